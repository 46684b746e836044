/*
 * lfasm.h -- C ABI of the B200 (sm_100a) LithoFEM system-assembly library
 * (liblfasm.so).
 *
 * Drop-in for the reference's in-process assembly classes
 *   AsmGpu        solver/asm_gpu.inc:271-425
 *   AsmGpuGlobal  solver/asm_gpu.inc:498-599
 * fed by the same extracted per-mesh data (AsmData, solver/asm_data.inc:77-97)
 * and problem tables (Problem/Region, solver/problem_common.inc:18-65).
 *
 * Conventions (all entry points):
 *   - return 0 (LFASM_OK) on success, a nonzero LFASM_ERR_* code on failure;
 *     lfasm_last_error() returns the message, and a CUDA failure also prints
 *     one "asm_gpu: CUDA error '<msg>' at <file>:<line>" line, the reference's
 *     diagnostic (asm_gpu.inc:255-263);
 *   - plain pointers and sizes only; host arrays are read during the call;
 *   - device buffers are owned by the handle and freed by lfasm_destroy
 *     into a per-device memory pool of the library, which keeps the blocks
 *     for the next handle (lfasm_trim_pool hands them back to the driver); the
 *     device CSR returned by lfasm_get_csr is borrowed (the cuDSS contract of
 *     solver/cudss_solver.inc:75-110: int32 0-based row pointer, sorted int32
 *     columns, interleaved complex128 {re, im} values, general matrix);
 *   - work runs on the handle's stream (lfasm_set_stream, default: the legacy
 *     default stream) and every stage ends with a stream synchronize, as the
 *     reference's stages end with cudaDeviceSynchronize, unless the handle
 *     was switched to asynchronous mode (lfasm_set_async).
 *   - there is no CPU fallback: without a usable CUDA device every call that
 *     needs one fails with LFASM_ERR_CUDA.
 */
#ifndef LFASM_H
#define LFASM_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  LFASM_OK = 0,
  LFASM_ERR_ARG = 1,         /* invalid argument / inconsistent sizes      */
  LFASM_ERR_CUDA = 2,        /* CUDA runtime error                         */
  LFASM_ERR_UNSUPPORTED = 3, /* outside the supported envelope (p > 3 ...) */
  LFASM_ERR_STATE = 4,       /* call order (e.g. scatter before build)     */
  LFASM_ERR_CSR = 5,         /* given sparsity misses an element coupling  */
  LFASM_ERR_INJECTED = 6     /* failure injected on the host: the variable
                                LITHOFEM_ASM_FORCE_FAIL is set (the
                                reference's switch, lithofem_solve.cpp:757-762) */
};

/* Integrator selection bits, identical to the reference's mask enum
 * (asm_gpu.inc:51-58). */
enum {
  LFASM_CURLCURL = 1, /* rule_cc:  curl-curl with Lambda^-1                 */
  LFASM_MASS = 2,     /* rule_mass: -k0^2 eps Lambda mass                   */
  LFASM_CROSS0 = 4,   /* rule_mass: MixedVectorCurl (i K Lambda^-1)         */
  LFASM_CROSS1 = 8,   /* rule_mass: MixedVectorWeakCurl (i Lambda^-1 K)     */
  LFASM_KLK = 16      /* rule_mass: -K Lambda^-1 K mass                     */
};

/* Region kinds (problem_common.inc:18-27, parse_problem_core :296-318). */
enum {
  LFASM_REGION_BACKGROUND = 0,
  LFASM_REGION_FRUSTUM = 1,
  LFASM_REGION_PML_BOTTOM = 2,
  LFASM_REGION_PML_TOP = 3
};

/* Reference tables at one quadrature rule: AsmRefRule (asm_data.inc:38-45). */
typedef struct lfasm_ref_rule {
  int nq;
  const double *ip;     /* nq*3 reference coordinates                      */
  const double *w;      /* nq weights                                      */
  const double *vshape; /* nq*nd*3, [q*nd*3 + k*3 + d]                      */
  const double *curl;   /* nq*nd*3                                         */
} lfasm_ref_rule;

/* Per-mesh extracted data: AsmData (asm_data.inc:77-97). I/Jcol may be NULL:
 * the symbolic CSR (build_csr_symbolic, asm_data.inc:178-210) is then built
 * on the device by lfasm_build_global. */
typedef struct lfasm_asm_data {
  int ne, nd, p, height, has_kpar;
  const int *dof;      /* ne*nd decoded global dof                         */
  const double *sign;  /* ne*nd +-1                                        */
  const int *fo;       /* ne*4 face orientations 0..5 (NULL for p = 1)     */
  const int *attr;     /* ne 1-based region attribute                      */
  const double *J;     /* ne*9 row-major Jacobian                          */
  const double *Jinv;  /* ne*9 row-major inverse                           */
  const double *detJ;  /* ne                                               */
  const double *v0;    /* ne*3 image of the reference origin               */
  lfasm_ref_rule rule_cc, rule_mass;
  const int *I;        /* height+1 row pointer, or NULL                    */
  const int *Jcol;     /* nnz sorted columns, or NULL                      */
  long long nnz;
} lfasm_asm_data;

/* Problem scalars and region table the path reads (Problem,
 * problem_common.inc:40-65; PML parameters, asm_gpu.inc:31-36). */
typedef struct lfasm_problem {
  double k0, kx, ky;
  double z_min, z_max, pml_thick, pml_order, pml_target;
  int n_regions;
  const double *region_eps;       /* 2*n_regions {re, im}                  */
  const int *region_kind;         /* n_regions LFASM_REGION_*              */
  const int *region_slab;         /* n_regions                             */
  const double *region_delta_eps; /* 2*n_regions, eps - eps_bg (frustum)   */
  const double *elem_eps;         /* NULL, or 2*ne per-element eps that
                                     overrides the region value            */
} lfasm_problem;

/* One incident-field part on every slab: SlabWave tables
 * (problem_common.inc:11-16, filled at lithofem_solve.cpp:577-598).
 * Arrays have n_slab entries; A/B are 3 complex {re, im} per slab. */
typedef struct lfasm_incident_part {
  int n_slab;
  const double *qA, *qB; /* 2*n_slab                                       */
  const double *zA, *zB; /* n_slab                                         */
  const double *A, *B;   /* 6*n_slab                                       */
} lfasm_incident_part;

typedef struct lfasm_handle lfasm_handle;

/* Last error message of the calling thread ("" if none). */
const char *lfasm_last_error(void);

/* Number of CUDA kernels this library launched in the process. */
long long lfasm_launch_count(void);

/* AsmGpu::Init (asm_gpu.inc:276-322): select device, upload geometry,
 * topology, rules and coefficient tables, allocate the element-matrix
 * buffer (ne*nd*nd complex128). */
int lfasm_init(const lfasm_asm_data *ad, const lfasm_problem *prob, int gpu_id,
               lfasm_handle **out);

/* Stream for all work of this handle (a cudaStream_t; NULL = default). */
int lfasm_set_stream(lfasm_handle *h, void *stream);

/* 0: every stage synchronizes its stream at the end (default);
 * 1: stages return after enqueueing (errors surface at the next sync). */
int lfasm_set_async(lfasm_handle *h, int async_mode);

/* AsmGpu::ComputeLocal (asm_gpu.inc:326-351): element matrices of the
 * integrators selected by mask_cc (rule_cc) and mask_mass (rule_mass), with
 * the dual face-orientation transform when apply_te != 0 (p >= 2), into the
 * handle's element buffer, row-major nd x nd per element, without dof signs. */
int lfasm_compute_local(lfasm_handle *h, int mask_cc, int mask_mass, int apply_te);

/* Device element buffer (borrowed): ne*nd*nd interleaved complex128. */
int lfasm_get_local(lfasm_handle *h, void **d_local);

/* AsmGpu::DownloadLocal (asm_gpu.inc:355-362), test-only: copies the element
 * buffer (2*ne*nd*nd doubles) and prints the reference's test-download
 * marker line "asm_gpu_test_download (test-only D2H)". */
int lfasm_download_local(lfasm_handle *h, double *host_out);

/* AsmGpuGlobal::BuildGlobal (asm_gpu.inc:501-514): upload the essential
 * (PEC) dof list and build the device CSR: the given I/Jcol, or the symbolic
 * CSR built on the device, plus the row -> (element, local row) map and the
 * element-entry -> CSR-slot map used by the atomic-free scatter. */
int lfasm_build_global(lfasm_handle *h, const int *ess_list, int n_ess);

/* AsmGpuGlobal::ScatterEliminate (asm_gpu.inc:517-530): element buffer from
 * lfasm_compute_local -> CSR values with dof signs; eliminate != 0 zeroes
 * essential rows/columns and puts 1+0i on their diagonal. */
int lfasm_scatter_eliminate(lfasm_handle *h, int eliminate);

/* Production path, the fused equivalent of ComputeLocal(CURLCURL,
 * MASS[|CROSS0|CROSS1|KLK when k-parallel != 0], te) + ScatterEliminate
 * (lithofem_solve.cpp:782-788): element matrices are written with signs,
 * transform and elimination applied, then gathered row-wise into the CSR. */
int lfasm_assemble(lfasm_handle *h, int eliminate);

/* AsmGpuGlobal accessors (asm_gpu.inc:579-583): borrowed device CSR. */
int lfasm_get_csr(lfasm_handle *h, int **d_rowptr, int **d_cols, void **d_vals,
                  int *n, long long *nnz);

/* Host copy of the symbolic CSR (height+1 and nnz ints). */
int lfasm_download_csr(lfasm_handle *h, int *host_I, int *host_J);

/* AsmGpuGlobal::DownloadValues (asm_gpu.inc:569-577), test-only: 2*nnz
 * doubles, prints the test-download marker line. */
int lfasm_download_values(lfasm_handle *h, double *host_out);

/* AsmGpuGlobal::Residual (asm_gpu.inc:533-565): ||A X - B|| / ||B|| with X
 * and B host vectors in the production [re(0..n-1); im(0..n-1)] layout. */
int lfasm_residual(lfasm_handle *h, const double *X, const double *B, double *rel);

/* Device variant: x, b interleaved complex128 device vectors of length n. */
int lfasm_residual_device(lfasm_handle *h, const void *d_x, const void *d_b,
                          double *rel);

/* Allocation-free residual (no counterpart in the reference): ||A x - b|| /
 * ||b|| for a device CSR given by plain pointers (int32 row pointer and
 * columns, interleaved complex128 values, x and b of length n), computed on
 * `stream` (a cudaStream_t; NULL = default) of the current device and
 * returned in *rel.  For callers that cannot call cudaMalloc while they run
 * (a solver loop whose memory is all held by its factorization, or a host
 * framework that owns every device allocation): it allocates nothing.  Its
 * partial sums use a fixed 4 MiB device array inside the library, which
 * bounds n to 2,097,152 rows (larger n fails with LFASM_ERR_UNSUPPORTED).
 * Each call enqueues its two kernels and a copy of the result on `stream`,
 * then synchronizes `stream` and returns with *rel set.  The first call on a
 * device looks up that array's address (and looks it up again after the
 * device's context was reset); make that first call before any stream
 * capture.  All calls share the array: calls that overlap on the GPU (other
 * streams, other host threads) race and must be serialized by the caller. */
int lfasm_csr_residual_noalloc(int n, const int *d_rowptr, const int *d_cols, const void *d_vals,
                               const void *d_x, const void *d_b, double *rel, void *stream);

/* y = A x on device vectors (interleaved complex128, length n). */
int lfasm_spmv(lfasm_handle *h, const void *d_x, void *d_y);

/* Scattered-field right-hand side (ScatterSource, problem_common.inc:218-266,
 * assembled as the reference's ComplexLinearForm with
 * VectorFEDomainLFIntegrator, lithofem_solve.cpp:678-684), using the
 * rule_mass points.  Part i goes into column col_of_part[i] of d_b
 * (n x ncol, column-major, interleaved complex128): parts sharing a column
 * are summed (one source with s and p parts), distinct columns give a
 * multi-RHS block.  Essential rows are zeroed (form_rhs_only,
 * lithofem_solve.cpp:732-742) when eliminate != 0. */
int lfasm_assemble_rhs(lfasm_handle *h, const lfasm_incident_part *parts,
                       int n_parts, const int *col_of_part, int ncol,
                       int eliminate, void *d_b);

/* Adjoint contraction for per-element permittivity.  For a linear
 * functional l(u) = c^T u of the solution of A(eps) u = b(eps) and the
 * adjoint solution A^T lambda = c (device vectors, interleaved complex128),
 * writes d_grad[e] = dl/deps_e = lambda^T (db/deps_e - dA/deps_e u) for
 * every non-PML element (0 for PML elements; ne complex128 entries):
 * dA_e/deps_e = -k0^2 M_e (the Lambda-weighted mass matrix of the mass
 * integrator, problem_common.inc:123-148) and db_e/deps_e = k0^2 int v.Ehat
 * (ScatterSource, problem_common.inc:238-266) with the incident parts of the
 * source (summed).  No counterpart in the reference (it has no adjoint). */
int lfasm_eps_gradient(lfasm_handle *h, const lfasm_incident_part *parts, int n_parts,
                       const void *d_u, const void *d_lambda, void *d_grad);

/* Autotuner: times the bulk-element kernel variants on this mesh -- 0: the
 * SIMT k_bulk, 1 and 2: the FP64 tensor-core k_bulk_mma with 4 or 2 tiles
 * per warp, 3 and 4: the same without block barriers (k_bulk_mma_nb), 5:
 * k_bulk_mma with 4 tiles per warp and the element records staged into
 * shared memory by the bulk-copy engine (k_bulk_tma) -- and
 * keeps the fastest.  The first lfasm_assemble of a handle
 * whose variant was not set takes the decision from a per-process cache
 * keyed by device, order p, k-parallel terms and the power-of-two class of
 * the bulk element count, and runs the autotuner only on a miss; an explicit
 * lfasm_autotune always times and refreshes the cache.  lfasm_get_tuning
 * reports the choice and one timing per variant (ms, LFASM_BULK_VARIANTS
 * floats). */
#define LFASM_BULK_VARIANTS 6
int lfasm_autotune(lfasm_handle *h);
int lfasm_set_bulk_variant(lfasm_handle *h, int variant);
int lfasm_get_tuning(lfasm_handle *h, int *bulk_variant, float *ms);

/* The PML-element kernel: 0 k_pml_mma, 1 k_pml_ws (warp-specialised
 * producer/consumer pipeline, p = 3 only), 2 k_pml_sym (the element matrix
 * split into its symmetric part, upper tiles only, and the cross part).  The
 * autotuner times the variants on the mesh (the cached decision carries
 * it); lfasm_set_pml_variant fixes one.  lfasm_get_pml_tuning reports the
 * choice and three timings in ms (0 for a variant not timed). */
int lfasm_set_pml_variant(lfasm_handle *h, int variant);
int lfasm_get_pml_tuning(lfasm_handle *h, int *pml_variant, float *ms3);

/* Field sampling and the orders' adjoint seed (the reference samples planes
 * with MFEM FindPoints/GetVectorValue, solver/lithofem_solve.cpp:951-1004,
 * and takes orders by FFT, src/lithofem/orders.py:36-67).
 * lfasm_set_basis hands over the element basis for evaluation away from the
 * quadrature points: nmono monomials x^a y^b z^c (exps[3 m .. 3 m + 2],
 * a + b + c <= p) and the coefficients of the nd functions and of their
 * curls, coef[(k * 3 + d) * nmono + m] (component d of function k).
 * lfasm_sample_plane: E and curl E of the device solution d_u (n
 * complex128, global coefficients) at the points ((i + 1/2) lx / nx +
 * 3.1e-7, (j + 1/2) ly / ny + 1.7e-7, z - 4.9e-7), j-major, into d_e and
 * d_curl (ny * nx * 3 complex128 each, either may be NULL), as the
 * reference's sampler; LFASM_ERR_ARG if a point lies outside the mesh.
 * lfasm_plane_seed: d_c (n complex128, overwritten) with c^T u equal to the
 * (m, q) Fourier coefficient (1 / (nx ny)) sum_{j,i} E_comp(x_ij)
 * exp(-2 pi i (m i / nx + q j / ny)) of component comp of those samples. */
int lfasm_set_basis(lfasm_handle *h, int nmono, const int *exps, const double *coef,
                    const double *curl_coef);
int lfasm_sample_plane(lfasm_handle *h, double lx, double ly, double z, int nx, int ny,
                       const void *d_u, void *d_e, void *d_curl);
int lfasm_plane_seed(lfasm_handle *h, double lx, double ly, double z, int nx, int ny, int comp,
                     int m, int q, void *d_c);

/* Several planes and their diffraction orders on the device (the reference
 * samples its reflection and transmission planes one after the other,
 * solver/lithofem_solve.cpp:951-1015, then FFTs each on the host,
 * src/lithofem/orders.py:36-67, and forms the order efficiencies of
 * src/lithofem/outputs.py:219-269).
 * lfasm_sample_planes: lfasm_sample_plane for nz planes at heights z[0 ..
 * nz) (host array) in one pass; d_e / d_curl hold nz blocks of ny * nx * 3
 * complex128 (plane-major).  At most LFASM_MAX_PLANES planes and 2^24 points.
 * lfasm_plane_orders: for every plane iz of such samples d_e and every
 * grid index o = b nx + a of the order (m, n) = (a or a - nx above nx / 2,
 * b or b - ny above ny / 2): d_coef[(iz nx ny + o) 3 + c] = (1 / (nx ny))
 * sum_{j,i} E_c(x_ij) exp(-2 pi i (a i / nx + b j / ny)) (numpy's fft2
 * divided by nx ny), and d_eff[iz nx ny + o] the order's efficiency: with
 * kx = args->kx + 2 pi m / lx, ky likewise, qz = sqrt(k0^2 eps - kx^2 -
 * ky^2) (Im qz >= 0) and c' = c exp(-i d qz (z - z_ref)) plus bg00 for the
 * (0, 0) order when has_bg00, eff = d Re[(c' x conj(k x c' / k0))_z] lx ly /
 * (2 inc_flux), k = (kx, ky, d qz), d = direction (+1: up-going orders of a
 * reflection plane, -1: down-going of a transmission plane). */
#define LFASM_MAX_PLANES 256
typedef struct {
  double z, z_ref;       /* sampled height, reference plane of the efficiency */
  double eps_re, eps_im; /* permittivity of the one-way region */
  int direction;         /* +1 or -1 */
  int has_bg00;          /* add bg00 to the (0, 0) coefficient at z_ref */
  double bg00[6];        /* analytic (0, 0) background, 3 complex (re, im) */
} lfasm_order_plane;
typedef struct {
  double lx, ly;   /* cell */
  double k0;       /* vacuum wavenumber */
  double kx, ky;   /* Bloch wavevector of the incidence */
  double inc_flux; /* incident flux through the cell */
} lfasm_order_args;
int lfasm_sample_planes(lfasm_handle *h, double lx, double ly, int nz, const double *z, int nx,
                        int ny, const void *d_u, void *d_e, void *d_curl);
int lfasm_plane_orders(lfasm_handle *h, int nz, int nx, int ny, const void *d_e,
                       const lfasm_order_plane *planes, const lfasm_order_args *args,
                       void *d_coef, double *d_eff);

/* Per-mesh data on the device (the reference's extract_asm_data over MFEM's
 * Nedelec space, solver/asm_data.inc:99-173, run on the host there):
 * from ne tetrahedra with topological vertex ids tv[4 e + i] (0 .. nv-1,
 * after periodic identification) and their own vertex coordinates
 * xv[(4 e + i) 3 + d], at order p, the lfasm_asm_data arrays: dof and sign
 * (ne * nd), fo (ne * 4, p >= 2; may be NULL at p = 1), J, Jinv (ne * 9
 * row-major), detJ (ne), v0 (ne * 3), the DOF count *height and the sorted
 * essential DOFs (every DOF of a face that one element alone references,
 * with its edges) into ess (*n_ess of them; LFASM_ERR_ARG when more than
 * ess_cap).  Element-local vertex order: ascending id, the last two
 * swapped where that makes detJ > 0; edges and faces numbered by first
 * occurrence (element-major, local edge / face order); a face's global
 * vertex order is that of its first occurrence.  nv < 2^21. */
int lfasm_extract(int gpu_id, int ne, int nv, int p, const int *tv, const double *xv, int *dof,
                  double *sign, int *fo, double *J, double *Jinv, double *detJ, double *v0,
                  int *ess, long long ess_cap, int *height, int *n_ess);

/* Per-stage CUDA-event timing of lfasm_assemble (the analogue of the
 * reference's asm_gpu_*_s sub-timers, lithofem_solve.cpp:773-793):
 * lfasm_set_profile(h, 1) then, after an lfasm_assemble, ms3 receives the
 * milliseconds of {coefficient prep + bulk elements, PML elements, CSR
 * gather}. */
int lfasm_set_profile(lfasm_handle *h, int on);
int lfasm_stage_times(lfasm_handle *h, float *ms3);

/* Element counts of the two device paths (elements whose quadrature points
 * all lie outside the PML, and the rest). */
int lfasm_path_counts(lfasm_handle *h, int *n_bulk, int *n_pml);

void lfasm_destroy(lfasm_handle *h);

/* 1 in the bounds-checked debug build (liblfasm_bounds.so, compiled with
 * -DLFASM_BOUNDS: device index checks in the gather record a failure,
 * skip the access and make the call return LFASM_ERR_CUDA), else 0. */
int lfasm_bounds_checked(void);

/* Bounds-checked debug build only (LFASM_ERR_UNSUPPORTED elsewhere; no
 * counterpart in the reference): on device gpu_id, every bounded mbarrier
 * wait of the warp-specialised PML kernel gives up after wait_limit
 * try-wait rounds (<= 0: the default 2^20), and drop_first != 0 withholds
 * the producers' arrivals on the first chunk barrier of block 0, so that the
 * consumers' first wait there runs out: lfasm_assemble then returns
 * LFASM_ERR_CUDA ("a bounded wait ran out") with the device still usable.
 * Exercises the failure path without a GPU fault. */
int lfasm_debug_wait_test(int gpu_id, long long wait_limit, int drop_first);

/* Batched assembly of several meshes on one device (the reference assembles
 * one mesh per process; no counterpart).  lfasm_batch_create takes n built
 * handles (lfasm_build_global done) of one device; they must outlive the
 * batch and keep their structure (no new build, no lfasm_set_bulk_variant)
 * while it exists.  lfasm_batch_assemble(b, eliminate) has the effect of
 * lfasm_assemble(h_i, eliminate) on every handle: the first call for an
 * eliminate flag tunes each handle and captures all of them into one CUDA
 * graph (one branch per handle, concurrent), later calls launch that graph
 * once; it returns after the graph has completed on the batch stream
 * (lfasm_batch_set_stream, default: a stream of the batch). */
typedef struct lfasm_batch lfasm_batch;
int lfasm_batch_create(lfasm_handle *const *handles, int n, lfasm_batch **out);
int lfasm_batch_set_stream(lfasm_batch *b, void *stream);
int lfasm_batch_assemble(lfasm_batch *b, int eliminate);
void lfasm_batch_destroy(lfasm_batch *b);

/* Hands the device memory cached by the library's pool on device gpu_id
 * (blocks of destroyed handles and temporaries) back to the driver; live
 * handles keep theirs.  No counterpart in the reference, whose handles
 * cudaMalloc and cudaFree their buffers directly. */
int lfasm_trim_pool(int gpu_id);

#ifdef __cplusplus
}
#endif

#endif /* LFASM_H */
