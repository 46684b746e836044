/*
 * lfsolve.h -- C ABI of the B200 (sm_100a) sparse direct solver for the
 * assembled LithoFEM systems (liblfsolve.so).
 *
 * Takes the place of the reference's cuDSS solver (solver/cudss_solver.inc:
 * SolveDeviceCsr :79-110, FactorDevice :186-203, FactorCore :205-285,
 * Backsolve :287-309), which is not available in this image.  It keeps that
 * solver's input contract: the device CSR of the assembly library is
 * borrowed zero-copy (int32 0-based row pointer, sorted int32 columns,
 * interleaved complex128 {re, im} values, general matrix, BASE_ZERO,
 * solver/cudss_solver.inc:217-220), and right-hand sides / solutions are
 * dense n x nrhs column-major device blocks (:222-227).
 *
 * Method: multifrontal LU.  The ordering is a nested dissection of the mesh
 * (element bisection; a separator is the set of DOFs shared by both halves),
 * computed on the host from the element DOF lists and element centroids
 * (the reference lets cuDSS reorder the CSR graph).  Fronts are factored
 * depth level by depth level on the device in complex64 or complex128 with
 * partial pivoting inside each front's pivot block; a complex64
 * factorization is refined in FP64 against the complex128 CSR
 * (lfsolve_solve_refined).  The same factors solve with A^T (the adjoint:
 * A^T(k_par) = A(-k_par) for the Bloch-envelope system).
 *
 * Essential (PEC) rows given to lfsolve_analyze are identity rows of the
 * eliminated system (as lfasm_assemble(h, 1) writes them): x = b there.
 *
 * Conventions as in lfasm.h: 0 on success, an LFSOLVE_ERR_* code otherwise,
 * lfsolve_last_error() for the message; work runs on the solver's stream
 * and every call returns after synchronizing it.  No CPU fallback.
 */
#ifndef LFSOLVE_H
#define LFSOLVE_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  LFSOLVE_OK = 0,
  LFSOLVE_ERR_ARG = 1,        /* invalid argument / inconsistent sizes       */
  LFSOLVE_ERR_CUDA = 2,       /* CUDA runtime or library error               */
  LFSOLVE_ERR_STATE = 3,      /* call order (factor before analyze ...)      */
  LFSOLVE_ERR_SINGULAR = 4,   /* a zero pivot in a front                     */
  LFSOLVE_ERR_NOCONV = 5      /* refinement did not reach the tolerance      */
};

enum { LFSOLVE_C64 = 0, LFSOLVE_C128 = 1 };  /* factorization precision */

typedef struct lfsolve lfsolve;

typedef struct lfsolve_stats {
  int n, n_ess, n_fronts, depth, max_front, max_pivots;
  long long factor_entries;   /* stored L and U entries                    */
  double factor_flops;        /* real flops of the numeric factorization   */
  long long peak_front_entries; /* front workspace of the two busiest depths */
  double analyze_s;           /* host seconds of lfsolve_analyze           */
  float factor_ms;            /* device ms of the last lfsolve_factor      */
  float solve_ms;             /* device ms of the last triangular solve    */
  int refine_iters;           /* iterations of the last refined solve      */
  double refine_rel;          /* its final max relative residual           */
} lfsolve_stats;

const char *lfsolve_last_error(void);

/* Solver on device gpu_id (its stream: lfsolve_set_stream, default the
 * legacy default stream). */
int lfsolve_create(int gpu_id, lfsolve **out);
int lfsolve_set_stream(lfsolve *s, void *stream);

/* Ordering and symbolic factorization (host).  n rows with the CSR
 * structure I (n + 1), J (nnz) of the matrix to be factored (host copies of
 * the device CSR's structure), the mesh's ne elements with nd DOFs each
 * (elem_dof, ne * nd) and their centroids (ne * 3), and the n_ess essential
 * rows.  Subdomains of at most leaf_elements elements (<= 0: 32) are not
 * split further. */
int lfsolve_analyze(lfsolve *s, int n, const int *I, const int *J, long long nnz, int ne,
                    int nd, const int *elem_dof, const double *centroid, const int *ess,
                    int n_ess, int leaf_elements);

/* Numeric factorization of the device CSR values d_vals (nnz interleaved
 * complex128, the structure given to lfsolve_analyze) in precision prec
 * (LFSOLVE_C64 or LFSOLVE_C128).  Replaces the previous factors. */
int lfsolve_factor(lfsolve *s, const void *d_vals, int prec);

/* d_x = A^-1 d_b (transpose != 0: A^-T d_b) with the factors alone, in
 * their precision; d_b, d_x: n x nrhs column-major complex128 device blocks
 * (d_x may equal d_b). */
int lfsolve_solve(lfsolve *s, int nrhs, const void *d_b, void *d_x, int transpose);

/* Refined solve: x_{i+1} = x_i + A_f^-1 (b - A x_i), with the residual in
 * FP64 on the device CSR (d_I, d_J, d_vals: the matrix that was factored,
 * complex128) and the correction from the factors A_f, from x_0 = A_f^-1 b,
 * until every column's ||b - A x|| / ||b|| <= tol or max_iter corrections
 * (LFSOLVE_ERR_NOCONV, with *rel set, if the tolerance is not reached).
 * rel_out (nrhs doubles, may be NULL) receives the final relative residuals
 * and *iters_out (may be NULL) the corrections applied.  transpose != 0
 * solves A^T x = b (residual with A^T).  When a correction reduces the
 * worst relative residual by less than half (refinement stalls, e.g. when
 * the factors are far from A), the solve switches to GMRES-based
 * refinement: per column, restarted GMRES(30) on A x = b in FP64 from the
 * current x, right-preconditioned by the factors, up to 10 max_iter Arnoldi
 * steps; *iters_out then counts the corrections plus the Arnoldi steps.
 * The environment variable LFSOLVE_GMRES=1 uses GMRES from the start,
 * LFSOLVE_GMRES=0 never. */
int lfsolve_solve_refined(lfsolve *s, const int *d_I, const int *d_J, const void *d_vals,
                          int nrhs, const void *d_b, void *d_x, int transpose, double tol,
                          int max_iter, double *rel_out, int *iters_out);

int lfsolve_get_stats(lfsolve *s, lfsolve_stats *out);

/* The ordering (host): perm[i] = the original row eliminated i-th, for the
 * n - n_ess non-essential rows; node_of[i] = the front that eliminates it. */
int lfsolve_get_ordering(lfsolve *s, int *perm, int *node_of);

/* The elimination tree (host), n_fronts entries each, fronts in preorder:
 * parent front (-1 for the root), depth, pivots k and rows m (any pointer
 * may be NULL). */
int lfsolve_get_fronts(lfsolve *s, int *parent, int *depth, int *k, int *m);

/* Releases the factors and the front workspace (the analysis stays). */
int lfsolve_release_factors(lfsolve *s);

void lfsolve_destroy(lfsolve *s);

#ifdef __cplusplus
}
#endif

#endif /* LFSOLVE_H */
