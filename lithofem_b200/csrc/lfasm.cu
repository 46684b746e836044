// liblfasm: B200 (sm_100a) LithoFEM system assembly behind the C ABI of
// include/lfasm.h.  Host side of the handle; the kernels live in
// lfasm_kernels.cuh.
//
// Call sequence mirrors the reference (solver/lithofem_solve.cpp:765-795):
//   lfasm_init          <- AsmGpu::Init            (asm_gpu.inc:276-322)
//   lfasm_build_global  <- AsmGpuGlobal::BuildGlobal (asm_gpu.inc:501-514)
//   lfasm_assemble      <- ComputeLocal + ScatterEliminate (asm_gpu.inc:326-351, 517-530)
//   lfasm_get_csr       <- DeviceI/DeviceJ/DeviceValues  (asm_gpu.inc:579-583)
//   lfasm_residual      <- Residual                (asm_gpu.inc:533-565)

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <map>
#include <atomic>
#include <mutex>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "../../include/lfasm.h"
#include "lfasm_kernels.cuh"
#include "lfextract.cuh"

using namespace lfasm_dev;

namespace {

thread_local std::string g_err;
std::atomic<long long> g_launches{0};

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define LF_CUDA(call)                                                          \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      std::printf("asm_gpu: CUDA error '%s' at %s:%d\n",                       \
                  cudaGetErrorString(e_), __FILE__, __LINE__);                 \
      std::fflush(stdout);                                                     \
      return fail(LFASM_ERR_CUDA, "CUDA error '%s' at %s:%d",                  \
                  cudaGetErrorString(e_), __FILE__, __LINE__);                 \
    }                                                                          \
  } while (0)

#define LF_LAUNCHED() g_launches.fetch_add(1, std::memory_order_relaxed)

// Device memory of the handles.  Blocks of BIG_BLOCK bytes and more (the
// element buffer, the CSR values, columns and slot maps) are cudaMalloc'd in
// 2 MiB multiples and, when released, kept in a per-device cache keyed by
// size: a request is served by the smallest cached block that is at least
// as large and at most 1/8 larger, so a new handle on a mesh of the same size
// (one handle per design iteration) gets the same blocks back without a
// cudaMalloc/cudaFree round trip or a growing, fragmented pool.  Smaller
// blocks come from a stream-ordered pool per device (release threshold:
// keep everything), allocated and freed on the legacy default stream.  Every
// release happens after the work that used the block has completed.
// lfasm_trim_pool hands all cached memory back to the driver.
constexpr int MAX_DEV = 64;
constexpr size_t BIG_BLOCK = size_t(16) << 20;
constexpr size_t BIG_ROUND = size_t(2) << 20;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[MAX_DEV] = {};
std::multimap<size_t, void *> g_big_free[MAX_DEV];
std::map<void *, size_t> g_big_live[MAX_DEV];

cudaError_t dev_pool(int dev, cudaMemPool_t *out) {  // g_pool_mu held
  if (!g_pool[dev]) {
    cudaMemPoolProps pp;
    std::memset(&pp, 0, sizeof(pp));
    pp.allocType = cudaMemAllocationTypePinned;
    pp.handleTypes = cudaMemHandleTypeNone;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = dev;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = cudaMemPoolCreate(&pool, &pp);
    if (e != cudaSuccess) return e;
    unsigned long long keep = ~0ull;
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) {
      cudaMemPoolDestroy(pool);
      return e;
    }
    g_pool[dev] = pool;
  }
  *out = g_pool[dev];
  return cudaSuccess;
}

// frees the cached big blocks of `dev` (g_pool_mu held, dev current)
void drop_big_cache(int dev) {
  for (auto &kv : g_big_free[dev]) cudaFree(kv.second);
  g_big_free[dev].clear();
}

cudaError_t dmalloc_bytes(void **out, size_t bytes) {
  *out = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= MAX_DEV) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (bytes < BIG_BLOCK) {
    cudaMemPool_t pool;
    if ((e = dev_pool(dev, &pool)) != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(out, std::max<size_t>(bytes, 1), pool, 0);
  }
  const size_t want = (bytes + BIG_ROUND - 1) / BIG_ROUND * BIG_ROUND;
  auto it = g_big_free[dev].lower_bound(want);
  if (it != g_big_free[dev].end() && it->first <= want + want / 8) {
    *out = it->second;
    g_big_live[dev][it->second] = it->first;
    g_big_free[dev].erase(it);
    return cudaSuccess;
  }
  e = cudaMalloc(out, want);
  if (e == cudaErrorMemoryAllocation) {  // give the cache back and retry once
    cudaGetLastError();
    drop_big_cache(dev);
    e = cudaMalloc(out, want);
  }
  if (e != cudaSuccess) return e;
  g_big_live[dev][*out] = want;
  return cudaSuccess;
}

void dfree_bytes(void *p) {
  if (!p) return;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEV) return;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto it = g_big_live[dev].find(p);
  if (it != g_big_live[dev].end()) {
    g_big_free[dev].emplace(it->second, p);
    g_big_live[dev].erase(it);
    return;
  }
  cudaFreeAsync(p, 0);
}

template <typename T>
cudaError_t dmalloc(T *&dst, size_t count) {
  void *p = nullptr;
  cudaError_t e = dmalloc_bytes(&p, std::max<size_t>(count, 1) * sizeof(T));
  dst = static_cast<T *>(p);
  return e;
}

template <typename T>
cudaError_t upload(T *&dst, const T *src, size_t count) {
  dst = nullptr;
  if (count == 0) return cudaSuccess;
  cudaError_t e = dmalloc(dst, count);
  if (e != cudaSuccess) return e;
  return cudaMemcpy(dst, src, count * sizeof(T), cudaMemcpyHostToDevice);
}

template <typename T>
void dfree(T *&p) {
  if (p) { dfree_bytes((void *)p); p = nullptr; }
}

struct DevRule {
  int nq = 0, ldt = 0;
  double *ip = nullptr, *w = nullptr, *v = nullptr, *c = nullptr;
  double *vt = nullptr, *ct = nullptr;  // component-major, zero-padded columns
  Rule view() const {
    Rule r;
    r.nq = nq; r.ip = ip; r.w = w; r.v = v; r.c = c; r.vt = vt; r.ct = ct; r.ldt = ldt;
    return r;
  }
};

// [q][k][d] (k < nd) -> [d][q][k] with ldt columns, zero past nd
std::vector<double> component_major(const double *t, int nq, int nd, int ldt) {
  std::vector<double> out((size_t)3 * nq * ldt, 0.0);
  if (!t) return out;
  for (int d = 0; d < 3; ++d)
    for (int q = 0; q < nq; ++q)
      for (int k = 0; k < nd; ++k)
        out[((size_t)d * nq + q) * ldt + k] = t[((size_t)q * nd + k) * 3 + d];
  return out;
}

}  // namespace

struct lfasm_handle {
  int dev = 0;
  cudaStream_t stream = nullptr;
  int async_mode = 0;
  int ne = 0, nd = 0, p = 0, n = 0, has_kpar = 0;
  int ndp = 0, ndp4 = 0, rs = 0;
  int sm_count = 148;
  int smem_optin = 48 * 1024;  // max dynamic shared memory per block (opt-in)
  long long nnz = 0;
  // element data
  int *dof = nullptr;
  double *sign = nullptr;
  int *attr = nullptr;
  double *J = nullptr, *Jinv = nullptr, *detJ = nullptr, *v0 = nullptr;
  unsigned *fopack = nullptr;
  unsigned long long *signmask = nullptr, *essmask = nullptr;
  DevRule rcc, rm;
  dcplx *eps_tab = nullptr, *elem_eps = nullptr;
  PmlParams pml{};
  int *bulk_list = nullptr, *pml_list = nullptr;
  int n_bulk = 0, n_pml = 0;
  double *S = nullptr;
  double *rec = nullptr;
  // tensor-core bulk variant and the autotuned choice
  double *S_mma = nullptr, *rec_mma = nullptr;
  double *S_mmaf = nullptr;  // B operand of the fused Bloch layout
  // 0: k_bulk (SIMT), 1/2: k_bulk_mma (DMMA, 4/2 tiles per warp),
  // 3/4: k_bulk_mma_nb (the same without block barriers, 4/2 tiles per warp)
  int bulk_variant = 0;
  int tuned = 0;             // autotune done
  int forced = 0;            // variant fixed by lfasm_set_bulk_variant
  float tune_ms[LFASM_BULK_VARIANTS] = {};
  // PML kernel: 0 k_pml_mma, 1 k_pml_ws (warp-specialised, p = 3 only),
  // 2 k_pml_sym (symmetric split)
  int pml_variant = 0;
  int pml_forced = 0;
  float pml_ms[3] = {0.f, 0.f, 0.f};
  int *err = nullptr;  // device error word of the bounded-wait kernels
  // element basis for sampling away from the quadrature points
  int nmono = 0;
  int *bexps = nullptr;
  double *bcoef = nullptr, *bccoef = nullptr;
  dcplx *Ae = nullptr;
  // RHS data
  int *slab_of = nullptr;
  dcplx *delta = nullptr;
  int *src_list = nullptr, *src_slot = nullptr;
  int n_src = 0;
  int max_src_slab = -1;  // largest slab index among RHS source elements
  int max_bulk_slab = -1; // largest slab index among the non-PML (design) elements
  // global
  int built = 0, locals_valid = 0;
  int *I = nullptr, *Jc = nullptr;
  dcplx *vals = nullptr;
  unsigned char *ess = nullptr;
  int *ea_ptr = nullptr, *ea = nullptr;
  uint16_t *off = nullptr;
  int max_row = 0;
  // chunked lfasm_assemble: elements in chunks of consecutive centroid
  // height; after each chunk, the rows it completes are gathered while its
  // element rows are in L2 (and then discarded from it)
  int nchunk = 0;                            // 0: one pass (no chunking)
  std::vector<int> chunk_b, chunk_q, chunk_r; // nchunk + 1 offsets: bulk list,
                                             // PML list, row order
  int *row_order = nullptr;                  // rows by completion chunk
  cudaStream_t gstream = nullptr;            // gather stream of the chunks
  cudaStream_t cstream = nullptr;            // capture stream (the handle's own
                                             // stream may be the legacy stream)
  cudaGraphExec_t cexec[2] = {nullptr, nullptr};  // captured chunk sequence
  long long ckernels[2] = {0, 0};
  int cvar_bulk[2] = {-1, -1}, cvar_pml[2] = {-1, -1};  // variants captured
  int row_cap = 0;            // gather: rows up to row_cap entries in shared memory
  int *long_rows = nullptr;   // the longer rows
  int n_long = 0;
  double *partials = nullptr, *red = nullptr;
  int n_part_blocks = 0;
  // optional per-stage events of lfasm_assemble: prep+bulk, pml, gather
  int profile = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // side stream for the PML elements, overlapped with the bulk elements
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // host copies of a caller-given symbolic CSR (read at init)
  std::vector<int> h_I, h_J;
};

namespace {

// bounds-checked build: the first failed device index check, if any
int bounds_status() {
#ifdef LFASM_BOUNDS
  int e = 0;
  LF_CUDA(cudaMemcpyFromSymbol(&e, g_bounds_err, sizeof(int)));
  if (e) {
    const int zero = 0;
    LF_CUDA(cudaMemcpyToSymbol(g_bounds_err, &zero, sizeof(int)));
    return fail(LFASM_ERR_CUDA, "device bounds check %d failed (%s)", e,
                e == BOUNDS_SLOT ? "slot offset outside its CSR row"
                                 : "row-list entry outside the element buffer");
  }
#endif
  return LFASM_OK;
}

int sync_if(lfasm_handle *h) {
  LF_CUDA(cudaGetLastError());
  if (!h->async_mode) {
    LF_CUDA(cudaStreamSynchronize(h->stream));
    if (int rb = bounds_status()) return rb;
    if ((h->pml_variant == 1 || h->bulk_variant == 5) && h->err) {
      int e = 0;
      LF_CUDA(cudaMemcpy(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost));
      if (e) {
        LF_CUDA(cudaMemset(h->err, 0, sizeof(int)));
        return fail(LFASM_ERR_CUDA,
                    "PML pipeline or staged bulk records: a bounded wait ran out (results "
                    "undefined)");
      }
    }
  }
  return LFASM_OK;
}

// Element-independent tables of the bulk path, quadrature sums of reference
// shape products with the element's own rules (exact for these polynomial
// integrands):  Scc_t[k][l] = sum_q w_q rc_k,a rc_l,b (+ the (b,a) term for
// a != b), Svv_t likewise with vshapes, Rvc_jj'[k][l] = sum_q w_q rv_k,j rc_l,j'.
// Packed per bulk-kernel thread (I, l >= 2I), value-major for coalesced
// loads: [cc(2I,l) 6, vv(2I,l) 6, cc(2I+1,l) 6, vv(2I+1,l) 6,
//         Rvc(2I,l) 9, Rvc(2I+1,l) 9, Rvc(l,2I) 9, Rvc(l,2I+1) 9].
int bulk_threads(int ndp) { const int H = ndp / 2; return H * H + H; }

void build_S(const lfasm_asm_data *ad, int ndp, std::vector<double> &S) {
  const int nd = ad->nd;
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  const lfasm_ref_rule &rc = ad->rule_cc, &rm = ad->rule_mass;
  // full tables first: [9][nd][nd] each
  std::vector<double> Rcc((size_t)9 * nd * nd, 0.0), Rvv(Rcc.size(), 0.0), Rvc(Rcc.size(), 0.0);
  auto at = [&](std::vector<double> &T, int j, int k, int l) -> double & {
    return T[((size_t)j * nd + k) * nd + l];
  };
  for (int k = 0; k < nd; ++k)
    for (int l = 0; l < nd; ++l) {
      for (int q = 0; q < rc.nq; ++q) {
        const double *ck = rc.curl + ((size_t)q * nd + k) * 3;
        const double *cl = rc.curl + ((size_t)q * nd + l) * 3;
        for (int j = 0; j < 3; ++j)
          for (int jj = 0; jj < 3; ++jj) at(Rcc, j * 3 + jj, k, l) += rc.w[q] * ck[j] * cl[jj];
      }
      for (int q = 0; q < rm.nq; ++q) {
        const double *vk = rm.vshape + ((size_t)q * nd + k) * 3;
        const double *vl = rm.vshape + ((size_t)q * nd + l) * 3;
        const double *cl = rm.curl + ((size_t)q * nd + l) * 3;
        for (int j = 0; j < 3; ++j)
          for (int jj = 0; jj < 3; ++jj) {
            at(Rvv, j * 3 + jj, k, l) += rm.w[q] * vk[j] * vl[jj];
            at(Rvc, j * 3 + jj, k, l) += rm.w[q] * vk[j] * cl[jj];
          }
      }
    }
  auto sym = [&](std::vector<double> &T, int t, int k, int l) -> double {
    if (k >= nd || l >= nd) return 0.0;
    const int a = pa[t], b = pb[t];
    return a == b ? at(T, a * 3 + a, k, l) : at(T, a * 3 + b, k, l) + at(T, b * 3 + a, k, l);
  };
  auto rvc = [&](int j, int k, int l) -> double {
    return (k >= nd || l >= nd) ? 0.0 : at(Rvc, j, k, l);
  };
  const int nthr = bulk_threads(ndp);
  S.assign((size_t)60 * nthr, 0.0);
  int f = 0;
  for (int I = 0; I < ndp / 2; ++I)
    for (int l = 2 * I; l < ndp; ++l, ++f) {
      for (int a = 0; a < 2; ++a) {
        const int r = 2 * I + a;
        for (int t = 0; t < 6; ++t) {
          S[(size_t)(12 * a + t) * nthr + f] = sym(Rcc, t, r, l);
          S[(size_t)(12 * a + 6 + t) * nthr + f] = sym(Rvv, t, r, l);
        }
        for (int j = 0; j < 9; ++j) {
          S[(size_t)(24 + 9 * a + j) * nthr + f] = rvc(j, r, l);
          S[(size_t)(42 + 9 * a + j) * nthr + f] = rvc(j, l, r);
        }
      }
    }
}

// B operand of the tensor-core bulk variant (k_bulk_mma): the same
// quadrature sums, term-major [BK][ntiles*8], entries in pair-block order
// n = 4 (I*H + J) + 2a + b for entry (2I+a, 2J+b), H = ndp/2; terms 0..5 Scc,
// 6..11 Svv (symmetric pairs), 12..20 Rvc_jj', 21..29 Rcv_jj'.
int bulk_tiles(int ndp) { return 2 * (ndp / 2) * ((ndp + 7) / 8); }

// fused: the fused Bloch layout of k_bulk_mma<..., FUSED> -- terms 0..11 as
// above, 12..17 Svv again (imaginary row), 18..26 D_ab = Rvc_ab - Rcv_ba.
void build_S_mma(const lfasm_asm_data *ad, int ndp, bool fused, std::vector<double> &S) {
  const int nd = ad->nd;
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  const lfasm_ref_rule &rc = ad->rule_cc, &rm = ad->rule_mass;
  std::vector<double> Rcc((size_t)9 * nd * nd, 0.0), Rvv(Rcc.size(), 0.0), Rvc(Rcc.size(), 0.0),
      Rcv(Rcc.size(), 0.0);
  auto at = [&](std::vector<double> &T, int j, int k, int l) -> double & {
    return T[((size_t)j * nd + k) * nd + l];
  };
  for (int k = 0; k < nd; ++k)
    for (int l = 0; l < nd; ++l) {
      for (int q = 0; q < rc.nq; ++q) {
        const double *ck = rc.curl + ((size_t)q * nd + k) * 3;
        const double *cl = rc.curl + ((size_t)q * nd + l) * 3;
        for (int j = 0; j < 3; ++j)
          for (int jj = 0; jj < 3; ++jj) at(Rcc, j * 3 + jj, k, l) += rc.w[q] * ck[j] * cl[jj];
      }
      for (int q = 0; q < rm.nq; ++q) {
        const double *vk = rm.vshape + ((size_t)q * nd + k) * 3;
        const double *vl = rm.vshape + ((size_t)q * nd + l) * 3;
        const double *ck = rm.curl + ((size_t)q * nd + k) * 3;
        const double *cl = rm.curl + ((size_t)q * nd + l) * 3;
        for (int j = 0; j < 3; ++j)
          for (int jj = 0; jj < 3; ++jj) {
            at(Rvv, j * 3 + jj, k, l) += rm.w[q] * vk[j] * vl[jj];
            at(Rvc, j * 3 + jj, k, l) += rm.w[q] * vk[j] * cl[jj];
            at(Rcv, j * 3 + jj, k, l) += rm.w[q] * ck[j] * vl[jj];
          }
      }
    }
  const int ncb = (ndp + 7) / 8, ntiles = bulk_tiles(ndp), N = ntiles * 8;
  S.assign((size_t)BK * N, 0.0);
  for (int I = 0; I < ndp / 2; ++I)
    for (int cb = 0; cb < ncb; ++cb)
      for (int a = 0; a < 2; ++a)
        for (int c = 0; c < 8; ++c) {
          const int k = 2 * I + a, l = 8 * cb + c;
          if (k >= nd || l >= nd) continue;
          const size_t n = (size_t)(2 * (I * ncb + cb) + a) * 8 + c;
          for (int t = 0; t < 6; ++t) {
            const int x = pa[t], y = pb[t];
            S[(size_t)t * N + n] = x == y ? at(Rcc, x * 3 + x, k, l)
                                          : at(Rcc, x * 3 + y, k, l) + at(Rcc, y * 3 + x, k, l);
            S[(size_t)(6 + t) * N + n] = x == y ? at(Rvv, x * 3 + x, k, l)
                                                : at(Rvv, x * 3 + y, k, l) + at(Rvv, y * 3 + x, k, l);
          }
          if (fused) {
            for (int t = 0; t < 6; ++t) S[(size_t)(12 + t) * N + n] = S[(size_t)(6 + t) * N + n];
            for (int a2 = 0; a2 < 3; ++a2)
              for (int b2 = 0; b2 < 3; ++b2)
                S[(size_t)(18 + a2 * 3 + b2) * N + n] =
                    at(Rvc, a2 * 3 + b2, k, l) - at(Rcv, b2 * 3 + a2, k, l);
          } else {
            for (int j = 0; j < 9; ++j) {
              S[(size_t)(12 + j) * N + n] = at(Rvc, j, k, l);
              S[(size_t)(21 + j) * N + n] = at(Rcv, j, k, l);
            }
          }
        }
}

// 2x2 blocks relating element-local face DOF pairs to the global pairs for
// the six face permutations, derived from the tangent pairs
// (b - a, c - a) vs (B - A, C - A); column-major like asm_data.inc:26-34.
void build_tinv(double out[24]) {
  const int perms[6][3] = {{0, 1, 2}, {1, 0, 2}, {1, 2, 0}, {2, 1, 0}, {2, 0, 1}, {0, 2, 1}};
  const double G[3][2] = {{0, 0}, {1, 0}, {0, 1}};
  for (int o = 0; o < 6; ++o) {
    const double *a = G[perms[o][0]], *b = G[perms[o][1]], *c = G[perms[o][2]];
    const double m00 = b[0] - a[0], m01 = b[1] - a[1];
    const double m10 = c[0] - a[0], m11 = c[1] - a[1];
    out[4 * o + 0] = m00;
    out[4 * o + 1] = m10;
    out[4 * o + 2] = m01;
    out[4 * o + 3] = m11;
  }
}

// index of the first i < n with bad(i), else n; scans in blocks with a
// branch-free reduction (vectorised) and locates the index only in a block
// that has one
template <class F>
size_t first_bad_range(size_t lo, size_t hi, F &bad) {
  constexpr size_t B = 8192;
  for (size_t c = lo; c < hi; c += B) {
    const size_t e = std::min(hi, c + B);
    int any = 0;
    for (size_t i = c; i < e; ++i) any |= bad(i);
    if (any)
      for (size_t i = c; i < e; ++i)
        if (bad(i)) return i;
  }
  return hi;
}

// large arrays are split over a few host threads; the answer is still the
// lowest offending index
template <class F>
size_t first_bad(size_t n, F bad) {
  constexpr size_t PAR_MIN = size_t(1) << 20;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned nt = n < PAR_MIN ? 1u : std::min(8u, hw);
  if (nt == 1) return first_bad_range(0, n, bad);
  std::vector<size_t> res(nt, n);
  std::vector<std::thread> th;
  const size_t step = (n + nt - 1) / nt;
  for (unsigned t = 0; t < nt; ++t) {
    const size_t lo = std::min(n, t * step), hi = std::min(n, lo + step);
    th.emplace_back([&, t, lo, hi] {
      const size_t r = first_bad_range(lo, hi, bad);
      res[t] = r < hi ? r : n;
    });
  }
  for (std::thread &x : th) x.join();
  return *std::min_element(res.begin(), res.end());
}

// reference S tables depend only on p and the two rules: cached per process
// on the exact rule contents
struct STables {
  std::vector<double> key, S, S_mma, S_mmaf;
};
std::mutex g_stab_mu;
std::vector<STables> g_stab;

std::vector<double> rule_key(const lfasm_asm_data *ad, int ndp) {
  std::vector<double> k = {(double)ad->p, (double)ad->nd, (double)ndp};
  const int nd = ad->nd;
  for (const lfasm_ref_rule *r : {&ad->rule_cc, &ad->rule_mass}) {
    k.push_back((double)r->nq);
    k.insert(k.end(), r->ip, r->ip + (size_t)r->nq * 3);
    k.insert(k.end(), r->w, r->w + r->nq);
    k.push_back(r->vshape ? 1.0 : 0.0);
    if (r->vshape) k.insert(k.end(), r->vshape, r->vshape + (size_t)r->nq * nd * 3);
    k.insert(k.end(), r->curl, r->curl + (size_t)r->nq * nd * 3);
  }
  return k;
}

}  // namespace

extern "C" {

const char *lfasm_last_error(void) { return g_err.c_str(); }

long long lfasm_launch_count(void) { return g_launches.load(); }

int lfasm_bounds_checked(void) {
#ifdef LFASM_BOUNDS
  return 1;
#else
  return 0;
#endif
}

int lfasm_debug_wait_test(int gpu_id, long long wait_limit, int drop_first) {
  g_err.clear();
#ifdef LFASM_BOUNDS
  LF_CUDA(cudaSetDevice(gpu_id));
  const long long lim = wait_limit > 0 ? wait_limit : WS_WAIT_LIMIT;
  const int drop = drop_first ? 1 : 0;
  LF_CUDA(cudaMemcpyToSymbol(g_ws_wait_limit, &lim, sizeof lim));
  LF_CUDA(cudaMemcpyToSymbol(g_ws_drop_first, &drop, sizeof drop));
  return LFASM_OK;
#else
  (void)gpu_id; (void)wait_limit; (void)drop_first;
  return fail(LFASM_ERR_UNSUPPORTED, "wait test settings exist only in the bounds-checked build");
#endif
}

int lfasm_init(const lfasm_asm_data *ad, const lfasm_problem *prob, int gpu_id,
               lfasm_handle **out) {
  g_err.clear();
  if (!out) return fail(LFASM_ERR_ARG, "out handle pointer is NULL");
  *out = nullptr;
  const char *inject = std::getenv("LITHOFEM_ASM_FORCE_FAIL");
  if (inject && inject[0]) {
    std::printf("asm_gpu: forced failure injected (LITHOFEM_ASM_FORCE_FAIL)\n");
    std::fflush(stdout);
    return fail(LFASM_ERR_INJECTED, "forced failure injected (LITHOFEM_ASM_FORCE_FAIL)");
  }
  if (!ad || !prob) return fail(LFASM_ERR_ARG, "NULL asm data or problem");
  if (ad->ne <= 0) return fail(LFASM_ERR_ARG, "empty mesh (ne = %d)", ad->ne);
  if (ad->p < 1 || ad->p > 3)
    return fail(LFASM_ERR_UNSUPPORTED, "ND order p = %d outside the supported 1..3", ad->p);
  const int nd = ad->p * (ad->p + 2) * (ad->p + 3) / 2;
  if (ad->nd != nd) return fail(LFASM_ERR_ARG, "nd = %d does not match p = %d", ad->nd, ad->p);
  if (ad->height <= 0) return fail(LFASM_ERR_ARG, "height must be positive");
  if (!ad->dof || !ad->sign || !ad->attr || !ad->J || !ad->Jinv || !ad->detJ || !ad->v0)
    return fail(LFASM_ERR_ARG, "missing element array");
  if (ad->p >= 2 && !ad->fo) return fail(LFASM_ERR_ARG, "face orientations required for p >= 2");
  if (ad->rule_cc.nq <= 0 || ad->rule_mass.nq <= 0 || !ad->rule_cc.ip || !ad->rule_mass.ip ||
      !ad->rule_cc.curl || !ad->rule_mass.curl || !ad->rule_mass.vshape || !ad->rule_cc.w ||
      !ad->rule_mass.w)
    return fail(LFASM_ERR_ARG, "missing reference rule tables");
  if (ad->rule_cc.nq + ad->rule_mass.nq > PML_MAXQ)
    return fail(LFASM_ERR_UNSUPPORTED, "%d + %d quadrature points exceed the %d per element supported",
                ad->rule_cc.nq, ad->rule_mass.nq, PML_MAXQ);
  if (prob->n_regions <= 0 || !prob->region_eps || !prob->region_kind)
    return fail(LFASM_ERR_ARG, "missing region table");
  if (!(prob->pml_thick > 0.0) || !(prob->k0 > 0.0))
    return fail(LFASM_ERR_ARG, "k0 and pml thickness must be positive");
  const size_t ne = ad->ne;
  const size_t nen = ne * nd;
  {
    const int *dof = ad->dof, *attr = ad->attr, *fo = ad->fo;
    const double *detJ = ad->detJ;
    const unsigned hgt = (unsigned)ad->height, nreg = (unsigned)prob->n_regions;
    size_t i = first_bad(nen, [&](size_t k) { return (int)((unsigned)dof[k] >= hgt); });
    if (i < nen)
      return fail(LFASM_ERR_ARG, "dof[%zu] = %d out of range [0, %d)", i, ad->dof[i], ad->height);
    const size_t ea = first_bad(ne, [&](size_t k) { return (int)((unsigned)(attr[k] - 1) >= nreg); });
    const size_t ed = first_bad(ne, [&](size_t k) { return (int)!(detJ[k] > 0.0); });
    if (ea < ne && ea <= ed)
      return fail(LFASM_ERR_ARG, "attr[%zu] = %d outside 1..%d", ea, ad->attr[ea], prob->n_regions);
    if (ed < ne) return fail(LFASM_ERR_ARG, "detJ[%zu] not positive", ed);
    if (ad->p >= 2) {
      i = first_bad(ne * 4, [&](size_t k) { return (int)((unsigned)fo[k] > 5u); });
      if (i < ne * 4) return fail(LFASM_ERR_ARG, "fo[%zu] = %d outside 0..5", i, ad->fo[i]);
    }
  }

  int ndev = 0;
  LF_CUDA(cudaGetDeviceCount(&ndev));
  if (gpu_id < 0 || gpu_id >= ndev)
    return fail(LFASM_ERR_ARG, "gpu_id %d outside the %d visible devices", gpu_id, ndev);
  LF_CUDA(cudaSetDevice(gpu_id));

  lfasm_handle *h = new lfasm_handle();
  h->dev = gpu_id;
  h->ne = ad->ne;
  h->nd = nd;
  h->p = ad->p;
  h->n = ad->height;
  h->has_kpar = (prob->kx != 0.0 || prob->ky != 0.0) ? 1 : 0;
  h->ndp = (nd + 1) & ~1;
  h->rs = (nd + 7) & ~7;  // fused element-buffer row stride: rows on 128-byte lines
  h->ndp4 = (nd + 3) & ~3;
  if (ad->I || ad->Jcol) {
    if (!ad->I || !ad->Jcol || ad->nnz <= 0) {
      delete h;
      return fail(LFASM_ERR_ARG, "I and Jcol must be given together with nnz > 0");
    }
    if (ad->I[0] != 0 || ad->I[ad->height] != ad->nnz) {
      delete h;
      return fail(LFASM_ERR_ARG, "row pointer does not span [0, nnz)");
    }
    h->h_I.assign(ad->I, ad->I + ad->height + 1);
    h->h_J.assign(ad->Jcol, ad->Jcol + ad->nnz);
  }
  auto bail = [&](int code) { lfasm_destroy(h); return code; };
#define LF_CUDA_H(call)                                                        \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      std::printf("asm_gpu: CUDA error '%s' at %s:%d\n",                       \
                  cudaGetErrorString(e_), __FILE__, __LINE__);                 \
      std::fflush(stdout);                                                     \
      fail(LFASM_ERR_CUDA, "CUDA error '%s' at %s:%d", cudaGetErrorString(e_), \
           __FILE__, __LINE__);                                                \
      return bail(LFASM_ERR_CUDA);                                             \
    }                                                                          \
  } while (0)

  double tinv[24];
  build_tinv(tinv);
  LF_CUDA_H(cudaMemcpyToSymbol(c_tinv, tinv, sizeof(tinv)));

  LF_CUDA_H(upload(h->dof, ad->dof, nen));
  LF_CUDA_H(upload(h->sign, ad->sign, nen));
  LF_CUDA_H(upload(h->attr, ad->attr, ne));
  LF_CUDA_H(upload(h->J, ad->J, ne * 9));
  LF_CUDA_H(upload(h->Jinv, ad->Jinv, ne * 9));
  LF_CUDA_H(upload(h->detJ, ad->detJ, ne));
  LF_CUDA_H(upload(h->v0, ad->v0, ne * 3));
  // packed per-element orientation and sign bits, formed on the device
  {
    int *dfo = nullptr;
    if (ad->p >= 2) LF_CUDA_H(upload(dfo, ad->fo, ne * 4));
    LF_CUDA_H(dmalloc(h->fopack, ne));
    LF_CUDA_H(dmalloc(h->signmask, ne));
    k_pack<<<(unsigned)((ne + 255) / 256), 256>>>((int)ne, nd, ad->p, h->sign, dfo, h->fopack,
                                                  h->signmask);
    LF_LAUNCHED();
    LF_CUDA_H(cudaGetLastError());
    dfree(dfo);
  }
  auto up_rule = [&](DevRule &d, const lfasm_ref_rule &r) -> cudaError_t {
    d.nq = r.nq;
    cudaError_t e;
    if ((e = upload(d.ip, r.ip, (size_t)r.nq * 3)) != cudaSuccess) return e;
    if ((e = upload(d.w, r.w, (size_t)r.nq)) != cudaSuccess) return e;
    if (r.vshape && (e = upload(d.v, r.vshape, (size_t)r.nq * nd * 3)) != cudaSuccess) return e;
    if ((e = upload(d.c, r.curl, (size_t)r.nq * nd * 3)) != cudaSuccess) return e;
    d.ldt = (nd + 7) & ~7;
    const std::vector<double> vt = component_major(r.vshape, r.nq, nd, d.ldt);
    const std::vector<double> ct = component_major(r.curl, r.nq, nd, d.ldt);
    if ((e = upload(d.vt, vt.data(), vt.size())) != cudaSuccess) return e;
    return upload(d.ct, ct.data(), ct.size());
  };
  LF_CUDA_H(up_rule(h->rcc, ad->rule_cc));
  LF_CUDA_H(up_rule(h->rm, ad->rule_mass));

  std::vector<dcplx> eps(prob->n_regions);
  for (int r = 0; r < prob->n_regions; ++r)
    eps[r] = dcplx{prob->region_eps[2 * r], prob->region_eps[2 * r + 1]};
  LF_CUDA_H(upload(h->eps_tab, eps.data(), eps.size()));
  if (prob->elem_eps) {
    LF_CUDA_H(upload(h->elem_eps, reinterpret_cast<const dcplx *>(prob->elem_eps), ne));
  }

  PmlParams &pm = h->pml;
  pm.z_min = prob->z_min;
  pm.z_max = prob->z_max;
  pm.thick = prob->pml_thick;
  pm.order = prob->pml_order;
  pm.k0 = prob->k0;
  pm.kx = prob->kx;
  pm.ky = prob->ky;
  double n_bot = 1.0, n_top = 1.0;
  for (int r = 0; r < prob->n_regions; ++r) {
    const double er = prob->region_eps[2 * r], ei = prob->region_eps[2 * r + 1];
    // |sqrt(eps)| = |eps|^(1/2)
    const double nm = std::sqrt(std::sqrt(er * er + ei * ei));
    if (prob->region_kind[r] == LFASM_REGION_PML_BOTTOM) n_bot = nm;
    if (prob->region_kind[r] == LFASM_REGION_PML_TOP) n_top = nm;
  }
  pm.smax_bot = -std::log(prob->pml_target) * (prob->pml_order + 1) /
                (2.0 * prob->k0 * n_bot * prob->pml_thick);
  pm.smax_top = -std::log(prob->pml_target) * (prob->pml_order + 1) /
                (2.0 * prob->k0 * n_top * prob->pml_thick);

  // classify on the device: bulk iff s(z_q) == 1 exactly at every point of
  // both rules; both element lists stay in ascending element order
  std::vector<int> has_bulk(prob->n_regions, 0);
  {
    int *flag = nullptr, *pos = nullptr, *rhb = nullptr;
    unsigned char *tmp = nullptr;
    size_t tmp_bytes = 0;
    LF_CUDA_H(dmalloc(flag, ne + 1));
    LF_CUDA_H(dmalloc(pos, ne + 1));
    LF_CUDA_H(dmalloc(rhb, (size_t)prob->n_regions));
    LF_CUDA_H(dmalloc(h->bulk_list, ne));
    LF_CUDA_H(dmalloc(h->pml_list, ne));
    LF_CUDA_H(cudaMemsetAsync(flag, 0, (ne + 1) * sizeof(int), 0));
    LF_CUDA_H(cudaMemsetAsync(rhb, 0, (size_t)prob->n_regions * sizeof(int), 0));
    const unsigned gb = (unsigned)((ne + 255) / 256);
    k_classify<<<gb, 256>>>((int)ne, h->rcc.view(), h->rm.view(), h->J, h->v0, h->attr,
                            pm.z_min, pm.z_max, flag, rhb);
    LF_LAUNCHED();
    LF_CUDA_H(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, flag, pos, (int)ne + 1, 0));
    LF_CUDA_H(dmalloc(tmp, tmp_bytes));
    LF_CUDA_H(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, flag, pos, (int)ne + 1, 0));
    k_split_lists<<<gb, 256>>>((int)ne, flag, pos, h->bulk_list, h->pml_list);
    LF_LAUNCHED();
    int nb = 0;
    LF_CUDA_H(cudaMemcpy(&nb, pos + ne, sizeof(int), cudaMemcpyDeviceToHost));
    LF_CUDA_H(cudaMemcpy(has_bulk.data(), rhb, has_bulk.size() * sizeof(int),
                         cudaMemcpyDeviceToHost));
    dfree(flag); dfree(pos); dfree(rhb); dfree(tmp);
    h->n_bulk = nb;
    h->n_pml = (int)ne - nb;
  }
  if (h->n_bulk) LF_CUDA_H(dmalloc(h->rec, (size_t)h->n_bulk * REC));

  {
    std::vector<double> key = rule_key(ad, h->ndp);
    std::lock_guard<std::mutex> lk(g_stab_mu);
    const STables *hit = nullptr;
    for (const STables &t : g_stab)
      if (t.key == key) { hit = &t; break; }
    if (!hit) {
      STables t;
      t.key = std::move(key);
      build_S(ad, h->ndp, t.S);
      build_S_mma(ad, h->ndp, false, t.S_mma);
      build_S_mma(ad, h->ndp, true, t.S_mmaf);
      if (g_stab.size() >= 16) g_stab.erase(g_stab.begin());
      g_stab.push_back(std::move(t));
      hit = &g_stab.back();
    }
    LF_CUDA_H(upload(h->S, hit->S.data(), hit->S.size()));
    LF_CUDA_H(upload(h->S_mma, hit->S_mma.data(), hit->S_mma.size()));
    LF_CUDA_H(upload(h->S_mmaf, hit->S_mmaf.data(), hit->S_mmaf.size()));
  }
  if (h->n_bulk)
    LF_CUDA_H(dmalloc(h->rec_mma, (size_t)h->n_bulk * BREC));

  // RHS source elements: frustum regions (delta = region eps - eps_bg) or,
  // with per-element eps, every non-PML element whose eps differs from its
  // slab background.
  {
    std::vector<int> slab(ne, 0), src, slot(ne, -1);
    std::vector<dcplx> del(ne, dcplx{0.0, 0.0});
    std::vector<int> bg_of_slab(prob->n_regions + 1, -1);
    int max_slab = 0;
    for (int r = 0; r < prob->n_regions; ++r)
      if (prob->region_slab) max_slab = std::max(max_slab, prob->region_slab[r]);
    std::vector<int> bg(max_slab + 2, -1);
    for (int r = 0; r < prob->n_regions; ++r)
      if (prob->region_kind[r] == LFASM_REGION_BACKGROUND && prob->region_slab &&
          prob->region_slab[r] >= 0)
        bg[prob->region_slab[r]] = r;
    for (size_t e = 0; e < ne; ++e) {
      const int r = ad->attr[e] - 1;
      const int kind = prob->region_kind[r];
      slab[e] = prob->region_slab ? prob->region_slab[r] : 0;
      dcplx d{0.0, 0.0};
      if (kind == LFASM_REGION_FRUSTUM && prob->region_delta_eps)
        d = dcplx{prob->region_delta_eps[2 * r], prob->region_delta_eps[2 * r + 1]};
      if (prob->elem_eps && (kind == LFASM_REGION_BACKGROUND || kind == LFASM_REGION_FRUSTUM) &&
          slab[e] >= 0 && bg[slab[e]] >= 0) {
        const int b = bg[slab[e]];
        d = dcplx{prob->elem_eps[2 * e] - prob->region_eps[2 * b],
                  prob->elem_eps[2 * e + 1] - prob->region_eps[2 * b + 1]};
      }
      del[e] = d;
      if (d.re != 0.0 || d.im != 0.0) {
        slot[e] = (int)src.size();
        src.push_back((int)e);
        h->max_src_slab = std::max(h->max_src_slab, slab[e]);
      }
    }
    h->n_src = (int)src.size();
    for (int r = 0; r < prob->n_regions; ++r)
      if (has_bulk[r])
        h->max_bulk_slab = std::max(h->max_bulk_slab, prob->region_slab ? prob->region_slab[r] : 0);
    LF_CUDA_H(upload(h->slab_of, slab.data(), ne));
    LF_CUDA_H(upload(h->delta, del.data(), ne));
    LF_CUDA_H(upload(h->src_list, src.data(), src.size()));
    LF_CUDA_H(upload(h->src_slot, slot.data(), ne));
  }

  // element buffer: dense nd x nd rows for lfasm_compute_local, padded row
  // stride ndp (even) for the fused path so every row starts on a 32-byte
  // sector and column pairs fill whole sectors
  LF_CUDA_H(dmalloc(h->Ae, ne * nd * h->rs));
  LF_CUDA_H(dmalloc(h->err, 1));
  LF_CUDA_H(cudaMemset(h->err, 0, sizeof(int)));
  LF_CUDA_H(cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, gpu_id));
  LF_CUDA_H(cudaDeviceGetAttribute(&h->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, gpu_id));
  LF_CUDA_H(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
  LF_CUDA_H(cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming));
  LF_CUDA_H(cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming));
  LF_CUDA_H(cudaDeviceSynchronize());
#undef LF_CUDA_H
  *out = h;
  return LFASM_OK;
}

int lfasm_set_stream(lfasm_handle *h, void *stream) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  h->stream = (cudaStream_t)stream;
  return LFASM_OK;
}

int lfasm_set_async(lfasm_handle *h, int async_mode) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  h->async_mode = async_mode ? 1 : 0;
  return LFASM_OK;
}

int lfasm_path_counts(lfasm_handle *h, int *n_bulk, int *n_pml) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  if (n_bulk) *n_bulk = h->n_bulk;
  if (n_pml) *n_pml = h->n_pml;
  return LFASM_OK;
}

}  // extern "C"

// PML elements pml_list[q0 .. q0 + nq) (nq < 0: the whole list)
template <int NDP8>
static int launch_pml(lfasm_handle *h, bool cross, int mode, int mask_cc, int mask_mass, int te,
                      int eliminate, int rs, cudaStream_t st, int q0 = 0, int nq = -1) {
  if (nq < 0) nq = h->n_pml - q0;
  if (nq <= 0) return LFASM_OK;
  const int *plist = h->pml_list + q0;
  size_t smem = PmlShape<NDP8>::smem(PmlShape<NDP8>::QC, h->rcc.nq + h->rm.nq);
  const int threads = NDP8 * 4;
  auto go = [&](auto kern) -> int {
    LF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    LF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
    const int grid = std::max(1, std::min(nq, std::max(per_sm, 1) * h->sm_count));
    kern<<<grid, threads, smem, st>>>(
        nq, plist, h->nd, rs, h->p, h->rcc.view(), h->rm.view(), h->J, h->Jinv,
        h->detJ, h->v0, h->attr, h->eps_tab, h->elem_eps, h->pml, mask_cc, mask_mass, te,
        eliminate, h->fopack, h->signmask, h->essmask, h->Ae);
    LF_LAUNCHED();
    return LFASM_OK;
  };
  if (NDP8 == 48 && h->pml_variant == 1) {
    const size_t wsm = PmlWsShape::smem(h->rcc.nq + h->rm.nq);
    auto ws = [&](auto kern) -> int {
      LF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm));
      const int grid = std::max(1, std::min(nq, h->sm_count));
      kern<<<grid, WS_THREADS, wsm, st>>>(
          nq, plist, h->nd, rs, h->p, h->rcc.view(), h->rm.view(), h->J, h->Jinv,
          h->detJ, h->v0, h->attr, h->eps_tab, h->elem_eps, h->pml, mask_cc, mask_mass, te,
          eliminate, h->fopack, h->signmask, h->essmask, h->Ae, h->err);
      LF_LAUNCHED();
      return LFASM_OK;
    };
    if (cross) return mode ? ws(k_pml_ws<true, 1>) : ws(k_pml_ws<true, 0>);
    return mode ? ws(k_pml_ws<false, 1>) : ws(k_pml_ws<false, 0>);
  }
  if (h->pml_variant == 2) {
    // mask_cc never carries the cross bits, so cross = cross terms in mask_mass
    smem = PmlSymShape<NDP8>::smem(h->rcc.nq + h->rm.nq, cross);
    if (cross) return mode ? go(k_pml_sym<NDP8, true, 1>) : go(k_pml_sym<NDP8, true, 0>);
    return mode ? go(k_pml_sym<NDP8, false, 1>) : go(k_pml_sym<NDP8, false, 0>);
  }
  if (cross) return mode ? go(k_pml_mma<NDP8, true, 1>) : go(k_pml_mma<NDP8, true, 0>);
  return mode ? go(k_pml_mma<NDP8, false, 1>) : go(k_pml_mma<NDP8, false, 0>);
}

// bulk elements bulk_list[b0 .. b0 + nb): the coefficient records (prep)
// and / or the element matrices (body), on stream st
static int launch_bulk(lfasm_handle *h, int mask, int te, int mode, int eliminate, int rs,
                       int b0, int nb, bool prep, bool body, cudaStream_t st) {
  if (nb <= 0) return LFASM_OK;
  const bool cross = (mask & (LFASM_CROSS0 | LFASM_CROSS1)) != 0;
  const int *blist = h->bulk_list + b0;
  if (h->bulk_variant == 0) {
    if (prep) {
      k_prep_bulk<<<(nb + 127) / 128, 128, 0, st>>>(nb, blist, h->J, h->Jinv, h->detJ, h->attr,
                                                    h->eps_tab, h->elem_eps, h->pml, mask,
                                                    h->rec + (size_t)b0 * REC);
      LF_LAUNCHED();
    }
    if (!body) return LFASM_OK;
    const int nthr = bulk_threads(h->ndp);
    const int ytiles = (nthr + BULK_THREADS - 1) / BULK_THREADS;
    const long long want = (long long)h->sm_count * 8;
    int chunk = (int)std::max<long long>(16, ((long long)nb * ytiles + want - 1) / want);
    chunk = (chunk + BULK_EB - 1) / BULK_EB * BULK_EB;
    dim3 grid((nb + chunk - 1) / chunk, ytiles);
#define LF_BULK(C, M)                                                             \
  k_bulk<C, M><<<grid, BULK_THREADS, 0, st>>>(                                    \
      nb, blist, h->rec + (size_t)b0 * REC, h->S, nthr, h->nd, h->ndp, h->p, chunk, te,       \
      eliminate, rs, (mask & LFASM_CROSS0) ? 1 : 0, (mask & LFASM_CROSS1) ? 1 : 0,  \
      h->fopack, h->signmask, h->essmask, h->Ae)
    if (cross) { if (mode) LF_BULK(true, 1); else LF_BULK(true, 0); }
    else { if (mode) LF_BULK(false, 1); else LF_BULK(false, 0); }
#undef LF_BULK
    LF_LAUNCHED();
  } else {
    // both cross terms or neither: the fused Bloch layout (7 k-steps a tile)
    const bool fused = ((mask & LFASM_CROSS0) != 0) == ((mask & LFASM_CROSS1) != 0);
    double *recm = h->rec_mma + (size_t)b0 * (fused ? BK : BREC);
    if (prep) {
      k_prep_bulk_mma<<<(nb + 127) / 128, 128, 0, st>>>(nb, blist, h->J, h->Jinv, h->detJ,
                                                        h->attr, h->eps_tab, h->elem_eps, h->pml,
                                                        mask, fused ? 1 : 0, recm);
      LF_LAUNCHED();
    }
    if (!body) return LFASM_OK;
    const int ntiles = bulk_tiles(h->ndp);
    const int TT = (h->bulk_variant == 2 || h->bulk_variant == 4) ? 2 : 4;  // tiles per warp
    const bool nobar = h->bulk_variant == 3 || h->bulk_variant == 4;
    const bool tma = h->bulk_variant == 5;
    const int ytiles = (ntiles + BULK_WARPS * TT - 1) / (BULK_WARPS * TT);
    // k_bulk_mma writes 16-byte-aligned double4 pairs: needs rs even (the
    // fused layout); the dense ComputeLocal layout uses the SIMT kernel
    const int nbat = (nb + 7) / 8;
    const long long want = (long long)h->sm_count * 8;
    const int bchunk = (int)std::max<long long>(1, ((long long)nbat * ytiles + want - 1) / want);
    dim3 grid((nbat + bchunk - 1) / bchunk, ytiles);
#define LF_BULKM(C, M, T, F)                                                      \
  do {                                                                            \
    if (tma)                                                                      \
      k_bulk_tma<C, M, T, F><<<grid, BULK_WARPS * 32, 0, st>>>(                   \
          nb, blist, recm, F ? h->S_mmaf : h->S_mma, ntiles, h->nd, h->ndp, h->p, \
          bchunk, te, eliminate, rs, h->fopack, h->signmask, h->essmask, h->Ae,   \
          h->err);                                                                \
    else                                                                          \
      (nobar ? k_bulk_mma_nb<C, M, T, F> : k_bulk_mma<C, M, T, F>)                \
          <<<grid, BULK_WARPS * 32, 0, st>>>(                                     \
          nb, blist, recm, F ? h->S_mmaf : h->S_mma, ntiles, h->nd, h->ndp,       \
          h->p, bchunk, te, eliminate, rs, h->fopack, h->signmask, h->essmask,    \
          h->Ae);                                                                 \
  } while (0)
#define LF_BULKM_T(T, F)                                                          \
  do {                                                                            \
    if (cross) { if (mode) LF_BULKM(true, 1, T, F); else LF_BULKM(true, 0, T, F); }   \
    else { if (mode) LF_BULKM(false, 1, T, F); else LF_BULKM(false, 0, T, F); }       \
  } while (0)
    if (TT == 4) {
      if (fused) LF_BULKM_T(4, true); else LF_BULKM_T(4, false);
    } else {
      if (fused) LF_BULKM_T(2, true); else LF_BULKM_T(2, false);
    }
#undef LF_BULKM_T
#undef LF_BULKM
    LF_LAUNCHED();
  }
  return LFASM_OK;
}

extern "C" {

static int launch_local(lfasm_handle *h, int mask_cc, int mask_mass, int te, int mode,
                        int eliminate) {
  if ((mask_cc & ~LFASM_CURLCURL) || (mask_mass & LFASM_CURLCURL) || (mask_mass & ~31))
    return fail(LFASM_ERR_UNSUPPORTED,
                "mask_cc may select only CURLCURL and mask_mass only MASS|CROSS0|CROSS1|KLK");
  LF_CUDA(cudaSetDevice(h->dev));
  const int mask = mask_cc | mask_mass;
  const bool cross = (mask & (LFASM_CROSS0 | LFASM_CROSS1)) != 0;
  const bool prof = mode == 1 && h->profile;
  // every element is written by exactly one of the two paths: no memset.
  // The PML elements (tensor-pipe bound) run on the side stream next to the
  // bulk elements (HBM bound) unless stage timing is requested.
  const bool overlap = !prof && h->n_bulk > 0 && h->n_pml > 0;
  cudaStream_t pst = overlap ? h->side : h->stream;
  if (prof) LF_CUDA(cudaEventRecord(h->ev[0], h->stream));
  if (overlap) {
    LF_CUDA(cudaEventRecord(h->fork, h->stream));
    LF_CUDA(cudaStreamWaitEvent(h->side, h->fork, 0));
  }
  const int rs = mode ? h->rs : h->nd;
  if (h->n_bulk) {
    int rc = launch_bulk(h, mask, te, mode, eliminate, rs, 0, h->n_bulk, true, true, h->stream);
    if (rc) return rc;
  }
  if (prof) LF_CUDA(cudaEventRecord(h->ev[1], h->stream));
  if (h->n_pml) {
    int rc = h->p == 1 ? launch_pml<8>(h, cross, mode, mask_cc, mask_mass, te, eliminate, rs, pst)
           : h->p == 2 ? launch_pml<24>(h, cross, mode, mask_cc, mask_mass, te, eliminate, rs, pst)
                       : launch_pml<48>(h, cross, mode, mask_cc, mask_mass, te, eliminate, rs, pst);
    if (rc) return rc;
  }
  if (overlap) {
    LF_CUDA(cudaEventRecord(h->join, h->side));
    LF_CUDA(cudaStreamWaitEvent(h->stream, h->join, 0));
  }
  if (prof) LF_CUDA(cudaEventRecord(h->ev[2], h->stream));
  return LFASM_OK;
}

int lfasm_compute_local(lfasm_handle *h, int mask_cc, int mask_mass, int apply_te) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  g_err.clear();
  if (!mask_cc && !mask_mass) {
    LF_CUDA(cudaSetDevice(h->dev));
    LF_CUDA(cudaMemsetAsync(h->Ae, 0, (size_t)h->ne * h->nd * h->nd * sizeof(dcplx), h->stream));
  } else {
    int rc = launch_local(h, mask_cc, mask_mass, apply_te ? 1 : 0, 0, 0);
    if (rc) return rc;
  }
  h->locals_valid = 1;
  return sync_if(h);
}

int lfasm_get_local(lfasm_handle *h, void **d_local) {
  if (!h || !d_local) return fail(LFASM_ERR_ARG, "NULL argument");
  *d_local = h->Ae;
  return LFASM_OK;
}

int lfasm_download_local(lfasm_handle *h, double *host_out) {
  if (!h || !host_out) return fail(LFASM_ERR_ARG, "NULL argument");
  std::printf("asm_gpu_test_download (test-only D2H)\n");
  std::fflush(stdout);
  LF_CUDA(cudaSetDevice(h->dev));
  LF_CUDA(cudaStreamSynchronize(h->stream));
  LF_CUDA(cudaMemcpy(host_out, h->Ae, (size_t)h->ne * h->nd * h->nd * sizeof(dcplx),
                     cudaMemcpyDeviceToHost));
  return LFASM_OK;
}

}  // extern "C"

// symbolic CSR + row maps
static int build_maps(lfasm_handle *h, const int *hI, const int *hJ, long long nnz_given) {
  const int n = h->n, nd = h->nd;
  const long long total = (long long)h->ne * nd;
  // int32 CSR (the cuDSS contract) and int32 row-list positions: the
  // candidate count ne * nd^2 bounds nnz and every position used here
  if (total * nd > (long long)INT_MAX)
    return fail(LFASM_ERR_UNSUPPORTED,
                "%lld element couplings exceed the int32 CSR (ne * nd^2 must stay below 2^31)",
                total * nd);
  int *cnt = nullptr, *fill = nullptr, *dmax = nullptr, *err = nullptr;
  int *tmpJ = nullptr;  // every row's unique columns at its candidate offset
  unsigned char *tmp = nullptr;
  size_t tmp_bytes = 0;
  LF_CUDA(dmalloc(cnt, (size_t)(n + 1)));
  LF_CUDA(dmalloc(fill, (size_t)n));
  LF_CUDA(dmalloc(dmax, 2));
  LF_CUDA(dmalloc(err, 1));
  LF_CUDA(cudaMemsetAsync(cnt, 0, (size_t)(n + 1) * sizeof(int), h->stream));
  LF_CUDA(cudaMemsetAsync(fill, 0, (size_t)n * sizeof(int), h->stream));
  LF_CUDA(cudaMemsetAsync(dmax, 0, 2 * sizeof(int), h->stream));
  LF_CUDA(cudaMemsetAsync(err, 0, sizeof(int), h->stream));
  LF_CUDA(dmalloc(h->ea_ptr, (size_t)(n + 1)));
  LF_CUDA(dmalloc(h->ea, (size_t)total));
  const int tb = 256;
  const unsigned gb = (unsigned)((total + tb - 1) / tb);
  k_count_rows<<<gb, tb, 0, h->stream>>>(total, h->dof, cnt);
  LF_LAUNCHED();
  LF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt, h->ea_ptr, n + 1, h->stream));
  LF_CUDA(dmalloc(tmp, tmp_bytes));
  LF_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cnt, h->ea_ptr, n + 1, h->stream));
  k_fill_rows<<<gb, tb, 0, h->stream>>>(total, h->dof, h->ea_ptr, fill, h->ea);
  LF_LAUNCHED();
  k_max_reduce<<<256, 256, 0, h->stream>>>(n, h->ea_ptr, 1, dmax);
  LF_LAUNCHED();
  int mmax = 0;
  LF_CUDA(cudaMemcpyAsync(&mmax, dmax, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  LF_CUDA(cudaStreamSynchronize(h->stream));
  if (mmax > 64) {
    dfree(cnt); dfree(fill); dfree(dmax); dfree(err); dfree(tmp);
    return fail(LFASM_ERR_UNSUPPORTED, "a dof belongs to %d elements (max 64)", mmax);
  }
  int cap = 32;
  while (cap < mmax * nd) cap <<= 1;
  const int wpb = 4;
  const size_t smem = (size_t)wpb * (cap + 64) * sizeof(int);
  const unsigned rb = (unsigned)((n + wpb - 1) / wpb);
  LF_CUDA(dmalloc(h->off, (size_t)total * nd));
  if (!hI) {
    LF_CUDA(dmalloc(tmpJ, (size_t)total * nd));
    LF_CUDA(cudaFuncSetAttribute(k_row_symbolic<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_row_symbolic<1><<<rb, wpb * 32, smem, h->stream>>>(n, nd, h->dof, h->ea_ptr, h->ea, cap,
                                                          cnt, nullptr, nullptr, tmpJ, h->off, err);
    LF_LAUNCHED();
    LF_CUDA(dmalloc(h->I, (size_t)(n + 1)));
    LF_CUDA(cudaMemsetAsync(cnt + n, 0, sizeof(int), h->stream));
    LF_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cnt, h->I, n + 1, h->stream));
    int nnz = 0;
    LF_CUDA(cudaMemcpyAsync(&nnz, h->I + n, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    LF_CUDA(cudaStreamSynchronize(h->stream));
    h->nnz = nnz;
    LF_CUDA(dmalloc(h->Jc, (size_t)std::max(nnz, 1)));
    k_row_compact<<<(unsigned)((n + 7) / 8), 256, 0, h->stream>>>(n, nd, h->ea_ptr, h->I, tmpJ,
                                                                   h->Jc);
    LF_LAUNCHED();
  } else {
    // map every row's candidates into the caller's sparsity
    h->nnz = nnz_given;
    LF_CUDA(upload(h->I, hI, (size_t)n + 1));
    LF_CUDA(upload(h->Jc, hJ, (size_t)nnz_given));
    LF_CUDA(cudaFuncSetAttribute(k_row_symbolic<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_row_symbolic<3><<<rb, wpb * 32, smem, h->stream>>>(n, nd, h->dof, h->ea_ptr, h->ea, cap,
                                                          nullptr, h->I, h->Jc, nullptr, h->off, err);
    LF_LAUNCHED();
  }
  k_max_reduce<<<256, 256, 0, h->stream>>>(n, h->I, 1, dmax + 1);
  LF_LAUNCHED();
  int herr = 0, mrow = 0;
  LF_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  LF_CUDA(cudaMemcpyAsync(&mrow, dmax + 1, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  LF_CUDA(cudaStreamSynchronize(h->stream));
  dfree(cnt); dfree(fill); dfree(dmax); dfree(err); dfree(tmp); dfree(tmpJ);
  if (herr == 1) return fail(LFASM_ERR_CSR, "CSR position missing: the given sparsity lacks an element coupling");
  if (herr) return fail(LFASM_ERR_UNSUPPORTED, "row map overflow");
  if (mrow > 65535) return fail(LFASM_ERR_UNSUPPORTED, "row with %d entries exceeds 65535", mrow);
  h->max_row = std::max(mrow, 1);
  // gather: rows up to GATHER_ROW_CAP entries accumulate in shared memory
  constexpr int GATHER_ROW_CAP = 256;
  h->row_cap = std::min(h->max_row, GATHER_ROW_CAP);
  h->n_long = 0;
  if (h->max_row > h->row_cap) {
    int *cnt_d = nullptr;
    LF_CUDA(dmalloc(cnt_d, 1));
    LF_CUDA(dmalloc(h->long_rows, (size_t)n));
    LF_CUDA(cudaMemsetAsync(cnt_d, 0, sizeof(int), h->stream));
    k_long_rows<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(n, h->I, h->row_cap,
                                                                   h->long_rows, cnt_d);
    LF_LAUNCHED();
    LF_CUDA(cudaMemcpyAsync(&h->n_long, cnt_d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    LF_CUDA(cudaStreamSynchronize(h->stream));
    dfree(cnt_d);
  }
  return LFASM_OK;
}

// Chunks for lfasm_assemble (fused element rows only: rs a multiple of 8,
// so that each element row is whole 128-byte lines), when LFASM_CHUNK_MB
// sets the element-row megabytes per chunk (default 0: one pass).  On the
// 1.35M-DOF line grating the chunked sequence measured 3.0-3.1 ms per
// assembly at 32-96 MB chunks against 2.70 ms in one pass (about 9 us of
// kernel ramp and tail per chunk on the chunk -> gather chain, and no
// overlap with the PML kernel, which fills every SM's register file), so it
// stays an option.
// The bulk elements are ordered by centroid height and cut into chunks of
// equal size; the PML elements (at the two ends in height) form one launch
// of their own.  Rows are ordered by the last bulk chunk that holds one of
// their element rows, and rows touching a PML element come last (group
// nchunk).
static int setup_chunks(lfasm_handle *h) {
  h->nchunk = 0;
  double mb = 0.0;
  if (const char *e = std::getenv("LFASM_CHUNK_MB")) mb = std::atof(e);
  if (mb <= 0.0 || h->rs % 8 != 0 || h->n_bulk <= 0) return LFASM_OK;
  const double row_bytes = (double)h->nd * h->rs * sizeof(dcplx);
  const int per = std::max(1, (int)(mb * 1048576.0 / row_bytes));
  const int nb = h->n_bulk;
  const int nc = (nb + per - 1) / per;
  if (nc < 2) return LFASM_OK;
  cudaStream_t st = h->stream;
  const int ne = h->ne, n = h->n;
  double *key = nullptr, *key2 = nullptr;
  int *ids = nullptr, *chunk_of = nullptr, *ki = nullptr, *ko = nullptr, *vi = nullptr;
  void *tmp = nullptr;
  size_t tb = 0, tneed = 0;
  const int mx = std::max(std::max(ne, n), 1);
  LF_CUDA(dmalloc(key, (size_t)ne));
  LF_CUDA(dmalloc(key2, (size_t)ne));
  LF_CUDA(dmalloc(ids, (size_t)ne));
  LF_CUDA(dmalloc(chunk_of, (size_t)ne));
  LF_CUDA(dmalloc(ki, (size_t)mx));
  LF_CUDA(dmalloc(ko, (size_t)mx));
  LF_CUDA(dmalloc(vi, (size_t)mx));
  LF_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tneed, key, key2, ids, ids, nb, 0, 64, st));
  tb = std::max(tb, tneed);
  LF_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tneed, ki, ko, vi, vi, n, 0, 32, st));
  tb = std::max(tb, tneed);
  LF_CUDA(dmalloc_bytes(&tmp, std::max<size_t>(tb, 16)));
  // bulk elements by height: keys of the bulk list, sorted into bulk_list
  k_list_zkey<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(nb, h->bulk_list, h->J, h->v0, key, ids);
  LF_LAUNCHED();
  LF_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, key, key2, ids, h->bulk_list, nb, 0, 64, st));
  k_fill_int<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(ne, nc, chunk_of);
  LF_LAUNCHED();
  k_chunk_of<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(nb, h->bulk_list, per, chunk_of);
  LF_LAUNCHED();
  h->chunk_b.assign(nc + 1, nb);
  for (int c = 0; c < nc; ++c) h->chunk_b[c] = c * per;
  // rows by completion group
  k_row_chunk<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, h->ea_ptr, h->ea, h->nd, chunk_of,
                                                            ki, vi);
  LF_LAUNCHED();
  dfree(h->row_order);
  LF_CUDA(dmalloc(h->row_order, (size_t)n));
  size_t t2 = tb;
  LF_CUDA(cub::DeviceRadixSort::SortPairs(tmp, t2, ki, ko, vi, h->row_order, n, 0, 32, st));
  std::vector<int> keys(n);
  LF_CUDA(cudaMemcpyAsync(keys.data(), ko, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  LF_CUDA(cudaStreamSynchronize(st));
  h->chunk_r.assign(nc + 2, n);
  h->chunk_r[0] = 0;
  for (int c = 1; c <= nc; ++c)
    h->chunk_r[c] = (int)(std::lower_bound(keys.begin(), keys.end(), c) - keys.begin());
  dfree(key); dfree(key2); dfree(ids); dfree(chunk_of); dfree(ki); dfree(ko); dfree(vi);
  dfree_bytes(tmp);
  if (!h->gstream) LF_CUDA(cudaStreamCreateWithFlags(&h->gstream, cudaStreamNonBlocking));
  if (!h->cstream) LF_CUDA(cudaStreamCreateWithFlags(&h->cstream, cudaStreamNonBlocking));
  h->nchunk = nc;
  return LFASM_OK;
}

static int build_global_csr(lfasm_handle *h, const int *hI, const int *hJ, long long nnz) {
  int rc = build_maps(h, hI, hJ, nnz);
  if (rc) return rc;
  LF_CUDA(dmalloc(h->vals, (size_t)std::max<long long>(h->nnz, 1)));
  h->n_part_blocks = (h->n + 7) / 8;
  LF_CUDA(dmalloc(h->partials, (size_t)h->n_part_blocks * 2));
  LF_CUDA(dmalloc(h->red, 2));
  if ((rc = setup_chunks(h))) return rc;
  h->built = 1;
  return sync_if(h);
}

extern "C" {

int lfasm_build_global(lfasm_handle *h, const int *ess_list, int n_ess) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  g_err.clear();
  if (h->built) return fail(LFASM_ERR_STATE, "global structure already built");
  if (n_ess < 0 || (n_ess > 0 && !ess_list)) return fail(LFASM_ERR_ARG, "bad essential list");
  LF_CUDA(cudaSetDevice(h->dev));
  std::vector<unsigned char> ess(h->n, 0);
  for (int i = 0; i < n_ess; ++i) {
    if (ess_list[i] < 0 || ess_list[i] >= h->n)
      return fail(LFASM_ERR_ARG, "essential dof %d out of range", ess_list[i]);
    ess[ess_list[i]] = 1;
  }
  LF_CUDA(upload(h->ess, ess.data(), ess.size()));
  LF_CUDA(dmalloc(h->essmask, (size_t)h->ne));
  k_essmask<<<(h->ne + 255) / 256, 256, 0, h->stream>>>(h->ne, h->nd, h->dof, h->ess, h->essmask);
  LF_LAUNCHED();
  if (h->h_I.empty()) return build_global_csr(h, nullptr, nullptr, 0);
  return build_global_csr(h, h->h_I.data(), h->h_J.data(), (long long)h->h_J.size());
}

static int gather(lfasm_handle *h, bool raw, int eliminate) {
  // one warp per row, each with the row's accumulator in shared memory
  // (h->row_cap entries); the few longer rows (h->long_rows) go to a second,
  // small launch that accumulates in place in global memory, so that they do
  // not cut the occupancy of the whole gather.  The kernels' dynamic shared
  // memory limit is the device maximum (an upper bound only), so launches of
  // several handles can share the kernels.
  const int cap = h->row_cap;
  const int wpb = 8;
  const size_t smem = (size_t)wpb * cap * sizeof(dcplx);
  const unsigned nb = (unsigned)((h->n + wpb - 1) / wpb);
  const unsigned nl = (unsigned)((h->n_long + wpb - 1) / wpb);
  const int rs = raw ? h->nd : h->rs;
#define LF_GATHER(R, L, grid, rows, sm)                                                       \
  k_gather<R, L><<<grid, wpb * 32, sm, h->stream>>>(rows, h->long_rows, h->ea_ptr, h->ea,      \
                                                    h->off, h->I, h->Jc, h->Ae, h->nd, rs,     \
                                                    h->ess, h->sign, h->dof, eliminate, cap,   \
                                                    (long long)h->ne * h->nd, h->vals)
  if (raw) {
    LF_CUDA(cudaFuncSetAttribute(k_gather<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, h->smem_optin));
    LF_GATHER(true, false, nb, h->n, smem);
    LF_LAUNCHED();
    if (h->n_long) { LF_GATHER(true, true, nl, h->n_long, 0); LF_LAUNCHED(); }
  } else {
    LF_CUDA(cudaFuncSetAttribute(k_gather<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, h->smem_optin));
    LF_GATHER(false, false, nb, h->n, smem);
    LF_LAUNCHED();
    if (h->n_long) { LF_GATHER(false, true, nl, h->n_long, 0); LF_LAUNCHED(); }
  }
#undef LF_GATHER
  return LFASM_OK;
}

int lfasm_scatter_eliminate(lfasm_handle *h, int eliminate) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  g_err.clear();
  if (!h->built) return fail(LFASM_ERR_STATE, "lfasm_build_global has not run");
  if (!h->locals_valid) return fail(LFASM_ERR_STATE, "lfasm_compute_local has not run");
  LF_CUDA(cudaSetDevice(h->dev));
  int rc = gather(h, true, eliminate ? 1 : 0);
  if (rc) return rc;
  return sync_if(h);
}

}  // extern "C"

// Per-process cache of autotuner decisions, keyed by device, order p,
// k-parallel terms and the power-of-two class of the bulk element count.
namespace {
struct TuneEntry {
  int variant;
  float ms[LFASM_BULK_VARIANTS];
  int pml_variant;
  float pml_ms[3];
};
std::mutex g_tune_mu;
std::map<std::array<int, 4>, TuneEntry> g_tune;

std::array<int, 4> tune_key(const lfasm_handle *h) {
  int cls = 0;
  while ((1 << cls) < h->n_bulk && cls < 30) ++cls;
  return {h->dev, h->p, h->has_kpar, cls};
}
}  // namespace

extern "C" {

// Autotuner: times each bulk-element variant on this mesh (two launches
// each, the second timed with CUDA events) and keeps the faster one.
int lfasm_autotune(lfasm_handle *h) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  if (!h->built) return fail(LFASM_ERR_STATE, "lfasm_build_global has not run");
  LF_CUDA(cudaSetDevice(h->dev));
  const int mm = LFASM_MASS | (h->has_kpar ? (LFASM_CROSS0 | LFASM_CROSS1 | LFASM_KLK) : 0);
  cudaEvent_t a, b;
  LF_CUDA(cudaEventCreate(&a));
  LF_CUDA(cudaEventCreate(&b));
  const int keep_n_pml = h->n_pml;
  h->n_pml = 0;  // time the bulk path alone
  int rc = LFASM_OK;
  for (int v = 0; v < LFASM_BULK_VARIANTS && !rc; ++v) {
    h->bulk_variant = v;
    for (int rep = 0; rep < 2 && !rc; ++rep) {
      LF_CUDA(cudaEventRecord(a, h->stream));
      rc = launch_local(h, LFASM_CURLCURL, mm, 1, 1, 1);
      LF_CUDA(cudaEventRecord(b, h->stream));
    }
    if (!rc) {
      LF_CUDA(cudaEventSynchronize(b));
      LF_CUDA(cudaEventElapsedTime(&h->tune_ms[v], a, b));
    }
  }
  h->n_pml = keep_n_pml;
  int ebulk = 0;
  if (!rc) {
    // the staged-record variant (5) is never chosen if one of its waits ran out
    LF_CUDA(cudaMemcpy(&ebulk, h->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (ebulk) LF_CUDA(cudaMemset(h->err, 0, sizeof(int)));
  }
  int best = 0;
  for (int v = 1; v < LFASM_BULK_VARIANTS; ++v)
    if (h->tune_ms[v] < h->tune_ms[best] && !(v == 5 && ebulk)) best = v;
  h->bulk_variant = best;
  if (!rc && h->n_pml > 0 && !h->pml_forced) {
    // PML kernels (the warp-specialised one at p = 3 only), the PML path alone
    const int keep_n_bulk = h->n_bulk;
    h->n_bulk = 0;
    for (int v = 0; v < 3 && !rc; ++v) {
      h->pml_ms[v] = 0.f;
      if (v == 1 && h->p != 3) continue;
      h->pml_variant = v;
      for (int rep = 0; rep < 2 && !rc; ++rep) {
        LF_CUDA(cudaEventRecord(a, h->stream));
        rc = launch_local(h, LFASM_CURLCURL, mm, 1, 1, 1);
        LF_CUDA(cudaEventRecord(b, h->stream));
      }
      if (!rc) {
        LF_CUDA(cudaEventSynchronize(b));
        LF_CUDA(cudaEventElapsedTime(&h->pml_ms[v], a, b));
      }
    }
    h->n_bulk = keep_n_bulk;
    if (!rc) {
      int e = 0;
      LF_CUDA(cudaMemcpy(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost));
      // a variant whose waits ran out is never chosen
      int bestp = 0;
      for (int v = 1; v < 3; ++v) {
        if (h->pml_ms[v] <= 0.f || (v == 1 && e)) continue;
        if (h->pml_ms[v] < h->pml_ms[bestp]) bestp = v;
      }
      h->pml_variant = bestp;
      if (e) LF_CUDA(cudaMemset(h->err, 0, sizeof(int)));
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  h->tuned = 1;
  h->locals_valid = 0;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    TuneEntry &t = g_tune[tune_key(h)];
    t.variant = best;
    for (int v = 0; v < LFASM_BULK_VARIANTS; ++v) t.ms[v] = h->tune_ms[v];
    t.pml_variant = h->pml_variant;
    for (int v = 0; v < 3; ++v) t.pml_ms[v] = h->pml_ms[v];
  }
  return sync_if(h);
}

int lfasm_set_bulk_variant(lfasm_handle *h, int variant) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  if (variant < 0 || variant >= LFASM_BULK_VARIANTS)
    return fail(LFASM_ERR_ARG, "bulk variant must be 0 .. %d", LFASM_BULK_VARIANTS - 1);
  h->bulk_variant = variant;
  h->forced = 1;
  h->tuned = 1;
  return LFASM_OK;
}

int lfasm_set_pml_variant(lfasm_handle *h, int variant) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  if (variant < 0 || variant > 2) return fail(LFASM_ERR_ARG, "PML variant must be 0, 1 or 2");
  if (variant == 1 && h->p != 3)
    return fail(LFASM_ERR_UNSUPPORTED, "the warp-specialised PML kernel is for p = 3");
  h->pml_variant = variant;
  h->pml_forced = 1;
  return LFASM_OK;
}

int lfasm_get_pml_tuning(lfasm_handle *h, int *pml_variant, float *ms3) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  if (pml_variant) *pml_variant = h->pml_variant;
  if (ms3) for (int i = 0; i < 3; ++i) ms3[i] = h->pml_ms[i];
  return LFASM_OK;
}

int lfasm_get_tuning(lfasm_handle *h, int *bulk_variant, float *ms) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  if (bulk_variant) *bulk_variant = h->bulk_variant;
  if (ms) for (int i = 0; i < LFASM_BULK_VARIANTS; ++i) ms[i] = h->tune_ms[i];
  return LFASM_OK;
}

// the kernel variants of a handle that has none set: the per-process cached
// decision for its kind of mesh, else the autotuner
static int ensure_tuned(lfasm_handle *h) {
  if (h->tuned) return LFASM_OK;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(tune_key(h));
    if (it != g_tune.end()) {
      h->bulk_variant = it->second.variant;
      for (int v = 0; v < LFASM_BULK_VARIANTS; ++v) h->tune_ms[v] = it->second.ms[v];
      if (!h->pml_forced) h->pml_variant = it->second.pml_variant;
      for (int v = 0; v < 3; ++v) h->pml_ms[v] = it->second.pml_ms[v];
      h->tuned = 1;
      return LFASM_OK;
    }
  }
  return lfasm_autotune(h);
}

}  // extern "C"

namespace {

// The chunked fused assembly, enqueued on h->cstream (bulk elements; it is
// the capture stream), h->side (all PML elements, one launch) and
// h->gstream (gathers): chunk c's gather waits for chunk c's bulk kernel
// only, so it runs while the next chunk's elements are computed; the rows
// touching PML elements follow the PML launch; rows longer than the shared
// accumulator are gathered at the end without discarding.  Captured into a
// graph by assemble_chunked.
int enqueue_chunked(lfasm_handle *h, int eliminate, std::vector<cudaEvent_t> &evs) {
  const int mm = LFASM_MASS | (h->has_kpar ? (LFASM_CROSS0 | LFASM_CROSS1 | LFASM_KLK) : 0);
  const int mask = LFASM_CURLCURL | mm;
  const bool cross = (mask & (LFASM_CROSS0 | LFASM_CROSS1)) != 0;
  cudaStream_t A = h->cstream, P = h->side, G = h->gstream;
  const int rs = h->rs;
  size_t ei = 0;
  auto ev = [&]() { return evs[ei++]; };
  const int wpb = 8;
  const size_t smem = (size_t)wpb * h->row_cap * sizeof(dcplx);
  LF_CUDA(cudaFuncSetAttribute(k_gather_list, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               h->smem_optin));
  auto gather_group = [&](int c) {
    const int r0 = h->chunk_r[c], nr = h->chunk_r[c + 1] - r0;
    if (nr > 0) {
      k_gather_list<<<(unsigned)((nr + wpb - 1) / wpb), wpb * 32, smem, G>>>(
          nr, h->row_order + r0, h->ea_ptr, h->ea, h->off, h->I, h->Jc, h->Ae, h->nd, rs, h->ess,
          eliminate, h->row_cap, (long long)h->ne * h->nd, h->vals);
      LF_LAUNCHED();
    }
  };
  // fork: the PML elements in one launch on P; the bulk records on A
  cudaEvent_t e0 = ev();
  LF_CUDA(cudaEventRecord(e0, A));
  LF_CUDA(cudaStreamWaitEvent(P, e0, 0));
  LF_CUDA(cudaStreamWaitEvent(G, e0, 0));
  if (h->n_pml > 0) {
    int rc = h->p == 1 ? launch_pml<8>(h, cross, 1, LFASM_CURLCURL, mm, 1, eliminate, rs, P)
           : h->p == 2 ? launch_pml<24>(h, cross, 1, LFASM_CURLCURL, mm, 1, eliminate, rs, P)
                       : launch_pml<48>(h, cross, 1, LFASM_CURLCURL, mm, 1, eliminate, rs, P);
    if (rc) return rc;
  }
  if (int rc = launch_bulk(h, mask, 1, 1, eliminate, rs, 0, h->n_bulk, true, false, A)) return rc;
  // bulk chunks, each followed by the gather of the rows it completes
  for (int c = 0; c < h->nchunk; ++c) {
    const int b0 = h->chunk_b[c], nb = h->chunk_b[c + 1] - b0;
    if (int rc = launch_bulk(h, mask, 1, 1, eliminate, rs, b0, nb, false, true, A)) return rc;
    cudaEvent_t ea = ev();
    LF_CUDA(cudaEventRecord(ea, A));
    LF_CUDA(cudaStreamWaitEvent(G, ea, 0));
    gather_group(c);
  }
  // the rows that touch PML elements, once those are done
  cudaEvent_t ep = ev();
  LF_CUDA(cudaEventRecord(ep, P));
  LF_CUDA(cudaStreamWaitEvent(G, ep, 0));
  gather_group(h->nchunk);
  cudaEvent_t eg = ev();
  LF_CUDA(cudaEventRecord(eg, G));
  LF_CUDA(cudaStreamWaitEvent(A, eg, 0));
  if (h->n_long) {
    const unsigned nl = (unsigned)((h->n_long + wpb - 1) / wpb);
    k_gather<false, true><<<nl, wpb * 32, 0, A>>>(h->n_long, h->long_rows, h->ea_ptr, h->ea,
                                                  h->off, h->I, h->Jc, h->Ae, h->nd, rs, h->ess,
                                                  h->sign, h->dof, eliminate, h->row_cap,
                                                  (long long)h->ne * h->nd, h->vals);
    LF_LAUNCHED();
  }
  return LFASM_OK;
}

// lfasm_assemble through the chunks: the sequence captured once per
// eliminate flag (and per chosen variants), then one graph launch a call
int assemble_chunked(lfasm_handle *h, int eliminate) {
  const int slot = eliminate ? 1 : 0;
  if (h->cexec[slot] &&
      (h->cvar_bulk[slot] != h->bulk_variant || h->cvar_pml[slot] != h->pml_variant)) {
    cudaGraphExecDestroy(h->cexec[slot]);
    h->cexec[slot] = nullptr;
  }
  if (!h->cexec[slot]) {
    std::vector<cudaEvent_t> evs(3 * (size_t)h->nchunk + 8, nullptr);
    for (auto &e : evs) LF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    const long long l0 = g_launches.load();
    LF_CUDA(cudaStreamBeginCapture(h->cstream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_chunked(h, eliminate, evs);
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(h->cstream, &graph);
    h->ckernels[slot] = g_launches.load() - l0;
    g_launches -= h->ckernels[slot];  // counted when the graph runs
    if (rc || ee != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      for (auto &e : evs) cudaEventDestroy(e);
      if (rc) return rc;
      LF_CUDA(ee);
    }
    const cudaError_t ie = cudaGraphInstantiate(&h->cexec[slot], graph, 0);
    cudaGraphDestroy(graph);
    for (auto &e : evs) cudaEventDestroy(e);
    LF_CUDA(ie);
    h->cvar_bulk[slot] = h->bulk_variant;
    h->cvar_pml[slot] = h->pml_variant;
  }
  LF_CUDA(cudaGraphLaunch(h->cexec[slot], h->stream));
  g_launches += h->ckernels[slot];
  return LFASM_OK;
}

}  // namespace

extern "C" {

int lfasm_assemble(lfasm_handle *h, int eliminate) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  g_err.clear();
  if (!h->built) return fail(LFASM_ERR_STATE, "lfasm_build_global has not run");
  if (int rt = ensure_tuned(h)) return rt;
  if (h->nchunk > 1 && !h->profile) {
    // chunked, element rows kept in L2 (the stage profile uses one pass)
    LF_CUDA(cudaSetDevice(h->dev));
    int rc = assemble_chunked(h, eliminate ? 1 : 0);
    if (rc) return rc;
    h->locals_valid = 0;
    return sync_if(h);
  }
  const int mm = LFASM_MASS | (h->has_kpar ? (LFASM_CROSS0 | LFASM_CROSS1 | LFASM_KLK) : 0);
  int rc = launch_local(h, LFASM_CURLCURL, mm, 1, 1, eliminate ? 1 : 0);
  if (rc) return rc;
  h->locals_valid = 0;  // the element buffer now holds signed entries
  rc = gather(h, false, eliminate ? 1 : 0);
  if (rc) return rc;
  if (h->profile) LF_CUDA(cudaEventRecord(h->ev[3], h->stream));
  return sync_if(h);
}

}  // extern "C"

// Batched assembly: several handles (meshes) of one device assembled by one
// CUDA-graph launch.  The graph holds, per handle, the element kernels and
// the gather of lfasm_assemble on a branch stream of its own (the PML side
// stream of the handle joins that branch), all branches forked from and
// joined into one capture stream, so small meshes run concurrently.
struct lfasm_batch {
  int dev = 0;
  std::vector<lfasm_handle *> hs;
  cudaStream_t cs = nullptr;         // capture / launch stream
  cudaStream_t user = nullptr;       // lfasm_batch_set_stream
  std::vector<cudaStream_t> bs;      // per-handle branch streams
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};  // per eliminate flag
  long long kernels[2] = {0, 0};                 // kernel nodes per graph
};

namespace {

void batch_free(lfasm_batch *b) {
  for (int i = 0; i < 2; ++i)
    if (b->exec[i]) cudaGraphExecDestroy(b->exec[i]);
  for (cudaEvent_t e : b->joins)
    if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  for (cudaStream_t st : b->bs)
    if (st) cudaStreamDestroy(st);
  if (b->cs) cudaStreamDestroy(b->cs);
  delete b;
}

// capture every handle's fused assembly into one graph
int batch_capture(lfasm_batch *b, int eliminate) {
  const int slot = eliminate ? 1 : 0;
  for (lfasm_handle *h : b->hs)
    if (int rt = ensure_tuned(h)) return rt;
  LF_CUDA(cudaStreamBeginCapture(b->cs, cudaStreamCaptureModeThreadLocal));
  int rc = LFASM_OK;
  cudaError_t ce = cudaEventRecord(b->fork, b->cs);
  std::vector<cudaStream_t> keep(b->hs.size());
  std::vector<int> keep_prof(b->hs.size());
  for (size_t i = 0; i < b->hs.size() && rc == LFASM_OK && ce == cudaSuccess; ++i) {
    lfasm_handle *h = b->hs[i];
    keep[i] = h->stream;
    keep_prof[i] = h->profile;
    h->stream = b->bs[i];
    h->profile = 0;
    ce = cudaStreamWaitEvent(b->bs[i], b->fork, 0);
    if (ce == cudaSuccess) {
      const int mm = LFASM_MASS | (h->has_kpar ? (LFASM_CROSS0 | LFASM_CROSS1 | LFASM_KLK) : 0);
      rc = launch_local(h, LFASM_CURLCURL, mm, 1, 1, eliminate);
      h->locals_valid = 0;
      if (rc == LFASM_OK) rc = gather(h, false, eliminate);
      if (rc == LFASM_OK) ce = cudaEventRecord(b->joins[i], b->bs[i]);
      if (rc == LFASM_OK && ce == cudaSuccess) ce = cudaStreamWaitEvent(b->cs, b->joins[i], 0);
    }
    h->stream = keep[i];
    h->profile = keep_prof[i];
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(b->cs, &graph);
  if (rc != LFASM_OK || ce != cudaSuccess || ee != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    if (rc != LFASM_OK) return rc;
    LF_CUDA(ce != cudaSuccess ? ce : ee);
  }
  size_t nn = 0;
  LF_CUDA(cudaGraphGetNodes(graph, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  LF_CUDA(cudaGraphGetNodes(graph, nodes.data(), &nn));
  long long nk = 0;
  for (cudaGraphNode_t nd_ : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd_, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++nk;
  }
  const cudaError_t ie = cudaGraphInstantiate(&b->exec[slot], graph, 0);
  cudaGraphDestroy(graph);
  LF_CUDA(ie);
  b->kernels[slot] = nk;
  return LFASM_OK;
}

}  // namespace

extern "C" {

int lfasm_batch_create(lfasm_handle *const *handles, int n, lfasm_batch **out) {
  g_err.clear();
  if (!out) return fail(LFASM_ERR_ARG, "out batch pointer is NULL");
  *out = nullptr;
  if (n <= 0 || !handles) return fail(LFASM_ERR_ARG, "empty batch");
  for (int i = 0; i < n; ++i) {
    if (!handles[i]) return fail(LFASM_ERR_ARG, "handle %d is NULL", i);
    if (handles[i]->dev != handles[0]->dev)
      return fail(LFASM_ERR_ARG, "handle %d is on device %d, handle 0 on %d", i, handles[i]->dev,
                  handles[0]->dev);
    if (!handles[i]->built)
      return fail(LFASM_ERR_STATE, "handle %d: lfasm_build_global has not run", i);
    for (int j = 0; j < i; ++j)
      if (handles[j] == handles[i]) return fail(LFASM_ERR_ARG, "handle %d repeats handle %d", i, j);
  }
  LF_CUDA(cudaSetDevice(handles[0]->dev));
  lfasm_batch *b = new lfasm_batch();
  b->dev = handles[0]->dev;
  b->hs.assign(handles, handles + n);
  b->bs.assign(n, nullptr);
  b->joins.assign(n, nullptr);
  cudaError_t e = cudaStreamCreateWithFlags(&b->cs, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    e = cudaStreamCreateWithFlags(&b->bs[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->joins[i], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    batch_free(b);
    LF_CUDA(e);
  }
  *out = b;
  return LFASM_OK;
}

int lfasm_batch_set_stream(lfasm_batch *b, void *stream) {
  if (!b) return fail(LFASM_ERR_ARG, "NULL batch");
  b->user = (cudaStream_t)stream;
  return LFASM_OK;
}

int lfasm_batch_assemble(lfasm_batch *b, int eliminate) {
  if (!b) return fail(LFASM_ERR_ARG, "NULL batch");
  g_err.clear();
  LF_CUDA(cudaSetDevice(b->dev));
  const int slot = eliminate ? 1 : 0;
  if (!b->exec[slot]) {
    int rc = batch_capture(b, eliminate);
    if (rc) return rc;
  }
  cudaStream_t st = b->user ? b->user : b->cs;
  LF_CUDA(cudaGraphLaunch(b->exec[slot], st));
  g_launches.fetch_add(b->kernels[slot], std::memory_order_relaxed);
  LF_CUDA(cudaStreamSynchronize(st));
  if (int rb = bounds_status()) return rb;
  for (size_t i = 0; i < b->hs.size(); ++i) {
    lfasm_handle *h = b->hs[i];
    if (h->pml_variant != 1 && h->bulk_variant != 5) continue;
    int e = 0;
    LF_CUDA(cudaMemcpy(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
      LF_CUDA(cudaMemset(h->err, 0, sizeof(int)));
      return fail(LFASM_ERR_CUDA, "handle %zu: a bounded wait ran out", i);
    }
  }
  return LFASM_OK;
}

void lfasm_batch_destroy(lfasm_batch *b) {
  if (!b) return;
  cudaSetDevice(b->dev);
  if (b->cs) cudaStreamSynchronize(b->cs);
  if (b->user) cudaStreamSynchronize(b->user);
  batch_free(b);
}

int lfasm_set_basis(lfasm_handle *h, int nmono, const int *exps, const double *coef,
                    const double *curl_coef) {
  if (!h || !exps || !coef || !curl_coef) return fail(LFASM_ERR_ARG, "NULL argument");
  if (nmono <= 0 || nmono > BASIS_MAX_MONO)
    return fail(LFASM_ERR_UNSUPPORTED, "%d monomials (at most %d)", nmono, BASIS_MAX_MONO);
  for (int m = 0; m < nmono; ++m) {
    const int a = exps[3 * m], b = exps[3 * m + 1], c = exps[3 * m + 2];
    if (a < 0 || b < 0 || c < 0 || a + b + c > h->p)
      return fail(LFASM_ERR_ARG, "monomial %d has exponents (%d,%d,%d) beyond degree %d", m, a, b,
                  c, h->p);
  }
  LF_CUDA(cudaSetDevice(h->dev));
  dfree(h->bexps); dfree(h->bcoef); dfree(h->bccoef);
  const size_t nc = (size_t)h->nd * 3 * nmono;
  LF_CUDA(upload(h->bexps, exps, (size_t)nmono * 3));
  LF_CUDA(upload(h->bcoef, coef, nc));
  LF_CUDA(upload(h->bccoef, curl_coef, nc));
  h->nmono = nmono;
  return LFASM_OK;
}

}  // extern "C"

namespace {

// locate the nx x ny sample points of the plane z: element and reference
// coordinates per point (device arrays owned by the caller afterwards)
// Device buffers of one call, freed when it returns (on every path).
struct DevBufs {
  std::vector<void *> v;
  ~DevBufs() {
    for (void *q : v) dfree_bytes(q);
  }
  template <typename T>
  cudaError_t get(T *&d, size_t n) {
    cudaError_t e = dmalloc(d, n);
    if (e == cudaSuccess) v.push_back((void *)d);
    return e;
  }
};

// Sample points of nz planes (heights zs, host) located in the mesh: per
// plane the elements whose z-range holds it (flags [iz][e], one scan, one
// compaction), then a warp per point over its plane's candidates; *elem
// and *xi (device, nz * nx * ny points) are the caller's to free.
int plane_locate(lfasm_handle *h, const PlaneGrid &G, int nz, const double *zs, int **elem,
                 double **xi) {
  const int ne = h->ne, npts = G.nx * G.ny;
  const long long nf = (long long)ne * nz, ntot = (long long)npts * nz;
  int *flag = nullptr, *pos = nullptr, *cand = nullptr, *miss = nullptr;
  double *dz = nullptr;
  unsigned char *tmp = nullptr;
  size_t tb = 0;
  LF_CUDA(dmalloc(flag, (size_t)nf + 1));
  LF_CUDA(dmalloc(pos, (size_t)nf + 1));
  LF_CUDA(dmalloc(cand, (size_t)nf));
  LF_CUDA(dmalloc(miss, 1));
  LF_CUDA(dmalloc(dz, (size_t)nz));
  LF_CUDA(dmalloc(*elem, (size_t)ntot));
  LF_CUDA(dmalloc(*xi, (size_t)ntot * 3));
  LF_CUDA(cudaMemcpyAsync(dz, zs, sizeof(double) * nz, cudaMemcpyHostToDevice, h->stream));
  LF_CUDA(cudaMemsetAsync(flag + nf, 0, sizeof(int), h->stream));
  LF_CUDA(cudaMemsetAsync(miss, 0, sizeof(int), h->stream));
  const unsigned gb = (unsigned)((nf + 255) / 256);
  k_plane_cand<<<gb, 256, 0, h->stream>>>(ne, nz, h->J, h->v0, dz, flag);
  LF_LAUNCHED();
  LF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag, pos, (int)(nf + 1), h->stream));
  LF_CUDA(dmalloc(tmp, tb));
  LF_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, flag, pos, (int)(nf + 1), h->stream));
  k_compact<<<gb, 256, 0, h->stream>>>((int)nf, flag, pos, cand);
  LF_LAUNCHED();
  const int wpb = 8;
  k_plane_locate<<<(unsigned)((ntot + wpb - 1) / wpb), wpb * 32, 0, h->stream>>>(
      G, nz, dz, ne, pos, cand, h->Jinv, h->v0, *elem, *xi, miss);
  LF_LAUNCHED();
  int nmiss = 0;
  LF_CUDA(cudaMemcpyAsync(&nmiss, miss, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  LF_CUDA(cudaStreamSynchronize(h->stream));
  dfree(flag); dfree(pos); dfree(cand); dfree(miss); dfree(tmp); dfree(dz);
  if (nmiss) {
    dfree(*elem); dfree(*xi);
    if (nz == 1)
      return fail(LFASM_ERR_ARG, "%d of %d sample points of the plane z = %g lie outside the mesh",
                  nmiss, npts, zs[0]);
    return fail(LFASM_ERR_ARG, "%d of %lld sample points of the %d planes lie outside the mesh",
                nmiss, ntot, nz);
  }
  return LFASM_OK;
}

int plane_args(lfasm_handle *h, double lx, double ly, double z, int nx, int ny, PlaneGrid &G) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  if (!h->nmono) return fail(LFASM_ERR_STATE, "lfasm_set_basis has not run");
  if (nx <= 0 || ny <= 0 || (long long)nx * ny > (1ll << 24) || !(lx > 0) || !(ly > 0))
    return fail(LFASM_ERR_ARG, "bad sampling grid %d x %d over %g x %g", nx, ny, lx, ly);
  G.lx = lx; G.ly = ly; G.z = z; G.nx = nx; G.ny = ny;
  return LFASM_OK;
}

}  // namespace

extern "C" {

int lfasm_sample_plane(lfasm_handle *h, double lx, double ly, double z, int nx, int ny,
                       const void *d_u, void *d_e, void *d_curl) {
  PlaneGrid G;
  int rc = plane_args(h, lx, ly, z, nx, ny, G);
  if (rc) return rc;
  if (!d_u || (!d_e && !d_curl)) return fail(LFASM_ERR_ARG, "NULL vector");
  g_err.clear();
  LF_CUDA(cudaSetDevice(h->dev));
  int *elem = nullptr;
  double *xi = nullptr;
  if ((rc = plane_locate(h, G, 1, &z, &elem, &xi))) return rc;
  const int npts = nx * ny, wpb = 8;
  k_plane_eval<<<(unsigned)((npts + wpb - 1) / wpb), wpb * 32, 0, h->stream>>>(
      npts, elem, xi, h->nd, h->p, h->nmono, h->bexps, h->bcoef, h->bccoef, h->dof, h->sign,
      h->fopack, h->J, h->Jinv, h->detJ, (const dcplx *)d_u, (dcplx *)d_e, (dcplx *)d_curl);
  LF_LAUNCHED();
  LF_CUDA(cudaStreamSynchronize(h->stream));
  dfree(elem); dfree(xi);
  return sync_if(h);
}

int lfasm_plane_seed(lfasm_handle *h, double lx, double ly, double z, int nx, int ny, int comp,
                     int m, int q, void *d_c) {
  PlaneGrid G;
  int rc = plane_args(h, lx, ly, z, nx, ny, G);
  if (rc) return rc;
  if (!d_c) return fail(LFASM_ERR_ARG, "NULL vector");
  if (comp < 0 || comp > 2) return fail(LFASM_ERR_ARG, "component %d outside 0..2", comp);
  g_err.clear();
  LF_CUDA(cudaSetDevice(h->dev));
  int *elem = nullptr;
  double *xi = nullptr;
  if ((rc = plane_locate(h, G, 1, &z, &elem, &xi))) return rc;
  const int npts = nx * ny, wpb = 8;
  LF_CUDA(cudaMemsetAsync(d_c, 0, (size_t)h->n * sizeof(dcplx), h->stream));
  k_plane_seed<<<(unsigned)((npts + wpb - 1) / wpb), wpb * 32, 0, h->stream>>>(
      G, elem, xi, h->nd, h->p, h->nmono, h->bexps, h->bcoef, h->bccoef, h->dof, h->sign,
      h->fopack, h->J, h->Jinv, h->detJ, comp, m, q, (double *)d_c);
  LF_LAUNCHED();
  LF_CUDA(cudaStreamSynchronize(h->stream));
  dfree(elem); dfree(xi);
  return sync_if(h);
}

int lfasm_sample_planes(lfasm_handle *h, double lx, double ly, int nz, const double *z, int nx,
                        int ny, const void *d_u, void *d_e, void *d_curl) {
  PlaneGrid G;
  int rc = plane_args(h, lx, ly, 0.0, nx, ny, G);
  if (rc) return rc;
  if (nz <= 0 || nz > LFASM_MAX_PLANES || !z)
    return fail(LFASM_ERR_ARG, "bad plane list (%d planes, at most %d)", nz, LFASM_MAX_PLANES);
  if ((long long)nx * ny * nz > (1ll << 24))
    return fail(LFASM_ERR_ARG, "%d planes of %d x %d points exceed 2^24 points", nz, nx, ny);
  if (!d_u || (!d_e && !d_curl)) return fail(LFASM_ERR_ARG, "NULL vector");
  g_err.clear();
  LF_CUDA(cudaSetDevice(h->dev));
  int *elem = nullptr;
  double *xi = nullptr;
  if ((rc = plane_locate(h, G, nz, z, &elem, &xi))) return rc;
  const long long npts = (long long)nx * ny * nz;
  const int wpb = 8;
  k_plane_eval<<<(unsigned)((npts + wpb - 1) / wpb), wpb * 32, 0, h->stream>>>(
      (int)npts, elem, xi, h->nd, h->p, h->nmono, h->bexps, h->bcoef, h->bccoef, h->dof, h->sign,
      h->fopack, h->J, h->Jinv, h->detJ, (const dcplx *)d_u, (dcplx *)d_e, (dcplx *)d_curl);
  LF_LAUNCHED();
  LF_CUDA(cudaStreamSynchronize(h->stream));
  dfree(elem); dfree(xi);
  return sync_if(h);
}

int lfasm_plane_orders(lfasm_handle *h, int nz, int nx, int ny, const void *d_e,
                       const lfasm_order_plane *planes, const lfasm_order_args *args,
                       void *d_coef, double *d_eff) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  if (nz <= 0 || nz > LFASM_MAX_PLANES || !planes || !args)
    return fail(LFASM_ERR_ARG, "bad plane list (%d planes, at most %d)", nz, LFASM_MAX_PLANES);
  if (nx <= 0 || ny <= 0 || (long long)nx * ny * nz > (1ll << 24))
    return fail(LFASM_ERR_ARG, "bad sampling grid %d x %d x %d planes", nx, ny, nz);
  if (!d_e || !d_coef || !d_eff) return fail(LFASM_ERR_ARG, "NULL vector");
  const lfasm_order_args &a = *args;
  if (!(a.lx > 0) || !(a.ly > 0) || !(a.k0 > 0) || !(a.inc_flux > 0))
    return fail(LFASM_ERR_ARG, "bad cell %g x %g, k0 %g or incident flux %g", a.lx, a.ly, a.k0,
                a.inc_flux);
  for (int i = 0; i < nz; ++i)
    if (planes[i].direction != 1 && planes[i].direction != -1)
      return fail(LFASM_ERR_ARG, "plane %d: direction %d is not +1 or -1", i,
                  planes[i].direction);
  g_err.clear();
  LF_CUDA(cudaSetDevice(h->dev));
  // per-plane scalars packed into one upload: z, z_ref, eps (2), background (6)
  std::vector<double> hp((size_t)nz * 10);
  std::vector<int> hd(nz);
  bool any_bg = false;
  for (int i = 0; i < nz; ++i) {
    const lfasm_order_plane &q = planes[i];
    double *r = hp.data() + (size_t)i * 10;
    r[0] = q.z; r[1] = q.z_ref; r[2] = q.eps_re; r[3] = q.eps_im;
    for (int c = 0; c < 6; ++c) r[4 + c] = q.bg00[c];
    any_bg = any_bg || q.has_bg00;
    if (!q.has_bg00)
      for (int c = 0; c < 6; ++c) r[4 + c] = 0.0;
    hd[i] = q.direction;
  }
  double *dp = nullptr;
  int *dd = nullptr;
  LF_CUDA(dmalloc(dp, hp.size()));
  LF_CUDA(dmalloc(dd, hd.size()));
  LF_CUDA(cudaMemcpyAsync(dp, hp.data(), sizeof(double) * hp.size(), cudaMemcpyHostToDevice,
                          h->stream));
  LF_CUDA(cudaMemcpyAsync(dd, hd.data(), sizeof(int) * hd.size(), cudaMemcpyHostToDevice,
                          h->stream));
  // split the packed rows into the kernel's arrays: z, z_ref, eps, background
  double *zs = nullptr;
  LF_CUDA(dmalloc(zs, (size_t)nz * 10));
  k_unpack_planes<<<(nz + 127) / 128, 128, 0, h->stream>>>(nz, dp, zs, zs + nz, zs + 2 * nz,
                                                            zs + 4 * nz);
  LF_LAUNCHED();
  OrderArgs A{a.lx, a.ly, a.k0, a.kx, a.ky, a.inc_flux};
  k_plane_orders<<<dim3((unsigned)(nx * ny), (unsigned)nz), ORDER_THREADS, 0, h->stream>>>(
      nx, ny, (const dcplx *)d_e, zs, zs + nz, dd, zs + 2 * nz, any_bg ? zs + 4 * nz : nullptr,
      A, (dcplx *)d_coef, d_eff);
  LF_LAUNCHED();
  LF_CUDA(cudaStreamSynchronize(h->stream));
  dfree(dp); dfree(dd); dfree(zs);
  return sync_if(h);
}

int lfasm_extract(int gpu_id, int ne, int nv, int p, const int *tv, const double *xv, int *dof,
                  double *sign, int *fo, double *J, double *Jinv, double *detJ, double *v0,
                  int *ess, long long ess_cap, int *height, int *n_ess) {
  if (ne <= 0 || nv <= 0) return fail(LFASM_ERR_ARG, "empty mesh (%d elements, %d vertices)", ne, nv);
  if (p < 1 || p > 3) return fail(LFASM_ERR_UNSUPPORTED, "order p = %d outside 1..3", p);
  if (nv >= (1 << 21)) return fail(LFASM_ERR_ARG, "%d vertices: face keys hold 21 bits", nv);
  if ((long long)ne * 6 >= INT_MAX / 2) return fail(LFASM_ERR_ARG, "%d elements: too many", ne);
  if (!tv || !xv || !dof || !sign || (p >= 2 && !fo) || !J || !Jinv || !detJ || !v0 || !height ||
      !n_ess || (ess_cap > 0 && !ess))
    return fail(LFASM_ERR_ARG, "NULL argument");
  for (long long i = 0; i < 4LL * ne; ++i)
    if (tv[i] < 0 || tv[i] >= nv)
      return fail(LFASM_ERR_ARG, "element %lld vertex %lld: id %d outside 0..%d", i / 4, i % 4,
                  tv[i], nv - 1);
  g_err.clear();
  LF_CUDA(cudaSetDevice(gpu_id));
  const int nd = p * (p + 2) * (p + 3) / 2;
  DevBufs B;  // every device buffer of the call, freed on every return
  cudaStream_t st = 0;
  int *d_tvin, *d_tv, *d_err;
  double *d_xv, *d_J, *d_Ji, *d_det, *d_v0;
  LF_CUDA(B.get(d_tvin, (size_t)ne * 4));
  LF_CUDA(B.get(d_tv, (size_t)ne * 4));
  LF_CUDA(B.get(d_err, 2));
  LF_CUDA(B.get(d_xv, (size_t)ne * 12));
  LF_CUDA(B.get(d_J, (size_t)ne * 9));
  LF_CUDA(B.get(d_Ji, (size_t)ne * 9));
  LF_CUDA(B.get(d_det, (size_t)ne));
  LF_CUDA(B.get(d_v0, (size_t)ne * 3));
  LF_CUDA(cudaMemcpyAsync(d_tvin, tv, sizeof(int) * 4 * ne, cudaMemcpyHostToDevice, st));
  LF_CUDA(cudaMemcpyAsync(d_xv, xv, sizeof(double) * 12 * ne, cudaMemcpyHostToDevice, st));
  LF_CUDA(cudaMemsetAsync(d_err, 0, 2 * sizeof(int), st));
  lfasm_ex::k_ex_local<<<(ne + 127) / 128, 128, 0, st>>>(ne, d_tvin, d_xv, d_tv, d_J, d_Ji, d_det,
                                                          d_v0, d_err, d_err + 1);
  LF_LAUNCHED();
  int herr[2] = {0, 0};
  LF_CUDA(cudaMemcpyAsync(herr, d_err, sizeof(herr), cudaMemcpyDeviceToHost, st));
  LF_CUDA(cudaStreamSynchronize(st));
  if (herr[0] == lfasm_ex::EX_ERR_REPEATED)
    return fail(LFASM_ERR_ARG, "element %d repeats a vertex", herr[1]);
  if (herr[0]) return fail(LFASM_ERR_ARG, "element %d is degenerate (detJ <= 0)", herr[1]);

  // ids by first occurrence of the key in row order (edges, then faces)
  auto number = [&](long long n, unsigned long long *key, int *row, int *id, int **first_of,
                    int **count_of, int *nuniq) -> int {
    unsigned long long *ks;
    int *rs, *head, *run, *rfirst, *rlen, *ridx, *sfirst, *srun, *rank;
    LF_CUDA(B.get(ks, (size_t)n));
    LF_CUDA(B.get(rs, (size_t)n));
    LF_CUDA(B.get(head, (size_t)n));
    LF_CUDA(B.get(run, (size_t)n));
    size_t tb = 0, tb2 = 0;
    LF_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key, ks, row, rs, (int)n, 0, 64, st));
    LF_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb2, head, run, (int)n, st));
    unsigned char *tmp;
    LF_CUDA(B.get(tmp, std::max(tb, tb2)));
    tb = std::max(tb, tb2);
    LF_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, key, ks, row, rs, (int)n, 0, 64, st));
    const unsigned g = (unsigned)((n + 255) / 256);
    lfasm_ex::k_ex_heads<<<g, 256, 0, st>>>(n, ks, head);
    LF_LAUNCHED();
    LF_CUDA(cub::DeviceScan::InclusiveSum(tmp, tb, head, run, (int)n, st));
    int nrun = 0;
    LF_CUDA(cudaMemcpyAsync(&nrun, run + n - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    LF_CUDA(cudaStreamSynchronize(st));
    LF_CUDA(B.get(rfirst, (size_t)nrun));
    LF_CUDA(B.get(rlen, (size_t)nrun));
    LF_CUDA(B.get(ridx, (size_t)nrun));
    LF_CUDA(B.get(sfirst, (size_t)nrun));
    LF_CUDA(B.get(srun, (size_t)nrun));
    LF_CUDA(B.get(rank, (size_t)nrun));
    LF_CUDA(B.get(*first_of, (size_t)nrun));
    LF_CUDA(B.get(*count_of, (size_t)nrun));
    LF_CUDA(cudaMemsetAsync(rlen, 0, sizeof(int) * nrun, st));
    lfasm_ex::k_ex_runs<<<g, 256, 0, st>>>(n, head, run, rs, rfirst, rlen, ridx);
    LF_LAUNCHED();
    size_t tb3 = 0;
    LF_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb3, rfirst, sfirst, ridx, srun, nrun, 0, 32,
                                            st));
    unsigned char *tmp3;
    LF_CUDA(B.get(tmp3, tb3));
    LF_CUDA(cub::DeviceRadixSort::SortPairs(tmp3, tb3, rfirst, sfirst, ridx, srun, nrun, 0, 32,
                                            st));
    lfasm_ex::k_ex_rank<<<(nrun + 255) / 256, 256, 0, st>>>(nrun, srun, rank);
    LF_LAUNCHED();
    lfasm_ex::k_ex_ids<<<g, 256, 0, st>>>(n, run, rs, rank, rfirst, rlen, id, *first_of,
                                          *count_of);
    LF_LAUNCHED();
    *nuniq = nrun;
    return LFASM_OK;
  };
  const long long n6 = 6LL * ne, n4 = 4LL * ne;
  unsigned long long *ekey, *fkey;
  int *erow, *eid, *frow, *fid, *efirst, *ecount, *ffirst, *fcount, *d_fo, *d_dof, *flag, *pos;
  signed char *esgn;
  double *d_sign;
  LF_CUDA(B.get(ekey, (size_t)n6));
  LF_CUDA(B.get(erow, (size_t)n6));
  LF_CUDA(B.get(eid, (size_t)n6));
  LF_CUDA(B.get(esgn, (size_t)n6));
  lfasm_ex::k_ex_edge_keys<<<(unsigned)((n6 + 255) / 256), 256, 0, st>>>(ne, d_tv, ekey, erow, esgn);
  LF_LAUNCHED();
  int nE = 0, nF = 0, rc;
  if ((rc = number(n6, ekey, erow, eid, &efirst, &ecount, &nE))) return rc;
  LF_CUDA(B.get(fkey, (size_t)n4));
  LF_CUDA(B.get(frow, (size_t)n4));
  LF_CUDA(B.get(fid, (size_t)n4));
  LF_CUDA(B.get(d_fo, (size_t)n4));
  lfasm_ex::k_ex_face_keys<<<(unsigned)((n4 + 255) / 256), 256, 0, st>>>(ne, d_tv, fkey, frow);
  LF_LAUNCHED();
  if ((rc = number(n4, fkey, frow, fid, &ffirst, &fcount, &nF))) return rc;
  lfasm_ex::k_ex_face_orient<<<(unsigned)((n4 + 255) / 256), 256, 0, st>>>(ne, d_tv, fid, ffirst,
                                                                          d_fo, d_err, d_err + 1);
  LF_LAUNCHED();
  const long long ndof_f = (long long)p * (p - 1), nint = nd - 6 * p - 4 * ndof_f;
  const long long hgt = (long long)nE * p + nF * ndof_f + (long long)ne * nint;
  if (hgt >= INT_MAX) return fail(LFASM_ERR_ARG, "%lld DOFs exceed 32-bit indices", hgt);
  LF_CUDA(B.get(d_dof, (size_t)ne * nd));
  LF_CUDA(B.get(d_sign, (size_t)ne * nd));
  lfasm_ex::k_ex_dofs<<<(ne + 127) / 128, 128, 0, st>>>(ne, p, nd, nE * p, (int)(nF * ndof_f), eid,
                                                         esgn, fid, d_fo, d_dof, d_sign);
  LF_LAUNCHED();
  LF_CUDA(B.get(flag, (size_t)hgt + 1));
  LF_CUDA(B.get(pos, (size_t)hgt + 1));
  LF_CUDA(cudaMemsetAsync(flag, 0, sizeof(int) * (hgt + 1), st));
  lfasm_ex::k_ex_ess<<<(unsigned)((n4 + 255) / 256), 256, 0, st>>>(ne, p, nd, fid, fcount, d_dof,
                                                                     flag);
  LF_LAUNCHED();
  size_t tb = 0;
  LF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag, pos, (int)(hgt + 1), st));
  unsigned char *tmp;
  LF_CUDA(B.get(tmp, tb));
  LF_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, flag, pos, (int)(hgt + 1), st));
  int ness = 0;
  LF_CUDA(cudaMemcpyAsync(&ness, pos + hgt, sizeof(int), cudaMemcpyDeviceToHost, st));
  LF_CUDA(cudaMemcpyAsync(herr, d_err, sizeof(herr), cudaMemcpyDeviceToHost, st));
  LF_CUDA(cudaStreamSynchronize(st));
  if (herr[0]) return fail(LFASM_ERR_ARG, "element %d: inconsistent face vertices", herr[1]);
  *height = (int)hgt;
  *n_ess = ness;
  if (ness > ess_cap)
    return fail(LFASM_ERR_ARG, "%d essential DOFs exceed the buffer of %lld", ness, ess_cap);
  int *d_ess;
  LF_CUDA(B.get(d_ess, (size_t)std::max(ness, 1)));
  lfasm_ex::k_ex_compact<<<(unsigned)((hgt + 255) / 256), 256, 0, st>>>((int)hgt, flag, pos, d_ess);
  LF_LAUNCHED();
  LF_CUDA(cudaMemcpyAsync(dof, d_dof, sizeof(int) * ne * nd, cudaMemcpyDeviceToHost, st));
  LF_CUDA(cudaMemcpyAsync(sign, d_sign, sizeof(double) * ne * nd, cudaMemcpyDeviceToHost, st));
  if (p >= 2)
    LF_CUDA(cudaMemcpyAsync(fo, d_fo, sizeof(int) * 4 * ne, cudaMemcpyDeviceToHost, st));
  LF_CUDA(cudaMemcpyAsync(J, d_J, sizeof(double) * 9 * ne, cudaMemcpyDeviceToHost, st));
  LF_CUDA(cudaMemcpyAsync(Jinv, d_Ji, sizeof(double) * 9 * ne, cudaMemcpyDeviceToHost, st));
  LF_CUDA(cudaMemcpyAsync(detJ, d_det, sizeof(double) * ne, cudaMemcpyDeviceToHost, st));
  LF_CUDA(cudaMemcpyAsync(v0, d_v0, sizeof(double) * 3 * ne, cudaMemcpyDeviceToHost, st));
  if (ness) LF_CUDA(cudaMemcpyAsync(ess, d_ess, sizeof(int) * ness, cudaMemcpyDeviceToHost, st));
  LF_CUDA(cudaStreamSynchronize(st));
  return LFASM_OK;
}

int lfasm_set_profile(lfasm_handle *h, int on) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  LF_CUDA(cudaSetDevice(h->dev));
  if (on && !h->ev[0])
    for (int i = 0; i < 4; ++i) LF_CUDA(cudaEventCreate(&h->ev[i]));
  h->profile = on ? 1 : 0;
  return LFASM_OK;
}

int lfasm_stage_times(lfasm_handle *h, float *ms3) {
  if (!h || !ms3) return fail(LFASM_ERR_ARG, "NULL argument");
  if (!h->profile) return fail(LFASM_ERR_STATE, "profiling is off");
  LF_CUDA(cudaSetDevice(h->dev));
  LF_CUDA(cudaEventSynchronize(h->ev[3]));
  for (int i = 0; i < 3; ++i) LF_CUDA(cudaEventElapsedTime(ms3 + i, h->ev[i], h->ev[i + 1]));
  return LFASM_OK;
}

int lfasm_get_csr(lfasm_handle *h, int **d_rowptr, int **d_cols, void **d_vals, int *n,
                  long long *nnz) {
  if (!h) return fail(LFASM_ERR_ARG, "NULL handle");
  if (!h->built) return fail(LFASM_ERR_STATE, "lfasm_build_global has not run");
  if (d_rowptr) *d_rowptr = h->I;
  if (d_cols) *d_cols = h->Jc;
  if (d_vals) *d_vals = h->vals;
  if (n) *n = h->n;
  if (nnz) *nnz = h->nnz;
  return LFASM_OK;
}

int lfasm_download_csr(lfasm_handle *h, int *host_I, int *host_J) {
  if (!h || !host_I || !host_J) return fail(LFASM_ERR_ARG, "NULL argument");
  if (!h->built) return fail(LFASM_ERR_STATE, "lfasm_build_global has not run");
  LF_CUDA(cudaSetDevice(h->dev));
  LF_CUDA(cudaStreamSynchronize(h->stream));
  LF_CUDA(cudaMemcpy(host_I, h->I, (size_t)(h->n + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  LF_CUDA(cudaMemcpy(host_J, h->Jc, (size_t)h->nnz * sizeof(int), cudaMemcpyDeviceToHost));
  return LFASM_OK;
}

int lfasm_download_values(lfasm_handle *h, double *host_out) {
  if (!h || !host_out) return fail(LFASM_ERR_ARG, "NULL argument");
  if (!h->built) return fail(LFASM_ERR_STATE, "lfasm_build_global has not run");
  std::printf("asm_gpu_test_download (test-only D2H)\n");
  std::fflush(stdout);
  LF_CUDA(cudaSetDevice(h->dev));
  LF_CUDA(cudaStreamSynchronize(h->stream));
  LF_CUDA(cudaMemcpy(host_out, h->vals, (size_t)h->nnz * sizeof(dcplx), cudaMemcpyDeviceToHost));
  return LFASM_OK;
}

static int residual_core(lfasm_handle *h, const dcplx *dx, const dcplx *db, double *rel) {
  const int wpb = 8;
  const unsigned nb = (unsigned)((h->n + wpb - 1) / wpb);
  k_spmv_resid<<<nb, wpb * 32, 0, h->stream>>>(h->n, h->I, h->Jc, h->vals, dx, db, nullptr,
                                                h->partials);
  LF_LAUNCHED();
  k_sum_partials<<<1, 1024, 0, h->stream>>>((int)nb, h->partials, h->red);
  LF_LAUNCHED();
  double hr[2];
  LF_CUDA(cudaMemcpyAsync(hr, h->red, sizeof(hr), cudaMemcpyDeviceToHost, h->stream));
  LF_CUDA(cudaStreamSynchronize(h->stream));
  *rel = hr[1] > 0.0 ? std::sqrt(hr[0] / hr[1]) : 0.0;
  return LFASM_OK;
}

int lfasm_residual(lfasm_handle *h, const double *X, const double *B, double *rel) {
  if (!h || !X || !B || !rel) return fail(LFASM_ERR_ARG, "NULL argument");
  if (!h->built) return fail(LFASM_ERR_STATE, "lfasm_build_global has not run");
  LF_CUDA(cudaSetDevice(h->dev));
  double *d2 = nullptr;
  dcplx *dx = nullptr, *db = nullptr;
  const size_t n = h->n;
  LF_CUDA(dmalloc(d2, 2 * n));
  LF_CUDA(dmalloc(dx, n));
  LF_CUDA(dmalloc(db, n));
  const unsigned g = (unsigned)((n + 255) / 256);
  LF_CUDA(cudaMemcpyAsync(d2, X, 2 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  k_split_to_cplx<<<g, 256, 0, h->stream>>>((int)n, d2, dx);
  LF_LAUNCHED();
  LF_CUDA(cudaMemcpyAsync(d2, B, 2 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  k_split_to_cplx<<<g, 256, 0, h->stream>>>((int)n, d2, db);
  LF_LAUNCHED();
  int rc = residual_core(h, dx, db, rel);
  dfree(d2);
  dfree(dx);
  dfree(db);
  return rc;
}

int lfasm_residual_device(lfasm_handle *h, const void *d_x, const void *d_b, double *rel) {
  if (!h || !d_x || !d_b || !rel) return fail(LFASM_ERR_ARG, "NULL argument");
  if (!h->built) return fail(LFASM_ERR_STATE, "lfasm_build_global has not run");
  LF_CUDA(cudaSetDevice(h->dev));
  return residual_core(h, (const dcplx *)d_x, (const dcplx *)d_b, rel);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free residual.
//
// For callers that must not allocate device memory once they are running:
// a solver loop that has handed all remaining memory to its factorization,
// or a host framework whose own pool owns every device allocation and
// forbids side allocations.  The partial sums of the residual live in this
// file-scope device array instead of memory from cudaMalloc; every GPU that
// loads the library keeps it (64 KiB per 4096 blocks, 4 MiB in total) until
// the process exits.  Host code must not pass the symbol itself to a kernel
// (on the host it only names a stand-in object): its device address is
// looked up once per device with cudaGetSymbolAddress, on the first call
// made on that device.
// ---------------------------------------------------------------------------
namespace {
constexpr int NOALLOC_WPB = 8;                    // rows (warps) per block
constexpr int NOALLOC_MAX_BLOCKS = 1 << 18;       // 262144 blocks
static __device__ __align__(256) double g_noalloc_scratch[2 * NOALLOC_MAX_BLOCKS + 2];

// The array's device address per device, with the id of the CUDA context it
// was looked up in.  A device reset (cudaDeviceReset) destroys that context
// and the module with it; the next call sees a new context id and looks the
// address up again instead of handing a dead address to the kernels.
struct NoallocSlot {
  unsigned long long ctx_id = 0;
  double *ptr = nullptr;
};
std::mutex g_noalloc_mu;
NoallocSlot g_noalloc[64];

// id of the calling thread's current context (0 if none or unknown), read
// through driver entry points obtained from the runtime (no allocation, no
// link against the driver library)
unsigned long long current_ctx_id() {
  using GetCurrent = int (*)(void **);
  using GetId = int (*)(void *, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    resolved = true;
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
    cudaGetLastError();
  }
  if (!get_current || !get_id) return 0;
  void *ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

int noalloc_scratch(int dev, double **out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (dev < 0 || dev >= 64) return fail(LFASM_ERR_UNSUPPORTED, "device ordinal %d >= 64", dev);
  NoallocSlot &sl = g_noalloc[dev];
  const unsigned long long id = current_ctx_id();
  if (!sl.ptr || id == 0 || id != sl.ctx_id) {
    // set-up: with the device current, the symbol's address in this
    // context (the lookup also makes the device's context current)
    void *ptr = nullptr;
    LF_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    sl.ptr = static_cast<double *>(ptr);
    sl.ctx_id = current_ctx_id();
  }
  *out = sl.ptr;
  return LFASM_OK;
}
}  // namespace

extern "C" {

int lfasm_csr_residual_noalloc(int n, const int *d_rowptr, const int *d_cols, const void *d_vals,
                               const void *d_x, const void *d_b, double *rel, void *stream) {
  g_err.clear();
  if (!rel) return fail(LFASM_ERR_ARG, "NULL result pointer");
  if (n < 0) return fail(LFASM_ERR_ARG, "negative row count %d", n);
  const long long max_rows = (long long)NOALLOC_WPB * NOALLOC_MAX_BLOCKS;
  if (n > max_rows)
    return fail(LFASM_ERR_UNSUPPORTED,
                "n = %d rows exceeds the allocation-free residual limit of %lld rows", n, max_rows);
  if (n == 0) { *rel = 0.0; return LFASM_OK; }
  if (!d_rowptr || !d_cols || !d_vals || !d_x || !d_b) return fail(LFASM_ERR_ARG, "NULL argument");
  int dev = 0;
  LF_CUDA(cudaGetDevice(&dev));
  double *scratch = nullptr;
  int rc = noalloc_scratch(dev, &scratch);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (n + NOALLOC_WPB - 1) / NOALLOC_WPB;
  // every block writes its own partial pair and k_sum_partials overwrites
  // the two result slots: nothing carries over from an earlier call
  k_spmv_resid<<<nb, NOALLOC_WPB * 32, 0, st>>>(n, d_rowptr, d_cols, (const dcplx *)d_vals,
                                                 (const dcplx *)d_x, (const dcplx *)d_b, nullptr,
                                                 scratch);
  LF_LAUNCHED();
  k_sum_partials<<<1, 1024, 0, st>>>(nb, scratch, scratch + 2 * NOALLOC_MAX_BLOCKS);
  LF_LAUNCHED();
  double hr[2];
  LF_CUDA(cudaMemcpyAsync(hr, scratch + 2 * NOALLOC_MAX_BLOCKS, sizeof(hr),
                          cudaMemcpyDeviceToHost, st));
  LF_CUDA(cudaStreamSynchronize(st));
  *rel = hr[1] > 0.0 ? std::sqrt(hr[0] / hr[1]) : 0.0;
  return LFASM_OK;
}

int lfasm_spmv(lfasm_handle *h, const void *d_x, void *d_y) {
  if (!h || !d_x || !d_y) return fail(LFASM_ERR_ARG, "NULL argument");
  if (!h->built) return fail(LFASM_ERR_STATE, "lfasm_build_global has not run");
  LF_CUDA(cudaSetDevice(h->dev));
  const int wpb = 8;
  const unsigned nb = (unsigned)((h->n + wpb - 1) / wpb);
  k_spmv_resid<<<nb, wpb * 32, 0, h->stream>>>(h->n, h->I, h->Jc, h->vals, (const dcplx *)d_x,
                                                nullptr, (dcplx *)d_y, nullptr);
  LF_LAUNCHED();
  return sync_if(h);
}

int lfasm_assemble_rhs(lfasm_handle *h, const lfasm_incident_part *parts, int n_parts,
                       const int *col_of_part, int ncol, int eliminate, void *d_b) {
  if (!h || (n_parts > 0 && (!parts || !col_of_part)) || ncol <= 0 || !d_b)
    return fail(LFASM_ERR_ARG, "bad RHS arguments");
  if (!h->built) return fail(LFASM_ERR_STATE, "lfasm_build_global has not run");
  LF_CUDA(cudaSetDevice(h->dev));
  int n_slab = n_parts > 0 ? parts[0].n_slab : 1;
  if (n_parts > 0 && h->max_src_slab >= n_slab)
    return fail(LFASM_ERR_ARG, "incident tables have %d slabs; source elements reach slab %d",
                n_slab, h->max_src_slab);
  std::vector<SlabWaveD> waves((size_t)std::max(n_parts, 1) * n_slab);
  for (int pi = 0; pi < n_parts; ++pi) {
    const lfasm_incident_part &P = parts[pi];
    if (P.n_slab != n_slab) return fail(LFASM_ERR_ARG, "parts disagree on the slab count");
    if (col_of_part[pi] < 0 || col_of_part[pi] >= ncol)
      return fail(LFASM_ERR_ARG, "part %d mapped to column %d of %d", pi, col_of_part[pi], ncol);
    for (int s = 0; s < n_slab; ++s) {
      SlabWaveD &w = waves[(size_t)pi * n_slab + s];
      w.qA = dcplx{P.qA[2 * s], P.qA[2 * s + 1]};
      w.qB = dcplx{P.qB[2 * s], P.qB[2 * s + 1]};
      w.zA = P.zA[s];
      w.zB = P.zB[s];
      for (int d = 0; d < 3; ++d) {
        w.A[d] = dcplx{P.A[6 * s + 2 * d], P.A[6 * s + 2 * d + 1]};
        w.B[d] = dcplx{P.B[6 * s + 2 * d], P.B[6 * s + 2 * d + 1]};
      }
    }
  }
  SlabWaveD *dw = nullptr;
  int *dcol = nullptr;
  dcplx *be = nullptr;
  LF_CUDA(upload(dw, waves.data(), waves.size()));
  std::vector<int> cols(col_of_part, col_of_part + n_parts);
  if (n_parts) LF_CUDA(upload(dcol, cols.data(), cols.size()));
  if (h->n_src) LF_CUDA(dmalloc(be, (size_t)h->n_src * ncol * h->nd));
  if (h->n_src && n_parts) {
    const int wpb = 4;
    k_rhs_elem<<<(h->n_src + wpb - 1) / wpb, wpb * 32, 0, h->stream>>>(
        h->n_src, h->src_list, h->nd, h->p, h->rm.view(), h->J, h->Jinv, h->detJ, h->v0,
        h->slab_of, h->delta, dw, n_slab, n_parts, dcol, ncol, h->pml.k0, h->fopack, be);
    LF_LAUNCHED();
  } else if (h->n_src) {
    LF_CUDA(cudaMemsetAsync(be, 0, (size_t)h->n_src * ncol * h->nd * sizeof(dcplx), h->stream));
  }
  k_rhs_gather<<<(h->n + 255) / 256, 256, 0, h->stream>>>(h->n, h->ea_ptr, h->ea, h->nd,
                                                          h->src_slot, h->sign, be, ncol, h->ess,
                                                          eliminate ? 1 : 0, (dcplx *)d_b);
  LF_LAUNCHED();
  LF_CUDA(cudaStreamSynchronize(h->stream));
  dfree(dw);
  dfree(dcol);
  dfree(be);
  return sync_if(h);
}

static int upload_waves(const lfasm_incident_part *parts, int n_parts, int n_slab_min,
                        std::vector<SlabWaveD> &waves, int &n_slab) {
  n_slab = n_parts > 0 ? parts[0].n_slab : 1;
  if (n_parts > 0 && n_slab_min >= n_slab)
    return fail(LFASM_ERR_ARG, "incident tables have %d slabs; elements reach slab %d", n_slab,
                n_slab_min);
  waves.assign((size_t)std::max(n_parts, 1) * n_slab, SlabWaveD{});
  for (int pi = 0; pi < n_parts; ++pi) {
    const lfasm_incident_part &P = parts[pi];
    if (P.n_slab != n_slab) return fail(LFASM_ERR_ARG, "parts disagree on the slab count");
    for (int s = 0; s < n_slab; ++s) {
      SlabWaveD &w = waves[(size_t)pi * n_slab + s];
      w.qA = dcplx{P.qA[2 * s], P.qA[2 * s + 1]};
      w.qB = dcplx{P.qB[2 * s], P.qB[2 * s + 1]};
      w.zA = P.zA[s];
      w.zB = P.zB[s];
      for (int d = 0; d < 3; ++d) {
        w.A[d] = dcplx{P.A[6 * s + 2 * d], P.A[6 * s + 2 * d + 1]};
        w.B[d] = dcplx{P.B[6 * s + 2 * d], P.B[6 * s + 2 * d + 1]};
      }
    }
  }
  return LFASM_OK;
}

int lfasm_eps_gradient(lfasm_handle *h, const lfasm_incident_part *parts, int n_parts,
                       const void *d_u, const void *d_lambda, void *d_grad) {
  if (!h || !d_u || !d_lambda || !d_grad || n_parts < 0 || (n_parts > 0 && !parts))
    return fail(LFASM_ERR_ARG, "bad gradient arguments");
  g_err.clear();
  if (!h->built) return fail(LFASM_ERR_STATE, "lfasm_build_global has not run");
  LF_CUDA(cudaSetDevice(h->dev));
  std::vector<SlabWaveD> waves;
  int n_slab = 1;
  // the design elements are the non-PML ones; their slabs must be tabulated
  int rc = upload_waves(parts, n_parts, h->max_bulk_slab, waves, n_slab);
  if (rc) return rc;
  SlabWaveD *dw = nullptr;
  LF_CUDA(upload(dw, waves.data(), waves.size()));
  LF_CUDA(cudaMemsetAsync(d_grad, 0, (size_t)h->ne * sizeof(dcplx), h->stream));
  if (h->n_bulk) {
    const int wpb = 4;
    k_eps_grad<<<(h->n_bulk + wpb - 1) / wpb, wpb * 32, 0, h->stream>>>(
        h->n_bulk, h->bulk_list, h->nd, h->p, h->rm.view(), h->J, h->Jinv, h->detJ, h->v0,
        h->dof, h->sign, h->fopack, h->pml, h->slab_of, dw, n_slab, n_parts,
        (const dcplx *)d_u, (const dcplx *)d_lambda, (dcplx *)d_grad);
    LF_LAUNCHED();
  }
  LF_CUDA(cudaStreamSynchronize(h->stream));
  dfree(dw);
  return sync_if(h);
}

void lfasm_destroy(lfasm_handle *h) {
  if (!h) return;
  cudaSetDevice(h->dev);
  // the buffers go back to the pool on the legacy stream: the handle's own
  // streams (possibly non-blocking) finish first
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->side) cudaStreamSynchronize(h->side);
  dfree(h->dof); dfree(h->sign); dfree(h->attr); dfree(h->J); dfree(h->Jinv); dfree(h->detJ);
  dfree(h->v0); dfree(h->fopack); dfree(h->signmask); dfree(h->essmask);
  for (DevRule *r : {&h->rcc, &h->rm}) {
    dfree(r->ip); dfree(r->w); dfree(r->v); dfree(r->c); dfree(r->vt); dfree(r->ct);
  }
  dfree(h->eps_tab); dfree(h->elem_eps); dfree(h->bulk_list); dfree(h->pml_list);
  dfree(h->S); dfree(h->err); dfree(h->bexps); dfree(h->bcoef); dfree(h->bccoef); dfree(h->rec); dfree(h->S_mma); dfree(h->S_mmaf); dfree(h->rec_mma); dfree(h->Ae); dfree(h->slab_of); dfree(h->delta);
  dfree(h->src_list); dfree(h->src_slot); dfree(h->I); dfree(h->Jc); dfree(h->vals);
  dfree(h->ess); dfree(h->ea_ptr); dfree(h->ea); dfree(h->long_rows); dfree(h->off); dfree(h->partials);
  dfree(h->red); dfree(h->row_order);
  for (int i = 0; i < 2; ++i)
    if (h->cexec[i]) cudaGraphExecDestroy(h->cexec[i]);
  for (cudaStream_t *sp : {&h->gstream, &h->cstream})
    if (*sp) {
      cudaStreamSynchronize(*sp);
      cudaStreamDestroy(*sp);
    }
  for (int i = 0; i < 4; ++i)
    if (h->ev[i]) cudaEventDestroy(h->ev[i]);
  if (h->fork) cudaEventDestroy(h->fork);
  if (h->join) cudaEventDestroy(h->join);
  if (h->side) cudaStreamDestroy(h->side);
  delete h;
}

int lfasm_trim_pool(int gpu_id) {
  if (gpu_id < 0 || gpu_id >= MAX_DEV) return fail(LFASM_ERR_ARG, "gpu_id %d out of range", gpu_id);
  int cur = 0;
  LF_CUDA(cudaGetDevice(&cur));
  cudaError_t e = cudaSuccess;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pool[gpu_id] && g_big_free[gpu_id].empty()) return LFASM_OK;
    e = cudaSetDevice(gpu_id);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) {
      drop_big_cache(gpu_id);
      if (g_pool[gpu_id]) e = cudaMemPoolTrimTo(g_pool[gpu_id], 0);
    }
  }
  cudaSetDevice(cur);
  LF_CUDA(e);
  return LFASM_OK;
}

}  // extern "C"
