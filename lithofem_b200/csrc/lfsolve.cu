// liblfsolve.so -- multifrontal sparse LU for the assembled LithoFEM systems
// on B200 (sm_100a), in place of the reference's cuDSS solver
// (solver/cudss_solver.inc:79-309).  C ABI: include/lfsolve.h.
//
// Pipeline
//   analyze (host): nested dissection of the mesh by element bisection (a
//     subdomain's elements are split at the median centroid coordinate
//     along the axis that gives the smallest separator; the separator is the
//     set of still unnumbered DOFs that elements of both halves touch), the
//     postorder elimination tree, every front's index list (its pivots, then
//     the ancestor DOFs its subtree touches) and the maps below;
//   factor (device): depth by depth from the deepest level, the fronts of a
//     level are zeroed, receive their original entries (CSR position ->
//     front offset map) and their children's Schur complements (extend-add),
//     and are partially factored: P [F11 F12] = L11 [U11 U12] with partial
//     pivoting among the front's pivot rows (library getrf on the k x m pivot
//     row panel), L21 = F21 U11^-1 (library trsm), F22 -= L21 U12 (library
//     gemm); the L and U blocks are copied to the factor store;
//   solve (device): forward and backward sweeps over the tree, each front's
//     right-hand side gathered from the global vector and its children's
//     update vectors (no atomics); fronts up to SMALL_M rows in one block
//     each (the vector in shared memory), larger ones through library
//     trsm / gemm; A^T is solved with the same factors (U^T forward, L^T
//     backward, inverse pivots last);
//   refine: FP64 residual on the complex128 CSR, corrections from the
//     factors, per right-hand-side column.
#include <cublas_v2.h>
#include <cuComplex.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lfsolve.h"

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define LS_CUDA(call)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      std::printf("lfsolve: CUDA error '%s' at %s:%d\n", cudaGetErrorString(e_),        \
                  __FILE__, __LINE__);                                                  \
      std::fflush(stdout);                                                              \
      return fail(LFSOLVE_ERR_CUDA, "CUDA error '%s' at %s:%d", cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                  \
    }                                                                                   \
  } while (0)

#define LS_BLAS(call)                                                                     \
  do {                                                                                    \
    const int s_ = (int)(call);                                                           \
    if (s_ != 0)                                                                          \
      return fail(LFSOLVE_ERR_CUDA, "library status %d at %s:%d", s_, __FILE__, __LINE__); \
  } while (0)

constexpr long long ALIGN = 32;  // front / factor block alignment (entries)
inline long long align_up(long long x) { return (x + ALIGN - 1) / ALIGN * ALIGN; }
// pivot blocks and leading dimensions of the fronts are padded to this many
// entries, so that F11, F12, F21 and F22 all start on 128-byte boundaries
// (256 for complex128) with row strides of whole 128-byte lines
constexpr int FPAD = 16;
inline int pad_up(int x) { return (x + FPAD - 1) / FPAD * FPAD; }

// fronts with at most SMALL_M rows, SMALL_K pivots and 2 k + r <= SMALL_BWD
// are solved by one block each, with the right-hand-side block in shared
// memory: m x nrhs entries forward, (2 k + r) x nrhs backward, at most
// 192 kB in complex128 (two right-hand sides a pass); the block takes one
// barrier per pivot, so fronts with more pivots go to the library path
constexpr int SMALL_M = 4096;
constexpr int SMALL_K = 256;
constexpr int SMALL_BWD = 6144;
constexpr int SOLVE_THREADS = 256;
constexpr int MAX_NRHS_PASS = 2;  // right-hand sides per solve pass
constexpr int LANES = 8;          // streams (and library handles) for the fronts
constexpr int BATCH_MIN = 128;    // depths with this many fronts use batched calls
// complex64 fronts whose Schur update F22 -= L21 U12 has at least this many
// complex multiply-adds use three TF32 tensor-core GEMMs on split operands
constexpr double TF32X3_MIN_MACS = 2e9;

// ---------------------------------------------------------------------------
// analysis (host)
// ---------------------------------------------------------------------------
struct Node {
  int parent = -1, nchild = 0, child[2] = {-1, -1};
  int depth = 0;
  int p0 = 0, k = 0, m = 0;   // pivots [p0, p0 + k) of the new numbering; k + r rows
  std::vector<int> R;         // update rows: new indices, ascending
  long long arena_off = 0;    // front offset in its depth's arena (entries)
  long long fac_off = 0;      // factor block offset: P (m x k) then U12 (k x r)
  long long r_off = 0;        // offset of its update rows' original indices
  long long rel_off = 0;      // offset of its rows' positions in the parent front
  long long vec_off = 0;      // solve vector block offset (rows)
  int el0 = 0, el1 = 0;       // element range (leaves)
  int ld = 0;                 // leading dimension of its front in the arena
  int roff = 0;               // front row of its first update row (k, or the
                              // padded pivot count of a batched depth)
};

// host array of n values left uninitialised (filled by the caller), the
// assembly map's hundreds of MB not zeroed first
template <typename T>
struct HostBuf {
  std::unique_ptr<T[]> p;
  size_t n = 0;
  void resize(size_t m) { p.reset(m ? new T[m] : nullptr); n = m; }
  T *data() { return p.get(); }
  const T *data() const { return p.get(); }
  T &operator[](size_t i) { return p[i]; }
  const T &operator[](size_t i) const { return p[i]; }
  size_t size() const { return n; }
  bool empty() const { return n == 0; }
};

struct Plan {
  int n = 0, n_ess = 0, nn = 0;       // rows, essential rows, numbered rows
  long long nnz = 0;
  std::vector<Node> nodes;            // preorder ids
  std::vector<int> post;              // postorder
  std::vector<int> perm, iperm;       // new -> original, original -> new (-1: essential)
  std::vector<int> node_of;           // new index -> node
  std::vector<std::vector<int>> by_depth;
  std::vector<long long> arena_size;  // per depth (entries)
  long long factor_entries = 0, vec_rows = 0;
  std::vector<int> r_orig;            // update rows (original indices), node blocks
  std::vector<int> rel;               // rows of each child in its parent front
  std::vector<int> rel_fac;           // the same in the parent's (padded) front layout
  // depths with many fronts are factored by batched calls on a uniform
  // padded layout: kpad pivot rows (dummy identity pivots after the real
  // ones), rpad update rows (zero rows after the real ones), stride per front
  std::vector<char> batched;
  std::vector<int> kpad, rpad;
  std::vector<long long> stride;
  std::vector<int> ess;
  // assembly map per depth: CSR position -> arena offset
  std::vector<HostBuf<int>> asm_src;        // every entry is written: no zero fill
  std::vector<HostBuf<long long>> asm_dst;
  HostBuf<int> tpos;                  // CSR position of the transposed entry
  double flops = 0.0;
  int max_front = 0, max_k = 0, max_depth = 0;
  long long peak_front_entries = 0;
};

// Nested dissection by element bisection.  Returns the nodes in preorder.
void bisect(int n, int ne, int nd, const int *edof, const double *cen,
            const std::vector<char> &is_ess, int leaf, Plan &P, std::vector<int> &owner,
            std::vector<int> &elems) {
  elems.resize(ne);
  std::iota(elems.begin(), elems.end(), 0);
  owner.assign(n, -1);
  std::vector<int> markL(n, -1), markR(n, -1);
  int stamp = 0;
  struct Item { int a, b, parent, depth, slot; };
  std::vector<Item> stack{{0, ne, -1, 0, 0}};
  std::vector<int> trial, best;
  while (!stack.empty()) {
    const Item it = stack.back();
    stack.pop_back();
    const int id = (int)P.nodes.size();
    P.nodes.emplace_back();
    Node &nd_ = P.nodes.back();
    nd_.parent = it.parent;
    nd_.depth = it.depth;
    nd_.el0 = it.a;
    nd_.el1 = it.b;
    if (it.parent >= 0) {
      Node &par = P.nodes[it.parent];
      par.child[it.slot] = id;
      par.nchild = std::max(par.nchild, it.slot + 1);
    }
    const int cnt = it.b - it.a;
    if (cnt <= leaf) {  // leaf: every unnumbered DOF of its elements
      for (int e = it.a; e < it.b; ++e)
        for (int q = 0; q < nd; ++q) {
          const int d = edof[(size_t)elems[e] * nd + q];
          if (owner[d] < 0 && !is_ess[d]) owner[d] = id;
        }
      continue;
    }
    const int mid = it.a + cnt / 2;
    long long best_sep = -1;
    for (int ax = 0; ax < 3; ++ax) {
      trial.assign(elems.begin() + it.a, elems.begin() + it.b);
      std::nth_element(trial.begin(), trial.begin() + (mid - it.a), trial.end(),
                       [&](int x, int y) {
                         const double cx = cen[(size_t)x * 3 + ax], cy = cen[(size_t)y * 3 + ax];
                         return cx < cy || (cx == cy && x < y);
                       });
      ++stamp;
      for (int t = 0; t < mid - it.a; ++t)
        for (int q = 0; q < nd; ++q) markL[edof[(size_t)trial[t] * nd + q]] = stamp;
      long long sep = 0;
      for (int t = mid - it.a; t < cnt; ++t)
        for (int q = 0; q < nd; ++q) {
          const int d = edof[(size_t)trial[t] * nd + q];
          if (markL[d] == stamp && markR[d] != stamp && owner[d] < 0 && !is_ess[d]) {
            markR[d] = stamp;
            ++sep;
          }
        }
      if (best_sep < 0 || sep < best_sep) {
        best_sep = sep;
        best.swap(trial);
      }
    }
    std::copy(best.begin(), best.end(), elems.begin() + it.a);
    ++stamp;
    for (int e = it.a; e < mid; ++e)
      for (int q = 0; q < nd; ++q) markL[edof[(size_t)elems[e] * nd + q]] = stamp;
    for (int e = mid; e < it.b; ++e)
      for (int q = 0; q < nd; ++q) {
        const int d = edof[(size_t)elems[e] * nd + q];
        if (markL[d] == stamp && owner[d] < 0 && !is_ess[d]) owner[d] = id;
      }
    stack.push_back({mid, it.b, id, it.depth + 1, 1});
    stack.push_back({it.a, mid, id, it.depth + 1, 0});
  }
}

// f(item, worker) for every item of [0, n) on the host threads, items handed
// out one at a time (the fronts' work varies by orders of magnitude)
template <typename F>
void parallel_items(int n, F f) {
  int T = (int)std::min(32u, std::max(1u, std::thread::hardware_concurrency()));
  T = std::max(1, std::min(T, n));
  std::atomic<int> next{0};
  auto run = [&](int w) {
    for (int i = next++; i < n; i = next++) f(i, w);
  };
  if (T == 1) { run(0); return; }
  std::vector<std::thread> th;
  for (int w = 0; w < T; ++w) th.emplace_back(run, w);
  for (auto &t : th) t.join();
}
inline int host_workers(int n) {
  return std::max(1, std::min((int)std::min(32u, std::max(1u, std::thread::hardware_concurrency())), n));
}

int build_plan(int n, const int *I, const int *J, long long nnz, int ne, int nd,
               const int *edof, const double *cen, const int *ess, int n_ess, int leaf,
               Plan &P) {
  P = Plan();
  P.n = n;
  P.nnz = nnz;
  std::vector<char> is_ess(n, 0);
  for (int i = 0; i < n_ess; ++i) {
    if (ess[i] < 0 || ess[i] >= n) return fail(LFSOLVE_ERR_ARG, "essential row %d out of range", ess[i]);
    is_ess[ess[i]] = 1;
  }
  for (int i = 0; i < n; ++i)
    if (is_ess[i]) P.ess.push_back(i);
  P.n_ess = (int)P.ess.size();
  for (long long t = 0; t < (long long)ne * nd; ++t)
    if (edof[t] < 0 || edof[t] >= n) return fail(LFSOLVE_ERR_ARG, "element DOF %d out of range", edof[t]);
  // LFSOLVE_PROFILE set: host seconds of the analysis phases printed
  const bool prof = std::getenv("LFSOLVE_PROFILE") != nullptr;
  auto tick = std::chrono::steady_clock::now();
  auto phase = [&](const char *what) {
    if (!prof) return;
    const auto now = std::chrono::steady_clock::now();
    std::printf("lfsolve analysis: %-28s %8.3f s\n", what,
                std::chrono::duration<double>(now - tick).count());
    std::fflush(stdout);
    tick = now;
  };
  std::vector<int> owner, elems;
  bisect(n, ne, nd, edof, cen, is_ess, leaf, P, owner, elems);
  phase("nested dissection");
  for (int i = 0; i < n; ++i)
    if (!is_ess[i] && owner[i] < 0)
      return fail(LFSOLVE_ERR_ARG, "row %d is touched by no element", i);
  const int ns = (int)P.nodes.size();
  // postorder (children before parents)
  P.post.reserve(ns);
  {
    std::vector<std::pair<int, int>> st{{0, 0}};
    while (!st.empty()) {
      auto &[u, i] = st.back();
      if (i < P.nodes[u].nchild) {
        const int c = P.nodes[u].child[i++];
        st.push_back({c, 0});
      } else {
        P.post.push_back(u);
        st.pop_back();
      }
    }
  }
  // pivots of each node (ascending original index) and the new numbering
  std::vector<std::vector<int>> piv(ns);
  for (int i = 0; i < n; ++i)
    if (owner[i] >= 0) piv[owner[i]].push_back(i);
  P.perm.clear();
  P.iperm.assign(n, -1);
  P.node_of.clear();
  for (int s : P.post) {
    Node &N = P.nodes[s];
    N.p0 = (int)P.perm.size();
    N.k = (int)piv[s].size();
    for (int i : piv[s]) {
      P.iperm[i] = (int)P.perm.size();
      P.perm.push_back(i);
      P.node_of.push_back(s);
    }
  }
  P.nn = (int)P.perm.size();
  // update rows, bottom-up
  for (int s : P.post) {
    Node &N = P.nodes[s];
    std::vector<int> R;
    if (N.nchild == 0) {
      for (int e = N.el0; e < N.el1; ++e)
        for (int q = 0; q < nd; ++q) {
          const int d = edof[(size_t)elems[e] * nd + q];
          const int v = P.iperm[d];
          if (v >= N.p0 + N.k) R.push_back(v);
        }
    } else {
      for (int c = 0; c < N.nchild; ++c)
        for (int v : P.nodes[N.child[c]].R)
          if (v >= N.p0 + N.k) R.push_back(v);
    }
    std::sort(R.begin(), R.end());
    R.erase(std::unique(R.begin(), R.end()), R.end());
    N.R.swap(R);
    N.m = N.k + (int)N.R.size();
    P.max_front = std::max(P.max_front, N.m);
    P.max_k = std::max(P.max_k, N.k);
    P.max_depth = std::max(P.max_depth, N.depth);
    const double k = N.k, r = (double)N.R.size();
    P.flops += 8.0 * (k * k * k / 3.0 + k * k * r + k * r * r);
  }
  phase("numbering, update rows");
  // layouts
  P.by_depth.assign(P.max_depth + 1, {});
  for (int s : P.post) P.by_depth[P.nodes[s].depth].push_back(s);
  P.arena_size.assign(P.max_depth + 1, 0);
  P.batched.assign(P.max_depth + 1, 0);
  P.kpad.assign(P.max_depth + 1, 0);
  P.rpad.assign(P.max_depth + 1, 0);
  P.stride.assign(P.max_depth + 1, 0);
  // LFSOLVE_BATCH_MIN overrides the front count from which a depth is batched
  int batch_min = BATCH_MIN;
  if (const char *e = std::getenv("LFSOLVE_BATCH_MIN")) batch_min = std::max(1, std::atoi(e));
  for (int d = 0; d <= P.max_depth; ++d) {
    if ((int)P.by_depth[d].size() < batch_min) continue;
    int kp = 0, rp = 0;
    for (int s : P.by_depth[d]) {
      kp = std::max(kp, P.nodes[s].k);
      rp = std::max(rp, P.nodes[s].m - P.nodes[s].k);
    }
    if (kp == 0) continue;
    P.batched[d] = 1;
    P.kpad[d] = pad_up(kp);
    P.rpad[d] = pad_up(P.kpad[d] + rp) - P.kpad[d];
    const long long ld = P.kpad[d] + P.rpad[d];
    P.stride[d] = align_up(ld * ld);
  }
  long long fac = 0, roff = 0, vec = 0;
  for (int d = 0; d <= P.max_depth; ++d)
    for (int s : P.by_depth[d]) {
      Node &N = P.nodes[s];
      N.arena_off = P.arena_size[d];
      if (P.batched[d]) {
        N.ld = P.kpad[d] + P.rpad[d];
        N.roff = P.kpad[d];
        P.arena_size[d] += P.stride[d];
      } else {
        // dummy identity pivots k .. roff-1 after the real ones, zero rows
        // and columns past the update rows up to ld
        N.roff = pad_up(N.k);
        N.ld = pad_up(N.roff + (N.m - N.k));
        P.arena_size[d] += align_up((long long)N.ld * N.ld);
      }
      N.fac_off = fac;
      const long long r = (long long)N.R.size();
      fac += align_up((long long)N.m * N.k + (long long)N.k * r);
      N.r_off = roff;
      roff += r;
      N.vec_off = vec;
      vec += N.m;
    }
  P.factor_entries = fac;
  P.vec_rows = vec;
  for (int d = 0; d <= P.max_depth; ++d)
    P.peak_front_entries = std::max(P.peak_front_entries,
                                    P.arena_size[d] + (d < P.max_depth ? P.arena_size[d + 1] : 0));
  P.r_orig.resize(roff);
  for (int s = 0; s < ns; ++s) {
    const Node &N = P.nodes[s];
    for (size_t t = 0; t < N.R.size(); ++t) P.r_orig[N.r_off + t] = P.perm[N.R[t]];
  }
  // each child's update rows located in its parent's front
  std::vector<int> loc(P.nn, -1);
  P.rel.assign(roff, 0);
  P.rel_fac.assign(roff, 0);
  for (int s = 0; s < ns; ++s) {
    const Node &N = P.nodes[s];
    if (N.nchild == 0) continue;
    for (int t = 0; t < N.k; ++t) loc[N.p0 + t] = t;
    for (size_t t = 0; t < N.R.size(); ++t) loc[N.R[t]] = N.k + (int)t;
    for (int c = 0; c < N.nchild; ++c) {
      Node &C = P.nodes[N.child[c]];
      C.rel_off = C.r_off;
      for (size_t t = 0; t < C.R.size(); ++t) {
        const int l = loc[C.R[t]];
        if (l < 0) return fail(LFSOLVE_ERR_ARG, "internal: child row missing from its parent front");
        P.rel[C.r_off + t] = l;
        P.rel_fac[C.r_off + t] = l < N.k ? l : N.roff + (l - N.k);
      }
    }
    for (int t = 0; t < N.k; ++t) loc[N.p0 + t] = -1;
    for (int v : N.R) loc[v] = -1;
  }
  phase("layouts, child row maps");
  // transposed positions: entry (i, j) -> the position of (j, i), by binary
  // search in row j (columns sorted); the structure must be symmetric
  P.tpos.resize(nnz);  // every entry written below (or the call fails)
  {
    std::atomic<long long> bad{-1};
    constexpr int ROWS = 4096;  // rows an item
    parallel_items((n + ROWS - 1) / ROWS, [&](int it, int) {
      for (int i = it * ROWS; i < std::min(n, (it + 1) * ROWS); ++i)
        for (long long p = I[i]; p < I[i + 1]; ++p) {
          const int j = J[p];
          const int *b = J + I[j], *e = J + I[j + 1];
          const int *f = std::lower_bound(b, e, i);
          if (f == e || *f != i) {
            long long expect = -1;
            bad.compare_exchange_strong(expect, (long long)i << 32 | (unsigned)j);
            return;
          }
          P.tpos[p] = (int)(f - J);
        }
    });
    if (bad >= 0)
      return fail(LFSOLVE_ERR_ARG, "the CSR structure is not symmetric (row %d, column %d)",
                  (int)(bad >> 32), (int)(bad & 0xffffffff));
  }
  phase("transposed positions");
  // assembly map: every entry (i, j) with i eliminated at front s and j not
  // eliminated before it goes to its front position (and the transposed
  // entry, when j is an update row); per depth, fronts in index order, each
  // front's entries in row order.  A counting pass sizes every front's
  // slice, then the fronts fill their slices on the host threads.
  P.asm_src.clear();
  P.asm_src.resize(P.max_depth + 1);
  P.asm_dst.clear();
  P.asm_dst.resize(P.max_depth + 1);
  {
    const int W = host_workers(ns);
    std::vector<std::vector<int>> wloc(W, std::vector<int>(P.nn, -1));
    std::vector<long long> cnt(ns, 0), off(ns, 0);
    parallel_items(ns, [&](int s, int) {
      const Node &N = P.nodes[s];
      long long c = 0;
      for (int t = 0; t < N.k; ++t) {
        const int i = P.perm[N.p0 + t];
        for (long long p = I[i]; p < I[i + 1]; ++p) {
          const int vj = P.iperm[J[p]];
          if (vj < N.p0) continue;  // essential, or eliminated further down
          c += vj >= N.p0 + N.k ? 2 : 1;
        }
      }
      cnt[s] = c;
    });
    std::vector<long long> total(P.max_depth + 1, 0);
    for (int s = 0; s < ns; ++s) {
      off[s] = total[P.nodes[s].depth];
      total[P.nodes[s].depth] += cnt[s];
    }
    for (int d = 0; d <= P.max_depth; ++d) {
      P.asm_src[d].resize(total[d]);
      P.asm_dst[d].resize(total[d]);
    }
    std::atomic<int> outside{0};
    parallel_items(ns, [&](int s, int w) {
      const Node &N = P.nodes[s];
      std::vector<int> &lc = wloc[w];
      for (int t = 0; t < N.k; ++t) lc[N.p0 + t] = t;
      for (size_t t = 0; t < N.R.size(); ++t) lc[N.R[t]] = N.roff + (int)t;
      int *src = P.asm_src[N.depth].data() + off[s];
      long long *dst = P.asm_dst[N.depth].data() + off[s];
      long long q = 0;
      for (int t = 0; t < N.k; ++t) {
        const int i = P.perm[N.p0 + t];
        const long long li = t;
        for (long long p = I[i]; p < I[i + 1]; ++p) {
          const int vj = P.iperm[J[p]];
          if (vj < N.p0) continue;
          const long long lj = lc[vj];
          if (lj < 0) { outside = 1; continue; }
          src[q] = (int)p;
          dst[q++] = N.arena_off + li + lj * N.ld;
          if (vj >= N.p0 + N.k) {
            src[q] = P.tpos[p];
            dst[q++] = N.arena_off + lj + li * N.ld;
          }
        }
      }
      for (int t = 0; t < N.k; ++t) lc[N.p0 + t] = -1;
      for (int v : N.R) lc[v] = -1;
    });
    if (outside) return fail(LFSOLVE_ERR_ARG, "internal: coupling outside the front");
  }
  phase("assembly map");
  return LFSOLVE_OK;
}

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
template <typename T> struct CT;
template <> struct CT<cuComplex> {
  using R = float;
  __host__ __device__ static cuComplex mk(double a, double b) { return make_cuComplex((float)a, (float)b); }
};
template <> struct CT<cuDoubleComplex> {
  using R = double;
  __host__ __device__ static cuDoubleComplex mk(double a, double b) { return make_cuDoubleComplex(a, b); }
};
__device__ __forceinline__ cuComplex cmul(cuComplex a, cuComplex b) { return cuCmulf(a, b); }
__device__ __forceinline__ cuDoubleComplex cmul(cuDoubleComplex a, cuDoubleComplex b) { return cuCmul(a, b); }
__device__ __forceinline__ cuComplex csub(cuComplex a, cuComplex b) { return cuCsubf(a, b); }
__device__ __forceinline__ cuDoubleComplex csub(cuDoubleComplex a, cuDoubleComplex b) { return cuCsub(a, b); }
__device__ __forceinline__ cuComplex cadd(cuComplex a, cuComplex b) { return cuCaddf(a, b); }
__device__ __forceinline__ cuDoubleComplex cadd(cuDoubleComplex a, cuDoubleComplex b) { return cuCadd(a, b); }
__device__ __forceinline__ cuComplex cdiv(cuComplex a, cuComplex b) { return cuCdivf(a, b); }
__device__ __forceinline__ cuDoubleComplex cdiv(cuDoubleComplex a, cuDoubleComplex b) { return cuCdiv(a, b); }
template <typename T> __device__ __forceinline__ T czero() { return CT<T>::mk(0.0, 0.0); }
// a - b c
template <typename T> __device__ __forceinline__ T cfms(T a, T b, T c) { return csub(a, cmul(b, c)); }

// original entries into the fronts of one depth
template <typename T>
__global__ void k_assemble(long long cnt, const int *__restrict__ src,
                           const long long *__restrict__ dst, const double2 *__restrict__ vals,
                           T *__restrict__ arena) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cnt;
       t += (long long)gridDim.x * blockDim.x) {
    const double2 v = __ldg(vals + src[t]);
    arena[dst[t]] = CT<T>::mk(v.x, v.y);
  }
}

// Extend-add of one child slot: item = (child node, first column of a strip
// of 32 update columns); F_parent[rel[a], rel[b]] += U_child[a, b].
struct EaItem { int child, col0; };
struct NodeDev {  // per-node data the kernels read
  long long arena_off, fac_off, r_off, vec_off;
  int parent, k, m, p0, depth, ld, roff;
};
template <typename T>
__global__ void k_extend_add(const EaItem *__restrict__ items, const NodeDev *__restrict__ nodes,
                             const int *__restrict__ rel, const T *__restrict__ child_arena,
                             T *__restrict__ arena) {
  const EaItem it = items[blockIdx.x];
  const NodeDev C = nodes[it.child];
  const NodeDev Pn = nodes[C.parent];
  const int r = C.m - C.k;
  const T *U = child_arena + C.arena_off + C.roff + (long long)C.roff * C.ld;  // child's F22
  T *F = arena + Pn.arena_off;
  const int *rl = rel + C.r_off;  // child rows in the parent's front layout
  const int c1 = min(it.col0 + 32, r);
  for (int b = it.col0; b < c1; ++b) {
    const long long cb = (long long)rl[b] * Pn.ld;
    const T *Ub = U + (long long)b * C.ld;
    for (int a = threadIdx.x; a < r; a += blockDim.x) {
      T *f = F + rl[a] + cb;
      *f = cadd(*f, Ub[a]);
    }
  }
}

// copy the L and U blocks of the factored fronts to the factor store:
// P = F[:, 0:k] (m x k) then U12 = F[0:k, k:m] (k x r); item = (node, col0)
template <typename T>
__global__ void k_copy_out(const EaItem *__restrict__ items, const NodeDev *__restrict__ nodes,
                           const T *__restrict__ arena, T *__restrict__ fac) {
  const EaItem it = items[blockIdx.x];
  const NodeDev N = nodes[it.child];
  const T *F = arena + N.arena_off;
  T *Pf = fac + N.fac_off;
  T *U12 = Pf + (long long)N.m * N.k;
  const int c1 = min(it.col0 + 32, N.m);
  for (int c = it.col0; c < c1; ++c) {
    // compact column c: a pivot column (< k) or update column c - k, which
    // sits at front column roff + c - k
    const int fc = c < N.k ? c : N.roff + (c - N.k);
    const T *Fc = F + (long long)fc * N.ld;
    if (c < N.k) {
      T *dst = Pf + (long long)c * N.m;
      for (int a = threadIdx.x; a < N.m; a += blockDim.x)
        dst[a] = Fc[a < N.k ? a : N.roff + (a - N.k)];
    } else {
      T *dst = U12 + (long long)(c - N.k) * N.k;
      for (int a = threadIdx.x; a < N.k; a += blockDim.x) dst[a] = Fc[a];
    }
  }
}

// the row interchanges of a front's pivot block (ipiv, 1-based, applied in
// order) on ncol columns of ld-strided storage: a thread per column
template <typename T>
__global__ void k_swap_cols(int k, int ncol, const int *__restrict__ ipiv, T *__restrict__ A,
                            int ld) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  T *col = A + (long long)c * ld;
  for (int i = 0; i < k; ++i) {
    const int p = ipiv[i] - 1;
    if (p != i) {
      const T t = col[i];
      col[i] = col[p];
      col[p] = t;
    }
  }
}

// dummy identity pivots of each front (rows / columns k .. roff-1), one
// block per front of the depth (list in arena order)
template <typename T>
__global__ void k_dummy_diag(const int *__restrict__ list, const NodeDev *__restrict__ nodes,
                             T *__restrict__ arena) {
  const NodeDev N = nodes[list[blockIdx.x]];
  T *F = arena + N.arena_off;
  for (int i = N.k + threadIdx.x; i < N.roff; i += blockDim.x)
    F[i + (long long)i * N.ld] = CT<T>::mk(1.0, 0.0);
}

// pointer arrays of a batched depth: F11, F12 and F21 of front i
template <typename T>
__global__ void k_make_ptrs(int cnt, T *arena, long long stride, int kpad, int ld, T **p11,
                            T **p12, T **p21) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  T *F = arena + (long long)i * stride;
  p11[i] = F;
  p12[i] = F + (long long)kpad * ld;
  p21[i] = F + kpad;
}

// the real part of the batched pivots / infos to the per-node arrays
__global__ void k_take_pivots(const int *__restrict__ list, const NodeDev *__restrict__ nodes,
                              int kpad, const int *__restrict__ piv, const int *__restrict__ inf,
                              int *__restrict__ ipiv, int *__restrict__ info) {
  const int i = blockIdx.x;
  const int id = list[i];
  const NodeDev N = nodes[id];
  for (int t = threadIdx.x; t < N.k; t += blockDim.x) ipiv[N.p0 + t] = piv[(long long)i * kpad + t];
  if (threadIdx.x == 0) info[id] = inf[i];
}

// batched depths: the fronts' row interchanges on their update columns,
// item = (front, first of 32 columns)
template <typename T>
__global__ void k_swap_cols_batched(const EaItem *__restrict__ items,
                                    const NodeDev *__restrict__ nodes,
                                    const int *__restrict__ ipiv, T *__restrict__ arena) {
  const EaItem it = items[blockIdx.x];
  const NodeDev N = nodes[it.child];
  const int r = N.m - N.k;
  const int c = it.col0 + threadIdx.x;
  if (threadIdx.x >= 32 || c >= r) return;
  T *col = arena + N.arena_off + (long long)(N.roff + c) * N.ld;
  const int *pv = ipiv + N.p0;
  for (int i = 0; i < N.k; ++i) {
    const int q = pv[i] - 1;
    if (q != i) {
      const T t = col[i];
      col[i] = col[q];
      col[q] = t;
    }
  }
}

// y = A x (or A^T x through the transposed positions) in FP64, a warp per
// row; one column
__global__ void k_spmv(int n, const int *__restrict__ I, const int *__restrict__ J,
                       const double2 *__restrict__ vals, const int *__restrict__ tpos,
                       const double2 *__restrict__ x, double2 *__restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= n) return;
  double ar = 0.0, ai = 0.0;
  for (int p = I[row] + lane; p < I[row + 1]; p += 32) {
    const double2 a = vals[tpos ? tpos[p] : p];
    const double2 xv = x[J[p]];
    ar = fma(a.x, xv.x, ar); ar = fma(-a.y, xv.y, ar);
    ai = fma(a.x, xv.y, ai); ai = fma(a.y, xv.x, ai);
  }
  for (int o = 16; o; o >>= 1) {
    ar += __shfl_xor_sync(0xffffffffu, ar, o);
    ai += __shfl_xor_sync(0xffffffffu, ai, o);
  }
  if (lane == 0) y[row] = make_double2(ar, ai);
}

// Error-compensated TF32 operands of F22 -= L21 U12 (complex64, kk pivot
// columns incl. dummies, r update rows), in a real formulation: the complex
// product is the real product of A (2r x 2kk; column 2j is column j of L21
// read as (re, im) float pairs, column 2j + 1 that of i L21) and B (2kk x r;
// U12 read as (re, im) pairs), and the real result read as floats is F22
// itself (leading dimension 2 ld).  Every float x is split as hi = its TF32
// rounding (cvt.rna.tf32.f32, 10 mantissa bits) and lo = x - hi;
// hi hi' + hi lo' + lo hi' carries the product to about 2^-22 relative on
// TF32 tensor cores.  A is stored as [hi | lo] (2r x 4kk, leading dimension
// lda), B as [lo ; hi] (4kk x r, leading dimension 4kk), so that two GEMMs
// ([hi | lo] [lo ; hi] and hi hi) cover the three products.
__device__ __forceinline__ float tf32_round(float x) {
  unsigned u;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(x));
  return __uint_as_float(u);
}
__device__ __forceinline__ void tf32_split(cuComplex v, float2 &h, float2 &l) {
  h = make_float2(tf32_round(v.x), tf32_round(v.y));
  l = make_float2(v.x - h.x, v.y - h.y);
}
// nb fronts of the same shape: front f's block at L + f sL, its operand at
// A + f sA (B + f sB)
__global__ void k_split_a(int r, int kk, const cuComplex *__restrict__ L, int ld,
                          float *__restrict__ A, int lda, int nb, long long sL, long long sA) {
  const long long per = (long long)r * kk, n = per * nb, lo_off = (long long)2 * kk * lda;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const long long f = t / per, u = t - f * per;
    const int i = (int)(u % r), j = (int)(u / r);
    float2 h, l;
    tf32_split(L[f * sL + i + (long long)j * ld], h, l);
    float *c0 = A + f * sA + (long long)(2 * j) * lda + 2 * i;  // column 2j; 2j + 1 one lda on
    *reinterpret_cast<float2 *>(c0) = h;
    *reinterpret_cast<float2 *>(c0 + lda) = make_float2(-h.y, h.x);
    *reinterpret_cast<float2 *>(c0 + lo_off) = l;
    *reinterpret_cast<float2 *>(c0 + lo_off + lda) = make_float2(-l.y, l.x);
  }
}
__global__ void k_split_b(int kk, int r, const cuComplex *__restrict__ U, int ld,
                          float *__restrict__ B, int nb, long long sU, long long sB) {
  const long long per = (long long)kk * r, n = per * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const long long f = t / per, u = t - f * per;
    const int j = (int)(u % kk), c = (int)(u / kk);
    float2 h, l;
    tf32_split(U[f * sU + j + (long long)c * ld], h, l);
    float *col = B + f * sB + (long long)c * 4 * kk;
    *reinterpret_cast<float2 *>(col + 2 * j) = l;
    *reinterpret_cast<float2 *>(col + 2 * kk + 2 * j) = h;
  }
}

// ---------------------------------------------------------------------------
// solve kernels.  Vector blocks: node s owns V[vec_off .. vec_off + m) per
// right-hand-side column, columns nrhs apart by vec_rows (VR).
// ---------------------------------------------------------------------------
// gather: v[0:k] = b[perm[p0 + t]], v[k:m] = 0, plus the children's update
// rows (v_child[k_c + t] at rel[t]); one block per node of the depth
template <typename T>
__global__ void k_gather_rhs(const int *__restrict__ list, const NodeDev *__restrict__ nodes,
                             const int *__restrict__ child, const int *__restrict__ rel,
                             const int *__restrict__ perm, const T *__restrict__ b, int ldb,
                             T *__restrict__ V, long long VR, int nrhs) {
  const int s = list[blockIdx.x];
  const NodeDev N = nodes[s];
  for (int c = 0; c < nrhs; ++c) {
    T *v = V + N.vec_off + c * VR;
    const T *bc = b + (long long)c * ldb;
    for (int a = threadIdx.x; a < N.m; a += blockDim.x)
      v[a] = a < N.k ? bc[perm[N.p0 + a]] : czero<T>();
  }
  __syncthreads();
  for (int q = 0; q < 2; ++q) {  // children in turn: no two writers of one row
    const int cs = child[2 * s + q];
    if (cs < 0) continue;
    const NodeDev C = nodes[cs];
    const int r = C.m - C.k;
    const int *rl = rel + C.r_off;
    for (int c = 0; c < nrhs; ++c) {
      T *v = V + N.vec_off + c * VR;
      const T *u = V + C.vec_off + C.k + c * VR;
      for (int a = threadIdx.x; a < r; a += blockDim.x) v[rl[a]] = cadd(v[rl[a]], u[a]);
    }
    __syncthreads();
  }
}

// forward elimination of small fronts, in place on the vector block:
// TRANS = 0: pivots, L11 (unit) and L21: v[0:k] = y1, v[k:m] -= L21 y1;
// TRANS = 1: U11^T z1 = v[0:k], v[k:m] -= U12^T z1
template <typename T, int TRANS>
__global__ void __launch_bounds__(SOLVE_THREADS)
k_fwd_small(const int *__restrict__ list, const NodeDev *__restrict__ nodes,
            const T *__restrict__ fac, const int *__restrict__ ipiv, T *__restrict__ V,
            long long VR, int nrhs) {
  extern __shared__ unsigned char smraw[];
  T *sv = reinterpret_cast<T *>(smraw);  // m x nrhs
  __shared__ T red[SOLVE_THREADS / 32][MAX_NRHS_PASS];
  const int s = list[blockIdx.x];
  const NodeDev N = nodes[s];
  const int m = N.m, k = N.k, tid = threadIdx.x;
  const T *Pf = fac + N.fac_off;
  const T *U12 = Pf + (long long)m * k;
  for (int c = 0; c < nrhs; ++c)
    for (int a = tid; a < m; a += blockDim.x) sv[a + c * m] = V[N.vec_off + a + c * VR];
  __syncthreads();
  if (TRANS == 0) {
    if (tid == 0)
      for (int i = 0; i < k; ++i) {
        const int p = ipiv[N.p0 + i] - 1;
        if (p != i)
          for (int c = 0; c < nrhs; ++c) {
            const T t = sv[i + c * m];
            sv[i + c * m] = sv[p + c * m];
            sv[p + c * m] = t;
          }
      }
    __syncthreads();
    for (int j = 0; j < k; ++j) {
      const T *col = Pf + (long long)j * m;
      T y[MAX_NRHS_PASS];
      for (int c = 0; c < nrhs; ++c) y[c] = sv[j + c * m];
      for (int a = j + 1 + tid; a < m; a += blockDim.x) {
        const T l = col[a];
        for (int c = 0; c < nrhs; ++c) sv[a + c * m] = cfms(sv[a + c * m], l, y[c]);
      }
      __syncthreads();
    }
  } else {
    // z_j = (v_j - sum_{i<j} U[i][j] z_i) / U[j][j]: column j of U11 is
    // contiguous; one block reduction per pivot
    const int lane = tid & 31, w = tid >> 5;
    for (int j = 0; j < k; ++j) {
      const T *col = Pf + (long long)j * m;
      T acc[MAX_NRHS_PASS];
      for (int c = 0; c < nrhs; ++c) acc[c] = czero<T>();
      for (int i = tid; i < j; i += blockDim.x) {
        const T u = col[i];
        for (int c = 0; c < nrhs; ++c) acc[c] = cadd(acc[c], cmul(u, sv[i + c * m]));
      }
      for (int c = 0; c < nrhs; ++c)
        for (int o = 16; o; o >>= 1) {
          acc[c].x += __shfl_xor_sync(0xffffffffu, acc[c].x, o);
          acc[c].y += __shfl_xor_sync(0xffffffffu, acc[c].y, o);
        }
      if (lane == 0)
        for (int c = 0; c < nrhs; ++c) red[w][c] = acc[c];
      __syncthreads();
      if (tid == 0) {
        const T d = col[j];
        for (int c = 0; c < nrhs; ++c) {
          T sum = czero<T>();
          for (int q = 0; q < (int)(blockDim.x >> 5); ++q) sum = cadd(sum, red[q][c]);
          sv[j + c * m] = cdiv(csub(sv[j + c * m], sum), d);
        }
      }
      __syncthreads();
    }
    // v[k + t] -= sum_i U12[i][t] z_i: a warp per update row, column t of
    // U12 contiguous
    const int r = m - k;
    for (int t = w; t < r; t += blockDim.x >> 5) {
      const T *col = U12 + (long long)t * k;
      T acc[MAX_NRHS_PASS];
      for (int c = 0; c < nrhs; ++c) acc[c] = czero<T>();
      for (int i = lane; i < k; i += 32) {
        const T u = col[i];
        for (int c = 0; c < nrhs; ++c) acc[c] = cadd(acc[c], cmul(u, sv[i + c * m]));
      }
      for (int c = 0; c < nrhs; ++c)
        for (int o = 16; o; o >>= 1) {
          acc[c].x += __shfl_xor_sync(0xffffffffu, acc[c].x, o);
          acc[c].y += __shfl_xor_sync(0xffffffffu, acc[c].y, o);
        }
      if (lane == 0)
        for (int c = 0; c < nrhs; ++c) sv[k + t + c * m] = csub(sv[k + t + c * m], acc[c]);
    }
    __syncthreads();
  }
  for (int c = 0; c < nrhs; ++c)
    for (int a = tid; a < m; a += blockDim.x) V[N.vec_off + a + c * VR] = sv[a + c * m];
}

// backward substitution of small fronts; x (original numbering, ld ldx):
// TRANS = 0: x1 = U11^-1 (y1 - U12 x_R);
// TRANS = 1: w = L11^-T (z1 - L21^T x_R), then the inverse row swaps
template <typename T, int TRANS>
__global__ void __launch_bounds__(SOLVE_THREADS)
k_bwd_small(const int *__restrict__ list, const NodeDev *__restrict__ nodes,
            const T *__restrict__ fac, const int *__restrict__ ipiv,
            const int *__restrict__ perm, const int *__restrict__ r_orig,
            const T *__restrict__ V, long long VR, T *__restrict__ x, int ldx, int nrhs) {
  extern __shared__ unsigned char smraw[];
  const int s = list[blockIdx.x];
  const NodeDev N = nodes[s];
  const int m = N.m, k = N.k, r = m - k, tid = threadIdx.x;
  T *st = reinterpret_cast<T *>(smraw);  // k x nrhs: right-hand side
  T *sx = st + (size_t)k * nrhs;         // k x nrhs: solution
  T *sr = sx + (size_t)k * nrhs;         // r x nrhs: x of the update rows
  __shared__ T red[SOLVE_THREADS / 32][MAX_NRHS_PASS];
  const T *Pf = fac + N.fac_off;
  const T *U12 = Pf + (long long)m * k;
  const int *ro = r_orig + N.r_off;
  for (int c = 0; c < nrhs; ++c) {
    for (int a = tid; a < k; a += blockDim.x) st[a + c * k] = V[N.vec_off + a + c * VR];
    for (int a = tid; a < r; a += blockDim.x) sr[a + c * r] = x[(long long)c * ldx + ro[a]];
  }
  __syncthreads();
  const int lane = tid & 31, w = tid >> 5;
  if (TRANS == 0) {
    // st -= U12 x_R: a thread per pivot row, U12 columns contiguous
    for (int i = tid; i < k; i += blockDim.x) {
      T acc[MAX_NRHS_PASS];
      for (int c = 0; c < nrhs; ++c) acc[c] = st[i + c * k];
      for (int t = 0; t < r; ++t) {
        const T u = U12[i + (long long)t * k];
        for (int c = 0; c < nrhs; ++c) acc[c] = cfms(acc[c], u, sr[t + c * r]);
      }
      for (int c = 0; c < nrhs; ++c) st[i + c * k] = acc[c];
    }
    __syncthreads();
    // back substitution with U11: one barrier per pivot (st[j] is final at
    // step j; the solution goes to sx, which nobody reads in the loop)
    for (int j = k - 1; j >= 0; --j) {
      const T *col = Pf + (long long)j * m;
      const T d = col[j];
      T xj[MAX_NRHS_PASS];
      for (int c = 0; c < nrhs; ++c) xj[c] = cdiv(st[j + c * k], d);
      if (tid == 0)
        for (int c = 0; c < nrhs; ++c) sx[j + c * k] = xj[c];
      for (int i = tid; i < j; i += blockDim.x) {
        const T u = col[i];
        for (int c = 0; c < nrhs; ++c) st[i + c * k] = cfms(st[i + c * k], u, xj[c]);
      }
      __syncthreads();
    }
  } else {
    // st -= L21^T x_R: a warp per pivot column, rows k..m-1 of P contiguous
    for (int j = w; j < k; j += blockDim.x >> 5) {
      const T *col = Pf + (long long)j * m + k;
      T acc[MAX_NRHS_PASS];
      for (int c = 0; c < nrhs; ++c) acc[c] = czero<T>();
      for (int t = lane; t < r; t += 32) {
        const T l = col[t];
        for (int c = 0; c < nrhs; ++c) acc[c] = cadd(acc[c], cmul(l, sr[t + c * r]));
      }
      for (int c = 0; c < nrhs; ++c)
        for (int o = 16; o; o >>= 1) {
          acc[c].x += __shfl_xor_sync(0xffffffffu, acc[c].x, o);
          acc[c].y += __shfl_xor_sync(0xffffffffu, acc[c].y, o);
        }
      if (lane == 0)
        for (int c = 0; c < nrhs; ++c) st[j + c * k] = csub(st[j + c * k], acc[c]);
    }
    __syncthreads();
    // L11^T (unit upper) back substitution: w_j = st_j - sum_{i>j} L[i][j] w_i
    for (int j = k - 1; j >= 0; --j) {
      const T *col = Pf + (long long)j * m;
      T acc[MAX_NRHS_PASS];
      for (int c = 0; c < nrhs; ++c) acc[c] = czero<T>();
      for (int i = j + 1 + tid; i < k; i += blockDim.x) {
        const T l = col[i];
        for (int c = 0; c < nrhs; ++c) acc[c] = cadd(acc[c], cmul(l, sx[i + c * k]));
      }
      for (int c = 0; c < nrhs; ++c)
        for (int o = 16; o; o >>= 1) {
          acc[c].x += __shfl_xor_sync(0xffffffffu, acc[c].x, o);
          acc[c].y += __shfl_xor_sync(0xffffffffu, acc[c].y, o);
        }
      if (lane == 0)
        for (int c = 0; c < nrhs; ++c) red[w][c] = acc[c];
      __syncthreads();
      if (tid == 0)
        for (int c = 0; c < nrhs; ++c) {
          T sum = czero<T>();
          for (int q = 0; q < (int)(blockDim.x >> 5); ++q) sum = cadd(sum, red[q][c]);
          sx[j + c * k] = csub(st[j + c * k], sum);
        }
      __syncthreads();
    }
    if (tid == 0)
      for (int i = k - 1; i >= 0; --i) {
        const int p = ipiv[N.p0 + i] - 1;
        if (p != i)
          for (int c = 0; c < nrhs; ++c) {
            const T t = sx[i + c * k];
            sx[i + c * k] = sx[p + c * k];
            sx[p + c * k] = t;
          }
      }
    __syncthreads();
  }
  for (int c = 0; c < nrhs; ++c)
    for (int a = tid; a < k; a += blockDim.x) x[(long long)c * ldx + perm[N.p0 + a]] = sx[a + c * k];
}

// big fronts: row swaps of the pivot rows of a vector block (forward,
// TRANS = 0) or the inverse swaps (TRANS = 1); one thread
template <typename T, int INV>
__global__ void k_laswp(int k, const int *__restrict__ ipiv, T *__restrict__ v, int ldv, int nrhs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int q = 0; q < k; ++q) {
    const int i = INV ? k - 1 - q : q;
    const int p = ipiv[i] - 1;
    if (p != i)
      for (int c = 0; c < nrhs; ++c) {
        const T t = v[i + (long long)c * ldv];
        v[i + (long long)c * ldv] = v[p + (long long)c * ldv];
        v[p + (long long)c * ldv] = t;
      }
  }
}

// Pivot permutation of every front: the front's sequential row swaps
// (ipiv, 1-based) applied to the identity, so that the swapped vector is
// v[perm[i]] at row i and the inverse swaps put row i at perm[i]; a block
// per front, the swaps in shared memory up to cap pivots (global beyond)
constexpr int PERM_CAP = 12288;
__device__ void perm_from_ipiv(int k, const int *__restrict__ pv, int *__restrict__ dst,
                               int *__restrict__ sp) {
  int *w = k <= PERM_CAP ? sp : dst;
  for (int i = threadIdx.x; i < k; i += blockDim.x) w[i] = i;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int q = 0; q < k; ++q) {
      const int p = pv[q] - 1;
      if (p != q && p >= 0 && p < k) {
        const int t = w[q];
        w[q] = w[p];
        w[p] = t;
      }
    }
  __syncthreads();
  if (k <= PERM_CAP)
    for (int i = threadIdx.x; i < k; i += blockDim.x) dst[i] = sp[i];
}
__global__ void k_ipiv_to_perm(const NodeDev *__restrict__ nodes, const int *__restrict__ ipiv,
                               int *__restrict__ perm) {
  __shared__ int sp[PERM_CAP];
  const NodeDev N = nodes[blockIdx.x];
  perm_from_ipiv(N.k, ipiv + N.p0, perm + N.p0, sp);
}
// one front's permutation (k pivots at pv) into perm
__global__ void k_ipiv_to_perm_one(int k, const int *__restrict__ pv, int *__restrict__ perm) {
  __shared__ int sp[PERM_CAP];
  perm_from_ipiv(k, pv, perm, sp);
}
// the factorization's row interchanges on the ncol update columns of a
// front (A: the first k rows of column c at A + c ld): a block per column,
// the k rows staged in shared memory, row i taking row perm[i]
template <typename T>
__global__ void k_perm_cols(int k, const int *__restrict__ perm, T *__restrict__ A, int ld) {
  extern __shared__ unsigned char pc_sm[];
  T *sv = reinterpret_cast<T *>(pc_sm);
  T *col = A + (long long)blockIdx.x * ld;
  for (int i = threadIdx.x; i < k; i += blockDim.x) sv[i] = col[i];
  __syncthreads();
  for (int i = threadIdx.x; i < k; i += blockDim.x) col[i] = sv[perm[i]];
}

// big fronts: the pivot rows of a vector block permuted (INV = 0: row i
// takes row perm[i]; INV = 1: row i goes to perm[i]); a block per column,
// the k rows staged in shared memory
template <typename T, int INV>
__global__ void k_perm_pivots(int k, const int *__restrict__ perm, T *__restrict__ v, int ldv) {
  extern __shared__ unsigned char perm_sm[];
  T *sv = reinterpret_cast<T *>(perm_sm);
  T *vc = v + (long long)blockIdx.x * ldv;
  for (int i = threadIdx.x; i < k; i += blockDim.x) sv[i] = vc[i];
  __syncthreads();
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    if (INV) vc[perm[i]] = sv[i];
    else vc[i] = sv[perm[i]];
  }
}
// pivots of a vector block that the shared-memory permutation can take
template <typename T>
constexpr int perm_smem_max() { return (int)(160 * 1024 / sizeof(T)); }

// big fronts: x_R gathered into a dense block (r x nrhs, ld r), and the
// pivots' solution scattered back to x
template <typename T>
__global__ void k_gather_rows(int r, const int *__restrict__ ro, const T *__restrict__ x,
                              int ldx, T *__restrict__ out, int nrhs) {
  for (int c = 0; c < nrhs; ++c)
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < r; a += gridDim.x * blockDim.x)
      out[a + (long long)c * r] = x[(long long)c * ldx + ro[a]];
}
template <typename T>
__global__ void k_scatter_pivots(int k, const int *__restrict__ pv, const T *__restrict__ v,
                                 long long VR, T *__restrict__ x, int ldx, int nrhs) {
  for (int c = 0; c < nrhs; ++c)
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < k; a += gridDim.x * blockDim.x)
      x[(long long)c * ldx + pv[a]] = v[a + c * VR];
}

// x[ess] = b[ess]
template <typename T>
__global__ void k_ess_copy(int ne, const int *__restrict__ ess, const T *__restrict__ b, int ldb,
                           T *__restrict__ x, int ldx, int nrhs) {
  for (int c = 0; c < nrhs; ++c)
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < ne; a += gridDim.x * blockDim.x)
      x[(long long)c * ldx + ess[a]] = b[(long long)c * ldb + ess[a]];
}

// conversions: out = (T)(in * scale[c]);  acc += scale[c] * (double)d
template <typename T>
__global__ void k_to_prec(long long n, int ncol, const double2 *__restrict__ in,
                          const double *__restrict__ scale, T *__restrict__ out) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * ncol;
       t += (long long)gridDim.x * blockDim.x) {
    const double s = scale ? scale[t / n] : 1.0;
    out[t] = CT<T>::mk(in[t].x * s, in[t].y * s);
  }
}
template <typename T>
__global__ void k_from_prec(long long n, int ncol, const T *__restrict__ d,
                            const double *__restrict__ scale, double2 *__restrict__ acc,
                            int accumulate) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * ncol;
       t += (long long)gridDim.x * blockDim.x) {
    const double s = scale ? scale[t / n] : 1.0;
    const double2 v = make_double2((double)d[t].x * s, (double)d[t].y * s);
    acc[t] = accumulate ? make_double2(acc[t].x + v.x, acc[t].y + v.y) : v;
  }
}

// FP64 residual r = b - A x (or A^T x through the transposed positions), a
// warp per row, and per column partial sums of |r|^2, |b|^2, max |r|
__global__ void k_resid(int n, int ncol, const int *__restrict__ I, const int *__restrict__ J,
                        const double2 *__restrict__ vals, const int *__restrict__ tpos,
                        const double2 *__restrict__ x, const double2 *__restrict__ b,
                        double2 *__restrict__ r, double *__restrict__ part) {
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int c = blockIdx.y;
  double rn = 0.0, bn = 0.0, rmax = 0.0;
  if (row < n) {
    const double2 *xc = x + (long long)c * n;
    double ar = 0.0, ai = 0.0;
    for (int p = I[row] + lane; p < I[row + 1]; p += 32) {
      const double2 a = vals[tpos ? tpos[p] : p];
      const double2 xv = xc[J[p]];
      ar = fma(a.x, xv.x, ar); ar = fma(-a.y, xv.y, ar);
      ai = fma(a.x, xv.y, ai); ai = fma(a.y, xv.x, ai);
    }
    for (int o = 16; o; o >>= 1) {
      ar += __shfl_xor_sync(0xffffffffu, ar, o);
      ai += __shfl_xor_sync(0xffffffffu, ai, o);
    }
    if (lane == 0) {
      const double2 bv = b[(long long)c * n + row];
      const double dr = bv.x - ar, di = bv.y - ai;
      r[(long long)c * n + row] = make_double2(dr, di);
      rn = dr * dr + di * di;
      bn = bv.x * bv.x + bv.y * bv.y;
      rmax = fmax(fabs(dr), fabs(di));
    }
  }
  __shared__ double red[3][32];
  const int w = threadIdx.x >> 5;
  if (lane == 0) { red[0][w] = rn; red[1][w] = bn; red[2][w] = rmax; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
      a0 += red[0][q]; a1 += red[1][q]; a2 = fmax(a2, red[2][q]);
    }
    double *pp = part + 3 * ((long long)c * gridDim.x + blockIdx.x);
    pp[0] = a0; pp[1] = a1; pp[2] = a2;
  }
}
__global__ void k_resid_sum(int nblk, int ncol, const double *__restrict__ part,
                            double *__restrict__ out) {
  const int c = blockIdx.x;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
    const double *pp = part + 3 * ((long long)c * nblk + i);
    a0 += pp[0]; a1 += pp[1]; a2 = fmax(a2, pp[2]);
  }
  __shared__ double red[3][32];
  for (int o = 16; o; o >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 = fmax(a2, __shfl_xor_sync(0xffffffffu, a2, o));
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { red[0][w] = a0; red[1][w] = a1; red[2][w] = a2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
      s0 += red[0][q]; s1 += red[1][q]; s2 = fmax(s2, red[2][q]);
    }
    out[3 * c] = s0; out[3 * c + 1] = s1; out[3 * c + 2] = s2;
  }
}

// ---------------------------------------------------------------------------
// library dispatch by precision
// ---------------------------------------------------------------------------
inline cusolverStatus_t getrf_buf(cusolverDnHandle_t h, int m, int n, cuComplex *A, int lda, int *lw) {
  return cusolverDnCgetrf_bufferSize(h, m, n, A, lda, lw);
}
inline cusolverStatus_t getrf_buf(cusolverDnHandle_t h, int m, int n, cuDoubleComplex *A, int lda, int *lw) {
  return cusolverDnZgetrf_bufferSize(h, m, n, A, lda, lw);
}
inline cusolverStatus_t getrf(cusolverDnHandle_t h, int m, int n, cuComplex *A, int lda, cuComplex *w, int *ip, int *info) {
  return cusolverDnCgetrf(h, m, n, A, lda, w, ip, info);
}
inline cusolverStatus_t getrf(cusolverDnHandle_t h, int m, int n, cuDoubleComplex *A, int lda, cuDoubleComplex *w, int *ip, int *info) {
  return cusolverDnZgetrf(h, m, n, A, lda, w, ip, info);
}
inline cublasStatus_t trsm(cublasHandle_t h, cublasSideMode_t sd, cublasFillMode_t ul, cublasOperation_t tr,
                           cublasDiagType_t dg, int m, int n, const cuComplex *al, const cuComplex *A, int lda,
                           cuComplex *B, int ldb) {
  return cublasCtrsm(h, sd, ul, tr, dg, m, n, al, A, lda, B, ldb);
}
inline cublasStatus_t trsm(cublasHandle_t h, cublasSideMode_t sd, cublasFillMode_t ul, cublasOperation_t tr,
                           cublasDiagType_t dg, int m, int n, const cuDoubleComplex *al, const cuDoubleComplex *A,
                           int lda, cuDoubleComplex *B, int ldb) {
  return cublasZtrsm(h, sd, ul, tr, dg, m, n, al, A, lda, B, ldb);
}
inline cublasStatus_t gemm(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k,
                           const cuComplex *al, const cuComplex *A, int lda, const cuComplex *B, int ldb,
                           const cuComplex *be, cuComplex *C, int ldc) {
  return cublasCgemm(h, ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc);
}
inline cublasStatus_t gemm(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k,
                           const cuDoubleComplex *al, const cuDoubleComplex *A, int lda,
                           const cuDoubleComplex *B, int ldb, const cuDoubleComplex *be, cuDoubleComplex *C,
                           int ldc) {
  return cublasZgemm(h, ta, tb, m, n, k, al, A, lda, B, ldb, be, C, ldc);
}

inline cublasStatus_t getrf_batched(cublasHandle_t h, int n, cuComplex *const A[], int lda, int *piv,
                                   int *info, int b) {
  return cublasCgetrfBatched(h, n, A, lda, piv, info, b);
}
inline cublasStatus_t getrf_batched(cublasHandle_t h, int n, cuDoubleComplex *const A[], int lda,
                                   int *piv, int *info, int b) {
  return cublasZgetrfBatched(h, n, A, lda, piv, info, b);
}
inline cublasStatus_t trsm_batched(cublasHandle_t h, cublasSideMode_t sd, cublasFillMode_t ul,
                                   cublasOperation_t tr, cublasDiagType_t dg, int m, int n,
                                   const cuComplex *al, const cuComplex *const A[], int lda,
                                   cuComplex *const B[], int ldb, int b) {
  return cublasCtrsmBatched(h, sd, ul, tr, dg, m, n, al, A, lda, B, ldb, b);
}
inline cublasStatus_t trsm_batched(cublasHandle_t h, cublasSideMode_t sd, cublasFillMode_t ul,
                                   cublasOperation_t tr, cublasDiagType_t dg, int m, int n,
                                   const cuDoubleComplex *al, const cuDoubleComplex *const A[],
                                   int lda, cuDoubleComplex *const B[], int ldb, int b) {
  return cublasZtrsmBatched(h, sd, ul, tr, dg, m, n, al, A, lda, B, ldb, b);
}
inline cublasStatus_t gemm_sb(cublasHandle_t h, int m, int n, int k, const cuComplex *al,
                              const cuComplex *A, int lda, long long sa, const cuComplex *B, int ldb,
                              long long sb, const cuComplex *be, cuComplex *C, int ldc, long long sc,
                              int b) {
  return cublasCgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, al, A, lda, sa, B, ldb,
                                   sb, be, C, ldc, sc, b);
}
inline cublasStatus_t gemm_sb(cublasHandle_t h, int m, int n, int k, const cuDoubleComplex *al,
                              const cuDoubleComplex *A, int lda, long long sa,
                              const cuDoubleComplex *B, int ldb, long long sb,
                              const cuDoubleComplex *be, cuDoubleComplex *C, int ldc, long long sc,
                              int b) {
  return cublasZgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, al, A, lda, sa, B, ldb,
                                   sb, be, C, ldc, sc, b);
}

}  // namespace

// ---------------------------------------------------------------------------
// solver object
// ---------------------------------------------------------------------------
struct lfsolve {
  int dev = 0;
  cudaStream_t stream = nullptr;
  bool analyzed = false, uploaded = false;
  Plan P;
  lfsolve_stats st{};
  // device copies of the plan
  NodeDev *d_nodes = nullptr;
  int *d_child = nullptr, *d_rel = nullptr, *d_perm = nullptr, *d_rorig = nullptr,
      *d_ess = nullptr, *d_tpos = nullptr;
  std::vector<int *> d_asm_src;
  std::vector<long long *> d_asm_dst;
  std::vector<EaItem *> d_ea[2], d_co;    // per depth: extend-add items per slot, copy-out items
  std::vector<int> n_ea[2], n_co;
  std::vector<int *> d_small, d_all;      // per depth: small fronts, all fronts
  int *d_rel_fac = nullptr;               // child rows in the parents' front layout
  std::vector<EaItem *> d_sw;             // batched depths: swap items (front, columns)
  std::vector<int> n_sw;
  void **d_ptrs = nullptr;                // batched pointer arrays (3 x max fronts)
  int *d_bpiv = nullptr, *d_binf = nullptr;
  std::vector<std::vector<int>> big;      // per depth: big fronts (host ids)
  std::vector<int> n_small;
  // factors
  int prec = -1;
  void *d_fac = nullptr;
  int *d_ipiv = nullptr, *d_info = nullptr;
  int *d_pperm = nullptr;  // per-front pivot permutations (from d_ipiv)
  // lanes
  cudaStream_t lane[LANES] = {};
  cublasHandle_t blas[LANES] = {};
  cusolverDnHandle_t sol[LANES] = {};
  void *work[LANES] = {};
  size_t work_bytes[LANES] = {};
  cudaEvent_t ev_main = nullptr, ev_lane[LANES] = {};
  // the front workspace comes from a private pool that keeps its memory
  // between depths and factorizations (a pool that hands memory back to the
  // driver at every synchronize re-maps gigabytes per depth)
  cudaMemPool_t pool = nullptr;
  // 3xTF32 Schur updates of large complex64 fronts: per-lane split buffers
  void *split[LANES] = {};
  size_t split_bytes[LANES] = {};
  int *lpiv[LANES] = {};  // pivots of a front's padded pivot block
  int lpiv_n[LANES] = {};
  cublasHandle_t blas_main = nullptr;
  // solve scratch
  void *d_V = nullptr, *d_bw = nullptr, *d_xr = nullptr;
  size_t xr_lane = 0;  // entries of one lane's x_R scratch
  size_t V_bytes = 0, bw_bytes = 0, xr_bytes = 0;
  double2 *d_r = nullptr, *d_x64 = nullptr;
  size_t r_bytes = 0;
  double *d_part = nullptr, *d_scale = nullptr;
  size_t part_bytes = 0;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
};

namespace {

template <typename T>
int upload(T **dst, const HostBuf<T> &v, cudaStream_t st) {
  *dst = nullptr;
  if (v.empty()) return LFSOLVE_OK;
  LS_CUDA(cudaMalloc((void **)dst, v.size() * sizeof(T)));
  LS_CUDA(cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return LFSOLVE_OK;
}
template <typename T>
int upload(T **dst, const std::vector<T> &v, cudaStream_t st) {
  *dst = nullptr;
  if (v.empty()) return LFSOLVE_OK;
  LS_CUDA(cudaMalloc((void **)dst, v.size() * sizeof(T)));
  LS_CUDA(cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return LFSOLVE_OK;
}

bool is_small(const Node &N) {
  return N.m <= SMALL_M && N.k <= SMALL_K && 2 * N.k + (N.m - N.k) <= SMALL_BWD;
}

int ensure_uploaded(lfsolve *s) {
  if (s->uploaded) return LFSOLVE_OK;
  Plan &P = s->P;
  const int ns = (int)P.nodes.size();
  std::vector<NodeDev> nd(ns);
  std::vector<int> child(2 * ns, -1);
  for (int i = 0; i < ns; ++i) {
    const Node &N = P.nodes[i];
    nd[i] = {N.arena_off, N.fac_off, N.r_off, N.vec_off, N.parent, N.k, N.m, N.p0, N.depth,
             N.ld, N.roff};
    child[2 * i] = N.child[0];
    child[2 * i + 1] = N.nchild > 1 ? N.child[1] : -1;
  }
  cudaStream_t st = s->stream;
  int rc;
  if ((rc = upload(&s->d_nodes, nd, st))) return rc;
  if ((rc = upload(&s->d_child, child, st))) return rc;
  if ((rc = upload(&s->d_rel, P.rel, st))) return rc;
  if ((rc = upload(&s->d_rel_fac, P.rel_fac, st))) return rc;
  if ((rc = upload(&s->d_perm, P.perm, st))) return rc;
  if ((rc = upload(&s->d_rorig, P.r_orig, st))) return rc;
  if ((rc = upload(&s->d_ess, P.ess, st))) return rc;
  if ((rc = upload(&s->d_tpos, P.tpos, st))) return rc;
  const int D = P.max_depth + 1;
  s->d_asm_src.assign(D, nullptr);
  s->d_asm_dst.assign(D, nullptr);
  for (int q = 0; q < 2; ++q) { s->d_ea[q].assign(D, nullptr); s->n_ea[q].assign(D, 0); }
  s->d_co.assign(D, nullptr);
  s->n_co.assign(D, 0);
  s->d_small.assign(D, nullptr);
  s->d_all.assign(D, nullptr);
  s->n_small.assign(D, 0);
  s->big.assign(D, {});
  s->d_sw.assign(D, nullptr);
  s->n_sw.assign(D, 0);
  long long maxb = 1, maxpiv = 1;
  for (int d = 0; d < D; ++d)
    if (P.batched[d]) {
      maxb = std::max<long long>(maxb, (long long)P.by_depth[d].size());
      maxpiv = std::max<long long>(maxpiv, (long long)P.by_depth[d].size() * P.kpad[d]);
    }
  LS_CUDA(cudaMalloc((void **)&s->d_ptrs, sizeof(void *) * 3 * maxb));
  LS_CUDA(cudaMalloc((void **)&s->d_bpiv, sizeof(int) * maxpiv));
  LS_CUDA(cudaMalloc((void **)&s->d_binf, sizeof(int) * maxb));
  for (int d = 0; d < D; ++d) {
    if ((rc = upload(&s->d_asm_src[d], P.asm_src[d], st))) return rc;
    if ((rc = upload(&s->d_asm_dst[d], P.asm_dst[d], st))) return rc;
    std::vector<EaItem> ea[2], co;
    std::vector<int> small;
    for (int id : P.by_depth[d]) {
      const Node &N = P.nodes[id];
      for (int q = 0; q < N.nchild; ++q) {
        const Node &C = P.nodes[N.child[q]];
        const int r = C.m - C.k;
        for (int c0 = 0; c0 < r; c0 += 32) ea[q].push_back({N.child[q], c0});
      }
      for (int c0 = 0; c0 < N.m; c0 += 32) co.push_back({id, c0});
      if (is_small(N)) small.push_back(id);
      else s->big[d].push_back(id);
    }
    for (int q = 0; q < 2; ++q) {
      if ((rc = upload(&s->d_ea[q][d], ea[q], st))) return rc;
      s->n_ea[q][d] = (int)ea[q].size();
    }
    if (P.batched[d]) {
      std::vector<EaItem> sw;
      for (int id : P.by_depth[d]) {
        const Node &N = P.nodes[id];
        for (int c0 = 0; c0 < N.m - N.k; c0 += 32) sw.push_back({id, c0});
      }
      if ((rc = upload(&s->d_sw[d], sw, st))) return rc;
      s->n_sw[d] = (int)sw.size();
    }
    if ((rc = upload(&s->d_co[d], co, st))) return rc;
    s->n_co[d] = (int)co.size();
    if ((rc = upload(&s->d_small[d], small, st))) return rc;
    s->n_small[d] = (int)small.size();
    if ((rc = upload(&s->d_all[d], P.by_depth[d], st))) return rc;
  }
  LS_CUDA(cudaStreamSynchronize(st));
  s->uploaded = true;
  return LFSOLVE_OK;
}

int ensure_lanes(lfsolve *s) {
  if (s->blas_main) return LFSOLVE_OK;
  LS_BLAS(cublasCreate(&s->blas_main));
  LS_BLAS(cublasSetStream(s->blas_main, s->stream));
  // the vector permutations stage up to 160 kB of pivot rows
  LS_CUDA(cudaFuncSetAttribute(k_perm_pivots<cuComplex, 0>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
  LS_CUDA(cudaFuncSetAttribute(k_perm_pivots<cuComplex, 1>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
  LS_CUDA(cudaFuncSetAttribute(k_perm_pivots<cuDoubleComplex, 0>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
  LS_CUDA(cudaFuncSetAttribute(k_perm_pivots<cuDoubleComplex, 1>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
  LS_CUDA(cudaFuncSetAttribute(k_perm_cols<cuComplex>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
  LS_CUDA(cudaFuncSetAttribute(k_perm_cols<cuDoubleComplex>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
  for (int l = 0; l < LANES; ++l) {
    LS_CUDA(cudaStreamCreateWithFlags(&s->lane[l], cudaStreamNonBlocking));
    LS_BLAS(cublasCreate(&s->blas[l]));
    LS_BLAS(cublasSetStream(s->blas[l], s->lane[l]));
    LS_BLAS(cusolverDnCreate(&s->sol[l]));
    LS_BLAS(cusolverDnSetStream(s->sol[l], s->lane[l]));
    LS_CUDA(cudaEventCreateWithFlags(&s->ev_lane[l], cudaEventDisableTiming));
  }
  LS_CUDA(cudaEventCreateWithFlags(&s->ev_main, cudaEventDisableTiming));
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = s->dev;
  LS_CUDA(cudaMemPoolCreate(&s->pool, &props));
  unsigned long long keep = ~0ull;
  LS_CUDA(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  LS_CUDA(cudaEventCreate(&s->t0));
  LS_CUDA(cudaEventCreate(&s->t1));
  return LFSOLVE_OK;
}

// main stream -> every lane, and back
int fork_lanes(lfsolve *s) {
  LS_CUDA(cudaEventRecord(s->ev_main, s->stream));
  for (int l = 0; l < LANES; ++l) LS_CUDA(cudaStreamWaitEvent(s->lane[l], s->ev_main, 0));
  return LFSOLVE_OK;
}
int join_lanes(lfsolve *s) {
  for (int l = 0; l < LANES; ++l) {
    LS_CUDA(cudaEventRecord(s->ev_lane[l], s->lane[l]));
    LS_CUDA(cudaStreamWaitEvent(s->stream, s->ev_lane[l], 0));
  }
  return LFSOLVE_OK;
}

int grid_for(long long n, int threads) {
  return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 16));
}

// fronts from this many complex multiply-adds of Schur update on
// (LFSOLVE_TF32X3_MIN overrides TF32X3_MIN_MACS)
double tf32x3_min() {
  const char *e = std::getenv("LFSOLVE_TF32X3_MIN");
  return e ? std::atof(e) : TF32X3_MIN_MACS;
}

// the 3xTF32 path: complex64 only, off with LFSOLVE_TF32X3=0
template <typename T> bool use_tf32x3(lfsolve *) { return false; }
template <> bool use_tf32x3<cuComplex>(lfsolve *) {
  const char *e = std::getenv("LFSOLVE_TF32X3");
  return !(e && e[0] == '0');
}

// F22 -= L21 U12 of one complex64 front (at F, leading dimension ld, kk
// pivot rows incl. dummies, r update rows) on lane l: split both operands,
// then the two TF32 tensor-core GEMMs of the real formulation with FP32
// accumulation into F22
int schur_tf32x3(lfsolve *s, int l, cuComplex *F, int ld, int kk, int r) {
  const long long lda = ((2LL * r + 31) / 32) * 32;
  const size_t na = (size_t)lda * 4 * kk, need = (na + (size_t)4 * kk * r) * sizeof(float);
  if (s->split_bytes[l] < need) {
    LS_CUDA(cudaStreamSynchronize(s->lane[l]));
    if (s->split[l]) LS_CUDA(cudaFree(s->split[l]));
    LS_CUDA(cudaMalloc(&s->split[l], need));
    s->split_bytes[l] = need;
  }
  float *A = static_cast<float *>(s->split[l]);
  float *B = A + na;
  const int g = grid_for((long long)r * kk, 256);
  k_split_a<<<g, 256, 0, s->lane[l]>>>(r, kk, F + kk, ld, A, (int)lda, 1, 0, 0);
  LS_CUDA(cudaGetLastError());
  k_split_b<<<g, 256, 0, s->lane[l]>>>(kk, r, F + (long long)kk * ld, ld, B, 1, 0, 0);
  LS_CUDA(cudaGetLastError());
  const float mone = -1.f, one = 1.f;
  float *C = reinterpret_cast<float *>(F + kk + (long long)kk * ld);
  LS_BLAS(cublasGemmEx(s->blas[l], CUBLAS_OP_N, CUBLAS_OP_N, 2 * r, r, 4 * kk, &mone, A,
                       CUDA_R_32F, (int)lda, B, CUDA_R_32F, 4 * kk, &one, C, CUDA_R_32F, 2 * ld,
                       CUBLAS_COMPUTE_32F_FAST_TF32, CUBLAS_GEMM_DEFAULT));
  LS_BLAS(cublasGemmEx(s->blas[l], CUBLAS_OP_N, CUBLAS_OP_N, 2 * r, r, 2 * kk, &mone, A,
                       CUDA_R_32F, (int)lda, B + 2 * kk, CUDA_R_32F, 4 * kk, &one, C,
                       CUDA_R_32F, 2 * ld, CUBLAS_COMPUTE_32F_FAST_TF32, CUBLAS_GEMM_DEFAULT));
  return LFSOLVE_OK;
}

// The same for all cnt fronts of a batched depth (uniform kk x r blocks,
// front stride S entries, leading dimension ld) on the main stream, the
// split operands in the solver's pool for the duration of the call
int schur_tf32x3_batched(lfsolve *s, cuComplex *arena, long long S, int ld, int kk, int r,
                         int cnt) {
  cudaStream_t st = s->stream;
  const long long lda = ((2LL * r + 31) / 32) * 32;
  const long long na = lda * 4 * kk, nbf = 4LL * kk * r;
  float *A = nullptr;
  LS_CUDA(cudaMallocFromPoolAsync((void **)&A, sizeof(float) * (size_t)(na + nbf) * cnt, s->pool,
                                  st));
  float *B = A + na * cnt;
  const int g = grid_for((long long)r * kk * cnt, 256);
  k_split_a<<<g, 256, 0, st>>>(r, kk, arena + kk, ld, A, (int)lda, cnt, S, na);
  LS_CUDA(cudaGetLastError());
  k_split_b<<<g, 256, 0, st>>>(kk, r, arena + (long long)kk * ld, ld, B, cnt, S, nbf);
  LS_CUDA(cudaGetLastError());
  const float mone = -1.f, one = 1.f;
  float *C = reinterpret_cast<float *>(arena + kk + (long long)kk * ld);
  LS_BLAS(cublasGemmStridedBatchedEx(s->blas_main, CUBLAS_OP_N, CUBLAS_OP_N, 2 * r, r, 4 * kk,
                                     &mone, A, CUDA_R_32F, (int)lda, na, B, CUDA_R_32F, 4 * kk,
                                     nbf, &one, C, CUDA_R_32F, 2 * ld, 2 * S, cnt,
                                     CUBLAS_COMPUTE_32F_FAST_TF32, CUBLAS_GEMM_DEFAULT));
  LS_BLAS(cublasGemmStridedBatchedEx(s->blas_main, CUBLAS_OP_N, CUBLAS_OP_N, 2 * r, r, 2 * kk,
                                     &mone, A, CUDA_R_32F, (int)lda, na, B + 2 * kk, CUDA_R_32F,
                                     4 * kk, nbf, &one, C, CUDA_R_32F, 2 * ld, 2 * S, cnt,
                                     CUBLAS_COMPUTE_32F_FAST_TF32, CUBLAS_GEMM_DEFAULT));
  LS_CUDA(cudaFreeAsync(A, st));
  return LFSOLVE_OK;
}

template <typename T>
int factor_impl(lfsolve *s, const double2 *vals) {
  Plan &P = s->P;
  cudaStream_t st = s->stream;
  const int D = P.max_depth + 1;
  // LFSOLVE_PROFILE set: per-depth device times printed after the call
  const bool prof = std::getenv("LFSOLVE_PROFILE") != nullptr;
  std::vector<cudaEvent_t> evs;
  if (prof) {
    evs.resize(2 * D);
    for (auto &e : evs) LS_CUDA(cudaEventCreate(&e));
  }
  T *fac = static_cast<T *>(s->d_fac);
  std::vector<T *> arena(D, nullptr);
  const T one = CT<T>::mk(1.0, 0.0), mone = CT<T>::mk(-1.0, 0.0);
  for (int d = D - 1; d >= 0; --d) {
    if (prof) LS_CUDA(cudaEventRecord(evs[2 * d], st));
    const size_t bytes = (size_t)P.arena_size[d] * sizeof(T);
    LS_CUDA(cudaMallocFromPoolAsync((void **)&arena[d], std::max<size_t>(bytes, 256), s->pool, st));
    LS_CUDA(cudaMemsetAsync(arena[d], 0, bytes, st));
    const long long na = (long long)P.asm_src[d].size();
    if (na > 0) {
      k_assemble<T><<<grid_for(na, 256), 256, 0, st>>>(na, s->d_asm_src[d], s->d_asm_dst[d], vals,
                                                       arena[d]);
      LS_CUDA(cudaGetLastError());
    }
    if (d + 1 < D) {
      for (int q = 0; q < 2; ++q)
        if (s->n_ea[q][d] > 0) {
          k_extend_add<T><<<s->n_ea[q][d], 256, 0, st>>>(s->d_ea[q][d], s->d_nodes, s->d_rel_fac,
                                                         arena[d + 1], arena[d]);
          LS_CUDA(cudaGetLastError());
        }
      LS_CUDA(cudaFreeAsync(arena[d + 1], st));
      arena[d + 1] = nullptr;
    }
    if (P.batched[d]) {
      // the whole depth at once on the uniform padded layout
      const int cnt = (int)P.by_depth[d].size();
      const int kp = P.kpad[d], rp = P.rpad[d], ld = kp + rp;
      const long long S = P.stride[d];
      k_dummy_diag<T><<<cnt, 128, 0, st>>>(s->d_all[d], s->d_nodes, arena[d]);
      LS_CUDA(cudaGetLastError());
      T **p11 = reinterpret_cast<T **>(s->d_ptrs);
      T **p12 = p11 + cnt, **p21 = p12 + cnt;
      k_make_ptrs<T><<<(cnt + 127) / 128, 128, 0, st>>>(cnt, arena[d], S, kp, ld, p11, p12, p21);
      LS_CUDA(cudaGetLastError());
      LS_BLAS(getrf_batched(s->blas_main, kp, p11, ld, s->d_bpiv, s->d_binf, cnt));
      k_take_pivots<<<cnt, 128, 0, st>>>(s->d_all[d], s->d_nodes, kp, s->d_bpiv, s->d_binf,
                                         s->d_ipiv, s->d_info);
      LS_CUDA(cudaGetLastError());
      if (rp > 0) {
        if (s->n_sw[d] > 0) {
          k_swap_cols_batched<T><<<s->n_sw[d], 32, 0, st>>>(s->d_sw[d], s->d_nodes, s->d_ipiv,
                                                            arena[d]);
          LS_CUDA(cudaGetLastError());
        }
        LS_BLAS(trsm_batched(s->blas_main, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                             CUBLAS_DIAG_UNIT, kp, rp, &one, p11, ld, p12, ld, cnt));
        LS_BLAS(trsm_batched(s->blas_main, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                             CUBLAS_DIAG_NON_UNIT, rp, kp, &one, p11, ld, p21, ld, cnt));
        if (use_tf32x3<T>(s) && (double)rp * rp * kp * cnt >= tf32x3_min()) {
          int rc3 = schur_tf32x3_batched(s, reinterpret_cast<cuComplex *>(arena[d]), S, ld, kp, rp,
                                         cnt);
          if (rc3) return rc3;
        } else {
          LS_BLAS(gemm_sb(s->blas_main, rp, rp, kp, &mone, arena[d] + kp, ld, S,
                          arena[d] + (long long)kp * ld, ld, S, &one,
                          arena[d] + kp + (long long)kp * ld, ld, S, cnt));
        }
      }
      if (s->n_co[d] > 0) {
        k_copy_out<T><<<s->n_co[d], 256, 0, st>>>(s->d_co[d], s->d_nodes, arena[d], fac);
        LS_CUDA(cudaGetLastError());
      }
      if (prof) LS_CUDA(cudaEventRecord(evs[2 * d + 1], st));
      continue;
    }
    // workspace and pivot scratch for the largest front of the depth
    int lw_max = 0, kk_max = 0;
    for (int id : P.by_depth[d]) {
      const Node &N = P.nodes[id];
      if (N.k == 0) continue;
      int lw = 0;
      LS_BLAS(getrf_buf(s->sol[0], N.roff, N.roff, arena[d] + N.arena_off, N.ld, &lw));
      lw_max = std::max(lw_max, lw);
      kk_max = std::max(kk_max, N.roff);
    }
    for (int l = 0; l < LANES; ++l) {
      if (s->work_bytes[l] < (size_t)lw_max * sizeof(T)) {
        LS_CUDA(cudaStreamSynchronize(st));
        if (s->work[l]) LS_CUDA(cudaFree(s->work[l]));
        s->work_bytes[l] = (size_t)lw_max * sizeof(T);
        LS_CUDA(cudaMalloc(&s->work[l], s->work_bytes[l]));
      }
      if (s->lpiv_n[l] < kk_max) {
        LS_CUDA(cudaStreamSynchronize(st));
        if (s->lpiv[l]) LS_CUDA(cudaFree(s->lpiv[l]));
        s->lpiv_n[l] = kk_max;
        LS_CUDA(cudaMalloc((void **)&s->lpiv[l], sizeof(int) * kk_max));
      }
    }
    const int cnt = (int)P.by_depth[d].size();
    k_dummy_diag<T><<<cnt, 128, 0, st>>>(s->d_all[d], s->d_nodes, arena[d]);
    LS_CUDA(cudaGetLastError());
    int rc = fork_lanes(s);
    if (rc) return rc;
    // largest fronts first, spread over the lanes
    std::vector<int> order(P.by_depth[d]);
    std::sort(order.begin(), order.end(),
              [&](int a, int b) { return P.nodes[a].m > P.nodes[b].m; });
    int li = 0;
    for (int id : order) {
      const Node &N = P.nodes[id];
      if (N.k == 0) continue;
      const int l = li++ % LANES;
      T *F = arena[d] + N.arena_off;
      const int k = N.k, r = N.m - N.k, kk = N.roff, ld = N.ld;
      // P F11 = L11 U11 (library getrf on the kk x kk block: the k real
      // pivots, then dummy identity pivots that never swap), the real swaps
      // on F12, U12 = L11^-1 P F12, L21 = F21 U11^-1, F22 -= L21 U12
      LS_BLAS(getrf(s->sol[l], kk, kk, F, ld, static_cast<T *>(s->work[l]), s->lpiv[l],
                    s->d_info + id));
      LS_CUDA(cudaMemcpyAsync(s->d_ipiv + N.p0, s->lpiv[l], sizeof(int) * k,
                              cudaMemcpyDeviceToDevice, s->lane[l]));
      if (r > 0) {
        if (k <= perm_smem_max<T>()) {
          k_ipiv_to_perm_one<<<1, 256, 0, s->lane[l]>>>(k, s->d_ipiv + N.p0, s->lpiv[l]);
          k_perm_cols<T><<<r, 256, (size_t)k * sizeof(T), s->lane[l]>>>(
              k, s->lpiv[l], F + (long long)kk * ld, ld);
        } else {
          k_swap_cols<T><<<(r + 127) / 128, 128, 0, s->lane[l]>>>(k, r, s->d_ipiv + N.p0,
                                                                  F + (long long)kk * ld, ld);
        }
        LS_CUDA(cudaGetLastError());
        LS_BLAS(trsm(s->blas[l], CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                     CUBLAS_DIAG_UNIT, kk, r, &one, F, ld, F + (long long)kk * ld, ld));
        LS_BLAS(trsm(s->blas[l], CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                     CUBLAS_DIAG_NON_UNIT, r, kk, &one, F, ld, F + kk, ld));
        if (use_tf32x3<T>(s) && (double)r * r * kk >= tf32x3_min()) {
          int rc3 = schur_tf32x3(s, l, reinterpret_cast<cuComplex *>(F), ld, kk, r);
          if (rc3) return rc3;
        } else {
          LS_BLAS(gemm(s->blas[l], CUBLAS_OP_N, CUBLAS_OP_N, r, r, kk, &mone, F + kk, ld,
                       F + (long long)kk * ld, ld, &one, F + kk + (long long)kk * ld, ld));
        }
      }
    }
    if ((rc = join_lanes(s))) return rc;
    if (s->n_co[d] > 0) {
      k_copy_out<T><<<s->n_co[d], 256, 0, st>>>(s->d_co[d], s->d_nodes, arena[d], fac);
      LS_CUDA(cudaGetLastError());
    }
    if (prof) LS_CUDA(cudaEventRecord(evs[2 * d + 1], st));
  }
  LS_CUDA(cudaFreeAsync(arena[0], st));
  if (prof) {
    LS_CUDA(cudaStreamSynchronize(st));
    for (int d = D - 1; d >= 0; --d) {
      float ms = 0.f;
      LS_CUDA(cudaEventElapsedTime(&ms, evs[2 * d], evs[2 * d + 1]));
      double fl = 0.0;
      int mmax = 0;
      for (int id : P.by_depth[d]) {
        const Node &N = P.nodes[id];
        const double k = N.k, r = N.m - N.k;
        fl += 8.0 * (k * k * k / 3.0 + k * k * r + k * r * r);
        mmax = std::max(mmax, N.m);
      }
      std::printf("lfsolve profile: depth %2d fronts %5zu max m %5d  %8.2f ms  %7.2f TFLOP/s\n", d,
                  P.by_depth[d].size(), mmax, ms, fl / (ms * 1e-3) / 1e12);
    }
    std::fflush(stdout);
    for (auto &e : evs) cudaEventDestroy(e);
  }
  return LFSOLVE_OK;
}

size_t small_fwd_smem(int m, int nrhs, size_t es) { return (size_t)m * nrhs * es; }

// one pass of at most MAX_NRHS_PASS columns: b (n x nr, ld n, precision T,
// original numbering) -> x (same layout)
template <typename T>
int solve_pass(lfsolve *s, int nr, const T *b, T *x, int trans) {
  Plan &P = s->P;
  cudaStream_t st = s->stream;
  const int D = P.max_depth + 1;
  const T *fac = static_cast<const T *>(s->d_fac);
  T *V = static_cast<T *>(s->d_V);
  const long long VR = P.vec_rows;
  const T one = CT<T>::mk(1.0, 0.0), mone = CT<T>::mk(-1.0, 0.0);
  const int n = P.n;
  // LFSOLVE_PROFILE set: per-depth device times of both sweeps
  const bool prof = std::getenv("LFSOLVE_PROFILE") != nullptr;
  std::vector<cudaEvent_t> evs;
  if (prof) {
    evs.resize(4 * D);
    for (auto &e : evs) LS_CUDA(cudaEventCreate(&e));
  }
  // forward, deepest level first
  for (int d = D - 1; d >= 0; --d) {
    if (prof) LS_CUDA(cudaEventRecord(evs[4 * d], st));
    const int cnt = (int)P.by_depth[d].size();
    k_gather_rhs<T><<<cnt, 256, 0, st>>>(s->d_all[d], s->d_nodes, s->d_child, s->d_rel,
                                         s->d_perm, b, n, V, VR, nr);
    LS_CUDA(cudaGetLastError());
    if (s->n_small[d] > 0) {
      int mmax = 0;
      for (int id : P.by_depth[d])
        if (is_small(P.nodes[id])) mmax = std::max(mmax, P.nodes[id].m);
      const size_t sm = small_fwd_smem(mmax, nr, sizeof(T));
      if (trans) {
        LS_CUDA(cudaFuncSetAttribute(k_fwd_small<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_fwd_small<T, 1><<<s->n_small[d], SOLVE_THREADS, sm, st>>>(s->d_small[d], s->d_nodes, fac,
                                                                    s->d_ipiv, V, VR, nr);
      } else {
        LS_CUDA(cudaFuncSetAttribute(k_fwd_small<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_fwd_small<T, 0><<<s->n_small[d], SOLVE_THREADS, sm, st>>>(s->d_small[d], s->d_nodes, fac,
                                                                    s->d_ipiv, V, VR, nr);
      }
      LS_CUDA(cudaGetLastError());
    }
    // large fronts: library calls, the fronts of the depth spread over the
    // lanes (independent vector blocks)
    if (!s->big[d].empty()) {
      int rc = fork_lanes(s);
      if (rc) return rc;
      int li = 0;
      for (int id : s->big[d]) {
        const Node &N = P.nodes[id];
        const int m = N.m, k = N.k, r = m - k;
        if (k == 0) continue;  // the gathered block is its update already
        const int l = li++ % LANES;
        cublasHandle_t bh = s->blas[l];
        T *v = V + N.vec_off;
        const T *Pf = fac + N.fac_off;
        const T *U12 = Pf + (long long)m * k;
        if (!trans) {
          if (k <= perm_smem_max<T>())
            k_perm_pivots<T, 0><<<nr, 1024, (size_t)k * sizeof(T), s->lane[l]>>>(
                k, s->d_pperm + N.p0, v, (int)VR);
          else
            k_laswp<T, 0><<<1, 32, 0, s->lane[l]>>>(k, s->d_ipiv + N.p0, v, (int)VR, nr);
          LS_CUDA(cudaGetLastError());
          LS_BLAS(trsm(bh, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                       CUBLAS_DIAG_UNIT, k, nr, &one, Pf, m, v, (int)VR));
          if (r > 0)
            LS_BLAS(gemm(bh, CUBLAS_OP_N, CUBLAS_OP_N, r, nr, k, &mone, Pf + k, m, v, (int)VR,
                         &one, v + k, (int)VR));
        } else {
          LS_BLAS(trsm(bh, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T,
                       CUBLAS_DIAG_NON_UNIT, k, nr, &one, Pf, m, v, (int)VR));
          if (r > 0)
            LS_BLAS(gemm(bh, CUBLAS_OP_T, CUBLAS_OP_N, r, nr, k, &mone, U12, k, v, (int)VR,
                         &one, v + k, (int)VR));
        }
      }
      if ((rc = join_lanes(s))) return rc;
    }
    if (prof) LS_CUDA(cudaEventRecord(evs[4 * d + 1], st));
  }
  // essential rows
  if (P.n_ess > 0) {
    k_ess_copy<T><<<grid_for(P.n_ess, 256), 256, 0, st>>>(P.n_ess, s->d_ess, b, n, x, n, nr);
    LS_CUDA(cudaGetLastError());
  }
  // backward, root first
  for (int d = 0; d < D; ++d) {
    if (prof) LS_CUDA(cudaEventRecord(evs[4 * d + 2], st));
    if (s->n_small[d] > 0) {
      int need = 0;  // rows of the largest (2 k + r) shared block
      for (int id : P.by_depth[d]) {
        const Node &N = P.nodes[id];
        if (is_small(N)) need = std::max(need, 2 * N.k + (N.m - N.k));
      }
      const size_t sm = (size_t)need * nr * sizeof(T);
      if (trans) {
        LS_CUDA(cudaFuncSetAttribute(k_bwd_small<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_bwd_small<T, 1><<<s->n_small[d], SOLVE_THREADS, sm, st>>>(
            s->d_small[d], s->d_nodes, fac, s->d_ipiv, s->d_perm, s->d_rorig, V, VR, x, n, nr);
      } else {
        LS_CUDA(cudaFuncSetAttribute(k_bwd_small<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_bwd_small<T, 0><<<s->n_small[d], SOLVE_THREADS, sm, st>>>(
            s->d_small[d], s->d_nodes, fac, s->d_ipiv, s->d_perm, s->d_rorig, V, VR, x, n, nr);
      }
      LS_CUDA(cudaGetLastError());
    }
    if (!s->big[d].empty()) {
      int rc = fork_lanes(s);
      if (rc) return rc;
      int li = 0;
      for (int id : s->big[d]) {
        const Node &N = P.nodes[id];
        const int m = N.m, k = N.k, r = m - k;
        if (k == 0) continue;
        const int l = li++ % LANES;
        cublasHandle_t bh = s->blas[l];
        cudaStream_t ls = s->lane[l];
        T *v = V + N.vec_off;
        const T *Pf = fac + N.fac_off;
        const T *U12 = Pf + (long long)m * k;
        T *xr = static_cast<T *>(s->d_xr) + (size_t)l * s->xr_lane;  // this lane's scratch
        if (r > 0) {
          k_gather_rows<T><<<grid_for(r, 256), 256, 0, ls>>>(r, s->d_rorig + N.r_off, x, n, xr, nr);
          LS_CUDA(cudaGetLastError());
        }
        if (!trans) {
          if (r > 0)
            LS_BLAS(gemm(bh, CUBLAS_OP_N, CUBLAS_OP_N, k, nr, r, &mone, U12, k, xr, r, &one, v,
                         (int)VR));
          LS_BLAS(trsm(bh, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                       CUBLAS_DIAG_NON_UNIT, k, nr, &one, Pf, m, v, (int)VR));
        } else {
          if (r > 0)
            LS_BLAS(gemm(bh, CUBLAS_OP_T, CUBLAS_OP_N, k, nr, r, &mone, Pf + k, m, xr, r, &one, v,
                         (int)VR));
          LS_BLAS(trsm(bh, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T,
                       CUBLAS_DIAG_UNIT, k, nr, &one, Pf, m, v, (int)VR));
          if (k <= perm_smem_max<T>())
            k_perm_pivots<T, 1><<<nr, 1024, (size_t)k * sizeof(T), ls>>>(
                k, s->d_pperm + N.p0, v, (int)VR);
          else
            k_laswp<T, 1><<<1, 32, 0, ls>>>(k, s->d_ipiv + N.p0, v, (int)VR, nr);
          LS_CUDA(cudaGetLastError());
        }
        k_scatter_pivots<T><<<grid_for(k, 256), 256, 0, ls>>>(k, s->d_perm + N.p0, v, VR, x, n, nr);
        LS_CUDA(cudaGetLastError());
      }
      if ((rc = join_lanes(s))) return rc;
    }
    if (prof) LS_CUDA(cudaEventRecord(evs[4 * d + 3], st));
  }
  if (prof) {
    LS_CUDA(cudaStreamSynchronize(st));
    for (int d = D - 1; d >= 0; --d) {
      float f = 0.f, b = 0.f;
      LS_CUDA(cudaEventElapsedTime(&f, evs[4 * d], evs[4 * d + 1]));
      LS_CUDA(cudaEventElapsedTime(&b, evs[4 * d + 2], evs[4 * d + 3]));
      std::printf("lfsolve solve profile (%s, %d rhs): depth %2d fronts %5zu (%zu large)  "
                  "forward %7.3f ms  backward %7.3f ms\n", trans ? "A^T" : "A", nr, d,
                  P.by_depth[d].size(), s->big[d].size(), f, b);
    }
    std::fflush(stdout);
    for (auto &e : evs) cudaEventDestroy(e);
  }
  return LFSOLVE_OK;
}

int ensure_solve_scratch(lfsolve *s, size_t es) {
  Plan &P = s->P;
  const size_t V = (size_t)P.vec_rows * MAX_NRHS_PASS * es;
  if (s->V_bytes < V) {
    if (s->d_V) LS_CUDA(cudaFree(s->d_V));
    LS_CUDA(cudaMalloc(&s->d_V, V));
    s->V_bytes = V;
  }
  size_t rmax = 1;
  for (const Node &N : P.nodes) rmax = std::max(rmax, (size_t)(N.m - N.k));
  s->xr_lane = rmax * MAX_NRHS_PASS;
  const size_t xr = s->xr_lane * LANES * es;
  if (s->xr_bytes < xr) {
    if (s->d_xr) LS_CUDA(cudaFree(s->d_xr));
    LS_CUDA(cudaMalloc(&s->d_xr, xr));
    s->xr_bytes = xr;
  }
  const size_t bw = (size_t)P.n * 2 * MAX_NRHS_PASS * es;  // b and x in the factor precision
  if (s->bw_bytes < bw) {
    if (s->d_bw) LS_CUDA(cudaFree(s->d_bw));
    LS_CUDA(cudaMalloc(&s->d_bw, bw));
    s->bw_bytes = bw;
  }
  return LFSOLVE_OK;
}

// complex128 in / out, any nrhs, optional per-column scale of the input
// (the output is scaled back): x = A_f^-1 (b * s) / s, accumulate: x += ...
template <typename T>
int solve_any(lfsolve *s, int nrhs, const double2 *b, double2 *x, int trans,
              const double *d_scale, int accumulate) {
  int rc = ensure_solve_scratch(s, sizeof(T));
  if (rc) return rc;
  const int n = s->P.n;
  T *bw = static_cast<T *>(s->d_bw);
  T *xw = bw + (size_t)n * MAX_NRHS_PASS;
  cudaStream_t st = s->stream;
  for (int c0 = 0; c0 < nrhs; c0 += MAX_NRHS_PASS) {
    const int nr = std::min(MAX_NRHS_PASS, nrhs - c0);
    k_to_prec<T><<<grid_for((long long)n * nr, 256), 256, 0, st>>>(
        n, nr, b + (size_t)c0 * n, d_scale ? d_scale + c0 : nullptr, bw);
    LS_CUDA(cudaGetLastError());
    if ((rc = solve_pass<T>(s, nr, bw, xw, trans))) return rc;
    if (d_scale) {
      // the scale was applied to b; undo it on x: pass 1 / scale
      k_from_prec<T><<<grid_for((long long)n * nr, 256), 256, 0, st>>>(
          n, nr, xw, d_scale + nrhs + c0, x + (size_t)c0 * n, accumulate);
    } else {
      k_from_prec<T><<<grid_for((long long)n * nr, 256), 256, 0, st>>>(
          n, nr, xw, nullptr, x + (size_t)c0 * n, accumulate);
    }
    LS_CUDA(cudaGetLastError());
  }
  return LFSOLVE_OK;
}

int solve_dispatch(lfsolve *s, int nrhs, const double2 *b, double2 *x, int trans,
                   const double *d_scale, int accumulate) {
  return s->prec == LFSOLVE_C64 ? solve_any<cuComplex>(s, nrhs, b, x, trans, d_scale, accumulate)
                                : solve_any<cuDoubleComplex>(s, nrhs, b, x, trans, d_scale, accumulate);
}

// GMRES-IR for one column: restarted GMRES(m) on A x = b in FP64 (complex128
// vectors, modified Gram-Schmidt Arnoldi, complex Givens rotations), right
// preconditioned by the factors (M^-1 v: one triangular solve of the
// factorization's precision), from the current x.  The Krylov basis, the
// Hessenberg solve and the update x += M^-1 (V y) follow the standard
// algorithm (Saad and Schultz 1986; with a low-precision preconditioner,
// Carson and Higham's GMRES-based iterative refinement, 2017-2018).  *iters
// counts the Arnoldi steps; *rel is the final true relative residual.
int gmres_column(lfsolve *s, const int *d_I, const int *d_J, const double2 *vals, const int *tp,
                 const double2 *b, double2 *x, int trans, double tol, int max_steps, int m,
                 double *rel, int *iters) {
  using cd = std::complex<double>;
  const int n = s->P.n;
  cudaStream_t st = s->stream;
  int rc = ensure_lanes(s);
  if (rc) return rc;
  cublasHandle_t hb = s->blas_main;
  LS_BLAS(cublasSetPointerMode(hb, CUBLAS_POINTER_MODE_HOST));
  double2 *V = nullptr, *z = nullptr, *w = nullptr;
  LS_CUDA(cudaMalloc((void **)&V, sizeof(double2) * (size_t)n * (m + 1)));
  LS_CUDA(cudaMalloc((void **)&z, sizeof(double2) * (size_t)n));
  LS_CUDA(cudaMalloc((void **)&w, sizeof(double2) * (size_t)n));
  struct Free {
    void *a, *b, *c;
    ~Free() { cudaFree(a); cudaFree(b); cudaFree(c); }
  } guard{V, z, w};
  auto spmv = [&](const double2 *in, double2 *out) -> int {
    k_spmv<<<(n + 7) / 8, 256, 0, st>>>(n, d_I, d_J, vals, tp, in, out);
    LS_CUDA(cudaGetLastError());
    return LFSOLVE_OK;
  };
  auto zc = [](cuDoubleComplex v) { return cd(v.x, v.y); };
  auto cz = [](cd v) { return make_cuDoubleComplex(v.real(), v.imag()); };
  double bn = 0.0;
  LS_BLAS(cublasDznrm2(hb, n, reinterpret_cast<const cuDoubleComplex *>(b), 1, &bn));
  if (bn == 0.0) bn = 1.0;
  std::vector<cd> H((size_t)(m + 1) * m), g(m + 1), sn(m), y(m);
  std::vector<double> cs(m);
  int steps = 0;
  *rel = 1.0;
  while (true) {
    // r = b - A x into V[0]
    if ((rc = spmv(x, w))) return rc;
    LS_CUDA(cudaMemcpyAsync(V, b, sizeof(double2) * n, cudaMemcpyDeviceToDevice, st));
    const cuDoubleComplex mone = make_cuDoubleComplex(-1.0, 0.0);
    auto *V0 = reinterpret_cast<cuDoubleComplex *>(V);
    LS_BLAS(cublasZaxpy(hb, n, &mone, reinterpret_cast<const cuDoubleComplex *>(w), 1, V0, 1));
    double beta = 0.0;
    LS_BLAS(cublasDznrm2(hb, n, V0, 1, &beta));
    *rel = beta / bn;
    if (*rel <= tol || steps >= max_steps || beta == 0.0) break;
    const double ib = 1.0 / beta;
    LS_BLAS(cublasZdscal(hb, n, &ib, V0, 1));
    std::fill(g.begin(), g.end(), cd(0.0));
    g[0] = beta;
    int k = 0;
    for (; k < m && steps < max_steps; ++k) {
      auto *Vk = reinterpret_cast<cuDoubleComplex *>(V + (size_t)k * n);
      // w = A M^-1 v_k
      if ((rc = solve_dispatch(s, 1, reinterpret_cast<const double2 *>(Vk), z, trans, nullptr, 0)))
        return rc;
      if ((rc = spmv(z, w))) return rc;
      auto *W = reinterpret_cast<cuDoubleComplex *>(w);
      for (int i = 0; i <= k; ++i) {
        auto *Vi = reinterpret_cast<cuDoubleComplex *>(V + (size_t)i * n);
        cuDoubleComplex hij;
        LS_BLAS(cublasZdotc(hb, n, Vi, 1, W, 1, &hij));
        H[(size_t)i * m + k] = zc(hij);
        const cuDoubleComplex neg = make_cuDoubleComplex(-hij.x, -hij.y);
        LS_BLAS(cublasZaxpy(hb, n, &neg, Vi, 1, W, 1));
      }
      double hn = 0.0;
      LS_BLAS(cublasDznrm2(hb, n, W, 1, &hn));
      H[(size_t)(k + 1) * m + k] = hn;
      if (hn > 0.0) {
        const double ih = 1.0 / hn;
        LS_CUDA(cudaMemcpyAsync(V + (size_t)(k + 1) * n, w, sizeof(double2) * n,
                                cudaMemcpyDeviceToDevice, st));
        LS_BLAS(cublasZdscal(hb, n, &ih,
                             reinterpret_cast<cuDoubleComplex *>(V + (size_t)(k + 1) * n), 1));
      }
      // earlier rotations on column k, then the one that zeroes H[k+1][k]
      for (int i = 0; i < k; ++i) {
        const cd a = H[(size_t)i * m + k], c = H[(size_t)(i + 1) * m + k];
        H[(size_t)i * m + k] = cs[i] * a + sn[i] * c;
        H[(size_t)(i + 1) * m + k] = -std::conj(sn[i]) * a + cs[i] * c;
      }
      const cd a = H[(size_t)k * m + k];
      const double bb = hn, r = std::hypot(std::abs(a), bb);
      if (std::abs(a) == 0.0) {
        cs[k] = 0.0;
        sn[k] = 1.0;
        H[(size_t)k * m + k] = bb;
      } else {
        const cd ph = a / std::abs(a);
        cs[k] = std::abs(a) / r;
        sn[k] = ph * bb / r;
        H[(size_t)k * m + k] = ph * r;
      }
      H[(size_t)(k + 1) * m + k] = 0.0;
      g[k + 1] = -std::conj(sn[k]) * g[k];
      g[k] = cs[k] * g[k];
      ++steps;
      if (std::abs(g[k + 1]) / bn <= 0.5 * tol || hn == 0.0) {
        ++k;
        break;
      }
    }
    // y = H^-1 g (upper triangular k x k), u = V y, x += M^-1 u
    for (int i = k - 1; i >= 0; --i) {
      cd t = g[i];
      for (int j = i + 1; j < k; ++j) t -= H[(size_t)i * m + j] * y[j];
      y[i] = t / H[(size_t)i * m + i];
    }
    LS_CUDA(cudaMemsetAsync(w, 0, sizeof(double2) * n, st));
    for (int i = 0; i < k; ++i) {
      const cuDoubleComplex yi = cz(y[i]);
      LS_BLAS(cublasZaxpy(hb, n, &yi, reinterpret_cast<const cuDoubleComplex *>(V + (size_t)i * n),
                          1, reinterpret_cast<cuDoubleComplex *>(w), 1));
    }
    if ((rc = solve_dispatch(s, 1, w, x, trans, nullptr, 1))) return rc;
  }
  *iters = steps;
  LS_CUDA(cudaStreamSynchronize(st));
  return LFSOLVE_OK;
}

void free_factors(lfsolve *s) {
  if (s->d_fac) cudaFree(s->d_fac);
  s->d_fac = nullptr;
  s->prec = -1;
}

}  // namespace

extern "C" {

const char *lfsolve_last_error(void) { return g_err.c_str(); }

int lfsolve_create(int gpu_id, lfsolve **out) {
  g_err.clear();
  if (!out) return fail(LFSOLVE_ERR_ARG, "NULL output pointer");
  *out = nullptr;
  lfsolve *s = new lfsolve();
  s->dev = gpu_id;
  *out = s;
  return LFSOLVE_OK;
}

int lfsolve_set_stream(lfsolve *s, void *stream) {
  if (!s) return fail(LFSOLVE_ERR_ARG, "NULL solver");
  s->stream = (cudaStream_t)stream;
  if (s->blas_main) LS_BLAS(cublasSetStream(s->blas_main, s->stream));
  return LFSOLVE_OK;
}

int lfsolve_analyze(lfsolve *s, int n, const int *I, const int *J, long long nnz, int ne, int nd,
                    const int *elem_dof, const double *centroid, const int *ess, int n_ess,
                    int leaf_elements) {
  g_err.clear();
  if (!s || !I || !J || !elem_dof || !centroid || (n_ess > 0 && !ess))
    return fail(LFSOLVE_ERR_ARG, "NULL argument");
  if (n <= 0 || ne <= 0 || nd <= 0 || nnz <= 0 || n_ess < 0)
    return fail(LFSOLVE_ERR_ARG, "sizes must be positive");
  if (nnz >= (1LL << 31)) return fail(LFSOLVE_ERR_ARG, "nnz beyond the int32 CSR contract");
  if (I[0] != 0 || I[n] != nnz) return fail(LFSOLVE_ERR_ARG, "row pointer does not span nnz");
  const auto t0 = std::chrono::steady_clock::now();
  const int leaf = leaf_elements > 0 ? leaf_elements : 32;
  const int rc = build_plan(n, I, J, nnz, ne, nd, elem_dof, centroid, ess, n_ess, leaf, s->P);
  if (rc) return rc;
  const auto t1 = std::chrono::steady_clock::now();
  s->analyzed = true;
  s->uploaded = false;
  lfsolve_stats &st = s->st;
  st = lfsolve_stats{};
  st.n = n;
  st.n_ess = s->P.n_ess;
  st.n_fronts = (int)s->P.nodes.size();
  st.depth = s->P.max_depth + 1;
  st.max_front = s->P.max_front;
  st.max_pivots = s->P.max_k;
  st.factor_entries = s->P.factor_entries;
  st.factor_flops = s->P.flops;
  st.peak_front_entries = s->P.peak_front_entries;
  st.analyze_s = std::chrono::duration<double>(t1 - t0).count();
  return LFSOLVE_OK;
}

int lfsolve_get_ordering(lfsolve *s, int *perm, int *node_of) {
  if (!s || !s->analyzed) return fail(LFSOLVE_ERR_STATE, "lfsolve_analyze has not run");
  if (perm) std::copy(s->P.perm.begin(), s->P.perm.end(), perm);
  if (node_of) std::copy(s->P.node_of.begin(), s->P.node_of.end(), node_of);
  return LFSOLVE_OK;
}

int lfsolve_get_fronts(lfsolve *s, int *parent, int *depth, int *k, int *m) {
  if (!s || !s->analyzed) return fail(LFSOLVE_ERR_STATE, "lfsolve_analyze has not run");
  const std::vector<Node> &nodes = s->P.nodes;
  for (size_t i = 0; i < nodes.size(); ++i) {
    if (parent) parent[i] = nodes[i].parent;
    if (depth) depth[i] = nodes[i].depth;
    if (k) k[i] = nodes[i].k;
    if (m) m[i] = nodes[i].m;
  }
  return LFSOLVE_OK;
}

int lfsolve_get_stats(lfsolve *s, lfsolve_stats *out) {
  if (!s || !out) return fail(LFSOLVE_ERR_ARG, "NULL argument");
  *out = s->st;
  return LFSOLVE_OK;
}

int lfsolve_factor(lfsolve *s, const void *d_vals, int prec) {
  g_err.clear();
  if (!s || !d_vals) return fail(LFSOLVE_ERR_ARG, "NULL argument");
  if (!s->analyzed) return fail(LFSOLVE_ERR_STATE, "lfsolve_analyze has not run");
  if (prec != LFSOLVE_C64 && prec != LFSOLVE_C128) return fail(LFSOLVE_ERR_ARG, "unknown precision %d", prec);
  LS_CUDA(cudaSetDevice(s->dev));
  int rc = ensure_lanes(s);
  if (rc) return rc;
  if ((rc = ensure_uploaded(s))) return rc;
  const size_t es = prec == LFSOLVE_C64 ? sizeof(cuComplex) : sizeof(cuDoubleComplex);
  if (s->prec != prec) {
    free_factors(s);
    LS_CUDA(cudaMalloc(&s->d_fac, std::max<size_t>((size_t)s->P.factor_entries * es, 256)));
    s->prec = prec;
  }
  if (!s->d_ipiv) LS_CUDA(cudaMalloc((void **)&s->d_ipiv, sizeof(int) * std::max(1, s->P.nn)));
  if (!s->d_info) LS_CUDA(cudaMalloc((void **)&s->d_info, sizeof(int) * s->P.nodes.size()));
  LS_CUDA(cudaMemsetAsync(s->d_info, 0, sizeof(int) * s->P.nodes.size(), s->stream));
  LS_CUDA(cudaEventRecord(s->t0, s->stream));
  rc = prec == LFSOLVE_C64 ? factor_impl<cuComplex>(s, static_cast<const double2 *>(d_vals))
                           : factor_impl<cuDoubleComplex>(s, static_cast<const double2 *>(d_vals));
  if (rc) return rc;
  // the fronts' pivot permutations for the solves' row interchanges
  if (!s->d_pperm) LS_CUDA(cudaMalloc((void **)&s->d_pperm, sizeof(int) * std::max(1, s->P.nn)));
  k_ipiv_to_perm<<<(unsigned)s->P.nodes.size(), 128, 0, s->stream>>>(s->d_nodes, s->d_ipiv,
                                                                      s->d_pperm);
  LS_CUDA(cudaGetLastError());
  LS_CUDA(cudaEventRecord(s->t1, s->stream));
  LS_CUDA(cudaStreamSynchronize(s->stream));
  LS_CUDA(cudaEventElapsedTime(&s->st.factor_ms, s->t0, s->t1));
  std::vector<int> info(s->P.nodes.size());
  LS_CUDA(cudaMemcpy(info.data(), s->d_info, sizeof(int) * info.size(), cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < info.size(); ++i)
    if (info[i] != 0)
      return fail(LFSOLVE_ERR_SINGULAR, "front %zu: zero pivot at position %d of %d", i, info[i],
                  s->P.nodes[i].k);
  return LFSOLVE_OK;
}

int lfsolve_solve(lfsolve *s, int nrhs, const void *d_b, void *d_x, int transpose) {
  g_err.clear();
  if (!s || !d_b || !d_x || nrhs <= 0) return fail(LFSOLVE_ERR_ARG, "bad arguments");
  if (!s->d_fac) return fail(LFSOLVE_ERR_STATE, "lfsolve_factor has not run");
  LS_CUDA(cudaSetDevice(s->dev));
  LS_CUDA(cudaEventRecord(s->t0, s->stream));
  int rc = solve_dispatch(s, nrhs, static_cast<const double2 *>(d_b), static_cast<double2 *>(d_x),
                          transpose != 0, nullptr, 0);
  if (rc) return rc;
  LS_CUDA(cudaEventRecord(s->t1, s->stream));
  LS_CUDA(cudaStreamSynchronize(s->stream));
  LS_CUDA(cudaEventElapsedTime(&s->st.solve_ms, s->t0, s->t1));
  return LFSOLVE_OK;
}

int lfsolve_solve_refined(lfsolve *s, const int *d_I, const int *d_J, const void *d_vals,
                          int nrhs, const void *d_b, void *d_x, int transpose, double tol,
                          int max_iter, double *rel_out, int *iters_out) {
  g_err.clear();
  if (!s || !d_I || !d_J || !d_vals || !d_b || !d_x || nrhs <= 0)
    return fail(LFSOLVE_ERR_ARG, "bad arguments");
  if (!s->d_fac) return fail(LFSOLVE_ERR_STATE, "lfsolve_factor has not run");
  if (d_b == d_x) return fail(LFSOLVE_ERR_ARG, "the refined solve needs x and b apart");
  LS_CUDA(cudaSetDevice(s->dev));
  const int n = s->P.n;
  cudaStream_t st = s->stream;
  const size_t rb = (size_t)n * nrhs * sizeof(double2);
  if (s->r_bytes < rb) {
    if (s->d_r) LS_CUDA(cudaFree(s->d_r));
    LS_CUDA(cudaMalloc((void **)&s->d_r, rb));
    s->r_bytes = rb;
  }
  const int wpb = 8;
  const int nblk = (n + wpb - 1) / wpb;
  const size_t pb = (size_t)3 * nblk * nrhs * sizeof(double) + (size_t)3 * nrhs * sizeof(double);
  if (s->part_bytes < pb) {
    if (s->d_part) LS_CUDA(cudaFree(s->d_part));
    LS_CUDA(cudaMalloc((void **)&s->d_part, pb));
    s->part_bytes = pb;
    if (s->d_scale) LS_CUDA(cudaFree(s->d_scale));
    LS_CUDA(cudaMalloc((void **)&s->d_scale, sizeof(double) * 2 * nrhs));
  }
  double *sums = s->d_part + (size_t)3 * nblk * nrhs;
  const double2 *b = static_cast<const double2 *>(d_b);
  double2 *x = static_cast<double2 *>(d_x);
  const int *tp = transpose ? s->d_tpos : nullptr;
  std::vector<double> h(3 * nrhs), sc(2 * nrhs);
  auto residual = [&](double *worst) -> int {
    k_resid<<<dim3(nblk, nrhs), wpb * 32, 0, st>>>(n, nrhs, d_I, d_J,
                                                   static_cast<const double2 *>(d_vals), tp, x, b,
                                                   s->d_r, s->d_part);
    LS_CUDA(cudaGetLastError());
    k_resid_sum<<<nrhs, 1024, 0, st>>>(nblk, nrhs, s->d_part, sums);
    LS_CUDA(cudaGetLastError());
    LS_CUDA(cudaMemcpyAsync(h.data(), sums, sizeof(double) * 3 * nrhs, cudaMemcpyDeviceToHost, st));
    LS_CUDA(cudaStreamSynchronize(st));
    *worst = 0.0;
    for (int c = 0; c < nrhs; ++c) {
      const double rel = h[3 * c + 1] > 0 ? std::sqrt(h[3 * c] / h[3 * c + 1]) : std::sqrt(h[3 * c]);
      if (rel_out) rel_out[c] = rel;
      *worst = std::max(*worst, rel);
      // the correction's right-hand side is scaled to a unit max entry
      const double mx = h[3 * c + 2] > 0 ? h[3 * c + 2] : 1.0;
      sc[c] = 1.0 / mx;
      sc[nrhs + c] = mx;
    }
    return LFSOLVE_OK;
  };
  LS_CUDA(cudaEventRecord(s->t0, st));
  int rc = solve_dispatch(s, nrhs, b, x, transpose != 0, nullptr, 0);
  if (rc) return rc;
  double worst = 0.0;
  int it = 0, steps = 0;
  if ((rc = residual(&worst))) return rc;
  // classical refinement while it contracts; when a correction reduces the
  // worst residual by less than half (or LFSOLVE_GMRES=1 asks for it from
  // the start), GMRES-IR takes over, column by column, with up to
  // 10 max_iter Arnoldi steps (LFSOLVE_GMRES=0: never)
  const char *ge = std::getenv("LFSOLVE_GMRES");
  bool gmres = ge && ge[0] == '1';
  const bool no_gmres = ge && ge[0] == '0';  // classical refinement only
  // (comparisons written so that a NaN residual counts as not converged)
  while (!gmres && !(worst <= tol) && it < max_iter) {
    LS_CUDA(cudaMemcpyAsync(s->d_scale, sc.data(), sizeof(double) * 2 * nrhs, cudaMemcpyHostToDevice, st));
    if ((rc = solve_dispatch(s, nrhs, s->d_r, x, transpose != 0, s->d_scale, 1))) return rc;
    ++it;
    const double prev = worst;
    if ((rc = residual(&worst))) return rc;
    if (!(worst <= tol) && !(worst <= 0.5 * prev) && !no_gmres) gmres = true;
  }
  if (gmres && !(worst <= tol)) {
    // a diverged refinement leaves x worse than zero: start from x = 0
    if (!(worst < 1.0)) LS_CUDA(cudaMemsetAsync(x, 0, sizeof(double2) * (size_t)n * nrhs, st));
    for (int c = 0; c < nrhs; ++c) {
      double rel = 0.0;
      int k = 0;
      if ((rc = gmres_column(s, d_I, d_J, static_cast<const double2 *>(d_vals), tp,
                             b + (size_t)c * n, x + (size_t)c * n, transpose != 0, tol,
                             10 * std::max(1, max_iter), 30, &rel, &k)))
        return rc;
      steps += k;
    }
    if ((rc = residual(&worst))) return rc;
  }
  it += steps;
  LS_CUDA(cudaEventRecord(s->t1, st));
  LS_CUDA(cudaStreamSynchronize(st));
  LS_CUDA(cudaEventElapsedTime(&s->st.solve_ms, s->t0, s->t1));
  s->st.refine_iters = it;
  s->st.refine_rel = worst;
  if (iters_out) *iters_out = it;
  if (!(worst <= tol))
    return fail(LFSOLVE_ERR_NOCONV,
                "refinement stopped at relative residual %.3e after %d corrections / GMRES steps",
                worst, it);
  return LFSOLVE_OK;
}

int lfsolve_release_factors(lfsolve *s) {
  if (!s) return fail(LFSOLVE_ERR_ARG, "NULL solver");
  cudaSetDevice(s->dev);
  free_factors(s);
  if (s->pool) {
    if (s->stream) cudaStreamSynchronize(s->stream);
    cudaMemPoolTrimTo(s->pool, 0);
  }
  return LFSOLVE_OK;
}

void lfsolve_destroy(lfsolve *s) {
  if (!s) return;
  cudaSetDevice(s->dev);
  if (s->stream) cudaStreamSynchronize(s->stream);
  free_factors(s);
  void *bufs[] = {s->d_nodes, s->d_child, s->d_rel, s->d_perm, s->d_rorig, s->d_ess, s->d_tpos,
                  s->d_ipiv, s->d_info, s->d_V, s->d_bw, s->d_xr, s->d_r, s->d_part, s->d_scale,
                  s->d_pperm};
  for (void *p : bufs)
    if (p) cudaFree(p);
  for (auto *p : s->d_asm_src) if (p) cudaFree(p);
  for (auto *p : s->d_asm_dst) if (p) cudaFree(p);
  for (int q = 0; q < 2; ++q) for (auto *p : s->d_ea[q]) if (p) cudaFree(p);
  for (auto *p : s->d_co) if (p) cudaFree(p);
  for (auto *p : s->d_small) if (p) cudaFree(p);
  for (auto *p : s->d_sw) if (p) cudaFree(p);
  if (s->d_rel_fac) cudaFree(s->d_rel_fac);
  if (s->d_ptrs) cudaFree(s->d_ptrs);
  if (s->d_bpiv) cudaFree(s->d_bpiv);
  if (s->d_binf) cudaFree(s->d_binf);
  for (auto *p : s->d_all) if (p) cudaFree(p);
  for (int l = 0; l < LANES; ++l) {
    if (s->work[l]) cudaFree(s->work[l]);
    if (s->split[l]) cudaFree(s->split[l]);
    if (s->lpiv[l]) cudaFree(s->lpiv[l]);
    if (s->blas[l]) cublasDestroy(s->blas[l]);
    if (s->sol[l]) cusolverDnDestroy(s->sol[l]);
    if (s->lane[l]) cudaStreamDestroy(s->lane[l]);
    if (s->ev_lane[l]) cudaEventDestroy(s->ev_lane[l]);
  }
  if (s->blas_main) cublasDestroy(s->blas_main);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  if (s->ev_main) cudaEventDestroy(s->ev_main);
  if (s->t0) cudaEventDestroy(s->t0);
  if (s->t1) cudaEventDestroy(s->t1);
  delete s;
}

}  // extern "C"
