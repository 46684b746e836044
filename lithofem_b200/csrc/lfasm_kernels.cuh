// Device kernels of liblfasm (sm_100a).  Included once by lfasm.cu.
//
// Element-matrix evaluation follows the reference's arithmetic
// (solver/asm_gpu.inc:70-214 and the CPU twin solver/asm_data.inc:218-370):
// physical shapes v = refv . Jinv, curls c = J . refc / detJ, weight
// w_q detJ, PML stretch s(z) per quadrature point (asm_gpu.inc:40-48) and the
// five integrator tensors.  Two device paths share that arithmetic:
//
//  * bulk elements (every quadrature point outside the PML, where s == 1
//    exactly): the integrand coefficients are constant on the element, so
//    A_e = sum_t G_e[t] S_t with 3x3 geometry coefficients G_e (from J, Jinv,
//    detJ, eps, k-parallel) and element-independent tables S_t of reference
//    quadrature sums (w_q refX_k,j refY_l,j'), evaluated with the same rules
//    and exact for these polynomial integrands;
//  * PML elements: per-quadrature-point contraction A += X_q^T (W_q X_q)
//    with X_q the (face-transformed) physical shapes and W_q the complex
//    coefficient tensors, on FP64 tensor cores (mma.sync m8n8k4 .f64).

#pragma once

#include <cstdint>

namespace lfasm_dev {

// Bounds-checked debug build (-DLFASM_BOUNDS): index checks in the gather
// record the code of the first failure in g_bounds_err and skip the access
// (never trap); the host reads the word after each synchronising call.
#ifdef LFASM_BOUNDS
__device__ int g_bounds_err;
#define LF_CHECK(cond, code) ((cond) ? true : (atomicCAS(&g_bounds_err, 0, (code)), false))
#else
#define LF_CHECK(cond, code) true
#endif
constexpr int BOUNDS_SLOT = 1;      // slot offset outside its CSR row
constexpr int BOUNDS_ELEM_ROW = 2;  // row-list entry outside the element buffer

struct dcplx {
  double re, im;
};

struct PmlParams {  // asm_gpu.inc:31-36
  double z_min, z_max, thick, order;
  double smax_bot, smax_top;
  double k0, kx, ky;
};

struct Rule {
  int nq;
  const double *ip, *w, *v, *c;
  // component-major copies, [d][q][k] with ldt (nd rounded up to 8, zero
  // padded) columns: a column pair is one aligned 16-byte load
  const double *vt, *ct;
  int ldt;
};

constexpr int REC = 28;        // doubles per bulk-element coefficient record
constexpr int NT_CC = 6;       // symmetric (j <= j') pairs
constexpr int NT_ALL = 30;     // 6 cc + 6 vv + 9 vc + 9 cv
constexpr int BULK_THREADS = 128;

__constant__ double c_tinv[24];   // 2x2 column-major blocks per orientation

__device__ __forceinline__ dcplx mk(double r, double i) { dcplx z; z.re = r; z.im = i; return z; }
__device__ __forceinline__ dcplx cmul(dcplx a, dcplx b) {
  return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__device__ __forceinline__ dcplx cinv(dcplx a) {
  const double d = a.re * a.re + a.im * a.im;
  return mk(a.re / d, -a.im / d);
}
__device__ __forceinline__ dcplx cscale(double s, dcplx a) { return mk(s * a.re, s * a.im); }
__device__ __forceinline__ dcplx cadd(dcplx a, dcplx b) { return mk(a.re + b.re, a.im + b.im); }

// PML stretch s(z) (problem_common.inc:69-90 with the per-side maximum
// precomputed as at asm_gpu.inc:310-319).
__device__ __forceinline__ dcplx pml_s(const PmlParams &p, double z) {
  double d = -1.0, smax = 0.0;
  if (z < p.z_min) { d = (p.z_min - z) / p.thick; smax = p.smax_bot; }
  else if (z > p.z_max) { d = (z - p.z_max) / p.thick; smax = p.smax_top; }
  if (d < 0.0) return mk(1.0, 0.0);
  if (d > 1.0) d = 1.0;
  return mk(1.0, smax * pow(d, p.order));
}

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ int face_of(int k, int p) {
  const int f0 = 6 * p, nf = p * (p - 1);
  if (nf == 0 || k < f0 || k >= f0 + 4 * nf) return -1;
  return (k - f0) / nf;
}

// ---------------------------------------------------------------------------
// bulk-element coefficient records (REC doubles per element)
//   [0,6)   gcc: J^T J / detJ at the symmetric pairs (00,11,22,01,02,12)
//   [6,18)  gvv: detJ Jinv (-k0^2 eps I - K K) Jinv^T, complex, same pairs
//   [18,27) gx : Jinv K J (the cross coefficients, i factored out), j*3+j'
// With these, A = Sym + i (c0 X - c1 X^T): Sym = sum gcc Scc + gvv Svv is
// symmetric and X = sum gx Rvc; the MixedVectorWeakCurl coefficient is
// J^T K Jinv^T = -(Jinv K J)^T, which turns its term into -X^T.
// ---------------------------------------------------------------------------
__global__ void k_prep_bulk(int nb, const int *__restrict__ list,
                            const double *__restrict__ J9, const double *__restrict__ Ji9,
                            const double *__restrict__ detJ, const int *__restrict__ attr,
                            const dcplx *__restrict__ eps_tab,
                            const dcplx *__restrict__ elem_eps, PmlParams pml,
                            int mask, double *__restrict__ rec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const int e = list[i];
  double J[9], Ji[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    J[t] = J9[(size_t)e * 9 + t];
    Ji[t] = Ji9[(size_t)e * 9 + t];
  }
  const double det = detJ[e];
  const dcplx eps = elem_eps ? elem_eps[e] : eps_tab[attr[e] - 1];
  double *r = rec + (size_t)i * REC;
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  const bool cc = mask & 1, ms = mask & 2, kl = mask & 16;
  const double kx = pml.kx, ky = pml.ky, k2 = pml.k0 * pml.k0;
  // K = [[0,0,ky],[0,0,-kx],[-ky,kx,0]] (fill_K, problem_common.inc:150-158)
  const double K[9] = {0.0, 0.0, ky, 0.0, 0.0, -kx, -ky, kx, 0.0};
  // -K K (real symmetric), the KLK tensor where Lambda = I
  const double mKK[9] = {ky * ky, -kx * ky, 0.0, -kx * ky, kx * kx, 0.0, 0.0, 0.0,
                         kx * kx + ky * ky};
  const double me_re = -k2 * eps.re, me_im = -k2 * eps.im;
  for (int t = 0; t < 6; ++t) {
    const int a = pa[t], b = pb[t];
    double g = 0.0;
    if (cc) g = (J[a] * J[b] + J[3 + a] * J[3 + b] + J[6 + a] * J[6 + b]) / det;
    r[t] = g;
    const double jj = Ji[a * 3 + 0] * Ji[b * 3 + 0] + Ji[a * 3 + 1] * Ji[b * 3 + 1] +
                      Ji[a * 3 + 2] * Ji[b * 3 + 2];
    double vr = 0.0, vi = 0.0;
    if (ms) { vr += me_re * jj; vi += me_im * jj; }
    if (kl) {
      double s = 0.0;
      for (int rr = 0; rr < 3; ++rr)
        for (int c2 = 0; c2 < 3; ++c2) s += Ji[a * 3 + rr] * mKK[rr * 3 + c2] * Ji[b * 3 + c2];
      vr += s;
    }
    r[6 + 2 * t] = det * vr;
    r[7 + 2 * t] = det * vi;
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double gx = 0.0;
      for (int rr = 0; rr < 3; ++rr)
        for (int c2 = 0; c2 < 3; ++c2) {
          const double k = K[rr * 3 + c2];
          if (k != 0.0) gx += Ji[a * 3 + rr] * k * J[c2 * 3 + b];
        }
      r[18 + a * 3 + b] = gx;
    }
  r[27] = 0.0;
}

// ---------------------------------------------------------------------------
// bulk element kernel.  Thread <-> (row pair I, column l >= 2I): it produces
// A(2I+a, l) and, when l >= 2I+2, the mirrored A(l, 2I+a), a = 0, 1, from NV
// table values held in registers (symmetric tables at (2I+a, l), cross
// tables at (2I+a, l) and (l, 2I+a)).  Element records are staged through
// shared memory in batches of BULK_EB.  Face transforms: the row pair is
// thread-local, the partner column / row l^1 sits in the neighbouring lane.
// MODE 0: raw local matrix (ComputeLocal); MODE 1: signs + elimination.
// ---------------------------------------------------------------------------
constexpr int BULK_EB = 8;

template <bool CROSS, int MODE>
__global__ void __launch_bounds__(BULK_THREADS, 3)
k_bulk(int nb, const int *__restrict__ list, const double *__restrict__ rec,
       const double *__restrict__ S, int nthr, int nd, int ndp, int p, int chunk, int te,
       int eliminate, int rs, int c0, int c1, const unsigned *__restrict__ fopack,
       const unsigned long long *__restrict__ signmask,
       const unsigned long long *__restrict__ essmask, dcplx *__restrict__ Ae) {
  constexpr int NV = CROSS ? 60 : 24;
  __shared__ double sg[BULK_EB * REC];
  __shared__ int se[BULK_EB];
  __shared__ unsigned sfo[BULK_EB];
  __shared__ unsigned long long ssm[BULK_EB], sem[BULK_EB];
  const int tid = threadIdx.x;
  const int f = blockIdx.y * BULK_THREADS + tid;
  const bool valid = f < nthr;
  int I = 0, l = 0;
  if (valid) {
    int rem = f;
    while (rem >= ndp - 2 * I) { rem -= ndp - 2 * I; ++I; }
    l = 2 * I + rem;
  }
  const bool mirror = valid && l >= 2 * I + 2;
  const int r0 = 2 * I, r1 = 2 * I + 1;
  double sv[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) sv[v] = valid ? S[(size_t)v * nthr + f] : 0.0;
  const int frow = valid ? face_of(r0, p) : -1;
  const int fcol = valid ? face_of(l & ~1, p) : -1;
  const int cp = l & 1;
  const double fc0 = c0 ? 1.0 : 0.0, fc1 = c1 ? 1.0 : 0.0;
  const int i0 = blockIdx.x * chunk;
  const int i1 = min(nb, i0 + chunk);
  // records of the next batch are loaded into registers while the current
  // batch is computed (BULK_EB * REC <= 2 * BULK_THREADS)
  constexpr int PF = (BULK_EB * REC + BULK_THREADS - 1) / BULK_THREADS;
  double pf[PF];
  int pfe = -1;
  unsigned pfo = 0u;
  unsigned long long psm = 0ull, pem = 0ull;
  auto prefetch = [&](int ib) {
    const int nbat = min(BULK_EB, i1 - ib);
#pragma unroll
    for (int u = 0; u < PF; ++u) {
      const int j = tid + u * BULK_THREADS;
      pf[u] = (ib < i1 && j < nbat * REC) ? rec[(size_t)ib * REC + j] : 0.0;
    }
    pfe = (ib < i1 && tid < nbat) ? list[ib + tid] : -1;
    if (pfe >= 0) {
      pfo = fopack[pfe];
      psm = MODE == 1 ? signmask[pfe] : 0ull;
      pem = (MODE == 1 && eliminate) ? essmask[pfe] : 0ull;
    }
  };
  prefetch(i0);
  for (int ib = i0; ib < i1; ib += BULK_EB) {
    const int nbat = min(BULK_EB, i1 - ib);
    __syncthreads();
#pragma unroll
    for (int u = 0; u < PF; ++u) {
      const int j = tid + u * BULK_THREADS;
      if (j < BULK_EB * REC) sg[j] = pf[u];
    }
    if (tid < nbat) {
      se[tid] = pfe;
      sfo[tid] = pfo;
      ssm[tid] = psm;
      sem[tid] = pem;
    }
    __syncthreads();
    prefetch(ib + BULK_EB);
    for (int b = 0; b < nbat; ++b) {
      const double *g = sg + b * REC;
      double sr0 = 0.0, si0 = 0.0, sr1 = 0.0, si1 = 0.0;
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const double gc = g[t];
        sr0 = fma(gc, sv[t], sr0);
        sr1 = fma(gc, sv[12 + t], sr1);
      }
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const double gr = g[6 + 2 * t], gi = g[7 + 2 * t];
        sr0 = fma(gr, sv[6 + t], sr0);
        si0 = fma(gi, sv[6 + t], si0);
        sr1 = fma(gr, sv[18 + t], sr1);
        si1 = fma(gi, sv[18 + t], si1);
      }
      // primary A(r0|r1, l) and mirror A(l, r0|r1)
      double pr0 = sr0, pi0 = si0, pr1 = sr1, pi1 = si1;
      double mr0 = sr0, mi0 = si0, mr1 = sr1, mi1 = si1;
      if (CROSS) {
        double x0 = 0.0, x1 = 0.0, y0 = 0.0, y1 = 0.0;
#pragma unroll
        for (int t = 0; t < 9; ++t) {
          const double gx = g[18 + t];
          x0 = fma(gx, sv[(24 + t) % NV], x0);
          x1 = fma(gx, sv[(33 + t) % NV], x1);
          y0 = fma(gx, sv[(42 + t) % NV], y0);
          y1 = fma(gx, sv[(51 + t) % NV], y1);
        }
        pi0 += fc0 * x0 - fc1 * y0;
        pi1 += fc0 * x1 - fc1 * y1;
        mi0 += fc0 * y0 - fc1 * x0;
        mi1 += fc0 * y1 - fc1 * x1;
      }
      const int e = se[b];
      if (te && p >= 2) {
        const unsigned fp = sfo[b];
        // primary: columns (partner lane holds column l^1), then rows
        const double qpr0 = __shfl_xor_sync(0xffffffffu, pr0, 1);
        const double qpi0 = __shfl_xor_sync(0xffffffffu, pi0, 1);
        const double qpr1 = __shfl_xor_sync(0xffffffffu, pr1, 1);
        const double qpi1 = __shfl_xor_sync(0xffffffffu, pi1, 1);
        // mirror: rows l / l^1 across the lane pair, columns local
        const double qmr0 = __shfl_xor_sync(0xffffffffu, mr0, 1);
        const double qmi0 = __shfl_xor_sync(0xffffffffu, mi0, 1);
        const double qmr1 = __shfl_xor_sync(0xffffffffu, mr1, 1);
        const double qmi1 = __shfl_xor_sync(0xffffffffu, mi1, 1);
        if (fcol >= 0) {
          const double *T = c_tinv + 4 * ((fp >> (8 * fcol)) & 0xffu);
          // M[c'][c] = T[2c + c']: new[cp] = own * T[2cp+cp] + other * T[2cp+1-cp]
          const double own = T[2 * cp + cp], oth = T[2 * cp + 1 - cp];
          double n0 = own * pr0 + oth * qpr0, n1 = own * pi0 + oth * qpi0;
          double n2 = own * pr1 + oth * qpr1, n3 = own * pi1 + oth * qpi1;
          pr0 = n0; pi0 = n1; pr1 = n2; pi1 = n3;
          n0 = own * mr0 + oth * qmr0; n1 = own * mi0 + oth * qmi0;
          n2 = own * mr1 + oth * qmr1; n3 = own * mi1 + oth * qmi1;
          mr0 = n0; mi0 = n1; mr1 = n2; mi1 = n3;
        }
        if (frow >= 0) {
          const double *T = c_tinv + 4 * ((fp >> (8 * frow)) & 0xffu);
          double n0 = T[0] * pr0 + T[1] * pr1, n1 = T[0] * pi0 + T[1] * pi1;
          double n2 = T[2] * pr0 + T[3] * pr1, n3 = T[2] * pi0 + T[3] * pi1;
          pr0 = n0; pi0 = n1; pr1 = n2; pi1 = n3;
          n0 = T[0] * mr0 + T[1] * mr1; n1 = T[0] * mi0 + T[1] * mi1;
          n2 = T[2] * mr0 + T[3] * mr1; n3 = T[2] * mi0 + T[3] * mi1;
          mr0 = n0; mi0 = n1; mr1 = n2; mi1 = n3;
        }
      }
      if (MODE == 1 && valid) {
        const unsigned long long sm = ssm[b];
        const double sl = ((sm >> l) & 1ull) ? -1.0 : 1.0;
        const double sa = (((sm >> r0) & 1ull) ? -1.0 : 1.0) * sl;
        const double sb = (((sm >> r1) & 1ull) ? -1.0 : 1.0) * sl;
        pr0 *= sa; pi0 *= sa; pr1 *= sb; pi1 *= sb;
        mr0 *= sa; mi0 *= sa; mr1 *= sb; mi1 *= sb;
        if (eliminate) {
          const unsigned long long em = sem[b];
          const bool el = (em >> l) & 1ull;
          if (el || ((em >> r0) & 1ull)) { pr0 = pi0 = mr0 = mi0 = 0.0; }
          if (el || ((em >> r1) & 1ull)) { pr1 = pi1 = mr1 = mi1 = 0.0; }
        }
      }
      if (valid && l < nd) {
        dcplx *dst = Ae + (size_t)e * nd * rs;
        dst[(size_t)r0 * rs + l] = mk(pr0, pi0);
        if (r1 < nd) dst[(size_t)r1 * rs + l] = mk(pr1, pi1);
        if (mirror) {
          dst[(size_t)l * rs + r0] = mk(mr0, mi0);
          if (r1 < nd) dst[(size_t)l * rs + r1] = mk(mr1, mi1);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Bulk elements as a tensor-core GEMM (alternative to k_bulk, chosen by the
// autotuner).  A_e = sum_t G_e[t] S_t written as C (8 elements x 8 entries)
// = A (8 x 32 terms) B (32 x 8) per m8n8k4 DMMA tile: A = the element
// coefficient rows (a real row: terms 0..11, an imaginary row: 6..29), B = S
// in pair-block-major entry order n = 4 pb + 2a + b for entry (2I+a, 2J+b).
// Terms: 0..5 curl-curl and 6..11 mass+KLK at the symmetric pairs, 12..20
// MixedVectorCurl (Jinv K J), 21..29 MixedVectorWeakCurl (J^T K Jinv^T).
// Each warp keeps its B fragments and its per-tile entry indices in
// registers; the face table is read from shared memory (lanes hold different
// elements).
// ---------------------------------------------------------------------------
constexpr int BK = 32;          // coefficient terms (padded)
constexpr int BREC = 2 * BK;    // doubles per element record: real row, imaginary row
constexpr int BULK_T = 4;       // N tiles (8 entries) per warp
constexpr int BULK_WARPS = 4;

// One coefficient row of 32 terms for the fused Bloch layout (both cross
// terms on, or neither): [0..5] curl-curl and [6..11] mass+KLK real parts at
// the symmetric pairs, [12..17] mass imaginary parts, [18..26] G^vc =
// Jinv K J.  Because K is antisymmetric, G^cv = J^T K Jinv^T = -(G^vc)^T,
// so the two cross terms i(G^vc : R^vc + G^cv : R^cv) collapse onto
// G^vc : D with D_ab = R^vc_ab - R^cv_ba (a table column of the B operand).
__device__ __forceinline__ void bulk_record_fused(const double *J, const double *Ji, double det,
                                                  double me_re, double me_im, const double *K,
                                                  const double *mKK, bool cc, bool ms,
                                                  bool cross, bool kl, double *r) {
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  for (int t = 0; t < BK; ++t) r[t] = 0.0;
  for (int t = 0; t < 6; ++t) {
    const int a = pa[t], b = pb[t];
    if (cc) r[t] = (J[a] * J[b] + J[3 + a] * J[3 + b] + J[6 + a] * J[6 + b]) / det;
    const double jj = Ji[a * 3 + 0] * Ji[b * 3 + 0] + Ji[a * 3 + 1] * Ji[b * 3 + 1] +
                      Ji[a * 3 + 2] * Ji[b * 3 + 2];
    double vr = 0.0, vi = 0.0;
    if (ms) { vr += me_re * jj; vi += me_im * jj; }
    if (kl) {
      double s = 0.0;
      for (int rr = 0; rr < 3; ++rr)
        for (int c2 = 0; c2 < 3; ++c2) s += Ji[a * 3 + rr] * mKK[rr * 3 + c2] * Ji[b * 3 + c2];
      vr += s;
    }
    r[6 + t] = det * vr;
    r[12 + t] = det * vi;
  }
  if (cross)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double gvc = 0.0;
        for (int rr = 0; rr < 3; ++rr)
          for (int c2 = 0; c2 < 3; ++c2) {
            const double k = K[rr * 3 + c2];
            if (k == 0.0) continue;
            gvc += Ji[a * 3 + rr] * k * J[c2 * 3 + b];
          }
        r[18 + a * 3 + b] = gvc;
      }
}

__global__ void k_prep_bulk_mma(int nb, const int *__restrict__ list,
                            const double *__restrict__ J9, const double *__restrict__ Ji9,
                            const double *__restrict__ detJ, const int *__restrict__ attr,
                            const dcplx *__restrict__ eps_tab,
                            const dcplx *__restrict__ elem_eps, PmlParams pml,
                            int mask, int fused, double *__restrict__ rec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const int e = list[i];
  double J[9], Ji[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    J[t] = J9[(size_t)e * 9 + t];
    Ji[t] = Ji9[(size_t)e * 9 + t];
  }
  const double det = detJ[e];
  const dcplx eps = elem_eps ? elem_eps[e] : eps_tab[attr[e] - 1];
  double *re = rec + (size_t)i * BREC, *im = re + BK;
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  const bool cc = mask & 1, ms = mask & 2, c0 = mask & 4, c1 = mask & 8, kl = mask & 16;
  const double kx = pml.kx, ky = pml.ky, k2 = pml.k0 * pml.k0;
  // K = [[0,0,ky],[0,0,-kx],[-ky,kx,0]] (fill_K, problem_common.inc:150-158)
  const double K[9] = {0.0, 0.0, ky, 0.0, 0.0, -kx, -ky, kx, 0.0};
  // -K K (real symmetric), the KLK tensor where Lambda = I
  const double mKK[9] = {ky * ky, -kx * ky, 0.0, -kx * ky, kx * kx, 0.0, 0.0, 0.0,
                         kx * kx + ky * ky};
  const double me_re = -k2 * eps.re, me_im = -k2 * eps.im;
  if (fused) {
    bulk_record_fused(J, Ji, det, me_re, me_im, K, mKK, cc, ms, c0 && c1, kl,
                      rec + (size_t)i * BK);
    return;
  }
  for (int t = 0; t < BK; ++t) { re[t] = 0.0; im[t] = 0.0; }
  for (int t = 0; t < 6; ++t) {
    const int a = pa[t], b = pb[t];
    if (cc) re[t] = (J[a] * J[b] + J[3 + a] * J[3 + b] + J[6 + a] * J[6 + b]) / det;
    const double jj = Ji[a * 3 + 0] * Ji[b * 3 + 0] + Ji[a * 3 + 1] * Ji[b * 3 + 1] +
                      Ji[a * 3 + 2] * Ji[b * 3 + 2];
    double vr = 0.0, vi = 0.0;
    if (ms) { vr += me_re * jj; vi += me_im * jj; }
    if (kl) {
      double s = 0.0;
      for (int rr = 0; rr < 3; ++rr)
        for (int c2 = 0; c2 < 3; ++c2) s += Ji[a * 3 + rr] * mKK[rr * 3 + c2] * Ji[b * 3 + c2];
      vr += s;
    }
    re[6 + t] = det * vr;
    im[6 + t] = det * vi;
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double gvc = 0.0, gcv = 0.0;
      for (int rr = 0; rr < 3; ++rr)
        for (int c2 = 0; c2 < 3; ++c2) {
          const double k = K[rr * 3 + c2];
          if (k == 0.0) continue;
          gvc += Ji[a * 3 + rr] * k * J[c2 * 3 + b];
          gcv += J[rr * 3 + a] * k * Ji[b * 3 + c2];
        }
      if (c0) im[12 + a * 3 + b] = gvc;
      if (c1) im[21 + a * 3 + b] = gcv;
    }
}

// One row-pair block of a bulk DMMA tile for 8 elements: the DMMA
// contraction (every lane, the instruction is warp-wide), then for this
// lane's element (ok) the dual face transform, signs and essential zeroing
// and the store of c[a][i] = entry (row + a, col + i).
template <bool CROSS, int MODE, int KS, bool FUSED>
__device__ __forceinline__ void bulk_rowpair(const double (&bfj)[2][KS], const double (&ar)[3],
                                             const double (&ai)[KS], bool ok, unsigned fp,
                                             unsigned long long sm, unsigned long long em,
                                             int row, int col, int fr, int fc, const double *sT,
                                             int nd, int rs, dcplx *base) {
  double cr[2][2], ci[2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    cr[a][0] = cr[a][1] = ci[a][0] = ci[a][1] = 0.0;
#pragma unroll
    for (int ks = 0; ks < 3; ++ks) dmma(cr[a][0], cr[a][1], ar[ks], bfj[a][ks]);
    if (FUSED) {
#pragma unroll
      for (int ks = 3; ks < (CROSS ? 7 : 5); ++ks) dmma(ci[a][0], ci[a][1], ai[ks], bfj[a][ks]);
    } else {
#pragma unroll
      for (int ks = 1; ks < (CROSS ? KS : 3); ++ks) dmma(ci[a][0], ci[a][1], ai[ks], bfj[a][ks]);
    }
  }
  if (!ok) return;
  if (fc >= 0) {  // columns: A <- A M
    const double *T = sT + 4 * ((fp >> (8 * fc)) & 0xffu);
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const double n0 = T[0] * cr[a][0] + T[1] * cr[a][1], n1 = T[2] * cr[a][0] + T[3] * cr[a][1];
      const double m0 = T[0] * ci[a][0] + T[1] * ci[a][1], m1 = T[2] * ci[a][0] + T[3] * ci[a][1];
      cr[a][0] = n0; cr[a][1] = n1; ci[a][0] = m0; ci[a][1] = m1;
    }
  }
  if (fr >= 0) {  // rows: A <- M^T A
    const double *T = sT + 4 * ((fp >> (8 * fr)) & 0xffu);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const double n0 = T[0] * cr[0][i] + T[1] * cr[1][i], n1 = T[2] * cr[0][i] + T[3] * cr[1][i];
      const double m0 = T[0] * ci[0][i] + T[1] * ci[1][i], m1 = T[2] * ci[0][i] + T[3] * ci[1][i];
      cr[0][i] = n0; cr[1][i] = n1; ci[0][i] = m0; ci[1][i] = m1;
    }
  }
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const int r = row + a;
    if (r >= nd) continue;
    if (MODE == 1) {
      const unsigned long long rbit = (sm >> r) & 1ull, cbits = sm >> col;
      const double s0 = ((rbit ^ cbits) & 1ull) ? -1.0 : 1.0;
      const double s1 = ((rbit ^ (cbits >> 1)) & 1ull) ? -1.0 : 1.0;
      cr[a][0] *= s0; ci[a][0] *= s0; cr[a][1] *= s1; ci[a][1] *= s1;
      const unsigned long long eb = em >> col;
      const bool er = (em >> r) & 1ull;
      if (er || (eb & 1ull)) { cr[a][0] = 0.0; ci[a][0] = 0.0; }
      if (er || (eb & 2ull)) { cr[a][1] = 0.0; ci[a][1] = 0.0; }
    }
    dcplx *dst = base + (size_t)r * rs + col;
    if (col + 1 < nd && (reinterpret_cast<uintptr_t>(dst) & 31u) == 0) {
      reinterpret_cast<double4 *>(dst)[0] = make_double4(cr[a][0], ci[a][0], cr[a][1], ci[a][1]);
    } else {
      dst[0] = mk(cr[a][0], ci[a][0]);
      if (col + 1 < nd) dst[1] = mk(cr[a][1], ci[a][1]);
    }
  }
}

// Tiles are 8 consecutive columns of one row: tile t = 2 (I * ncb + cb) + a
// covers entry (2I + a, 8 cb + c), c = 0..7, so a warp's C fragment for one
// element is one full 128-byte line of the (row-padded) element matrix.  A
// warp owns BULK_T/2 row-pair blocks (I, cb), i.e. both rows of each pair:
// the row transform is thread-local, the column pair is thread-local.
// FUSED: the fused Bloch layout (one 32-term coefficient row per element,
// real part from k-steps 0..2, imaginary part from 3..4, or 3..6 with the
// cross terms); otherwise the general layout (a real row and an imaginary
// row of 32 terms, k-steps 0..2 and 1..7).
template <bool CROSS, int MODE, int TT, bool FUSED>
__global__ void __launch_bounds__(BULK_WARPS * 32)
k_bulk_mma(int nb, const int *__restrict__ list, const double *__restrict__ rec,
           const double *__restrict__ S, int ntiles, int nd, int ndp, int p, int bchunk, int te,
           int eliminate, int rs, const unsigned *__restrict__ fopack,
           const unsigned long long *__restrict__ signmask,
           const unsigned long long *__restrict__ essmask, dcplx *__restrict__ Ae) {
  __shared__ double sA[8 * BREC];
  __shared__ double sT[24];
  __shared__ int se[8];
  __shared__ unsigned sfo[8];
  __shared__ unsigned long long ssm[8], sem[8];
  constexpr int PB = TT / 2;               // row-pair blocks per warp
  constexpr int KS = FUSED ? 7 : BK / 4;   // B k-steps held in registers
  constexpr int RECW = FUSED ? BK : BREC;  // doubles per element record
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int ncb = (ndp + 7) / 8;           // column blocks of 8
  const int npb = (ndp / 2) * ncb;         // row-pair blocks
  if (tid < 24) sT[tid] = c_tinv[tid];
  double bf[PB][2][KS];
  int rowv[PB], colv[PB], frv[PB], fcv[PB], okv[PB];
  const int pb0 = (blockIdx.y * BULK_WARPS + w) * PB;
#pragma unroll
  for (int j = 0; j < PB; ++j) {
    const int pb = pb0 + j;
    const bool ok = pb < npb;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const int tile = 2 * pb + a;
#pragma unroll
      for (int ks = 0; ks < KS; ++ks)
        bf[j][a][ks] = ok ? S[(size_t)(ks * 4 + t4) * ntiles * 8 + tile * 8 + g] : 0.0;
    }
    const int I = ok ? pb / ncb : 0, cb = ok ? pb - I * ncb : 0;
    rowv[j] = 2 * I;
    colv[j] = 8 * cb + 2 * t4;
    okv[j] = ok && rowv[j] < nd && colv[j] < nd;
    frv[j] = (te && p >= 2) ? face_of(2 * I, p) : -1;
    fcv[j] = (te && p >= 2) ? face_of(colv[j], p) : -1;
  }
  const int nbat = (nb + 7) / 8;
  const int b0 = blockIdx.x * bchunk, b1 = min(nbat, b0 + bchunk);
  // the next batch's records and element metadata are loaded into registers
  // while the current batch is computed
  constexpr int PF = (8 * RECW + BULK_WARPS * 32 - 1) / (BULK_WARPS * 32);
  double pf[PF];
  int pfe = -1;
  unsigned pfo = 0u;
  unsigned long long psm = 0ull, pem = 0ull;
  auto prefetch = [&](int bt) {
    const int ebase = bt * 8;
    const int nel = bt < b1 ? min(8, nb - ebase) : 0;
#pragma unroll
    for (int u = 0; u < PF; ++u) {
      const int j = tid + u * BULK_WARPS * 32;
      pf[u] = (j < 8 * RECW && (j / RECW) < nel) ? rec[(size_t)ebase * RECW + j] : 0.0;
    }
    pfe = tid < nel ? list[ebase + tid] : -1;
    if (pfe >= 0) {
      pfo = fopack[pfe];
      psm = MODE == 1 ? signmask[pfe] : 0ull;
      pem = (MODE == 1 && eliminate) ? essmask[pfe] : 0ull;
    }
  };
  prefetch(b0);
  for (int bt = b0; bt < b1; ++bt) {
    __syncthreads();
#pragma unroll
    for (int u = 0; u < PF; ++u) {
      const int j = tid + u * BULK_WARPS * 32;
      if (j < 8 * RECW) sA[j] = pf[u];
    }
    if (tid < 8) {
      se[tid] = pfe;
      sfo[tid] = pfe >= 0 ? pfo : 0u;
      ssm[tid] = pfe >= 0 ? psm : 0ull;
      sem[tid] = pfe >= 0 ? pem : 0ull;
    }
    __syncthreads();
    prefetch(bt + 1);
    double ar[3], ai[KS];
#pragma unroll
    for (int ks = 0; ks < 3; ++ks) ar[ks] = sA[g * RECW + ks * 4 + t4];
#pragma unroll
    for (int ks = 0; ks < KS; ++ks)
      ai[ks] = FUSED ? (ks >= 3 ? sA[g * RECW + ks * 4 + t4] : 0.0) : sA[g * RECW + BK + ks * 4 + t4];
    const int e = se[g];
    const unsigned fp = sfo[g];
    const unsigned long long sm = ssm[g], em = sem[g];
    dcplx *base = e >= 0 ? Ae + (size_t)e * nd * rs : Ae;
#pragma unroll
    for (int j = 0; j < PB; ++j)
      bulk_rowpair<CROSS, MODE, KS, FUSED>(bf[j], ar, ai, okv[j] && e >= 0, fp, sm, em, rowv[j],
                                           colv[j], frv[j], fcv[j], sT, nd, rs, base);
  }
}

// k_bulk_mma without block barriers: each lane reads the record terms and
// the metadata of its own element (row g of the batch of 8) straight from
// global memory -- the records are L2 resident and the block's warps share
// them through L1 -- one batch ahead in registers, so the warps of a block
// run independently.  Same tiles, operands and epilogue as k_bulk_mma.
template <bool CROSS, int MODE, int TT, bool FUSED>
__global__ void __launch_bounds__(BULK_WARPS * 32)
k_bulk_mma_nb(int nb, const int *__restrict__ list, const double *__restrict__ rec,
              const double *__restrict__ S, int ntiles, int nd, int ndp, int p, int bchunk,
              int te, int eliminate, int rs, const unsigned *__restrict__ fopack,
              const unsigned long long *__restrict__ signmask,
              const unsigned long long *__restrict__ essmask, dcplx *__restrict__ Ae) {
  __shared__ double sT[24];
  constexpr int PB = TT / 2;
  constexpr int KS = FUSED ? 7 : BK / 4;
  constexpr int RECW = FUSED ? BK : BREC;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int ncb = (ndp + 7) / 8;
  const int npb = (ndp / 2) * ncb;
  if (tid < 24) sT[tid] = c_tinv[tid];
  double bf[PB][2][KS];
  int rowv[PB], colv[PB], frv[PB], fcv[PB], okv[PB];
  const int pb0 = (blockIdx.y * BULK_WARPS + w) * PB;
#pragma unroll
  for (int j = 0; j < PB; ++j) {
    const int pb = pb0 + j;
    const bool ok = pb < npb;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const int tile = 2 * pb + a;
#pragma unroll
      for (int ks = 0; ks < KS; ++ks)
        bf[j][a][ks] = ok ? S[(size_t)(ks * 4 + t4) * ntiles * 8 + tile * 8 + g] : 0.0;
    }
    const int I = ok ? pb / ncb : 0, cb = ok ? pb - I * ncb : 0;
    rowv[j] = 2 * I;
    colv[j] = 8 * cb + 2 * t4;
    okv[j] = ok && rowv[j] < nd && colv[j] < nd;
    frv[j] = (te && p >= 2) ? face_of(2 * I, p) : -1;
    fcv[j] = (te && p >= 2) ? face_of(colv[j], p) : -1;
  }
  __syncthreads();  // the face tables; no barrier after this
  const int nbat = (nb + 7) / 8;
  const int b0 = blockIdx.x * bchunk, b1 = min(nbat, b0 + bchunk);
  double nar[3], nai[KS];
  int ne = -1;
  unsigned nfo = 0u;
  unsigned long long nsm = 0ull, nem = 0ull;
  // element of this lane one batch further ahead: the metadata loads of a
  // batch index by it and so never wait for the list load
  auto elem_of = [&](int bt) {
    const int i = bt * 8 + g;
    return (bt < b1 && i < nb) ? list[i] : -1;
  };
  int e_ahead = elem_of(b0);
  auto load = [&](int bt) {
    const int i = bt * 8 + g;
    const bool ok = bt < b1 && i < nb;
    const double *r = rec + (size_t)(ok ? i : 0) * RECW;
#pragma unroll
    for (int ks = 0; ks < 3; ++ks) nar[ks] = ok ? r[ks * 4 + t4] : 0.0;
#pragma unroll
    for (int ks = 0; ks < KS; ++ks)
      nai[ks] = !ok ? 0.0 : FUSED ? (ks >= 3 ? r[ks * 4 + t4] : 0.0) : r[BK + ks * 4 + t4];
    ne = e_ahead;
    nfo = ne >= 0 ? fopack[ne] : 0u;
    nsm = (MODE == 1 && ne >= 0) ? signmask[ne] : 0ull;
    nem = (MODE == 1 && eliminate && ne >= 0) ? essmask[ne] : 0ull;
    e_ahead = elem_of(bt + 1);
  };
  load(b0);
  for (int bt = b0; bt < b1; ++bt) {
    double ar[3], ai[KS];
#pragma unroll
    for (int ks = 0; ks < 3; ++ks) ar[ks] = nar[ks];
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) ai[ks] = nai[ks];
    const int e = ne;
    const unsigned fp = nfo;
    const unsigned long long sm = nsm, em = nem;
    load(bt + 1);
    dcplx *base = e >= 0 ? Ae + (size_t)e * nd * rs : Ae;
#pragma unroll
    for (int j = 0; j < PB; ++j)
      bulk_rowpair<CROSS, MODE, KS, FUSED>(bf[j], ar, ai, okv[j] && e >= 0, fp, sm, em, rowv[j],
                                           colv[j], frv[j], fcv[j], sT, nd, rs, base);
  }
}

// ---------------------------------------------------------------------------
// PML element kernel on FP64 tensor cores (mma.sync m8n8k4 .f64, DMMA).
//
// Per element: A_e = sum_r X[r]^T Y[r] over the staged rows r (3 curl rows
// per cc-rule point; 3 shape rows, plus 3 curl rows when the k-parallel
// cross terms are on, per mass-rule point), X real, Y = W X complex kept as
// two real planes.  As a GEMM: C (M x N) = A (M x K) B (K x N) with
// A[m][r] = X[r][m], B[r][n] = Yre/Yim[r][n]; M = N = NDP8 (nd rounded up
// to 8).  One warp per 8-column tile (real and imaginary planes), all
// M tiles, so the epilogue holds both parts of each entry.  Rows are staged
// in chunks of 8 points (p = 3) or 4; blocks are persistent over the PML elements.
//
// The stretch coefficients of every point of both rules (one pow() each)
// are formed once per element by all threads in parallel, into a table in
// shared memory; each chunk then needs two block barriers (rows staged /
// rows consumed).
// ---------------------------------------------------------------------------
constexpr int PML_QC = 8;     // quadrature points staged per round
constexpr int PML_MAXQ = 40;  // cc-rule + mass-rule points per element (p = 3: 11 + 24)

struct QCoef {  // per quadrature point, already multiplied by w_q detJ
  dcplx a00, a01, a10, a11, a22;      // (Md + M2) entries (cc rule: Lambda^-1 diagonal)
  dcplx b02, b12, b20, b21;           // M0 = i K Lambda^-1
  dcplx c02, c12, c20, c21;           // M1 = i Lambda^-1 K
};

template <int NDP8>
struct PmlShape {
  static constexpr int NW = NDP8 / 8;                    // warps = column tiles
  static constexpr int MT = NDP8 / 8;                    // row tiles
  // row stride = 4 mod 16 doubles: the fragment loads of one DMMA (lane
  // (g, t4) reads row r0 + t4, column 8 m + g) then fall on 16 distinct
  // 8-byte bank pairs in each half-warp
  static constexpr int LD = NDP8 + ((4 - NDP8 % 16) + 16) % 16;
  // points per chunk: 8 at p = 3, 4 below (smaller blocks, more per SM)
  static constexpr int QC = NDP8 >= 48 ? PML_QC : 4;
  // shared memory for chunks of qc points (rmax = 6 qc staged rows) and a
  // coefficient table of nq_all points
  static size_t smem(int qc, int nq_all) {
    return (size_t)3 * (6 * qc) * LD * sizeof(double) + (size_t)nq_all * sizeof(QCoef);
  }
  // blocks per SM the register budget is cut for (shared memory allows it)
  // p = 3 stays at 2 blocks (a 3-block register cap spills and runs slower)
  static constexpr int MINB = NDP8 >= 48 ? 2 : NDP8 >= 24 ? 5 : 16;
};

// Coefficients of one quadrature point (rule 0: curl-curl, rule 1: mass and
// k-parallel terms), asm_gpu.inc:86-161 restated per point.
__device__ __forceinline__ QCoef pml_qcoef(const PmlParams &pml, int rule, int mask, double z,
                                          double wq, dcplx eps) {
  const double k2 = pml.k0 * pml.k0;
  const double K02 = pml.ky, K12 = -pml.kx, K20 = -pml.ky, K21 = pml.kx;
  const dcplx s = pml_s(pml, z);
  const dcplx si = cinv(s);
  QCoef c;
  if (rule == 0) {
    c.a00 = cscale(wq, si); c.a11 = c.a00; c.a22 = cscale(wq, s);
    c.a01 = mk(0, 0); c.a10 = mk(0, 0);
    c.b02 = c.b12 = c.b20 = c.b21 = c.c02 = c.c12 = c.c20 = c.c21 = mk(0, 0);
    return c;
  }
  const dcplx li0 = si, li1 = si, li2 = s;
  dcplx a00 = mk(0, 0), a01 = mk(0, 0), a10 = mk(0, 0), a11 = mk(0, 0), a22 = mk(0, 0);
  if (mask & 2) {
    const dcplx me = cscale(-k2, eps);
    a00 = cmul(me, s); a11 = a00; a22 = cmul(me, si);
  }
  if (mask & 16) {
    a00 = cadd(a00, cscale(-K02 * K20, li2));
    a01 = cadd(a01, cscale(-K02 * K21, li2));
    a10 = cadd(a10, cscale(-K12 * K20, li2));
    a11 = cadd(a11, cscale(-K12 * K21, li2));
    a22 = cadd(a22, cadd(cscale(-K20 * K02, li0), cscale(-K21 * K12, li1)));
  }
  c.a00 = cscale(wq, a00); c.a01 = cscale(wq, a01); c.a10 = cscale(wq, a10);
  c.a11 = cscale(wq, a11); c.a22 = cscale(wq, a22);
  const dcplx iu = mk(0.0, 1.0);
  if (mask & 4) {
    c.b02 = cscale(wq * K02, cmul(iu, li2)); c.b12 = cscale(wq * K12, cmul(iu, li2));
    c.b20 = cscale(wq * K20, cmul(iu, li0)); c.b21 = cscale(wq * K21, cmul(iu, li1));
  } else { c.b02 = c.b12 = c.b20 = c.b21 = mk(0, 0); }
  if (mask & 8) {
    c.c02 = cscale(wq * K02, cmul(iu, li0)); c.c12 = cscale(wq * K12, cmul(iu, li1));
    c.c20 = cscale(wq * K20, cmul(iu, li2)); c.c21 = cscale(wq * K21, cmul(iu, li2));
  } else { c.c02 = c.c12 = c.c20 = c.c21 = mk(0, 0); }
  return c;
}

// Physical shapes v and curls c of the element-local columns k = 2 pr,
// 2 pr + 1 at quadrature point q, with the dual face transform applied.
__device__ __forceinline__ void pml_shapes_pair(int pr, int q, const Rule &R, int p, int te,
                                                bool need_v, bool need_c, const double *sJ,
                                                const double *sJi, double sidet, unsigned sfo,
                                                double (&v)[2][3], double (&c)[2][3]) {
  {
    // reference shapes / curls of columns 2 pr, 2 pr + 1 (zero past nd)
    double2 rv[3], rc[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const size_t o = ((size_t)r * R.nq + q) * R.ldt + 2 * pr;
      rv[r] = need_v ? *reinterpret_cast<const double2 *>(R.vt + o) : make_double2(0.0, 0.0);
      rc[r] = need_c ? *reinterpret_cast<const double2 *>(R.ct + o) : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      v[0][d] = rv[0].x * sJi[0 * 3 + d] + rv[1].x * sJi[1 * 3 + d] + rv[2].x * sJi[2 * 3 + d];
      v[1][d] = rv[0].y * sJi[0 * 3 + d] + rv[1].y * sJi[1 * 3 + d] + rv[2].y * sJi[2 * 3 + d];
      c[0][d] = (rc[0].x * sJ[d * 3 + 0] + rc[1].x * sJ[d * 3 + 1] + rc[2].x * sJ[d * 3 + 2]) * sidet;
      c[1][d] = (rc[0].y * sJ[d * 3 + 0] + rc[1].y * sJ[d * 3 + 1] + rc[2].y * sJ[d * 3 + 2]) * sidet;
    }
  }
  if (te && p >= 2) {
    const int f = face_of(2 * pr, p);
    if (f >= 0) {
      const double *T = c_tinv + 4 * ((sfo >> (8 * f)) & 0xffu);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double v0_ = v[0][d], v1_ = v[1][d], c0_ = c[0][d], c1_ = c[1][d];
        v[0][d] = v0_ * T[0] + v1_ * T[1];
        v[1][d] = v0_ * T[2] + v1_ * T[3];
        c[0][d] = c0_ * T[0] + c1_ * T[1];
        c[1][d] = c0_ * T[2] + c1_ * T[3];
      }
    }
  }
}

// One staged pair of PML rows: element-local columns k = 2 pr, 2 pr + 1 of
// quadrature point q (chunk row block qi): physical shapes/curls, the dual
// face transform, and X (real), Y = W X (two planes) at row stride LD.
// PAIR: both columns of a row in one 16-byte store (the p = 3 kernels; at
// lower p the narrower register budget keeps one store per entry).
template <int LD, bool PAIR = true>
__device__ __forceinline__ void pml_stage_pair(int qi, int pr, int q, const Rule &R, int nd, int p,
                                               int te, bool need_v, bool need_c, int rule, int rq,
                                               const double *sJ, const double *sJi, double sidet,
                                               unsigned sfo, const QCoef &C, double *Xs,
                                               double *Yr, double *Yi) {
  double v[2][3], c[2][3];
  pml_shapes_pair(pr, q, R, p, te, need_v, need_c, sJ, sJi, sidet, sfo, v, c);
  if constexpr (!PAIR) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = 2 * pr + h;
      const int rb = qi * rq;
      if (rule == 0) {
#pragma unroll
        for (int d = 0; d < 3; ++d) Xs[(rb + d) * LD + k] = c[h][d];
        const dcplx y0 = cscale(c[h][0], C.a00), y1 = cscale(c[h][1], C.a11),
                    y2 = cscale(c[h][2], C.a22);
        Yr[(rb + 0) * LD + k] = y0.re; Yi[(rb + 0) * LD + k] = y0.im;
        Yr[(rb + 1) * LD + k] = y1.re; Yi[(rb + 1) * LD + k] = y1.im;
        Yr[(rb + 2) * LD + k] = y2.re; Yi[(rb + 2) * LD + k] = y2.im;
      } else {
        const double *vv = v[h], *cc = c[h];
#pragma unroll
        for (int d = 0; d < 3; ++d) Xs[(rb + d) * LD + k] = vv[d];
        dcplx y0 = cadd(cscale(vv[0], C.a00), cscale(vv[1], C.a01));
        dcplx y1 = cadd(cscale(vv[0], C.a10), cscale(vv[1], C.a11));
        dcplx y2 = cscale(vv[2], C.a22);
        if (need_c) {
          y0 = cadd(y0, cscale(cc[2], C.b02));
          y1 = cadd(y1, cscale(cc[2], C.b12));
          y2 = cadd(y2, cadd(cscale(cc[0], C.b20), cscale(cc[1], C.b21)));
#pragma unroll
          for (int d = 0; d < 3; ++d) Xs[(rb + 3 + d) * LD + k] = cc[d];
          const dcplx z0 = cscale(vv[2], C.c02), z1 = cscale(vv[2], C.c12),
                      z2 = cadd(cscale(vv[0], C.c20), cscale(vv[1], C.c21));
          Yr[(rb + 3) * LD + k] = z0.re; Yi[(rb + 3) * LD + k] = z0.im;
          Yr[(rb + 4) * LD + k] = z1.re; Yi[(rb + 4) * LD + k] = z1.im;
          Yr[(rb + 5) * LD + k] = z2.re; Yi[(rb + 5) * LD + k] = z2.im;
        }
        Yr[(rb + 0) * LD + k] = y0.re; Yi[(rb + 0) * LD + k] = y0.im;
        Yr[(rb + 1) * LD + k] = y1.re; Yi[(rb + 1) * LD + k] = y1.im;
        Yr[(rb + 2) * LD + k] = y2.re; Yi[(rb + 2) * LD + k] = y2.im;
      }
    }
    return;
  }
  // row d of both columns: one 16-byte store a plane (columns 2 pr,
  // 2 pr + 1 side by side, LD even); the shape rows first, then (cross
  // terms) the curl rows
  const int o = qi * rq * LD + 2 * pr;
  auto put = [&](int d, double x0, double x1, dcplx y0, dcplx y1) {
    *reinterpret_cast<double2 *>(Xs + o + d * LD) = make_double2(x0, x1);
    *reinterpret_cast<double2 *>(Yr + o + d * LD) = make_double2(y0.re, y1.re);
    *reinterpret_cast<double2 *>(Yi + o + d * LD) = make_double2(y0.im, y1.im);
  };
  if (rule == 0) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const dcplx a = d == 0 ? C.a00 : d == 1 ? C.a11 : C.a22;
      put(d, c[0][d], c[1][d], cscale(c[0][d], a), cscale(c[1][d], a));
    }
    return;
  }
  {
    dcplx y[2][3];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const double *vv = v[h], *cc = c[h];
      y[h][0] = cadd(cscale(vv[0], C.a00), cscale(vv[1], C.a01));
      y[h][1] = cadd(cscale(vv[0], C.a10), cscale(vv[1], C.a11));
      y[h][2] = cscale(vv[2], C.a22);
      if (need_c) {
        y[h][0] = cadd(y[h][0], cscale(cc[2], C.b02));
        y[h][1] = cadd(y[h][1], cscale(cc[2], C.b12));
        y[h][2] = cadd(y[h][2], cadd(cscale(cc[0], C.b20), cscale(cc[1], C.b21)));
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) put(d, v[0][d], v[1][d], y[0][d], y[1][d]);
  }
  if (need_c) {
    dcplx z[2][3];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const double *vv = v[h];
      z[h][0] = cscale(vv[2], C.c02);
      z[h][1] = cscale(vv[2], C.c12);
      z[h][2] = cadd(cscale(vv[0], C.c20), cscale(vv[1], C.c21));
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) put(3 + d, c[0][d], c[1][d], z[0][d], z[1][d]);
  }
}

template <int NDP8, bool CROSS, int MODE>
__global__ void __launch_bounds__(NDP8 * 4, PmlShape<NDP8>::MINB)
k_pml_mma(int npml, const int *__restrict__ list, int nd, int rs, int p, Rule rcc, Rule rm,
          const double *__restrict__ J9, const double *__restrict__ Ji9,
          const double *__restrict__ detJ, const double *__restrict__ v0,
          const int *__restrict__ attr, const dcplx *__restrict__ eps_tab,
          const dcplx *__restrict__ elem_eps, PmlParams pml, int mask_cc, int mask_mass,
          int te, int eliminate, const unsigned *__restrict__ fopack,
          const unsigned long long *__restrict__ signmask,
          const unsigned long long *__restrict__ essmask, dcplx *__restrict__ Ae) {
  using Sh = PmlShape<NDP8>;
  constexpr int LD = Sh::LD, MT = Sh::MT, QC = Sh::QC, RMAX = 6 * QC;
  extern __shared__ __align__(16) double smem[];
  double *Xs = smem;
  double *Yr = Xs + RMAX * LD;
  double *Yi = Yr + RMAX * LD;
  QCoef *qtab = reinterpret_cast<QCoef *>(Yi + RMAX * LD);
  __shared__ double sJ[9], sJi[9], sidet;
  __shared__ unsigned sfo;

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  constexpr int npair = NDP8 / 2;
  const int nq_all = rcc.nq + rm.nq;  // <= PML_MAXQ, checked by the host

  for (int ie = blockIdx.x; ie < npml; ie += gridDim.x) {
    const int e = list[ie];
    // element scalars and the coefficient table; the previous element's
    // last barrier already ordered every read of both before these writes
    if (tid < 9) { sJ[tid] = J9[(size_t)e * 9 + tid]; sJi[tid] = Ji9[(size_t)e * 9 + tid]; }
    if (tid == 0) { sidet = 1.0 / detJ[e]; sfo = fopack[e]; }
    for (int j = tid; j < nq_all; j += blockDim.x) {
      const int rule = j < rcc.nq ? 0 : 1;
      const int q = rule == 0 ? j : j - rcc.nq;
      const Rule &R = rule == 0 ? rcc : rm;
      const double *Jz = J9 + (size_t)e * 9 + 6;
      const double z = v0[(size_t)e * 3 + 2] + Jz[0] * R.ip[q * 3 + 0] +
                       Jz[1] * R.ip[q * 3 + 1] + Jz[2] * R.ip[q * 3 + 2];
      const dcplx eps = elem_eps ? elem_eps[e] : eps_tab[attr[e] - 1];
      qtab[j] = pml_qcoef(pml, rule, rule == 0 ? mask_cc : mask_mass, z, R.w[q] * detJ[e], eps);
    }
    double cr[MT][2], ci[MT][2];
#pragma unroll
    for (int m = 0; m < MT; ++m) { cr[m][0] = cr[m][1] = ci[m][0] = ci[m][1] = 0.0; }
    __syncthreads();

    for (int rule = 0; rule < 2; ++rule) {
      const int mask = rule == 0 ? mask_cc : mask_mass;
      if (!mask) continue;
      const Rule R = rule == 0 ? rcc : rm;
      const QCoef *qc = qtab + (rule == 0 ? 0 : rcc.nq);
      const bool need_c = rule == 0 ? true : (CROSS && (mask & (4 | 8)));
      const bool need_v = rule == 1;
      const int rq = rule == 0 ? 3 : (need_c ? 6 : 3);
      for (int q0 = 0; q0 < R.nq; q0 += QC) {
        const int nqc = min(QC, R.nq - q0);
        const int nrows = nqc * rq, nrows4 = (nrows + 3) & ~3;
        // zero the padding rows up to a multiple of 4
        for (int i = tid; i < (nrows4 - nrows) * LD; i += blockDim.x) {
          const int r = nrows + i / LD, k = i % LD;
          Xs[r * LD + k] = 0.0; Yr[r * LD + k] = 0.0; Yi[r * LD + k] = 0.0;
        }
        for (int it = tid; it < nqc * npair; it += blockDim.x) {
          const int qi = it / npair, pr = it - qi * npair;
          pml_stage_pair<LD, (NDP8 >= 48)>(qi, pr, q0 + qi, R, nd, p, te, need_v, need_c, rule,
                                           rq, sJ, sJi, sidet, sfo, qc[q0 + qi], Xs, Yr, Yi);
        }
        __syncthreads();
        // tensor-core contraction of the staged rows
        for (int r0 = 0; r0 < nrows4; r0 += 4) {
          const double br = Yr[(r0 + t4) * LD + w * 8 + g];
          const double bi = Yi[(r0 + t4) * LD + w * 8 + g];
#pragma unroll
          for (int m = 0; m < MT; ++m) {
            const double a = Xs[(r0 + t4) * LD + m * 8 + g];
            dmma(cr[m][0], cr[m][1], a, br);
            dmma(ci[m][0], ci[m][1], a, bi);
          }
        }
        __syncthreads();
      }
    }
    // epilogue: C[row = m*8 + g][col = w*8 + 2*t4 + i]
    const unsigned long long sm = MODE == 1 ? signmask[e] : 0ull;
    const unsigned long long em = (MODE == 1 && eliminate) ? essmask[e] : 0ull;
    dcplx *dst = Ae + (size_t)e * nd * rs;
    const int col = w * 8 + 2 * t4;
#pragma unroll
    for (int m = 0; m < MT; ++m) {
      const int row = m * 8 + g;
      if (row >= nd) continue;
      dcplx v2[2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int l = col + i;
        double re = cr[m][i], im = ci[m][i];
        if (MODE == 1) {
          const double sg = ((((sm >> row) ^ (sm >> l)) & 1ull) ? -1.0 : 1.0);
          re *= sg; im *= sg;
          if (((em >> row) | (em >> l)) & 1ull) { re = 0.0; im = 0.0; }
        }
        v2[i] = mk(re, im);
      }
      if (col + 1 < nd) {
        dst[(size_t)row * rs + col] = v2[0];
        dst[(size_t)row * rs + col + 1] = v2[1];
      } else if (col < nd) {
        dst[(size_t)row * rs + col] = v2[0];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// PML elements with the element matrix split by symmetry (alternative to
// k_pml_mma, chosen by the autotuner).
//
// Per mass-rule point the cross coefficients satisfy M1 = -M0^T entry by
// entry (c02 = -b20, c12 = -b21, c20 = -b02, c21 = -b12: K is antisymmetric
// and Lambda^-1 diagonal), so
//   A_e = S + alpha P - beta P^T,   P_kl = sum_q v_k . (M0 c_l),
// with S the complex-symmetric part (curl-curl with diagonal Lambda^-1, mass,
// KLK) and alpha / beta the CROSS0 / CROSS1 selections.  Pass 1 contracts
// all tiles of P (X = v, Y = M0 c) into shared memory; pass 2 contracts only
// the tiles of S on or above the diagonal (X = c, Y = W c; X = v, Y = A v);
// the epilogue writes each S tile and its mirror with the P terms added.
// Every point stages 3 rows.  DMMA work at p = 3 with the cross terms:
// (36 + 21) tiles x 3 rows per mass point and 21 x 3 per curl point, against
// 36 x 6 and 36 x 3 in k_pml_mma; without them 21 of 36 tiles.
//
// The upper tiles are dealt to the warps in a folded order (column MT-1-j,
// then column j, ...), so each warp's tiles lie in at most two columns and
// the warps' tile counts differ by at most one.
// ---------------------------------------------------------------------------
template <int NDP8>
struct PmlSymShape {
  static constexpr int MT = NDP8 / 8;
  static constexpr int LD = PmlShape<NDP8>::LD;
  static constexpr int NT = MT * (MT + 1) / 2;      // tiles on or above the diagonal
  static constexpr int TPW = (NT + MT - 1) / MT;    // most upper tiles of one warp
  static constexpr int QS = NDP8 >= 48 ? 16 : 8;    // points per chunk (3 rows each)
  // P row stride: odd, so that the fragment-ordered stores and the
  // transposed reads of P spread over the banks
  static constexpr int LDP = LD + 1;
  // stage planes X, Yre, Yim of 3 QS rows, the coefficient table, and
  // (with the cross terms) P as two planes of NDP8 rows
  static size_t smem(int nq_all, bool cross) {
    return (size_t)3 * (3 * QS) * LD * sizeof(double) + (size_t)nq_all * sizeof(QCoef) +
           (cross ? (size_t)2 * NDP8 * LDP * sizeof(double) : 0);
  }
};

// Upper tile t of an MT x MT tile grid in the folded order.
template <int MT>
__host__ __device__ constexpr void sym_tile(int t, int &m, int &n) {
  for (int j = 0; j < MT / 2; ++j) {
    if (t < MT - j) { m = t; n = MT - 1 - j; return; }
    t -= MT - j;
    if (t < j + 1) { m = t; n = j; return; }
    t -= j + 1;
  }
  m = t;
  n = MT / 2;
}

// One staged pair of rows of the split kernel.  kind 0: curl-curl (X = c,
// Y = diag(Lambda^-1 terms) c); 1: symmetric mass part (X = v, Y = A v);
// 2: cross part (X = v, Y = M0 c).
template <int LD>
__device__ __forceinline__ void pml_sym_stage_pair(int qi, int pr, int q, const Rule &R, int p,
                                                   int te, int kind, const double *sJ,
                                                   const double *sJi, double sidet, unsigned sfo,
                                                   const QCoef &C, double *Xs, double *Yr,
                                                   double *Yi) {
  double v[2][3], c[2][3];
  pml_shapes_pair(pr, q, R, p, te, kind != 0, kind != 1, sJ, sJi, sidet, sfo, v, c);
  double x[2][3];
  dcplx y[2][3];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (kind == 0) {
#pragma unroll
      for (int d = 0; d < 3; ++d) x[h][d] = c[h][d];
      y[h][0] = cscale(c[h][0], C.a00); y[h][1] = cscale(c[h][1], C.a11);
      y[h][2] = cscale(c[h][2], C.a22);
    } else if (kind == 1) {
#pragma unroll
      for (int d = 0; d < 3; ++d) x[h][d] = v[h][d];
      y[h][0] = cadd(cscale(v[h][0], C.a00), cscale(v[h][1], C.a01));
      y[h][1] = cadd(cscale(v[h][0], C.a10), cscale(v[h][1], C.a11));
      y[h][2] = cscale(v[h][2], C.a22);
    } else {
#pragma unroll
      for (int d = 0; d < 3; ++d) x[h][d] = v[h][d];
      y[h][0] = cscale(c[h][2], C.b02); y[h][1] = cscale(c[h][2], C.b12);
      y[h][2] = cadd(cscale(c[h][0], C.b20), cscale(c[h][1], C.b21));
    }
  }
  // columns 2 pr, 2 pr + 1 side by side: one 16-byte store a row (LD even)
  const int o = 3 * qi * LD + 2 * pr;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    *reinterpret_cast<double2 *>(Xs + o + d * LD) = make_double2(x[0][d], x[1][d]);
    *reinterpret_cast<double2 *>(Yr + o + d * LD) = make_double2(y[0][d].re, y[1][d].re);
    *reinterpret_cast<double2 *>(Yi + o + d * LD) = make_double2(y[0][d].im, y[1][d].im);
  }
}

template <int NDP8, bool CROSS, int MODE>
__global__ void __launch_bounds__(NDP8 * 4, PmlShape<NDP8>::MINB)
k_pml_sym(int npml, const int *__restrict__ list, int nd, int rs, int p, Rule rcc, Rule rm,
          const double *__restrict__ J9, const double *__restrict__ Ji9,
          const double *__restrict__ detJ, const double *__restrict__ v0,
          const int *__restrict__ attr, const dcplx *__restrict__ eps_tab,
          const dcplx *__restrict__ elem_eps, PmlParams pml, int mask_cc, int mask_mass,
          int te, int eliminate, const unsigned *__restrict__ fopack,
          const unsigned long long *__restrict__ signmask,
          const unsigned long long *__restrict__ essmask, dcplx *__restrict__ Ae) {
  using Sh = PmlSymShape<NDP8>;
  constexpr int LD = Sh::LD, MT = Sh::MT, QS = Sh::QS, TPW = Sh::TPW;
  extern __shared__ __align__(16) double smem[];
  double *Xs = smem;
  double *Yr = Xs + 3 * QS * LD;
  double *Yi = Yr + 3 * QS * LD;
  const int nq_all = rcc.nq + rm.nq;  // <= PML_MAXQ, checked by the host
  QCoef *qtab = reinterpret_cast<QCoef *>(Yi + 3 * QS * LD);
  double *Pr = reinterpret_cast<double *>(qtab + nq_all);
  constexpr int LDP = Sh::LDP;
  double *Pi = Pr + NDP8 * LDP;
  __shared__ double sJ[9], sJi[9], sidet;
  __shared__ unsigned sfo;

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  constexpr int npair = NDP8 / 2;
  const bool cross = CROSS && (mask_mass & 12);
  // M0's coefficients are needed whenever either cross term is selected
  const int mask_coef = cross ? (mask_mass | 4) : mask_mass;

  // this warp's upper tiles: rows tm[i], column na or nb
  int tm[TPW];
  bool tok[TPW], tsec[TPW];
  int na = -1, nb = -1;
  {
    const int t0 = w * Sh::NT / MT, t1 = (w + 1) * Sh::NT / MT;
#pragma unroll
    for (int i = 0; i < TPW; ++i) {
      int m = 0, n = 0;
      tok[i] = t0 + i < t1;
      if (tok[i]) sym_tile<MT>(t0 + i, m, n);
      if (tok[i] && na < 0) na = n;
      tsec[i] = tok[i] && n != na;
      if (tsec[i]) nb = n;
      tm[i] = m;
    }
    if (na < 0) na = 0;
    if (nb < 0) nb = na;
  }

  for (int ie = blockIdx.x; ie < npml; ie += gridDim.x) {
    const int e = list[ie];
    if (tid < 9) { sJ[tid] = J9[(size_t)e * 9 + tid]; sJi[tid] = Ji9[(size_t)e * 9 + tid]; }
    if (tid == 0) { sidet = 1.0 / detJ[e]; sfo = fopack[e]; }
    for (int j = tid; j < nq_all; j += blockDim.x) {
      const int rule = j < rcc.nq ? 0 : 1;
      const int q = rule == 0 ? j : j - rcc.nq;
      const Rule &R = rule == 0 ? rcc : rm;
      const double *Jz = J9 + (size_t)e * 9 + 6;
      const double z = v0[(size_t)e * 3 + 2] + Jz[0] * R.ip[q * 3 + 0] +
                       Jz[1] * R.ip[q * 3 + 1] + Jz[2] * R.ip[q * 3 + 2];
      const dcplx eps = elem_eps ? elem_eps[e] : eps_tab[attr[e] - 1];
      qtab[j] = pml_qcoef(pml, rule, rule == 0 ? mask_cc : mask_coef, z, R.w[q] * detJ[e], eps);
    }
    __syncthreads();

    // one pass over a rule's points in chunks of QS: stage 3 rows a point,
    // then contract them (CONTRACT(r0) runs per 4-row k-step)
    auto pass = [&](const Rule &R, const QCoef *qc, int kind, auto &&contract) {
      for (int q0 = 0; q0 < R.nq; q0 += QS) {
        const int nqc = min(QS, R.nq - q0);
        const int nrows = 3 * nqc, nrows4 = (nrows + 3) & ~3;
        for (int i = tid; i < (nrows4 - nrows) * LD; i += blockDim.x) {
          const int r = nrows + i / LD, k = i % LD;
          Xs[r * LD + k] = 0.0; Yr[r * LD + k] = 0.0; Yi[r * LD + k] = 0.0;
        }
        for (int it = tid; it < nqc * npair; it += blockDim.x) {
          const int qi = it / npair, pr = it - qi * npair;
          pml_sym_stage_pair<LD>(qi, pr, q0 + qi, R, p, te, kind, sJ, sJi, sidet, sfo,
                                 qc[q0 + qi], Xs, Yr, Yi);
        }
        __syncthreads();
        for (int r0 = 0; r0 < nrows4; r0 += 4) contract(r0);
        __syncthreads();
      }
    };

    // pass 1: P = sum v^T (M0 c), all tiles, warp w owns column tile w
    if (cross) {
      double pr_[MT][2], pi_[MT][2];
#pragma unroll
      for (int m = 0; m < MT; ++m) { pr_[m][0] = pr_[m][1] = pi_[m][0] = pi_[m][1] = 0.0; }
      pass(rm, qtab + rcc.nq, 2, [&](int r0) {
        const double br = Yr[(r0 + t4) * LD + w * 8 + g];
        const double bi = Yi[(r0 + t4) * LD + w * 8 + g];
#pragma unroll
        for (int m = 0; m < MT; ++m) {
          const double a = Xs[(r0 + t4) * LD + m * 8 + g];
          dmma(pr_[m][0], pr_[m][1], a, br);
          dmma(pi_[m][0], pi_[m][1], a, bi);
        }
      });
#pragma unroll
      for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int k = m * 8 + g, l = w * 8 + 2 * t4 + i;
          Pr[k * LDP + l] = pr_[m][i];
          Pi[k * LDP + l] = pi_[m][i];
        }
    }

    // pass 2: the upper tiles of S
    double sr[TPW][2], si[TPW][2];
#pragma unroll
    for (int i = 0; i < TPW; ++i) { sr[i][0] = sr[i][1] = si[i][0] = si[i][1] = 0.0; }
    auto contract_s = [&](int r0) {
      const double bar = Yr[(r0 + t4) * LD + na * 8 + g];
      const double bai = Yi[(r0 + t4) * LD + na * 8 + g];
      double bbr = bar, bbi = bai;
      if (nb != na) {
        bbr = Yr[(r0 + t4) * LD + nb * 8 + g];
        bbi = Yi[(r0 + t4) * LD + nb * 8 + g];
      }
#pragma unroll
      for (int i = 0; i < TPW; ++i) {
        if (!tok[i]) continue;
        const double a = Xs[(r0 + t4) * LD + tm[i] * 8 + g];
        dmma(sr[i][0], sr[i][1], a, tsec[i] ? bbr : bar);
        dmma(si[i][0], si[i][1], a, tsec[i] ? bbi : bai);
      }
    };
    if (mask_cc) pass(rcc, qtab, 0, contract_s);
    if (mask_mass) pass(rm, qtab + rcc.nq, 1, contract_s);
    if (cross) __syncthreads();  // P complete before the epilogue reads it

    // epilogue: entry (k, l) of each upper tile and its mirror (l, k)
    const unsigned long long sm = MODE == 1 ? signmask[e] : 0ull;
    const unsigned long long em = (MODE == 1 && eliminate) ? essmask[e] : 0ull;
    const bool al = mask_mass & 4, be = mask_mass & 8;
    dcplx *dst = Ae + (size_t)e * nd * rs;
#pragma unroll
    for (int i = 0; i < TPW; ++i) {
      if (!tok[i]) continue;
      const int n = tsec[i] ? nb : na;
      const int k = tm[i] * 8 + g;
      dcplx up[2], lo[2];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int l = n * 8 + 2 * t4 + c;
        double ur = sr[i][c], ui = si[i][c], lr = ur, li = ui;
        if (cross) {
          const double pkr = Pr[k * LDP + l], pki = Pi[k * LDP + l];
          const double plr = Pr[l * LDP + k], pli = Pi[l * LDP + k];
          if (al) { ur += pkr; ui += pki; lr += plr; li += pli; }
          if (be) { ur -= plr; ui -= pli; lr -= pkr; li -= pki; }
        }
        if (MODE == 1) {
          const double sg = ((((sm >> k) ^ (sm >> l)) & 1ull) ? -1.0 : 1.0);
          ur *= sg; ui *= sg; lr *= sg; li *= sg;
          if (((em >> k) | (em >> l)) & 1ull) { ur = ui = lr = li = 0.0; }
        }
        up[c] = mk(ur, ui);
        lo[c] = mk(lr, li);
      }
      const int l0 = n * 8 + 2 * t4;
      if (k < nd) {
        if (l0 + 1 < nd) {
          dst[(size_t)k * rs + l0] = up[0];
          dst[(size_t)k * rs + l0 + 1] = up[1];
        } else if (l0 < nd) {
          dst[(size_t)k * rs + l0] = up[0];
        }
      }
      if (n != tm[i] && k < nd) {
#pragma unroll
        for (int c = 0; c < 2; ++c)
          if (l0 + c < nd) dst[(size_t)(l0 + c) * rs + k] = lo[c];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// PML elements at p = 3, warp-specialised (alternative to k_pml_mma<48>,
// chosen by the autotuner).  WS_PROD producer warps: WS_STAGE threads stage
// the rows of the next chunks into a ring of WS_NBUF buffers, the others
// form the next element's coefficient table in a second table slot; while
// WS_CONS consumer warps run the DMMA contraction of the oldest buffer.
// Each consumer warp owns a block of WS_CM x WS_CN of the 6 x 6 tiles (real
// and imaginary planes), one consumer per SM sub-partition.  Staging takes
// more instructions than the contraction, so most of the warps are
// producers.  The buffers are handed over through mbarriers (full: every
// staging thread arrives after its stores; empty: every consumer thread
// arrives after its loads).
// Every wait is bounded: a wait that runs out sets *err, and that
// thread then skips its remaining waits but keeps to the same loop, so the
// kernel always finishes (with the error reported, results undefined).
// ---------------------------------------------------------------------------
constexpr int WS_CM = 3, WS_CN = 3;  // row / column tiles per consumer warp
constexpr int WS_CONS = (6 / WS_CM) * (6 / WS_CN), WS_PROD = 16 - WS_CONS;
constexpr int WS_NBUF = 3;  // staging buffers in the ring
// producer threads that stage rows (one column pair each of a full chunk of
// 8 points x 24 pairs); the other producer threads form the next element's
// coefficient table meanwhile
constexpr int WS_STAGE = 8 * 24;
static_assert(WS_STAGE < WS_PROD * 32, "no producer threads left for the table");
constexpr int WS_THREADS = (WS_CONS + WS_PROD) * 32;
constexpr long long WS_WAIT_LIMIT = 1ll << 20;  // try_wait rounds before giving up

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
#ifdef LFASM_BOUNDS
// Debug build only: the wait limit and a test injection that withholds the
// stagers' arrivals on block 0's first chunk barrier, so that the consumers'
// first wait on it must run out (set by lfasm_debug_wait_test).
__device__ long long g_ws_wait_limit = WS_WAIT_LIMIT;
__device__ int g_ws_drop_first = 0;
#define WS_LIMIT g_ws_wait_limit
#else
#define WS_LIMIT WS_WAIT_LIMIT
#endif
// bounded wait for the completion of the phase with the given parity;
// false (and *err set) if it did not complete
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, int *err) {
  const long long limit = WS_LIMIT;
  for (long long it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  atomicExch(err, 1);
  return false;
}

// ---------------------------------------------------------------------------
// k_bulk_mma with the element records staged by the bulk-copy engine: thread
// 0 issues one cp.async.bulk (global -> shared, completion counted on an
// mbarrier in bytes) per batch of 8 elements, one batch ahead into the other
// of two shared buffers, so the records reach shared memory without passing
// through registers.  Every wait on a copy is bounded (a wait that runs out
// sets *err, skips the rest of its waits and the block still finishes);
// before returning, thread 0 waits (bounded) for any copy still in flight.
// Same tiles, operands and epilogue as k_bulk_mma.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// bytes (a multiple of 16) from src (16-byte aligned) to the 16-byte aligned
// shared dst, completion on bar
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes,
                                         unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

template <bool CROSS, int MODE, int TT, bool FUSED>
__global__ void __launch_bounds__(BULK_WARPS * 32)
k_bulk_tma(int nb, const int *__restrict__ list, const double *__restrict__ rec,
           const double *__restrict__ S, int ntiles, int nd, int ndp, int p, int bchunk, int te,
           int eliminate, int rs, const unsigned *__restrict__ fopack,
           const unsigned long long *__restrict__ signmask,
           const unsigned long long *__restrict__ essmask, dcplx *__restrict__ Ae,
           int *__restrict__ err) {
  constexpr int PB = TT / 2;
  constexpr int KS = FUSED ? 7 : BK / 4;
  constexpr int RECW = FUSED ? BK : BREC;
  __shared__ alignas(128) double sA[2][8 * RECW];
  __shared__ unsigned long long bar[2];
  __shared__ double sT[24];
  __shared__ int se[8];
  __shared__ unsigned sfo[8];
  __shared__ unsigned long long ssm[8], sem[8];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int ncb = (ndp + 7) / 8;
  const int npb = (ndp / 2) * ncb;
  if (tid < 24) sT[tid] = c_tinv[tid];
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
  }
  double bf[PB][2][KS];
  int rowv[PB], colv[PB], frv[PB], fcv[PB], okv[PB];
  const int pb0 = (blockIdx.y * BULK_WARPS + w) * PB;
#pragma unroll
  for (int j = 0; j < PB; ++j) {
    const int pb = pb0 + j;
    const bool ok = pb < npb;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const int tile = 2 * pb + a;
#pragma unroll
      for (int ks = 0; ks < KS; ++ks)
        bf[j][a][ks] = ok ? S[(size_t)(ks * 4 + t4) * ntiles * 8 + tile * 8 + g] : 0.0;
    }
    const int I = ok ? pb / ncb : 0, cb = ok ? pb - I * ncb : 0;
    rowv[j] = 2 * I;
    colv[j] = 8 * cb + 2 * t4;
    okv[j] = ok && rowv[j] < nd && colv[j] < nd;
    frv[j] = (te && p >= 2) ? face_of(2 * I, p) : -1;
    fcv[j] = (te && p >= 2) ? face_of(colv[j], p) : -1;
  }
  const int nbat = (nb + 7) / 8;
  const int b0 = blockIdx.x * bchunk, b1 = min(nbat, b0 + bchunk);
  // batch bt goes to buffer (bt - b0) & 1, the k-th use of a buffer
  // completing its barrier's phase k & 1
  auto issue = [&](int bt) {
    const int ebase = bt * 8, nel = min(8, nb - ebase), buf = (bt - b0) & 1;
    const unsigned bytes = (unsigned)(nel * RECW * sizeof(double));
    // the buffer's previous contents were read through the generic proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bar[buf], bytes);
    bulk_g2s(sA[buf], rec + (size_t)ebase * RECW, bytes, &bar[buf]);
  };
  int pfe = -1;
  unsigned pfo = 0u;
  unsigned long long psm = 0ull, pem = 0ull;
  auto meta = [&](int bt) {
    const int ebase = bt * 8;
    const int nel = bt < b1 ? min(8, nb - ebase) : 0;
    pfe = tid < nel ? list[ebase + tid] : -1;
    if (pfe >= 0) {
      pfo = fopack[pfe];
      psm = MODE == 1 ? signmask[pfe] : 0ull;
      pem = (MODE == 1 && eliminate) ? essmask[pfe] : 0ull;
    }
  };
  __syncthreads();  // barriers initialised
  if (tid == 0 && b0 < b1) issue(b0);
  meta(b0);
  bool live = true;
  for (int bt = b0; bt < b1; ++bt) {
    const int buf = (bt - b0) & 1;
    const unsigned par = (unsigned)(((bt - b0) >> 1) & 1);
    __syncthreads();  // the previous batch is done: its buffer may be refilled
    if (tid < 8) {
      se[tid] = pfe;
      sfo[tid] = pfe >= 0 ? pfo : 0u;
      ssm[tid] = pfe >= 0 ? psm : 0ull;
      sem[tid] = pfe >= 0 ? pem : 0ull;
    }
    if (tid == 0 && bt + 1 < b1) issue(bt + 1);
    __syncthreads();
    meta(bt + 1);
    if (live) live = mbar_wait(&bar[buf], par, err);
    const double *A = sA[buf];
    double ar[3], ai[KS];
#pragma unroll
    for (int ks = 0; ks < 3; ++ks) ar[ks] = A[g * RECW + ks * 4 + t4];
#pragma unroll
    for (int ks = 0; ks < KS; ++ks)
      ai[ks] = FUSED ? (ks >= 3 ? A[g * RECW + ks * 4 + t4] : 0.0) : A[g * RECW + BK + ks * 4 + t4];
    const int e = se[g];
    const unsigned fp = sfo[g];
    const unsigned long long sm = ssm[g], em = sem[g];
    dcplx *base = e >= 0 ? Ae + (size_t)e * nd * rs : Ae;
#pragma unroll
    for (int j = 0; j < PB; ++j)
      bulk_rowpair<CROSS, MODE, KS, FUSED>(bf[j], ar, ai, okv[j] && e >= 0, fp, sm, em, rowv[j],
                                           colv[j], frv[j], fcv[j], sT, nd, rs, base);
  }
  // a copy whose wait ran out may still be in flight: drain the last use of
  // each buffer before the block's shared memory is released
  if (!live && tid == 0)
    for (int last = b1 - 1; last >= b0 && last >= b1 - 2; --last)
      mbar_wait(&bar[(last - b0) & 1], (unsigned)(((last - b0) >> 1) & 1), err);
}

struct PmlWsShape {
  static constexpr int NDP8 = 48, LD = 52, MT = 6, QC = 8, RMAX = 6 * QC;
  static constexpr size_t BUF = (size_t)3 * RMAX * LD;  // doubles per ring buffer
  // the ring, then two coefficient tables (this element's, the next one's)
  static size_t smem(int nq_all) {
    return WS_NBUF * BUF * sizeof(double) + (size_t)2 * nq_all * sizeof(QCoef);
  }
};

template <bool CROSS, int MODE>
__global__ void __launch_bounds__(WS_THREADS, 1)
k_pml_ws(int npml, const int *__restrict__ list, int nd, int rs, int p, Rule rcc, Rule rm,
         const double *__restrict__ J9, const double *__restrict__ Ji9,
         const double *__restrict__ detJ, const double *__restrict__ v0,
         const int *__restrict__ attr, const dcplx *__restrict__ eps_tab,
         const dcplx *__restrict__ elem_eps, PmlParams pml, int mask_cc, int mask_mass, int te,
         int eliminate, const unsigned *__restrict__ fopack,
         const unsigned long long *__restrict__ signmask,
         const unsigned long long *__restrict__ essmask, dcplx *__restrict__ Ae,
         int *__restrict__ err) {
  using Sh = PmlWsShape;
  constexpr int LD = Sh::LD, QC = Sh::QC, RMAX = Sh::RMAX, NDP8 = Sh::NDP8;
  extern __shared__ double smem[];
  QCoef *qtab = reinterpret_cast<QCoef *>(smem + WS_NBUF * Sh::BUF);  // [2][nq_all]
  __shared__ unsigned long long full[WS_NBUF], empty[WS_NBUF];
  __shared__ double sJ[2][9], sJi[2][9], sidet[2];
  __shared__ unsigned sfo[2];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int b = 0; b < WS_NBUF; ++b) {
      mbar_init(&full[b], WS_STAGE);
      mbar_init(&empty[b], WS_CONS * 32);
    }
  }
  __syncthreads();
  const int nq_all = rcc.nq + rm.nq;
  bool live = true;  // false after a wait ran out: no more waiting

  if (warp >= WS_CONS) {
    // ------------------------------------------------------------ producers
    // Element tables in two slots.  Producer threads 0 .. WS_STAGE - 1 stage
    // the current element's rows (one column pair each) and alone arrive on
    // the chunk barriers; the other producer threads form the next
    // element's coefficient table and geometry in the other slot meanwhile.
    // One producer barrier an element makes the new slot visible and frees
    // the old one.
    const int ptid = tid - WS_CONS * 32;
    constexpr int npair = NDP8 / 2;
    static_assert(QC * npair == WS_STAGE, "one column pair a staging thread");
    constexpr int NFILL = WS_PROD * 32 - WS_STAGE;
    const int nfill_items = max(nq_all, 9);
    auto fill = [&](int ie, int slot, int t) {
      const int e = list[ie];
      if (t < 9) {
        sJ[slot][t] = J9[(size_t)e * 9 + t];
        sJi[slot][t] = Ji9[(size_t)e * 9 + t];
      }
      if (t == 0) { sidet[slot] = 1.0 / detJ[e]; sfo[slot] = fopack[e]; }
      if (t < nq_all) {
        const int rule = t < rcc.nq ? 0 : 1;
        const int q = rule == 0 ? t : t - rcc.nq;
        const Rule &R = rule == 0 ? rcc : rm;
        const double *Jz = J9 + (size_t)e * 9 + 6;
        const double z = v0[(size_t)e * 3 + 2] + Jz[0] * R.ip[q * 3 + 0] +
                         Jz[1] * R.ip[q * 3 + 1] + Jz[2] * R.ip[q * 3 + 2];
        const dcplx eps = elem_eps ? elem_eps[e] : eps_tab[attr[e] - 1];
        qtab[slot * nq_all + t] =
            pml_qcoef(pml, rule, rule == 0 ? mask_cc : mask_mass, z, R.w[q] * detJ[e], eps);
      }
    };
    if (blockIdx.x < npml)
      for (int t = ptid; t < nfill_items; t += WS_PROD * 32) fill(blockIdx.x, 0, t);
    asm volatile("bar.sync 1, %0;" ::"n"(WS_PROD * 32) : "memory");  // producers only
    unsigned c = 0;
    int slot = 0;
    for (int ie = blockIdx.x; ie < npml; ie += gridDim.x, slot ^= 1) {
      if (ptid >= WS_STAGE) {
        const int ien = ie + gridDim.x;
        if (ien < npml)
          for (int t = ptid - WS_STAGE; t < nfill_items; t += NFILL) fill(ien, slot ^ 1, t);
      } else {
        const double *tJ = sJ[slot], *tJi = sJi[slot];
        const double tdet = sidet[slot];
        const unsigned tfo = sfo[slot];
        for (int rule = 0; rule < 2; ++rule) {
          const int mask = rule == 0 ? mask_cc : mask_mass;
          if (!mask) continue;
          const Rule R = rule == 0 ? rcc : rm;
          const QCoef *qc = qtab + slot * nq_all + (rule == 0 ? 0 : rcc.nq);
          const bool need_c = rule == 0 ? true : (CROSS && (mask & (4 | 8)));
          const bool need_v = rule == 1;
          const int rq = rule == 0 ? 3 : (need_c ? 6 : 3);
          for (int q0 = 0; q0 < R.nq; q0 += QC, ++c) {
            const int nqc = min(QC, R.nq - q0);
            const int nrows = nqc * rq, nrows4 = (nrows + 3) & ~3;
            const unsigned b = c % WS_NBUF, use = c / WS_NBUF;
            if (live) live = mbar_wait(&empty[b], (use & 1u) ^ 1u, err);
            double *Xs = smem + b * Sh::BUF;
            double *Yr = Xs + RMAX * LD;
            double *Yi = Yr + RMAX * LD;
            for (int i = ptid; i < (nrows4 - nrows) * LD; i += WS_STAGE) {
              const int r = nrows + i / LD, k = i % LD;
              Xs[r * LD + k] = 0.0; Yr[r * LD + k] = 0.0; Yi[r * LD + k] = 0.0;
            }
            if (ptid < nqc * npair) {
              const int qi = ptid / npair, pr = ptid - qi * npair;
              pml_stage_pair<LD>(qi, pr, q0 + qi, R, nd, p, te, need_v, need_c, rule, rq, tJ,
                                 tJi, tdet, tfo, qc[q0 + qi], Xs, Yr, Yi);
            }
#ifdef LFASM_BOUNDS
            if (!(g_ws_drop_first && blockIdx.x == 0 && c == 0))
#endif
              mbar_arrive(&full[b]);
          }
        }
      }
      asm volatile("bar.sync 1, %0;" ::"n"(WS_PROD * 32) : "memory");  // next slot ready
    }
    return;
  }

  // -------------------------------------------------------------- consumers
  const int g = lane >> 2, t4 = lane & 3;
  const int m0 = (warp / (6 / WS_CN)) * WS_CM, n0 = (warp % (6 / WS_CN)) * WS_CN;
  unsigned c = 0;
  for (int ie = blockIdx.x; ie < npml; ie += gridDim.x) {
    const int e = list[ie];
    double cr[WS_CM][WS_CN][2], ci[WS_CM][WS_CN][2];
#pragma unroll
    for (int m = 0; m < WS_CM; ++m)
#pragma unroll
      for (int n = 0; n < WS_CN; ++n) cr[m][n][0] = cr[m][n][1] = ci[m][n][0] = ci[m][n][1] = 0.0;
    for (int rule = 0; rule < 2; ++rule) {
      const int mask = rule == 0 ? mask_cc : mask_mass;
      if (!mask) continue;
      const Rule R = rule == 0 ? rcc : rm;
      const bool need_c = rule == 0 ? true : (CROSS && (mask & (4 | 8)));
      const int rq = rule == 0 ? 3 : (need_c ? 6 : 3);
      for (int q0 = 0; q0 < R.nq; q0 += QC, ++c) {
        const int nqc = min(QC, R.nq - q0);
        const int nrows4 = (nqc * rq + 3) & ~3;
        const unsigned b = c % WS_NBUF, use = c / WS_NBUF;
        if (live) live = mbar_wait(&full[b], use & 1u, err);
        const double *Xs = smem + b * Sh::BUF;
        const double *Yr = Xs + RMAX * LD;
        const double *Yi = Yr + RMAX * LD;
        for (int r0 = 0; r0 < nrows4; r0 += 4) {
          double br[WS_CN], bi[WS_CN];
#pragma unroll
          for (int n = 0; n < WS_CN; ++n) {
            br[n] = Yr[(r0 + t4) * LD + (n0 + n) * 8 + g];
            bi[n] = Yi[(r0 + t4) * LD + (n0 + n) * 8 + g];
          }
#pragma unroll
          for (int m = 0; m < WS_CM; ++m) {
            const double a = Xs[(r0 + t4) * LD + (m0 + m) * 8 + g];
#pragma unroll
            for (int n = 0; n < WS_CN; ++n) {
              dmma(cr[m][n][0], cr[m][n][1], a, br[n]);
              dmma(ci[m][n][0], ci[m][n][1], a, bi[n]);
            }
          }
        }
        mbar_arrive(&empty[b]);
      }
    }
    // epilogue: C[row = (m0 + m) 8 + g][col = (n0 + n) 8 + 2 t4 + i]
    const unsigned long long sm = MODE == 1 ? signmask[e] : 0ull;
    const unsigned long long em = (MODE == 1 && eliminate) ? essmask[e] : 0ull;
    dcplx *dst = Ae + (size_t)e * nd * rs;
#pragma unroll
    for (int m = 0; m < WS_CM; ++m)
#pragma unroll
    for (int n = 0; n < WS_CN; ++n) {
      const int row = (m0 + m) * 8 + g;
      const int col = (n0 + n) * 8 + 2 * t4;
      if (row >= nd) continue;
      dcplx v2[2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int l = col + i;
        double re = cr[m][n][i], im = ci[m][n][i];
        if (MODE == 1) {
          const double sg = ((((sm >> row) ^ (sm >> l)) & 1ull) ? -1.0 : 1.0);
          re *= sg; im *= sg;
          if (((em >> row) | (em >> l)) & 1ull) { re = 0.0; im = 0.0; }
        }
        v2[i] = mk(re, im);
      }
      if (col + 1 < nd) {
        dst[(size_t)row * rs + col] = v2[0];
        dst[(size_t)row * rs + col + 1] = v2[1];
      } else if (col < nd) {
        dst[(size_t)row * rs + col] = v2[0];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Row-owner gather: one warp per CSR row sums the element-row contributions
// through the precomputed entry -> slot-offset map (no atomics).
// RAW: element buffer without signs/elimination (ComputeLocal output).
// ---------------------------------------------------------------------------
// The row's element contributions summed into acc[0..nr) (shared memory, or
// the row's own CSR values for rows longer than the shared accumulator),
// the unit diagonal of an essential row set.  Inlined twice so that the
// shared-memory path keeps shared-memory instructions.
// row-list entries whose element-row loads a gather warp issues together
// (2 measured best on the benchmark mesh: 0.96 ms against 1.04 for 1 and
// 1.22 for 4, whose registers cost occupancy)
#ifndef GATHER_UNROLL
#define GATHER_UNROLL 2
#endif
template <bool RAW>
__device__ __forceinline__ void gather_row_q(dcplx *acc, int r, int rb, int nr, int lane,
                                             int p0, int p1, bool row_ess,
                                             const int *__restrict__ ea,
                                             const uint16_t *__restrict__ off,
                                             const int *__restrict__ Jc,
                                             const dcplx *__restrict__ Ae, int nd, int rs,
                                             const unsigned char *__restrict__ ess,
                                             const double *__restrict__ sign,
                                             const int *__restrict__ dof, int eliminate,
                                             long long n_erows) {
  for (int j = lane; j < nr; j += 32) acc[j] = mk(0.0, 0.0);
  __syncwarp();
  if (!RAW && nd <= 16) {
    // short element rows (p = 1): 32 / nd row-list entries per pass, one
    // lane per (entry, column); their loads issue together, the additions
    // go entry by entry (two entries may share a slot)
    const int epi = 32 / nd;
    const int sub = lane / nd, b = lane - sub * nd;
    for (int q0 = p0; q0 < p1; q0 += epi) {
      const int pp = q0 + sub;
      dcplx v = mk(0.0, 0.0);
      int j = -1;
      if (sub < epi && pp < p1) {
        const int id = ea[pp];
        if (LF_CHECK(id >= 0 && id < n_erows, BOUNDS_ELEM_ROW)) {
          v = Ae[(size_t)id * rs + b];
          j = off[(size_t)pp * nd + b];
          if (!LF_CHECK(j < nr, BOUNDS_SLOT)) j = -1;
        }
      }
      for (int t = 0; t < epi; ++t) {
        if (sub == t && j >= 0) { acc[j].re += v.re; acc[j].im += v.im; }
        __syncwarp();
      }
    }
  } else if (!RAW && nd <= 64 && GATHER_UNROLL > 1) {
    // GATHER_UNROLL row-list entries a step: every lane loads its columns of
    // all of them first (independent loads in flight together), then the
    // additions go entry by entry (two entries may share a slot)
    constexpr int U = GATHER_UNROLL;
    for (int q0 = p0; q0 < p1; q0 += U) {
      dcplx v[U][2];
      int j[U][2];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int pp = q0 + u;
        j[u][0] = j[u][1] = -1;
        if (pp < p1) {
          const int id = ea[pp];
          if (LF_CHECK(id >= 0 && id < n_erows, BOUNDS_ELEM_ROW)) {
            const dcplx *src = Ae + (size_t)id * rs;
            const uint16_t *o = off + (size_t)pp * nd;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int b = lane + 32 * h;
              if (b < nd) {
                v[u][h] = src[b];
                const int jj = o[b];
                j[u][h] = LF_CHECK(jj < nr, BOUNDS_SLOT) ? jj : -1;
              }
            }
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
#pragma unroll
        for (int h = 0; h < 2; ++h)
          if (j[u][h] >= 0) {
            acc[j[u][h]].re += v[u][h].re;
            acc[j[u][h]].im += v[u][h].im;
          }
        __syncwarp();
      }
    }
  } else {
    for (int pp = p0; pp < p1; ++pp) {
      const int id = ea[pp];  // the same in every lane
      if (!LF_CHECK(id >= 0 && id < n_erows, BOUNDS_ELEM_ROW)) continue;
      const dcplx *src = Ae + (size_t)id * rs;
      const uint16_t *o = off + (size_t)pp * nd;
      double sa = 1.0;
      int ebase = 0;
      if (RAW) { sa = sign[id]; ebase = (id / nd) * nd; }
      for (int b = lane; b < nd; b += 32) {
        dcplx v = src[b];
        const int j = o[b];
        if (!LF_CHECK(j < nr, BOUNDS_SLOT)) continue;
        if (RAW) {
          const double s = sa * sign[ebase + b];
          v.re *= s; v.im *= s;
          if (eliminate && (row_ess || ess[dof[ebase + b]])) v = mk(0.0, 0.0);
        }
        acc[j].re += v.re;
        acc[j].im += v.im;
      }
      __syncwarp();
    }
  }
  if (row_ess && lane == 0) {
    int lo = 0, hi = nr - 1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (Jc[rb + mid] < r) lo = mid + 1; else hi = mid;
    }
    acc[lo] = mk(1.0, 0.0);
  }
  __syncwarp();
}

template <bool RAW>
__device__ __forceinline__ void gather_row(dcplx *acc, int r, int rb, int nr, int lane,
                                           const int *__restrict__ ea_ptr,
                                           const int *__restrict__ ea,
                                           const uint16_t *__restrict__ off,
                                           const int *__restrict__ Jc,
                                           const dcplx *__restrict__ Ae, int nd, int rs,
                                           const unsigned char *__restrict__ ess,
                                           const double *__restrict__ sign,
                                           const int *__restrict__ dof, int eliminate,
                                           long long n_erows) {
  gather_row_q<RAW>(acc, r, rb, nr, lane, ea_ptr[r], ea_ptr[r + 1], eliminate && ess[r], ea, off,
                    Jc, Ae, nd, rs, ess, sign, dof, eliminate, n_erows);
}

// LONG = false: one warp per row r < n, accumulator in shared memory; rows
// longer than maxrow are skipped.  LONG = true: one warp per entry of
// long_rows (the rows longer than maxrow), accumulating in place in the
// row's CSR values, still owned by this warp alone.
template <bool RAW, bool LONG>
__global__ void k_gather(int n, const int *__restrict__ long_rows, const int *__restrict__ ea_ptr,
                         const int *__restrict__ ea,
                         const uint16_t *__restrict__ off, const int *__restrict__ I,
                         const int *__restrict__ Jc, const dcplx *__restrict__ Ae, int nd, int rs,
                         const unsigned char *__restrict__ ess,
                         const double *__restrict__ sign, const int *__restrict__ dof,
                         int eliminate, int maxrow, long long n_erows, dcplx *__restrict__ vals) {
  extern __shared__ dcplx sacc[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int w = blockIdx.x * (blockDim.x >> 5) + wib;
  if (w >= n) return;
  const int r = LONG ? long_rows[w] : w;
  const int rb = I[r], nr = I[r + 1] - rb;
  if (!LONG && nr > maxrow) return;
  dcplx *acc = LONG ? vals + rb : sacc + (size_t)wib * maxrow;
  gather_row<RAW>(acc, r, rb, nr, lane, ea_ptr, ea, off, Jc, Ae, nd, rs, ess, sign, dof,
                  eliminate, n_erows);
  if (!LONG)
    for (int j = lane; j < nr; j += 32) vals[rb + j] = acc[j];
}

// ---------------------------------------------------------------------------
// Chunked assembly: the bulk elements are taken in chunks of consecutive
// centroid height, and the CSR rows whose last element lies in a chunk are
// gathered right after that chunk, while its element rows are still in L2.  Each
// element row is read by exactly one CSR row, so after reading it the warp
// discards its 128-byte lines from L2 (discard.global.L2: the lines are
// dropped without being written back), and the element buffer does not have
// to travel to DRAM and back.
// ---------------------------------------------------------------------------
// centroid heights of the elements of a list (sort keys) and the list
__global__ void k_list_zkey(int n, const int *__restrict__ list, const double *__restrict__ J9,
                            const double *__restrict__ v0, double *__restrict__ key,
                            int *__restrict__ ids) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int e = list[i];
  const double *Jz = J9 + (size_t)e * 9 + 6;
  key[i] = v0[(size_t)e * 3 + 2] + 0.25 * (Jz[0] + Jz[1] + Jz[2]);
  ids[i] = e;
}

__global__ void k_fill_int(int n, int v, int *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = v;
}

// chunk of each element from its rank in the height order
__global__ void k_chunk_of(int ne, const int *__restrict__ sorted, int per_chunk,
                           int *__restrict__ chunk_of) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ne) chunk_of[sorted[i]] = i / per_chunk;
}

// completion chunk of each CSR row (the last chunk holding one of its
// element rows) and the identity permutation of the rows
__global__ void k_row_chunk(int n, const int *__restrict__ ea_ptr, const int *__restrict__ ea,
                            int nd, const int *__restrict__ chunk_of, int *__restrict__ comp,
                            int *__restrict__ ids) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  int c = 0;
  for (int pp = ea_ptr[r]; pp < ea_ptr[r + 1]; ++pp) c = max(c, chunk_of[ea[pp] / nd]);
  comp[r] = c;
  ids[r] = r;
}

__device__ __forceinline__ void discard_l2_line(const void *p) {
  asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

// Gather of the rows rows[0..n) (rows longer than maxrow are left to the
// long-row launch), signed element rows as lfasm_assemble writes them, each
// element row's lines discarded from L2 once the warp has added it.
// rs is a multiple of 8: an element row is rs / 8 whole 128-byte lines.
__global__ void k_gather_list(int n, const int *__restrict__ rows, const int *__restrict__ ea_ptr,
                              const int *__restrict__ ea, const uint16_t *__restrict__ off,
                              const int *__restrict__ I, const int *__restrict__ Jc,
                              const dcplx *__restrict__ Ae, int nd, int rs,
                              const unsigned char *__restrict__ ess, int eliminate, int maxrow,
                              long long n_erows, dcplx *__restrict__ vals) {
  extern __shared__ dcplx sacc[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int w = blockIdx.x * (blockDim.x >> 5) + wib;
  if (w >= n) return;
  const int r = rows[w];
  const int rb = I[r], nr = I[r + 1] - rb;
  if (nr > maxrow) return;
  dcplx *acc = sacc + (size_t)wib * maxrow;
  for (int j = lane; j < nr; j += 32) acc[j] = mk(0.0, 0.0);
  __syncwarp();
  const int p0 = ea_ptr[r], p1 = ea_ptr[r + 1];
  const int lines = rs >> 3;
  if (nd <= 16) {
    const int epi = 32 / nd;
    const int sub = lane / nd, b = lane - sub * nd;
    for (int q0 = p0; q0 < p1; q0 += epi) {
      const int pp = q0 + sub;
      dcplx v = mk(0.0, 0.0);
      int j = -1, id = -1;
      if (sub < epi && pp < p1) {
        id = ea[pp];
        if (LF_CHECK(id >= 0 && id < n_erows, BOUNDS_ELEM_ROW)) {
          v = Ae[(size_t)id * rs + b];
          j = off[(size_t)pp * nd + b];
          if (!LF_CHECK(j < nr, BOUNDS_SLOT)) j = -1;
        } else {
          id = -1;
        }
      }
      for (int t = 0; t < epi; ++t) {
        if (sub == t && j >= 0) { acc[j].re += v.re; acc[j].im += v.im; }
        __syncwarp();
      }
      if (id >= 0 && b < lines) discard_l2_line(Ae + (size_t)id * rs + 8 * b);
    }
  } else {
    for (int pp = p0; pp < p1; ++pp) {
      const int id = ea[pp];
      if (!LF_CHECK(id >= 0 && id < n_erows, BOUNDS_ELEM_ROW)) continue;
      const dcplx *src = Ae + (size_t)id * rs;
      const uint16_t *o = off + (size_t)pp * nd;
      for (int b = lane; b < nd; b += 32) {
        const dcplx v = src[b];
        const int j = o[b];
        if (!LF_CHECK(j < nr, BOUNDS_SLOT)) continue;
        acc[j].re += v.re;
        acc[j].im += v.im;
      }
      __syncwarp();  // every lane's loads of this element row are consumed
      if (lane < lines) discard_l2_line(src + 8 * lane);
    }
  }
  if (eliminate && ess[r] && lane == 0) {
    int lo = 0, hi = nr - 1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (Jc[rb + mid] < r) lo = mid + 1; else hi = mid;
    }
    acc[lo] = mk(1.0, 0.0);
  }
  __syncwarp();
  for (int j = lane; j < nr; j += 32) vals[rb + j] = acc[j];
}

// rows longer than cap, in any order
__global__ void k_long_rows(int n, const int *__restrict__ I, int cap, int *__restrict__ out,
                            int *__restrict__ count) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n && I[r + 1] - I[r] > cap) out[atomicAdd(count, 1)] = r;
}

// ---------------------------------------------------------------------------
// symbolic CSR on the device
// ---------------------------------------------------------------------------
__global__ void k_count_rows(long long total, const int *__restrict__ dof, int *__restrict__ cnt) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) atomicAdd(cnt + dof[i], 1);
}

__global__ void k_fill_rows(long long total, const int *__restrict__ dof,
                            const int *__restrict__ ptr, int *__restrict__ fill,
                            int *__restrict__ ea) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) {
    const int r = dof[i];
    ea[ptr[r] + atomicAdd(fill + r, 1)] = (int)i;
  }
}

__global__ void k_max_reduce(int n, const int *__restrict__ ptr, int diff, int *__restrict__ out) {
  // diff != 0: max of ptr[i+1]-ptr[i]; else max of ptr[i]
  int m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    m = max(m, diff ? ptr[i + 1] - ptr[i] : ptr[i]);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Warp-wide bitonic sort of 32 K ints held in registers, element i at
// x[i >> 5] of lane i & 31: partners closer than 32 are exchanged by
// shuffles, farther ones are register swaps inside a lane.
template <int K>
__device__ __forceinline__ void warp_sort_reg(int (&x)[K], int lane) {
#pragma unroll
  for (int k = 2; k <= 32 * K; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
        const int J = j >> 5;
#pragma unroll
        for (int s = 0; s < K; ++s) {
          if ((s & J) == 0) {
            const bool up = ((s << 5) & k) == 0;
            const int a = x[s], b = x[s | J];
            const int lo = min(a, b), hi = max(a, b);
            x[s] = up ? lo : hi;
            x[s | J] = up ? hi : lo;
          }
        }
      } else {
#pragma unroll
        for (int s = 0; s < K; ++s) {
          const bool up = (((s << 5) | lane) & k) == 0;
          const int v = x[s];
          const int o = __shfl_xor_sync(0xffffffffu, v, j);
          x[s] = (((lane & j) == 0) == up) ? min(v, o) : max(v, o);
        }
      }
    }
  }
}

// the row's candidate columns (sentinel-padded to 32 K), sorted in registers
// and compacted to the unique list in buf; returns its length
template <int K>
__device__ __forceinline__ int row_unique_reg(const int *lst, int tot, int nd,
                                              const int *__restrict__ dof, int *buf, int lane) {
  int x[K];
#pragma unroll
  for (int s = 0; s < K; ++s) {
    const int i = (s << 5) | lane;
    int v = 0x7fffffff;
    if (i < tot) {
      const int id = lst[i / nd];
      v = dof[(size_t)(id / nd) * nd + (i % nd)];
    }
    x[s] = v;
  }
  warp_sort_reg<K>(x, lane);
  int nr = 0, last = -1;
#pragma unroll
  for (int s = 0; s < K; ++s) {
    const int v = x[s];
    int prev = __shfl_up_sync(0xffffffffu, v, 1);
    if (lane == 0) prev = last;
    last = __shfl_sync(0xffffffffu, v, 31);
    const bool keep = v != 0x7fffffff && v != prev;
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    if (keep) buf[nr + __popc(bal & ((1u << lane) - 1u))] = v;
    nr += __popc(bal);
  }
  __syncwarp();
  return nr;
}

// one warp per row.  Both passes first sort the row's (element, row) list
// (the gather sums in that order).
// PASS 1: sort the candidate columns (every dof of every listed element),
// padded only to the next power of two of this row's own count; write the
// unique columns to the row's candidate segment of tmpJ (offset
// ea_ptr[r] * nd, which has room for all candidates), their count and the
// slot offsets (positions within the row, independent of where it starts).
// PASS 3: given columns (I/Jcol from the caller): offsets by binary search.
template <int PASS>
__global__ void k_row_symbolic(int n, int nd, const int *__restrict__ dof,
                               const int *__restrict__ ea_ptr, int *__restrict__ ea,
                               int cap, int *__restrict__ cnt, const int *__restrict__ I,
                               const int *__restrict__ Jc, int *__restrict__ tmpJ,
                               uint16_t *__restrict__ off, int *__restrict__ err) {
  extern __shared__ int sh[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int r = blockIdx.x * (blockDim.x >> 5) + wib;
  if (r >= n) return;
  int *buf = sh + (size_t)wib * (cap + 64);
  int *lst = buf + cap;  // up to 64 (element,row) ids
  const int p0 = ea_ptr[r], m = ea_ptr[r + 1] - p0;
  if (m > 64) { if (lane == 0) atomicExch(err, 2); return; }
  if (lane < m) lst[lane] = ea[p0 + lane];
  if (lane + 32 < m) lst[lane + 32] = ea[p0 + lane + 32];
  __syncwarp();
  if (lane == 0) {  // insertion sort (m is small)
    for (int a = 1; a < m; ++a) {
      const int v = lst[a];
      int b = a - 1;
      while (b >= 0 && lst[b] > v) { lst[b + 1] = lst[b]; --b; }
      lst[b + 1] = v;
    }
  }
  __syncwarp();
  if (lane < m) ea[p0 + lane] = lst[lane];
  if (lane + 32 < m) ea[p0 + lane + 32] = lst[lane + 32];
  const int tot = m * nd;
  if (PASS == 3) {
    const int rb = I[r], re = I[r + 1];
    for (int i = lane; i < tot; i += 32) {
      const int id = lst[i / nd];
      const int col = dof[(size_t)(id / nd) * nd + (i % nd)];
      int lo = rb, hi = re;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (Jc[mid] < col) lo = mid + 1; else hi = mid;
      }
      if (lo >= re || Jc[lo] != col) { atomicExch(err, 1); lo = rb; }
      off[(size_t)p0 * nd + i] = (uint16_t)(lo - rb);
    }
    return;
  }
  int len = 32;  // this row's sort length; tot <= cap
  while (len < tot) len <<= 1;
  int nr = 0;
  if (len <= 1024) {
    switch (len) {
      case 32: nr = row_unique_reg<1>(lst, tot, nd, dof, buf, lane); break;
      case 64: nr = row_unique_reg<2>(lst, tot, nd, dof, buf, lane); break;
      case 128: nr = row_unique_reg<4>(lst, tot, nd, dof, buf, lane); break;
      case 256: nr = row_unique_reg<8>(lst, tot, nd, dof, buf, lane); break;
      case 512: nr = row_unique_reg<16>(lst, tot, nd, dof, buf, lane); break;
      default: nr = row_unique_reg<32>(lst, tot, nd, dof, buf, lane); break;
    }
  } else {
    for (int i = lane; i < len; i += 32) {
      int v = 0x7fffffff;
      if (i < tot) {
        const int id = lst[i / nd];
        v = dof[(size_t)(id / nd) * nd + (i % nd)];
      }
      buf[i] = v;
    }
    __syncwarp();
    // bitonic sort (ascending); each lane takes compare pairs (i, i | j)
    for (int k = 2; k <= len; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int pi = lane; pi < (len >> 1); pi += 32) {
          const int i = ((pi & ~(j - 1)) << 1) | (pi & (j - 1));
          const int ixj = i | j;
          const int a = buf[i], b = buf[ixj];
          if ((a > b) == ((i & k) == 0)) { buf[i] = b; buf[ixj] = a; }
        }
        __syncwarp();
      }
    }
    // unique, compacted in place (a chunk writes only at or below what it read)
    int last = -1;
    for (int c0 = 0; c0 < len; c0 += 32) {
      const int v = buf[c0 + lane];
      int prev = __shfl_up_sync(0xffffffffu, v, 1);
      if (lane == 0) prev = last;
      last = __shfl_sync(0xffffffffu, v, 31);
      const bool keep = v != 0x7fffffff && v != prev;
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      __syncwarp();
      if (keep) buf[nr + __popc(bal & ((1u << lane) - 1u))] = v;
      nr += __popc(bal);
      __syncwarp();
    }
  }
  if (lane == 0) cnt[r] = nr;
  int *dst = tmpJ + (size_t)p0 * nd;
  for (int j = lane; j < nr; j += 32) dst[j] = buf[j];
  // offsets: binary search of each candidate in the unique list
  for (int i = lane; i < tot; i += 32) {
    const int id = lst[i / nd];
    const int col = dof[(size_t)(id / nd) * nd + (i % nd)];
    int lo = 0, hi = nr - 1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (buf[mid] < col) lo = mid + 1; else hi = mid;
    }
    off[(size_t)p0 * nd + i] = (uint16_t)lo;
  }
}

// one warp per row: the row's unique columns from its candidate segment of
// tmpJ into the final CSR column array
__global__ void k_row_compact(int n, int nd, const int *__restrict__ ea_ptr,
                              const int *__restrict__ I, const int *__restrict__ tmpJ,
                              int *__restrict__ Jc) {
  const int lane = threadIdx.x & 31;
  const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= n) return;
  const int *src = tmpJ + (size_t)ea_ptr[r] * nd;
  const int rb = I[r], len = I[r + 1] - rb;
  for (int j = lane; j < len; j += 32) Jc[rb + j] = src[j];
}

// ---------------------------------------------------------------------------
// init-time passes over the uploaded element arrays
// ---------------------------------------------------------------------------
// per element: the four face orientation codes in one word (8 bits each)
// and the dof sign bits
__global__ void k_pack(int ne, int nd, int p, const double *__restrict__ sign,
                       const int *__restrict__ fo, unsigned *__restrict__ fopack,
                       unsigned long long *__restrict__ signmask) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  unsigned f = 0u;
  if (p >= 2)
    for (int k = 0; k < 4; ++k) f |= (unsigned)fo[(size_t)e * 4 + k] << (8 * k);
  unsigned long long m = 0ull;
  for (int k = 0; k < nd; ++k)
    if (sign[(size_t)e * nd + k] < 0.0) m |= 1ull << k;
  fopack[e] = f;
  signmask[e] = m;
}

// bulk iff every quadrature point of both rules has z_min <= z <= z_max
// (the stretch is then exactly 1); z is formed with explicit roundings, in
// the order z0 + J20 x + J21 y + J22 z, so that the result does not depend on
// multiply-add contraction.  flag[e] = 1 for bulk; region_has_bulk marks the
// regions that own a bulk element.
__global__ void k_classify(int ne, Rule rcc, Rule rm, const double *__restrict__ J9,
                           const double *__restrict__ v0, const int *__restrict__ attr,
                           double z_min, double z_max, int *__restrict__ flag,
                           int *__restrict__ region_has_bulk) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const double z0 = v0[(size_t)e * 3 + 2];
  const double a = J9[(size_t)e * 9 + 6], b = J9[(size_t)e * 9 + 7], c = J9[(size_t)e * 9 + 8];
  bool bulk = true;
  for (int rr = 0; rr < 2 && bulk; ++rr) {
    const Rule &R = rr == 0 ? rcc : rm;
    for (int q = 0; q < R.nq && bulk; ++q) {
      const double z = __dadd_rn(__dadd_rn(__dadd_rn(z0, __dmul_rn(a, R.ip[q * 3])),
                                           __dmul_rn(b, R.ip[q * 3 + 1])),
                                 __dmul_rn(c, R.ip[q * 3 + 2]));
      if (z < z_min || z > z_max) bulk = false;
    }
  }
  flag[e] = bulk ? 1 : 0;
  if (bulk) region_has_bulk[attr[e] - 1] = 1;
}

// ordered split of 0..ne-1 into the bulk and PML lists from the exclusive
// scan of the bulk flags
__global__ void k_split_lists(int ne, const int *__restrict__ flag, const int *__restrict__ pos,
                              int *__restrict__ bulk_list, int *__restrict__ pml_list) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  if (flag[e]) bulk_list[pos[e]] = e;
  else pml_list[e - pos[e]] = e;
}

__global__ void k_essmask(int ne, int nd, const int *__restrict__ dof,
                          const unsigned char *__restrict__ ess,
                          unsigned long long *__restrict__ mask) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  unsigned long long m = 0ull;
  for (int k = 0; k < nd; ++k)
    if (ess[dof[(size_t)e * nd + k]]) m |= 1ull << k;
  mask[e] = m;
}

// ---------------------------------------------------------------------------
// CSR SpMV with fused residual partial norms (warp per row)
// ---------------------------------------------------------------------------
__global__ void k_spmv_resid(int n, const int *__restrict__ I, const int *__restrict__ Jc,
                             const dcplx *__restrict__ vals, const dcplx *__restrict__ x,
                             const dcplx *__restrict__ b, dcplx *__restrict__ y,
                             double *__restrict__ partials) {
  __shared__ double red[2][32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int r = blockIdx.x * (blockDim.x >> 5) + wib;
  double rn = 0.0, bn = 0.0;
  if (r < n) {
    double ar = 0.0, ai = 0.0;
    for (int k = I[r] + lane; k < I[r + 1]; k += 32) {
      const dcplx a = vals[k], xv = x[Jc[k]];
      ar = fma(a.re, xv.re, ar); ar = fma(-a.im, xv.im, ar);
      ai = fma(a.re, xv.im, ai); ai = fma(a.im, xv.re, ai);
    }
    for (int o = 16; o; o >>= 1) {
      ar += __shfl_xor_sync(0xffffffffu, ar, o);
      ai += __shfl_xor_sync(0xffffffffu, ai, o);
    }
    if (lane == 0) {
      if (y) y[r] = mk(ar, ai);
      if (b) {
        const dcplx bv = b[r];
        const double dr = ar - bv.re, di = ai - bv.im;
        rn = dr * dr + di * di;
        bn = bv.re * bv.re + bv.im * bv.im;
      }
    }
  }
  if (!partials) return;
  if (lane == 0) { red[0][wib] = rn; red[1][wib] = bn; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { s0 += red[0][w]; s1 += red[1][w]; }
    partials[2 * blockIdx.x] = s0;
    partials[2 * blockIdx.x + 1] = s1;
  }
}

__global__ void k_sum_partials(int nblk, const double *__restrict__ partials,
                               double *__restrict__ out) {
  __shared__ double red[2][32];
  double s0 = 0.0, s1 = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
    s0 += partials[2 * i];
    s1 += partials[2 * i + 1];
  }
  for (int o = 16; o; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { red[0][w] = s0; red[1][w] = s1; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, c = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { a += red[0][i]; c += red[1][i]; }
    out[0] = a;
    out[1] = c;
  }
}

// host [re; im] halves <-> interleaved
__global__ void k_split_to_cplx(int n, const double *__restrict__ h2n, dcplx *__restrict__ z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = mk(h2n[i], h2n[n + i]);
}

// ---------------------------------------------------------------------------
// scattered-field RHS (ScatterSource, problem_common.inc:218-266)
// ---------------------------------------------------------------------------
struct SlabWaveD {
  dcplx qA, qB;
  double zA, zB;
  dcplx A[3], B[3];
};

// one warp per source element; lanes over local dofs
__global__ void k_rhs_elem(int nsrc, const int *__restrict__ list, int nd, int p, Rule rm,
                           const double *__restrict__ J9, const double *__restrict__ Ji9,
                           const double *__restrict__ detJ, const double *__restrict__ v0,
                           const int *__restrict__ slab_of, const dcplx *__restrict__ delta,
                           const SlabWaveD *__restrict__ waves, int n_slab, int n_parts,
                           const int *__restrict__ col_of_part, int ncol, double k0,
                           const unsigned *__restrict__ fopack, dcplx *__restrict__ be) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= nsrc) return;
  const int e = list[i];
  double J[9], Ji[9];
  for (int t = 0; t < 9; ++t) { J[t] = J9[(size_t)e * 9 + t]; Ji[t] = Ji9[(size_t)e * 9 + t]; }
  const double det = detJ[e];
  const double x0[3] = {v0[(size_t)e * 3], v0[(size_t)e * 3 + 1], v0[(size_t)e * 3 + 2]};
  const int slab = slab_of[e];
  const dcplx fac = cscale(k0 * k0, delta[e]);
  const unsigned fp = fopack ? fopack[e] : 0u;
  for (int c = 0; c < ncol; ++c) {
    for (int kb = 0; kb < nd; kb += 32) {
      const int k = kb + lane;
      double br = 0.0, bi = 0.0;
      for (int q = 0; q < rm.nq; ++q) {
        const double *xi = rm.ip + q * 3;
        const double z = x0[2] + J[6] * xi[0] + J[7] * xi[1] + J[8] * xi[2];
        dcplx ev[3] = {mk(0, 0), mk(0, 0), mk(0, 0)};
        for (int pi = 0; pi < n_parts; ++pi) {
          if (col_of_part[pi] != c) continue;
          const SlabWaveD &sw = waves[(size_t)pi * n_slab + slab];
          // exp(i q (z - zA)) = exp(-Im(q) dz) (cos(Re(q) dz) + i sin(Re(q) dz))
          const double da = z - sw.zA, db = z - sw.zB;
          const double ma = exp(-sw.qA.im * da), mb = exp(-sw.qB.im * db);
          double sa, ca, sb, cb;
          sincos(sw.qA.re * da, &sa, &ca);
          sincos(sw.qB.re * db, &sb, &cb);
          const dcplx up = mk(ma * ca, ma * sa), dn = mk(mb * cb, mb * sb);
          for (int d = 0; d < 3; ++d)
            ev[d] = cadd(ev[d], cadd(cmul(sw.A[d], up), cmul(sw.B[d], dn)));
        }
        const double w = rm.w[q] * det;
        if (k < nd) {
          const double *rv = rm.v + ((size_t)q * nd + k) * 3;
          for (int d = 0; d < 3; ++d) {
            const double pv = rv[0] * Ji[0 * 3 + d] + rv[1] * Ji[1 * 3 + d] + rv[2] * Ji[2 * 3 + d];
            const dcplx f = cmul(fac, ev[d]);
            br += w * pv * f.re;
            bi += w * pv * f.im;
          }
        }
      }
      // dual transform on the element vector: b <- M^T b on face pairs
      const double obr = __shfl_xor_sync(0xffffffffu, br, 1);
      const double obi = __shfl_xor_sync(0xffffffffu, bi, 1);
      const int f = (p >= 2 && k < nd) ? face_of(k & ~1, p) : -1;
      if (f >= 0) {
        const double *T = c_tinv + 4 * ((fp >> (8 * f)) & 0xffu);
        const int cp = k & 1;
        const double own = T[2 * cp + cp], oth = T[2 * cp + (1 - cp)];
        const double nr = own * br + oth * obr, ni = own * bi + oth * obi;
        br = nr; bi = ni;
      }
      if (k < nd) be[((size_t)i * ncol + c) * nd + k] = mk(br, bi);
    }
  }
}

__global__ void k_rhs_gather(int n, const int *__restrict__ ea_ptr, const int *__restrict__ ea,
                             int nd, const int *__restrict__ src_slot,
                             const double *__restrict__ sign, const dcplx *__restrict__ be,
                             int ncol, const unsigned char *__restrict__ ess, int eliminate,
                             dcplx *__restrict__ b) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  for (int c = 0; c < ncol; ++c) {
    double br = 0.0, bi = 0.0;
    if (!(eliminate && ess[r])) {
      for (int pp = ea_ptr[r]; pp < ea_ptr[r + 1]; ++pp) {
        const int id = ea[pp];
        const int e = id / nd, a = id - e * nd;
        const int s = src_slot[e];
        if (s < 0) continue;
        const dcplx v = be[((size_t)s * ncol + c) * nd + a];
        br += sign[id] * v.re;
        bi += sign[id] * v.im;
      }
    }
    b[(size_t)c * n + r] = mk(br, bi);
  }
}

// ---------------------------------------------------------------------------
// Adjoint contraction for per-element permittivity (one warp per element).
//
// For l(u) = c^T u with A(eps) u = b(eps) and A^T lambda = c:
//   dl/deps_e = lambda^T (db/deps_e - dA/deps_e u)
//             = k0^2 sum_q w_q detJ [ sum_i Lam_i (lt . v_i)(ut . v_i)
//                                     + src_e sum_i (lt . v_i) Ehat_i(z_q) ]
// with dA_e/deps_e = -k0^2 M_e^Lambda (the mass integrator,
// problem_common.inc:123-148), db_e/deps_e = k0^2 int v . Ehat
// (ScatterSource, problem_common.inc:238-266), Lam = (s, s, 1/s), v the
// physical shapes and lt, ut the element-local coefficients of lambda and u
// (signs and the face transform applied: local = M (sign * global)).
// ---------------------------------------------------------------------------
__global__ void k_eps_grad(int nsel, const int *__restrict__ list, int nd, int p, Rule rm,
                           const double *__restrict__ J9, const double *__restrict__ Ji9,
                           const double *__restrict__ detJ, const double *__restrict__ v0,
                           const int *__restrict__ dof, const double *__restrict__ sign,
                           const unsigned *__restrict__ fopack, PmlParams pml,
                           const int *__restrict__ slab_of, const SlabWaveD *__restrict__ waves,
                           int n_slab, int n_parts, const dcplx *__restrict__ u,
                           const dcplx *__restrict__ lam, dcplx *__restrict__ grad) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= nsel) return;
  const int e = list[i];
  double J[9], Ji[9];
  for (int t = 0; t < 9; ++t) { J[t] = J9[(size_t)e * 9 + t]; Ji[t] = Ji9[(size_t)e * 9 + t]; }
  const double det = detJ[e];
  const double z0 = v0[(size_t)e * 3 + 2];
  const unsigned fp = fopack ? fopack[e] : 0u;
  // local coefficients for k = lane and k = lane + 32
  dcplx lt[2], ut[2];
  for (int hh = 0; hh < 2; ++hh) {
    const int k = lane + 32 * hh;
    dcplx lg = mk(0, 0), ug = mk(0, 0);
    if (k < nd) {
      const double sg = sign[(size_t)e * nd + k];
      const int d = dof[(size_t)e * nd + k];
      lg = cscale(sg, lam[d]);
      ug = cscale(sg, u[d]);
    }
    // face pairs: local = M global, M[r][c] = T[2c + r] (column-major)
    const double olr = __shfl_xor_sync(0xffffffffu, lg.re, 1);
    const double oli = __shfl_xor_sync(0xffffffffu, lg.im, 1);
    const double our = __shfl_xor_sync(0xffffffffu, ug.re, 1);
    const double oui = __shfl_xor_sync(0xffffffffu, ug.im, 1);
    const int f = (p >= 2 && k < nd) ? face_of(k & ~1, p) : -1;
    if (f >= 0) {
      const double *T = c_tinv + 4 * ((fp >> (8 * f)) & 0xffu);
      const int r = k & 1;
      const double own = T[2 * r + r], oth = T[2 * (1 - r) + r];
      lg = mk(own * lg.re + oth * olr, own * lg.im + oth * oli);
      ug = mk(own * ug.re + oth * our, own * ug.im + oth * oui);
    }
    lt[hh] = lg;
    ut[hh] = ug;
  }
  const int slab = slab_of[e];
  double gr = 0.0, gi = 0.0;
  for (int q = 0; q < rm.nq; ++q) {
    dcplx Lv[3] = {mk(0, 0), mk(0, 0), mk(0, 0)}, Uv[3] = {mk(0, 0), mk(0, 0), mk(0, 0)};
    for (int hh = 0; hh < 2; ++hh) {
      const int k = lane + 32 * hh;
      if (k >= nd) continue;
      const double *rv = rm.v + ((size_t)q * nd + k) * 3;
      for (int d = 0; d < 3; ++d) {
        const double pv = rv[0] * Ji[0 * 3 + d] + rv[1] * Ji[1 * 3 + d] + rv[2] * Ji[2 * 3 + d];
        Lv[d] = cadd(Lv[d], cscale(pv, lt[hh]));
        Uv[d] = cadd(Uv[d], cscale(pv, ut[hh]));
      }
    }
    for (int o = 16; o; o >>= 1)
      for (int d = 0; d < 3; ++d) {
        Lv[d].re += __shfl_xor_sync(0xffffffffu, Lv[d].re, o);
        Lv[d].im += __shfl_xor_sync(0xffffffffu, Lv[d].im, o);
        Uv[d].re += __shfl_xor_sync(0xffffffffu, Uv[d].re, o);
        Uv[d].im += __shfl_xor_sync(0xffffffffu, Uv[d].im, o);
      }
    if (lane == 0) {
      const double *xi = rm.ip + q * 3;
      const double z = z0 + J[6] * xi[0] + J[7] * xi[1] + J[8] * xi[2];
      const dcplx s = pml_s(pml, z);
      const dcplx Lam[3] = {s, s, cinv(s)};
      dcplx acc = mk(0, 0);
      for (int d = 0; d < 3; ++d) acc = cadd(acc, cmul(Lam[d], cmul(Lv[d], Uv[d])));
      if (slab >= 0 && n_parts > 0) {
        dcplx ev[3] = {mk(0, 0), mk(0, 0), mk(0, 0)};
        for (int pi = 0; pi < n_parts; ++pi) {
          const SlabWaveD &sw = waves[(size_t)pi * n_slab + slab];
          const double da = z - sw.zA, db = z - sw.zB;
          const double ma = exp(-sw.qA.im * da), mb = exp(-sw.qB.im * db);
          double sa, ca, sb, cb;
          sincos(sw.qA.re * da, &sa, &ca);
          sincos(sw.qB.re * db, &sb, &cb);
          const dcplx up = mk(ma * ca, ma * sa), dn = mk(mb * cb, mb * sb);
          for (int d = 0; d < 3; ++d)
            ev[d] = cadd(ev[d], cadd(cmul(sw.A[d], up), cmul(sw.B[d], dn)));
        }
        for (int d = 0; d < 3; ++d) acc = cadd(acc, cmul(Lv[d], ev[d]));
      }
      const double w = rm.w[q] * det;
      gr += w * acc.re;
      gi += w * acc.im;
    }
  }
  if (lane == 0) {
    const double k2 = pml.k0 * pml.k0;
    grad[e] = mk(k2 * gr, k2 * gi);
  }
}

// ---------------------------------------------------------------------------
// Field sampling on a z-plane (the reference's plane sampler,
// solver/lithofem_solve.cpp:951-1004) and the adjoint seed of one Fourier
// order of the samples (src/lithofem/orders.py:36-67).
// ---------------------------------------------------------------------------
constexpr int BASIS_MAX_MONO = 20;  // monomials of degree <= 3

struct PlaneGrid {
  double lx, ly, z;
  int nx, ny;
};

// sample point (i, j) of a plane at height z: cell-centred with the
// reference's fixed nudges
__device__ __forceinline__ void plane_point(const PlaneGrid &G, int pt, double z, double x[3]) {
  const int i = pt % G.nx, j = pt / G.nx;
  x[0] = (i + 0.5) * G.lx / G.nx + 3.1e-7;
  x[1] = (j + 0.5) * G.ly / G.ny + 1.7e-7;
  x[2] = z - 4.9e-7;
}

// elements whose z-range contains the nudged height of plane iz (vertex
// z = v0z + J20 / J21 / J22); flags [iz][e] for nz planes
__global__ void k_plane_cand(int ne, int nz, const double *__restrict__ J9,
                             const double *__restrict__ v0, const double *__restrict__ zs,
                             int *__restrict__ flag) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)ne * nz) return;
  const int e = (int)(t % ne), iz = (int)(t / ne);
  const double z = zs[iz] - 4.9e-7;
  const double z0 = v0[(size_t)e * 3 + 2];
  double lo = z0, hi = z0;
  for (int c = 0; c < 3; ++c) {
    const double zc = z0 + J9[(size_t)e * 9 + 6 + c];
    lo = fmin(lo, zc);
    hi = fmax(hi, zc);
  }
  const double tol = 1e-9 * (1.0 + fabs(z));
  flag[t] = (z >= lo - tol && z <= hi + tol) ? 1 : 0;
}

__global__ void k_compact(int n, const int *__restrict__ flag, const int *__restrict__ pos,
                          int *__restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n && flag[e]) out[pos[e]] = e;
}

// one warp per sample point of nz planes (point pt of plane pt / (nx ny)):
// the candidate element of its plane (cand[pos[iz ne] .. pos[(iz + 1) ne]))
// in which the point is most interior (largest smallest barycentric
// coordinate; lower index on a tie) and the point's reference coordinates;
// *missing counts points that lie outside every candidate
__global__ void k_plane_locate(PlaneGrid G, int nz, const double *__restrict__ zs, int ne,
                               const int *__restrict__ pos, const int *__restrict__ cand,
                               const double *__restrict__ Ji9, const double *__restrict__ v0,
                               int *__restrict__ elem, double *__restrict__ xi,
                               int *__restrict__ missing) {
  const int lane = threadIdx.x & 31;
  const int npts = G.nx * G.ny;
  const long long ptg = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5);
  if (ptg >= (long long)npts * nz) return;
  const int iz = (int)(ptg / npts), pt = (int)ptg;
  double x[3];
  plane_point(G, pt % npts, zs[iz], x);
  double best = -1e300;
  int be = 0x7fffffff;
  // the compaction kept flattened (plane, element) indices iz ne + e
  const int c0 = pos[(size_t)iz * ne], c1 = pos[(size_t)(iz + 1) * ne];
  for (int i = c0 + lane; i < c1; i += 32) {
    const int e = cand[i] - iz * ne;
    const double *Ji = Ji9 + (size_t)e * 9;
    const double d0 = x[0] - v0[(size_t)e * 3], d1 = x[1] - v0[(size_t)e * 3 + 1],
                 d2 = x[2] - v0[(size_t)e * 3 + 2];
    const double a = Ji[0] * d0 + Ji[1] * d1 + Ji[2] * d2;
    const double b = Ji[3] * d0 + Ji[4] * d1 + Ji[5] * d2;
    const double c = Ji[6] * d0 + Ji[7] * d1 + Ji[8] * d2;
    const double m = fmin(fmin(1.0 - a - b - c, a), fmin(b, c));
    if (m > best || (m == best && e < be)) { best = m; be = e; }
  }
  for (int o = 16; o; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int oe = __shfl_xor_sync(0xffffffffu, be, o);
    if (ob > best || (ob == best && oe < be)) { best = ob; be = oe; }
  }
  if (lane == 0) {
    if (be == 0x7fffffff || best < -1e-9) {
      atomicAdd(missing, 1);
      elem[pt] = -1;
      return;
    }
    elem[pt] = be;
    const double *Ji = Ji9 + (size_t)be * 9;
    const double d0 = x[0] - v0[(size_t)be * 3], d1 = x[1] - v0[(size_t)be * 3 + 1],
                 d2 = x[2] - v0[(size_t)be * 3 + 2];
    xi[pt * 3 + 0] = Ji[0] * d0 + Ji[1] * d1 + Ji[2] * d2;
    xi[pt * 3 + 1] = Ji[3] * d0 + Ji[4] * d1 + Ji[5] * d2;
    xi[pt * 3 + 2] = Ji[6] * d0 + Ji[7] * d1 + Ji[8] * d2;
  }
}

// Global basis functions of element e at reference point xi for the pair of
// local functions (2 pr, 2 pr + 1): physical values psi (covariant map,
// v J^-1) and physical curls (J c / detJ), with the face transform applied
// like in the element kernels.  k >= nd gives zeros.
__device__ __forceinline__ void basis_pair(int e, int pr, const double *xi, int nd, int p,
                                           int nmono, const int *__restrict__ exps,
                                           const double *__restrict__ coef,
                                           const double *__restrict__ ccoef,
                                           const double *__restrict__ J9,
                                           const double *__restrict__ Ji9,
                                           const double *__restrict__ detJ, unsigned fo,
                                           double v[2][3], double c[2][3]) {
  double mono[BASIS_MAX_MONO];
  for (int m = 0; m < nmono; ++m) {
    double t = 1.0;
    for (int a = 0; a < exps[3 * m + 0]; ++a) t *= xi[0];
    for (int a = 0; a < exps[3 * m + 1]; ++a) t *= xi[1];
    for (int a = 0; a < exps[3 * m + 2]; ++a) t *= xi[2];
    mono[m] = t;
  }
  const double *J = J9 + (size_t)e * 9, *Ji = Ji9 + (size_t)e * 9;
  const double idet = 1.0 / detJ[e];
  for (int h = 0; h < 2; ++h) {
    const int k = 2 * pr + h;
    double r[3] = {0.0, 0.0, 0.0}, q[3] = {0.0, 0.0, 0.0};
    if (k < nd)
      for (int d = 0; d < 3; ++d)
        for (int m = 0; m < nmono; ++m) {
          r[d] += coef[((size_t)k * 3 + d) * nmono + m] * mono[m];
          q[d] += ccoef[((size_t)k * 3 + d) * nmono + m] * mono[m];
        }
    for (int d = 0; d < 3; ++d) {
      v[h][d] = r[0] * Ji[0 * 3 + d] + r[1] * Ji[1 * 3 + d] + r[2] * Ji[2 * 3 + d];
      c[h][d] = (J[d * 3 + 0] * q[0] + J[d * 3 + 1] * q[1] + J[d * 3 + 2] * q[2]) * idet;
    }
  }
  if (p >= 2) {
    const int f = face_of(2 * pr, p);
    if (f >= 0) {
      const double *T = c_tinv + 4 * ((fo >> (8 * f)) & 0xffu);
      for (int d = 0; d < 3; ++d) {
        const double v0_ = v[0][d], v1_ = v[1][d], c0_ = c[0][d], c1_ = c[1][d];
        v[0][d] = v0_ * T[0] + v1_ * T[1];
        v[1][d] = v0_ * T[2] + v1_ * T[3];
        c[0][d] = c0_ * T[0] + c1_ * T[1];
        c[1][d] = c0_ * T[2] + c1_ * T[3];
      }
    }
  }
}

// one warp per sample point: E and curl E of u (global coefficients, dof
// signs) at the located point; out layout [pt][3] complex
__global__ void k_plane_eval(int npts, const int *__restrict__ elem, const double *__restrict__ xi,
                             int nd, int p, int nmono, const int *__restrict__ exps,
                             const double *__restrict__ coef, const double *__restrict__ ccoef,
                             const int *__restrict__ dof, const double *__restrict__ sign,
                             const unsigned *__restrict__ fopack, const double *__restrict__ J9,
                             const double *__restrict__ Ji9, const double *__restrict__ detJ,
                             const dcplx *__restrict__ u, dcplx *__restrict__ E,
                             dcplx *__restrict__ curlE) {
  const int lane = threadIdx.x & 31;
  const int pt = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (pt >= npts) return;
  const int e = elem[pt];
  double acc[12];
  for (int i = 0; i < 12; ++i) acc[i] = 0.0;
  const int npair = (nd + 1) / 2;
  if (e >= 0 && lane < npair) {
    double v[2][3], c[2][3];
    basis_pair(e, lane, xi + (size_t)pt * 3, nd, p, nmono, exps, coef, ccoef, J9, Ji9, detJ,
               fopack[e], v, c);
    for (int h = 0; h < 2; ++h) {
      const int k = 2 * lane + h;
      if (k >= nd) continue;
      const dcplx g = u[dof[(size_t)e * nd + k]];
      const double s = sign[(size_t)e * nd + k];
      for (int d = 0; d < 3; ++d) {
        acc[2 * d] += s * g.re * v[h][d];
        acc[2 * d + 1] += s * g.im * v[h][d];
        acc[6 + 2 * d] += s * g.re * c[h][d];
        acc[6 + 2 * d + 1] += s * g.im * c[h][d];
      }
    }
  }
  for (int i = 0; i < 12; ++i)
    for (int o = 16; o; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
  if (lane == 0) {
    for (int d = 0; d < 3; ++d) {
      if (E) E[(size_t)pt * 3 + d] = mk(acc[2 * d], acc[2 * d + 1]);
      if (curlE) curlE[(size_t)pt * 3 + d] = mk(acc[6 + 2 * d], acc[6 + 2 * d + 1]);
    }
  }
}

// adjoint seed of the (m, q) Fourier coefficient of component comp of the
// sampled E: c[dof_k] += sign_k psi_k(x_pt)[comp] exp(-2 pi i (m i/nx + q j/ny)) / (nx ny)
__global__ void k_plane_seed(PlaneGrid G, const int *__restrict__ elem,
                             const double *__restrict__ xi, int nd, int p, int nmono,
                             const int *__restrict__ exps, const double *__restrict__ coef,
                             const double *__restrict__ ccoef, const int *__restrict__ dof,
                             const double *__restrict__ sign, const unsigned *__restrict__ fopack,
                             const double *__restrict__ J9, const double *__restrict__ Ji9,
                             const double *__restrict__ detJ, int comp, int m, int q,
                             double *__restrict__ cvec) {
  const int lane = threadIdx.x & 31;
  const int npts = G.nx * G.ny;
  const int pt = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (pt >= npts) return;
  const int e = elem[pt];
  const int npair = (nd + 1) / 2;
  if (e < 0 || lane >= npair) return;
  const int i = pt % G.nx, j = pt / G.nx;
  // phase -2 pi (m i / nx + q j / ny), reduced to one period first
  const long long num = ((long long)m * i * G.ny + (long long)q * j * G.nx) %
                        ((long long)G.nx * G.ny);
  const double ang = -2.0 * 3.141592653589793238 * (double)num / ((double)G.nx * G.ny);
  double sn, cs;
  sincos(ang, &sn, &cs);
  const double inv = 1.0 / npts;
  double v[2][3], c[2][3];
  basis_pair(e, lane, xi + (size_t)pt * 3, nd, p, nmono, exps, coef, ccoef, J9, Ji9, detJ,
             fopack[e], v, c);
  for (int h = 0; h < 2; ++h) {
    const int k = 2 * lane + h;
    if (k >= nd) continue;
    const double w = sign[(size_t)e * nd + k] * v[h][comp] * inv;
    double *dst = cvec + 2 * (size_t)dof[(size_t)e * nd + k];
    atomicAdd(dst, w * cs);
    atomicAdd(dst + 1, w * sn);
  }
}

// ---------------------------------------------------------------------------
// Fourier orders of sampled planes and their efficiencies (the reference's
// orders_from_plane and order efficiency, src/lithofem/orders.py:36-67 and
// src/lithofem/outputs.py:219-269).  Block (order o, plane iz): the
// coefficient c = (1 / (nx ny)) sum_{j,i} E(x_ij) exp(-2 pi i (a i / nx +
// b j / ny)) of the order at grid index o = b nx + a (order m = a, or
// a - nx above nx / 2; n likewise), its qz = sqrt(k0^2 eps - kx^2 - ky^2)
// with Im qz >= 0, and the efficiency of the coefficient carried to the
// reference plane, c' = c exp(-i d qz (z - z_ref)) (+ the analytic (0,0)
// background there): d Re[(c' x conj(k x c' / k0))_z] area / (2 inc_flux),
// k = (kx, ky, d qz), d = +1 (reflection side) or -1 (transmission side).
// ---------------------------------------------------------------------------
struct OrderArgs {
  double lx, ly, k0, kx, ky, inc_flux;
};
constexpr int ORDER_THREADS = 128;

// principal square root (Re >= 0), the half-angle formulas evaluated
// without cancellation on either sign of the real part
__device__ __forceinline__ dcplx csqrt_principal(dcplx w) {
  const double r = hypot(w.re, w.im);
  if (r == 0.0) return mk(0.0, 0.0);
  if (w.re >= 0.0) {
    const double t = sqrt(0.5 * (r + w.re));
    return mk(t, w.im / (2.0 * t));
  }
  const double t = sqrt(0.5 * (r - w.re));
  return mk(fabs(w.im) / (2.0 * t), copysign(t, w.im));
}

// rows of 10 (z, z_ref, eps re/im, background 3 complex) to separate arrays
__global__ void k_unpack_planes(int nz, const double *__restrict__ rows, double *__restrict__ z,
                                double *__restrict__ zref, double *__restrict__ eps2,
                                double *__restrict__ bg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nz) return;
  const double *r = rows + (size_t)i * 10;
  z[i] = r[0];
  zref[i] = r[1];
  eps2[2 * i] = r[2];
  eps2[2 * i + 1] = r[3];
  for (int c = 0; c < 6; ++c) bg[6 * i + c] = r[4 + c];
}

__global__ void __launch_bounds__(ORDER_THREADS)
k_plane_orders(int nx, int ny, const dcplx *__restrict__ E, const double *__restrict__ zs,
               const double *__restrict__ zref, const int *__restrict__ dirs,
               const double *__restrict__ eps2, const double *__restrict__ bg, OrderArgs A,
               dcplx *__restrict__ coef, double *__restrict__ eff) {
  const int npts = nx * ny, o = blockIdx.x, iz = blockIdx.y;
  const int a = o % nx, b = o / nx;
  const dcplx *Ez = E + (size_t)iz * npts * 3;
  const long long per = (long long)nx * ny;
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (int pt = threadIdx.x; pt < npts; pt += ORDER_THREADS) {
    const int i = pt % nx, j = pt / nx;
    // phase -2 pi (a i / nx + b j / ny), reduced to one period first
    const long long num = ((long long)a * i * ny + (long long)b * j * nx) % per;
    double sn, cs;
    sincospi(-2.0 * (double)num / (double)per, &sn, &cs);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const dcplx u = Ez[(size_t)pt * 3 + c];
      s[2 * c] += u.re * cs - u.im * sn;
      s[2 * c + 1] += u.re * sn + u.im * cs;
    }
  }
  __shared__ double red[6][ORDER_THREADS];
#pragma unroll
  for (int q = 0; q < 6; ++q) red[q][threadIdx.x] = s[q];
  __syncthreads();
  for (int w = ORDER_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int q = 0; q < 6; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x) return;
  const double inv = 1.0 / (double)npts;
  dcplx c[3];
  for (int q = 0; q < 3; ++q) {
    c[q] = mk(red[2 * q][0] * inv, red[2 * q + 1][0] * inv);
    coef[((size_t)iz * npts + o) * 3 + q] = c[q];
  }
  const int m = a <= nx / 2 ? a : a - nx, n = b <= ny / 2 ? b : b - ny;
  const double kx = A.kx + 2.0 * 3.141592653589793238 / A.lx * m;
  const double ky = A.ky + 2.0 * 3.141592653589793238 / A.ly * n;
  const dcplx ep = mk(eps2[2 * iz], eps2[2 * iz + 1]);
  dcplx qz = csqrt_principal(mk(A.k0 * A.k0 * ep.re - kx * kx - ky * ky, A.k0 * A.k0 * ep.im));
  if (qz.im < 0.0) qz = mk(-qz.re, -qz.im);
  const int d = dirs[iz];
  // c' = c exp(-i d qz dz) = c e^{d dz Im qz} (cos(d dz Re qz) - i sin(d dz Re qz))
  const double dz = zs[iz] - zref[iz];
  const double g = exp(d * dz * qz.im);
  double sn, cs;
  sincos(d * dz * qz.re, &sn, &cs);
  const dcplx ph = mk(g * cs, -g * sn);
  for (int q = 0; q < 3; ++q) {
    c[q] = cmul(c[q], ph);
    if (m == 0 && n == 0 && bg) c[q] = cadd(c[q], mk(bg[6 * iz + 2 * q], bg[6 * iz + 2 * q + 1]));
  }
  const dcplx kz = mk(d * qz.re, d * qz.im);
  // h = k x c / k0 (x and y components)
  const dcplx hx = cscale(1.0 / A.k0, cadd(cscale(ky, c[2]), cscale(-1.0, cmul(kz, c[1]))));
  const dcplx hy = cscale(1.0 / A.k0, cadd(cmul(kz, c[0]), cscale(-kx, c[2])));
  // Re[(c x conj(h))_z] = Re[c_x conj(h_y) - c_y conj(h_x)]
  const double sz = (c[0].re * hy.re + c[0].im * hy.im) - (c[1].re * hx.re + c[1].im * hx.im);
  eff[(size_t)iz * npts + o] = d * 0.5 * sz * A.lx * A.ly / A.inc_flux;
}

}  // namespace lfasm_dev
