// Test-infrastructure build of the REFERENCE assembly code, compiled from the
// reference tree's own files (solver/problem_common.inc, asm_data.inc,
// asm_gpu.inc; included, never copied) against mfem_shim.hpp, and exposed
// through a small C API for the parity tests and the CPU baseline:
//
//   ref_set_problem       fills the reference's global `prob`
//                         (Problem/Region, problem_common.inc:18-67)
//   ref_ctx_create        builds the reference's AsmData (asm_data.inc:77-97)
//                         from caller arrays (the MFEM extraction step is
//                         replaced by the caller's own extraction)
//   ref_ctx_build_csr     build_csr_symbolic   (asm_data.inc:178-210)
//   ref_ctx_reassemble    reassemble_all       (asm_data.inc:374-402)
//   ref_ctx_element       reassemble_element   (asm_data.inc:218-370)
//   ref_ctx_gpu_local     AsmGpu::Init + ComputeLocal + DownloadLocal
//   ref_ctx_gpu_global    AsmGpuGlobal::BuildGlobal + ScatterEliminate
//   ref_ctx_set_csr       a caller-given CSR for the context (element shares)
//   ref_set_incident      the incident tables of the global problem
//   ref_incident_at       incident_at          (problem_common.inc:219-236)
//   ref_scatter_source    ScatterSource::Eval  (problem_common.inc:239-266)
//
// Built by oracle/Makefile into oracle/_ref/libref_asm.so.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "mfem_shim.hpp"
#include "thirdparty/json.hpp"

using namespace mfem;
using json = nlohmann::json;
using C = std::complex<double>;

namespace {
#include "problem_common.inc"
#include "asm_data.inc"
#include "asm_gpu.inc"
#include "ref_fill.inc"
}  // namespace


extern "C" {

int ref_set_problem(double k0, double kx, double ky, double z_min, double z_max,
                    double pml_thick, double pml_order, double pml_target, int order,
                    int n_regions, const double *eps, const int *kind, const int *slab,
                    const double *delta_eps) {
  return fill_problem(k0, kx, ky, z_min, z_max, pml_thick, pml_order, pml_target, order,
                      n_regions, eps, kind, slab, delta_eps);
}

void *ref_ctx_create(int ne, int nd, int p, int height, const int *dof, const double *sign,
                     const int *fo, const int *attr, const double *J, const double *Jinv,
                     const double *detJ, const double *v0, int nq_cc, const double *ip_cc,
                     const double *w_cc, const double *v_cc, const double *c_cc, int nq_m,
                     const double *ip_m, const double *w_m, const double *v_m,
                     const double *c_m) {
  return make_asm_data(ne, nd, p, height, dof, sign, fo, attr, J, Jinv, detJ, v0, nq_cc, ip_cc,
                       w_cc, v_cc, c_cc, nq_m, ip_m, w_m, v_m, c_m);
}

void ref_ctx_destroy(void *ctx) { delete static_cast<AsmData *>(ctx); }

long long ref_ctx_build_csr(void *ctx) {
  AsmData *ad = static_cast<AsmData *>(ctx);
  build_csr_symbolic(*ad);
  return (long long)ad->Jcol.size();
}

int ref_ctx_get_csr(void *ctx, int *I, int *J) {
  AsmData *ad = static_cast<AsmData *>(ctx);
  std::copy(ad->I.begin(), ad->I.end(), I);
  std::copy(ad->Jcol.begin(), ad->Jcol.end(), J);
  return 0;
}

int ref_ctx_reassemble(void *ctx, double *vre, double *vim) {
  AsmData *ad = static_cast<AsmData *>(ctx);
  std::vector<double> re, im;
  reassemble_all(*ad, re, im);
  std::copy(re.begin(), re.end(), vre);
  std::copy(im.begin(), im.end(), vim);
  return 0;
}

// reassemble_all on the context, output discarded; returns seconds
double ref_ctx_time_reassemble(void *ctx) {
  AsmData *ad = static_cast<AsmData *>(ctx);
  std::vector<double> re, im;
  const auto t0 = std::chrono::steady_clock::now();
  reassemble_all(*ad, re, im);
  const auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

int ref_ctx_element(void *ctx, int e, double *out) {
  AsmData *ad = static_cast<AsmData *>(ctx);
  std::vector<C> Ae;
  reassemble_element(*ad, e, Ae);
  for (size_t i = 0; i < Ae.size(); ++i) {
    out[2 * i] = Ae[i].real();
    out[2 * i + 1] = Ae[i].imag();
  }
  return 0;
}

int ref_ctx_gpu_local(void *ctx, int mask_cc, int mask_mass, int te, double *out, double *ms) {
  AsmData *ad = static_cast<AsmData *>(ctx);
  AsmGpu g;
  if (!g.Init(*ad, 0)) return 1;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a);
  if (!g.ComputeLocal(mask_cc, mask_mass, te != 0)) return 2;
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float t = 0.f;
  cudaEventElapsedTime(&t, a, b);
  if (ms) *ms = t;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  std::vector<DC> h;
  if (out) {
    if (!g.DownloadLocal(h)) return 3;
    std::memcpy(out, h.data(), h.size() * sizeof(DC));
  }
  return 0;
}

// Replaces the context's CSR (height + 1 row pointer, nnz columns) with a
// caller-given one: a share of the elements can then be reassembled into the
// full rows of the mesh's own sparsity (rows the share does not touch empty).
int ref_ctx_set_csr(void *ctx, const int *I, long long nnz, const int *J) {
  AsmData *ad = static_cast<AsmData *>(ctx);
  ad->I.assign(I, I + (size_t)ad->height + 1);
  ad->Jcol.assign(J, J + (size_t)nnz);
  return 0;
}

// Incident-field tables of the global problem (prob.incident, parts x slabs;
// problem_common.inc:11-16, 43-57): n_parts * n_slab SlabWave records, part
// major; qA/qB {re, im}, A/B 3 x {re, im} per record.  Call after
// ref_set_problem, which resets the problem.
int ref_set_incident(int n_parts, int n_slab, const double *z_lo, const double *z_hi,
                     const double *qA, const double *qB, const double *zA, const double *zB,
                     const double *A, const double *B) {
  prob.incident.assign(n_parts, std::vector<SlabWave>(n_slab));
  prob.active_parts.clear();
  for (int p = 0; p < n_parts; ++p)
    for (int s = 0; s < n_slab; ++s) {
      const size_t r = (size_t)p * n_slab + s;
      SlabWave &w = prob.incident[p][s];
      w.z_lo = z_lo[s];
      w.z_hi = z_hi[s];
      w.zA = zA[r];
      w.zB = zB[r];
      w.qA = C(qA[2 * r], qA[2 * r + 1]);
      w.qB = C(qB[2 * r], qB[2 * r + 1]);
      for (int i = 0; i < 3; ++i) {
        w.A[i] = C(A[6 * r + 2 * i], A[6 * r + 2 * i + 1]);
        w.B[i] = C(B[6 * r + 2 * i], B[6 * r + 2 * i + 1]);
      }
    }
  return 0;
}

// incident_at (problem_common.inc:219-236): Ehat(z) in slab `slab`, summed
// over the parts; out = 3 x {re, im}.
int ref_incident_at(int slab, double z, double *out) {
  C e[3];
  incident_at(slab, z, e);
  for (int i = 0; i < 3; ++i) {
    out[2 * i] = e[i].real();
    out[2 * i + 1] = e[i].imag();
  }
  return 0;
}

// ScatterSource::Eval (problem_common.inc:239-266), real and imaginary
// coefficient, at reference point xi of the affine element (J row-major,
// v0) with attribute attr: out = 3 x {re, im} of k0^2 (eps - eps_bg) Ehat.
int ref_scatter_source(int attr, const double *J, const double *v0, const double *xi,
                       double *out) {
  ElementTransformation T;
  T.Attribute = attr;
  T.affine = true;
  for (int i = 0; i < 9; ++i) T.J[i] = J[i];
  for (int i = 0; i < 3; ++i) T.v0[i] = v0[i];
  IntegrationPoint ip;
  ip.Set3(xi[0], xi[1], xi[2]);
  ScatterSource sre(false), sim(true);
  Vector fr(3), fi(3);
  sre.Eval(fr, T, ip);
  sim.Eval(fi, T, ip);
  for (int i = 0; i < 3; ++i) {
    out[2 * i] = fr(i);
    out[2 * i + 1] = fi(i);
  }
  return 0;
}

// ref_scatter_source over ne elements (attr[ne], J[ne*9], v0[ne*3]) at nq
// reference points ip[nq*3]: out[(e*nq + q)*6 ...] = 3 x {re, im}.
int ref_scatter_source_elems(int ne, const int *attr, const double *J, const double *v0,
                             int nq, const double *ip, double *out) {
  for (int e = 0; e < ne; ++e)
    for (int q = 0; q < nq; ++q)
      ref_scatter_source(attr[e], J + (size_t)e * 9, v0 + (size_t)e * 3, ip + (size_t)q * 3,
                         out + ((size_t)e * nq + q) * 6);
  return 0;
}

// Full reference GPU path: ComputeLocal(CC, MASS[|kpar terms], te) +
// ScatterEliminate, repeated `iters` times after one warm-up; ms_* are the
// per-iteration averages of the two stages.
int ref_ctx_gpu_global(void *ctx, const int *ess, int n_ess, int eliminate, int iters,
                       double *vals_out, double *ms_local, double *ms_scatter) {
  AsmData *ad = static_cast<AsmData *>(ctx);
  if (ad->Jcol.empty()) build_csr_symbolic(*ad);
  Array<int> ess_list;
  for (int i = 0; i < n_ess; ++i) ess_list.Append(ess[i]);
  AsmGpuGlobal g;
  if (!g.Init(*ad, 0)) return 1;
  if (!g.BuildGlobal(*ad, ess_list)) return 2;
  const bool kpar = prob.kx != 0.0 || prob.ky != 0.0;
  const int mm = ASM_MASS | (kpar ? ASM_CROSS0 | ASM_CROSS1 | ASM_KLK : 0);
  cudaEvent_t a, b, c;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventCreate(&c);
  double tl = 0.0, ts = 0.0;
  for (int it = -1; it < std::max(iters, 1); ++it) {
    cudaEventRecord(a);
    if (!g.ComputeLocal(ASM_CURLCURL, mm, true)) return 3;
    cudaEventRecord(b);
    if (!g.ScatterEliminate(eliminate != 0)) return 4;
    cudaEventRecord(c);
    cudaEventSynchronize(c);
    float t1 = 0.f, t2 = 0.f;
    cudaEventElapsedTime(&t1, a, b);
    cudaEventElapsedTime(&t2, b, c);
    if (it >= 0) { tl += t1; ts += t2; }
  }
  const int n_it = std::max(iters, 1);
  if (ms_local) *ms_local = tl / n_it;
  if (ms_scatter) *ms_scatter = ts / n_it;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaEventDestroy(c);
  if (vals_out) {
    std::vector<DC> h;
    if (!g.DownloadValues(h)) return 5;
    std::memcpy(vals_out, h.data(), h.size() * sizeof(DC));
  }
  return 0;
}

}  // extern "C"
