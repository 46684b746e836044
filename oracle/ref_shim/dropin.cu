// Test infrastructure: the drop-in call site of INTEGRATION.md section 2
// (gpu_assemble, the code a maintainer adds to solver/lithofem_solve.cpp in
// place of AsmGpu / AsmGpuGlobal, :765-795), compiled against the
// reference's own AsmData, Region and Problem (solver/asm_data.inc,
// solver/problem_common.inc, included from the reference tree, never
// copied) and linked against liblfasm.so.  The snippet is extracted from
// INTEGRATION.md by oracle/Makefile into _build/dropin_snippet.inc, so the
// document's code is the code that is compiled.
//
//   dropin_set_problem   the reference's global `prob` (as ref_set_problem)
//   dropin_ctx_create    the reference's AsmData (as ref_ctx_create)
//   dropin_assemble      gpu_assemble(ad, ess, &h), then the borrowed device
//                        CSR (lfasm_get_csr) copied to the host
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "mfem_shim.hpp"
#include "thirdparty/json.hpp"
#include "lfasm.h"

using namespace mfem;
using json = nlohmann::json;
using C = std::complex<double>;

namespace {
#include "problem_common.inc"
#include "asm_data.inc"
#include "ref_fill.inc"
#include "dropin_snippet.inc"
}  // namespace

extern "C" {

int dropin_set_problem(double k0, double kx, double ky, double z_min, double z_max,
                       double pml_thick, double pml_order, double pml_target, int order,
                       int n_regions, const double *eps, const int *kind, const int *slab,
                       const double *delta_eps) {
  return fill_problem(k0, kx, ky, z_min, z_max, pml_thick, pml_order, pml_target, order,
                      n_regions, eps, kind, slab, delta_eps);
}

void *dropin_ctx_create(int ne, int nd, int p, int height, const int *dof, const double *sign,
                        const int *fo, const int *attr, const double *J, const double *Jinv,
                        const double *detJ, const double *v0, int nq_cc, const double *ip_cc,
                        const double *w_cc, const double *v_cc, const double *c_cc, int nq_m,
                        const double *ip_m, const double *w_m, const double *v_m,
                        const double *c_m) {
  return make_asm_data(ne, nd, p, height, dof, sign, fo, attr, J, Jinv, detJ, v0, nq_cc, ip_cc,
                       w_cc, v_cc, c_cc, nq_m, ip_m, w_m, v_m, c_m);
}

void dropin_ctx_destroy(void *ctx) { delete static_cast<AsmData *>(ctx); }

// gpu_assemble on the context, then the CSR it leaves on the device: n + 1
// row pointers, nnz columns and 2 nnz values (NULL outputs: sizes only).
// Returns 0, or the step that failed (1 gpu_assemble, 2 lfasm_get_csr,
// 3 a copy).
int dropin_assemble(void *ctx, const int *ess, int n_ess, int *n_out, long long *nnz_out,
                    int *I_out, int *J_out, double *vals_out) {
  AsmData *ad = static_cast<AsmData *>(ctx);
  prob.gpu_id = 0;
  Array<int> ess_list;
  for (int i = 0; i < n_ess; ++i) ess_list.Append(ess[i]);
  lfasm_handle *h = nullptr;
  int rc = 0;
  if (!gpu_assemble(*ad, ess_list, &h)) {
    rc = 1;
  } else {
    int *dI = nullptr, *dJ = nullptr;
    void *dV = nullptr;
    int n = 0;
    long long nnz = 0;
    if (lfasm_get_csr(h, &dI, &dJ, &dV, &n, &nnz)) {
      rc = 2;
    } else {
      *n_out = n;
      *nnz_out = nnz;
      if (I_out && (cudaMemcpy(I_out, dI, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost) ||
                    cudaMemcpy(J_out, dJ, sizeof(int) * nnz, cudaMemcpyDeviceToHost) ||
                    cudaMemcpy(vals_out, dV, 16 * nnz, cudaMemcpyDeviceToHost)))
        rc = 3;
    }
  }
  if (h) lfasm_destroy(h);
  return rc;
}

}  // extern "C"
