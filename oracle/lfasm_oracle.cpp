// ORACLE -- test infrastructure, not product code.
//
// Serial CPU restatement of the reference's assembly path, used only by
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg to check
// and time the CUDA library.  Inputs are the same C structs the library
// takes (include/lfasm.h), so both run on identical data.
//
//   orc_local     element matrices per integrator mask + dual transform:
//                 reassemble_element, solver/asm_data.inc:218-370, with the
//                 integrator masks of asm_local_kernel (asm_gpu.inc:51-58,
//                 148-205) and s(z) of problem_common.inc:69-98
//   orc_csr       build_csr_symbolic, asm_data.inc:178-210
//   orc_assemble  reassemble_all scatter (asm_data.inc:374-402) + essential
//                 elimination (asm_eliminate_kernel, asm_gpu.inc:461-478)
//   orc_spmv      y = A x (asm_spmv_kernel, asm_gpu.inc:480-493) and the
//                 residual norm of AsmGpuGlobal::Residual (asm_gpu.inc:533-565)
//   orc_rhs       ScatterSource + incident_at (problem_common.inc:218-266)
//                 integrated as VectorFEDomainLFIntegrator at the rule_mass
//                 points, dual transform, signed scatter, essential rows
//                 zeroed (form_rhs_only, lithofem_solve.cpp:732-742)
//
// Parity of this restatement is pinned against the reference's own
// reassembler compiled from its sources (oracle/ref_shim, oracle/_ref) by
// the golden fixtures in tests/golden.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "../include/lfasm.h"

using C = std::complex<double>;

namespace {

struct Pml {
  double z_min, z_max, thick, order, smax_bot, smax_top;
};

Pml make_pml(const lfasm_problem *pr) {
  Pml p{pr->z_min, pr->z_max, pr->pml_thick, pr->pml_order, 0.0, 0.0};
  double n_bot = 1.0, n_top = 1.0;
  for (int r = 0; r < pr->n_regions; ++r) {
    const C e(pr->region_eps[2 * r], pr->region_eps[2 * r + 1]);
    if (pr->region_kind[r] == LFASM_REGION_PML_BOTTOM) n_bot = std::abs(std::sqrt(e));
    if (pr->region_kind[r] == LFASM_REGION_PML_TOP) n_top = std::abs(std::sqrt(e));
  }
  p.smax_bot = -std::log(pr->pml_target) * (pr->pml_order + 1) / (2.0 * pr->k0 * n_bot * pr->pml_thick);
  p.smax_top = -std::log(pr->pml_target) * (pr->pml_order + 1) / (2.0 * pr->k0 * n_top * pr->pml_thick);
  return p;
}

// problem_common.inc:69-90
C s_z(const Pml &p, double z) {
  double d = -1.0, smax = 0.0;
  if (z < p.z_min) { d = (p.z_min - z) / p.thick; smax = p.smax_bot; }
  else if (z > p.z_max) { d = (z - p.z_max) / p.thick; smax = p.smax_top; }
  if (d < 0.0) return {1.0, 0.0};
  if (d > 1.0) d = 1.0;
  return {1.0, smax * std::pow(d, p.order)};
}

C eps_of(const lfasm_asm_data *ad, const lfasm_problem *pr, int e) {
  if (pr->elem_eps) return C(pr->elem_eps[2 * e], pr->elem_eps[2 * e + 1]);
  const int r = ad->attr[e] - 1;
  return C(pr->region_eps[2 * r], pr->region_eps[2 * r + 1]);
}

// column-major 2x2 face blocks: local pair = M (global pair), for the face
// vertex permutations (0,1,2),(1,0,2),(1,2,0),(2,1,0),(2,0,1),(0,2,1)
void tinv_table(double T[24]) {
  const int perms[6][3] = {{0, 1, 2}, {1, 0, 2}, {1, 2, 0}, {2, 1, 0}, {2, 0, 1}, {0, 2, 1}};
  const double G[3][2] = {{0, 0}, {1, 0}, {0, 1}};
  for (int o = 0; o < 6; ++o) {
    const double *a = G[perms[o][0]], *b = G[perms[o][1]], *c = G[perms[o][2]];
    T[4 * o + 0] = b[0] - a[0];
    T[4 * o + 1] = c[0] - a[0];
    T[4 * o + 2] = b[1] - a[1];
    T[4 * o + 3] = c[1] - a[1];
  }
}

// asm_data.inc:337-369: TInv(fo)^T on face-DOF pairs, columns then rows
void dual_transform(int nd, int p, const int *fo, C *Ae) {
  if (p < 2) return;
  double T[24];
  tinv_table(T);
  const int foff = 6 * p, ntd = p * (p - 1);
  for (int axis = 0; axis < 2; ++axis)
    for (int f = 0; f < 4; ++f) {
      const double *Ti = T + 4 * fo[f];
      for (int i = 0; i < ntd / 2; ++i) {
        const int d0 = foff + f * ntd + 2 * i;
        for (int r = 0; r < nd; ++r) {
          C &a = axis == 0 ? Ae[(size_t)r * nd + d0] : Ae[(size_t)d0 * nd + r];
          C &b = axis == 0 ? Ae[(size_t)r * nd + d0 + 1] : Ae[(size_t)(d0 + 1) * nd + r];
          const C na = Ti[0] * a + Ti[1] * b;
          const C nb = Ti[2] * a + Ti[3] * b;
          a = na;
          b = nb;
        }
      }
    }
}

// one element, operation order of reassemble_element (asm_data.inc:218-335)
void element(const lfasm_asm_data *ad, const lfasm_problem *pr, const Pml &pm, int e,
             int mask_cc, int mask_mass, bool te, std::vector<C> &Ae) {
  const int nd = ad->nd;
  const double *J = ad->J + (size_t)e * 9;
  const double *Ji = ad->Jinv + (size_t)e * 9;
  const double detJ = ad->detJ[e];
  const double *v0 = ad->v0 + (size_t)e * 3;
  const C eps = eps_of(ad, pr, e);
  const double k2 = pr->k0 * pr->k0;
  Ae.assign((size_t)nd * nd, C(0.0, 0.0));
  std::vector<double> pc((size_t)nd * 3), pv((size_t)nd * 3);
  if (mask_cc & LFASM_CURLCURL) {
    const lfasm_ref_rule &rc = ad->rule_cc;
    for (int q = 0; q < rc.nq; ++q) {
      const double *xi = rc.ip + (size_t)q * 3;
      const double z = v0[2] + J[6] * xi[0] + J[7] * xi[1] + J[8] * xi[2];
      const C s = s_z(pm, z);
      const C li[3] = {1.0 / s, 1.0 / s, s};
      const double w = rc.w[q] * detJ;
      const double *cs = rc.curl + (size_t)q * nd * 3;
      for (int k = 0; k < nd; ++k)
        for (int i = 0; i < 3; ++i)
          pc[(size_t)k * 3 + i] =
              (cs[k * 3 + 0] * J[i * 3 + 0] + cs[k * 3 + 1] * J[i * 3 + 1] + cs[k * 3 + 2] * J[i * 3 + 2]) / detJ;
      for (int k = 0; k < nd; ++k)
        for (int l = 0; l < nd; ++l) {
          C sum(0.0, 0.0);
          for (int i = 0; i < 3; ++i) sum += pc[(size_t)k * 3 + i] * li[i] * pc[(size_t)l * 3 + i];
          Ae[(size_t)k * nd + l] += w * sum;
        }
    }
  }
  if (mask_mass) {
    const lfasm_ref_rule &rm = ad->rule_mass;
    double K[9] = {0.0, 0.0, pr->ky, 0.0, 0.0, -pr->kx, -pr->ky, pr->kx, 0.0};
    const bool need_c = mask_mass & (LFASM_CROSS0 | LFASM_CROSS1);
    for (int q = 0; q < rm.nq; ++q) {
      const double *xi = rm.ip + (size_t)q * 3;
      const double z = v0[2] + J[6] * xi[0] + J[7] * xi[1] + J[8] * xi[2];
      const C s = s_z(pm, z);
      const C lam[3] = {s, s, 1.0 / s};
      const C li[3] = {1.0 / s, 1.0 / s, s};
      const double w = rm.w[q] * detJ;
      const double *vs = rm.vshape + (size_t)q * nd * 3;
      const double *cs = rm.curl + (size_t)q * nd * 3;
      for (int k = 0; k < nd; ++k)
        for (int i = 0; i < 3; ++i) {
          pv[(size_t)k * 3 + i] = vs[k * 3 + 0] * Ji[0 * 3 + i] + vs[k * 3 + 1] * Ji[1 * 3 + i] +
                                  vs[k * 3 + 2] * Ji[2 * 3 + i];
          if (need_c)
            pc[(size_t)k * 3 + i] =
                (cs[k * 3 + 0] * J[i * 3 + 0] + cs[k * 3 + 1] * J[i * 3 + 1] + cs[k * 3 + 2] * J[i * 3 + 2]) / detJ;
        }
      const C md[3] = {-k2 * eps * lam[0], -k2 * eps * lam[1], -k2 * eps * lam[2]};
      if (mask_mass & LFASM_MASS)
        for (int k = 0; k < nd; ++k)
          for (int l = 0; l < nd; ++l) {
            C s2(0.0, 0.0);
            for (int i = 0; i < 3; ++i) s2 += pv[(size_t)k * 3 + i] * md[i] * pv[(size_t)l * 3 + i];
            Ae[(size_t)k * nd + l] += w * s2;
          }
      if (mask_mass & (LFASM_CROSS0 | LFASM_CROSS1 | LFASM_KLK)) {
        const C iu(0.0, 1.0);
        for (int k = 0; k < nd; ++k)
          for (int l = 0; l < nd; ++l) {
            C s0(0.0, 0.0), s1(0.0, 0.0), s2b(0.0, 0.0);
            for (int r = 0; r < 3; ++r)
              for (int c = 0; c < 3; ++c) {
                const double krc = K[r * 3 + c];
                if (krc != 0.0) {
                  if (mask_mass & LFASM_CROSS0)
                    s0 += pv[(size_t)k * 3 + r] * (iu * krc * li[c]) * pc[(size_t)l * 3 + c];
                  if (mask_mass & LFASM_CROSS1)
                    s1 += pc[(size_t)k * 3 + r] * (iu * li[r] * krc) * pv[(size_t)l * 3 + c];
                }
                if (mask_mass & LFASM_KLK) {
                  C m2(0.0, 0.0);
                  for (int t = 0; t < 3; ++t) m2 += K[r * 3 + t] * li[t] * K[t * 3 + c];
                  s2b -= pv[(size_t)k * 3 + r] * m2 * pv[(size_t)l * 3 + c];
                }
              }
            Ae[(size_t)k * nd + l] += w * (s0 + s1 + s2b);
          }
      }
    }
  }
  if (te) dual_transform(nd, ad->p, ad->fo + (size_t)e * 4, Ae.data());
}

}  // namespace

extern "C" {

int orc_local(const lfasm_asm_data *ad, const lfasm_problem *pr, int mask_cc, int mask_mass,
              int te, double *out) {
  const Pml pm = make_pml(pr);
  std::vector<C> Ae;
  const size_t n2 = (size_t)ad->nd * ad->nd;
  for (int e = 0; e < ad->ne; ++e) {
    element(ad, pr, pm, e, mask_cc, mask_mass, te != 0, Ae);
    std::memcpy(out + 2 * n2 * e, Ae.data(), n2 * sizeof(C));
  }
  return 0;
}

// asm_data.inc:178-210.  J_out == NULL: only count.
long long orc_csr(const lfasm_asm_data *ad, int *I_out, int *J_out) {
  const int n = ad->height, nd = ad->nd;
  std::vector<std::vector<int>> cols(n);
  for (int e = 0; e < ad->ne; ++e) {
    const int *ed = ad->dof + (size_t)e * nd;
    for (int a = 0; a < nd; ++a)
      for (int b = 0; b < nd; ++b) cols[ed[a]].push_back(ed[b]);
  }
  long long nnz = 0;
  if (I_out) I_out[0] = 0;
  for (int r = 0; r < n; ++r) {
    std::vector<int> &row = cols[r];
    std::sort(row.begin(), row.end());
    row.erase(std::unique(row.begin(), row.end()), row.end());
    if (J_out) std::copy(row.begin(), row.end(), J_out + nnz);
    nnz += (long long)row.size();
    if (I_out) I_out[r + 1] = (int)nnz;
  }
  return nnz;
}

// asm_data.inc:374-402 scatter (lower_bound in the sorted row) followed by
// the elimination of asm_gpu.inc:461-478
int orc_assemble(const lfasm_asm_data *ad, const lfasm_problem *pr, const int *I,
                 const int *Jc, const int *ess_list, int n_ess, int eliminate, double *vals) {
  const Pml pm = make_pml(pr);
  const long long nnz = I[ad->height];
  std::fill(vals, vals + 2 * nnz, 0.0);
  const int mm = LFASM_MASS | ((pr->kx != 0.0 || pr->ky != 0.0)
                                   ? (LFASM_CROSS0 | LFASM_CROSS1 | LFASM_KLK) : 0);
  std::vector<C> Ae;
  const int nd = ad->nd;
  for (int e = 0; e < ad->ne; ++e) {
    element(ad, pr, pm, e, LFASM_CURLCURL, mm, true, Ae);
    const int *ed = ad->dof + (size_t)e * nd;
    const double *es = ad->sign + (size_t)e * nd;
    for (int a = 0; a < nd; ++a) {
      const int row = ed[a];
      const int *jb = Jc + I[row], *je = Jc + I[row + 1];
      for (int b = 0; b < nd; ++b) {
        const int *pos = std::lower_bound(jb, je, ed[b]);
        if (pos == je || *pos != ed[b]) return 1;
        const size_t k = (size_t)(pos - Jc);
        const C v = es[a] * es[b] * Ae[(size_t)a * nd + b];
        vals[2 * k] += v.real();
        vals[2 * k + 1] += v.imag();
      }
    }
  }
  if (eliminate) {
    std::vector<unsigned char> is_ess(ad->height, 0);
    for (int i = 0; i < n_ess; ++i) is_ess[ess_list[i]] = 1;
    for (int r = 0; r < ad->height; ++r)
      for (int k = I[r]; k < I[r + 1]; ++k) {
        const int c = Jc[k];
        if (is_ess[r] || is_ess[c]) {
          vals[2 * (size_t)k] = (is_ess[r] && c == r) ? 1.0 : 0.0;
          vals[2 * (size_t)k + 1] = 0.0;
        }
      }
  }
  return 0;
}

// y = A x (interleaved complex); returns ||A x - b|| / ||b|| when b != NULL
double orc_spmv(int n, const int *I, const int *Jc, const double *vals, const double *x,
                const double *b, double *y) {
  double rn = 0.0, bn = 0.0;
  for (int r = 0; r < n; ++r) {
    C acc(0.0, 0.0);
    for (int k = I[r]; k < I[r + 1]; ++k)
      acc += C(vals[2 * (size_t)k], vals[2 * (size_t)k + 1]) * C(x[2 * (size_t)Jc[k]], x[2 * (size_t)Jc[k] + 1]);
    if (y) { y[2 * (size_t)r] = acc.real(); y[2 * (size_t)r + 1] = acc.imag(); }
    if (b) {
      const C bb(b[2 * (size_t)r], b[2 * (size_t)r + 1]);
      rn += std::norm(acc - bb);
      bn += std::norm(bb);
    }
  }
  return bn > 0.0 ? std::sqrt(rn / bn) : 0.0;
}

// problem_common.inc:218-266; parts with col_of_part[i] == c form column c
int orc_rhs(const lfasm_asm_data *ad, const lfasm_problem *pr, const lfasm_incident_part *parts,
            int n_parts, const int *col_of_part, int ncol, const int *ess_list, int n_ess,
            int eliminate, double *b) {
  const int nd = ad->nd, n = ad->height;
  std::fill(b, b + 2 * (size_t)n * ncol, 0.0);
  // background region of each slab, for per-element eps contrasts
  std::vector<int> bg(64, -1);
  for (int r = 0; r < pr->n_regions; ++r)
    if (pr->region_kind[r] == LFASM_REGION_BACKGROUND && pr->region_slab[r] >= 0 &&
        pr->region_slab[r] < 64)
      bg[pr->region_slab[r]] = r;
  const lfasm_ref_rule &rm = ad->rule_mass;
  std::vector<C> be(nd);
  for (int e = 0; e < ad->ne; ++e) {
    const int r = ad->attr[e] - 1;
    const int kind = pr->region_kind[r];
    const int slab = pr->region_slab[r];
    C delta(0.0, 0.0);
    if (kind == LFASM_REGION_FRUSTUM)
      delta = C(pr->region_delta_eps[2 * r], pr->region_delta_eps[2 * r + 1]);
    if (pr->elem_eps && (kind == LFASM_REGION_BACKGROUND || kind == LFASM_REGION_FRUSTUM) &&
        slab >= 0 && bg[slab] >= 0)
      delta = C(pr->elem_eps[2 * e], pr->elem_eps[2 * e + 1]) -
              C(pr->region_eps[2 * bg[slab]], pr->region_eps[2 * bg[slab] + 1]);
    if (delta == C(0.0, 0.0)) continue;
    const double *J = ad->J + (size_t)e * 9;
    const double *Ji = ad->Jinv + (size_t)e * 9;
    const double *v0 = ad->v0 + (size_t)e * 3;
    const C fac = pr->k0 * pr->k0 * delta;
    for (int c = 0; c < ncol; ++c) {
      std::fill(be.begin(), be.end(), C(0.0, 0.0));
      for (int q = 0; q < rm.nq; ++q) {
        const double *xi = rm.ip + (size_t)q * 3;
        const double z = v0[2] + J[6] * xi[0] + J[7] * xi[1] + J[8] * xi[2];
        C ev[3] = {0.0, 0.0, 0.0};
        for (int pi = 0; pi < n_parts; ++pi) {
          if (col_of_part[pi] != c) continue;
          const lfasm_incident_part &P = parts[pi];
          const C qA(P.qA[2 * slab], P.qA[2 * slab + 1]), qB(P.qB[2 * slab], P.qB[2 * slab + 1]);
          const C up = std::exp(C(0, 1) * qA * (z - P.zA[slab]));
          const C dn = std::exp(C(0, 1) * qB * (z - P.zB[slab]));
          for (int d = 0; d < 3; ++d)
            ev[d] += C(P.A[6 * slab + 2 * d], P.A[6 * slab + 2 * d + 1]) * up +
                     C(P.B[6 * slab + 2 * d], P.B[6 * slab + 2 * d + 1]) * dn;
        }
        const double w = rm.w[q] * ad->detJ[e];
        const double *vs = rm.vshape + (size_t)q * nd * 3;
        for (int k = 0; k < nd; ++k)
          for (int d = 0; d < 3; ++d) {
            const double pv = vs[k * 3 + 0] * Ji[0 * 3 + d] + vs[k * 3 + 1] * Ji[1 * 3 + d] +
                              vs[k * 3 + 2] * Ji[2 * 3 + d];
            be[k] += w * pv * (fac * ev[d]);
          }
      }
      if (ad->p >= 2) {  // rows of the dual transform
        double T[24];
        tinv_table(T);
        const int foff = 6 * ad->p, ntd = ad->p * (ad->p - 1);
        for (int f = 0; f < 4; ++f) {
          const double *Ti = T + 4 * ad->fo[(size_t)e * 4 + f];
          for (int i = 0; i < ntd / 2; ++i) {
            const int d0 = foff + f * ntd + 2 * i;
            const C a = be[d0], bb = be[d0 + 1];
            be[d0] = Ti[0] * a + Ti[1] * bb;
            be[d0 + 1] = Ti[2] * a + Ti[3] * bb;
          }
        }
      }
      for (int k = 0; k < nd; ++k) {
        const size_t row = (size_t)ad->dof[(size_t)e * nd + k];
        const C v = ad->sign[(size_t)e * nd + k] * be[k];
        b[2 * ((size_t)c * n + row)] += v.real();
        b[2 * ((size_t)c * n + row) + 1] += v.imag();
      }
    }
  }
  if (eliminate)
    for (int i = 0; i < n_ess; ++i)
      for (int c = 0; c < ncol; ++c) {
        b[2 * ((size_t)c * n + ess_list[i])] = 0.0;
        b[2 * ((size_t)c * n + ess_list[i]) + 1] = 0.0;
      }
  return 0;
}

}  // extern "C"
