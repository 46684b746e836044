"""The adjoint gradient on the benchmark's C4 configuration at its size: the
contact hole (96 x 96 nm cell, 60 nm absorber with a 48 x 48 nm hole at 85
deg, p = 2, theta = 6 deg, ~255k DOF) with per-element permittivity of the
absorber elements jittered +-2 % in n and k, objective the zeroth up-going
order efficiency on a plane above the structure.

* Mixed-precision gradient (complex64 factors, FP64-refined solve and
  transposed solve) against the FP64 reference gradient (complex128
  factors, refined to 1e-13): 1e-8 relative over the absorber elements.
* Against central finite differences, step h = 1e-6 in Re eps_e and in
  Im eps_e, on 20 seeded absorber elements, each to 1e-5 relative.  A
  perturbation of one element changes eta by ~1e-12 of itself, so
  subtracting two computed efficiencies would lose the difference to
  rounding; the same central quotient is evaluated without cancellation:
  for eps' = eps +- h e, the solution change du solves A(eps') du =
  b(eps') - A(eps') u (residual in FP64, refined against the unperturbed
  factors), and eta(u + du) - eta(u) = kappa (2 Re(c^H Q dc) + dc^H Q dc)
  with dc = S du (eta = kappa c^H Q c is a quadratic form of the order
  coefficient c = S u + c_bg).
"""

from __future__ import annotations

import numpy as np
import pytest

from lithofem_b200 import adjoint, configs, incident
from lithofem_b200.solver import C128

pytestmark = pytest.mark.gpu
H = 1e-6


@pytest.fixture(scope="module")
def c4():
    import torch
    c = configs.config(4)
    st = c.stack
    parts = [incident.planewave_parts(st, c.theta, 0.0, "s")]
    z_plane = st.z_max - 0.25 * (st.z_max - st.slabs[-2])
    mixed = adjoint.EffAdjoint(c.ad, c.prob, parts, z_plane, st.lx, st.ly, nx=16, ny=16)
    eta, g_re, g_im = mixed.value_and_grad(c.prob.elem_eps)
    ref = adjoint.EffAdjoint(c.ad, c.prob, parts, z_plane, st.lx, st.ly, nx=16, ny=16,
                             prec=C128, tol=1e-13)
    eta64, r_re, r_im = ref.value_and_grad(c.prob.elem_eps)
    yield c, mixed, (eta, g_re, g_im), (eta64, r_re, r_im)
    del mixed, ref
    torch.cuda.empty_cache()


def _absorber(c):
    e0 = c.prob.eps_table()[c.ad.attr - 1]
    return np.nonzero(np.abs(c.prob.elem_eps - e0) > 0)[0]


def test_c4_mixed_gradient_equals_fp64_gradient(c4):
    c, _, (eta, g_re, g_im), (eta64, r_re, r_im) = c4
    sel = _absorber(c)
    assert len(sel) > 1000
    assert abs(eta - eta64) <= 1e-10 * abs(eta64)
    for got, want in ((g_re, r_re), (g_im, r_im)):
        rel = np.linalg.norm(got[sel] - want[sel]) / np.linalg.norm(want[sel])
        print(f"C4: n={c.ad.height} eta={eta:.6e} gradient vs FP64 reference {rel:.2e}")
        assert rel <= 1e-8, rel


def test_c4_gradient_vs_central_differences_on_20_elements(c4):
    import torch
    c, adj, (eta, g_re, g_im), _ = c4
    g, lu, u = adj.last
    ad = c.ad
    sel = np.random.default_rng(configs.SEED).choice(_absorber(c), 20, replace=False)
    ud = torch.from_numpy(u).cuda()
    cvec = adj.coefficient(u)
    Q, kappa = adj.Q(), adj.kappa()
    S = adj._seeds

    def delta_eta(eps2):
        g2, b2 = adj._assemble(eps2)           # A(eps'), b(eps') on the device
        y = torch.empty_like(ud)
        assert g2.SpMV(ud.data_ptr(), y.data_ptr())
        r = (b2 - y).contiguous()              # FP64 residual of u for the perturbed system
        du = torch.empty_like(r)
        ok, rel, _ = lu.s.SolveRefined(g2, 1, r.data_ptr(), du.data_ptr(), False, 1e-12)
        assert ok, lu.s.last_error
        dc = S @ du.cpu().numpy()
        g2.Release()
        return kappa * float(2.0 * np.real(np.conj(cvec) @ Q @ dc) + np.real(np.conj(dc) @ Q @ dc))

    worst = 0.0
    for e in sel:
        for part, grad in ((1.0, g_re), (1j, g_im)):
            eps_p = c.prob.elem_eps.copy()
            eps_m = c.prob.elem_eps.copy()
            eps_p[e] += part * H
            eps_m[e] -= part * H
            fd = (delta_eta(eps_p) - delta_eta(eps_m)) / (2 * H)
            err = abs(grad[e] - fd) / abs(fd)
            worst = max(worst, err)
            assert err <= 1e-5, (int(e), part, grad[e], fd)
    print(f"C4: central differences on 20 elements, worst relative error {worst:.2e}")
