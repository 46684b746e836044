"""Adjoint gradient w.r.t. per-element permittivity.

1. The kernel's dF/deps_e for F(eps) = lambda^T (b(eps) - A(eps) u) (any u,
   lambda vanishing on the PEC dofs) equals central differences of the
   GPU-assembled F -- A and b are affine in each eps_e, so this is exact up
   to rounding.
2. The full adjoint gradient of J = |l(u)|^2 (l = plane mean of a scattered
   component, the (0,0) order building block) matches central finite
   differences (step 1e-6) on 20 seeded elements to 1e-5 relative.
"""

from __future__ import annotations

import copy

import numpy as np
import pytest

from lithofem_b200 import adjoint, configs, incident, mesh, problem, space
from lithofem_b200.asm import AsmGpuGlobal

pytestmark = pytest.mark.gpu


def _hole_case(p=2, h=3.0, theta=6.0):
    st = mesh.Stack(lx=12.0, ly=12.0, z_min=0.0, z_max=24.0, wavelength=configs.WAVELENGTH,
                    layers=[(0.0, 12.0, configs.ABSORBER)],
                    frustums=[mesh.Frustum(3.0, 9.0, 3.0, 9.0, 0.0, 12.0, 85.0, 1.0 + 0j)])
    ms = mesh.build_mesh(st, h)
    pr = problem.Problem.from_stack(st, p, incident.kpar_of(st, theta))
    ad = space.build_asm_data(ms, p, pr, local_order_seed=8)
    pr.elem_eps = configs.absorber_jitter(ad, pr)
    parts = [incident.planewave_parts(st, theta, 0.0, "s"), incident.planewave_parts(st, theta, 0.0, "p")]
    return st, ad, pr, parts


def _F(ad, pr, parts, eps, u, lam):
    import torch
    prb = copy.copy(pr)
    prb.elem_eps = eps
    g = AsmGpuGlobal(prb)
    assert g.Init(ad, 0) and g.BuildGlobal(ad.ess) and g.Assemble(True)
    b = torch.zeros(ad.height, dtype=torch.complex128, device="cuda")
    assert g.AssembleRHS(parts, [0] * len(parts), 1, True, b.data_ptr())
    y = torch.zeros_like(b)
    ud = torch.from_numpy(u).cuda()
    assert g.SpMV(ud.data_ptr(), y.data_ptr())
    return complex(lam @ (b - y).cpu().numpy()), g


def test_gradient_kernel_is_the_derivative_of_the_assembled_form():
    import torch
    st, ad, pr, parts = _hole_case()
    rng = np.random.default_rng(2)
    n = ad.height
    u = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    lam = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    u[ad.ess] = 0.0
    lam[ad.ess] = 0.0
    F0, g = _F(ad, pr, parts, pr.elem_eps, u, lam)
    gd = torch.zeros(ad.ne, dtype=torch.complex128, device="cuda")
    assert g.EpsGradient(parts, torch.from_numpy(u).cuda().data_ptr(),
                         torch.from_numpy(lam).cuda().data_ptr(), gd.data_ptr())
    grad = gd.cpu().numpy()
    is_pml = np.array([pr.regions[a - 1].is_pml for a in ad.attr])
    assert np.all(grad[is_pml] == 0) and np.all(grad[~is_pml] != 0)
    cand = np.nonzero(~is_pml)[0]
    for e in rng.choice(cand, size=6, replace=False):
        for dirn in (1.0, 1j):
            h = 1e-2
            ep = pr.elem_eps.copy()
            em = pr.elem_eps.copy()
            ep[e] += h * dirn
            em[e] -= h * dirn
            fd = (_F(ad, pr, parts, ep, u, lam)[0] - _F(ad, pr, parts, em, u, lam)[0]) / (2 * h)
            an = grad[e] * dirn
            assert abs(fd - an) <= 1e-8 * abs(an), (e, dirn, fd, an)


def test_adjoint_gradient_matches_central_fd_on_20_elements():
    st, ad, pr, parts = _hole_case()
    c = adjoint.plane_functional(ad, z=21.0, lx=st.lx, ly=st.ly, comp=1)
    adj = adjoint.EpsAdjoint(ad, pr, parts, c)
    ell, J, gre, gim, _ = adj.value_and_grad(pr.elem_eps)
    assert J > 0
    rng = np.random.default_rng(configs.SEED)
    is_pml = np.array([pr.regions[a - 1].is_pml for a in ad.attr])
    els = rng.choice(np.nonzero(~is_pml)[0], size=20, replace=False)
    scale = max(np.abs(gre).max(), np.abs(gim).max())
    h = 1e-6
    worst = 0.0
    for e in els:
        for comp, an in ((1.0, gre[e]), (1j, gim[e])):
            ep = pr.elem_eps.copy()
            em = pr.elem_eps.copy()
            ep[e] += h * comp
            em[e] -= h * comp
            fd = (abs(adj.value(ep)) ** 2 - abs(adj.value(em)) ** 2) / (2 * h)
            worst = max(worst, abs(fd - an) / scale)
    assert worst < 1e-5, worst


def test_autograd_function_backward():
    import torch
    st, ad, pr, parts = _hole_case(h=4.0)
    c = adjoint.plane_functional(ad, z=21.0, lx=st.lx, ly=st.ly, comp=0)
    adj = adjoint.EpsAdjoint(ad, pr, parts, c)
    Fn = adjoint.autograd_function(adj)
    er = torch.tensor(pr.elem_eps.real, dtype=torch.float64, requires_grad=True)
    ei = torch.tensor(pr.elem_eps.imag, dtype=torch.float64, requires_grad=True)
    J = Fn.apply(er, ei)
    J.backward()
    _, J2, gre, gim, _ = adj.value_and_grad(pr.elem_eps)
    assert abs(float(J) - J2) <= 1e-12 * J2
    assert np.allclose(er.grad.numpy(), gre) and np.allclose(ei.grad.numpy(), gim)


def test_efficiency_gradient_matches_central_fd_on_20_elements():
    """The zeroth up-order efficiency (the contact-hole objective) from the
    GPU plane seeds, and its adjoint gradient vs central FD (step 1e-6)."""
    st, ad, pr, parts = _hole_case()
    adj = adjoint.EffAdjoint(ad, pr, parts, z_plane=21.0, lx=st.lx, ly=st.ly, nx=8, ny=8)
    eta, gre, gim = adj.value_and_grad(pr.elem_eps)
    assert 0.0 < eta < 1.0
    rng = np.random.default_rng(configs.SEED)
    is_pml = np.array([pr.regions[a - 1].is_pml for a in ad.attr])
    els = rng.choice(np.nonzero(~is_pml)[0], size=20, replace=False)
    scale = max(np.abs(gre).max(), np.abs(gim).max())
    h = 1e-6
    worst = 0.0
    for e in els:
        for comp, an in ((1.0, gre[e]), (1j, gim[e])):
            ep = pr.elem_eps.copy()
            em = pr.elem_eps.copy()
            ep[e] += h * comp
            em[e] -= h * comp
            fd = (adj.value(ep) - adj.value(em)) / (2 * h)
            worst = max(worst, abs(fd - an) / scale)
    assert worst < 1e-5, worst


def test_bare_slab_zeroth_order_efficiency_is_the_tmm_reflectance():
    """Without contrast the scattered field vanishes and the (0,0)
    efficiency is the stack's reflectance |r|^2 (s polarisation)."""
    from lithofem_b200 import tmm
    st = mesh.Stack(lx=8.0, ly=8.0, z_min=0.0, z_max=24.0, wavelength=configs.WAVELENGTH,
                    layers=[(0.0, 12.0, configs.ABSORBER)])
    theta = 6.0
    ms = mesh.build_mesh(st, 2.5)
    pr = problem.Problem.from_stack(st, 2, incident.kpar_of(st, theta))
    ad = space.build_asm_data(ms, 2, pr, local_order_seed=3)
    parts = [incident.planewave_parts(st, theta, 0.0, "s")]
    eps = pr.eps_table()[ad.attr - 1].copy()
    adj = adjoint.EffAdjoint(ad, pr, parts, z_plane=20.0, lx=st.lx, ly=st.ly, nx=4, ny=4)
    eta = adj.value(eps)
    slabs = st.slabs
    eps_s = [st.eps_bg_of_slab(i) for i in range(len(slabs) - 1)]
    d = [slabs[i + 1] - slabs[i] for i in range(len(slabs) - 1)]
    kx, ky = incident.kpar_of(st, theta)
    res = tmm.solve(tmm.Stack(eps_in=eps_s[-1], eps_out=eps_s[0], eps=tuple(reversed(eps_s)),
                              d=tuple(reversed(d))), st.wavelength, kpar=float(np.hypot(kx, ky)),
                    pol="s")
    assert abs(eta - abs(res.r) ** 2) < 1e-10, (eta, abs(res.r) ** 2)
