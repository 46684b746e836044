"""Plane sampling and order seeds on the GPU (lfasm_sample_plane,
lfasm_plane_seed) against a host evaluation of the same field."""

from __future__ import annotations

import numpy as np
import pytest

from lithofem_b200 import configs, ndbasis, space
from lithofem_b200.asm import AsmGpuGlobal

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def _case(kind, p):
    if kind == "poly":
        return configs.small_poly_case(p, 6.0, seed=5)
    return configs.small_case(kind, p, 6.0, seed=13, h={1: 1.8, 2: 2.4, 3: 3.2}[p])


def _points(lx, ly, z, nx, ny):
    return np.array([[(i + 0.5) * lx / nx + 3.1e-7, (j + 0.5) * ly / ny + 1.7e-7, z - 4.9e-7]
                     for j in range(ny) for i in range(nx)])


def host_field(ad, p, X, u):
    """E and curl E of the global coefficients u at physical points X:
    most-interior element, local coefficients M (sign u) on face pairs."""
    ne, nd = ad.ne, ad.nd
    Jm, Ji = ad.J.reshape(ne, 3, 3), ad.Jinv.reshape(ne, 3, 3)
    v0, dof, sg = ad.v0.reshape(ne, 3), ad.dof.reshape(ne, nd), ad.sign.reshape(ne, nd)
    fo = ad.fo.reshape(ne, 4) if p > 1 else None
    el = ndbasis.nd_element(p)
    E = np.zeros((len(X), 3), dtype=complex)
    C = np.zeros((len(X), 3), dtype=complex)
    for n, x in enumerate(X):
        xi = np.einsum("eij,ej->ei", Ji, x[None, :] - v0)
        lam = np.column_stack([1 - xi.sum(1), xi]).min(1)
        e = int(np.argmax(lam))
        loc = sg[e] * u[dof[e]]
        if p > 1:
            for f in range(4):
                M = space.face_tinv(fo[e, f])
                for i in range(p * (p - 1) // 2):
                    d0 = 6 * p + f * p * (p - 1) + 2 * i
                    loc[d0:d0 + 2] = M @ loc[d0:d0 + 2]
        vs = el.vshape(xi[e][None])[0] @ Ji[e]                       # (nd, 3)
        cs = (el.curl(xi[e][None])[0] @ Jm[e].T) / ad.detJ[e]       # (nd, 3)
        E[n] = loc @ vs
        C[n] = loc @ cs
    return E, C


@pytest.mark.parametrize("kind,p", [("grating", 1), ("hole", 2), ("grating", 3), ("poly", 3)])
def test_sample_plane_matches_host(kind, p):
    import torch
    c = _case(kind, p)
    g = AsmGpuGlobal(c.prob)
    assert g.Init(c.ad, 0) and g.SetBasis(ndbasis.nd_element(p))
    rng = np.random.default_rng(3)
    u = rng.standard_normal(c.ad.height) + 1j * rng.standard_normal(c.ad.height)
    ud = torch.from_numpy(u).cuda()
    lx, ly = c.stack.lx, c.stack.ly
    z = c.stack.z_min + 0.37 * (c.stack.z_max - c.stack.z_min)
    nx, ny = 7, 5
    E = torch.empty(ny * nx * 3, dtype=torch.complex128, device="cuda")
    C = torch.empty_like(E)
    assert g.SamplePlane(lx, ly, z, nx, ny, ud.data_ptr(), E.data_ptr(), C.data_ptr())
    Eh, Ch = host_field(c.ad, p, _points(lx, ly, z, nx, ny), u)
    assert rel(E.cpu().numpy().reshape(-1, 3), Eh) < 1e-12
    assert rel(C.cpu().numpy().reshape(-1, 3), Ch) < 1e-12


def test_plane_seed_is_the_fft_coefficient():
    import torch
    c = _case("hole", 2)
    g = AsmGpuGlobal(c.prob)
    assert g.Init(c.ad, 0) and g.SetBasis(ndbasis.nd_element(2))
    rng = np.random.default_rng(4)
    u = torch.from_numpy(rng.standard_normal(c.ad.height)
                         + 1j * rng.standard_normal(c.ad.height)).cuda()
    lx, ly, z, nx, ny = c.stack.lx, c.stack.ly, 0.5 * c.stack.z_max + 1.3, 6, 4
    E = torch.empty(ny * nx * 3, dtype=torch.complex128, device="cuda")
    assert g.SamplePlane(lx, ly, z, nx, ny, u.data_ptr(), E.data_ptr())
    F = np.fft.fft2(E.cpu().numpy().reshape(ny, nx, 3), axes=(0, 1)) / (nx * ny)
    cvec = torch.empty(c.ad.height, dtype=torch.complex128, device="cuda")
    for comp, m, q in [(0, 0, 0), (1, 1, -1), (2, -2, 1), (0, 3, 2)]:
        assert g.PlaneSeed(lx, ly, z, nx, ny, comp, m, q, cvec.data_ptr())
        got = complex((cvec * u).sum().item())
        want = F[q % ny, m % nx, comp]
        assert abs(got - want) <= 1e-12 * np.abs(F).max(), (comp, m, q, got, want)


def test_plane_outside_mesh_and_missing_basis_are_errors():
    import torch
    c = _case("grating", 1)
    g = AsmGpuGlobal(c.prob)
    assert g.Init(c.ad, 0)
    u = torch.zeros(c.ad.height, dtype=torch.complex128, device="cuda")
    E = torch.empty(4 * 3, dtype=torch.complex128, device="cuda")
    lx, ly = c.stack.lx, c.stack.ly
    assert not g.SamplePlane(lx, ly, 0.0, 2, 2, u.data_ptr(), E.data_ptr())
    assert g.last_error[0] == 4
    assert g.SetBasis(ndbasis.nd_element(1))
    z_out = c.stack.z_max + 3 * c.stack.pml_thick
    assert not g.SamplePlane(lx, ly, z_out, 2, 2, u.data_ptr(), E.data_ptr())
    assert g.last_error[0] == 1 and "outside the mesh" in g.last_error[1]
