"""Background field (TMM, incident tables) and end-to-end physics.

TMM is pinned to the reference's own module by golden vectors
(tests/golden/make_tmm_golden.py imports src/lithofem/tmm.py); the
difference-layer solve checks the whole assembly chain against the analytic
scattered field, and must converge with the order p.
"""

from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from lithofem_b200 import configs, incident, mesh, tmm
from oracle import oracle

from . import fem_eval

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "tmm_golden.json").read_text())


def _c(v):
    return complex(v[0], v[1])


@pytest.mark.parametrize("case", GOLD, ids=[f"{g['pol']}{g['theta']:g}-{len(g['eps'])}L" for g in GOLD])
def test_tmm_matches_reference_golden(case):
    st = tmm.Stack(eps_in=_c(case["eps_in"]), eps_out=_c(case["eps_out"]),
                   eps=tuple(_c(e) for e in case["eps"]), d=tuple(case["d"]))
    r = tmm.solve(st, case["wavelength"], theta_deg=case["theta"], pol=case["pol"])
    assert abs(r.r - _c(case["r"])) < 1e-12 and abs(r.t - _c(case["t"])) < 1e-12
    for arr, key in ((r.a, "a"), (r.b, "b"), (r.q, "q")):
        assert np.allclose(arr, [_c(v) for v in case[key]], rtol=1e-12, atol=1e-14)


def test_tmm_fresnel_and_energy():
    n1, n2, th = 1.0, 1.5, 30.0
    for pol in ("s", "p"):
        r = tmm.solve(tmm.Stack(eps_in=n1 ** 2, eps_out=n2 ** 2), 500.0, theta_deg=th, pol=pol)
        c1 = math.cos(math.radians(th))
        c2 = math.sqrt(1 - (n1 / n2 * math.sin(math.radians(th))) ** 2)
        rs = (n1 * c1 - n2 * c2) / (n1 * c1 + n2 * c2)
        rp = (n2 * c1 - n1 * c2) / (n2 * c1 + n1 * c2)
        ref = rs if pol == "s" else rp
        assert abs(abs(r.r) - abs(ref)) < 1e-12   # sign conventions differ for p
    # lossless multilayer conserves energy (R + T = 1)
    st = tmm.Stack(eps_in=1.0, eps_out=2.25, eps=(1.9, 2.6), d=(80.0, 55.0))
    for pol in ("s", "p"):
        r = tmm.solve(st, 400.0, theta_deg=20.0, pol=pol)
        g_in = 1.0
        g_out = 1.0 if pol == "s" else 1.0 / 2.25
        T = abs(r.t) ** 2 * (r.q[-1] * g_out).real / (r.q[0] * g_in).real
        assert abs(abs(r.r) ** 2 + T - 1.0) < 1e-12


@pytest.mark.parametrize("pol", ["s", "p"])
def test_incident_tables_are_continuous_and_match_tmm(pol):
    st = configs.line_grating_stack()
    parts = incident.planewave_parts(st, 6.0, 0.0, pol)
    # tangential E continuous at every slab interface
    for a, b in zip(parts[:-1], parts[1:]):
        z = a.z_hi
        ea, eb = a.eval(z)[0], b.eval(z)[0]
        assert np.abs(ea[:2] - eb[:2]).max() < 1e-12 * max(1.0, np.abs(ea).max())
    if pol == "s":
        # s-polarised, phi = 0: E is along y and |Ey| is the TMM scalar |u|
        res = tmm.solve(tmm.Stack(eps_in=1.0, eps_out=configs.UNDERLAYER,
                                  eps=(1.0, 1.0, configs.UNDERLAYER), d=(30.0, 60.0, 40.0)),
                        st.wavelength, kpar=math.hypot(*incident.kpar_of(st, 6.0)), pol="s")
        z = np.array([85.0, 40.0, -10.0])
        ey = incident.eval_parts([parts], z)[:, 1]
        u = res.u(st.slabs[-1] - z)
        assert np.allclose(np.abs(ey), np.abs(u), rtol=1e-12)


def test_zero_scattering_without_contrast():
    st = mesh.Stack(lx=8, ly=8, z_min=0, z_max=20, wavelength=13.5,
                    layers=[(0, 10, configs.ABSORBER)])
    from lithofem_b200 import problem, space
    ms = mesh.build_mesh(st, 2.0)
    pr = problem.Problem.from_stack(st, 2, incident.kpar_of(st, 6.0))
    ad = space.build_asm_data(ms, 2, pr)
    b = oracle.rhs(ad, pr, [incident.planewave_parts(st, 6.0)], [0], 1, ad.ess, True)
    assert np.abs(b).max() == 0.0


def test_difference_layer_oracle_p2():
    st, ad, pr, parts, exact = fem_eval.difference_layer(2, 2.0)
    v = oracle.assemble(ad, pr, ad.I, ad.Jcol, ad.ess, True)
    b = oracle.rhs(ad, pr, parts, [0], 1, ad.ess, True)[0]
    A = sp.csr_matrix((v, ad.Jcol, ad.I), shape=(ad.height,) * 2)
    u = spl.splu(A.tocsc()).solve(b)
    assert np.linalg.norm(A @ u - b) / np.linalg.norm(b) < 1e-10
    assert fem_eval.field_error(ad, u, exact, parts) < 3e-2


@pytest.mark.gpu
@pytest.mark.parametrize("p,h,tol", [(2, 2.0, 3e-2), (3, 2.5, 5e-3)])
@pytest.mark.parametrize("pol", ["s", "p"])
def test_difference_layer_gpu(p, h, tol, pol):
    """GPU-assembled system and RHS reproduce the analytic scattered field."""
    import torch
    from lithofem_b200.asm import AsmGpuGlobal
    st, ad, pr, parts, exact = fem_eval.difference_layer(p, h, pol=pol)
    g = AsmGpuGlobal(pr)
    assert g.Init(ad, 0) and g.BuildGlobal(ad.ess) and g.Assemble(True)
    n = ad.height
    bd = torch.zeros(n, dtype=torch.complex128, device="cuda")
    assert g.AssembleRHS(parts, [0], 1, True, bd.data_ptr())
    I, J = g.DownloadCsr()
    A = sp.csr_matrix((g.DownloadValues(), J, I), shape=(n, n))
    b = bd.cpu().numpy()
    u = spl.splu(A.tocsc()).solve(b)
    ud = torch.from_numpy(u).cuda()
    ok, rel = g.ResidualDevice(ud.data_ptr(), bd.data_ptr())
    assert ok and rel < 1e-10
    assert fem_eval.field_error(ad, u, exact, parts) < tol


def test_plane_functional_is_the_plane_mean():
    from lithofem_b200 import adjoint
    st, ad, pr, parts, exact = fem_eval.difference_layer(2, 3.0)
    rng = np.random.default_rng(3)
    u = rng.standard_normal(ad.height) + 1j * rng.standard_normal(ad.height)
    c = adjoint.plane_functional(ad, z=30.0, lx=fem_eval.L, ly=fem_eval.L, comp=1, nx=4, ny=4)
    xs = (np.arange(4) + 0.5) * fem_eval.L / 4
    X = np.array([[x, y, 30.0] for y in xs for x in xs])
    direct = fem_eval.eval_field(ad, u, X)[:, 1].mean()
    assert abs(c @ u - direct) < 1e-12 * abs(direct)
