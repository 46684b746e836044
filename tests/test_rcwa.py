"""Absorber line gratings against the reference's RCWA oracle.

The GPU-assembled system (lfasm_assemble, lfasm_assemble_rhs), a host LU,
plane samples (lfasm_sample_plane) and the order post-processing give the
diffraction efficiencies of a y-invariant absorber line grating in vacuum;
they must match the RCWA efficiencies in tests/golden/rcwa_golden.json
(written by tests/golden/make_rcwa_golden.py from the reference's
tests/reference/rcwa.py) under the reference's own rule and gate
(tests/test_solver_m8.py:122-143: relative 1e-3 on orders with efficiency
>= 1e-3, absolute 1e-3 below).  The cell is the reference's scaled from a
48 nm period and 40 nm lines to 20 nm and 6 nm, so that the host LU of the
p=3 system (about 5e4 unknowns) ends in seconds.

The CPU tests pin the fixture (a uniform layer in RCWA is the
transfer-matrix result) and the efficiency post-processing.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from lithofem_b200 import incident, mesh, orders, problem, space, tmm

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "rcwa_golden.json").read_text())
GATE = 1e-3
LY, GAP, H = 2.0, 4.0, 2.5      # cell depth, vacuum above/below the lines, mesh size
NX, NY = 16, 2                  # plane samples


def _compare(fem: dict, ref_orders, ref_eff, tol: float) -> float:
    """The reference's rule: relative difference on orders with efficiency
    >= 1e-3, absolute below (tests/test_solver_m8.py:122-135)."""
    worst = 0.0
    for m, eff in zip(ref_orders, ref_eff):
        d = abs(fem.get((int(m), 0), 0.0) - eff)
        worst = max(worst, d / eff if eff >= 1e-3 else d)
    assert worst < tol, (worst, fem)
    return worst


@pytest.mark.parametrize("pol", ["TE", "TM"])
def test_uniform_layer_rcwa_is_the_tmm(pol):
    """The fixture's duty-1 layer equals our transfer-matrix solution, as the
    reference's tests/test_rcwa_selfcheck.py requires of RCWA."""
    case = GOLD["cases"]["uniform_" + pol.lower()]
    eps = complex(*GOLD["eps_line"])
    res = tmm.solve(tmm.Stack(eps_in=1.0, eps_out=1.0, eps=(eps,), d=(GOLD["height"],)),
                    GOLD["wavelength"], theta_deg=GOLD["theta"], pol="s" if pol == "TE" else "p")
    for m, r, t in zip(case["orders"], case["r_eff"], case["t_eff"]):
        want_r, want_t = (abs(res.r) ** 2, abs(res.t) ** 2) if m == 0 else (0.0, 0.0)
        assert abs(r - want_r) < 1e-10 and abs(t - want_t) < 1e-10, (m, r, t, want_r, want_t)


def test_order_efficiencies_of_sampled_plane_waves():
    """Two up-going orders sampled on a grid: each efficiency is that wave's
    flux over the incident flux; the (0,0) background adds in phase."""
    lx, ly, k0, nx, ny = 20.0, 2.0, 2 * np.pi / 13.5, 16, 2
    kx0 = k0 * np.sin(np.deg2rad(6.0))
    area = lx * ly
    waves = {(0, 0): 0.3 + 0.1j, (-1, 0): 0.05j}
    x = (np.arange(nx) + 0.5) * lx / nx
    samples = np.zeros((ny, nx, 3), dtype=complex)
    want = {}
    inc = orders.incident_flux(k0, 1.0, kx0, 0.0, area)
    bg = np.array([0.0, 0.2, 0.0], dtype=complex)
    for (m, n), a in waves.items():
        kx = kx0 + 2 * np.pi * m / lx
        qz = orders.order_qz(k0, 1.0, kx, 0.0)
        e = a * np.array([0.0, 1.0, 0.0])                # s-polarised: E along y
        samples += np.exp(1j * 2 * np.pi * m * x / lx)[None, :, None] * e[None, None, :]
        c = e + (bg if (m, n) == (0, 0) else 0)
        want[(m, n)] = 0.5 * (qz.real / k0) * abs(c[1]) ** 2 * area / inc
    oset = orders.orders_from_plane(samples, lx, ly, (kx0, 0.0), k0, 1.0)
    got = orders.order_efficiencies(oset, 3.0, 3.0, +1, area, inc, bg00=bg)
    for key, w in want.items():
        assert abs(got[key] - w) < 1e-14, (key, got[key], w)
    assert abs(got[(1, 0)]) < 1e-14


def _grating(duty: float, p: int = 3):
    """Absorber lines of width duty x period, centred in x, in vacuum."""
    per, hg = GOLD["period"], GOLD["height"]
    eps = complex(*GOLD["eps_line"])
    x0 = 0.5 * per * (1.0 - duty)
    st = mesh.Stack(lx=per, ly=LY, z_min=-GAP, z_max=hg + GAP, wavelength=GOLD["wavelength"],
                    pml_thickness_wavelengths=1.0,
                    frustums=[mesh.Frustum(x0, x0 + duty * per, 0.0, LY, 0.0, hg, 90.0, eps)])
    kpar = incident.kpar_of(st, GOLD["theta"])
    pr = problem.Problem.from_stack(st, p, kpar)
    ad = space.build_asm_data(mesh.build_mesh(st, H), p, pr, build_csr=True)
    return st, pr, ad, kpar


@pytest.mark.gpu
@pytest.mark.parametrize("duty", [0.5, 0.25])
def test_line_grating_matches_rcwa(duty):
    import torch
    from lithofem_b200 import ndbasis
    from lithofem_b200.adjoint import HostLU
    from lithofem_b200.asm import AsmGpuGlobal

    st, pr, ad, kpar = _grating(duty)
    g = AsmGpuGlobal(pr)
    assert g.Init(ad, 0) and g.BuildGlobal(ad.ess) and g.Assemble(True)
    assert g.SetBasis(ndbasis.nd_element(ad.p))
    lu = HostLU(g)
    area = st.lx * st.ly
    inc = orders.incident_flux(pr.k0, 1.0, kpar[0], kpar[1], area)
    planes = (("r", GOLD["height"] + GAP / 2, st.z_max, +1),
              ("t", -GAP / 2, st.z_min, -1))
    for pol in ("TE", "TM"):
        parts = [incident.planewave_parts(st, GOLD["theta"], 0.0, "s" if pol == "TE" else "p")]
        b = torch.zeros(ad.height, dtype=torch.complex128, device="cuda")
        assert g.AssembleRHS(parts, [0], 1, True, b.data_ptr())
        u = torch.from_numpy(lu.solve(b.cpu().numpy())).cuda()
        top, bot = parts[0][-1], parts[0][0]
        ref = GOLD["cases"][f"line_d{round(100 * duty)}_{pol.lower()}"]
        for side, z, z_ref, direction in planes:
            E = torch.empty(NY * NX * 3, dtype=torch.complex128, device="cuda")
            assert g.SamplePlane(st.lx, st.ly, z, NX, NY, u.data_ptr(), E.data_ptr())
            oset = orders.orders_from_plane(E.cpu().numpy().reshape(NY, NX, 3), st.lx, st.ly,
                                            kpar, pr.k0, 1.0)
            bg = (top.B * np.exp(1j * top.qB * (z_ref - top.zB)) if direction > 0
                  else bot.A * np.exp(1j * bot.qA * (z_ref - bot.zA)))
            eff = orders.order_efficiencies(oset, z, z_ref, direction, area, inc, bg00=bg)
            _compare(eff, ref["orders"], ref[side + "_eff"], GATE)


def test_order_efficiencies_refer_each_order_to_the_reference_plane():
    """In an absorbing medium an up-going order decays with height; sampled
    at two heights, the efficiency referred to z_ref is the same, and equals
    that of the amplitude the wave has at z_ref."""
    lx, ly, k0, nx, ny = 20.0, 2.0, 2 * np.pi / 13.5, 8, 2
    eps = 1.0 + 0.05j
    kx0 = k0 * np.sin(np.deg2rad(6.0))
    area = lx * ly
    inc = orders.incident_flux(k0, 1.0, kx0, 0.0, area)
    qz = orders.order_qz(k0, eps, kx0, 0.0)
    assert qz.imag > 0
    z_ref, a_ref = 10.0, 0.4 + 0.2j                # s-polarised amplitude at z_ref
    got = []
    for z in (4.0, 7.5):
        a = a_ref * np.exp(1j * qz * (z - z_ref))  # up-going: e^{i qz z}
        samples = np.zeros((ny, nx, 3), dtype=complex)
        samples[..., 1] = a
        oset = orders.orders_from_plane(samples, lx, ly, (kx0, 0.0), k0, eps)
        got.append(orders.order_efficiencies(oset, z, z_ref, +1, area, inc)[(0, 0)])
    c = np.array([0.0, a_ref, 0.0])
    want = orders.plane_wave_flux(c, kx0, 0.0, qz, k0, +1, area) / inc
    assert abs(got[0] - want) < 1e-13 * abs(want) and abs(got[1] - want) < 1e-13 * abs(want)
