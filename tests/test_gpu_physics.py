"""End-to-end physics through the device path (assembly, RHS, complex64
factorization refined in FP64 to 1e-10, plane sampling), at the reference's
own gates and configurations:

* the difference layer against the analytic TMM field (the reference's
  M6-2, tests/test_solver_m6.py:127-148: a 12 nm full-cell layer of
  eps = 1.9 + 0.15i over a 30 nm absorber, 10 nm cell, Nedelec p = 3 at 10
  elements per wavelength, total field on a 16 x 16 plane 12 nm above the
  layer, gate 1e-4; the reference measures 6.6e-5 at 10 epw);
* energy balance of the square contact hole (the reference's M8 4-5,
  tests/test_solver_m8.py:161-254: 32 nm cell, 26 nm absorber with a
  12 x 12 nm hole at 85 deg, p = 3, 4 epw): the net power entering through
  the top plane equals 1 - R with R from the reflected orders, to 1e-4
  (published ~1e-6), and the absorbed fraction (net in minus net out at the
  bottom plane) lies in (0, 1).

The meshes are this repository's structured conformal meshes at the
reference's size rule, lambda / (epw n_max) (src/lithofem/meshgen.py:
456-467); laterally the difference-layer field is uniform, so its cell uses
the reference's periodic minimum of five elements per period.
"""

from __future__ import annotations

import numpy as np
import pytest

from lithofem_b200 import configs, incident, mesh, ndbasis, orders, problem, space
from lithofem_b200.asm import AsmGpuGlobal
from lithofem_b200.solver import C64, DirectSolver

pytestmark = pytest.mark.gpu
WL = configs.WAVELENGTH


def n_max(eps_list) -> float:
    return max([1.0] + [max(abs(np.sqrt(complex(e)).real), abs(np.sqrt(complex(e))))
                        for e in eps_list])


def solve_device(pr, ad, parts, theta):
    """Assemble, factor (complex64), refined solve; returns (g, u, rel)."""
    import torch
    g = AsmGpuGlobal(pr)
    assert g.Init(ad, 0) and g.BuildGlobal(ad.ess) and g.Assemble(True)
    b = torch.zeros(ad.height, dtype=torch.complex128, device="cuda")
    assert g.AssembleRHS(parts, [0] * len(parts), 1, True, b.data_ptr())
    s = DirectSolver(0)
    assert s.AnalyzeAssembly(g, ad) and s.FactorDevice(g._csr()[2], C64), s.last_error
    u = torch.empty_like(b)
    ok, rel, it = s.SolveRefined(g, 1, b.data_ptr(), u.data_ptr(), tol=1e-10)
    assert ok and rel[0] <= 1e-10, (s.last_error, rel, it)
    s.Release()
    assert g.SetBasis(ndbasis.nd_element(ad.p))
    return g, u, rel[0]


def sample(g, st, u, z, nx, ny, curl=False):
    import torch
    E = torch.empty(ny * nx * 3, dtype=torch.complex128, device="cuda")
    C = torch.empty_like(E) if curl else None
    assert g.SamplePlane(st.lx, st.ly, z, nx, ny, u.data_ptr(), E.data_ptr(),
                         C.data_ptr() if curl else 0)
    E = E.cpu().numpy().reshape(ny, nx, 3)
    return (E, C.cpu().numpy().reshape(ny, nx, 3)) if curl else E


# ---------------------------------------------------------------------------
# M6-2: difference layer against TMM
# ---------------------------------------------------------------------------
EPS_DIFF = 1.9 + 0.15j
D_ABS, D_GAP, D_LAYER, LX = 30.0, 20.0, 12.0, 10.0


def difference_layer_case(theta, pol, p=3, epw=10.0):
    z1 = D_ABS + D_LAYER
    z_max = z1 + D_GAP
    st = mesh.Stack(lx=LX, ly=LX, z_min=0.0, z_max=z_max, wavelength=WL,
                    layers=[(0.0, D_ABS, configs.ABSORBER)], pml_thickness_wavelengths=0.75,
                    frustums=[mesh.Frustum(0.0, LX, 0.0, LX, D_ABS, D_LAYER, 90.0, EPS_DIFF)])
    h = WL / (epw * n_max([configs.ABSORBER, EPS_DIFF]))
    ms = mesh.build_mesh(st, h, h_xy=LX / 5.0)
    pr = problem.Problem.from_stack(st, p, incident.kpar_of(st, theta))
    ad = space.build_asm_data(ms, p, pr)
    parts = [incident.planewave_parts(st, theta, 0.0, pol)]
    ref_st = mesh.Stack(lx=LX, ly=LX, z_min=0.0, z_max=z_max, wavelength=WL,
                        layers=[(0.0, D_ABS, configs.ABSORBER), (D_ABS, z1, EPS_DIFF)],
                        pml_thickness_wavelengths=0.75)
    exact = [incident.planewave_parts(ref_st, theta, 0.0, pol)]
    return st, pr, ad, parts, exact, z1 + 0.6 * D_GAP


@pytest.mark.parametrize("pol", ["s", "p"])
@pytest.mark.parametrize("theta", [6.0, 17.0])
def test_difference_layer_vs_tmm_at_10_epw(theta, pol):
    st, pr, ad, parts, exact, z = difference_layer_case(theta, pol)
    g, u, _ = solve_device(pr, ad, parts, theta)
    E_sc = sample(g, st, u, z, 16, 16)
    # total envelope = scattered + incident background; the reference field
    # is the TMM of the stack with the layer as a real layer (the Bloch
    # phase is common to both and drops out)
    e_tot = E_sc + incident.eval_parts(parts, np.array([z]))[0][None, None, :]
    e_ref = np.broadcast_to(incident.eval_parts(exact, np.array([z]))[0], e_tot.shape)
    rel = float(np.linalg.norm(e_tot - e_ref) / np.linalg.norm(e_ref))
    print(f"difference layer theta={theta} pol={pol}: n={ad.height} rel={rel:.2e}")
    assert rel < 1e-4, rel
    g.Release()


# ---------------------------------------------------------------------------
# M8 4-5: energy balance of the square contact hole
# ---------------------------------------------------------------------------
def hole_case(p=3, epw=4.0):
    lx = 32.0
    st = mesh.Stack(lx=lx, ly=lx, z_min=-14.0, z_max=40.0, wavelength=WL,
                    layers=[(0.0, 26.0, configs.ABSORBER)], pml_thickness_wavelengths=0.75,
                    frustums=[mesh.Frustum(10.0, 22.0, 10.0, 22.0, 0.0, 26.0, 85.0, 1.0 + 0j)])
    h = min(WL / (epw * n_max([configs.ABSORBER])), lx / 5.0)
    pr = problem.Problem.from_stack(st, p, incident.kpar_of(st, 6.0))
    ad = space.build_asm_data(mesh.build_mesh(st, h), p, pr)
    parts = [incident.planewave_parts(st, 6.0, 0.0, "s")]
    return st, pr, ad, parts


def total_fields(st, pr, parts, E_sc, C_sc, z):
    """Total envelope E and Z0 H on a plane: scattered samples (E, curl E)
    plus the incident background; Z0 H = (curl E + i k_par x E) / (i k0)."""
    kpar = np.array([pr.kx, pr.ky, 0.0])
    H_sc = (C_sc + 1j * np.cross(kpar[None, None, :], E_sc)) / (1j * pr.k0)
    e_in = np.zeros(3, dtype=complex)
    h_in = np.zeros(3, dtype=complex)
    for slabs in parts:
        sw = next(s for s in slabs if s.z_lo <= z <= s.z_hi)
        a = sw.A * np.exp(1j * sw.qA * (z - sw.zA))
        bb = sw.B * np.exp(1j * sw.qB * (z - sw.zB))
        e_in += a + bb
        h_in += (np.cross([pr.kx, pr.ky, sw.qA], a) + np.cross([pr.kx, pr.ky, sw.qB], bb)) / pr.k0
    return E_sc + e_in, H_sc + h_in


def net_down(E, H, area) -> float:
    s_z = 0.5 * np.real(np.cross(E, np.conj(H))[..., 2])
    return -float(s_z.mean()) * area


def test_square_hole_energy_balance():
    st, pr, ad, parts = hole_case()
    g, u, _ = solve_device(pr, ad, parts, 6.0)
    area = st.lx * st.ly
    inc = orders.incident_flux(pr.k0, 1.0, pr.kx, pr.ky, area)
    z_top, z_bot = 34.0, -8.0
    E, C = sample(g, st, u, z_top, 16, 16, curl=True)
    Et, Ht = total_fields(st, pr, parts, E, C, z_top)
    p_in = net_down(Et, Ht, area)
    Eb, Cb = sample(g, st, u, z_bot, 16, 16, curl=True)
    Ebt, Hbt = total_fields(st, pr, parts, Eb, Cb, z_bot)
    p_out = net_down(Ebt, Hbt, area)
    oset = orders.orders_from_plane(E, st.lx, st.ly, (pr.kx, pr.ky), pr.k0, 1.0)
    top = parts[0][-1]
    bg = top.B * np.exp(1j * top.qB * (st.z_max - top.zB))
    eff = orders.order_efficiencies(oset, z_top, st.z_max, +1, area, inc, bg00=bg)
    r_tot = sum(v for v in eff.values() if v > 0)
    bal = abs(p_in / inc - (1.0 - r_tot))
    a_frac = (p_in - p_out) / inc
    print(f"square hole: n={ad.height} R={r_tot:.6f} in/inc={p_in / inc:.6f} "
          f"balance={bal:.2e} absorbed={a_frac:.4f}")
    assert bal < 1e-4, bal
    assert 0.0 < a_frac < 1.0
    g.Release()
