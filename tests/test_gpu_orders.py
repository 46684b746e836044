"""Batched plane sampling and the diffraction orders on the device.

* lfasm_sample_planes over several heights equals lfasm_sample_plane called
  once per height, bit for bit (the same location and evaluation kernels
  over all planes' points).
* lfasm_plane_orders: the Fourier coefficients and order efficiencies of
  sampled planes equal the host restatement of the reference's
  orders_from_plane / order efficiency (lithofem_b200.orders, itself
  src/lithofem/orders.py:36-67 and src/lithofem/outputs.py:219-269) on the
  same samples: coefficients to 1e-13 of the largest, efficiencies to
  1e-12 of the largest, for up-going and down-going planes, a lossy medium
  (evanescent and decaying orders) and the analytic (0,0) background.
* End to end on the square contact hole of the energy-balance gate: the
  reflected and transmitted order sums from one batched sampling pass and
  the device orders equal the host path's.
"""

from __future__ import annotations

import numpy as np
import pytest

from lithofem_b200 import configs, ndbasis, orders
from lithofem_b200.asm import AsmGpuGlobal

pytestmark = pytest.mark.gpu


def _global(case):
    g = AsmGpuGlobal(case.prob)
    assert g.Init(case.ad, 0) and g.BuildGlobal(case.ad.ess)
    assert g.SetBasis(ndbasis.nd_element(case.ad.p))
    return g


def test_sample_planes_equals_one_plane_at_a_time():
    import torch
    c = configs.small_case("grating", 3, 6.0)
    st = c.stack
    g = _global(c)
    rng = np.random.default_rng(3)
    u = torch.from_numpy(rng.standard_normal(c.ad.height) + 1j * rng.standard_normal(c.ad.height)).cuda()
    zs = [st.z_min + 0.3, 0.5 * (st.z_min + st.z_max), st.z_max - 0.7, 1.3]
    nx, ny = 12, 5
    npts = nx * ny * 3
    E = torch.empty(len(zs) * npts, dtype=torch.complex128, device="cuda")
    C = torch.empty_like(E)
    assert g.SamplePlanes(st.lx, st.ly, zs, nx, ny, u.data_ptr(), E.data_ptr(), C.data_ptr())
    for iz, z in enumerate(zs):
        e1 = torch.empty(npts, dtype=torch.complex128, device="cuda")
        c1 = torch.empty_like(e1)
        assert g.SamplePlane(st.lx, st.ly, z, nx, ny, u.data_ptr(), e1.data_ptr(), c1.data_ptr())
        assert torch.equal(E[iz * npts:(iz + 1) * npts], e1)
        assert torch.equal(C[iz * npts:(iz + 1) * npts], c1)
    # a plane outside the mesh (beyond the PML) fails the whole call
    assert not g.SamplePlanes(st.lx, st.ly, [0.0, st.z_max + 100.0], nx, ny, u.data_ptr(),
                              E.data_ptr())
    assert g.last_error[0] != 0 and "outside the mesh" in g.last_error[1]
    assert not g.SamplePlanes(st.lx, st.ly, [], nx, ny, u.data_ptr(), E.data_ptr())
    g.Release()


@pytest.mark.parametrize("nx,ny", [(16, 8), (9, 7)])
def test_plane_orders_equal_host_orders(nx, ny):
    import torch
    c = configs.small_case("slab", 1, 0.0)
    g = _global(c)
    rng = np.random.default_rng(11)
    lx, ly, k0 = 20.0, 14.0, 2 * np.pi / 13.5
    kpar = (k0 * np.sin(np.deg2rad(6.0)) * 0.8, k0 * np.sin(np.deg2rad(6.0)) * 0.6)
    planes = [dict(z=3.0, z_ref=10.0, eps=1.0, direction=1,
                   bg00=rng.standard_normal(3) + 1j * rng.standard_normal(3)),
              dict(z=-2.0, z_ref=-5.0, eps=2.25 + 0.3j, direction=-1),
              dict(z=7.5, z_ref=7.5, eps=1.0 + 0.05j, direction=1)]
    nz = len(planes)
    u = rng.standard_normal((nz, ny, nx, 3)) + 1j * rng.standard_normal((nz, ny, nx, 3))
    ud = torch.from_numpy(u.reshape(-1).copy()).cuda()
    inc = orders.incident_flux(k0, 1.0, kpar[0], kpar[1], lx * ly)
    got = orders.device_orders(g, nx, ny, ud.data_ptr(), planes, lx, ly, k0, kpar, inc)
    for iz, q in enumerate(planes):
        oset = orders.orders_from_plane(u[iz], lx, ly, kpar, k0, q["eps"])
        want = orders.order_efficiencies(oset, q["z"], q["z_ref"], q["direction"], lx * ly, inc,
                                         bg00=q.get("bg00"))
        coef, eff = got[iz]
        scale = np.abs(oset.coeffs).max()
        assert np.abs(coef - oset.coeffs).max() <= 1e-13 * scale
        assert set(eff) == set(want)
        escale = max(abs(v) for v in want.values())
        worst = max(abs(eff[k] - want[k]) for k in want)
        assert worst <= 1e-12 * escale, (iz, worst, escale)
    # argument checks
    bad = [dict(planes[0], direction=0)]
    args = dict(lx=lx, ly=ly, k0=k0, kx=kpar[0], ky=kpar[1], inc_flux=inc)
    assert not g.PlaneOrders(nx, ny, ud.data_ptr(), bad, args, ud.data_ptr(), ud.data_ptr())
    assert "direction" in g.last_error[1]
    assert not g.PlaneOrders(nx, ny, ud.data_ptr(), planes, dict(args, inc_flux=0.0),
                             ud.data_ptr(), ud.data_ptr())
    g.Release()


def test_square_hole_orders_from_one_batched_pass():
    """The energy-balance case: reflected and transmitted order sums from
    lfasm_sample_planes + lfasm_plane_orders equal the host post-processing
    of per-plane samples."""
    import torch
    from .test_gpu_physics import hole_case, solve_device
    st, pr, ad, parts = hole_case()
    g, u, _ = solve_device(pr, ad, parts, 6.0)
    area = st.lx * st.ly
    inc = orders.incident_flux(pr.k0, 1.0, pr.kx, pr.ky, area)
    top, bot = parts[0][-1], parts[0][0]
    z_top, z_bot, nx, ny = 34.0, -8.0, 16, 16
    bg_top = top.B * np.exp(1j * top.qB * (st.z_max - top.zB))
    # below the stack only the transmitted wave is present (the other amplitude is zero)
    bg_bot = (bot.A * np.exp(1j * bot.qA * (st.z_min - bot.zA))
              + bot.B * np.exp(1j * bot.qB * (st.z_min - bot.zB)))
    planes = [dict(z=z_top, z_ref=st.z_max, eps=1.0, direction=1, bg00=bg_top),
              dict(z=z_bot, z_ref=st.z_min, eps=st.eps_bg_of_slab(0), direction=-1, bg00=bg_bot)]
    E = torch.empty(2 * ny * nx * 3, dtype=torch.complex128, device="cuda")
    assert g.SamplePlanes(st.lx, st.ly, [z_top, z_bot], nx, ny, u.data_ptr(), E.data_ptr())
    got = orders.device_orders(g, nx, ny, E.data_ptr(), planes, st.lx, st.ly, pr.k0,
                               (pr.kx, pr.ky), inc)
    sums = []
    for iz, q in enumerate(planes):
        e1 = torch.empty(ny * nx * 3, dtype=torch.complex128, device="cuda")
        assert g.SamplePlane(st.lx, st.ly, q["z"], nx, ny, u.data_ptr(), e1.data_ptr())
        oset = orders.orders_from_plane(e1.cpu().numpy().reshape(ny, nx, 3), st.lx, st.ly,
                                        (pr.kx, pr.ky), pr.k0, q["eps"])
        want = orders.order_efficiencies(oset, q["z"], q["z_ref"], q["direction"], area, inc,
                                         bg00=q["bg00"])
        eff = got[iz][1]
        r_host = sum(v for v in want.values() if v > 0)
        r_dev = sum(v for v in eff.values() if v > 0)
        assert abs(r_dev - r_host) <= 1e-12, (iz, r_dev, r_host)
        sums.append(r_dev)
    print(f"square hole: R = {sums[0]:.6f}, T = {sums[1]:.6f} from one batched pass")
    assert 0.0 < sums[0] < 1.0 and 0.0 <= sums[1] < 1.0
    g.Release()
