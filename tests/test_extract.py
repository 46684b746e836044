"""Per-mesh data extraction on the device (lfasm_extract), against the host
build_asm_data (the restatement of the reference's extract_asm_data,
solver/asm_data.inc:99-173).

* CPU: argument checks precede any device call.
* GPU: on small meshes of every order and on the benchmark mesh at its size,
  every integer array (DOF map, signs, face orientations, attributes, the
  essential DOFs, the DOF count) and the Jacobians and origins are equal;
  Jinv and detJ (adjugate on the device, LU on the host) agree to 1e-14;
  the matrix assembled from the device-extracted data equals the one from
  the host data to 1e-13 of its largest entry.
"""

from __future__ import annotations

import ctypes as ct
import time

import numpy as np
import pytest

from lithofem_b200 import _lib, configs, space
from lithofem_b200._abi import c_double_p, c_int_p


def _call(ne, nv, p, tv, xv):
    nd = p * (p + 2) * (p + 3) // 2
    bufs = [np.empty(ne * nd, np.int32), np.empty(ne * nd), np.empty(ne * 4, np.int32),
            np.empty(ne * 9), np.empty(ne * 9), np.empty(ne), np.empty(ne * 3),
            np.empty(ne * nd, np.int32)]
    h, n = ct.c_int(), ct.c_int()
    ptr = [b.ctypes.data_as(c_int_p if b.dtype == np.int32 else c_double_p) for b in bufs]
    return _lib.lib().lfasm_extract(0, ne, nv, p, tv.ctypes.data_as(c_int_p),
                                    xv.ctypes.data_as(c_double_p), *ptr[:7], ptr[7], ne * nd,
                                    ct.byref(h), ct.byref(n))


def test_argument_checks_precede_device_use():
    m = configs.small_case("slab", 1, 0.0).mesh
    tv = np.ascontiguousarray(m.tv, dtype=np.int32)
    xv = np.ascontiguousarray(m.xv, dtype=np.float64)
    assert _call(m.ne, m.nv, 4, tv, xv) == 3
    assert b"outside 1..3" in _lib.lib().lfasm_last_error()
    bad = tv.copy()
    bad[7, 2] = m.nv
    assert _call(m.ne, m.nv, 1, bad, xv) == 1
    assert b"element 7 vertex 2" in _lib.lib().lfasm_last_error()
    assert _call(0, m.nv, 1, tv, xv) == 1
    assert _call(m.ne, 1 << 21, 1, tv, xv) == 1


def _compare(mesh, p, prob):
    t0 = time.perf_counter()
    host = space.build_asm_data(mesh, p, prob)
    t1 = time.perf_counter()
    dev = space.build_asm_data_device(mesh, p, prob)
    t2 = time.perf_counter()
    for f in ("dof", "sign", "fo", "attr", "ess", "J", "v0"):
        assert np.array_equal(getattr(host, f), getattr(dev, f)), f
    assert host.height == dev.height
    for f in ("Jinv", "detJ"):
        a, b = getattr(host, f), getattr(dev, f)
        assert np.abs(a - b).max() <= 1e-14 * np.abs(a).max(), f
    return host, dev, t1 - t0, t2 - t1


@pytest.mark.gpu
@pytest.mark.parametrize("kind,p", [("grating", 1), ("grating", 2), ("grating", 3), ("hole", 2),
                                    ("slab", 3)])
def test_device_extraction_equals_host(kind, p):
    from lithofem_b200.asm import AsmGpuGlobal
    c = configs.small_case(kind, p, 6.0, seed=None)
    host, dev, _, _ = _compare(c.mesh, p, c.prob)
    vals = []
    for ad in (host, dev):
        g = AsmGpuGlobal(c.prob)
        assert g.Init(ad, 0) and g.BuildGlobal(ad.ess) and g.Assemble(True)
        vals.append(g.DownloadValues())
        g.Release()
    assert np.array_equal(vals[0] != 0, vals[1] != 0)
    scale = np.abs(vals[0]).max()
    assert np.abs(vals[0] - vals[1]).max() <= 1e-13 * scale


@pytest.mark.gpu
def test_device_extraction_of_a_polygon_hole_mesh():
    from lithofem_b200.mesh_poly import build_poly_mesh
    rng = np.random.default_rng(9)
    st = configs.poly_hole_stack(rng, lx=24.0, ly=24.0, z_max=30.0, t_range=(10.0, 14.0),
                                 pml_wl=0.3)
    mesh = build_poly_mesh(st, st.frustums[0], 4.0)
    _compare(mesh, 3, None)


@pytest.mark.gpu
def test_device_extraction_at_the_benchmark_size():
    c = configs.config(3)
    _, dev, t_host, t_dev = _compare(c.mesh, 3, c.prob)
    print(f"C3 extraction: n={dev.height} host {t_host:.3f} s, device (incl. copies) {t_dev:.3f} s")
