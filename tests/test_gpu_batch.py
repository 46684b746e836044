"""Polygon-hole meshes on the GPU and batched (one CUDA graph) assembly.

Parity of the assembly on the batched workload's meshes against the oracle,
and lfasm_batch_assemble against per-handle lfasm_assemble (bit-identical:
the same kernels on the same data)."""

from __future__ import annotations

import ctypes as ct

import numpy as np
import pytest

from lithofem_b200 import _lib, configs
from lithofem_b200.asm import CROSS0, CROSS1, CURLCURL, KLK, MASS, AsmBatch, AsmGpu, AsmGpuGlobal
from lithofem_b200.asm import DeviceVector
from oracle import oracle

pytestmark = pytest.mark.gpu
TOL = 1e-13


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


_cache: dict = {}


def poly(p, theta, seed):
    key = (p, theta, seed)
    if key not in _cache:
        _cache[key] = configs.small_poly_case(p, theta, seed=seed)
    return _cache[key]


@pytest.mark.parametrize("p,theta,seed", [(1, 6.0, 3), (2, 6.0, 4), (3, 6.0, 5), (2, 0.0, 6)])
def test_polygon_hole_parity(p, theta, seed):
    c = poly(p, theta, seed)
    mm = MASS | ((CROSS0 | CROSS1 | KLK) if c.prob.has_kpar else 0)
    loc = AsmGpu(c.prob)
    assert loc.Init(c.ad, 0) and loc.ComputeLocal(CURLCURL, mm, True)
    assert rel(loc.DownloadLocal(), oracle.local(c.ad, c.prob, CURLCURL, mm, True)) < TOL
    g = AsmGpuGlobal(c.prob)
    assert g.Init(c.ad, 0) and g.BuildGlobal(c.ad.ess)
    I, J = g.DownloadCsr()
    Io, Jo = oracle.csr(c.ad)
    assert np.array_equal(I, Io) and np.array_equal(J, Jo)
    assert g.Assemble(True)
    assert rel(g.DownloadValues(), oracle.assemble(c.ad, c.prob, Io, Jo, c.ad.ess, True)) < TOL


def _zero_values(g):
    import torch
    _, _, V, _, nz = g._csr()
    torch.as_tensor(DeviceVector(V, (2 * nz,), "<f8"), device="cuda").zero_()
    torch.cuda.synchronize()


def test_batch_equals_per_handle_assembly():
    cases = [poly(1, 6.0, 3), poly(2, 6.0, 4), poly(3, 6.0, 5),
             configs.small_case("grating", 2, 6.0, seed=13, h=2.4)]
    hs = []
    for c in cases:
        g = AsmGpuGlobal(c.prob)
        assert g.Init(c.ad, 0) and g.BuildGlobal(c.ad.ess)
        hs.append(g)
    for elim in (True, False):
        ref = []
        for g in hs:
            assert g.Assemble(elim)
            ref.append(g.DownloadValues())
        b = AsmBatch(hs)
        for _ in range(2):
            for g in hs:
                _zero_values(g)
            n0 = _lib.lib().lfasm_launch_count()
            assert b.Assemble(elim)
            assert _lib.lib().lfasm_launch_count() - n0 >= 2 * len(hs)
            for g, r in zip(hs, ref):
                np.testing.assert_array_equal(g.DownloadValues(), r)
        b.Release()
    # the batch left the handles usable on their own
    assert hs[0].Assemble(True)


def test_handles_built_from_threads():
    """lfasm_init / lfasm_build_global from several host threads at once
    (the library's caches and memory pool are shared): every handle then
    assembles exactly what it does when built alone."""
    import concurrent.futures as cf
    cases = [poly(1, 6.0, 3), poly(2, 6.0, 4), poly(3, 6.0, 5),
             configs.small_case("hole", 2, 6.0, seed=13, h=2.4)]

    def make(c):
        g = AsmGpuGlobal(c.prob)
        ok = g.Init(c.ad, 0) and g.BuildGlobal(c.ad.ess)
        return g, ok

    ref = []
    for c in cases:
        g, ok = make(c)
        assert ok and g.Assemble(True)
        ref.append(g.DownloadValues())
        g.Release()
    for _ in range(2):
        with cf.ThreadPoolExecutor(max_workers=len(cases)) as ex:
            built = list(ex.map(make, cases))
        assert all(ok for _, ok in built)
        hs = [g for g, _ in built]
        b = AsmBatch(hs)
        assert b.Assemble(True)
        for g, r in zip(hs, ref):
            np.testing.assert_array_equal(g.DownloadValues(), r)
        b.Release()
        for g in hs:
            g.Release()


def test_batch_argument_errors():
    with pytest.raises(RuntimeError, match="empty batch"):
        AsmBatch([])
    c = poly(1, 6.0, 3)
    g = AsmGpuGlobal(c.prob)
    assert g.Init(c.ad, 0)
    with pytest.raises(RuntimeError, match="lfasm_build_global has not run"):
        AsmBatch([g])
    assert g.BuildGlobal(c.ad.ess)
    with pytest.raises(RuntimeError, match="repeats"):
        AsmBatch([g, g])
    h = ct.c_void_p()
    assert _lib.lib().lfasm_batch_assemble(h, 1) == 1
