"""Allocation-free residual entry point, checked against the regular one.

``lfasm_csr_residual_noalloc`` serves callers that cannot call cudaMalloc
while they run -- an iterative-refinement loop whose device memory is all
held by the sparse factorization, or a host framework that owns every
device allocation through its own pool.  It computes the same ||A x - b|| /
||b|| as ``lfasm_residual_device`` but keeps its partial sums in a fixed
array inside the library instead of allocating them.

The file name sorts last so that a run stopping at the first failure has
already run every other test; it also passes when run on its own.
"""

from __future__ import annotations

import ctypes as ct

import numpy as np
import pytest

from lithofem_b200 import _lib, configs
from lithofem_b200.asm import AsmGpuGlobal

pytestmark = pytest.mark.gpu
RTOL = 1e-12          # the residual tolerance of the other GPU tests
MAX_ROWS = 8 * (1 << 18)


def _noalloc(n, I, J, V, x, b):
    rel = ct.c_double(-1.0)
    rc = _lib.lib().lfasm_csr_residual_noalloc(int(n), ct.c_void_p(I), ct.c_void_p(J),
                                              ct.c_void_p(V), ct.c_void_p(x), ct.c_void_p(b),
                                              ct.byref(rel), None)
    return rc, rel.value


def test_noalloc_residual_matches_regular_entry_point():
    import torch
    c = configs.small_case("grating", 2, 6.0, seed=21)
    g = AsmGpuGlobal(c.prob)
    assert g.Init(c.ad, 0) and g.BuildGlobal(c.ad.ess) and g.Assemble(True)
    I, J, V, n, nnz = g._csr()
    rng = np.random.default_rng(9)
    x = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).cuda()
    for call in range(2):  # two calls in a row, different right-hand sides
        b = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n)).cuda()
        ok, ref = g.ResidualDevice(x.data_ptr(), b.data_ptr())
        assert ok
        rc, got = _noalloc(n, I, J, V, x.data_ptr(), b.data_ptr())
        assert rc == 0, _lib.lib().lfasm_last_error()
        assert abs(got - ref) <= RTOL * ref, (call, got, ref)
    # an exact solution gives zero
    y = torch.zeros(n, dtype=torch.complex128, device="cuda")
    assert g.SpMV(x.data_ptr(), y.data_ptr())
    rc, got = _noalloc(n, I, J, V, x.data_ptr(), y.data_ptr())
    assert rc == 0 and got < 1e-15


def test_noalloc_rejects_sizes_beyond_its_scratch():
    rc, _ = _noalloc(MAX_ROWS + 1, 0, 0, 0, 0, 0)
    assert rc == 3
    assert b"allocation-free residual limit" in _lib.lib().lfasm_last_error()


def test_noalloc_residual_at_its_row_limit():
    """n exactly at the limit (2,097,152 rows): the last block's partial sums
    sit next to the result slots.  A diagonal CSR gives the closed form
    ||d x - b|| / ||b||, checked on two calls in a row."""
    import torch
    n = MAX_ROWS
    rng = np.random.default_rng(17)
    I = torch.arange(n + 1, dtype=torch.int32, device="cuda")
    J = torch.arange(n, dtype=torch.int32, device="cuda")
    d = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    V = torch.from_numpy(d).cuda()
    xd = torch.from_numpy(x).cuda()
    for call in range(2):
        b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        if call == 1:
            b = d * x + 1e-3 * b          # a nearly exact right-hand side
        want = float(np.linalg.norm(d * x - b) / np.linalg.norm(b))
        bd = torch.from_numpy(b).cuda()
        rc, got = _noalloc(n, I.data_ptr(), J.data_ptr(), V.data_ptr(), xd.data_ptr(),
                           bd.data_ptr())
        assert rc == 0, _lib.lib().lfasm_last_error()
        assert abs(got - want) <= RTOL * want, (call, got, want)
