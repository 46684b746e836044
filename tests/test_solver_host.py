"""The sparse solver's host side (no GPU): the library loads and exports
every entry point of include/lfsolve.h; the nested-dissection analysis is a
valid elimination order for the mesh's system; the argument and state
checks; no CPU fallback.

Separator property: every coupling (i, j) of the matrix joins two rows
whose fronts lie on one root path (one is an ancestor of the other), so
eliminating a front never creates fill outside its own update rows.
"""

from __future__ import annotations

import ctypes as ct

import numpy as np
import pytest

from lithofem_b200 import configs, solver
from oracle import oracle


def test_library_exports_every_declared_entry_point():
    L = solver.lib()
    names = solver.exported_symbols()
    assert len(names) >= 10
    for nm in names:
        assert hasattr(L, nm), nm


def _analysed(kcase, **kw):
    c = configs.small_case(*kcase, seed=5, **kw)
    I, J = oracle.csr(c.ad)
    s = solver.DirectSolver(0)
    assert s.Analyze(c.ad, I, J), s.last_error
    return c, I, J, s


@pytest.mark.parametrize("kcase", [("grating", 3, 6.0), ("hole", 2, 6.0), ("slab", 1, 0.0)],
                         ids=["grating-p3", "hole-p2", "slab-p1"])
def test_ordering_is_a_valid_nested_dissection(kcase):
    c, I, J, s = _analysed(kcase)
    n = c.ad.height
    st = s.Stats()
    perm, node_of = s.Ordering()
    fr = s.Fronts()
    ess = np.zeros(n, dtype=bool)
    ess[c.ad.ess] = True
    # a bijection onto the non-essential rows
    assert len(perm) == n - ess.sum() == st["n"] - st["n_ess"]
    assert len(np.unique(perm)) == len(perm) and not ess[perm].any()
    # pivots of the fronts partition the numbered rows; depths follow parents
    assert fr["k"].sum() == len(perm)
    assert (fr["m"] >= fr["k"]).all() and fr["m"].max() == st["max_front"]
    par = fr["parent"]
    assert (par == -1).sum() == 1
    child = np.nonzero(par >= 0)[0]
    assert (fr["depth"][child] == fr["depth"][par[child]] + 1).all()
    assert np.bincount(node_of, minlength=len(par)).tolist() == fr["k"].tolist()
    # separator property over every coupling of the matrix
    iperm = np.full(n, -1)
    iperm[perm] = np.arange(len(perm))
    rows = np.repeat(np.arange(n), np.diff(I))
    keep = ~ess[rows] & ~ess[J]
    a = node_of[iperm[rows[keep]]]
    b = node_of[iperm[J[keep]]]
    depth = fr["depth"]

    def lift(x, d):
        x = x.copy()
        while True:
            up = depth[x] > d
            if not up.any():
                return x
            x[up] = par[x[up]]

    lo = np.minimum(depth[a], depth[b])
    ok = np.empty(len(a), dtype=bool)
    for d in np.unique(lo):
        sel = lo == d
        ok[sel] = lift(a[sel], d) == lift(b[sel], d)
    assert ok.all(), int((~ok).sum())
    assert st["factor_flops"] > 0 and st["factor_entries"] >= fr["k"].sum()
    s.Release()


def test_batched_depths_only_change_layout(monkeypatch):
    """The batching threshold changes the front layout, not the analysis."""
    out = []
    for env in ("100000", "4"):
        monkeypatch.setenv("LFSOLVE_BATCH_MIN", env)
        c, I, J, s = _analysed(("grating", 2, 6.0))
        perm, node = s.Ordering()
        st = s.Stats()
        out.append((perm, node, st["factor_entries"], st["factor_flops"],
                    st["peak_front_entries"]))
        s.Release()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2] and out[0][3] == out[1][3]
    assert out[1][4] >= out[0][4]        # padded fronts hold at least as much


def test_argument_and_state_checks():
    L = solver.lib()
    s = solver.DirectSolver(0)
    # factor and solve before any analysis
    assert L.lfsolve_factor(s._s, ct.c_void_p(1), 0) == 3
    assert L.lfsolve_solve(s._s, 1, ct.c_void_p(1), ct.c_void_p(1), 0) == 3
    c = configs.small_case("slab", 1, 0.0, seed=5)
    I, J = oracle.csr(c.ad)
    # a structure that is not symmetric is refused
    J2 = J.copy()
    r = 3
    J2[I[r]:I[r + 1]] = np.arange(I[r + 1] - I[r])   # rewrite one row's columns
    assert not s.Analyze(c.ad, I, J2)
    assert s.last_error[0] == 1
    # a row pointer that does not span the columns
    I2 = I.copy()
    I2[-1] -= 1
    assert not s.Analyze(c.ad, I2, J)
    assert s.last_error[0] == 1
    # unknown precision after a valid analysis
    assert s.Analyze(c.ad, I, J)
    assert L.lfsolve_factor(s._s, ct.c_void_p(1), 7) == 1
    s.Release()


def test_no_cpu_fallback():
    """Without a GPU the numeric factorization fails loudly."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    c, I, J, s = _analysed(("slab", 1, 0.0))
    rc = solver.lib().lfsolve_factor(s._s, ct.c_void_p(16), 0)
    assert rc == 2, rc
    assert b"CUDA error" in solver.lib().lfsolve_last_error()
    s.Release()
