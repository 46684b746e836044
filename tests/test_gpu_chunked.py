"""Chunked assembly (lfasm_assemble with the element rows kept in L2).

The elements are taken in chunks of consecutive centroid height and the
rows each chunk completes are gathered right after it, every element row
dropped from L2 once added (discard.global.L2).  Each row still sums its
element rows in the same order, so the chunked CSR equals the one-pass
assembly bit for bit.  The path is optional: LFASM_CHUNK_MB (element-row
megabytes per chunk, read when the structure is built; default 0, one
pass) turns it on; 0.05 makes many chunks of these small meshes.
"""

from __future__ import annotations

import numpy as np
import pytest

from lithofem_b200 import configs
from lithofem_b200.asm import AsmGpuGlobal
from oracle import oracle

pytestmark = pytest.mark.gpu

CASES = {"grating-p3": lambda: configs.small_case("grating", 3, 6.0, seed=13, h=3.2),
         "hole-p2": lambda: configs.small_case("hole", 2, 6.0, seed=13, h=2.4),
         "slab-p1": lambda: configs.small_case("slab", 1, 0.0, seed=13, h=1.8),
         "poly-p3": lambda: configs.small_poly_case(3, 6.0, seed=5)}


def _assemble(c, elim, mb, monkeypatch, reps=2):
    monkeypatch.setenv("LFASM_CHUNK_MB", mb)
    g = AsmGpuGlobal(c.prob)
    assert g.Init(c.ad, 0) and g.BuildGlobal(c.ad.ess)
    out = None
    for _ in range(reps):          # the captured sequence, launched again
        assert g.Assemble(elim), g.last_error
        v = g.DownloadValues()
        assert out is None or np.array_equal(v.view(np.float64), out.view(np.float64))
        out = v
    g.Release()
    return out


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("elim", [True, False])
def test_chunked_equals_one_pass_bitwise(name, elim, monkeypatch):
    c = CASES[name]()
    one = _assemble(c, elim, "0", monkeypatch)
    many = _assemble(c, elim, "0.05", monkeypatch)
    assert np.array_equal(one.view(np.float64), many.view(np.float64))
    I, J = oracle.csr(c.ad)
    ref = oracle.assemble(c.ad, c.prob, I, J, c.ad.ess, elim)
    assert np.abs(many - ref).max() / np.abs(ref).max() < 1e-13
