"""The oracle (CPU restatement) pinned to the reference's own assembler.

Golden fixtures in tests/golden were produced by the reference's
reassemble_all / build_csr_symbolic / reassemble_element compiled from its
sources (tests/golden/make_golden.py).  The live comparison runs where
oracle/_ref/libref_asm.so exists.
"""

from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np
import pytest

from lithofem_b200 import configs
from oracle import oracle

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import make_golden as G  # noqa: E402

GOLDEN = sorted((Path(__file__).resolve().parent / "golden").glob("ref_*.npz"))


def _case_from_name(path: Path):
    _, kind, p, t = path.stem.split("_")
    return kind, int(p[1:]), float(t[1:])


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_matches_reference_golden(path):
    g = np.load(path)
    kind, p, theta = _case_from_name(path)
    c = G.case_of(kind, p, theta)
    assert G.digest(c.ad) == str(g["digest"]), "inputs drifted from the fixture"
    I, J = oracle.csr(c.ad)
    assert np.array_equal(I, g["I"])
    assert G.sha(J) == str(g["J_sha"]) and len(J) == int(g["nnz"])
    vals = oracle.assemble(c.ad, c.prob, I, J, c.ad.ess, eliminate=False)
    ref_sub = g["vals_sub"]
    scale = np.abs(ref_sub).max()
    assert np.abs(vals[::G.STRIDE] - ref_sub).max() / scale < 1e-13
    cs = G.checksums(vals)
    assert np.allclose(cs, g["checksums"], rtol=1e-12, atol=0)
    loc = oracle.local(c.ad, c.prob, 1, 2 | (28 if c.prob.has_kpar else 0), True)
    for e, m in zip(g["elements"], g["element_mats"]):
        assert np.abs(loc[e] - m).max() / np.abs(m).max() < 1e-13


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("kind,p,theta", [("grating", 1, 6.0), ("hole", 2, 6.0), ("slab", 3, 0.0)])
def test_oracle_matches_reference_live(kind, p, theta):
    c = configs.small_case(kind, p, theta, seed=19, h={1: 2.0, 2: 3.0, 3: 4.0}[p])
    rc = oracle.RefContext(c.ad, c.prob)
    I, J = rc.build_csr()
    Io, Jo = oracle.csr(c.ad)
    assert np.array_equal(I, Io) and np.array_equal(J, Jo)
    v_ref = rc.reassemble()
    v = oracle.assemble(c.ad, c.prob, I, J, c.ad.ess, eliminate=False)
    assert np.abs(v - v_ref).max() / np.abs(v_ref).max() < 1e-13


@pytest.mark.parametrize("p", [1, 2, 3])
def test_symmetry_at_normal_incidence(p):
    """||A - A^T|| / ||A|| < 1e-12 at k-parallel = 0 (tests/test_mms.py:59)."""
    c = configs.small_case("hole", p, 0.0, h={1: 2.4, 2: 3.0, 3: 4.0}[p])
    I, J = oracle.csr(c.ad)
    v = oracle.assemble(c.ad, c.prob, I, J, c.ad.ess, eliminate=True)
    import scipy.sparse as sp
    A = sp.csr_matrix((v, J, I), shape=(c.ad.height,) * 2)
    assert abs(A - A.T).max() / abs(A).max() < 1e-12


@pytest.mark.parametrize("p", [1, 2])
def test_transpose_is_opposite_kpar(p):
    """A(k)^T = A(-k): the cross terms are antisymmetric, the rest symmetric."""
    c = configs.small_case("grating", p, 6.0, h={1: 2.4, 2: 3.0}[p])
    I, J = oracle.csr(c.ad)
    import copy
    import scipy.sparse as sp
    v = oracle.assemble(c.ad, c.prob, I, J, c.ad.ess, eliminate=False)
    pm = copy.copy(c.prob)
    pm.kx, pm.ky = -c.prob.kx, -c.prob.ky
    vm = oracle.assemble(c.ad, pm, I, J, c.ad.ess, eliminate=False)
    A = sp.csr_matrix((v, J, I), shape=(c.ad.height,) * 2)
    Am = sp.csr_matrix((vm, J, I), shape=(c.ad.height,) * 2)
    assert abs(A.T - Am).max() / abs(A).max() < 1e-12
    assert abs(A - A.T).max() / abs(A).max() > 1e-6  # genuinely non-symmetric


def test_host_csr_matches_oracle():
    c = configs.small_case("grating", 2, 0.0)
    I, J = oracle.csr(c.ad)
    assert np.array_equal(I, c.ad.I) and np.array_equal(J, c.ad.Jcol)


def test_spmv_residual():
    c = configs.small_case("slab", 1, 0.0)
    I, J = oracle.csr(c.ad)
    v = oracle.assemble(c.ad, c.prob, I, J, c.ad.ess, eliminate=True)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(c.ad.height) + 1j * rng.standard_normal(c.ad.height)
    y, rel = oracle.spmv(I, J, v, x, b=None)
    import scipy.sparse as sp
    A = sp.csr_matrix((v, J, I), shape=(c.ad.height,) * 2)
    assert np.abs(y - A @ x).max() / np.abs(y).max() < 1e-14
    _, rel = oracle.spmv(I, J, v, x, b=y)
    assert rel == 0.0
