"""The device sparse solver (liblfsolve.so) on assembled systems.

The CPU reference is SciPy's SuperLU (complex128, in place of UMFPACK, which
is not installed) on the same CSR, downloaded from the device.  Checked:
* complex128 factors: ||A x - b|| / ||b|| <= 1e-12 and the solution equal to
  SuperLU's to 1e-10;
* complex64 factors + FP64 refinement: residual <= 1e-10 (the stated target)
  and the solution within 1e-8 of the complex128 one;
* the transposed solve A^T x = b with the same factors (the adjoint system),
  plain and refined, against SuperLU on A^T;
* several right-hand sides at once (more than one solve pass), the s / p
  columns of a source;
* the benchmark's C1 mesh at its full size.
"""

from __future__ import annotations

import numpy as np
import pytest

from lithofem_b200 import configs, incident
from lithofem_b200.asm import AsmGpuGlobal
from lithofem_b200.solver import C64, C128, DirectSolver

pytestmark = pytest.mark.gpu
CASES = [("grating", 2, 6.0), ("hole", 3, 0.0), ("slab", 1, 0.0), ("hole", 1, 6.0),
         ("grating", 3, 6.0)]
H = {1: 1.6, 2: 2.0, 3: 3.4}    # mesh sizes: systems SuperLU factors in seconds
_cache: dict = {}


def system(kcase):
    """Assembled, eliminated system on the device with its s/p RHS."""
    import torch
    if kcase in _cache:
        return _cache[kcase]
    c = configs.small_case(*kcase, seed=5, h=H[kcase[1]])
    g = AsmGpuGlobal(c.prob)
    assert g.Init(c.ad, 0) and g.BuildGlobal(c.ad.ess) and g.Assemble(True)
    n = c.ad.height
    parts = [incident.planewave_parts(c.stack, c.theta, 0.0, pol, 1.0, True) for pol in ("s", "p")]
    b = torch.zeros(2 * n, dtype=torch.complex128, device="cuda")
    assert g.AssembleRHS(parts, [0, 1], 2, True, b.data_ptr())
    if float(b.abs().max()) == 0.0:   # no scatterer (the bare slab): a seeded RHS
        rng = np.random.default_rng(11)
        bh = rng.standard_normal((2, n)) + 1j * rng.standard_normal((2, n))
        bh[:, c.ad.ess] = 0.0
        b.copy_(torch.from_numpy(bh.reshape(-1)))
    _cache.clear()
    _cache[kcase] = (c, g, b)
    return _cache[kcase]


def host_matrix(g):
    import scipy.sparse as sp
    I, J = g.DownloadCsr()
    V = g.DownloadValues()
    n = len(I) - 1
    return sp.csr_matrix((V, J, I), shape=(n, n))


def superlu(A, B):
    import scipy.sparse.linalg as sla
    lu = sla.splu(A.tocsc())
    return np.stack([lu.solve(B[:, c]) for c in range(B.shape[1])], axis=1)


def rel_res(A, X, B):
    return max(np.linalg.norm(A @ X[:, c] - B[:, c]) / np.linalg.norm(B[:, c])
               for c in range(B.shape[1]))


def rel_err(X, Y):
    return float(np.linalg.norm(X - Y) / np.linalg.norm(Y))


@pytest.mark.parametrize("kcase", CASES, ids=[f"{k}-p{p}-t{t:g}" for k, p, t in CASES])
def test_complex128_factor_solve(kcase):
    import torch
    c, g, b = system(kcase)
    n = c.ad.height
    s = DirectSolver(0)
    assert s.AnalyzeAssembly(g, c.ad), s.last_error
    assert s.FactorDevice(g._csr()[2], C128), s.last_error
    x = torch.empty_like(b)
    assert s.Backsolve(2, b.data_ptr(), x.data_ptr()), s.last_error
    A = host_matrix(g)
    B = b.cpu().numpy().reshape(2, n).T
    X = x.cpu().numpy().reshape(2, n).T
    assert rel_res(A, X, B) <= 1e-12
    assert rel_err(X, superlu(A, B)) <= 1e-10
    st = s.Stats()
    assert st["n_fronts"] > 1 and st["factor_ms"] > 0
    s.Release()


@pytest.mark.parametrize("kcase", CASES, ids=[f"{k}-p{p}-t{t:g}" for k, p, t in CASES])
def test_complex64_refined_to_1e10(kcase):
    import torch
    c, g, b = system(kcase)
    n = c.ad.height
    s = DirectSolver(0)
    assert s.AnalyzeAssembly(g, c.ad)
    assert s.FactorDevice(g._csr()[2], C128)
    x128 = torch.empty_like(b)
    assert s.Backsolve(2, b.data_ptr(), x128.data_ptr())
    assert s.FactorDevice(g._csr()[2], C64), s.last_error
    x = torch.empty_like(b)
    ok, rel, iters = s.SolveRefined(g, 2, b.data_ptr(), x.data_ptr(), tol=1e-10)
    assert ok, (s.last_error, rel, iters)
    A = host_matrix(g)
    B = b.cpu().numpy().reshape(2, n).T
    X = x.cpu().numpy().reshape(2, n).T
    assert max(rel) <= 1e-10 and rel_res(A, X, B) <= 1e-10
    assert rel_err(X, x128.cpu().numpy().reshape(2, n).T) <= 1e-8
    s.Release()


@pytest.mark.parametrize("kcase", [("grating", 2, 6.0), ("hole", 1, 6.0), ("grating", 3, 6.0)],
                         ids=["grating-p2", "hole-p1", "grating-p3"])
def test_transposed_solve_with_the_same_factors(kcase):
    import torch
    c, g, b = system(kcase)
    n = c.ad.height
    A = host_matrix(g)
    B = b.cpu().numpy().reshape(2, n).T
    want = superlu(A.T.tocsr(), B)
    s = DirectSolver(0)
    assert s.AnalyzeAssembly(g, c.ad)
    assert s.FactorDevice(g._csr()[2], C128)
    x = torch.empty_like(b)
    assert s.Backsolve(2, b.data_ptr(), x.data_ptr(), transpose=True), s.last_error
    X = x.cpu().numpy().reshape(2, n).T
    assert rel_res(A.T.tocsr(), X, B) <= 1e-12
    assert rel_err(X, want) <= 1e-10
    assert s.FactorDevice(g._csr()[2], C64)
    ok, rel, _ = s.SolveRefined(g, 2, b.data_ptr(), x.data_ptr(), transpose=True, tol=1e-10)
    assert ok, (s.last_error, rel)
    X = x.cpu().numpy().reshape(2, n).T
    assert rel_res(A.T.tocsr(), X, B) <= 1e-10
    assert rel_err(X, want) <= 1e-8
    s.Release()


def test_several_right_hand_sides_in_passes():
    import torch
    c, g, b = system(("grating", 2, 6.0))
    n = c.ad.height
    rng = np.random.default_rng(3)
    Bh = rng.standard_normal((n, 5)) + 1j * rng.standard_normal((n, 5))
    Bh[c.ad.ess] = 0.0
    Bd = torch.from_numpy(np.ascontiguousarray(Bh.T)).cuda().reshape(-1)
    s = DirectSolver(0)
    assert s.AnalyzeAssembly(g, c.ad) and s.FactorDevice(g._csr()[2], C128)
    x = torch.empty_like(Bd)
    assert s.Backsolve(5, Bd.data_ptr(), x.data_ptr())
    X = x.cpu().numpy().reshape(5, n).T
    assert rel_res(host_matrix(g), X, Bh) <= 1e-12
    s.Release()


def test_full_size_c1_against_superlu():
    import torch
    c = configs.config(1)
    g = AsmGpuGlobal(c.prob)
    assert g.Init(c.ad, 0) and g.BuildGlobal(c.ad.ess) and g.Assemble(True)
    n = c.ad.height
    rng = np.random.default_rng(23)   # the bare slab has no scattered-field source
    bh = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    bh[c.ad.ess] = 0.0
    b = torch.from_numpy(bh).cuda()
    s = DirectSolver(0)
    assert s.AnalyzeAssembly(g, c.ad) and s.FactorDevice(g._csr()[2], C64)
    x = torch.empty_like(b)
    ok, rel, it = s.SolveRefined(g, 1, b.data_ptr(), x.data_ptr(), tol=1e-10)
    assert ok, (s.last_error, rel, it)
    A = host_matrix(g)
    B = b.cpu().numpy().reshape(n, 1)
    X = x.cpu().numpy().reshape(n, 1)
    assert rel_err(X, superlu(A, B)) <= 1e-8
    print(f"C1: n={n} refined in {it} corrections, residual {rel[0]:.2e}; {s.Stats()}")
    s.Release()
    g.Release()
