"""The device sparse solver (liblfsolve.so) on assembled systems.

The CPU reference is SciPy's SuperLU (complex128, in place of UMFPACK, which
is not installed) on the same CSR, downloaded from the device.  Checked:
* complex128 factors: ||A x - b|| / ||b|| <= 1e-11 (about cond(A) times the
  FP64 rounding unit) and the solution equal to SuperLU's to 1e-10;
* complex64 factors + FP64 refinement: residual <= 1e-10 (the stated target)
  and the solution within 1e-8 of the complex128 one;
* the transposed solve A^T x = b with the same factors (the adjoint system),
  plain and refined, against SuperLU on A^T;
* several right-hand sides at once (more than one solve pass), the s / p
  columns of a source;
* the benchmark's C1 mesh at its full size;
* the batched (padded) and per-front factorization paths on one system.
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
RES128 = 1e-11                  # residual bound of an unrefined complex128 solve
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
    assert rel_res(A, X, B) <= RES128
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
    assert rel_res(A.T.tocsr(), X, B) <= RES128
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
    assert rel_res(host_matrix(g), X, Bh) <= RES128
    s.Release()


def test_full_size_c1():
    """The benchmark's C1 mesh at full size (47k DOF, 4095 fronts, batched
    depths): the complex128 solve's residual on the host matrix, and the
    refined complex64 solve against it (SuperLU needs minutes here; it is
    the reference on the smaller systems above)."""
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
    assert s.AnalyzeAssembly(g, c.ad) and s.FactorDevice(g._csr()[2], C128)
    x128 = torch.empty_like(b)
    assert s.Backsolve(1, b.data_ptr(), x128.data_ptr())
    A = host_matrix(g)
    X128 = x128.cpu().numpy().reshape(n, 1)
    assert rel_res(A, X128, bh.reshape(n, 1)) <= RES128
    assert s.FactorDevice(g._csr()[2], C64)
    x = torch.empty_like(b)
    ok, rel, it = s.SolveRefined(g, 1, b.data_ptr(), x.data_ptr(), tol=1e-10)
    assert ok, (s.last_error, rel, it)
    assert rel_err(x.cpu().numpy().reshape(n, 1), X128) <= 1e-8
    print(f"C1: n={n} refined in {it} corrections, residual {rel[0]:.2e}; {s.Stats()}")
    s.Release()
    g.Release()


@pytest.mark.parametrize("kcase", [("grating", 3, 6.0), ("hole", 3, 0.0), ("grating", 2, 6.0)],
                         ids=["grating-p3", "hole-p3", "grating-p2"])
def test_batched_depths_equal_per_front_factorization(kcase, monkeypatch):
    """Depths with many fronts are factored by batched calls on a padded
    layout; forcing that path on every depth of at least 4 fronts gives the
    same solution as the per-front path, in both precisions."""
    import torch
    c, g, b = system(kcase)
    n = c.ad.height
    A = host_matrix(g)
    B = b.cpu().numpy().reshape(2, n).T
    out = {}
    for label, env in (("per-front", "100000"), ("batched", "4")):
        monkeypatch.setenv("LFSOLVE_BATCH_MIN", env)
        s = DirectSolver(0)
        assert s.AnalyzeAssembly(g, c.ad)
        for prec in (C128, C64):
            assert s.FactorDevice(g._csr()[2], prec), s.last_error
            x = torch.empty_like(b)
            assert s.Backsolve(2, b.data_ptr(), x.data_ptr()), s.last_error
            out[(label, prec)] = x.cpu().numpy().reshape(2, n).T
        ok, rel, _ = s.SolveRefined(g, 2, b.data_ptr(), x.data_ptr(), tol=1e-10)
        assert ok and max(rel) <= 1e-10, (label, s.last_error, rel)
        s.Release()
    assert rel_res(A, out[("batched", C128)], B) <= RES128
    assert rel_err(out[("batched", C128)], out[("per-front", C128)]) <= 1e-11
    # unrefined complex64 solutions carry the factorization's own error
    # (about cond(A) * 2^-24); both orders of arithmetic must be as accurate
    # as each other against complex128
    e_b = rel_err(out[("batched", C64)], out[("batched", C128)])
    e_p = rel_err(out[("per-front", C64)], out[("per-front", C128)])
    assert max(e_b, e_p) <= 1e-2 and max(e_b, e_p) <= 10 * min(e_b, e_p) + 1e-6, (e_b, e_p)


@pytest.mark.parametrize("batch_min", ["100000", "4"], ids=["per-front", "batched"])
@pytest.mark.parametrize("kcase", [("grating", 3, 6.0), ("hole", 3, 0.0)], ids=["grating-p3", "hole-p3"])
def test_tf32x3_schur_updates_refine_to_1e10(kcase, batch_min, monkeypatch):
    """Large complex64 fronts update their Schur complement with three TF32
    tensor-core GEMMs on split operands (about 2^-22 relative); forced on
    every front, on the per-front path and on the batched depths (strided
    batched GEMMs), the refined solve still reaches 1e-10 and agrees with
    the complex128 solution."""
    import torch
    c, g, b = system(kcase)
    monkeypatch.setenv("LFSOLVE_BATCH_MIN", batch_min)
    s = DirectSolver(0)
    assert s.AnalyzeAssembly(g, c.ad) and s.FactorDevice(g._csr()[2], C128)
    x128 = torch.empty_like(b)
    assert s.Backsolve(2, b.data_ptr(), x128.data_ptr())
    monkeypatch.setenv("LFSOLVE_TF32X3_MIN", "1")
    assert s.FactorDevice(g._csr()[2], C64), s.last_error
    x = torch.empty_like(b)
    ok, rel, it = s.SolveRefined(g, 2, b.data_ptr(), x.data_ptr(), tol=1e-10)
    assert ok and max(rel) <= 1e-10, (s.last_error, rel, it)
    assert rel_err(x.cpu().numpy(), x128.cpu().numpy()) <= 1e-8
    s.Release()


@pytest.mark.parametrize("transpose", [False, True], ids=["A", "AT"])
def test_gmres_ir_forced_from_the_start(transpose, monkeypatch):
    """GMRES-based refinement (restarted GMRES(30) in FP64, right
    preconditioned by the complex64 factors) reaches 1e-10 and agrees with
    the complex128 solution, for A and for A^T."""
    import torch
    c, g, b = system(("grating", 2, 6.0))
    s = DirectSolver(0)
    assert s.AnalyzeAssembly(g, c.ad) and s.FactorDevice(g._csr()[2], C128)
    xref = torch.empty_like(b)
    assert s.Backsolve(2, b.data_ptr(), xref.data_ptr(), transpose)
    assert s.FactorDevice(g._csr()[2], C64)
    monkeypatch.setenv("LFSOLVE_GMRES", "1")
    x = torch.empty_like(b)
    ok, rel, it = s.SolveRefined(g, 2, b.data_ptr(), x.data_ptr(), transpose, 1e-10)
    assert ok and max(rel) <= 1e-10, (s.last_error, rel, it)
    assert 1 <= it <= 60
    assert rel_err(x.cpu().numpy(), xref.cpu().numpy()) <= 1e-8
    s.Release()


def test_gmres_ir_takes_over_when_refinement_stalls(monkeypatch):
    """Factors of a perturbed matrix (every value times 1 + d u, u uniform in
    [-1, 1]): at the first d where classical refinement alone no longer
    converges, the automatic switch to GMRES-IR still reaches 1e-10 on the
    true matrix."""
    import torch
    c, g, b = system(("grating", 2, 6.0))
    V = g.DownloadValues()
    rng = np.random.default_rng(21)
    u = rng.uniform(-1.0, 1.0, V.shape)
    s = DirectSolver(0)
    assert s.AnalyzeAssembly(g, c.ad)
    x = torch.empty_like(b)
    seen = []
    for d in (1e-4, 1e-3, 3e-3, 1e-2, 3e-2):
        Vp = torch.from_numpy(V * (1.0 + d * u)).cuda()
        assert s.FactorDevice(Vp.data_ptr(), C64)
        monkeypatch.setenv("LFSOLVE_GMRES", "0")
        ok_ir, rel_ir, it_ir = s.SolveRefined(g, 2, b.data_ptr(), x.data_ptr(), False, 1e-10)
        monkeypatch.delenv("LFSOLVE_GMRES")
        ok, rel, it = s.SolveRefined(g, 2, b.data_ptr(), x.data_ptr(), False, 1e-10)
        seen.append((d, ok_ir, max(rel_ir), it_ir, ok, max(rel), it))
        print(f"perturbation {d:.0e}: refinement alone ok={ok_ir} rel={max(rel_ir):.2e} "
              f"({it_ir}); with GMRES-IR ok={ok} rel={max(rel):.2e} ({it})")
        if not ok_ir:
            assert ok and max(rel) <= 1e-10, seen
            break
    else:
        pytest.fail(f"refinement converged at every perturbation: {seen}")
    s.Release()
