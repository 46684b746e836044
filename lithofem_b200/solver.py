"""Sparse direct solve of the assembled system on the device (liblfsolve.so).

Mirrors the reference's cuDSS wrapper ``CuDssDirectSolver``
(solver/cudss_solver.inc:33-349): ``FactorDevice`` on the borrowed device
CSR of the assembly (the zero-copy entry, :186-203), ``Backsolve`` (:287-309)
and ``SolveDeviceCsr`` (:79-110, factor once, then solve; the factors are
reused by later calls), ``Release`` (:311).  The reference's methods return
``bool``; so do these, with the library's message in ``last_error``.  The
failure switch ``LITHOFEM_CUDSS_FORCE_FAIL`` (:81-86) makes
``SolveDeviceCsr`` fail the same way.

Beyond cuDSS: the factorization precision (complex64 or complex128), the
FP64-refined solve and the transposed solve A^T x = b with the same factors.
There is no CPU fallback: without the library or a device every call fails.
"""

from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

import numpy as np

from .asm import AsmGpuGlobal

LIB_PATH = Path(__file__).resolve().parent / "liblfsolve.so"
C64, C128 = 0, 1
_lib = None


class Stats(ct.Structure):
    _fields_ = [("n", ct.c_int), ("n_ess", ct.c_int), ("n_fronts", ct.c_int), ("depth", ct.c_int),
                ("max_front", ct.c_int), ("max_pivots", ct.c_int),
                ("factor_entries", ct.c_longlong), ("factor_flops", ct.c_double),
                ("peak_front_entries", ct.c_longlong), ("analyze_s", ct.c_double),
                ("factor_ms", ct.c_float), ("solve_ms", ct.c_float), ("refine_iters", ct.c_int),
                ("refine_rel", ct.c_double)]


def lib() -> ct.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__"
                           " as g; g.build()'` (the solver has no CPU fallback)")
    L = ct.CDLL(os.fspath(LIB_PATH))
    P, I, D, V = ct.c_void_p, ct.POINTER(ct.c_int), ct.POINTER(ct.c_double), ct.c_void_p
    sig = {
        "lfsolve_last_error": (ct.c_char_p, []),
        "lfsolve_create": (ct.c_int, [ct.c_int, ct.POINTER(P)]),
        "lfsolve_set_stream": (ct.c_int, [P, V]),
        "lfsolve_analyze": (ct.c_int, [P, ct.c_int, I, I, ct.c_longlong, ct.c_int, ct.c_int, I, D,
                                       I, ct.c_int, ct.c_int]),
        "lfsolve_factor": (ct.c_int, [P, V, ct.c_int]),
        "lfsolve_solve": (ct.c_int, [P, ct.c_int, V, V, ct.c_int]),
        "lfsolve_solve_refined": (ct.c_int, [P, V, V, V, ct.c_int, V, V, ct.c_int, ct.c_double,
                                             ct.c_int, D, I]),
        "lfsolve_get_stats": (ct.c_int, [P, ct.POINTER(Stats)]),
        "lfsolve_get_ordering": (ct.c_int, [P, I, I]),
        "lfsolve_get_fronts": (ct.c_int, [P, I, I, I, I]),
        "lfsolve_release_factors": (ct.c_int, [P]),
        "lfsolve_destroy": (None, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def exported_symbols() -> list[str]:
    """Entry points declared in include/lfsolve.h."""
    import re
    hdr = Path(__file__).resolve().parents[1] / "include" / "lfsolve.h"
    return sorted(set(re.findall(r"^(?:const\s+)?(?:int|void|const char)\s*\*?\s*(lfsolve_\w+)\s*\(",
                                 hdr.read_text(), flags=re.M)))


def centroids(ad) -> np.ndarray:
    """Element centroids v0 + J (1/4, 1/4, 1/4), (ne, 3)."""
    J = ad.J.reshape(ad.ne, 3, 3)
    return np.ascontiguousarray(ad.v0.reshape(ad.ne, 3) + J @ np.full(3, 0.25))


def _ip(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_int))


class DirectSolver:
    """Multifrontal LU of one assembled system on device ``gpu_id``."""

    def __init__(self, gpu_id: int = 0):
        self.gpu_id = gpu_id
        self.last_error = None
        self._s = ct.c_void_p()
        self._check(lib().lfsolve_create(gpu_id, ct.byref(self._s)))
        self._csr = None
        self.ready = False

    def _check(self, rc: int) -> bool:
        if rc != 0:
            self.last_error = (rc, lib().lfsolve_last_error().decode(errors="replace"))
            return False
        self.last_error = None
        return True

    def SetStream(self, stream: int) -> bool:
        return self._check(lib().lfsolve_set_stream(self._s, ct.c_void_p(stream)))

    def Analyze(self, ad, I: np.ndarray, J: np.ndarray, ess=None, leaf: int = 0) -> bool:
        """Ordering and symbolic factorization of the mesh's system: ad (the
        extracted mesh data), I/J (host CSR structure), ess (essential rows,
        default ad.ess)."""
        ess = np.ascontiguousarray(ad.ess if ess is None else ess, dtype=np.int32)
        I = np.ascontiguousarray(I, dtype=np.int32)
        J = np.ascontiguousarray(J, dtype=np.int32)
        dof = np.ascontiguousarray(ad.dof, dtype=np.int32)
        cen = centroids(ad)
        self._keep = (I, J, dof, cen, ess)
        ok = self._check(lib().lfsolve_analyze(self._s, int(ad.height), _ip(I), _ip(J), len(J),
                                               int(ad.ne), int(ad.nd), _ip(dof),
                                               cen.ctypes.data_as(ct.POINTER(ct.c_double)),
                                               _ip(ess), len(ess), int(leaf)))
        self.ready = False
        return ok

    def AnalyzeAssembly(self, g: AsmGpuGlobal, ad, leaf: int = 0) -> bool:
        """Analyze with the structure of an assembly handle's device CSR."""
        I, J = g.DownloadCsr()
        return self.Analyze(ad, I, J, g._ess, leaf)

    def FactorDevice(self, d_vals: int, prec: int = C64) -> bool:
        """Numeric factorization of the device CSR values (complex128)."""
        ok = self._check(lib().lfsolve_factor(self._s, ct.c_void_p(d_vals), int(prec)))
        self.ready = ok
        return ok

    def Backsolve(self, nrhs: int, d_b: int, d_x: int, transpose: bool = False) -> bool:
        return self._check(lib().lfsolve_solve(self._s, int(nrhs), ct.c_void_p(d_b),
                                               ct.c_void_p(d_x), int(transpose)))

    def SolveRefined(self, g: AsmGpuGlobal, nrhs: int, d_b: int, d_x: int,
                     transpose: bool = False, tol: float = 1e-10, max_iter: int = 30):
        """FP64-refined solve against the handle's complex128 CSR; returns
        (ok, relative residuals, corrections)."""
        I, J, V, _, _ = g._csr()
        rel = (ct.c_double * nrhs)()
        it = ct.c_int(0)
        ok = self._check(lib().lfsolve_solve_refined(
            self._s, ct.c_void_p(I), ct.c_void_p(J), ct.c_void_p(V), int(nrhs), ct.c_void_p(d_b),
            ct.c_void_p(d_x), int(transpose), float(tol), int(max_iter), rel, ct.byref(it)))
        return ok, list(rel), it.value

    def SolveDeviceCsr(self, g: AsmGpuGlobal, ad, nrhs: int, d_b: int, d_x: int,
                       prec: int = C128) -> bool:
        """The reference's zero-copy entry: factor the handle's device CSR on
        the first call (analysis included), reuse the factors afterwards,
        then back-solve."""
        if os.environ.get("LITHOFEM_CUDSS_FORCE_FAIL"):
            print("cudss: forced failure injected (LITHOFEM_CUDSS_FORCE_FAIL)", flush=True)
            self.last_error = (6, "forced failure injected (LITHOFEM_CUDSS_FORCE_FAIL)")
            return False
        if not self.ready:
            if not (self.AnalyzeAssembly(g, ad) and self.FactorDevice(g._csr()[2], prec)):
                return False
        else:
            print("cudss: factorization reused", flush=True)
        return self.Backsolve(nrhs, d_b, d_x)

    def Stats(self) -> dict:
        st = Stats()
        self._check(lib().lfsolve_get_stats(self._s, ct.byref(st)))
        return {f: getattr(st, f) for f, _ in Stats._fields_}

    def Ordering(self) -> tuple[np.ndarray, np.ndarray]:
        st = self.Stats()
        nn = st["n"] - st["n_ess"]
        perm = np.empty(nn, dtype=np.int32)
        node = np.empty(nn, dtype=np.int32)
        self._check(lib().lfsolve_get_ordering(self._s, _ip(perm), _ip(node)))
        return perm, node

    def Fronts(self) -> dict:
        """The elimination tree: parent, depth, pivots k and rows m per front."""
        nf = self.Stats()["n_fronts"]
        out = {key: np.empty(nf, dtype=np.int32) for key in ("parent", "depth", "k", "m")}
        self._check(lib().lfsolve_get_fronts(self._s, *[_ip(out[key]) for key in
                                                         ("parent", "depth", "k", "m")]))
        return out

    def Release(self) -> None:
        if self._s:
            lib().lfsolve_destroy(self._s)
            self._s = ct.c_void_p()
        self.ready = False

    def __del__(self):
        try:
            self.Release()
        except Exception:
            pass


class DeviceLU:
    """The device solver behind the adjoint's solve / solve_transposed
    interface: factors an assembly handle's device CSR (complex64 by
    default) and returns FP64-refined solutions of A x = b and A^T x = c.
    ``analysis`` is a DirectSolver already analysed for this mesh (the
    ordering depends on the mesh only, so design iterations reuse it)."""

    def __init__(self, g: AsmGpuGlobal, ad=None, prec: int = C64, tol: float = 1e-10,
                 analysis: "DirectSolver | None" = None, max_iter: int = 30):
        self.g, self.tol, self.max_iter = g, tol, max_iter
        self.s = analysis if analysis is not None else DirectSolver(g.gpu_id)
        if analysis is None and not self.s.AnalyzeAssembly(g, ad):
            raise RuntimeError(f"lfsolve_analyze: {self.s.last_error}")
        if not self.s.FactorDevice(g._csr()[2], prec):
            raise RuntimeError(f"lfsolve_factor: {self.s.last_error}")
        self.last = None

    def _run(self, rhs, transpose: bool):
        import torch
        b = rhs if isinstance(rhs, torch.Tensor) else torch.from_numpy(
            np.ascontiguousarray(rhs, dtype=np.complex128))
        b = b.to(device=f"cuda:{self.g.gpu_id}", dtype=torch.complex128).contiguous()
        x = torch.empty_like(b)
        ok, rel, it = self.s.SolveRefined(self.g, 1, b.data_ptr(), x.data_ptr(), transpose,
                                          self.tol, self.max_iter)
        if not ok:
            raise RuntimeError(f"lfsolve_solve_refined: {self.s.last_error}")
        self.last = (rel[0], it)
        return x

    def solve_device(self, b):
        return self._run(b, False)

    def solve_transposed_device(self, c):
        return self._run(c, True)

    def solve(self, b) -> np.ndarray:
        return self._run(b, False).cpu().numpy()

    def solve_transposed(self, c) -> np.ndarray:
        return self._run(c, True).cpu().numpy()
