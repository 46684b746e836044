"""ORACLE -- test infrastructure, not product code.

ctypes wrappers of the two CPU checkers built by oracle/Makefile:

* ``_build/liboracle.so``: this repository's serial restatement of the
  reference assembly path (oracle/lfasm_oracle.cpp);
* ``_ref/libref_asm.so``: the reference's own reassembler and CUDA kernels
  compiled from its sources (oracle/ref_shim/ref_asm.cu), present where the
  reference tree was available at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module.
"""

from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

import numpy as np

from lithofem_b200._abi import (AsmDataC, IncidentPartC, ProblemC, c_double_p, c_int_p,
                                marshal, marshal_parts)
from lithofem_b200.problem import Problem
from lithofem_b200.space import AsmData

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libref_asm.so"

_orc = None
_ref = None


def orc() -> ct.CDLL:
    global _orc
    if _orc is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"{ORACLE_SO} missing: run `make -C oracle`")
        L = ct.CDLL(os.fspath(ORACLE_SO))
        A, P = ct.POINTER(AsmDataC), ct.POINTER(ProblemC)
        L.orc_local.argtypes = [A, P, ct.c_int, ct.c_int, ct.c_int, c_double_p]
        L.orc_local.restype = ct.c_int
        L.orc_csr.argtypes = [A, c_int_p, c_int_p]
        L.orc_csr.restype = ct.c_longlong
        L.orc_assemble.argtypes = [A, P, c_int_p, c_int_p, c_int_p, ct.c_int, ct.c_int, c_double_p]
        L.orc_assemble.restype = ct.c_int
        L.orc_spmv.argtypes = [ct.c_int, c_int_p, c_int_p, c_double_p, c_double_p, c_double_p,
                               c_double_p]
        L.orc_spmv.restype = ct.c_double
        L.orc_rhs.argtypes = [A, P, ct.POINTER(IncidentPartC), ct.c_int, c_int_p, ct.c_int,
                              c_int_p, ct.c_int, ct.c_int, c_double_p]
        L.orc_rhs.restype = ct.c_int
        _orc = L
    return _orc


def ref_available() -> bool:
    return REF_SO.exists()


def ref() -> ct.CDLL:
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise RuntimeError(f"{REF_SO} missing: the reference tree was not available to build it")
        L = ct.CDLL(os.fspath(REF_SO))
        d, i = c_double_p, c_int_p
        L.ref_set_problem.argtypes = [ct.c_double] * 8 + [ct.c_int, ct.c_int, d, i, i, d]
        L.ref_set_problem.restype = ct.c_int
        L.ref_ctx_create.argtypes = ([ct.c_int] * 4 + [i, d, i, i, d, d, d, d] +
                                     [ct.c_int, d, d, d, d] * 2)
        L.ref_ctx_create.restype = ct.c_void_p
        L.ref_ctx_destroy.argtypes = [ct.c_void_p]
        L.ref_ctx_build_csr.argtypes = [ct.c_void_p]
        L.ref_ctx_build_csr.restype = ct.c_longlong
        L.ref_ctx_get_csr.argtypes = [ct.c_void_p, i, i]
        L.ref_ctx_reassemble.argtypes = [ct.c_void_p, d, d]
        L.ref_ctx_time_reassemble.argtypes = [ct.c_void_p]
        L.ref_ctx_time_reassemble.restype = ct.c_double
        L.ref_ctx_element.argtypes = [ct.c_void_p, ct.c_int, d]
        L.ref_ctx_gpu_local.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, d, d]
        L.ref_ctx_gpu_local.restype = ct.c_int
        L.ref_ctx_gpu_global.argtypes = [ct.c_void_p, i, ct.c_int, ct.c_int, ct.c_int, d, d, d]
        L.ref_ctx_gpu_global.restype = ct.c_int
        L.ref_ctx_set_csr.argtypes = [ct.c_void_p, i, ct.c_longlong, i]
        L.ref_set_incident.argtypes = [ct.c_int, ct.c_int] + [d] * 8
        L.ref_incident_at.argtypes = [ct.c_int, ct.c_double, d]
        L.ref_scatter_source_elems.argtypes = [ct.c_int, i, d, d, ct.c_int, d, d]
        _ref = L
    return _ref


# ---------------------------------------------------------------------------
# restatement
# ---------------------------------------------------------------------------

def local(ad: AsmData, prob: Problem, mask_cc: int, mask_mass: int, te: bool) -> np.ndarray:
    m = marshal(ad, prob)
    out = np.empty(2 * ad.ne * ad.nd * ad.nd)
    orc().orc_local(ct.byref(m.ad), ct.byref(m.prob), mask_cc, mask_mass, int(te),
                    out.ctypes.data_as(c_double_p))
    return out.view(np.complex128).reshape(ad.ne, ad.nd, ad.nd)


def csr(ad: AsmData) -> tuple[np.ndarray, np.ndarray]:
    m = marshal(ad, Problem(k0=1, lx=1, ly=1, z_min=0, z_max=1, pml_thick=1))
    I = np.empty(ad.height + 1, dtype=np.int32)
    nnz = orc().orc_csr(ct.byref(m.ad), I.ctypes.data_as(c_int_p), None)
    J = np.empty(nnz, dtype=np.int32)
    orc().orc_csr(ct.byref(m.ad), I.ctypes.data_as(c_int_p), J.ctypes.data_as(c_int_p))
    return I, J


def assemble(ad: AsmData, prob: Problem, I: np.ndarray, J: np.ndarray, ess,
             eliminate: bool) -> np.ndarray:
    m = marshal(ad, prob)
    ess = np.ascontiguousarray(np.asarray(ess, dtype=np.int32))
    vals = np.empty(2 * len(J))
    rc = orc().orc_assemble(ct.byref(m.ad), ct.byref(m.prob), I.ctypes.data_as(c_int_p),
                            J.ctypes.data_as(c_int_p), ess.ctypes.data_as(c_int_p), len(ess),
                            int(eliminate), vals.ctypes.data_as(c_double_p))
    if rc:
        raise RuntimeError("oracle: CSR position missing")
    return vals.view(np.complex128)


def spmv(I, J, vals: np.ndarray, x: np.ndarray, b: np.ndarray | None = None):
    vals = np.ascontiguousarray(vals, dtype=np.complex128)
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.empty_like(x)
    bb = None if b is None else np.ascontiguousarray(b, dtype=np.complex128)
    rel = orc().orc_spmv(len(I) - 1, np.ascontiguousarray(I, dtype=np.int32).ctypes.data_as(c_int_p),
                         np.ascontiguousarray(J, dtype=np.int32).ctypes.data_as(c_int_p),
                         vals.view(np.float64).ctypes.data_as(c_double_p),
                         x.view(np.float64).ctypes.data_as(c_double_p),
                         None if bb is None else bb.view(np.float64).ctypes.data_as(c_double_p),
                         y.view(np.float64).ctypes.data_as(c_double_p))
    return y, rel


def rhs(ad: AsmData, prob: Problem, parts, col_of_part, ncol: int, ess, eliminate: bool):
    m = marshal(ad, prob)
    arr, keep = marshal_parts(parts)
    cols = np.ascontiguousarray(np.asarray(col_of_part, dtype=np.int32))
    ess = np.ascontiguousarray(np.asarray(ess, dtype=np.int32))
    b = np.empty(2 * ad.height * ncol)
    orc().orc_rhs(ct.byref(m.ad), ct.byref(m.prob), arr, len(parts), cols.ctypes.data_as(c_int_p),
                  ncol, ess.ctypes.data_as(c_int_p), len(ess), int(eliminate),
                  b.ctypes.data_as(c_double_p))
    del keep
    return b.view(np.complex128).reshape(ncol, ad.height)


# ---------------------------------------------------------------------------
# reference build
# ---------------------------------------------------------------------------

def _c2(a) -> np.ndarray:
    a = np.asarray(a, dtype=np.complex128)
    return np.ascontiguousarray(np.stack([a.real, a.imag], axis=-1).reshape(-1))


def ref_set_problem(prob: Problem, order: int) -> None:
    """The reference's global problem (Problem/Region) from ours."""
    regs = prob.regions
    eps = _c2([r.eps for r in regs])
    dl = _c2([r.delta_eps for r in regs])
    kind = np.array([r.kind for r in regs], dtype=np.int32)
    slab = np.array([r.slab for r in regs], dtype=np.int32)
    ref().ref_set_problem(prob.k0, prob.kx, prob.ky, prob.z_min, prob.z_max, prob.pml_thick,
                          prob.pml_order, prob.pml_target, order, len(regs),
                          eps.ctypes.data_as(c_double_p), kind.ctypes.data_as(c_int_p),
                          slab.ctypes.data_as(c_int_p), dl.ctypes.data_as(c_double_p))


def ref_set_incident(parts) -> None:
    """The reference's incident tables (prob.incident) from per-slab
    SlabWave lists, one list per part; call after ref_set_problem."""
    n_parts, n_slab = len(parts), len(parts[0])
    zlo = np.array([sw.z_lo for sw in parts[0]], dtype=np.float64)
    zhi = np.array([sw.z_hi for sw in parts[0]], dtype=np.float64)
    flat = [sw for slabs in parts for sw in slabs]
    qA, qB = _c2([sw.qA for sw in flat]), _c2([sw.qB for sw in flat])
    zA = np.array([sw.zA for sw in flat], dtype=np.float64)
    zB = np.array([sw.zB for sw in flat], dtype=np.float64)
    A, B = _c2([sw.A for sw in flat]), _c2([sw.B for sw in flat])
    ref().ref_set_incident(n_parts, n_slab, *[x.ctypes.data_as(c_double_p)
                                              for x in (zlo, zhi, qA, qB, zA, zB, A, B)])


def ref_incident_at(slab: int, z: float) -> np.ndarray:
    out = np.empty(6)
    ref().ref_incident_at(slab, z, out.ctypes.data_as(c_double_p))
    return out.view(np.complex128)


def ref_scatter_source(ad: AsmData, prob: Problem, parts, elements=None,
                       rule=None) -> np.ndarray:
    """The reference's ScatterSource::Eval (problem_common.inc:239-266) at
    every point of ``rule`` (default: the mass rule) of the given elements:
    (len(elements), nq, 3) complex."""
    rule = ad.rule_mass if rule is None else rule
    sel = np.arange(ad.ne) if elements is None else np.asarray(elements)
    ref_set_problem(prob, ad.p)
    ref_set_incident(parts)
    attr = np.ascontiguousarray(ad.attr[sel], dtype=np.int32)
    J = np.ascontiguousarray(ad.J.reshape(ad.ne, 9)[sel].reshape(-1))
    v0 = np.ascontiguousarray(ad.v0.reshape(ad.ne, 3)[sel].reshape(-1))
    ip = np.ascontiguousarray(np.asarray(rule.ip, dtype=np.float64).reshape(-1))
    out = np.empty(len(sel) * rule.nq * 6)
    ref().ref_scatter_source_elems(len(sel), attr.ctypes.data_as(c_int_p),
                                   J.ctypes.data_as(c_double_p), v0.ctypes.data_as(c_double_p),
                                   rule.nq, ip.ctypes.data_as(c_double_p),
                                   out.ctypes.data_as(c_double_p))
    return out.view(np.complex128).reshape(len(sel), rule.nq, 3)


class RefContext:
    """The reference's AsmData + global problem, filled from our extraction."""

    def __init__(self, ad: AsmData, prob: Problem, elements: np.ndarray | None = None):
        L = ref()
        self._keep = []
        k = self._keep.append
        regs = prob.regions
        eps = np.ascontiguousarray(np.array([[r.eps.real, r.eps.imag] for r in regs]).reshape(-1))
        dl = np.ascontiguousarray(np.array([[r.delta_eps.real, r.delta_eps.imag] for r in regs]).reshape(-1))
        kind = np.array([r.kind for r in regs], dtype=np.int32)
        slab = np.array([r.slab for r in regs], dtype=np.int32)
        L.ref_set_problem(prob.k0, prob.kx, prob.ky, prob.z_min, prob.z_max, prob.pml_thick,
                          prob.pml_order, prob.pml_target, ad.p, len(regs),
                          eps.ctypes.data_as(c_double_p), kind.ctypes.data_as(c_int_p),
                          slab.ctypes.data_as(c_int_p), dl.ctypes.data_as(c_double_p))
        nd = ad.nd
        sel = np.arange(ad.ne) if elements is None else np.asarray(elements)
        ne = len(sel)

        def f(a, shape_per):
            a = np.ascontiguousarray(np.asarray(a).reshape(ad.ne, shape_per)[sel].reshape(-1))
            k(a)
            return a

        dof = f(ad.dof.astype(np.int32), nd)
        sign = f(ad.sign, nd)
        fo = f(ad.fo.astype(np.int32), 4) if ad.p >= 2 else np.zeros(4 * ne, dtype=np.int32)
        k(fo)
        attr = f(ad.attr.astype(np.int32), 1)
        J = f(ad.J, 9)
        Ji = f(ad.Jinv, 9)
        det = f(ad.detJ, 1)
        v0 = f(ad.v0, 3)

        def rule(r):
            arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (r.ip, r.w, r.vshape, r.curl)]
            for a in arrs:
                k(a)
            return [r.nq] + [a.ctypes.data_as(c_double_p) for a in arrs]

        self.ne, self.nd, self.height = ne, nd, ad.height
        self.ctx = L.ref_ctx_create(ne, nd, ad.p, ad.height, dof.ctypes.data_as(c_int_p),
                                    sign.ctypes.data_as(c_double_p), fo.ctypes.data_as(c_int_p),
                                    attr.ctypes.data_as(c_int_p), J.ctypes.data_as(c_double_p),
                                    Ji.ctypes.data_as(c_double_p), det.ctypes.data_as(c_double_p),
                                    v0.ctypes.data_as(c_double_p), *rule(ad.rule_cc),
                                    *rule(ad.rule_mass))
        self.nnz = None

    def build_csr(self):
        L = ref()
        self.nnz = int(L.ref_ctx_build_csr(self.ctx))
        I = np.empty(self.height + 1, dtype=np.int32)
        J = np.empty(self.nnz, dtype=np.int32)
        L.ref_ctx_get_csr(self.ctx, I.ctypes.data_as(c_int_p), J.ctypes.data_as(c_int_p))
        return I, J

    def set_csr(self, I: np.ndarray, J: np.ndarray) -> None:
        """Use a given CSR (height + 1 row pointer) instead of building one."""
        I = np.ascontiguousarray(I, dtype=np.int32)
        J = np.ascontiguousarray(J, dtype=np.int32)
        ref().ref_ctx_set_csr(self.ctx, I.ctypes.data_as(c_int_p), len(J),
                              J.ctypes.data_as(c_int_p))
        self.nnz = len(J)

    def reassemble(self) -> np.ndarray:
        if self.nnz is None:
            self.build_csr()
        re = np.empty(self.nnz)
        im = np.empty(self.nnz)
        ref().ref_ctx_reassemble(self.ctx, re.ctypes.data_as(c_double_p), im.ctypes.data_as(c_double_p))
        return re + 1j * im

    def time_reassemble(self) -> float:
        if self.nnz is None:
            self.build_csr()
        return float(ref().ref_ctx_time_reassemble(self.ctx))

    def element(self, e: int) -> np.ndarray:
        out = np.empty(2 * self.nd * self.nd)
        ref().ref_ctx_element(self.ctx, e, out.ctypes.data_as(c_double_p))
        return out.view(np.complex128).reshape(self.nd, self.nd)

    def gpu_local(self, mask_cc: int, mask_mass: int, te: bool):
        out = np.empty(2 * self.ne * self.nd * self.nd)
        ms = ct.c_double()
        rc = ref().ref_ctx_gpu_local(self.ctx, mask_cc, mask_mass, int(te),
                                     out.ctypes.data_as(c_double_p), ct.byref(ms))
        if rc:
            raise RuntimeError(f"reference GPU local failed ({rc})")
        return out.view(np.complex128).reshape(self.ne, self.nd, self.nd), ms.value

    def gpu_global(self, ess, eliminate: bool, iters: int = 1, download: bool = True):
        if self.nnz is None:
            self.build_csr()
        ess = np.ascontiguousarray(np.asarray(ess, dtype=np.int32))
        out = np.empty(2 * self.nnz) if download else None
        ml, msc = ct.c_double(), ct.c_double()
        rc = ref().ref_ctx_gpu_global(self.ctx, ess.ctypes.data_as(c_int_p), len(ess),
                                      int(eliminate), iters,
                                      None if out is None else out.ctypes.data_as(c_double_p),
                                      ct.byref(ml), ct.byref(msc))
        if rc:
            raise RuntimeError(f"reference GPU global failed ({rc})")
        vals = None if out is None else out.view(np.complex128)
        return vals, ml.value, msc.value

    def __del__(self):
        try:
            if getattr(self, "ctx", None):
                ref().ref_ctx_destroy(self.ctx)
                self.ctx = None
        except Exception:
            pass


def _ranges(starts: np.ndarray, lens: np.ndarray) -> np.ndarray:
    """Concatenation of arange(s, s + l) over (starts, lens), int64."""
    lens = np.asarray(lens, dtype=np.int64)
    tot = int(lens.sum())
    if tot == 0:
        return np.zeros(0, dtype=np.int64)
    off = np.concatenate(([0], np.cumsum(lens)[:-1]))
    return np.repeat(np.asarray(starts, dtype=np.int64) - off, lens) + np.arange(tot, dtype=np.int64)


def contiguous_shares(ne: int, n: int) -> list[np.ndarray]:
    """n disjoint contiguous element ranges covering 0..ne-1."""
    cuts = np.linspace(0, ne, n + 1).astype(np.int64)
    return [np.arange(cuts[s], cuts[s + 1]) for s in range(n)]


class RefShares:
    """The reference's reassemble_all (asm_data.inc:374-402) over disjoint
    element shares, one reference context per share.  Each share's context
    holds the full rows of the mesh's CSR (I, J) that its elements touch, so
    every binary search runs over a full-length row as in one serial
    reassembly of the whole mesh; over shares that cover the mesh, the
    shares' values summed entry by entry are the full reassembly.  All
    contexts share the reference's global problem (set identically by each
    context), so the shares can run on concurrent threads (ctypes releases
    the GIL)."""

    def __init__(self, ad: AsmData, prob: Problem, I: np.ndarray, J: np.ndarray,
                 shares: list[np.ndarray]):
        self.I, self.J = np.asarray(I), np.asarray(J)
        self.nnz = len(J)
        self.ctxs, self.rows, self.sizes = [], [], []
        dof = ad.dof.reshape(ad.ne, ad.nd)
        lens_all = np.diff(self.I.astype(np.int64))
        for sel in shares:
            sel = np.asarray(sel)
            rc = RefContext(ad, prob, elements=sel)
            rows = np.unique(dof[sel])
            lens = np.zeros(ad.height, dtype=np.int64)
            lens[rows] = lens_all[rows]
            Is = np.concatenate(([0], np.cumsum(lens))).astype(np.int32)
            Js = self.J[_ranges(self.I[rows], lens_all[rows])]
            rc.set_csr(Is, Js)
            self.ctxs.append(rc)
            self.rows.append(rows)
            self.sizes.append(len(sel))

    def time_parallel(self, threads: int) -> float:
        """Wall seconds of one reassembly of every share, `threads` at a time
        (shares handed out as threads free up)."""
        import concurrent.futures as cf
        import time
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            list(ex.map(lambda rc: rc.time_reassemble(), self.ctxs))
        return time.perf_counter() - t0

    def values(self, threads: int = 1) -> np.ndarray:
        """The sum over the shares of their reassemblies, complex (nnz,)."""
        import concurrent.futures as cf
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            parts = list(ex.map(lambda rc: rc.reassemble(), self.ctxs))
        out = np.zeros(self.nnz, dtype=np.complex128)
        lens_all = np.diff(self.I.astype(np.int64))
        for rows, v in zip(self.rows, parts):
            out[_ranges(self.I[rows], lens_all[rows])] += v   # distinct positions
        return out


DROPIN_SO = HERE / "_ref" / "libref_dropin.so"
_dropin = None


def dropin_available() -> bool:
    return DROPIN_SO.exists()


def dropin() -> ct.CDLL:
    """INTEGRATION.md's C++ call site compiled against the reference's types
    (oracle/ref_shim/dropin.cu), linked to liblfasm.so."""
    global _dropin
    if _dropin is None:
        L = ct.CDLL(os.fspath(DROPIN_SO))
        d, i = c_double_p, c_int_p
        L.dropin_set_problem.argtypes = [ct.c_double] * 8 + [ct.c_int, ct.c_int, d, i, i, d]
        L.dropin_ctx_create.argtypes = ([ct.c_int] * 4 + [i, d, i, i, d, d, d, d] +
                                        [ct.c_int, d, d, d, d] * 2)
        L.dropin_ctx_create.restype = ct.c_void_p
        L.dropin_ctx_destroy.argtypes = [ct.c_void_p]
        L.dropin_assemble.argtypes = [ct.c_void_p, i, ct.c_int, i, ct.POINTER(ct.c_longlong),
                                      i, i, d]
        L.dropin_assemble.restype = ct.c_int
        _dropin = L
    return _dropin


def dropin_assemble(ad: AsmData, prob: Problem):
    """The drop-in call site on (ad, prob): the reference's Problem and
    AsmData filled from ours, then gpu_assemble.  Returns (I, J, values)."""
    L = dropin()
    regs = prob.regions
    eps, dl = _c2([r.eps for r in regs]), _c2([r.delta_eps for r in regs])
    kind = np.array([r.kind for r in regs], dtype=np.int32)
    slab = np.array([r.slab for r in regs], dtype=np.int32)
    L.dropin_set_problem(prob.k0, prob.kx, prob.ky, prob.z_min, prob.z_max, prob.pml_thick,
                         prob.pml_order, prob.pml_target, ad.p, len(regs),
                         eps.ctypes.data_as(c_double_p), kind.ctypes.data_as(c_int_p),
                         slab.ctypes.data_as(c_int_p), dl.ctypes.data_as(c_double_p))
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data_as(c_int_p if dt == np.int32 else c_double_p)

    def rule(r):
        return [r.nq] + [arr(x, np.float64) for x in (r.ip, r.w, r.vshape, r.curl)]

    fo = ad.fo if ad.p >= 2 else np.zeros(4 * ad.ne, dtype=np.int32)
    ctx = L.dropin_ctx_create(ad.ne, ad.nd, ad.p, ad.height, arr(ad.dof, np.int32),
                              arr(ad.sign, np.float64), arr(fo, np.int32),
                              arr(ad.attr, np.int32), arr(ad.J, np.float64),
                              arr(ad.Jinv, np.float64), arr(ad.detJ, np.float64),
                              arr(ad.v0, np.float64), *rule(ad.rule_cc), *rule(ad.rule_mass))
    try:
        ess = np.ascontiguousarray(ad.ess, dtype=np.int32)
        n, nnz = ct.c_int(), ct.c_longlong()
        rc = L.dropin_assemble(ctx, ess.ctypes.data_as(c_int_p), len(ess), ct.byref(n),
                               ct.byref(nnz), None, None, None)
        if rc:
            raise RuntimeError(f"drop-in call site failed at step {rc}")
        I = np.empty(n.value + 1, dtype=np.int32)
        J = np.empty(nnz.value, dtype=np.int32)
        V = np.empty(2 * nnz.value)
        rc = L.dropin_assemble(ctx, ess.ctypes.data_as(c_int_p), len(ess), ct.byref(n),
                               ct.byref(nnz), I.ctypes.data_as(c_int_p), J.ctypes.data_as(c_int_p),
                               V.ctypes.data_as(c_double_p))
        if rc:
            raise RuntimeError(f"drop-in call site failed at step {rc}")
        return I, J, V.view(np.complex128)
    finally:
        L.dropin_ctx_destroy(ctx)
