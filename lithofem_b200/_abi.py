"""ctypes mirror of include/lfasm.h and marshalling of host arrays."""

from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field

import numpy as np

from .problem import Problem
from .space import AsmData

c_int_p = ct.POINTER(ct.c_int)
c_double_p = ct.POINTER(ct.c_double)

CURLCURL, MASS, CROSS0, CROSS1, KLK = 1, 2, 4, 8, 16
BULK_VARIANTS = 6   # LFASM_BULK_VARIANTS: bulk-element kernel variants of the autotuner
ERR_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_UNSUPPORTED", 4: "ERR_STATE",
             5: "ERR_CSR"}


class RefRule(ct.Structure):
    _fields_ = [("nq", ct.c_int), ("ip", c_double_p), ("w", c_double_p),
                ("vshape", c_double_p), ("curl", c_double_p)]


class AsmDataC(ct.Structure):
    _fields_ = [("ne", ct.c_int), ("nd", ct.c_int), ("p", ct.c_int), ("height", ct.c_int),
                ("has_kpar", ct.c_int),
                ("dof", c_int_p), ("sign", c_double_p), ("fo", c_int_p), ("attr", c_int_p),
                ("J", c_double_p), ("Jinv", c_double_p), ("detJ", c_double_p),
                ("v0", c_double_p), ("rule_cc", RefRule), ("rule_mass", RefRule),
                ("I", c_int_p), ("Jcol", c_int_p), ("nnz", ct.c_longlong)]


class ProblemC(ct.Structure):
    _fields_ = [("k0", ct.c_double), ("kx", ct.c_double), ("ky", ct.c_double),
                ("z_min", ct.c_double), ("z_max", ct.c_double), ("pml_thick", ct.c_double),
                ("pml_order", ct.c_double), ("pml_target", ct.c_double),
                ("n_regions", ct.c_int), ("region_eps", c_double_p),
                ("region_kind", c_int_p), ("region_slab", c_int_p),
                ("region_delta_eps", c_double_p), ("elem_eps", c_double_p)]


class IncidentPartC(ct.Structure):
    _fields_ = [("n_slab", ct.c_int), ("qA", c_double_p), ("qB", c_double_p),
                ("zA", c_double_p), ("zB", c_double_p), ("A", c_double_p), ("B", c_double_p)]


def _dp(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(c_double_p)


def _ip(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(c_int_p)


def _c2(z) -> np.ndarray:
    z = np.asarray(z, dtype=np.complex128)
    return np.ascontiguousarray(np.stack([z.real, z.imag], axis=-1).reshape(-1))


class OrderPlaneC(ct.Structure):
    """lfasm_order_plane: one sampled plane of lfasm_plane_orders."""
    _fields_ = [("z", ct.c_double), ("z_ref", ct.c_double), ("eps_re", ct.c_double),
                ("eps_im", ct.c_double), ("direction", ct.c_int), ("has_bg00", ct.c_int),
                ("bg00", ct.c_double * 6)]


class OrderArgsC(ct.Structure):
    """lfasm_order_args: cell, wavenumber, Bloch wavevector, incident flux."""
    _fields_ = [("lx", ct.c_double), ("ly", ct.c_double), ("k0", ct.c_double),
                ("kx", ct.c_double), ("ky", ct.c_double), ("inc_flux", ct.c_double)]


@dataclass
class Marshalled:
    """C structs plus the numpy buffers that keep their pointers alive."""

    ad: AsmDataC
    prob: ProblemC
    keep: list = field(default_factory=list)


def marshal(ad: AsmData, prob: Problem, with_csr: bool = False) -> Marshalled:
    keep: list = []

    def k(a):
        keep.append(a)
        return a

    def rule(r):
        return RefRule(r.nq, _dp(k(np.ascontiguousarray(r.ip, dtype=np.float64))),
                       _dp(k(np.ascontiguousarray(r.w, dtype=np.float64))),
                       _dp(k(np.ascontiguousarray(r.vshape, dtype=np.float64))),
                       _dp(k(np.ascontiguousarray(r.curl, dtype=np.float64))))

    c = AsmDataC()
    c.ne, c.nd, c.p, c.height = ad.ne, ad.nd, ad.p, ad.height
    c.has_kpar = int(prob.has_kpar)
    c.dof = _ip(k(np.ascontiguousarray(ad.dof, dtype=np.int32)))
    c.sign = _dp(k(np.ascontiguousarray(ad.sign, dtype=np.float64)))
    c.fo = _ip(k(np.ascontiguousarray(ad.fo, dtype=np.int32))) if ad.p >= 2 else None
    c.attr = _ip(k(np.ascontiguousarray(ad.attr, dtype=np.int32)))
    for name in ("J", "Jinv", "detJ", "v0"):
        setattr(c, name, _dp(k(np.ascontiguousarray(getattr(ad, name), dtype=np.float64))))
    c.rule_cc = rule(ad.rule_cc)
    c.rule_mass = rule(ad.rule_mass)
    if with_csr and ad.I is not None:
        c.I = _ip(k(np.ascontiguousarray(ad.I, dtype=np.int32)))
        c.Jcol = _ip(k(np.ascontiguousarray(ad.Jcol, dtype=np.int32)))
        c.nnz = int(ad.Jcol.shape[0])
    else:
        c.I = None
        c.Jcol = None
        c.nnz = 0
    p = ProblemC()
    p.k0, p.kx, p.ky = prob.k0, prob.kx, prob.ky
    p.z_min, p.z_max = prob.z_min, prob.z_max
    p.pml_thick, p.pml_order, p.pml_target = prob.pml_thick, prob.pml_order, prob.pml_target
    p.n_regions = len(prob.regions)
    p.region_eps = _dp(k(_c2([r.eps for r in prob.regions])))
    p.region_kind = _ip(k(np.array([r.kind for r in prob.regions], dtype=np.int32)))
    p.region_slab = _ip(k(np.array([r.slab for r in prob.regions], dtype=np.int32)))
    p.region_delta_eps = _dp(k(_c2([r.delta_eps for r in prob.regions])))
    p.elem_eps = _dp(k(_c2(prob.elem_eps))) if prob.elem_eps is not None else None
    return Marshalled(ad=c, prob=p, keep=keep)


def marshal_parts(parts) -> tuple[ct.Array, list]:
    """parts: list of per-slab wave tables (see ``incident.SlabWave``)."""
    keep: list = []
    arr = (IncidentPartC * max(1, len(parts)))()
    for i, slabs in enumerate(parts):
        qA = _c2([s.qA for s in slabs])
        qB = _c2([s.qB for s in slabs])
        zA = np.array([s.zA for s in slabs], dtype=np.float64)
        zB = np.array([s.zB for s in slabs], dtype=np.float64)
        A = _c2(np.array([s.A for s in slabs]))
        B = _c2(np.array([s.B for s in slabs]))
        keep += [qA, qB, zA, zB, A, B]
        arr[i] = IncidentPartC(len(slabs), _dp(qA), _dp(qB), _dp(zA), _dp(zB), _dp(A), _dp(B))
    return arr, keep
