"""Problem coefficients read by the assembly path.

Mirrors the reference's ``Problem``/``Region`` tables
(solver/problem_common.inc:18-65) as filled by ``parse_problem_core``
(problem_common.inc:271-324), the PML stretch s(z)
(problem_common.inc:69-90) and the per-side stretch maximum the device code
precomputes (solver/asm_gpu.inc:310-319).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .mesh import Stack

KIND_BACKGROUND, KIND_FRUSTUM, KIND_PML_BOTTOM, KIND_PML_TOP = 0, 1, 2, 3
_KIND = {"background": KIND_BACKGROUND, "frustum": KIND_FRUSTUM,
         "pml_bottom": KIND_PML_BOTTOM, "pml_top": KIND_PML_TOP}


@dataclass
class Region:
    slab: int
    eps: complex
    kind: int
    delta_eps: complex = 0j     # eps - eps_bg(slab), frustum regions only
    z0: float = 0.0
    z1: float = 0.0

    @property
    def is_pml(self) -> bool:
        return self.kind in (KIND_PML_BOTTOM, KIND_PML_TOP)

    @property
    def pml_top(self) -> bool:
        return self.kind == KIND_PML_TOP

    @property
    def is_frustum(self) -> bool:
        return self.kind == KIND_FRUSTUM


@dataclass
class Problem:
    k0: float
    lx: float
    ly: float
    z_min: float
    z_max: float
    kx: float = 0.0
    ky: float = 0.0
    order: int = 1
    pml_order: float = 2.0
    pml_target: float = 1e-8
    pml_thick: float = 0.0
    regions: list[Region] = field(default_factory=list)
    # optional per-element permittivity (design variables); None = per region
    elem_eps: np.ndarray | None = None

    @property
    def has_kpar(self) -> bool:
        return self.kx != 0.0 or self.ky != 0.0

    def n_med(self) -> tuple[float, float]:
        """|sqrt(eps)| of the bottom / top PML regions (1 if absent)."""
        n_bot = n_top = 1.0
        for r in self.regions:
            if r.is_pml and not r.pml_top:
                n_bot = abs(np.sqrt(complex(r.eps)))
            if r.is_pml and r.pml_top:
                n_top = abs(np.sqrt(complex(r.eps)))
        return n_bot, n_top

    def smax(self) -> tuple[float, float]:
        """-ln(R)(m+1) / (2 k0 n_med t) per side (asm_gpu.inc:310-319)."""
        n_bot, n_top = self.n_med()
        f = -math.log(self.pml_target) * (self.pml_order + 1)
        return (f / (2.0 * self.k0 * n_bot * self.pml_thick),
                f / (2.0 * self.k0 * n_top * self.pml_thick))

    def s_z(self, z: np.ndarray) -> np.ndarray:
        """PML stretch s(z) = 1 + i smax d^m (problem_common.inc:69-90)."""
        z = np.asarray(z, dtype=float)
        sb, st = self.smax()
        d = np.full(z.shape, -1.0)
        sm = np.zeros(z.shape)
        lo = z < self.z_min
        hi = z > self.z_max
        d[lo] = (self.z_min - z[lo]) / self.pml_thick
        sm[lo] = sb
        d[hi] = (z[hi] - self.z_max) / self.pml_thick
        sm[hi] = st
        out = np.ones(z.shape, dtype=complex)
        m = d >= 0.0
        dd = np.minimum(d[m], 1.0)
        out[m] = 1.0 + 1j * sm[m] * dd ** self.pml_order
        return out

    def eps_table(self) -> np.ndarray:
        return np.array([complex(r.eps) for r in self.regions], dtype=complex)

    @classmethod
    def from_stack(cls, stack: Stack, order: int, kpar: tuple[float, float] = (0.0, 0.0)
                   ) -> "Problem":
        regs = stack.regions()
        n_slab = len(stack.slabs) - 1
        bg = [stack.eps_bg_of_slab(i) for i in range(n_slab)]
        out: list[Region] = []
        for r in regs:
            kind = _KIND[r["kind"]]
            if kind in (KIND_PML_BOTTOM, KIND_PML_TOP):
                slab = n_slab - 1 if kind == KIND_PML_TOP else 0
                out.append(Region(slab=slab, eps=complex(r["eps"]), kind=kind,
                                  z0=r["z"][0], z1=r["z"][1]))
            else:
                d = complex(r["eps"]) - bg[r["slab"]] if kind == KIND_FRUSTUM else 0j
                out.append(Region(slab=r["slab"], eps=complex(r["eps"]), kind=kind,
                                  delta_eps=d, z0=r["z"][0], z1=r["z"][1]))
        return cls(k0=stack.k0, lx=stack.lx, ly=stack.ly, z_min=stack.z_min,
                   z_max=stack.z_max, kx=float(kpar[0]), ky=float(kpar[1]), order=order,
                   pml_order=float(stack.pml_order), pml_target=stack.pml_target,
                   pml_thick=stack.pml_thick, regions=out)
