"""1D multilayer transfer-matrix background (analytic incident field).

Restates the algorithm of the reference's TMM module (src/lithofem/tmm.py:
kz_branch :38-46, Stack :49-66, TMMResult :69-161, solve :169-270), which
supplies the background field whose contrast drives the scattered-field
right-hand side.  Conventions: e^{-i omega t}; Im(q) >= 0 branch; the solver
works in a coordinate zeta increasing along propagation, incidence
half-space at zeta <= 0, interfaces at the cumulative layer depths.

Per layer j the scalar field (s: Ey; p: Z0 Hy) is
    u_j(zeta) = a_j e^{+i q_j (zeta - z_lo[j])} + b_j e^{-i q_j (zeta - z_hi[j])}
("directional phase referencing": no growing exponentials), and continuity
of u and gamma du/dzeta (gamma = 1 for s, 1/eps for p) at every interface is
solved as one small linear system in (b_0, a_1, b_1, ..., a_{m+1}).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def kz_branch(eps: complex, k0: float, kpar: float) -> complex:
    """q = sqrt(k0^2 eps - kpar^2) with Im q >= 0 (Re q >= 0 when Im q == 0)."""
    q = np.sqrt(complex(eps) * k0 * k0 - kpar * kpar + 0j)
    if q.imag < 0.0 or (q.imag == 0.0 and q.real < 0.0):
        q = -q
    return complex(q)


@dataclass(frozen=True)
class Stack:
    """Layers in propagation order between two half-spaces."""

    eps_in: complex
    eps_out: complex
    eps: tuple = ()
    d: tuple = ()

    def __post_init__(self):
        if len(self.eps) != len(self.d):
            raise ValueError("eps and d must have equal length")
        if any(t <= 0 for t in self.d):
            raise ValueError("layer thicknesses must be positive")


@dataclass(frozen=True)
class TMMResult:
    wavelength: float
    kpar: float
    pol: str
    r: complex
    t: complex
    a: np.ndarray
    b: np.ndarray
    q: np.ndarray
    z_lo: np.ndarray
    z_hi: np.ndarray
    eps_all: np.ndarray

    @property
    def k0(self) -> float:
        return 2.0 * math.pi / self.wavelength

    def layer_of(self, zeta: np.ndarray) -> np.ndarray:
        edges = np.concatenate((self.z_lo[1:-1], self.z_hi[-1:]))
        return np.searchsorted(edges, zeta, side="right")

    def u(self, zeta) -> np.ndarray:
        zeta = np.asarray(zeta, dtype=float)
        j = self.layer_of(zeta)
        return (self.a[j] * np.exp(1j * self.q[j] * (zeta - self.z_lo[j]))
                + self.b[j] * np.exp(-1j * self.q[j] * (zeta - self.z_hi[j])))

    def du(self, zeta) -> np.ndarray:
        zeta = np.asarray(zeta, dtype=float)
        j = self.layer_of(zeta)
        up = self.a[j] * np.exp(1j * self.q[j] * (zeta - self.z_lo[j]))
        dn = self.b[j] * np.exp(-1j * self.q[j] * (zeta - self.z_hi[j]))
        return 1j * self.q[j] * (up - dn)


def solve(stack: Stack, wavelength: float, *, theta_deg: float = 0.0, pol: str = "s",
          kpar: float | None = None) -> TMMResult:
    if pol not in ("s", "p"):
        raise ValueError(f"pol must be 's' or 'p', got {pol!r}")
    k0 = 2.0 * math.pi / wavelength
    if kpar is None:
        if abs(complex(stack.eps_in).imag) > 0:
            raise ValueError("theta_deg needs a lossless incidence medium; pass kpar instead")
        kpar = k0 * math.sqrt(complex(stack.eps_in).real) * math.sin(math.radians(theta_deg))
    eps_all = np.array([complex(stack.eps_in), *[complex(e) for e in stack.eps],
                        complex(stack.eps_out)])
    m = len(stack.eps)
    q = np.array([kz_branch(e, k0, kpar) for e in eps_all])
    gam = np.ones(m + 2, dtype=complex) if pol == "s" else 1.0 / eps_all
    depth = np.concatenate(([0.0], np.cumsum(stack.d)))
    z_lo = np.concatenate(([0.0], depth[:-1], depth[-1:]))
    z_hi = np.concatenate(([0.0], depth[1:], depth[-1:]))
    ph = np.exp(1j * q[1:-1] * np.asarray(stack.d, dtype=float))   # |ph| <= 1

    # unknown vector: [b_0, a_1, b_1, ..., a_m, b_m, a_{m+1}]
    n = 2 * m + 2
    ia = lambda j: 2 * j - 1          # noqa: E731  a_j, j = 1..m+1
    ib = lambda j: 0 if j == 0 else 2 * j  # noqa: E731  b_j, j = 0..m
    M = np.zeros((n, n), dtype=complex)
    rhs = np.zeros(n, dtype=complex)
    for i in range(m + 1):
        L, R = i, i + 1
        # u and gamma*du at the interface: left layer at its exit side,
        # right layer at its entrance side
        la, lb = (1.0, 1.0) if L == 0 else (ph[L - 1], 1.0)
        ra, rb = (1.0, 0.0) if R == m + 1 else (1.0, ph[R - 1])
        cl, cr = 1j * q[L] * gam[L], 1j * q[R] * gam[R]
        row_u, row_d = 2 * i, 2 * i + 1
        if L == 0:
            rhs[row_u] -= la
            rhs[row_d] -= cl * la
        else:
            M[row_u, ia(L)] += la
            M[row_d, ia(L)] += cl * la
        M[row_u, ib(L)] += lb
        M[row_d, ib(L)] -= cl * lb
        M[row_u, ia(R)] -= ra
        M[row_d, ia(R)] -= cr * ra
        if R <= m:
            M[row_u, ib(R)] -= rb
            M[row_d, ib(R)] += cr * rb
    x = np.linalg.solve(M, rhs)
    a = np.empty(m + 2, dtype=complex)
    b = np.empty(m + 2, dtype=complex)
    a[0], b[0] = 1.0, x[0]
    for j in range(1, m + 1):
        a[j], b[j] = x[ia(j)], x[ib(j)]
    a[m + 1], b[m + 1] = x[-1], 0.0
    return TMMResult(wavelength=wavelength, kpar=float(kpar), pol=pol, r=complex(b[0]),
                     t=complex(a[m + 1]), a=a, b=b, q=q, z_lo=z_lo, z_hi=z_hi,
                     eps_all=eps_all)
