"""Planar multilayer background field (analytic incident field of the RHS).

The scattered-field right-hand side needs the field of the unpatterned
stack: a plane wave of unit amplitude entering from one half-space, passing
a sequence of homogeneous layers and leaving through the other half-space.
The reference computes it with its TMM module (src/lithofem/tmm.py: branch
rule :38-46, the result record :69-161, the solver :169-270); this module
produces the same record from a different scheme.

Scheme (Airy / Rouard recursion).  Work on a depth coordinate ``zeta`` that
grows along the propagation direction; the incidence half-space is zeta <= 0
and interface i sits at depth D_i (D_0 = 0, D_i = d_1 + ... + d_i).  The
scalar unknown is u = Ey for s and u = Z0 Hy for p; u and g du/dzeta are
continuous (g = 1 for s, 1/eps for p), so every interface is characterised
by the admittances Y_j = g_j q_j of its two sides.  Inside layer j

    u_j = f_j e^{+i q_j (zeta - D_{j-1})} + g_j e^{-i q_j (zeta - D_j)},

every exponential evaluated towards the layer's own interfaces, so no factor
ever exceeds 1 in modulus.  The stack is solved in two sweeps:

1. from the exit side upwards, the ratio G_j = (backward / forward wave) at
   the bottom face of layer j follows from the Fresnel coefficient of the
   interface below it and the ratio seen through the next layer,
   G_j = (r_j + G_{j+1} P_{j+1}^2) / (1 + r_j G_{j+1} P_{j+1}^2), with
   P = e^{i q d} the one-way phase of a layer and G = r at the last
   interface (nothing comes back from the exit half-space);
2. from the incidence side downwards, the forward amplitude is carried
   across each interface by whichever of the two continuity conditions
   (u, or g du/dzeta) is better conditioned there: |1 + rho| and |1 - rho|
   cannot both be small.

Conventions: time factor e^{-i omega t}; Im q >= 0 (Re q >= 0 when q is
real).  Amplitudes: a[j] = forward amplitude referenced at the layer's entry
face, b[j] = backward amplitude referenced at its exit face; a[0] = 1,
b[0] = r, a[-1] = t, b[-1] = 0; the two half-spaces are referenced at
zeta = 0 and zeta = D_m.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def kz_branch(eps: complex, k0: float, kpar: float) -> complex:
    """Normal wavenumber q = sqrt(k0^2 eps - kpar^2) on the decaying branch:
    Im q >= 0, and Re q >= 0 for a real q."""
    q = complex(np.sqrt(complex(k0 * k0 * complex(eps) - kpar * kpar)))
    flip = q.imag < 0.0 or (q.imag == 0.0 and q.real < 0.0)
    return -q if flip else q


@dataclass(frozen=True)
class Stack:
    """Half-space of incidence, finite layers in the order the wave meets
    them (permittivity ``eps[i]``, thickness ``d[i]`` in nm) and the exit
    half-space."""

    eps_in: complex
    eps_out: complex
    eps: tuple = ()
    d: tuple = ()

    def __post_init__(self):
        if len(self.eps) != len(self.d):
            raise ValueError(f"Stack: {len(self.eps)} permittivities given for "
                             f"{len(self.d)} thicknesses")
        bad = [t for t in self.d if not t > 0]
        if bad:
            raise ValueError(f"Stack: every layer needs a thickness > 0 (got {bad[0]!r})")


@dataclass(frozen=True)
class TMMResult:
    """Field of one polarisation in every region of the stack (index 0: the
    incidence half-space, 1..m: the layers, m + 1: the exit half-space)."""

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
    _edges: np.ndarray = field(repr=False, default=None)

    @property
    def k0(self) -> float:
        return 2.0 * math.pi / self.wavelength

    def layer_of(self, zeta) -> np.ndarray:
        """Region index of each depth (a depth on an interface belongs to the
        region below it)."""
        return np.searchsorted(self._edges, np.asarray(zeta, dtype=float), side="right")

    def _waves(self, zeta):
        zeta = np.asarray(zeta, dtype=float)
        j = self.layer_of(zeta)
        q = self.q[j]
        fwd = self.a[j] * np.exp(1j * q * (zeta - self.z_lo[j]))
        bwd = self.b[j] * np.exp(-1j * q * (zeta - self.z_hi[j]))
        return q, fwd, bwd

    def u(self, zeta) -> np.ndarray:
        _, fwd, bwd = self._waves(zeta)
        return fwd + bwd

    def du(self, zeta) -> np.ndarray:
        q, fwd, bwd = self._waves(zeta)
        return 1j * q * (fwd - bwd)


def _kpar_from_angle(stack: Stack, k0: float, theta_deg: float) -> float:
    e_in = complex(stack.eps_in)
    if e_in.imag != 0.0:
        raise ValueError("an incidence angle needs a lossless incidence half-space; "
                         "give kpar instead")
    return k0 * math.sqrt(e_in.real) * math.sin(math.radians(theta_deg))


def solve(stack: Stack, wavelength: float, *, theta_deg: float = 0.0, pol: str = "s",
          kpar: float | None = None) -> TMMResult:
    """Field of a unit plane wave of polarisation ``pol`` ('s' or 'p')
    through ``stack`` at vacuum wavelength ``wavelength`` (nm), with in-plane
    wavenumber ``kpar`` (rad/nm) or, from a lossless incidence half-space,
    the incidence angle ``theta_deg``."""
    if pol not in ("s", "p"):
        raise ValueError(f"polarisation must be 's' or 'p' (got {pol!r})")
    k0 = 2.0 * math.pi / wavelength
    if kpar is None:
        kpar = _kpar_from_angle(stack, k0, theta_deg)
    eps = np.array([stack.eps_in, *stack.eps, stack.eps_out], dtype=complex)
    nreg = eps.size                        # m layers + 2 half-spaces
    m = nreg - 2
    q = np.array([kz_branch(e, k0, kpar) for e in eps], dtype=complex)
    Y = q if pol == "s" else q / eps       # admittance of each region
    thick = np.asarray(stack.d, dtype=float)
    P = np.ones(nreg, dtype=complex)       # one-way phase across each region
    P[1:-1] = np.exp(1j * q[1:-1] * thick)

    # Fresnel reflection of interface i (region i above, region i + 1 below)
    r_if = (Y[:-1] - Y[1:]) / (Y[:-1] + Y[1:])
    # sweep 1 (upwards): G[i] = backward/forward ratio at the bottom face of
    # region i; rho[i] = the same ratio at the top face of region i + 1
    G = np.zeros(nreg, dtype=complex)
    rho = np.zeros(nreg - 1, dtype=complex)
    for i in range(m, -1, -1):
        below = G[i + 1] * P[i + 1] * P[i + 1] if i + 1 <= m else 0.0
        rho[i] = below
        G[i] = (r_if[i] + below) / (1.0 + r_if[i] * below)

    # sweep 2 (downwards): forward amplitude at each region's top face
    fwd_top = np.zeros(nreg, dtype=complex)
    fwd_top[0] = 1.0
    for i in range(m + 1):
        arrive = fwd_top[i] * P[i]         # forward wave at interface i, above it
        via_u = 1.0 + rho[i]
        via_flux = 1.0 - rho[i]
        if abs(via_u) >= abs(via_flux):
            fwd_top[i + 1] = arrive * (1.0 + G[i]) / via_u
        else:
            fwd_top[i + 1] = arrive * (Y[i] / Y[i + 1]) * (1.0 - G[i]) / via_flux

    a = fwd_top.copy()
    b = G * fwd_top * P                    # backward amplitude at each exit face
    b[-1] = 0.0
    depth = np.concatenate(([0.0], np.cumsum(thick)))      # D_0 .. D_m
    z_lo = np.concatenate(([0.0], depth))                  # entry face per region
    z_hi = np.concatenate(([0.0], depth[1:], depth[-1:]))  # exit face per region
    edges = depth.copy()                                   # region boundaries
    return TMMResult(wavelength=wavelength, kpar=float(kpar), pol=pol, r=complex(b[0]),
                     t=complex(a[-1]), a=a, b=b, q=q, z_lo=z_lo, z_hi=z_hi, eps_all=eps,
                     _edges=edges)
