"""Incident (background) field tables for the scattered-field right-hand side.

Restates the plane-wave construction of the reference
(src/lithofem/incident.py: _sp_basis :82-97, _planewave_field :121-205,
group_incident :208-240): the TMM solution of the unpatterned stack is
mapped to global coordinates as, per slab,

    Ehat(z) = A e^{i qA (z - zA)} + B e^{i qB (z - zB)},

one table per polarisation part, which is exactly what the device RHS
kernel evaluates (incident_at, solver/problem_common.inc:218-236).
Conventions (src/lithofem/constants.py): e^{-i omega t}; ``from_top`` means
the source sits above z_max and propagates toward -z; e_s = z x k / |z x k|
(e_s = y at normal incidence), e_p = k x e_s.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import tmm
from .mesh import Stack as MeshStack


@dataclass(frozen=True)
class SlabWave:
    z_lo: float
    z_hi: float
    qA: complex
    zA: float
    A: np.ndarray
    qB: complex
    zB: float
    B: np.ndarray

    def eval(self, z) -> np.ndarray:
        z = np.atleast_1d(np.asarray(z, dtype=float))
        return (np.exp(1j * self.qA * (z - self.zA))[:, None] * self.A[None, :]
                + np.exp(1j * self.qB * (z - self.zB))[:, None] * self.B[None, :])


def sp_basis(theta: float, phi: float, from_top: bool):
    th, ph = math.radians(theta), math.radians(phi)
    sz = -1.0 if from_top else 1.0
    k_hat = np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), sz * math.cos(th)])
    if theta == 0.0:
        e_s = np.array([0.0, 1.0, 0.0])
    else:
        e_s = np.cross([0.0, 0.0, 1.0], k_hat)
        e_s = e_s / np.linalg.norm(e_s)
    return e_s, np.cross(k_hat, e_s), k_hat


def kpar_of(stack: MeshStack, theta: float, phi: float = 0.0, from_top: bool = True):
    """In-plane wavevector k0 sin(theta) (cos phi, sin phi) of a plane-wave
    source: the reference defines a source's angle in vacuum whatever the
    incidence ambient (src/lithofem/config.py:472-473), so ``from_top`` does
    not enter."""
    del from_top
    kp = stack.k0 * math.sin(math.radians(theta))
    return (kp * math.cos(math.radians(phi)), kp * math.sin(math.radians(phi)))


def planewave_parts(stack: MeshStack, theta: float, phi: float = 0.0, pol: str = "s",
                    amp: complex = 1.0, from_top: bool = True) -> list[SlabWave]:
    """Per-slab global-frame tables for one plane wave of pure s or p pol."""
    slabs = stack.slabs
    n_slab = len(slabs) - 1
    k0 = stack.k0
    eps_s = [stack.eps_bg_of_slab(i) for i in range(n_slab)]
    d = [slabs[i + 1] - slabs[i] for i in range(n_slab)]
    if from_top:
        st = tmm.Stack(eps_in=eps_s[-1], eps_out=eps_s[0], eps=tuple(reversed(eps_s)),
                       d=tuple(reversed(d)))
        z_ref = slabs[-1]
    else:
        st = tmm.Stack(eps_in=eps_s[0], eps_out=eps_s[-1], eps=tuple(eps_s), d=tuple(d))
        z_ref = slabs[0]
    kx, ky = kpar_of(stack, theta, phi, from_top)
    kpar = math.hypot(kx, ky)
    res = tmm.solve(st, stack.wavelength, kpar=kpar, pol=pol)
    e_s, _, _ = sp_basis(theta, phi, from_top)
    ph = math.radians(phi)
    x_loc = np.array([math.cos(ph), math.sin(ph), 0.0])
    zeta_hat = np.array([0.0, 0.0, -1.0 if from_top else 1.0])
    y_loc = np.cross(zeta_hat, x_loc)
    align = float(np.dot(y_loc, e_s))
    s_sign = 1.0 if align > 0 else -1.0
    n_in = complex(np.sqrt(complex(st.eps_in)))
    amp_f = amp * s_sign if pol == "s" else amp * n_in
    R = np.stack([x_loc, y_loc, zeta_hat], axis=1)
    out = []
    for i in range(n_slab):
        j = (n_slab - i) if from_top else (i + 1)
        q, a, b = res.q[j], res.a[j], res.b[j]
        zl, zh = res.z_lo[j], res.z_hi[j]
        ej = res.eps_all[j]
        if pol == "s":
            va = np.array([0, 1, 0], dtype=complex) * a
            vb = np.array([0, 1, 0], dtype=complex) * b
        else:
            va = np.array([q / (k0 * ej), 0, -kpar / (k0 * ej)]) * a
            vb = np.array([-q / (k0 * ej), 0, -kpar / (k0 * ej)]) * b
        A = amp_f * (R @ va)
        B = amp_f * (R @ vb)
        if from_top:
            out.append(SlabWave(slabs[i], slabs[i + 1], -q, z_ref - zl, A, q, z_ref - zh, B))
        else:
            out.append(SlabWave(slabs[i], slabs[i + 1], q, z_ref + zl, A, -q, z_ref + zh, B))
    return out


def eval_parts(parts: list[list[SlabWave]], z) -> np.ndarray:
    """Ehat(z) summed over parts (no transverse phase factor), (n, 3)."""
    z = np.atleast_1d(np.asarray(z, dtype=float))
    out = np.zeros((len(z), 3), dtype=complex)
    for slabs in parts:
        edges = np.array([sw.z_lo for sw in slabs[1:]])
        idx = np.searchsorted(edges, z, side="right")
        for i, sw in enumerate(slabs):
            m = idx == i
            if m.any():
                out[m] += sw.eval(z[m])
    return out
