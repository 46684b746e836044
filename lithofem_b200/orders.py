"""Diffraction orders and order efficiencies from plane samples.

Restates the reference's post-processing: ``orders_from_plane`` (FFT of the
(ny, nx, 3) envelope samples, src/lithofem/orders.py:36-67),
``one_way_flux_z`` (:70-86) and the order efficiency of a one-way region
with the analytic (0,0) background term (src/lithofem/outputs.py:219-269).
The samples come from ``lfasm_sample_plane``; the adjoint seed of one
order's coefficient from ``lfasm_plane_seed``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class OrderSet:
    """Per-order envelope coefficients on a z-plane and their wavevectors."""

    ms: np.ndarray
    ns: np.ndarray
    coeffs: np.ndarray    # (n, 3) complex
    kx: np.ndarray
    ky: np.ndarray
    qz: np.ndarray        # complex, Im >= 0
    k0: float
    eps: complex


def order_qz(k0: float, eps: complex, kx: float, ky: float) -> complex:
    qz = np.sqrt(complex(k0 ** 2 * eps - kx ** 2 - ky ** 2))
    return -qz if qz.imag < 0 else qz


def orders_from_plane(u: np.ndarray, lx: float, ly: float, kpar: tuple[float, float],
                      k0: float, eps_medium: complex) -> OrderSet:
    """FFT the (ny, nx, 3) envelope samples into Fourier orders."""
    ny, nx, _ = u.shape
    c = np.fft.fft2(u, axes=(0, 1)) / (nx * ny)
    gx, gy = 2 * np.pi / lx, 2 * np.pi / ly
    ms, ns, coeffs, kxs, kys, qzs = [], [], [], [], [], []
    for j in range(ny):
        n_idx = j if j <= ny // 2 else j - ny
        for i in range(nx):
            m_idx = i if i <= nx // 2 else i - nx
            kx = kpar[0] + gx * m_idx
            ky = kpar[1] + gy * n_idx
            ms.append(m_idx)
            ns.append(n_idx)
            coeffs.append(c[j, i])
            kxs.append(kx)
            kys.append(ky)
            qzs.append(order_qz(k0, eps_medium, kx, ky))
    return OrderSet(ms=np.array(ms), ns=np.array(ns), coeffs=np.array(coeffs),
                    kx=np.array(kxs), ky=np.array(kys), qz=np.array(qzs), k0=k0,
                    eps=complex(eps_medium))


def plane_wave_flux(c: np.ndarray, kx: float, ky: float, qz: complex, k0: float,
                    direction: int, area: float) -> float:
    """z-power of one plane-wave order: Re[(E x (k x E / k0)*)_z] / 2 x area."""
    k = np.array([kx, ky, direction * qz])
    h = np.cross(k, c) / k0
    return 0.5 * float(np.real(np.cross(c, np.conj(h))[2])) * area


def one_way_flux_z(orders: OrderSet, direction: int, area: float) -> float:
    return sum(plane_wave_flux(orders.coeffs[i], orders.kx[i], orders.ky[i], orders.qz[i],
                               orders.k0, direction, 1.0) for i in range(len(orders.ms))) * area


def zeroth_order_efficiency(c00: np.ndarray, z: float, z_ref: float, kpar, k0: float,
                            eps_medium: complex, eps_in: complex, amp00: complex,
                            e_bg: np.ndarray, lx: float, ly: float, direction: int = 1) -> float:
    """Efficiency of the (0,0) order on the reflection (+1) or transmission
    (-1) side: the scattered coefficient c00 propagated to the reference
    plane z_ref, plus the analytic background amp00 e_bg, as a flux over the
    incident flux (outputs.py:219-269)."""
    qz = order_qz(k0, eps_medium, kpar[0], kpar[1])
    c = c00 * np.exp(-1j * direction * qz * (z - z_ref)) + amp00 * e_bg
    qz_in = np.sqrt(complex(k0 ** 2 * eps_in - kpar[0] ** 2 - kpar[1] ** 2))
    inc_flux = 0.5 * (qz_in.real / k0) * lx * ly
    return direction * plane_wave_flux(c, kpar[0], kpar[1], qz, k0, direction, lx * ly) / inc_flux


def incident_flux(k0: float, eps_in: complex, kx: float, ky: float, area: float) -> float:
    """z-flux of a unit-amplitude incident plane wave through the cell
    (outputs.py:235-238)."""
    qz_in = np.sqrt(complex(k0 ** 2 * eps_in - kx ** 2 - ky ** 2))
    return 0.5 * (qz_in.real / k0) * area


def order_efficiencies(oset: OrderSet, z: float, z_ref: float, direction: int, area: float,
                       inc_flux: float, bg00: np.ndarray | None = None
                       ) -> dict[tuple[int, int], float]:
    """Efficiency (flux / incident flux) of every order of a one-way region
    (outputs.py:219-269).  direction +1: reflection side, up-going orders
    sampled at height z; -1: transmission side, down-going.  Each scattered
    coefficient is carried from z to the reference plane z_ref (the domain's
    top or bottom); bg00 is the analytic (0,0) background at z_ref (the
    reflected wave above, the transmitted wave below) and adds to the (0,0)
    order there."""
    out: dict[tuple[int, int], float] = {}
    for i in range(len(oset.ms)):
        c = oset.coeffs[i] * np.exp(-1j * direction * oset.qz[i] * (z - z_ref))
        if oset.ms[i] == 0 and oset.ns[i] == 0 and bg00 is not None:
            c = c + bg00
        out[(int(oset.ms[i]), int(oset.ns[i]))] = direction * plane_wave_flux(
            c, oset.kx[i], oset.ky[i], oset.qz[i], oset.k0, direction, area) / inc_flux
    return out


def device_orders(g, nx: int, ny: int, e_ptr: int, planes, lx: float, ly: float, k0: float,
                  kpar: tuple[float, float], inc_flux: float):
    """Orders and efficiencies of nz sampled planes on the device
    (lfasm_plane_orders over samples written by lfasm_sample_planes at
    e_ptr).  planes: dicts with z, z_ref, eps, direction (+1 reflection,
    -1 transmission) and optional bg00.  Returns, per plane, the
    (ny * nx, 3) coefficients in orders_from_plane's order and the
    efficiency of every order keyed (m, n) as order_efficiencies."""
    import torch
    nz = len(planes)
    coef = torch.empty(nz * ny * nx * 3, dtype=torch.complex128, device="cuda")
    eff = torch.empty(nz * ny * nx, dtype=torch.float64, device="cuda")
    args = dict(lx=lx, ly=ly, k0=k0, kx=kpar[0], ky=kpar[1], inc_flux=inc_flux)
    if not g.PlaneOrders(nx, ny, e_ptr, planes, args, coef.data_ptr(), eff.data_ptr()):
        raise RuntimeError(f"lfasm_plane_orders failed: {g.last_error}")
    c = coef.cpu().numpy().reshape(nz, ny * nx, 3)
    e = eff.cpu().numpy().reshape(nz, ny * nx)
    ms = np.array([i if i <= nx // 2 else i - nx for _ in range(ny) for i in range(nx)])
    ns = np.array([j if j <= ny // 2 else j - ny for j in range(ny) for _ in range(nx)])
    out = []
    for iz in range(nz):
        out.append((c[iz], {(int(ms[o]), int(ns[o])): float(e[iz, o]) for o in range(ny * nx)}))
    return out
