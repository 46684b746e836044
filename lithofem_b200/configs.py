"""Synthetic workloads: the five benchmark workloads and small test cases.

Geometries follow the benchmark descriptions (EUV, lambda = 13.5 nm,
absorber n = 0.95 k = 0.031, eps = (n + i k)^2, z-PML of one wavelength,
order 2, R = 1e-8; conventions of src/lithofem/constants.py:30-40).  Mesh
densities are chosen to hit the stated DOF targets (the stated
elements-per-wavelength values would give far more DOFs than stated), and
the actual element, DOF and nonzero counts are reported by the callers.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from .mesh import Frustum, Stack, TetMesh, build_mesh, h_for_target_dofs
from .mesh_poly import PolyHole, build_poly_mesh, random_hole
from .problem import Problem
from .space import AsmData, build_asm_data

WAVELENGTH = 13.5
ABSORBER = complex(0.95, 0.031) ** 2
UNDERLAYER = complex(0.97, 0.01) ** 2
SEED = 20260806


def kpar_of(theta_deg: float, phi_deg: float = 0.0, n_in: float = 1.0) -> tuple[float, float]:
    k0 = 2.0 * math.pi / WAVELENGTH
    kp = k0 * n_in * math.sin(math.radians(theta_deg))
    return (kp * math.cos(math.radians(phi_deg)), kp * math.sin(math.radians(phi_deg)))


def slab_stack() -> Stack:
    """96 x 96 nm cell, z in [0, 120], absorber slab z in [0, 60] under vacuum."""
    return Stack(lx=96.0, ly=96.0, z_min=0.0, z_max=120.0, wavelength=WAVELENGTH,
                 layers=[(0.0, 60.0, ABSORBER)])


def contact_hole_stack() -> Stack:
    """Slab stack with a centred 48 x 48 nm vacuum frustum, h = 60, 85 deg walls."""
    st = slab_stack()
    st.frustums = [Frustum(24.0, 72.0, 24.0, 72.0, 0.0, 60.0, 85.0, 1.0 + 0j)]
    return st


def line_grating_stack() -> Stack:
    """Lines (pitch 64, CD 32) of a 60 nm absorber over a 40 nm underlayer."""
    return Stack(lx=64.0, ly=16.0, z_min=-40.0, z_max=90.0, wavelength=WAVELENGTH,
                 layers=[(-40.0, 0.0, UNDERLAYER)],
                 frustums=[Frustum(16.0, 48.0, 0.0, 16.0, 0.0, 60.0, 90.0, ABSORBER)])


@dataclass
class Case:
    name: str
    stack: Stack
    p: int
    theta: float
    ad: AsmData
    prob: Problem
    mesh: TetMesh | None = None
    h: float = 0.0
    # host seconds of the final mesh generation and of the space / per-mesh
    # data extraction (build_asm_data)
    host_s: dict = field(default_factory=dict)

    def summary(self) -> dict:
        nb = None
        return {"name": self.name, "p": self.p, "theta_deg": self.theta, "ne": self.ad.ne,
                "ndof": self.ad.height, "nnz": self.ad.nnz or nb}


def make_case(name: str, stack: Stack, p: int, theta: float, ndof_target: float | None = None,
              h: float | None = None, build_csr: bool = False,
              local_order_seed: int | None = None, elem_eps: bool = False) -> Case:
    prob = Problem.from_stack(stack, p, kpar_of(theta))
    if h is None:
        # grid lines on every interface round cell counts up: correct h once
        h = h_for_target_dofs(stack, p, ndof_target)
        trial = build_asm_data(build_mesh(stack, h), p, prob)
        h *= (trial.height / ndof_target) ** (1.0 / 3.0)
    t0 = time.perf_counter()
    mesh = build_mesh(stack, h)
    t1 = time.perf_counter()
    ad = build_asm_data(mesh, p, prob, build_csr=build_csr, local_order_seed=local_order_seed)
    t2 = time.perf_counter()
    if elem_eps:
        prob.elem_eps = absorber_jitter(ad, prob)
    return Case(name=name, stack=stack, p=p, theta=theta, ad=ad, prob=prob, mesh=mesh, h=h,
                host_s={"mesh": t1 - t0, "space": t2 - t1})


def make_poly_case(name: str, stack: Stack, p: int, theta: float,
                   ndof_target: float | None = None, h: float | None = None,
                   build_csr: bool = False, local_order_seed: int | None = None) -> Case:
    """A case on the polygon-hole mesh of ``stack`` (its single frustum is a
    PolyHole); h from the DOF target by one trial build at a coarser h."""
    hole = stack.frustums[0]
    prob = Problem.from_stack(stack, p, kpar_of(theta))
    if h is None:
        h0 = 1.6 * h_for_target_dofs(stack, p, ndof_target)
        trial = build_asm_data(build_poly_mesh(stack, hole, h0), p, prob)
        h = h0 * (trial.height / ndof_target) ** (1.0 / 3.0)
    mesh = build_poly_mesh(stack, hole, h)
    ad = build_asm_data(mesh, p, prob, build_csr=build_csr, local_order_seed=local_order_seed)
    return Case(name=name, stack=stack, p=p, theta=theta, ad=ad, prob=prob)


def poly_hole_stack(rng: np.random.Generator, lx: float = 96.0, ly: float = 96.0,
                    z_max: float = 120.0, t_range=(40.0, 70.0), pml_wl: float = 1.0) -> Stack:
    """Slab stack with one random polygonal vacuum hole through the absorber:
    U{3..8} vertices, side wall U(80, 90) deg, absorber thickness U(t_range)."""
    t = float(rng.uniform(*t_range))
    nv = int(rng.integers(3, 9))
    alpha = float(rng.uniform(80.0, 90.0))
    st = Stack(lx=lx, ly=ly, z_min=0.0, z_max=z_max, wavelength=WAVELENGTH,
               layers=[(0.0, t, ABSORBER)], pml_thickness_wavelengths=pml_wl)
    st.frustums = [random_hole(rng, lx, ly, 0.0, t, nv, alpha)]
    return st


def batch_config(scale: float = 1.0, n: int = 16, seed: int = SEED, theta: float = 6.0,
                 only: list[int] | None = None) -> list[Case]:
    """The batched workload: n seeded polygon-hole meshes, p cycled 1, 2, 3,
    DOF targets log-uniform in [20k, 400k] (times scale).  ``only`` builds a
    subset (one rank's share); the parameters of every mesh are still drawn
    in sequence, so mesh i is the same whichever subset is built."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        p = 1 + i % 3
        ndof = float(np.exp(rng.uniform(np.log(20e3), np.log(400e3)))) * scale
        st = poly_hole_stack(rng)
        if only is not None and i not in only:
            continue
        hole = st.frustums[0]
        name = (f"C5[{i}] polygon hole nv={len(hole.verts)} alpha={hole.alpha:.1f} "
                f"t={hole.h:.1f} p={p}")
        out.append(make_poly_case(name, st, p, theta, ndof))
    return out


def small_poly_case(p: int, theta: float, seed: int = 7, h: float | None = None,
                    local_order_seed: int | None = 7) -> Case:
    """Seconds-level polygon-hole case (shrunk cell) for the tests."""
    rng = np.random.default_rng(seed)
    st = poly_hole_stack(rng, lx=12.0, ly=12.0, z_max=12.0, t_range=(5.0, 7.0), pml_wl=0.4)
    hh = h if h is not None else {1: 2.0, 2: 3.0, 3: 4.0}[p]
    return make_poly_case(f"polygon hole p={p} theta={theta}", st, p, theta, h=hh,
                          build_csr=True, local_order_seed=local_order_seed)


def absorber_jitter(ad: AsmData, prob: Problem, seed: int = SEED, frac: float = 0.02
                    ) -> np.ndarray:
    """Per-element eps: absorber elements get U(+-frac) jitter of n and k."""
    eps = prob.eps_table()[ad.attr - 1].copy()
    rng = np.random.default_rng(seed)
    absorb = np.isclose(eps, ABSORBER) & ~np.array(
        [prob.regions[a - 1].is_pml for a in ad.attr])
    n = 0.95 * (1 + rng.uniform(-frac, frac, ad.ne))
    k = 0.031 * (1 + rng.uniform(-frac, frac, ad.ne))
    eps[absorb] = ((n + 1j * k) ** 2)[absorb]
    return eps


# -- the benchmark configurations -----------------------------------------

def config(idx: int, scale: float = 1.0, **kw) -> Case:
    """Benchmark config 1..4 (1-based, as listed); scale multiplies the DOF target."""
    if idx == 1:
        return make_case("C1 absorber slab p=1 theta=0", slab_stack(), 1, 0.0, 50e3 * scale, **kw)
    if idx == 2:
        return make_case("C2 contact hole p=2 theta=6", contact_hole_stack(), 2, 6.0,
                         300e3 * scale, **kw)
    if idx == 3:
        return make_case("C3 line grating p=3 theta=6", line_grating_stack(), 3, 6.0,
                         1.3e6 * scale, **kw)
    if idx == 4:
        return make_case("C4 contact hole p=2 theta=6 per-element eps", contact_hole_stack(), 2,
                         6.0, 300e3 * scale, elem_eps=True, **kw)
    raise ValueError(idx)


def small_case(kind: str, p: int, theta: float, seed: int | None = 7, h: float | None = None
               ) -> Case:
    """Seconds-level test meshes on the benchmark geometries (shrunk cells)."""
    if kind == "slab":
        st = Stack(lx=8.0, ly=8.0, z_min=0.0, z_max=12.0, wavelength=WAVELENGTH,
                   layers=[(0.0, 6.0, ABSORBER)], pml_thickness_wavelengths=0.4)
    elif kind == "hole":
        st = Stack(lx=12.0, ly=12.0, z_min=0.0, z_max=12.0, wavelength=WAVELENGTH,
                   layers=[(0.0, 6.0, ABSORBER)], pml_thickness_wavelengths=0.4,
                   frustums=[Frustum(3.0, 9.0, 3.0, 9.0, 0.0, 6.0, 80.0, 1.0 + 0j)])
    elif kind == "grating":
        st = Stack(lx=12.0, ly=4.0, z_min=-4.0, z_max=10.0, wavelength=WAVELENGTH,
                   layers=[(-4.0, 0.0, UNDERLAYER)], pml_thickness_wavelengths=0.4,
                   frustums=[Frustum(3.0, 9.0, 0.0, 4.0, 0.0, 6.0, 90.0, ABSORBER)])
    else:
        raise ValueError(kind)
    hh = h if h is not None else {1: 1.6, 2: 2.0, 3: 2.6}[p]
    return make_case(f"{kind} p={p} theta={theta}", st, p, theta, h=hh, build_csr=True,
                     local_order_seed=seed)
