"""Test helpers: difference-layer problem and FEM field evaluation.

The scattered-field envelope of a stack whose frustum fills the whole cell
in z in [z0, z0 + h] is known analytically: the TMM field of the modified
stack minus that of the background stack (the reference's M6-2 check,
tests/test_solver_m6.py:127-148).
"""

from __future__ import annotations

import numpy as np

from lithofem_b200 import configs, incident, mesh, ndbasis, problem, space

L = 8.0
EPS_D = (0.9 + 0.05j) ** 2


def difference_layer(p: int, h: float, theta: float = 6.0, pol: str = "s"):
    st = mesh.Stack(lx=L, ly=L, z_min=0.0, z_max=40.0, wavelength=configs.WAVELENGTH,
                    layers=[(0.0, 20.0, configs.ABSORBER)],
                    frustums=[mesh.Frustum(0.0, L, 0.0, L, 5.0, 10.0, 90.0, EPS_D)])
    ms = mesh.build_mesh(st, h)
    pr = problem.Problem.from_stack(st, p, incident.kpar_of(st, theta))
    ad = space.build_asm_data(ms, p, pr, build_csr=True, local_order_seed=4)
    parts = [incident.planewave_parts(st, theta, 0.0, pol)]
    st2 = mesh.Stack(lx=L, ly=L, z_min=0.0, z_max=40.0, wavelength=configs.WAVELENGTH,
                     layers=[(0.0, 5.0, configs.ABSORBER), (5.0, 15.0, EPS_D),
                             (15.0, 20.0, configs.ABSORBER)])
    exact = [incident.planewave_parts(st2, theta, 0.0, pol)]
    return st, ad, pr, parts, exact


def eval_field(ad, u: np.ndarray, X: np.ndarray) -> np.ndarray:
    """Physical envelope u(x) at points X (n, 3) from global DOF values."""
    ne, nd, p = ad.ne, ad.nd, ad.p
    Ji = ad.Jinv.reshape(ne, 3, 3)
    v0 = ad.v0.reshape(ne, 3)
    dof = ad.dof.reshape(ne, nd)
    sg = ad.sign.reshape(ne, nd)
    fo = ad.fo.reshape(ne, 4) if p > 1 else None
    el = ndbasis.nd_element(p)
    out = []
    for x in X:
        xi = np.einsum("eij,ej->ei", Ji, x[None, :] - v0)
        lam = np.column_stack([1 - xi.sum(1), xi])
        e = int(np.argmax((lam >= -1e-12).all(1)))
        g = sg[e] * u[dof[e]]
        c = g.copy()
        if p > 1:
            for f in range(4):
                M = space.face_tinv(fo[e, f])
                for i in range(p * (p - 1) // 2):
                    d0 = 6 * p + f * p * (p - 1) + 2 * i
                    c[d0:d0 + 2] = M @ g[d0:d0 + 2]
        ur = np.einsum("k,kd->d", c, el.vshape(xi[e][None])[0])
        out.append(ur @ Ji[e])
    return np.array(out)


def sample_points(n: int = 60, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.column_stack([rng.uniform(0.5, L - 0.5, n), rng.uniform(0.5, L - 0.5, n),
                            rng.uniform(1.0, 39.0, n)])


def field_error(ad, u, exact, parts) -> float:
    X = sample_points()
    got = eval_field(ad, u, X)
    ref = incident.eval_parts(exact, X[:, 2]) - incident.eval_parts(parts, X[:, 2])
    return float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
