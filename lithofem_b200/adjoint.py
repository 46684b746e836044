"""Adjoint gradient of a far-field objective with respect to per-element eps.

Objective: J = |l(u)|^2 with l(u) = c^T u the plane mean of one component of
the scattered envelope on a sampling plane, i.e. the (0,0) Rayleigh
coefficient of that component (the reference takes orders as plane FFTs,
src/lithofem/orders.py:36-67; the (0,0) term is the mean), and u the
solution of A(eps) u = b(eps) assembled by liblfasm.

Gradient (A, b holomorphic in eps_e):  with A^T lambda = c,
    dl/deps_e = lambda^T (db/deps_e - dA/deps_e u)      (lfasm_eps_gradient)
    dJ/dRe eps_e = 2 Re(conj(l) dl/deps_e),  dJ/dIm eps_e = -2 Im(conj(l) dl/deps_e).

The sparse solves are delegated to a solver object with ``solve(b)`` and
``solve_transposed(c)``.  The default is the device solver
(``solver.DeviceLU``: liblfsolve's complex64 factorization of the device
CSR, FP64-refined solves, the transposed solve with the same factors), the
role cuDSS has in the reference; the ordering is computed once per mesh and
reused by every design iteration.  ``HostLU`` (SuperLU on the host) is kept
as a CPU cross-check.  The assembly, right-hand side and gradient
contraction run on the GPU (liblfasm).
"""

from __future__ import annotations

import copy

import numpy as np

from . import ndbasis, space
from .asm import AsmGpuGlobal
from .solver import C64, DeviceLU, DirectSolver


class HostLU:
    """SuperLU factorisation of the device CSR on the host (CPU cross-check)."""

    def __init__(self, g: AsmGpuGlobal, ad=None):
        import scipy.sparse as sp
        import scipy.sparse.linalg as spl
        I, J = g.DownloadCsr()
        n = len(I) - 1
        A = sp.csr_matrix((g.DownloadValues(), J, I), shape=(n, n))
        self.lu = spl.splu(A.tocsc())

    def solve(self, b: np.ndarray) -> np.ndarray:
        return self.lu.solve(b)

    def solve_transposed(self, c: np.ndarray) -> np.ndarray:
        return self.lu.solve(c, trans="T")


class _Solvers:
    """Builds the solver for one assembled system: ``"device"`` (DeviceLU,
    the mesh's ordering computed once and reused) or a class taking (g, ad)
    such as HostLU."""

    def __init__(self, kind, gpu_id: int, prec: int, tol: float):
        self.kind, self.gpu_id, self.prec, self.tol = kind, gpu_id, prec, tol
        self.analysis = None

    def __call__(self, g: AsmGpuGlobal, ad):
        if self.kind != "device":
            return self.kind(g, ad)
        if self.analysis is None:
            self.analysis = DirectSolver(self.gpu_id)
            if not self.analysis.AnalyzeAssembly(g, ad):
                raise RuntimeError(f"lfsolve_analyze: {self.analysis.last_error}")
        return DeviceLU(g, prec=self.prec, tol=self.tol, analysis=self.analysis)


def plane_functional(ad: space.AsmData, z: float, lx: float, ly: float, comp: int,
                     nx: int = 8, ny: int = 8) -> np.ndarray:
    """c with c^T u = mean over an nx x ny plane grid of u_comp(x, y, z)."""
    xs = (np.arange(nx) + 0.5) * lx / nx
    ys = (np.arange(ny) + 0.5) * ly / ny
    X = np.array([[x, y, z] for y in ys for x in xs])
    ne, nd, p = ad.ne, ad.nd, ad.p
    Ji = ad.Jinv.reshape(ne, 3, 3)
    v0 = ad.v0.reshape(ne, 3)
    dof = ad.dof.reshape(ne, nd)
    sg = ad.sign.reshape(ne, nd)
    fo = ad.fo.reshape(ne, 4) if p > 1 else None
    el = ndbasis.nd_element(p)
    c = np.zeros(ad.height, dtype=complex)
    for x in X:
        xi = np.einsum("eij,ej->ei", Ji, x[None, :] - v0)
        lam = np.column_stack([1 - xi.sum(1), xi])
        e = int(np.argmax((lam >= -1e-12).all(1)))
        phys = el.vshape(xi[e][None])[0] @ Ji[e]          # (nd, 3) local basis values
        w = phys[:, comp] / len(X)                        # weight of local coefficient k
        # local coefficient = M (sign * global): fold M^T and the sign
        wg = w.copy()
        if p > 1:
            for f in range(4):
                M = space.face_tinv(fo[e, f])
                for i in range(p * (p - 1) // 2):
                    d0 = 6 * p + f * p * (p - 1) + 2 * i
                    wg[d0:d0 + 2] = M.T @ w[d0:d0 + 2]
        np.add.at(c, dof[e], sg[e] * wg)
    return c


class EpsAdjoint:
    """Assemble, solve and differentiate J = |c^T u|^2 w.r.t. per-element eps."""

    def __init__(self, ad, prob, parts, c: np.ndarray, gpu_id: int = 0, solver="device",
                 prec: int = C64, tol: float = 1e-12):
        self.ad, self.prob0, self.parts, self.c = ad, prob, parts, c
        self.gpu_id = gpu_id
        self.solver_cls = _Solvers(solver, gpu_id, prec, tol)

    def _assemble(self, eps: np.ndarray):
        import torch
        prob = copy.copy(self.prob0)
        prob.elem_eps = np.asarray(eps, dtype=complex)
        g = AsmGpuGlobal(prob)
        assert g.Init(self.ad, self.gpu_id) and g.BuildGlobal(self.ad.ess) and g.Assemble(True)
        b = torch.zeros(self.ad.height, dtype=torch.complex128, device=f"cuda:{self.gpu_id}")
        assert g.AssembleRHS(self.parts, [0] * len(self.parts), 1, True, b.data_ptr())
        return g, b

    def value(self, eps: np.ndarray) -> complex:
        g, b = self._assemble(eps)
        u = self.solver_cls(g, self.ad).solve(b.cpu().numpy())
        return complex(self.c @ u)

    def value_and_grad(self, eps: np.ndarray):
        """(l, J, dJ/dRe eps, dJ/dIm eps, dl/deps) for eps (ne complex)."""
        import torch
        g, b = self._assemble(eps)
        lu = self.solver_cls(g, self.ad)
        u = lu.solve(b.cpu().numpy())
        lam = lu.solve_transposed(self.c)
        ell = complex(self.c @ u)
        dev = b.device
        ud = torch.from_numpy(u).to(dev)
        ld = torch.from_numpy(lam).to(dev)
        gd = torch.zeros(self.ad.ne, dtype=torch.complex128, device=dev)
        assert g.EpsGradient(self.parts, ud.data_ptr(), ld.data_ptr(), gd.data_ptr())
        dl = gd.cpu().numpy()
        dJ_re = 2.0 * np.real(np.conj(ell) * dl)
        dJ_im = -2.0 * np.imag(np.conj(ell) * dl)
        return ell, abs(ell) ** 2, dJ_re, dJ_im, dl


class EffAdjoint:
    """The zeroth up-going order efficiency on a plane above the structure
    and its gradient with respect to per-element eps.

    eta = flux(c) / incident flux, c = the (0,0) Fourier coefficient of the
    scattered envelope sampled on the plane (three component seeds from
    lfasm_plane_seed, c_d = s_d^T u) plus the analytic reflected background
    at the same plane (the up-going part of the top slab's incident table);
    flux(c) = Re[(c x (k x c / k0)*)_z] / 2 x area with k = (kx, ky, qz) of
    the order (outputs.py:219-269, orders.py:70-86).  As a real quadratic
    form eta = kappa c^H Q c, so with g = kappa Q c the adjoint seed is
    sum_d conj(g_d) s_d and deta/deps_e = 2 Re / -2 Im of
    lambda^T (db/deps_e - dA/deps_e u) (lfasm_eps_gradient).
    """

    def __init__(self, ad, prob, parts, z_plane: float, lx: float, ly: float, nx: int = 8,
                 ny: int = 8, gpu_id: int = 0, solver="device", prec: int = C64,
                 tol: float = 1e-12):
        self.ad, self.prob0, self.parts = ad, prob, parts
        self.z, self.lx, self.ly, self.nx, self.ny = z_plane, lx, ly, nx, ny
        self.gpu_id = gpu_id
        self.solver_cls = _Solvers(solver, gpu_id, prec, tol)
        self.last = None     # (handle, solver, u) of the last value_and_grad
        k0 = prob.k0
        kx, ky = prob.kx, prob.ky
        # top-slab incident tables of every part (one plane wave's s/p parts
        # share the direction): A down-going incident, B up-going background
        tops = [part[-1] for part in parts]
        qz = tops[0].qB
        self.k = np.array([kx, ky, qz.real])
        self.k0 = k0
        self.c_bg = sum(t.B * np.exp(1j * t.qB * (z_plane - t.zB)) for t in tops)
        a_in = sum(t.A * np.exp(1j * t.qA * (z_plane - t.zA)) for t in tops)
        self.area = lx * ly
        self.inc_flux = abs(self._flux(a_in, np.array([kx, ky, tops[0].qA.real])))
        self._seeds = None

    def _flux(self, c, k) -> float:
        h = np.cross(k, c) / self.k0
        return 0.5 * float(np.real(np.cross(c, np.conj(h))[2])) * self.area

    def _Q(self) -> np.ndarray:
        kx, ky, kz = self.k
        return np.array([[kz, 0.0, -kx / 2], [0.0, kz, -ky / 2], [-kx / 2, -ky / 2, 0.0]])

    def _assemble(self, eps):
        import torch
        prob = copy.copy(self.prob0)
        prob.elem_eps = np.asarray(eps, dtype=complex)
        g = AsmGpuGlobal(prob)
        assert g.Init(self.ad, self.gpu_id) and g.BuildGlobal(self.ad.ess) and g.Assemble(True)
        dev = f"cuda:{self.gpu_id}"
        b = torch.zeros(self.ad.height, dtype=torch.complex128, device=dev)
        assert g.AssembleRHS(self.parts, [0] * len(self.parts), 1, True, b.data_ptr())
        if self._seeds is None:
            assert g.SetBasis(ndbasis.nd_element(self.ad.p))
            seeds = []
            for comp in range(3):
                sd = torch.empty(self.ad.height, dtype=torch.complex128, device=dev)
                assert g.PlaneSeed(self.lx, self.ly, self.z, self.nx, self.ny, comp, 0, 0,
                                   sd.data_ptr())
                seeds.append(sd.cpu().numpy())
            self._seeds = np.stack(seeds)
        return g, b

    def coefficient(self, u: np.ndarray) -> np.ndarray:
        return self._seeds @ u + self.c_bg

    def efficiency(self, c: np.ndarray) -> float:
        return self._flux(c, self.k) / self.inc_flux

    def value(self, eps) -> float:
        g, b = self._assemble(eps)
        u = self.solver_cls(g, self.ad).solve(b.cpu().numpy())
        return self.efficiency(self.coefficient(u))

    def kappa(self) -> float:
        """eta = kappa c^H Q c."""
        return 0.5 * self.area / (self.k0 * self.inc_flux)

    def Q(self) -> np.ndarray:
        return self._Q()

    def value_and_grad(self, eps):
        """(eta, deta/dRe eps, deta/dIm eps) for eps (ne complex)."""
        import torch
        g, b = self._assemble(eps)
        lu = self.solver_cls(g, self.ad)
        u = lu.solve(b.cpu().numpy())
        c = self.coefficient(u)
        eta = self.efficiency(c)
        kappa = self.kappa()
        gw = kappa * (self._Q() @ c)
        lam = lu.solve_transposed(np.conj(gw) @ self._seeds)
        dev = b.device
        ud = torch.from_numpy(u).to(dev)
        ld = torch.from_numpy(lam).to(dev)
        gd = torch.zeros(self.ad.ne, dtype=torch.complex128, device=dev)
        assert g.EpsGradient(self.parts, ud.data_ptr(), ld.data_ptr(), gd.data_ptr())
        dl = gd.cpu().numpy()
        self.last = (g, lu, u)
        return eta, 2.0 * np.real(dl), -2.0 * np.imag(dl)


def autograd_function(adj: EpsAdjoint):
    """torch.autograd.Function mapping (Re eps, Im eps) -> J = |l|^2."""
    import torch

    class _EpsObjective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, eps_re, eps_im):
            eps = eps_re.detach().cpu().numpy() + 1j * eps_im.detach().cpu().numpy()
            _, J, gre, gim, _ = adj.value_and_grad(eps)
            ctx.save_for_backward(torch.from_numpy(gre).to(eps_re), torch.from_numpy(gim).to(eps_im))
            return eps_re.new_tensor(J)

        @staticmethod
        def backward(ctx, gout):
            gre, gim = ctx.saved_tensors
            return gout * gre, gout * gim

    return _EpsObjective
