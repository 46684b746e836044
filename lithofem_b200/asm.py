"""Host-side mirror of the reference's GPU assembly classes.

``AsmGpu`` / ``AsmGpuGlobal`` keep the names, call order, argument meaning
and error behaviour of solver/asm_gpu.inc:271-425 and :498-599: every stage
returns ``True``/``False``, a CUDA failure prints the one-line
``asm_gpu: CUDA error '<msg>' at <file>:<line>`` diagnostic, and the
test-only downloads print the ``asm_gpu_test_download`` marker.  The
problem tables the reference reads from its global ``prob`` are passed to
the constructor.  Everything runs in liblfasm.so (CUDA, sm_100a); there is
no CPU fallback.
"""

from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _abi, _lib
from ._abi import (BULK_VARIANTS, CROSS0, CROSS1, CURLCURL, KLK, MASS, c_double_p, c_int_p, marshal,
                   marshal_parts)
from .problem import Problem
from .space import AsmData

__all__ = ["AsmGpu", "AsmGpuGlobal", "CURLCURL", "MASS", "CROSS0", "CROSS1", "KLK",
           "DeviceVector"]


class DeviceVector:
    """Minimal __cuda_array_interface__ view of a borrowed device buffer."""

    def __init__(self, ptr: int, shape: tuple, typestr: str):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr,
                                         "data": (int(ptr), False), "version": 2,
                                         "strides": None}


class AsmGpu:
    def __init__(self, prob: Problem):
        self.prob = prob
        self._h = ct.c_void_p()
        self._ne = self._nd = 0
        self._m = None
        self.gpu_id = 0

    # -- helpers ---------------------------------------------------------
    def _ok(self, rc: int) -> bool:
        if rc != 0:
            msg = _lib.lib().lfasm_last_error().decode(errors="replace")
            if rc != 2:  # CUDA errors were already printed by the library
                print(f"asm_gpu: {msg}", flush=True)
            self.last_error = (rc, msg)
            return False
        return True

    @property
    def handle(self) -> ct.c_void_p:
        return self._h

    # -- AsmGpu (asm_gpu.inc:276-376) -------------------------------------
    def Init(self, ad: AsmData, gpu_id: int = 0, with_csr: bool = False) -> bool:
        L = _lib.lib()
        self.Release()
        self._m = marshal(ad, self.prob, with_csr=with_csr)
        self._ne, self._nd = ad.ne, ad.nd
        self.gpu_id = gpu_id
        return self._ok(L.lfasm_init(ct.byref(self._m.ad), ct.byref(self._m.prob), gpu_id,
                                     ct.byref(self._h)))

    def SetStream(self, stream_ptr: int) -> bool:
        return self._ok(_lib.lib().lfasm_set_stream(self._h, ct.c_void_p(stream_ptr)))

    def SetAsync(self, on: bool) -> bool:
        return self._ok(_lib.lib().lfasm_set_async(self._h, int(bool(on))))

    def ComputeLocal(self, mask_cc: int, mask_mass: int, apply_te: bool) -> bool:
        return self._ok(_lib.lib().lfasm_compute_local(self._h, mask_cc, mask_mass,
                                                       int(bool(apply_te))))

    def DownloadLocal(self) -> np.ndarray | None:
        out = np.empty(2 * self._ne * self._nd * self._nd, dtype=np.float64)
        if not self._ok(_lib.lib().lfasm_download_local(self._h, out.ctypes.data_as(c_double_p))):
            return None
        return out.view(np.complex128).reshape(self._ne, self._nd, self._nd)

    def DeviceLocal(self) -> int:
        p = ct.c_void_p()
        _lib.check(_lib.lib().lfasm_get_local(self._h, ct.byref(p)))
        return int(p.value or 0)

    def SetProfile(self, on: bool) -> bool:
        return self._ok(_lib.lib().lfasm_set_profile(self._h, int(bool(on))))

    def StageTimes(self) -> list[float]:
        """ms of {prep + bulk elements, PML elements, CSR gather} of the last Assemble."""
        out = (ct.c_float * 3)()
        _lib.check(_lib.lib().lfasm_stage_times(self._h, out))
        return [float(x) for x in out]

    def Autotune(self) -> bool:
        return self._ok(_lib.lib().lfasm_autotune(self._h))

    def SetBulkVariant(self, variant: int) -> bool:
        """0: SIMT bulk-element kernel; 1, 2: FP64 tensor-core (DMMA) variant
        with 4 or 2 tiles per warp."""
        return self._ok(_lib.lib().lfasm_set_bulk_variant(self._h, int(variant)))

    def Tuning(self) -> tuple[int, list[float]]:
        v = ct.c_int()
        ms = (ct.c_float * BULK_VARIANTS)()
        _lib.check(_lib.lib().lfasm_get_tuning(self._h, ct.byref(v), ms))
        return v.value, [float(x) for x in ms]

    def SetPmlVariant(self, variant: int) -> bool:
        return self._ok(_lib.lib().lfasm_set_pml_variant(self._h, int(variant)))

    def PmlTuning(self) -> tuple[int, list[float]]:
        v = ct.c_int()
        ms = (ct.c_float * 3)()
        _lib.check(_lib.lib().lfasm_get_pml_tuning(self._h, ct.byref(v), ms))
        return v.value, [float(x) for x in ms]

    # -- field sampling (solver/lithofem_solve.cpp:951-1004) ---------------
    def SetBasis(self, el) -> bool:
        """Hand the element basis (ndbasis.NDElement) to the library."""
        self._bexps = np.ascontiguousarray(np.asarray(el.monos, dtype=np.int32).reshape(-1))
        self._bcoef = np.ascontiguousarray(el.coef, dtype=np.float64)
        self._bccoef = np.ascontiguousarray(el._curl_coef, dtype=np.float64)
        return self._ok(_lib.lib().lfasm_set_basis(
            self._h, len(el.monos), self._bexps.ctypes.data_as(c_int_p),
            self._bcoef.ctypes.data_as(c_double_p), self._bccoef.ctypes.data_as(c_double_p)))

    def SamplePlane(self, lx: float, ly: float, z: float, nx: int, ny: int, u_ptr: int,
                    e_ptr: int, curl_ptr: int = 0) -> bool:
        """E (and curl E) of the device solution at the reference's plane grid,
        [ny][nx][3] complex128 into e_ptr / curl_ptr (device)."""
        return self._ok(_lib.lib().lfasm_sample_plane(
            self._h, float(lx), float(ly), float(z), int(nx), int(ny), ct.c_void_p(u_ptr),
            ct.c_void_p(e_ptr or None), ct.c_void_p(curl_ptr or None)))

    def SamplePlanes(self, lx: float, ly: float, zs, nx: int, ny: int, u_ptr: int, e_ptr: int,
                     curl_ptr: int = 0) -> bool:
        """SamplePlane for every height of zs in one pass: [len(zs)][ny][nx][3]
        complex128 into e_ptr / curl_ptr (device)."""
        z = np.ascontiguousarray(zs, dtype=np.float64)
        return self._ok(_lib.lib().lfasm_sample_planes(
            self._h, float(lx), float(ly), len(z), z.ctypes.data_as(c_double_p), int(nx),
            int(ny), ct.c_void_p(u_ptr), ct.c_void_p(e_ptr or None),
            ct.c_void_p(curl_ptr or None)))

    def PlaneOrders(self, nx: int, ny: int, e_ptr: int, planes, args, coef_ptr: int,
                    eff_ptr: int) -> bool:
        """Fourier orders (coef_ptr: [nz][ny * nx][3] complex128) and order
        efficiencies (eff_ptr: [nz][ny * nx] float64) of sampled planes.
        planes: sequence of dicts with z, z_ref, eps, direction and optional
        bg00 (3 complex); args: dict with lx, ly, k0, kx, ky, inc_flux."""
        arr = (_abi.OrderPlaneC * len(planes))()
        for i, q in enumerate(planes):
            eps = complex(q["eps"])
            arr[i].z, arr[i].z_ref = float(q["z"]), float(q["z_ref"])
            arr[i].eps_re, arr[i].eps_im = eps.real, eps.imag
            arr[i].direction = int(q["direction"])
            bg = q.get("bg00")
            arr[i].has_bg00 = 0 if bg is None else 1
            if bg is not None:
                b = np.asarray(bg, dtype=np.complex128).reshape(3)
                for c in range(3):
                    arr[i].bg00[2 * c], arr[i].bg00[2 * c + 1] = b[c].real, b[c].imag
        a = _abi.OrderArgsC(float(args["lx"]), float(args["ly"]), float(args["k0"]),
                            float(args["kx"]), float(args["ky"]), float(args["inc_flux"]))
        return self._ok(_lib.lib().lfasm_plane_orders(
            self._h, len(planes), int(nx), int(ny), ct.c_void_p(e_ptr), arr, ct.byref(a),
            ct.c_void_p(coef_ptr), ct.c_void_p(eff_ptr)))

    def PlaneSeed(self, lx: float, ly: float, z: float, nx: int, ny: int, comp: int, m: int,
                  q: int, c_ptr: int) -> bool:
        """c (device, n complex128) with c^T u = the (m, q) Fourier coefficient
        of component comp of the plane samples."""
        return self._ok(_lib.lib().lfasm_plane_seed(
            self._h, float(lx), float(ly), float(z), int(nx), int(ny), int(comp), int(m),
            int(q), ct.c_void_p(c_ptr)))

    def PathCounts(self) -> tuple[int, int]:
        a, b = ct.c_int(), ct.c_int()
        _lib.check(_lib.lib().lfasm_path_counts(self._h, ct.byref(a), ct.byref(b)))
        return a.value, b.value

    def ne(self) -> int:
        return self._ne

    def nd(self) -> int:
        return self._nd

    def Release(self) -> None:
        if self._h:
            _lib.lib().lfasm_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.Release()
        except Exception:  # interpreter shutdown
            pass


class AsmGpuGlobal(AsmGpu):
    """Owns the device CSR handed zero-copy to the sparse solver."""

    def BuildGlobal(self, ess_list) -> bool:
        ess = np.ascontiguousarray(np.asarray(ess_list, dtype=np.int32))
        self._ess = ess
        return self._ok(_lib.lib().lfasm_build_global(
            self._h, ess.ctypes.data_as(c_int_p) if ess.size else None, int(ess.size)))

    def ScatterEliminate(self, eliminate: bool) -> bool:
        return self._ok(_lib.lib().lfasm_scatter_eliminate(self._h, int(bool(eliminate))))

    def Assemble(self, eliminate: bool = True) -> bool:
        """Production path: fused ComputeLocal(CC, MASS[+kpar], te) + ScatterEliminate."""
        return self._ok(_lib.lib().lfasm_assemble(self._h, int(bool(eliminate))))

    def _csr(self):
        I, J, V = ct.c_void_p(), ct.c_void_p(), ct.c_void_p()
        n, nnz = ct.c_int(), ct.c_longlong()
        _lib.check(_lib.lib().lfasm_get_csr(self._h, ct.byref(I), ct.byref(J), ct.byref(V),
                                            ct.byref(n), ct.byref(nnz)))
        return int(I.value or 0), int(J.value or 0), int(V.value or 0), n.value, nnz.value

    def n(self) -> int:
        return self._csr()[3]

    def nnz(self) -> int:
        return self._csr()[4]

    def DeviceI(self) -> int:
        return self._csr()[0]

    def DeviceJ(self) -> int:
        return self._csr()[1]

    def DeviceValues(self) -> int:
        return self._csr()[2]

    def DeviceCsrViews(self):
        """__cuda_array_interface__ views (I int32, J int32, vals complex128)."""
        I, J, V, n, nnz = self._csr()
        return (DeviceVector(I, (n + 1,), "<i4"), DeviceVector(J, (nnz,), "<i4"),
                DeviceVector(V, (nnz,), "<c16"))

    def DownloadCsr(self) -> tuple[np.ndarray, np.ndarray]:
        _, _, _, n, nnz = self._csr()
        I = np.empty(n + 1, dtype=np.int32)
        J = np.empty(nnz, dtype=np.int32)
        _lib.check(_lib.lib().lfasm_download_csr(self._h, I.ctypes.data_as(c_int_p),
                                                 J.ctypes.data_as(c_int_p)))
        return I, J

    def DownloadValues(self) -> np.ndarray | None:
        nnz = self.nnz()
        out = np.empty(2 * nnz, dtype=np.float64)
        if not self._ok(_lib.lib().lfasm_download_values(self._h, out.ctypes.data_as(c_double_p))):
            return None
        return out.view(np.complex128)

    def Residual(self, X: np.ndarray, B: np.ndarray) -> tuple[bool, float]:
        """||A X - B|| / ||B||; X, B in the production [re; im] 2n layout."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        B = np.ascontiguousarray(B, dtype=np.float64)
        rel = ct.c_double()
        ok = self._ok(_lib.lib().lfasm_residual(self._h, X.ctypes.data_as(c_double_p),
                                                B.ctypes.data_as(c_double_p), ct.byref(rel)))
        return ok, rel.value

    def ResidualDevice(self, x_ptr: int, b_ptr: int) -> tuple[bool, float]:
        rel = ct.c_double()
        ok = self._ok(_lib.lib().lfasm_residual_device(self._h, ct.c_void_p(x_ptr),
                                                       ct.c_void_p(b_ptr), ct.byref(rel)))
        return ok, rel.value

    def SpMV(self, x_ptr: int, y_ptr: int) -> bool:
        return self._ok(_lib.lib().lfasm_spmv(self._h, ct.c_void_p(x_ptr), ct.c_void_p(y_ptr)))

    def EpsGradient(self, parts, u_ptr: int, lam_ptr: int, grad_ptr: int) -> bool:
        """grad[e] = lambda^T (db/deps_e - dA/deps_e u) for the non-PML elements."""
        arr, keep = marshal_parts(parts)
        ok = self._ok(_lib.lib().lfasm_eps_gradient(self._h, arr, len(parts), ct.c_void_p(u_ptr),
                                                    ct.c_void_p(lam_ptr), ct.c_void_p(grad_ptr)))
        del keep
        return ok

    def AssembleRHS(self, parts, col_of_part, ncol: int, eliminate: bool, b_ptr: int) -> bool:
        arr, keep = marshal_parts(parts)
        cols = np.ascontiguousarray(np.asarray(col_of_part, dtype=np.int32))
        ok = self._ok(_lib.lib().lfasm_assemble_rhs(
            self._h, arr, len(parts), cols.ctypes.data_as(c_int_p), int(ncol),
            int(bool(eliminate)), ct.c_void_p(b_ptr)))
        del keep
        return ok


class AsmBatch:
    """Several built ``AsmGpuGlobal`` handles of one device assembled by one
    CUDA-graph launch (``lfasm_batch_*``).  The handles must outlive the
    batch; ``Assemble`` has the effect of ``Assemble`` on each of them."""

    def __init__(self, handles: list[AsmGpuGlobal]):
        self._members = list(handles)
        self._b = ct.c_void_p()
        self.last_error = None
        arr = (ct.c_void_p * max(1, len(handles)))(*[h.handle.value for h in handles])
        rc = _lib.lib().lfasm_batch_create(arr, len(handles), ct.byref(self._b))
        if rc != 0:
            self.last_error = (rc, _lib.lib().lfasm_last_error().decode(errors="replace"))
            raise RuntimeError(f"lfasm_batch_create: {self.last_error[1]}")

    def SetStream(self, stream_ptr: int) -> bool:
        return _lib.lib().lfasm_batch_set_stream(self._b, ct.c_void_p(stream_ptr)) == 0

    def Assemble(self, eliminate: bool = True) -> bool:
        rc = _lib.lib().lfasm_batch_assemble(self._b, int(bool(eliminate)))
        if rc != 0:
            self.last_error = (rc, _lib.lib().lfasm_last_error().decode(errors="replace"))
            print(f"asm_gpu: {self.last_error[1]}", flush=True)
            return False
        return True

    def Release(self) -> None:
        if self._b:
            _lib.lib().lfasm_batch_destroy(self._b)
            self._b = ct.c_void_p()

    def __del__(self):
        try:
            self.Release()
        except Exception:  # interpreter shutdown
            pass
