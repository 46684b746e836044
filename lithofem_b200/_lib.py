"""Loader for the in-tree CUDA library liblfasm.so.

There is deliberately no fallback: if the library is missing or cannot be
loaded, every entry point raises.
"""

from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

from ._abi import (AsmDataC, IncidentPartC, OrderArgsC, OrderPlaneC, ProblemC, c_double_p,
                   c_int_p)

LIB_PATH = Path(__file__).resolve().parent / "liblfasm.so"
# LFASM_LIBRARY selects another build of the same library (the
# bounds-checked liblfasm_bounds.so); the default is the in-tree liblfasm.so
if os.environ.get("LFASM_LIBRARY"):
    LIB_PATH = Path(os.environ["LFASM_LIBRARY"]).resolve()

_lib = None


class LfasmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"lfasm error {code}: {msg}")
        self.code = code


def lib() -> ct.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
            " (the assembly path has no CPU fallback)")
    L = ct.CDLL(os.fspath(LIB_PATH))
    H = ct.c_void_p
    sig = {
        "lfasm_last_error": (ct.c_char_p, []),
        "lfasm_launch_count": (ct.c_longlong, []),
        "lfasm_init": (ct.c_int, [ct.POINTER(AsmDataC), ct.POINTER(ProblemC), ct.c_int,
                                  ct.POINTER(H)]),
        "lfasm_set_stream": (ct.c_int, [H, ct.c_void_p]),
        "lfasm_set_async": (ct.c_int, [H, ct.c_int]),
        "lfasm_compute_local": (ct.c_int, [H, ct.c_int, ct.c_int, ct.c_int]),
        "lfasm_get_local": (ct.c_int, [H, ct.POINTER(ct.c_void_p)]),
        "lfasm_download_local": (ct.c_int, [H, c_double_p]),
        "lfasm_build_global": (ct.c_int, [H, c_int_p, ct.c_int]),
        "lfasm_scatter_eliminate": (ct.c_int, [H, ct.c_int]),
        "lfasm_assemble": (ct.c_int, [H, ct.c_int]),
        "lfasm_get_csr": (ct.c_int, [H, ct.POINTER(ct.c_void_p), ct.POINTER(ct.c_void_p),
                                     ct.POINTER(ct.c_void_p), ct.POINTER(ct.c_int),
                                     ct.POINTER(ct.c_longlong)]),
        "lfasm_download_csr": (ct.c_int, [H, c_int_p, c_int_p]),
        "lfasm_download_values": (ct.c_int, [H, c_double_p]),
        "lfasm_residual": (ct.c_int, [H, c_double_p, c_double_p, c_double_p]),
        "lfasm_residual_device": (ct.c_int, [H, ct.c_void_p, ct.c_void_p, c_double_p]),
        "lfasm_spmv": (ct.c_int, [H, ct.c_void_p, ct.c_void_p]),
        "lfasm_assemble_rhs": (ct.c_int, [H, ct.POINTER(IncidentPartC), ct.c_int, c_int_p,
                                          ct.c_int, ct.c_int, ct.c_void_p]),
        "lfasm_path_counts": (ct.c_int, [H, c_int_p, c_int_p]),
        "lfasm_set_profile": (ct.c_int, [H, ct.c_int]),
        "lfasm_stage_times": (ct.c_int, [H, ct.POINTER(ct.c_float)]),
        "lfasm_csr_residual_noalloc": (ct.c_int, [ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                                  ct.c_void_p, ct.c_void_p, c_double_p,
                                                  ct.c_void_p]),
        "lfasm_eps_gradient": (ct.c_int, [H, ct.POINTER(IncidentPartC), ct.c_int, ct.c_void_p,
                                          ct.c_void_p, ct.c_void_p]),
        "lfasm_autotune": (ct.c_int, [H]),
        "lfasm_set_bulk_variant": (ct.c_int, [H, ct.c_int]),
        "lfasm_get_tuning": (ct.c_int, [H, c_int_p, ct.POINTER(ct.c_float)]),
        "lfasm_set_pml_variant": (ct.c_int, [H, ct.c_int]),
        "lfasm_get_pml_tuning": (ct.c_int, [H, c_int_p, ct.POINTER(ct.c_float)]),
        "lfasm_destroy": (None, [H]),
        "lfasm_trim_pool": (ct.c_int, [ct.c_int]),
        "lfasm_bounds_checked": (ct.c_int, []),
        "lfasm_debug_wait_test": (ct.c_int, [ct.c_int, ct.c_longlong, ct.c_int]),
        "lfasm_set_basis": (ct.c_int, [H, ct.c_int, c_int_p, c_double_p, c_double_p]),
        "lfasm_sample_plane": (ct.c_int, [H, ct.c_double, ct.c_double, ct.c_double, ct.c_int,
                                          ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p]),
        "lfasm_plane_seed": (ct.c_int, [H, ct.c_double, ct.c_double, ct.c_double, ct.c_int,
                                        ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p]),
        "lfasm_sample_planes": (ct.c_int, [H, ct.c_double, ct.c_double, ct.c_int, c_double_p,
                                           ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p,
                                           ct.c_void_p]),
        "lfasm_plane_orders": (ct.c_int, [H, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p,
                                          ct.POINTER(OrderPlaneC), ct.POINTER(OrderArgsC),
                                          ct.c_void_p, ct.c_void_p]),
        "lfasm_extract": (ct.c_int, [ct.c_int, ct.c_int, ct.c_int, ct.c_int, c_int_p, c_double_p,
                                     c_int_p, c_double_p, c_int_p, c_double_p, c_double_p,
                                     c_double_p, c_double_p, c_int_p, ct.c_longlong,
                                     ct.POINTER(ct.c_int), ct.POINTER(ct.c_int)]),
        "lfasm_batch_create": (ct.c_int, [ct.POINTER(ct.c_void_p), ct.c_int, ct.POINTER(ct.c_void_p)]),
        "lfasm_batch_set_stream": (ct.c_int, [ct.c_void_p, ct.c_void_p]),
        "lfasm_batch_assemble": (ct.c_int, [ct.c_void_p, ct.c_int]),
        "lfasm_batch_destroy": (None, [ct.c_void_p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != 0:
        msg = lib().lfasm_last_error().decode(errors="replace")
        raise LfasmError(rc, msg)


def exported_symbols() -> list[str]:
    """Entry points declared in include/lfasm.h."""
    hdr = Path(__file__).resolve().parents[1] / "include" / "lfasm.h"
    import re
    names = re.findall(r"^(?:const\s+)?(?:int|void|long long|const char)\s*\*?\s*(lfasm_\w+)\s*\(",
                       hdr.read_text(), flags=re.M)
    return sorted(set(names))
