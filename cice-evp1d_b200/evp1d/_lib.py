"""ctypes binding of libevp1d.so (the C-ABI declared in include/evp1d.h).

The library is loaded from ``cice-evp1d_b200/lib/libevp1d.so``.  There is no
fallback: if the shared library is missing the import fails with the command
that builds it.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# EVP1D_LIBRARY=fma selects the FMA flavour (lib/libevp1d_fma.so); any other
# value is a path to a build of the library.
_FLAVOUR = os.environ.get("EVP1D_LIBRARY", "")
FLAVOUR = "fma" if _FLAVOUR == "fma" else ("exact" if not _FLAVOUR else "custom")
LIB_PATH = (os.path.join(PKG_ROOT, "lib", "libevp1d_fma.so") if _FLAVOUR == "fma"
            else _FLAVOUR or os.path.join(PKG_ROOT, "lib", "libevp1d.so"))

EVP1D_OK = 0
ERRORS = {
    -1: "EVP1D_ERR_INVALID_ARG", -2: "EVP1D_ERR_INDEX", -3: "EVP1D_ERR_CUDA",
    -4: "EVP1D_ERR_NOMEM", -5: "EVP1D_ERR_TIMEOUT", -6: "EVP1D_ERR_NO_DEVICE",
    -7: "EVP1D_ERR_STATE",
}

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int32)

PARAM_FIELDS = ("arlx1i", "denom1", "brlx", "capping", "e_factor", "epp2i",
                "deltaminEVP", "revp", "Ktens", "u0", "cosw", "sinw", "rhow")


class Params(C.Structure):
    """evp1d_params (include/evp1d.h)."""
    _fields_ = [(n, C.c_double) for n in PARAM_FIELDS]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n in PARAM_FIELDS}


class Fields(C.Structure):
    """evp1d_fields (include/evp1d.h)."""
    _fields_ = [
        ("skipT", _I), ("skipU", _I), ("stress", _D * 12),
        ("strength", _D), ("Cw", _D), ("aiu", _D), ("uocn", _D), ("vocn", _D),
        ("waterx", _D), ("watery", _D), ("forcex", _D), ("forcey", _D),
        ("umassdti", _D), ("fm", _D), ("Tbu", _D), ("uvel_init", _D),
        ("vvel_init", _D), ("uvel", _D), ("vvel", _D), ("strintx", _D),
        ("strinty", _D), ("Cb", _D), ("str", _D * 8),
    ]


class Grads(C.Structure):
    """evp1d_grads (include/evp1d.h)."""
    _fields_ = [
        ("strength", _D), ("Cw", _D), ("forcex", _D), ("forcey", _D),
        ("uvel", _D), ("vvel", _D), ("stress", _D * 12),
        ("uvel_init", _D), ("vvel_init", _D),
    ]


class EVP1DError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load() -> C.CDLL:
    """Load libevp1d.so once; raise ImportError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} not found: build it with `make -C {PKG_ROOT}` "
            "(nvcc, sm_100a)")
    L = C.CDLL(LIB_PATH)
    H = C.c_void_p
    L.evp1d_set_evp_parameters.argtypes = [C.POINTER(Params), C.c_int]
    L.evp1d_set_evp_parameters.restype = None
    L.evp1d_init.argtypes = ([C.POINTER(H), C.c_int, C.c_int] + [_I] * 6
                             + [_D] * 7 + [C.POINTER(Params), C.c_int])
    L.evp1d_finalize.argtypes = [H]
    L.evp1d_set_params.argtypes = [H, C.POINTER(Params)]
    L.evp1d_run.argtypes = [H, C.c_int, C.POINTER(Fields)]
    L.evp1d_upload.argtypes = [H, C.POINTER(Fields)]
    L.evp1d_subcycles.argtypes = [H, C.c_int]
    L.evp1d_subcycles_inner.argtypes = [H, C.c_int]
    L.evp1d_download.argtypes = [H, C.POINTER(Fields)]
    L.evp1d_stress_only.argtypes = [H, C.c_int]
    L.evp1d_stepu_only.argtypes = [H, C.c_int]
    L.evp1d_synchronize.argtypes = [H]
    L.evp1d_stream.argtypes = [H]
    L.evp1d_stream.restype = C.c_void_p
    L.evp1d_launch_count.argtypes = [H, C.c_int]
    L.evp1d_launch_count.restype = C.c_longlong
    L.evp1d_last_error.restype = C.c_char_p
    L.evp1d_last_error.argtypes = []
    L.evp1d_version.restype = C.c_char_p
    L.evp1d_binary_version.argtypes = [C.c_int]
    L.evp1d_binary_version.restype = C.c_int
    L.evp1d_init_batched.argtypes = ([C.POINTER(H), C.c_int, _I, _I] + [_I] * 6
                                     + [_D] * 7 + [C.POINTER(Params), C.c_int])
    L.evp1d_init_batched.restype = C.c_int
    L.evp1d_autotune.argtypes = [H, C.c_int, C.c_char_p, C.c_int]
    L.evp1d_autotune.restype = C.c_int
    L.evp1d_debug_trace.argtypes = [H, C.POINTER(C.c_longlong), C.c_int]
    L.evp1d_debug_trace.restype = C.c_int
    L.evp1d_debug_wait_timeout.argtypes = [H, C.c_longlong]
    L.evp1d_debug_wait_timeout.restype = C.c_int
    L.evp1d_debug_dep_wait_timeout.argtypes = [H, C.c_longlong]
    L.evp1d_debug_dep_wait_timeout.restype = C.c_int
    L.evp1d_kernel_path.argtypes = [H]
    L.evp1d_kernel_path.restype = C.c_char_p
    L.evp1d_build_index.argtypes = ([C.c_int, C.c_int, C.c_int, _I, C.c_int,
                                     C.c_int, C.POINTER(C.c_int),
                                     C.POINTER(C.c_int)] + [_I] * 9)
    L.evp1d_plan_stats.argtypes = [C.c_int, C.c_int] + [_I] * 6 + [C.POINTER(C.c_longlong)]
    L.evp1d_plan_check.argtypes = [C.c_int, C.c_int] + [_I] * 6 + [C.POINTER(C.c_longlong)]
    L.evp1d_run_checkpointed.argtypes = [H, C.c_int, C.POINTER(Fields), C.c_int]
    L.evp1d_record_subcycles.argtypes = [H, C.c_int, C.c_int]
    L.evp1d_adjoint.argtypes = [H, _D, _D, C.POINTER(_D), C.POINTER(Grads)]
    L.evp1d_adjoint_seed.argtypes = [H, _D, _D, C.POINTER(_D)]
    L.evp1d_adjoint_sweep.argtypes = [H]
    L.evp1d_adjoint_gradients.argtypes = [H, C.POINTER(Grads)]
    L.evp1d_adjoint_info.argtypes = [H, C.POINTER(C.c_longlong)]
    L.evp1d_set_adjoint_budget.argtypes = [H, C.c_longlong]
    L.evp1d_set_tile_points.argtypes = [C.c_int]
    L.evp1d_set_tile_points.restype = C.c_int
    L.evp1d_get_tile_points.argtypes = []
    L.evp1d_get_tile_points.restype = C.c_int
    L.evp1d_debug_fail_alloc.argtypes = [C.c_int]
    L.evp1d_debug_fail_alloc.restype = C.c_int
    L.evp1d_exchange_setup.argtypes = [H, C.c_int, _I, C.c_int, _I]
    L.evp1d_exchange_pack.argtypes = [H, C.c_void_p]
    L.evp1d_exchange_unpack.argtypes = [H, C.c_void_p]
    L.evp1d_exchange_buffers.argtypes = [H, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
    for name in ("evp1d_exchange_setup", "evp1d_exchange_pack", "evp1d_exchange_unpack",
                 "evp1d_exchange_buffers"):
        getattr(L, name).restype = C.c_int
    for name in ("evp1d_run_checkpointed", "evp1d_record_subcycles", "evp1d_adjoint",
                 "evp1d_adjoint_seed", "evp1d_adjoint_sweep", "evp1d_adjoint_gradients",
                 "evp1d_adjoint_info", "evp1d_set_adjoint_budget"):
        getattr(L, name).restype = C.c_int
    L.evp1d_host_alloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    L.evp1d_host_alloc.restype = C.c_int
    L.evp1d_host_free.argtypes = [C.c_void_p]
    L.evp1d_host_free.restype = C.c_int
    L.evp1d_run_device_noalloc.argtypes = ([C.c_int, C.c_int] + [C.c_void_p] * 13
                                           + [C.POINTER(Params), C.c_int,
                                              C.POINTER(Fields), C.c_void_p])
    L.evp1d_run_device_noalloc.restype = C.c_int
    for name in ("evp1d_plan_stats", "evp1d_plan_check", "evp1d_init", "evp1d_finalize", "evp1d_set_params",
                 "evp1d_run", "evp1d_upload", "evp1d_subcycles",
                 "evp1d_download", "evp1d_stress_only", "evp1d_stepu_only",
                 "evp1d_synchronize", "evp1d_build_index"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(rc: int, where: str) -> None:
    if rc != EVP1D_OK:
        msg = load().evp1d_last_error().decode(errors="replace")
        raise EVP1DError(rc, where, msg)
