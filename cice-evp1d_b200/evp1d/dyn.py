"""2D adapter: dyn_evp1d_init / dyn_evp1d_run / dyn_evp1d_finalize on global
2D arrays (integration/ice_dyn_evp1d.F90:65-255, 326-331) through the
library's evp1d_dyn_* entry points."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import Params, check

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int32)

STRESS = ("stressp_1", "stressp_2", "stressp_3", "stressp_4",
          "stressm_1", "stressm_2", "stressm_3", "stressm_4",
          "stress12_1", "stress12_2", "stress12_3", "stress12_4")
INPUTS = ("strength", "cdn_ocn", "aiu", "uocn", "vocn", "waterxU", "wateryU",
          "forcexU", "forceyU", "umassdti", "fmU", "Tbu")


class DynFields(C.Structure):
    _fields_ = ([("stress", _D * 12)] + [(k, _D) for k in INPUTS]
                + [("strintxU", _D), ("strintyU", _D), ("Cb", _D), ("uvel", _D),
                   ("vvel", _D), ("icetmask", _I), ("iceumask", _I)])


def _bind(L):
    if getattr(L, "_dyn_bound", False):
        return
    H = C.c_void_p
    L.evp1d_dyn_init.argtypes = [C.POINTER(H), C.c_int, C.c_int, C.c_int, _I] + [_D] * 5 + [
        C.POINTER(Params), C.c_int]
    L.evp1d_dyn_run.argtypes = [H, C.c_int, C.POINTER(DynFields)]
    L.evp1d_dyn_finalize.argtypes = [H]
    L.evp1d_dyn_sizes.argtypes = [H, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    for n in ("evp1d_dyn_init", "evp1d_dyn_run", "evp1d_dyn_finalize", "evp1d_dyn_sizes"):
        getattr(L, n).restype = C.c_int
    L._dyn_bound = True


def _f(a):
    a = np.asarray(a)
    if a.dtype != np.float64 or not a.flags.f_contiguous:
        raise ValueError("2D fields must be float64 and Fortran-ordered")
    return a.ctypes.data_as(_D)


class Dyn2D:
    """One 2D domain (global arrays [nx, ny] including ghost cells)."""

    def __init__(self, tmask, dyT, dxT, uarear, HTE, HTN, params: Params,
                 nghost: int = 1, device: int = 0):
        L = _lib.load()
        _bind(L)
        self._L = L
        nx, ny = np.asarray(tmask).shape
        self.shape = (nx, ny)
        m = np.asfortranarray(np.asarray(tmask, dtype=np.int32))
        h = C.c_void_p()
        check(L.evp1d_dyn_init(C.byref(h), nx, ny, nghost, m.ctypes.data_as(_I),
                               _f(dyT), _f(dxT), _f(uarear), _f(HTE), _f(HTN),
                               C.byref(params), int(device)), "evp1d_dyn_init")
        self.h = h

    @property
    def sizes(self):
        na, navel = C.c_int(), C.c_int()
        check(self._L.evp1d_dyn_sizes(self.h, C.byref(na), C.byref(navel)), "evp1d_dyn_sizes")
        return na.value, navel.value

    def run(self, ndte: int, fields: dict, icetmask, iceumask) -> dict:
        """dyn_evp1d_run: `fields` maps the reference's names (STRESS, INPUTS,
        strintxU, strintyU, Cb, uvel, vvel) to Fortran-ordered float64 arrays;
        the inout ones are updated in place."""
        f = DynFields()
        for k, n in enumerate(STRESS):
            f.stress[k] = _f(fields[n])
        for n in INPUTS:
            setattr(f, n, _f(fields[n]))
        for n in ("strintxU", "strintyU", "Cb", "uvel", "vvel"):
            setattr(f, n, _f(fields[n]))
        tm = np.asfortranarray(np.asarray(icetmask, dtype=np.int32))
        um = np.asfortranarray(np.asarray(iceumask, dtype=np.int32))
        f.icetmask, f.iceumask = tm.ctypes.data_as(_I), um.ctypes.data_as(_I)
        check(self._L.evp1d_dyn_run(self.h, int(ndte), C.byref(f)), "evp1d_dyn_run")
        return fields

    def finalize(self):
        if getattr(self, "h", None):
            check(self._L.evp1d_dyn_finalize(self.h), "evp1d_dyn_finalize")
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.finalize()

    def __del__(self):
        try:
            self.finalize()
        except Exception:
            pass


def fields_from_grid(g) -> dict:
    """The reference's dyn_evp1d_run field names for a synth.Grid2D."""
    F = {k: g.f[k].copy(order="F") for k in STRESS}
    rename = dict(strength="strength", cdn_ocn="Cw", aiu="aiu", uocn="uocn", vocn="vocn",
                  waterxU="waterx", wateryU="watery", forcexU="forcex", forceyU="forcey",
                  umassdti="umassdti", fmU="fm", Tbu="Tbu", strintxU="strintx",
                  strintyU="strinty", Cb="Cb", uvel="uvel", vvel="vvel")
    for k, src in rename.items():
        F[k] = g.f[src].copy(order="F")
    return F
