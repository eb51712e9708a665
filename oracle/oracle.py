"""ctypes front-end of the EVP-1D oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``liboracle_f1.so`` (bit-exact build, no FMA) or ``liboracle_f2.so``
(AVX2/FMA performance build) from this directory and runs the C restatement
of the reference's kernels (see evp_oracle.h for the file:line map).  Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
use this module; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict = {}

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int32)


class OracleParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "arlx1i", "denom1", "brlx", "capping", "e_factor", "epp2i",
        "deltaminEVP", "revp", "Ktens", "u0", "cosw", "sinw", "rhow")]


class Oracle1D(C.Structure):
    _fields_ = (
        [("na", C.c_int), ("navel", C.c_int)]
        + [(n, _I) for n in ("ee", "ne", "se", "nw", "sw", "sse", "skipT", "skipU")]
        + [(n, _D) for n in ("dxT", "dyT", "HTE", "HTN", "HTEm1", "HTNm1",
                             "strength", "Cw", "aiu", "uocn", "vocn", "waterx",
                             "watery", "forcex", "forcey", "umassdti", "fm",
                             "uarear", "Tbu", "uvel_init", "vvel_init")]
        + [("stress", _D * 12), ("uvel", _D), ("vvel", _D), ("str", _D * 8),
           ("strintx", _D), ("strinty", _D), ("Cb", _D)])


def build(quiet: bool = True) -> None:
    """Compile the oracle libraries with make (gcc)."""
    subprocess.run(["make", "-C", HERE], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def lib(flavour: str = "f1") -> C.CDLL:
    if flavour not in _LIBS:
        path = os.path.join(HERE, f"liboracle_{flavour}.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.oracle_set_params.argtypes = [C.POINTER(OracleParams), C.c_int]
        L.oracle_run_1d.argtypes = [C.POINTER(Oracle1D), C.c_int, C.POINTER(OracleParams)]
        L.oracle_stress_only_1d.argtypes = L.oracle_run_1d.argtypes
        L.oracle_stepu_only_1d.argtypes = L.oracle_run_1d.argtypes
        L.oracle_run_1d_omp.argtypes = [C.POINTER(Oracle1D), C.c_int,
                                        C.POINTER(OracleParams), C.c_int]
        L.oracle_run_1d_omp.restype = C.c_int
        L.oracle_omp_domain.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.oracle_build_index.restype = C.c_int
        L.oracle_build_index.argtypes = (
            [C.c_int, C.c_int, C.c_int, _I, C.c_int, C.c_int,
             C.POINTER(C.c_int), C.POINTER(C.c_int)] + [_I] * 9)
        L.oracle_stress_2d.argtypes = (
            [C.c_int, C.c_int, C.c_int, _I, _I] + [_D] * 12
            + [_D * 12, _D, C.POINTER(OracleParams)])
        L.oracle_stepu_2d.argtypes = (
            [C.c_int, C.c_int, C.c_int, _D, _I, _I] + [_D] * 20
            + [C.POINTER(OracleParams)])
        _LIBS[flavour] = L
    return _LIBS[flavour]


def params(ndte: int) -> OracleParams:
    p = OracleParams()
    lib().oracle_set_params(C.byref(p), int(ndte))
    return p


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def _ip(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I)


class State1D:
    """Owns contiguous copies of a Problem1D and the str scratch arrays."""

    def __init__(self, prob):
        self.na, self.navel = prob.na, prob.navel
        self.idx = {k: np.ascontiguousarray(v, dtype=np.int32) for k, v in prob.idx.items()}
        self.skipT = np.ascontiguousarray(prob.skipT, dtype=np.int32)
        self.skipU = np.ascontiguousarray(prob.skipU, dtype=np.int32)
        self.f = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in prob.f.items()}
        self.stress = np.ascontiguousarray(prob.stress, dtype=np.float64).copy()
        self.uvel = prob.uvel.astype(np.float64).copy()
        self.vvel = prob.vvel.astype(np.float64).copy()
        self.str = np.zeros((8, max(self.navel, 1)))
        self.strintx = prob.strintx.astype(np.float64).copy()
        self.strinty = prob.strinty.astype(np.float64).copy()
        self.Cb = prob.Cb.astype(np.float64).copy()
        s = Oracle1D()
        s.na, s.navel = self.na, self.navel
        for k in ("ee", "ne", "se", "nw", "sw", "sse"):
            setattr(s, k, _ip(self.idx[k]))
        s.skipT, s.skipU = _ip(self.skipT), _ip(self.skipU)
        for k in ("dxT", "dyT", "HTE", "HTN", "HTEm1", "HTNm1", "strength",
                  "Cw", "aiu", "uocn", "vocn", "waterx", "watery", "forcex",
                  "forcey", "umassdti", "fm", "uarear", "Tbu", "uvel_init",
                  "vvel_init"):
            setattr(s, k, _dp(self.f[k]))
        for k in range(12):
            s.stress[k] = self.stress[k].ctypes.data_as(_D)
        for k in range(8):
            s.str[k] = self.str[k].ctypes.data_as(_D)
        s.uvel, s.vvel = _dp(self.uvel), _dp(self.vvel)
        s.strintx, s.strinty, s.Cb = _dp(self.strintx), _dp(self.strinty), _dp(self.Cb)
        self.c = s

    def outputs(self) -> dict:
        return dict(stress=self.stress, uvel=self.uvel, vvel=self.vvel,
                    strintx=self.strintx, strinty=self.strinty, Cb=self.Cb,
                    str=self.str)


def run_1d(prob, ndte: int, p: OracleParams = None, mode: str = "fused",
           flavour: str = "f1", nthreads: int = 0, state: State1D = None) -> State1D:
    """Run the v2b 1D oracle on a copy of ``prob``.

    mode: 'fused' (serial ndte x {stress; stepu}), 'omp' (SPMD OpenMP),
    'stress' / 'stepu' (lindividual-style loops)."""
    L = lib(flavour)
    st = state if state is not None else State1D(prob)
    p = p if p is not None else params(ndte)
    if mode == "fused":
        L.oracle_run_1d(C.byref(st.c), int(ndte), C.byref(p))
    elif mode == "omp":
        L.oracle_run_1d_omp(C.byref(st.c), int(ndte), C.byref(p), int(nthreads))
    elif mode == "stress":
        L.oracle_stress_only_1d(C.byref(st.c), int(ndte), C.byref(p))
    elif mode == "stepu":
        L.oracle_stepu_only_1d(C.byref(st.c), int(ndte), C.byref(p))
    else:
        raise ValueError(mode)
    return st


def build_index(mask: np.ndarray, nghost: int = 1):
    """The adapter's index build through the C restatement.  Returns
    (na, navel, indxti, indxtj, indxtij, {ee..sse})."""
    L = lib()
    nx, ny = mask.shape
    m = np.ascontiguousarray(np.asarray(mask, dtype=np.int32).T).reshape(-1)  # F order
    cap = int(np.count_nonzero(m)) + 1
    capv = 7 * cap
    ti = np.zeros(cap, np.int32)
    tj = np.zeros(cap, np.int32)
    tij = np.zeros(capv, np.int32)
    nb = {k: np.zeros(cap, np.int32) for k in ("ee", "ne", "se", "nw", "sw", "sse")}
    na, navel = C.c_int(), C.c_int()
    rc = L.oracle_build_index(nx, ny, nghost, _ip(m), cap, capv, C.byref(na),
                              C.byref(navel), _ip(ti), _ip(tj), _ip(tij),
                              *[_ip(nb[k]) for k in ("ee", "ne", "se", "nw", "sw", "sse")])
    if rc != 0:
        raise RuntimeError(f"oracle_build_index failed: {rc}")
    n, nv = na.value, navel.value
    return n, nv, ti[:n], tj[:n], tij[:nv], {k: v[:n] for k, v in nb.items()}


def run_v0(grid, ndte: int, p: OracleParams = None) -> dict:
    """Run the v0 upstream 2D kernels (src/bench_v0.F90) for ndte subcycles on
    a copy of ``grid`` and return the 2D result fields (Fortran order).

    T list = ice T points, U list = ice U points, both j-outer / i-inner
    (the order CICE's icellt/icellu lists use).  The derived geometry arrays
    are computed as the v2 kernel derives them (src/bench_v2b.F90:139-147)."""
    L = lib()
    p = p if p is not None else params(ndte)
    nxb, nyb = grid.nxt, grid.nyt
    F = {k: np.asfortranarray(v.copy()) for k, v in grid.f.items()}
    HTE, HTN = F["HTE"], F["HTN"]
    HTEm1 = np.zeros_like(HTE)
    HTNm1 = np.zeros_like(HTN)
    HTEm1[1:, :] = HTE[:-1, :]
    HTNm1[:, 1:] = HTN[:, :-1]
    geo = {
        "cxp": 1.5 * HTN - 0.5 * HTNm1,
        "cyp": 1.5 * HTE - 0.5 * HTEm1,
        "cxm": -(1.5 * HTNm1 - 0.5 * HTN),
        "cym": -(1.5 * HTEm1 - 0.5 * HTE),
        "dxhy": 0.5 * (HTE - HTEm1),
        "dyhx": 0.5 * (HTN - HTNm1),
        "DminTarea": p.deltaminEVP * (F["dxT"] * F["dyT"]),
    }
    geo = {k: np.asfortranarray(v) for k, v in geo.items()}

    def lst(mask):
        jj, ii = np.nonzero(np.asarray(mask).T)
        return ((ii + 1).astype(np.int32), (jj + 1).astype(np.int32))

    ti, tj = lst(grid.iceT)
    ui, uj = lst(grid.iceU)

    def fp(a):
        assert a.flags.f_contiguous and a.dtype == np.float64
        return a.ctypes.data_as(_D)

    stress = [F[k] for k in (
        "stressp_1", "stressp_2", "stressp_3", "stressp_4",
        "stressm_1", "stressm_2", "stressm_3", "stressm_4",
        "stress12_1", "stress12_2", "stress12_3", "stress12_4")]
    sarr = (_D * 12)(*[fp(a) for a in stress])
    strtmp = np.zeros(nxb * nyb * 8)
    taubx = np.zeros((nxb, nyb), order="F")
    tauby = np.zeros((nxb, nyb), order="F")
    uinit, vinit = F["uvel"].copy(order="F"), F["vvel"].copy(order="F")
    for _ in range(ndte):
        L.oracle_stress_2d(nxb, nyb, ti.size, _ip(ti), _ip(tj), fp(F["uvel"]),
                           fp(F["vvel"]), fp(F["dxT"]), fp(F["dyT"]),
                           fp(geo["dxhy"]), fp(geo["dyhx"]), fp(geo["cxp"]),
                           fp(geo["cyp"]), fp(geo["cxm"]), fp(geo["cym"]),
                           fp(geo["DminTarea"]), fp(F["strength"]), sarr,
                           strtmp.ctypes.data_as(_D), C.byref(p))
        L.oracle_stepu_2d(nxb, nyb, ui.size, fp(F["Cw"]), _ip(ui), _ip(uj),
                          fp(F["aiu"]), strtmp.ctypes.data_as(_D), fp(F["uocn"]),
                          fp(F["vocn"]), fp(F["waterx"]), fp(F["watery"]),
                          fp(F["forcex"]), fp(F["forcey"]), fp(F["umassdti"]),
                          fp(F["fm"]), fp(F["uarear"]), fp(F["strintx"]),
                          fp(F["strinty"]), fp(taubx), fp(tauby), fp(uinit),
                          fp(vinit), fp(F["uvel"]), fp(F["vvel"]), fp(F["Tbu"]),
                          C.byref(p))
    F["taubx"], F["tauby"] = taubx, tauby
    F["str"] = strtmp.reshape((nxb, nyb, 8), order="F")
    return F


def output_files(stress: np.ndarray, strintx, strinty, uvel, vvel,
                 skipU: np.ndarray) -> tuple:
    """The two md5-compared output files (src/vars.F90:2233-2304):
    output_stress = 12 stress fields over the 1D list, output_stepu =
    strintx, strinty, uvel, vvel compacted over the non-skipU points."""
    na = stress.shape[1]
    keep = np.asarray(skipU[:na]) == 0
    f1 = np.ascontiguousarray(stress, dtype="<f8").tobytes()
    f2 = b"".join(np.ascontiguousarray(a[:na][keep], dtype="<f8").tobytes()
                  for a in (strintx, strinty, uvel, vvel))
    return f1, f2


def v0_output_files(grid, F2d: dict, prob) -> tuple:
    """Repack v0 2D results into the 1D output files using the 1D list of
    ``prob`` (src/vars.F90:534-584)."""
    i0, j0 = prob.indxti - 1, prob.indxtj - 1
    stress = np.stack([F2d[k][i0, j0] for k in (
        "stressp_1", "stressp_2", "stressp_3", "stressp_4",
        "stressm_1", "stressm_2", "stressm_3", "stressm_4",
        "stress12_1", "stress12_2", "stress12_3", "stress12_4")])
    return output_files(stress, F2d["strintx"][i0, j0], F2d["strinty"][i0, j0],
                        F2d["uvel"][i0, j0], F2d["vvel"][i0, j0], prob.skipU)
