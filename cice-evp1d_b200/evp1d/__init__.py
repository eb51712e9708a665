"""evp1d -- host-side interface of the B200 EVP-1D sea-ice dynamics solver.

Mirrors the reference's evp1d interface (dmidk/cice-evp1d):

* :func:`set_evp_parameters` -- ``set_evp_parameters`` (src/ice.F90:109-130);
* :func:`build_index` -- the 1D index space of ``dyn_evp1d_init``
  (integration/ice_dyn_evp1d.F90:559-589, 743-816);
* :class:`EVP1D` -- ``dyn_evp1d_init`` / ``dyn_evp1d_run`` /
  ``dyn_evp1d_finalize`` on the 1D layout, plus the ``lindividual``
  stress-only / stepu-only loops (src/evp_v2b.F90:127-155).

Every call goes through libevp1d.so (include/evp1d.h); the CUDA kernels are the
only compute path.
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _lib
from ._lib import EVP1DError, Fields, Params, check

__all__ = ["EVP1D", "EVP1DError", "Params", "set_evp_parameters",
           "build_index", "FieldSet", "version"]

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int32)


def version() -> str:
    return _lib.load().evp1d_version().decode()


def set_evp_parameters(ndte: int) -> Params:
    p = Params()
    _lib.load().evp1d_set_evp_parameters(C.byref(p), int(ndte))
    return p


def _d(a):
    return None if a is None else a.ctypes.data_as(_D)


def pinned_empty(shape, dtype=np.float64) -> np.ndarray:
    """A numpy array in page-locked host memory (evp1d_host_alloc), freed
    when the array is garbage collected."""
    L = _lib.load()
    count = int(np.prod(shape))
    nbytes = max(count * np.dtype(dtype).itemsize, 1)
    p = C.c_void_p()
    check(L.evp1d_host_alloc(C.byref(p), nbytes), "evp1d_host_alloc")
    buf = (C.c_char * nbytes).from_address(p.value)
    weakref.finalize(buf, L.evp1d_host_free, C.c_void_p(p.value))
    return np.frombuffer(buf, dtype=dtype, count=count).reshape(shape)


def pinned_copy(a) -> np.ndarray:
    """A page-locked copy of `a`."""
    a = np.asarray(a)
    out = pinned_empty(a.shape, a.dtype)
    out[...] = a
    return out


def _as_f64(a, n, name):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != (n,):
        raise ValueError(f"{name}: expected shape ({n},), got {a.shape}")
    return a


def _as_i32(a, n, name):
    a = np.ascontiguousarray(a, dtype=np.int32)
    if a.shape != (n,):
        raise ValueError(f"{name}: expected shape ({n},), got {a.shape}")
    return a


def build_index(mask: np.ndarray, nghost: int = 1):
    """1D list, halo slots and neighbour vectors of ``mask`` ([nx, ny], True =
    list point) through the library's native index build.  Returns
    ``(na, navel, indxti, indxtj, indxtij, {'ee','ne','se','nw','sw','sse'})``
    with 1-based values."""
    L = _lib.load()
    nx, ny = mask.shape
    m = np.ascontiguousarray(np.asarray(mask, dtype=np.int32).T).reshape(-1)
    na, navel = C.c_int(), C.c_int()
    rc = L.evp1d_build_index(nx, ny, nghost, m.ctypes.data_as(_I), 0, 0,
                             C.byref(na), C.byref(navel), *([None] * 9))
    if rc != 0 and na.value == 0 and navel.value == 0:
        check(rc, "evp1d_build_index")
    n, nv = na.value, navel.value
    ti = np.zeros(max(n, 1), np.int32)
    tj = np.zeros(max(n, 1), np.int32)
    tij = np.zeros(max(nv, 1), np.int32)
    nb = {k: np.zeros(max(n, 1), np.int32) for k in ("ee", "ne", "se", "nw", "sw", "sse")}
    rc = L.evp1d_build_index(nx, ny, nghost, m.ctypes.data_as(_I), n, nv,
                             C.byref(na), C.byref(navel),
                             ti.ctypes.data_as(_I), tj.ctypes.data_as(_I),
                             tij.ctypes.data_as(_I),
                             *[nb[k].ctypes.data_as(_I) for k in ("ee", "ne", "se", "nw", "sw", "sse")])
    check(rc, "evp1d_build_index")
    return n, nv, ti[:n], tj[:n], tij[:nv], {k: v[:n] for k, v in nb.items()}


def set_tile_points(points: int) -> None:
    """Largest tile (list points, 32..256) of the plans of handles created
    from now on (evp1d_set_tile_points); results do not depend on it."""
    check(_lib.load().evp1d_set_tile_points(int(points)), "evp1d_set_tile_points")


def get_tile_points() -> int:
    return int(_lib.load().evp1d_get_tile_points())


def tune_tile_points(prob, candidates=(256, 224, 192, 160, 128), nsub: int = 20,
                     device: int = 0) -> tuple:
    """The autotuner's tile-size dimension: for each candidate, build a handle
    planned with that largest tile for `prob` (a Problem1D, or an Ensemble for
    a batched handle), upload its fields and time `nsub` subcycles (best of
    two).  Leaves the fastest size set for later handles and returns
    (best, {points: microseconds per subcycle})."""
    import time
    batched = hasattr(prob, "combined")
    times = {}
    for n in candidates:
        set_tile_points(n)
        if batched:
            s = EVP1D.batched(prob, device=device)
            fs = FieldSet.from_problem(prob.combined)
        else:
            s = EVP1D.from_problem(prob, device=device)
            fs = FieldSet.from_problem(prob)
        with s:
            s.upload(fs)
            s.subcycles(2)
            s.synchronize()
            best = float("inf")
            for _ in range(2):
                t0 = time.perf_counter()
                s.subcycles(nsub)
                s.synchronize()
                best = min(best, time.perf_counter() - t0)
        times[int(n)] = best / nsub * 1e6
    pick = min(times, key=times.get)
    set_tile_points(pick)
    return pick, times


def debug_fail_alloc(n: int) -> None:
    """Host-side fault injection (evp1d_debug_fail_alloc): the n-th device
    allocation of the library from now on fails as out of memory; 0 disarms."""
    check(_lib.load().evp1d_debug_fail_alloc(int(n)), "evp1d_debug_fail_alloc")


def plan_check(na: int, navel: int, idx: dict) -> None:
    """Build the tile plan for these 1-based neighbour vectors and verify
    every index the kernels gather through (evp1d_plan_check; host only).
    Raises EVP1DError (EVP1D_ERR_INDEX) naming the first violation."""
    L = _lib.load()
    n = C.c_longlong(0)
    arrs = [_as_i32(idx[k], na, k) for k in ("ee", "ne", "se", "nw", "sw", "sse")]
    check(L.evp1d_plan_check(int(na), int(navel), *[a.ctypes.data_as(_I) for a in arrs],
                             C.byref(n)), "evp1d_plan_check")


def plan_stats(na: int, navel: int, idx: dict) -> dict:
    """Tile plan the solver builds for these 1-based neighbour vectors (host
    only, no GPU)."""
    L = _lib.load()
    st = (C.c_longlong * 8)()
    arrs = [_as_i32(idx[k], na, k) for k in ("ee", "ne", "se", "nw", "sw", "sse")]
    check(L.evp1d_plan_stats(int(na), int(navel), *[a.ctypes.data_as(_I) for a in arrs], st),
          "evp1d_plan_stats")
    return dict(tiles=st[0], slots=st[1], halo=st[2], from_coords=bool(st[3]),
                max_halo=st[4], max_tile=st[5], max_extras=st[6], max_run_tiles=st[7])


class FieldSet:
    """Host arrays of one dyn_evp1d_run call (evp1d_fields), kept alive while
    the ctypes struct points at them.  Arrays are updated in place by
    :meth:`EVP1D.run` / :meth:`EVP1D.download`."""

    DYN = ("strength", "Cw", "aiu", "uocn", "vocn", "waterx", "watery",
           "forcex", "forcey", "umassdti", "fm", "Tbu")

    def __init__(self, na: int, navel: int, *, skipT, skipU, stress, uvel,
                 vvel, strintx, strinty, Cb, uvel_init=None, vvel_init=None,
                 want_str: bool = False, **dyn):
        self.na, self.navel = na, navel
        self.skipT = _as_i32(skipT, na, "skipT")
        self.skipU = _as_i32(skipU, na, "skipU")
        stress = np.ascontiguousarray(stress, dtype=np.float64)
        if stress.shape != (12, na):
            raise ValueError(f"stress: expected (12, {na}), got {stress.shape}")
        self.stress = stress
        self.dyn = {k: _as_f64(dyn[k], na, k) for k in self.DYN}
        self.uvel = _as_f64(uvel, navel, "uvel")
        self.vvel = _as_f64(vvel, navel, "vvel")
        self.strintx = _as_f64(strintx, na, "strintx")
        self.strinty = _as_f64(strinty, na, "strinty")
        self.Cb = _as_f64(Cb, na, "Cb")
        self.uvel_init = None if uvel_init is None else _as_f64(uvel_init, na, "uvel_init")
        self.vvel_init = None if vvel_init is None else _as_f64(vvel_init, na, "vvel_init")
        self.str = np.zeros((8, navel)) if want_str else None
        f = Fields()
        f.skipT = self.skipT.ctypes.data_as(_I)
        f.skipU = self.skipU.ctypes.data_as(_I)
        for k in range(12):
            f.stress[k] = self.stress[k].ctypes.data_as(_D)
        for k in self.DYN:
            setattr(f, k, _d(self.dyn[k]))
        f.uvel_init = _d(self.uvel_init)
        f.vvel_init = _d(self.vvel_init)
        f.uvel, f.vvel = _d(self.uvel), _d(self.vvel)
        f.strintx, f.strinty, f.Cb = _d(self.strintx), _d(self.strinty), _d(self.Cb)
        for k in range(8):
            f.str[k] = self.str[k].ctypes.data_as(_D) if self.str is not None else None
        self.c = f

    @classmethod
    def from_problem(cls, prob, want_str: bool = False, copy: bool = True,
                     explicit_init: bool = False, pinned: bool = False) -> "FieldSet":
        """Fields of a :class:`evp1d.synth.Problem1D` (copied by default;
        into page-locked memory with ``pinned``)."""
        if pinned:
            cp = pinned_copy
        else:
            cp = (lambda a: np.array(a, copy=True)) if copy else (lambda a: a)
        dyn = {k: cp(prob.f[k]) for k in cls.DYN}
        return cls(prob.na, prob.navel, skipT=prob.skipT, skipU=prob.skipU,
                   stress=cp(prob.stress), uvel=cp(prob.uvel),
                   vvel=cp(prob.vvel), strintx=cp(prob.strintx),
                   strinty=cp(prob.strinty), Cb=cp(prob.Cb),
                   uvel_init=cp(prob.f["uvel_init"]) if explicit_init else None,
                   vvel_init=cp(prob.f["vvel_init"]) if explicit_init else None,
                   want_str=want_str, **dyn)

    def refill(self, prob) -> None:
        """Copy a problem's starting state and per-call fields into this
        set's arrays (keeping their memory, e.g. page-locked)."""
        self.stress[...] = prob.stress
        self.uvel[...] = prob.uvel
        self.vvel[...] = prob.vvel
        self.strintx[...] = prob.strintx
        self.strinty[...] = prob.strinty
        self.Cb[...] = prob.Cb
        self.skipT[...] = prob.skipT
        self.skipU[...] = prob.skipU
        for k in self.DYN:
            self.dyn[k][...] = prob.f[k]


class EVP1D:
    """One 1D EVP problem resident on a GPU (dyn_evp1d_init ... finalize)."""

    def __init__(self, na: int, navel: int, *, ee, ne, se, nw, sw, sse, dxT,
                 dyT, HTE, HTN, HTEm1, HTNm1, uarear, params: Params = None,
                 ndte: int = None, device: int = 0):
        L = _lib.load()
        self._L = L
        self.na, self.navel = int(na), int(navel)
        if params is None:
            if ndte is None:
                raise ValueError("give params or ndte")
            params = set_evp_parameters(ndte)
        self.params = params
        idx = [_as_i32(a, na, n) for a, n in
               ((ee, "ee"), (ne, "ne"), (se, "se"), (nw, "nw"), (sw, "sw"), (sse, "sse"))]
        geo = [_as_f64(a, na, n) for a, n in
               ((dxT, "dxT"), (dyT, "dyT"), (HTE, "HTE"), (HTN, "HTN"),
                (HTEm1, "HTEm1"), (HTNm1, "HTNm1"), (uarear, "uarear"))]
        h = C.c_void_p()
        rc = L.evp1d_init(C.byref(h), self.na, self.navel,
                          *[a.ctypes.data_as(_I) for a in idx],
                          *[a.ctypes.data_as(_D) for a in geo],
                          C.byref(params), int(device))
        check(rc, "evp1d_init")
        self.h = h

    @classmethod
    def batched(cls, ens, ndte: int = None, params: Params = None,
                device: int = 0) -> "EVP1D":
        """An ensemble handle (evp1d_init_batched) for a
        :class:`evp1d.synth.Ensemble`; FieldSets for it are built from
        ``ens.combined``."""
        L = _lib.load()
        pr = ens.combined
        if params is None:
            params = set_evp_parameters(ndte if ndte is not None else pr.ndte)
        f = pr.f
        idx = [_as_i32(pr.idx[k], pr.na, k) for k in ("ee", "ne", "se", "nw", "sw", "sse")]
        geo = [_as_f64(f[k], pr.na, k) for k in ("dxT", "dyT", "HTE", "HTN", "HTEm1", "HTNm1", "uarear")]
        na = np.ascontiguousarray(ens.na, dtype=np.int32)
        navel = np.ascontiguousarray(ens.navel, dtype=np.int32)
        h = C.c_void_p()
        rc = L.evp1d_init_batched(C.byref(h), len(na), na.ctypes.data_as(_I),
                                  navel.ctypes.data_as(_I),
                                  *[a.ctypes.data_as(_I) for a in idx],
                                  *[a.ctypes.data_as(_D) for a in geo],
                                  C.byref(params), int(device))
        check(rc, "evp1d_init_batched")
        self = cls.__new__(cls)
        self._L, self.h, self.params = L, h, params
        self.na, self.navel = pr.na, pr.navel
        return self

    def autotune(self, nsub: int = 20) -> str:
        """Pick the fastest kernel variant on the uploaded state
        (evp1d_autotune); returns the choice."""
        buf = C.create_string_buffer(128)
        check(self._L.evp1d_autotune(self.h, int(nsub), buf, 128), "evp1d_autotune")
        return buf.value.decode()

    @classmethod
    def from_problem(cls, prob, ndte: int = None, params: Params = None,
                     device: int = 0) -> "EVP1D":
        f = prob.f
        return cls(prob.na, prob.navel, **prob.idx, dxT=f["dxT"], dyT=f["dyT"],
                   HTE=f["HTE"], HTN=f["HTN"], HTEm1=f["HTEm1"],
                   HTNm1=f["HTNm1"], uarear=f["uarear"], params=params,
                   ndte=ndte if ndte is not None else prob.ndte, device=device)

    # -- dyn_evp1d_run -----------------------------------------------------
    def run(self, ndte: int, fields: FieldSet) -> FieldSet:
        check(self._L.evp1d_run(self.h, int(ndte), C.byref(fields.c)), "evp1d_run")
        return fields

    def upload(self, fields: FieldSet) -> None:
        check(self._L.evp1d_upload(self.h, C.byref(fields.c)), "evp1d_upload")

    def subcycles(self, ndte: int) -> None:
        check(self._L.evp1d_subcycles(self.h, int(ndte)), "evp1d_subcycles")

    def subcycles_inner(self, n: int) -> None:
        """Subcycles that do not end the call (evp1d_subcycles_inner): the
        state advances, strintx/strinty/Cb/str are not written."""
        check(self._L.evp1d_subcycles_inner(self.h, int(n)), "evp1d_subcycles_inner")

    def download(self, fields: FieldSet) -> FieldSet:
        check(self._L.evp1d_download(self.h, C.byref(fields.c)), "evp1d_download")
        return fields

    # -- lindividual -------------------------------------------------------
    def stress_only(self, n: int) -> None:
        check(self._L.evp1d_stress_only(self.h, int(n)), "evp1d_stress_only")

    def stepu_only(self, n: int) -> None:
        check(self._L.evp1d_stepu_only(self.h, int(n)), "evp1d_stepu_only")

    # -- adjoint ----------------------------------------------------------
    GRADS = ("strength", "Cw", "forcex", "forcey", "uvel", "vvel")

    def run_checkpointed(self, ndte: int, fields: FieldSet, interval: int = 0) -> FieldSet:
        """evp1d_run that also records what :meth:`adjoint` needs (interval > 0:
        checkpoints every `interval` subcycles; 0: sized to device memory)."""
        check(self._L.evp1d_run_checkpointed(self.h, int(ndte), C.byref(fields.c),
                                             int(interval)), "evp1d_run_checkpointed")
        return fields

    def record_subcycles(self, ndte: int, interval: int = 0) -> None:
        check(self._L.evp1d_record_subcycles(self.h, int(ndte), int(interval)),
              "evp1d_record_subcycles")

    def _lam_stress(self, lam_stress):
        if lam_stress is None:
            return None, None
        ls = np.ascontiguousarray(lam_stress, dtype=np.float64)
        if ls.shape != (12, self.na):
            raise ValueError(f"lam_stress: expected (12, {self.na})")
        arr = (_D * 12)(*[ls[k].ctypes.data_as(_D) for k in range(12)])
        return ls, arr

    def adjoint_seed(self, lam_u, lam_v, lam_stress=None) -> None:
        lu = _as_f64(lam_u, self.na, "lam_u")
        lv = _as_f64(lam_v, self.na, "lam_v")
        keep, arr = self._lam_stress(lam_stress)
        check(self._L.evp1d_adjoint_seed(self.h, _d(lu), _d(lv), arr), "evp1d_adjoint_seed")

    def adjoint_sweep(self) -> None:
        check(self._L.evp1d_adjoint_sweep(self.h), "evp1d_adjoint_sweep")

    def adjoint_gradients(self, want=GRADS, stress: bool = False,
                          init: bool = False) -> dict:
        out = {k: np.zeros(self.na) for k in want}
        g = _lib.Grads()
        for k, a in out.items():
            setattr(g, k, _d(a))
        if stress:
            out["stress"] = np.zeros((12, self.na))
            for k in range(12):
                g.stress[k] = out["stress"][k].ctypes.data_as(_D)
        if init:
            out["uvel_init"] = np.zeros(self.na)
            out["vvel_init"] = np.zeros(self.na)
            g.uvel_init, g.vvel_init = _d(out["uvel_init"]), _d(out["vvel_init"])
        check(self._L.evp1d_adjoint_gradients(self.h, C.byref(g)), "evp1d_adjoint_gradients")
        return out

    def adjoint(self, lam_u, lam_v, lam_stress=None, want=GRADS, stress: bool = False,
                init: bool = False) -> dict:
        """Gradients of J from dJ/d(final uvel, vvel) [na] (and optionally
        dJ/d(final stresses) [12, na]) for the last recorded forward."""
        self.adjoint_seed(lam_u, lam_v, lam_stress)
        self.adjoint_sweep()
        return self.adjoint_gradients(want, stress=stress, init=init)

    def adjoint_info(self) -> dict:
        info = (C.c_longlong * 8)()
        check(self._L.evp1d_adjoint_info(self.h, info), "evp1d_adjoint_info")
        keys = ("valid", "tape_subcycles", "interval", "checkpoints", "store_bytes",
                "work_bytes", "solver_bytes", "sweep_launches")
        return {k: int(v) for k, v in zip(keys, info)}

    def set_adjoint_budget(self, nbytes: int) -> None:
        """Device memory for the checkpoints and tape of sized recordings
        (interval 0); 0 = 80% of the free memory."""
        check(self._L.evp1d_set_adjoint_budget(self.h, int(nbytes)),
              "evp1d_set_adjoint_budget")

    def set_params(self, params: Params) -> None:
        check(self._L.evp1d_set_params(self.h, C.byref(params)), "evp1d_set_params")
        self.params = params

    def synchronize(self) -> None:
        check(self._L.evp1d_synchronize(self.h), "evp1d_synchronize")

    def debug_wait_timeout(self, ns: int) -> None:
        """Queue one bounded wait that runs out after ns nanoseconds
        (evp1d_debug_wait_timeout): the next synchronize raises the timeout."""
        check(self._L.evp1d_debug_wait_timeout(self.h, int(ns)), "evp1d_debug_wait_timeout")

    def debug_dep_wait_timeout(self, ns: int) -> None:
        """Queue one bounded wait of the multi-subcycle launch's kind, on a
        counter nothing raises (evp1d_debug_dep_wait_timeout): the next
        synchronize raises the timeout."""
        check(self._L.evp1d_debug_dep_wait_timeout(self.h, int(ns)),
              "evp1d_debug_dep_wait_timeout")

    @property
    def path(self) -> str:
        """Name of the kernel path the library runs."""
        return self._L.evp1d_kernel_path(self.h).decode()

    @property
    def stream(self) -> int:
        return self._L.evp1d_stream(self.h) or 0

    # -- a state split over handles (evp1d.bands) ---------------------------
    def exchange_setup(self, send_idx, recv_idx) -> None:
        """Velocity-exchange lists (evp1d_exchange_setup): 1-based local list
        points whose u, v are sent, and 1-based local positions that receive."""
        si = np.ascontiguousarray(send_idx, dtype=np.int32)
        ri = np.ascontiguousarray(recv_idx, dtype=np.int32)
        check(self._L.evp1d_exchange_setup(self.h, len(si), si.ctypes.data_as(_I), len(ri),
                                           ri.ctypes.data_as(_I)), "evp1d_exchange_setup")

    def exchange_pack(self, dev_ptr: int = 0) -> None:
        """u, v pairs of the sent points into a device buffer (0: the
        handle's own send buffer), on the handle's stream."""
        check(self._L.evp1d_exchange_pack(self.h, C.c_void_p(int(dev_ptr) or None)),
              "evp1d_exchange_pack")

    def exchange_unpack(self, dev_ptr: int = 0) -> None:
        """u, v pairs from a device buffer (0: the handle's own receive
        buffer) into the received positions."""
        check(self._L.evp1d_exchange_unpack(self.h, C.c_void_p(int(dev_ptr) or None)),
              "evp1d_exchange_unpack")

    def exchange_buffers(self) -> tuple:
        """Device addresses (send, receive) of the handle's own exchange
        buffers; 0 where a list is empty."""
        snd, rcv = C.c_void_p(), C.c_void_p()
        check(self._L.evp1d_exchange_buffers(self.h, C.byref(snd), C.byref(rcv)),
              "evp1d_exchange_buffers")
        return snd.value or 0, rcv.value or 0

    def launch_count(self, reset: bool = False) -> int:
        return int(self._L.evp1d_launch_count(self.h, 1 if reset else 0))

    def finalize(self) -> None:
        if getattr(self, "h", None):
            check(self._L.evp1d_finalize(self.h), "evp1d_finalize")
            self.h = None

    def __del__(self):
        try:
            self.finalize()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.finalize()
