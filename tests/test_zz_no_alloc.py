"""GPU tests of evp1d_run_device_noalloc, the allocation-free entry point.

The caller owns every device buffer (torch allocates them here, outside the
call); the library call itself allocates nothing.  Its results must be bitwise
equal to evp1d_run's on the same inputs, over two calls in a row on the same
arrays (the second starts from the first's state, and the shared scratch still
holds the first call's str1..str8).  The file is collected last so that it
runs both alone and after every other GPU test.
"""
import ctypes as C

import numpy as np
import pytest

import evp1d
from evp1d import _lib, synth

pytestmark = pytest.mark.gpu

MAX_NAVEL = 262144  # EVP1D_NOALLOC_MAX_NAVEL (include/evp1d.h)


def _dp(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))


def _ip(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_int32))


class DeviceCase:
    """One problem's arrays in device memory, in the reference 1D layout."""

    GEO = ("dxT", "dyT", "HTE", "HTN", "HTEm1", "HTNm1", "uarear")

    def __init__(self, pr, explicit_init=False, want_str=True):
        import torch
        dev = torch.device("cuda", 0)
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self.pr = pr
        self.nb = {k: T(pr.idx[k].astype(np.int32)) for k in ("ee", "ne", "se", "nw", "sw", "sse")}
        self.geo = {k: T(pr.f[k]) for k in self.GEO}
        self.skipT, self.skipU = T(pr.skipT.astype(np.int32)), T(pr.skipU.astype(np.int32))
        self.stress = T(pr.stress.copy())
        self.dyn = {k: T(pr.f[k]) for k in evp1d.FieldSet.DYN}
        self.uvel, self.vvel = T(pr.uvel.copy()), T(pr.vvel.copy())
        self.strintx, self.strinty, self.Cb = T(pr.strintx.copy()), T(pr.strinty.copy()), T(pr.Cb.copy())
        self.uinit = T(pr.f["uvel_init"]) if explicit_init else None
        self.vinit = T(pr.f["vvel_init"]) if explicit_init else None
        self.str = torch.full((8, pr.navel), 7.0, dtype=torch.float64, device=dev) if want_str else None
        f = _lib.Fields()
        f.skipT, f.skipU = _ip(self.skipT), _ip(self.skipU)
        for k in range(12):
            f.stress[k] = _dp(self.stress[k])
        for k in evp1d.FieldSet.DYN:
            setattr(f, k, _dp(self.dyn[k]))
        f.uvel_init = _dp(self.uinit) if explicit_init else None
        f.vvel_init = _dp(self.vinit) if explicit_init else None
        f.uvel, f.vvel = _dp(self.uvel), _dp(self.vvel)
        f.strintx, f.strinty, f.Cb = _dp(self.strintx), _dp(self.strinty), _dp(self.Cb)
        for k in range(8):
            f.str[k] = _dp(self.str[k]) if want_str else None
        self.c = f

    def run(self, ndte, params, na=None, navel=None, stream=None):
        import torch
        L = _lib.load()
        nb = [C.c_void_p(self.nb[k].data_ptr()) for k in ("ee", "ne", "se", "nw", "sw", "sse")]
        geo = [C.c_void_p(self.geo[k].data_ptr()) for k in self.GEO]
        st = torch.cuda.current_stream().cuda_stream if stream is None else stream
        return L.evp1d_run_device_noalloc(
            self.pr.na if na is None else na, self.pr.navel if navel is None else navel,
            *nb, *geo, C.byref(params), int(ndte), C.byref(self.c), C.c_void_p(st))

    def host(self):
        return dict(stress=self.stress.cpu().numpy(), uvel=self.uvel.cpu().numpy(),
                    vvel=self.vvel.cpu().numpy(), strintx=self.strintx.cpu().numpy(),
                    strinty=self.strinty.cpu().numpy(), Cb=self.Cb.cpu().numpy(),
                    str=None if self.str is None else self.str.cpu().numpy())


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def _assert_same(dev, fs, check_str=True):
    want = dict(stress=fs.stress, uvel=fs.uvel, vvel=fs.vvel, strintx=fs.strintx,
                strinty=fs.strinty, Cb=fs.Cb)
    for k, w in want.items():
        assert np.array_equal(_bits(dev[k]), _bits(w)), k
    if check_str:
        assert np.array_equal(_bits(dev["str"]), _bits(fs.str)), "str"


@pytest.mark.parametrize("explicit_init", [False, True])
def test_two_calls_match_evp1d_run(explicit_init):
    pr = synth.make_problem("grid400x300", nx=150, ny=110, ndte=17)
    assert pr.navel <= MAX_NAVEL
    ndte = pr.ndte
    params = evp1d.set_evp_parameters(ndte)
    fs = evp1d.FieldSet.from_problem(pr, want_str=True, explicit_init=explicit_init)
    dc = DeviceCase(pr, explicit_init=explicit_init)
    with evp1d.EVP1D.from_problem(pr, ndte=ndte) as s:
        for call in range(2):
            s.run(ndte, fs)
            _lib.check(dc.run(ndte, params), "evp1d_run_device_noalloc")
            _assert_same(dc.host(), fs)
    # the state moved: the second call did work
    assert not np.array_equal(fs.stress, pr.stress)


@pytest.mark.parametrize("explicit_init", [False, True])
def test_two_calls_match_the_oracle(oracle_mod, explicit_init):
    """The same two calls against the CPU oracle directly, bit for bit, with
    both reference output files md5-equal after each call."""
    from test_gpu_parity import assert_same, oracle_run
    pr = synth.make_problem("grid400x300", nx=140, ny=100, ndte=23)
    assert pr.navel <= MAX_NAVEL
    ndte = pr.ndte
    params = evp1d.set_evp_parameters(ndte)
    dc = DeviceCase(pr, explicit_init=explicit_init)
    cur = pr.copy()
    for call in range(2):
        _lib.check(dc.run(ndte, params), "evp1d_run_device_noalloc")
        st = oracle_run(oracle_mod, cur, ndte)
        got = dc.host()
        fs = evp1d.FieldSet.from_problem(cur, want_str=True)
        fs.stress[:], fs.strintx[:], fs.strinty[:], fs.Cb[:] = (
            got["stress"], got["strintx"], got["strinty"], got["Cb"])
        fs.uvel[:], fs.vvel[:], fs.str[:] = got["uvel"], got["vvel"], got["str"]
        assert_same(fs, st, cur)
        # the next call starts from this one's state; without explicit
        # uvel_init it also starts its uvel_init there
        cur = cur.copy()
        cur.stress[:] = st.stress
        cur.uvel[:] = st.uvel[: pr.navel]
        cur.vvel[:] = st.vvel[: pr.navel]
        cur.strintx[:], cur.strinty[:], cur.Cb[:] = st.strintx, st.strinty, st.Cb
        if not explicit_init:
            cur.f["uvel_init"] = st.uvel[: pr.na].copy()
            cur.f["vvel_init"] = st.vvel[: pr.na].copy()
    assert not np.array_equal(cur.uvel[: pr.na], pr.uvel[: pr.na])


def test_other_sizes_between_calls():
    """A smaller problem after a larger one: the shared scratch is cleared."""
    big = synth.make_problem("grid400x300", nx=90, ny=70, ndte=6)
    small = synth.to_1d(synth.make_grid(41, 29, seed=11, ndte=6, curvilinear=True))
    for pr in (big, small, big):
        params = evp1d.set_evp_parameters(pr.ndte)
        fs = evp1d.FieldSet.from_problem(pr, want_str=True)
        with evp1d.EVP1D.from_problem(pr, ndte=pr.ndte) as s:
            s.run(pr.ndte, fs)
        dc = DeviceCase(pr)
        _lib.check(dc.run(pr.ndte, params), "evp1d_run_device_noalloc")
        _assert_same(dc.host(), fs)


def test_rejects_oversize_and_bad_input():
    pr = synth.to_1d(synth.make_grid(30, 20, seed=5, ndte=3))
    params = evp1d.set_evp_parameters(3)
    dc = DeviceCase(pr)
    before = dc.host()
    L = _lib.load()
    rc = dc.run(3, params, navel=MAX_NAVEL + 1)
    assert rc == -1 and b"EVP1D_NOALLOC_MAX_NAVEL" in L.evp1d_last_error()
    # a neighbour outside 1..navel: rejected before any array is written
    dc.nb["sw"][pr.na // 2] = pr.navel + 1
    assert dc.run(3, params) == -2
    after = dc.host()
    for k in ("stress", "uvel", "vvel", "strintx", "strinty", "Cb"):
        assert np.array_equal(_bits(after[k]), _bits(before[k])), k
    dc.nb["sw"][pr.na // 2] = int(pr.idx["sw"][pr.na // 2])
    # a host pointer where device memory is required
    host_u = np.zeros(pr.navel)
    dc.c.uvel = host_u.ctypes.data_as(C.POINTER(C.c_double))
    assert dc.run(3, params) == -1
    assert b"uvel" in L.evp1d_last_error()
    dc.c.uvel = _dp(dc.uvel)
    rc = dc.run(3, params)
    assert rc == 0, L.evp1d_last_error()
