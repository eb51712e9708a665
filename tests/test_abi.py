"""CPU tests of the C-ABI library: it loads, exports every function that
include/evp1d.h declares, validates its arguments before touching a GPU, and
its native index build agrees with the oracle's restatement of the adapter."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, PKG

HEADER = os.path.join(ROOT, "include", "evp1d.h")
LIB = os.path.join(PKG, "lib", "libevp1d.so")


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-C", PKG], check=True, stdout=subprocess.DEVNULL)
    from evp1d import _lib
    return _lib.load()


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(evp1d_\w+)\s*\(", txt)))


def test_header_declares_api():
    names = declared_functions()
    for must in ("evp1d_init", "evp1d_run", "evp1d_finalize", "evp1d_stress_only",
                 "evp1d_stepu_only", "evp1d_build_index", "evp1d_last_error"):
        assert must in names


def test_every_declared_symbol_exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], check=True,
                         capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (evp1d_\w+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        assert hasattr(lib, n)


def test_library_is_sm100a(lib):
    """The build names its target in the version string (the Makefile's
    -gencode arch=compute_100a,code=sm_100a); the GPU test below asks the
    CUDA runtime for the kernel's binary version."""
    assert b"sm_100a" in lib.evp1d_version()
    mk = open(os.path.join(PKG, "Makefile")).read()
    assert "-gencode arch=compute_100a,code=sm_100a" in mk


@pytest.mark.gpu
def test_kernel_binary_is_sm100(lib):
    assert lib.evp1d_binary_version(0) == 100


def test_set_evp_parameters_matches_oracle(lib, oracle_mod):
    import evp1d
    for ndte in (1, 120, 1000):
        a = evp1d.set_evp_parameters(ndte).as_dict()
        b = oracle_mod.params(ndte)
        for k, v in a.items():
            assert v == getattr(b, k), (ndte, k)


def _init(lib, na, navel, idx, geo, params=None, device=0):
    import evp1d
    h = C.c_void_p()
    P = C.POINTER(C.c_int32)
    D = C.POINTER(C.c_double)
    params = params or evp1d.set_evp_parameters(10)
    rc = lib.evp1d_init(C.byref(h), na, navel,
                        *[None if a is None else a.ctypes.data_as(P) for a in idx],
                        *[None if a is None else a.ctypes.data_as(D) for a in geo],
                        C.byref(params), device)
    return rc, h


def test_init_rejects_bad_index_before_gpu(lib):
    na, navel = 4, 6
    ok = np.array([1, 2, 5, 6], np.int32)
    bad = np.array([1, 2, 7, 6], np.int32)   # 7 > navel
    zero = np.array([0, 2, 3, 4], np.int32)  # 0 is not a 1-based slot
    geo = [np.ones(na)] * 7
    rc, h = _init(lib, na, navel, [ok, ok, bad, ok, ok, ok], geo)
    assert rc == -2 and not h.value
    assert b"se(3) = 7" in lib.evp1d_last_error()
    rc, h = _init(lib, na, navel, [zero, ok, ok, ok, ok, ok], geo)
    assert rc == -2


def test_init_rejects_bad_sizes_and_nulls(lib):
    geo = [np.ones(3)] * 7
    ok = np.array([1, 2, 3], np.int32)
    rc, _ = _init(lib, 3, 2, [ok] * 6, geo)          # navel < na
    assert rc == -1
    rc, _ = _init(lib, 3, 3, [ok] * 5 + [None], geo)  # NULL neighbour vector
    assert rc == -1
    rc, _ = _init(lib, 3, 3, [ok] * 6, geo[:6] + [None])
    assert rc == -1
    assert lib.evp1d_init(None, 0, 0, *([None] * 13), None, 0) == -1


def test_null_handle_calls(lib):
    assert lib.evp1d_run(None, 1, None) == -1
    assert lib.evp1d_subcycles(None, 1) == -1
    assert lib.evp1d_stress_only(None, 1) == -1
    assert lib.evp1d_finalize(None) == 0
    assert lib.evp1d_launch_count(None, 0) == -1


@pytest.mark.parametrize("shape,frac,seed", [((40, 30), 0.6, 0), ((70, 21), 0.95, 5),
                                             ((5, 5), 0.0, 1)])
def test_native_index_build_matches_oracle(lib, oracle_mod, shape, frac, seed):
    import evp1d
    rng = np.random.default_rng(seed)
    mask = rng.random(shape) < frac
    mask[0, :] = mask[:, 0] = False
    got = evp1d.build_index(mask)
    want = oracle_mod.build_index(mask)
    assert got[0] == want[0] and got[1] == want[1]
    for a, b in zip(got[2:5], want[2:5]):
        assert np.array_equal(a, b)
    for k in want[5]:
        assert np.array_equal(got[5][k], want[5][k]), k


def test_native_index_build_capacity_error(lib):
    mask = np.ones((6, 6), np.int32)
    mask[0, :] = mask[:, 0] = 0
    m = np.ascontiguousarray(mask.T).reshape(-1)
    na, navel = C.c_int(), C.c_int()
    P = C.POINTER(C.c_int32)
    small = np.zeros(3, np.int32)
    rc = lib.evp1d_build_index(6, 6, 1, m.ctypes.data_as(P), 3, 3, C.byref(na),
                               C.byref(navel), *[small.ctypes.data_as(P)] * 9)
    assert rc == -1 and na.value == 25 and navel.value > 25


def test_header_compiles_as_c_and_layouts_match_bindings(lib, tmp_path):
    """A C99 caller of include/evp1d.h sees the struct layouts the Python
    binding uses, and host-only calls work from C."""
    import ctypes
    from evp1d import _lib
    from evp1d.dyn import DynFields
    exe = str(tmp_path / "abi_layout")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "native", "abi_layout.c"), "-o", exe,
                    "-L", os.path.dirname(LIB), "-levp1d",
                    "-Wl,-rpath," + os.path.dirname(LIB)], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    got = dict(line.rsplit(" ", 1) for line in out.strip().splitlines())
    py = {"evp1d_params": _lib.Params, "evp1d_fields": _lib.Fields,
          "evp1d_grads": _lib.Grads, "evp1d_dyn_fields": DynFields}
    for key, val in got.items():
        if "." in key:
            t, m = key.split(".")
            assert getattr(py[t], m).offset == int(val), key
        elif key in py:
            assert ctypes.sizeof(py[key]) == int(val), key
    assert got["brlx"] == "120.0"
    assert got["run_null"] == "-1,1"  # EVP1D_ERR_INVALID_ARG and a message
    assert got["version"] == "1"
