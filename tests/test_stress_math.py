"""CPU unit tests of the straight-line stress path.

The TMA kernel runs stress_update_std (cice-evp1d_b200/csrc/evp_math.cuh)
when the parameters allow it (std_params: capping = 1, Ktens = 0, revp = 0,
finite arlx1i).  It must give the very bits of the general stress_update
(src/bench_v2b.F90:170-310) on every input: here both are compiled for the
host (tests/native/stress_math_shim.cpp, no FMA contraction) and compared bit
for bit on random points and on the inputs that send stress_update_std to its
fallback: NaN strain rates, strength at or above 1e300*DminArea, a zero
deltaminEVP, zero and negative strength, zero velocities."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, PKG

SHIM = os.path.join(ROOT, "tests", "native", "stress_math_shim.cpp")
FIELDS = ("arlx1i", "denom1", "brlx", "capping", "e_factor", "epp2i",
          "deltaminEVP", "revp", "Ktens", "u0", "cosw", "sinw", "rhow")


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("shim") / "stress_math_shim.so")
    subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-ffp-contract=off",
                    "-I", os.path.join(PKG, "csrc"), "-I", os.path.join(ROOT, "include"),
                    "-I", "/usr/local/cuda/include", SHIM, "-o", out], check=True)
    L = C.CDLL(out)
    D = C.POINTER(C.c_double)
    L.shim_std_params.argtypes = [D]
    L.shim_std_params.restype = C.c_int
    L.shim_stress.argtypes = [C.c_int, C.c_int] + [D] * 7
    return L


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def std_vec(oracle_mod, **over):
    base = oracle_mod.params(120)
    return np.array([over.get(k, getattr(base, k)) for k in FIELDS], dtype=np.float64)


def run(shim, std, corners, geo, strength, q, S):
    n = strength.size
    s_out = np.zeros((12, n))
    str_out = np.zeros((8, n))
    shim.shim_stress(n, std, _p(corners), _p(geo), _p(strength), _p(q), _p(S),
                     _p(s_out), _p(str_out))
    return s_out, str_out


def points(rng, n):
    geo = rng.uniform(8e3, 12e3, (6, n))
    corners = rng.normal(0, 0.05, (8, n))
    corners[:, : n // 8] *= 1e-5          # Delta below DminArea
    corners[:, n // 8: n // 6] = 0.0      # Delta = 0
    S = rng.normal(0, 3e3, (12, n))
    strength = rng.uniform(0, 5e4, n)
    strength[: n // 16] = 0.0
    return np.ascontiguousarray(geo), np.ascontiguousarray(corners), np.ascontiguousarray(S), strength


def same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64))


def test_std_params_selection(oracle_mod, shim):
    assert shim.shim_std_params(_p(std_vec(oracle_mod))) == 1
    for over in (dict(capping=0.0), dict(Ktens=0.3), dict(revp=1.0),
                 dict(arlx1i=np.inf), dict(arlx1i=np.nan)):
        assert shim.shim_std_params(_p(std_vec(oracle_mod, **over))) == 0, over


def test_std_stress_bits_random(oracle_mod, shim):
    rng = np.random.default_rng(5)
    geo, corners, S, strength = points(rng, 4096)
    q = std_vec(oracle_mod)
    a = run(shim, 1, corners, geo, strength, q, S)
    b = run(shim, 0, corners, geo, strength, q, S)
    assert same_bits(a[0], b[0]) and same_bits(a[1], b[1])


def test_std_stress_bits_fallback_inputs(oracle_mod, shim):
    rng = np.random.default_rng(6)
    n = 64
    geo, corners, S, strength = points(rng, n)
    corners[0, 0:8] = np.nan                       # NaN Delta at some corners
    corners[3, 8:12] = np.inf
    strength[12:20] = 1e300 * 1e9                  # at or above 1e300 * DminArea
    strength[20:24] = -strength[20:24]             # negative strength
    strength[24:28] = np.nan
    for dmin in (None, 0.0, -1e-9):
        over = {} if dmin is None else dict(deltaminEVP=dmin)
        q = std_vec(oracle_mod, **over)
        a = run(shim, 1, corners, geo, strength, q, S)
        b = run(shim, 0, corners, geo, strength, q, S)
        assert same_bits(a[0], b[0]) and same_bits(a[1], b[1]), over
