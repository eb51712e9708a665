"""CPU unit tests of the library's per-point adjoint arithmetic.

cice-evp1d_b200/csrc/evp_adjoint_math.cuh is __host__ __device__ code; here
it is compiled for the host (tests/native/adjoint_math_shim.cpp) and its
vector-Jacobian products of stress and stepu are compared with torch
autograd of the taped restatement (oracle/evp_tape.py) on random points,
including points on both sides of max(Delta, DminArea), zero velocities
(zero-length square roots), a nonzero seabed stress and the general
parameter branches (capping = 0, Ktens, revp, turning angle)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, PKG

torch = pytest.importorskip("torch")

SHIM = os.path.join(ROOT, "tests", "native", "adjoint_math_shim.cpp")


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("shim") / "adjoint_math_shim.so")
    subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-ffp-contract=off",
                    "-I", os.path.join(PKG, "csrc"), "-I", os.path.join(ROOT, "include"),
                    "-I", "/usr/local/cuda/include", SHIM, "-o", out], check=True)
    L = C.CDLL(out)
    D = C.POINTER(C.c_double)
    L.shim_stress_adjoint.argtypes = [C.c_int] + [D] * 8
    L.shim_stepu_adjoint.argtypes = [C.c_int, D, D, D]
    return L


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


class P:
    """evp1d_params as a plain object."""

    FIELDS = ("arlx1i", "denom1", "brlx", "capping", "e_factor", "epp2i",
              "deltaminEVP", "revp", "Ktens", "u0", "cosw", "sinw", "rhow")

    def __init__(self, base, **over):
        for k in self.FIELDS:
            setattr(self, k, over.get(k, getattr(base, k)))

    def vec(self):
        return np.array([getattr(self, k) for k in self.FIELDS])


def param_sets(oracle_mod):
    base = oracle_mod.params(120)
    return [P(base), P(base, capping=0.0, Ktens=0.3, revp=1.0, cosw=0.9, sinw=0.4)]


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def random_points(rng, n):
    geo = rng.uniform(8e3, 12e3, (6, n))
    corners = rng.normal(0, 0.05, (8, n))
    corners[:, : n // 8] *= 1e-5          # Delta below DminArea
    corners[:, n // 8: n // 6] = 0.0      # Delta = 0
    S = rng.normal(0, 3e3, (12, n))
    strength = rng.uniform(0, 5e4, n)
    return geo, corners, S, strength


@pytest.mark.parametrize("which", [0, 1])
def test_stress_adjoint_matches_autograd(oracle_mod, shim, which):
    import evp_tape
    p = param_sets(oracle_mod)[which]
    rng = np.random.default_rng(11 + which)
    n = 512
    geo, corners, S0, strength = random_points(rng, n)
    lo = rng.normal(0, 1, (8, n))
    lS = rng.normal(0, 1, (12, n))
    # torch VJP
    tc = [torch.tensor(corners[k], requires_grad=True) for k in range(8)]
    tS = [torch.tensor(S0[k], requires_grad=True) for k in range(12)]
    tstr = torch.tensor(strength, requires_grad=True)
    g = evp_tape.geometry(*[torch.tensor(geo[k]) for k in range(6)], p.deltaminEVP)
    Snew, st = evp_tape.stress_point(tS, tc, g, tstr, p)
    obj = sum((Snew[k] * torch.tensor(lS[k])).sum() for k in range(12)) + \
        sum((st[k] * torch.tensor(lo[k])).sum() for k in range(8))
    obj.backward()
    # library arithmetic
    ls = lS.copy()
    lc = np.zeros((8, n))
    lstr = np.zeros(n)
    shim.shim_stress_adjoint(n, _p(corners), _p(geo), _p(strength), _p(p.vec()), _p(lo),
                             ls.ctypes.data_as(C.POINTER(C.c_double)),
                             lc.ctypes.data_as(C.POINTER(C.c_double)),
                             lstr.ctypes.data_as(C.POINTER(C.c_double)))
    assert rel_err(ls, np.stack([t.grad.numpy() for t in tS])) < 1e-12
    assert rel_err(lc, np.stack([t.grad.numpy() for t in tc])) < 1e-12
    assert rel_err(lstr, tstr.grad.numpy()) < 1e-12


@pytest.mark.parametrize("which", [0, 1])
def test_stepu_adjoint_matches_autograd(oracle_mod, shim, which):
    import evp_tape
    p = param_sets(oracle_mod)[which]
    rng = np.random.default_rng(31 + which)
    n = 512
    u = rng.normal(0, 0.05, n)
    v = rng.normal(0, 0.05, n)
    u[:16] = 0.0
    v[:16] = 0.0                          # |u| = 0
    f = dict(uocn=rng.normal(0, 0.2, n), vocn=rng.normal(0, 0.2, n),
             waterx=rng.normal(0, 1, n), watery=rng.normal(0, 1, n),
             umassdti=rng.uniform(0.2, 3.0, n), fm=rng.uniform(-0.5, 0.5, n),
             Tbu=np.where(rng.uniform(size=n) < 0.5, 0.0, rng.uniform(0, 2.0, n)),
             forcex=rng.normal(0, 0.1, n), forcey=rng.normal(0, 0.1, n),
             uinit=rng.normal(0, 0.05, n), vinit=rng.normal(0, 0.05, n))
    f["uocn"][16:24] = u[16:24]
    f["vocn"][16:24] = v[16:24]           # |u_ocn - u| = 0
    aiXrhow = rng.uniform(0.2, 1.0, n) * p.rhow
    Cw = np.full(n, 5.5e-3)
    sx, sy = rng.normal(0, 0.5, n), rng.normal(0, 0.5, n)
    lun, lvn = rng.normal(0, 1, n), rng.normal(0, 1, n)
    T = lambda a: torch.tensor(a, requires_grad=True)
    tu, tv, tsx, tsy, tCw = T(u), T(v), T(sx), T(sy), T(Cw)
    tf = {k: torch.tensor(a) for k, a in f.items()}
    tf["forcex"], tf["forcey"] = T(f["forcex"]), T(f["forcey"])
    tf["uinit"], tf["vinit"] = T(f["uinit"]), T(f["vinit"])
    tf["kvrel"] = torch.tensor(aiXrhow) * tCw
    un, vn = evp_tape.stepu_point(tu, tv, tsx, tsy, tf, p)
    ((un * torch.tensor(lun)).sum() + (vn * torch.tensor(lvn)).sum()).backward()
    kvrel = aiXrhow * Cw
    inp = np.stack([u, v, un.detach().numpy(), vn.detach().numpy(), lun, lvn, kvrel, aiXrhow,
                    f["uocn"], f["vocn"], f["waterx"], f["watery"], f["umassdti"], f["fm"],
                    f["Tbu"]])
    out = np.zeros((7, n))
    shim.shim_stepu_adjoint(n, _p(inp), _p(p.vec()), out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rel_err(out[0], tu.grad.numpy()) < 1e-10
    assert rel_err(out[1], tv.grad.numpy()) < 1e-10
    assert rel_err(out[2], tsx.grad.numpy()) < 1e-10
    assert rel_err(out[3], tsy.grad.numpy()) < 1e-10
    assert rel_err(out[2], tf["forcex"].grad.numpy()) < 1e-10
    assert rel_err(out[4], tCw.grad.numpy()) < 1e-10
    if p.revp != 0:
        assert rel_err(out[5], tf["uinit"].grad.numpy()) < 1e-10
        assert rel_err(out[6], tf["vinit"].grad.numpy()) < 1e-10
