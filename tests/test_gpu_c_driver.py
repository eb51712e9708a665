"""The solver driven from a plain C99 program (tests/native/c_driver.c)
linked against lib/libevp1d.so: the C-ABI as a C or Fortran host calls it,
with host pointers and no Python binding in the path.  Its results equal
the oracle's bit for bit, and the reference's two output files hash equal
(src/vars.F90:2233-2304)."""
import os
import subprocess

import numpy as np
import pytest

import helpers
from conftest import ROOT
from evp1d import synth
from test_gpu_parity import oracle_run

pytestmark = pytest.mark.gpu

LIBDIR = os.path.join(ROOT, "cice-evp1d_b200", "lib")
INPUTS = ("strength", "Cw", "aiu", "uocn", "vocn", "waterx", "watery", "forcex", "forcey",
          "umassdti", "fm", "Tbu")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cdrv") / "c_driver")
    subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Werror",
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "native", "c_driver.c"), "-o", exe,
                    "-L", LIBDIR, "-levp1d", "-Wl,-rpath," + LIBDIR], check=True)
    return exe


def _write(path, pr):
    i4 = lambda a: np.ascontiguousarray(a, dtype="<i4")  # noqa: E731
    f8 = lambda a: np.ascontiguousarray(a, dtype="<f8")  # noqa: E731
    with open(path, "wb") as f:
        i4([pr.na, pr.navel, pr.ndte]).tofile(f)
        for k in ("ee", "ne", "se", "nw", "sw", "sse"):
            i4(pr.idx[k]).tofile(f)
        i4(pr.skipT).tofile(f)
        i4(pr.skipU).tofile(f)
        for k in ("dxT", "dyT", "HTE", "HTN", "HTEm1", "HTNm1", "uarear"):
            f8(pr.f[k]).tofile(f)
        f8(pr.stress).tofile(f)
        for k in INPUTS:
            f8(pr.f[k]).tofile(f)
        for a in (pr.uvel, pr.vvel, pr.strintx, pr.strinty, pr.Cb):
            f8(a).tofile(f)


def _read(path, pr):
    d = np.fromfile(path, dtype="<f8")
    na, nv = pr.na, pr.navel
    assert d.size == 12 * na + 2 * nv + 3 * na
    o = dict(stress=d[: 12 * na].reshape(12, na))
    p = 12 * na
    o["uvel"], o["vvel"] = d[p: p + nv], d[p + nv: p + 2 * nv]
    p += 2 * nv
    o["strintx"], o["strinty"], o["Cb"] = d[p: p + na], d[p + na: p + 2 * na], d[p + 2 * na:]
    return o


@pytest.mark.parametrize("grid", ["plain", "curvilinear"])
def test_c_host_matches_the_oracle(oracle_mod, driver, tmp_path, grid):
    if grid == "plain":
        pr = synth.make_problem("grid400x300", nx=150, ny=110, ndte=20)
    else:
        pr = synth.to_1d(synth.make_grid(131, 77, seed=9, ndte=13, curvilinear=True))
    src, dst = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    _write(src, pr)
    r = subprocess.run([driver, src, dst], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == f"ok {pr.na} {pr.navel} {pr.ndte}"
    got = _read(dst, pr)
    ref = oracle_run(oracle_mod, pr, pr.ndte)
    na = pr.na
    for k in ("stress", "strintx", "strinty", "Cb"):
        assert np.array_equal(got[k].view(np.int64), np.asarray(getattr(ref, k)).view(np.int64)), k
    for k in ("uvel", "vvel"):
        assert np.array_equal(got[k][:na].view(np.int64), getattr(ref, k)[:na].view(np.int64)), k
        # halo slots are read as given and never written
        assert np.array_equal(got[k][na:], np.asarray(getattr(pr, k))[na:]), k
    f = helpers.output_files(got["stress"], got["strintx"], got["strinty"], got["uvel"],
                             got["vvel"], pr.skipU)
    g = helpers.output_files(ref.stress, ref.strintx, ref.strinty, ref.uvel, ref.vvel, pr.skipU)
    assert helpers.md5(f[0]) == helpers.md5(g[0]) and helpers.md5(f[1]) == helpers.md5(g[1])
