"""Parity at the configurations the bench numbers are quoted on.

- grid1600x1200 (1,180,692 points) at the full ndte = 1000: every output
  array bit for bit against the oracle, and both reference output files
  (src/vars.F90:2233-2304) md5-equal -- the reference's own acceptance method
  (README.md:44-127).  The oracle runs in its OpenMP SPMD mode on all host
  threads (src/evp_v2b.F90:91-110), which tests/test_oracle.py pins bit for
  bit to its serial mode.
- The FMA library on the same run: at most 1e-12 relative (max-norm) per
  output field against that oracle result, each field printed.
- The 64-member ensemble (ens64, ndte = 500): the batched handle bit for bit
  against a serial loop of one handle per member, for every member, and four
  members (the smallest, the largest, two others) bit for bit against the
  oracle.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import evp1d
from evp1d import synth
from conftest import PKG
from test_gpu_parity import assert_same, gpu_run

pytestmark = pytest.mark.gpu

FIELDS = ("stress", "uvel", "vvel", "strintx", "strinty", "Cb")


@pytest.fixture(scope="module")
def big():
    return synth.make_problem("grid1600x1200")


@pytest.fixture(scope="module")
def big_oracle(oracle_mod, big):
    """The oracle's 1000 subcycles of grid1600x1200 on every host thread."""
    assert big.ndte == 1000
    return oracle_mod.run_1d(big, big.ndte, mode="omp", nthreads=os.cpu_count() or 1)


def test_grid1600x1200_full_ndte_bitwise_and_md5(big, big_oracle):
    pr = big
    assert pr.na > 1_000_000
    fs = gpu_run(pr, pr.ndte)
    # every array and both output files; the state moved over the call
    assert_same(fs, big_oracle, pr)
    assert not np.array_equal(fs.uvel[: pr.na], pr.uvel[: pr.na])


FMA_CHILD = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import evp1d
from evp1d import synth, _lib
assert _lib.FLAVOUR == "fma"
pr = synth.make_problem("grid1600x1200")
fs = evp1d.FieldSet.from_problem(pr)
with evp1d.EVP1D.from_problem(pr) as s:
    s.run(pr.ndte, fs)
np.savez(sys.argv[2], stress=fs.stress, uvel=fs.uvel[:pr.na], vvel=fs.vvel[:pr.na],
         strintx=fs.strintx, strinty=fs.strinty, Cb=fs.Cb)
"""


def test_grid1600x1200_fma_library_within_1e12(big, big_oracle, tmp_path):
    lib = os.path.join(PKG, "lib", "libevp1d_fma.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", PKG], check=True, stdout=subprocess.DEVNULL)
    out = str(tmp_path / "fma.npz")
    env = dict(os.environ, EVP1D_LIBRARY="fma")
    subprocess.run([sys.executable, "-c", FMA_CHILD, PKG, out], check=True, env=env)
    got = np.load(out)
    na = big.na
    ref = dict(stress=big_oracle.stress, uvel=big_oracle.uvel[:na], vvel=big_oracle.vvel[:na],
               strintx=big_oracle.strintx, strinty=big_oracle.strinty, Cb=big_oracle.Cb)
    errs = {}
    for k in FIELDS:
        scale = max(np.abs(ref[k]).max(), 1e-300)
        errs[k] = float(np.abs(got[k] - ref[k]).max() / scale)
    print("grid1600x1200 FMA, max-norm relative error per field:",
          {k: f"{v:.2e}" for k, v in errs.items()})
    for k, e in errs.items():
        assert e <= 1e-12, (k, e)


@pytest.fixture(scope="module")
def ens64():
    cfg = dict(synth.ENSEMBLES["ens64"])
    assert cfg["ndte"] == 500 and cfg["n_members"] == 64
    return synth.make_ensemble(**cfg), cfg["ndte"]


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def test_ens64_batched_equals_serial_loop_and_oracle(oracle_mod, ens64):
    members, ndte = ens64
    ens = synth.concat(members)
    fb = evp1d.FieldSet.from_problem(ens.combined)
    with evp1d.EVP1D.batched(ens, ndte=ndte) as s:
        s.run(ndte, fb)
    off = 0
    us, vs = ens.split_slots(fb.uvel), ens.split_slots(fb.vvel)
    sizes = [m.na for m in members]
    sample = {int(np.argmin(sizes)), int(np.argmax(sizes)), 17, 42}
    for i, m in enumerate(members):
        fm = evp1d.FieldSet.from_problem(m)
        with evp1d.EVP1D.from_problem(m, ndte=ndte) as h:
            h.run(ndte, fm)
        sl = slice(off, off + m.na)
        got = dict(stress=fb.stress[:, sl], uvel=us[i][: m.na], vvel=vs[i][: m.na],
                   strintx=fb.strintx[sl], strinty=fb.strinty[sl], Cb=fb.Cb[sl])
        want = dict(stress=fm.stress, uvel=fm.uvel[: m.na], vvel=fm.vvel[: m.na],
                    strintx=fm.strintx, strinty=fm.strinty, Cb=fm.Cb)
        for k in FIELDS:
            assert np.array_equal(_bits(got[k]), _bits(want[k])), (i, k)
        if i in sample:
            st = oracle_mod.run_1d(m, ndte, mode="omp", nthreads=os.cpu_count() or 1)
            assert_same(fm, st, m, check_str=False)
        off += m.na
