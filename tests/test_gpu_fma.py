"""GPU test of the FMA flavour (lib/libevp1d_fma.so, EVP1D_LIBRARY=fma): the
same solver with a*b+c contracted into fused multiply-adds agrees with the
bit-exact oracle to <= 1e-12 relative (max-norm over each output field, each
field stated separately), on grid400x300 (ndte = 120) and on a small grid run for
1000 subcycles."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, PKG
from evp1d import synth

pytestmark = pytest.mark.gpu

FIELDS = ("stress", "uvel", "vvel", "strintx", "strinty", "Cb")

CHILD = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import evp1d
from evp1d import synth, _lib
assert _lib.FLAVOUR == "fma"
name, out = sys.argv[2], sys.argv[3]
pr = synth.make_problem("grid400x300") if name == "grid400x300" else \
    synth.to_1d(synth.make_grid(90, 70, seed=61, ndte=1000, curvilinear=True))
fs = evp1d.FieldSet.from_problem(pr)
with evp1d.EVP1D.from_problem(pr) as s:
    s.run(pr.ndte, fs)
np.savez(out, stress=fs.stress, uvel=fs.uvel[:pr.na], vvel=fs.vvel[:pr.na],
         strintx=fs.strintx, strinty=fs.strinty, Cb=fs.Cb)
"""


@pytest.mark.parametrize("case", ["grid400x300", "long"])
def test_fma_flavour_within_1e12(oracle_mod, case, tmp_path):
    lib = os.path.join(PKG, "lib", "libevp1d_fma.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", PKG], check=True, stdout=subprocess.DEVNULL)
    out = str(tmp_path / "fma.npz")
    env = dict(os.environ, EVP1D_LIBRARY="fma")
    subprocess.run([sys.executable, "-c", CHILD, PKG, case, out], check=True, env=env)
    got = np.load(out)
    pr = synth.make_problem("grid400x300") if case == "grid400x300" else \
        synth.to_1d(synth.make_grid(90, 70, seed=61, ndte=1000, curvilinear=True))
    st = oracle_mod.run_1d(pr, pr.ndte)
    ref = dict(stress=st.stress, uvel=st.uvel[: pr.na], vvel=st.vvel[: pr.na],
               strintx=st.strintx, strinty=st.strinty, Cb=st.Cb)
    errs = {}
    for k in FIELDS:
        scale = max(np.abs(ref[k]).max(), 1e-300)
        errs[k] = float(np.abs(got[k] - ref[k]).max() / scale)
    print(case, {k: f"{v:.1e}" for k, v in errs.items()})
    for k, e in errs.items():
        assert e <= 1e-12, (k, e)
