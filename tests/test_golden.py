"""The committed golden fixture: the oracle reproduces its recorded md5s (so
the checker itself cannot drift), the v0 and v2 md5s recorded in it agree,
and the closed-form smoke-test answer holds."""
import hashlib

import numpy as np

import golden_io
import helpers


def test_fixture_v0_equals_v2():
    _, _, exp = golden_io.load()
    assert exp["md5_stress_v0"] == exp["md5_stress_v2"]
    assert exp["md5_stepu_v0"] == exp["md5_stepu_v2"]


def test_oracle_reproduces_fixture(oracle_mod):
    pr, out, exp = golden_io.load()
    st = oracle_mod.run_1d(pr, pr.ndte)
    f1, f2 = helpers.output_files(st.stress, st.strintx, st.strinty, st.uvel, st.vvel, pr.skipU)
    assert helpers.md5(f1) == exp["md5_stress_v2"]
    assert helpers.md5(f2) == exp["md5_stepu_v2"]
    assert np.array_equal(st.str[:, : pr.navel], out["str"])


def test_standalone_fixture(oracle_mod):
    _, _, exp = golden_io.load()
    e = exp["standalone_ndte3_strength0"]
    sa = helpers.standalone_problem(ndte=3, strength=0.0)
    st = oracle_mod.run_1d(sa, 3)
    assert (sa.na, sa.navel) == (e["na"], e["navel"])
    assert hashlib.md5(np.ascontiguousarray(st.stress).tobytes()).hexdigest() == e["md5_stress"]
    p = oracle_mod.params(3)
    assert st.stress[0, 0] == 1.0 * p.denom1 * p.denom1 * p.denom1 == e["stressp_1"]
