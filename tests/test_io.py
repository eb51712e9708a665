"""The reference's 1D file formats: inputs round-trip, and the golden case
written to files and run by the oracle reproduces the fixture's md5 sums."""
import numpy as np

import golden_io
from evp1d import io as evio


def test_input_round_trip(tmp_path):
    pr, _, _ = golden_io.load()
    scal = dict(capping=1.0, e_factor=0.25, epp2i=0.25, deltaminEVP=1e-8)
    evio.write_inputs(str(tmp_path), pr, scal)
    q, s2 = evio.read_inputs(str(tmp_path), pr.na, pr.navel, pr.ndte)
    assert s2 == scal
    for k in pr.idx:
        assert np.array_equal(q.idx[k], pr.idx[k])
    for k in ("strength", "dxT", "dyT", "HTE", "HTN", "HTEm1", "HTNm1", "uarear", "Cw",
              "aiu", "uocn", "vocn", "waterx", "watery", "forcex", "forcey", "umassdti",
              "fm", "Tbu"):
        assert np.array_equal(q.f[k], pr.f[k]), k
    assert np.array_equal(q.stress, pr.stress)
    assert np.array_equal(q.uvel, pr.uvel) and np.array_equal(q.skipT, pr.skipT)
    assert np.array_equal(q.skipU, pr.skipU)


def test_file_case_reproduces_fixture_md5(tmp_path, oracle_mod):
    pr, _, exp = golden_io.load()
    p = oracle_mod.params(pr.ndte)
    scal = dict(capping=p.capping, e_factor=p.e_factor, epp2i=p.epp2i,
                deltaminEVP=p.deltaminEVP)
    evio.write_inputs(str(tmp_path), pr, scal)
    q, _ = evio.read_inputs(str(tmp_path), pr.na, pr.navel, pr.ndte)
    st = oracle_mod.run_1d(q, pr.ndte, p=p)
    h1, h2 = evio.write_outputs(str(tmp_path), "oracle", st.stress, st.strintx, st.strinty,
                                st.uvel, st.vvel, q.skipU)
    assert (h1, h2) == (exp["md5_stress_v2"], exp["md5_stepu_v2"])


def test_bad_sizes_rejected(tmp_path):
    pr, _, _ = golden_io.load()
    evio.write_inputs(str(tmp_path), pr, dict(capping=1.0, e_factor=0.25, epp2i=0.25,
                                              deltaminEVP=1e-8))
    import pytest
    with pytest.raises(ValueError):
        evio.read_inputs(str(tmp_path), pr.na + 1, pr.navel)
