"""The reference's 1D file formats: inputs round-trip, and the golden case
written to files and run by the oracle reproduces the fixture's md5 sums."""
import numpy as np
import pytest

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


def test_output_statistics_layout():
    """The output statistics mirror stat_out_1d (src/vars.F90:2209-2232): one
    line per field, a11 label then min, max, sum as f25.8."""
    from evp1d.io import output_statistics
    rng = np.random.default_rng(3)
    na, navel = 50, 57
    stress = rng.normal(0, 100, (12, na))
    strs = rng.normal(0, 1, (8, navel))
    lines = output_statistics(stress, strs, rng.normal(size=na), rng.normal(size=na),
                              rng.normal(size=navel), rng.normal(size=navel))
    assert len(lines) == 12 + 8 + 4
    assert lines[0].startswith(" stressp_1:") and lines[8].startswith("stress12_1:")
    assert lines[12].startswith("      str1:") and lines[-1].startswith("      vvel:")
    assert all(len(x) == 11 + 3 * 25 for x in lines)
    mn, mx, sm = (float(v) for v in lines[0][11:].split())
    assert abs(mn - stress[0].min()) < 1e-8 and abs(mx - stress[0].max()) < 1e-8
    assert abs(sm - stress[0].sum()) < 1e-6
    assert len(output_statistics(stress, None, stress[0], stress[0], strs[0], strs[0])) == 16


@pytest.mark.gpu
def test_run_case_from_files_matches_golden(tmp_path):
    """The file-driven runner (python -m evp1d.io): the golden case written
    in the reference's input format, run on the GPU, gives output files with
    the fixture's md5 sums, and --stats prints the 24 statistics lines."""
    import evp1d
    pr, out, exp = golden_io.load()
    p = evp1d.set_evp_parameters(pr.ndte)
    evio.write_inputs(str(tmp_path), pr,
                      {k: getattr(p, k) for k in ("capping", "e_factor", "epp2i", "deltaminEVP")})
    h1, h2, lines = evio.run_case(str(tmp_path), pr.na, pr.navel, pr.ndte, "t", stats=True)
    assert h1 == exp["md5_stress_v2"] and h2 == exp["md5_stepu_v2"]
    assert len(lines) == 24 and lines[-1].startswith("      vvel:")
