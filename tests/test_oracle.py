"""CPU tests of the oracle: the reference's own acceptance criterion (the v0
2D form and the v2 1D form give md5-identical output files, README.md:63-104),
the OpenMP SPMD loop, the index build, and closed-form known answers."""
import numpy as np
import pytest

from evp1d import synth
import helpers


@pytest.mark.parametrize("curvilinear", [False, True])
@pytest.mark.parametrize("nx,ny,seed,ndte", [(60, 40, 3, 20), (97, 55, 11, 7)])
def test_v0_equals_v2_md5(oracle_mod, nx, ny, seed, ndte, curvilinear):
    g = synth.make_grid(nx, ny, seed=seed, ndte=ndte, curvilinear=curvilinear)
    pr = synth.to_1d(g)
    assert pr.skipT.any() and pr.skipU.any()  # both skip kinds exercised
    st = oracle_mod.run_1d(pr, ndte)
    f1, f2 = helpers.output_files(st.stress, st.strintx, st.strinty, st.uvel,
                                  st.vvel, pr.skipU)
    F = oracle_mod.run_v0(g, ndte)
    g1, g2 = oracle_mod.v0_output_files(g, F, pr)
    assert helpers.md5(f1) == helpers.md5(g1)
    assert helpers.md5(f2) == helpers.md5(g2)
    # the state actually moved
    assert np.abs(st.stress).max() > 0
    assert not np.array_equal(st.uvel[: pr.na], pr.uvel[: pr.na])


def test_v0_equals_v2_grid400x300_short(oracle_mod):
    """The 400 x 300 configuration, 3 subcycles (the full 120 run lives in the
    GPU parity tests)."""
    g = synth.make_grid(**synth.CONFIGS["grid400x300"])
    pr = synth.to_1d(g)
    assert 40_000 < pr.na < 120_000
    st = oracle_mod.run_1d(pr, 3, p=oracle_mod.params(pr.ndte))
    f = helpers.output_files(st.stress, st.strintx, st.strinty, st.uvel, st.vvel, pr.skipU)
    F = oracle_mod.run_v0(g, 3, p=oracle_mod.params(pr.ndte))
    gg = oracle_mod.v0_output_files(g, F, pr)
    assert f == gg


@pytest.mark.parametrize("nthreads", [2, 3, 8])
def test_omp_spmd_equals_serial(oracle_mod, nthreads):
    pr = synth.make_problem("grid400x300", nx=120, ny=90, ndte=9)
    a = oracle_mod.run_1d(pr, 9)
    b = oracle_mod.run_1d(pr, 9, mode="omp", nthreads=nthreads)
    for k in ("stress", "uvel", "vvel", "strintx", "strinty", "Cb", "str"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_omp_domain_split(oracle_mod):
    """domp_get_domain (src/myomp.F90:85-124) tiles 1..n without gaps."""
    import ctypes as C
    L = oracle_mod.lib()
    for n in (1, 7, 100, 631387):
        for nt in (1, 3, 8, 36):
            lo, hi = C.c_int(), C.c_int()
            nxt = 1
            for t in range(nt):
                L.oracle_omp_domain(1, n, t, nt, C.byref(lo), C.byref(hi))
                if hi.value >= lo.value:
                    assert lo.value == nxt
                    nxt = hi.value + 1
            assert nxt == n + 1


def test_stress_only_then_stepu_only(oracle_mod):
    """lindividual loops (src/evp_v2b.F90:127-155) compose to one subcycle."""
    pr = synth.make_problem("grid400x300", nx=50, ny=40, ndte=5)
    a = oracle_mod.run_1d(pr, 1, p=oracle_mod.params(5))
    st = oracle_mod.State1D(pr)
    oracle_mod.run_1d(pr, 1, p=oracle_mod.params(5), mode="stress", state=st)
    oracle_mod.run_1d(pr, 1, p=oracle_mod.params(5), mode="stepu", state=st)
    assert np.array_equal(a.uvel, st.uvel) and np.array_equal(a.stress, st.stress)


@pytest.mark.parametrize("shape,frac,seed", [((40, 30), 0.5, 0), ((65, 33), 0.9, 1),
                                             ((10, 10), 0.0, 2), ((8, 9), 1.0, 3)])
def test_index_build_numpy_vs_oracle(oracle_mod, shape, frac, seed):
    rng = np.random.default_rng(seed)
    mask = rng.random(shape) < frac
    mask[0, :] = mask[:, 0] = False  # south/west ghost row/column
    ix = synth.build_index(mask)
    na, navel, ti, tj, tij, nb = oracle_mod.build_index(mask)
    assert (na, navel) == (ix.na, ix.navel)
    assert np.array_equal(ti, ix.indxti) and np.array_equal(tj, ix.indxtj)
    assert np.array_equal(tij, ix.indxtij)
    for k in nb:
        assert np.array_equal(nb[k], ix.nb[k]), k


def test_standalone_index_known_answer(oracle_mod):
    """21 x 21 square: 441 list points, one halo column + row + corner on each
    side of the stencil: navel = 441 + 2 * (21 + 21 + 1) = 527."""
    pr = helpers.standalone_problem()
    assert pr.na == 441 and pr.navel == 527
    na, navel, *_ = oracle_mod.build_index(helpers.standalone_grid().iceT)
    assert (na, navel) == (441, 527)


@pytest.mark.parametrize("ndte", [1, 5])
def test_standalone_closed_form(oracle_mod, ndte):
    """With strength = 0 the viscosities vanish, so every stress component
    relaxes as stress <- stress * denom1 each subcycle, interior and edge
    points alike (src/bench_v2b.F90:187-212)."""
    pr = helpers.standalone_problem(ndte=ndte, strength=0.0)
    p = oracle_mod.params(ndte)
    st = oracle_mod.run_1d(pr, ndte, p=p)
    want = pr.stress.copy()
    for _ in range(ndte):
        want = want * p.denom1
    assert np.array_equal(st.stress, want)
    assert np.all(st.Cb == 0.0)
    # vrel = 0 and fm = 0: u = strintx + u_old exactly when brlx = 1 (ndte=1)
    if ndte == 1:
        w = pr.skipU == 0
        assert np.array_equal(st.uvel[: pr.na][w], st.strintx[w] + pr.uvel[: pr.na][w])


def test_params_match_reference_defaults(oracle_mod):
    """set_evp_parameters (src/ice.F90:109-130) for ndte = 120."""
    p = oracle_mod.params(120)
    assert p.epp2i == 0.25 and p.e_factor == 0.25 and p.capping == 1.0
    assert p.brlx == 120.0 and p.arlx1i == 1.0 / (2 * 0.36 * 120)
    assert p.denom1 == 1.0 / (1.0 + p.arlx1i) and p.deltaminEVP == 1e-8
