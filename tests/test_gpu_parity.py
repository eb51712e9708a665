"""GPU parity: the CUDA path through the C-ABI against the oracle, bit for bit.

The tolerance is zero: with -fmad=false every output must be bitwise equal
to the oracle's no-FMA CPU restatement (the reference's f0/f1 semantics), and
the two md5-compared output files (src/vars.F90:2233-2304) must hash equal.
"""
import ctypes as C

import numpy as np
import pytest

import evp1d
from evp1d import synth
import helpers

pytestmark = pytest.mark.gpu


def gpu_run(pr, ndte, params=None, want_str=True, explicit_init=False, calls=1):
    fs = evp1d.FieldSet.from_problem(pr, want_str=want_str, explicit_init=explicit_init)
    with evp1d.EVP1D.from_problem(pr, ndte=ndte, params=params) as s:
        for _ in range(calls):
            s.run(ndte, fs)
    return fs


def oracle_run(oracle_mod, pr, ndte, params=None):
    p = params if params is not None else oracle_mod.params(ndte)
    op = oracle_mod.OracleParams(**{k: getattr(p, k) for k in evp1d._lib.PARAM_FIELDS})
    return oracle_mod.run_1d(pr, ndte, p=op)


def assert_same(fs, st, pr, check_str=True):
    na = pr.na
    for name, a, b in (("stress", fs.stress, st.stress), ("uvel", fs.uvel[:na], st.uvel[:na]),
                       ("vvel", fs.vvel[:na], st.vvel[:na]),
                       ("strintx", fs.strintx, st.strintx), ("strinty", fs.strinty, st.strinty),
                       ("Cb", fs.Cb, st.Cb)):
        assert np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64)), \
            f"{name}: {helpers.first_mismatch(a, b)}"
    if check_str and fs.str is not None:
        assert np.array_equal(fs.str.view(np.int64), st.str[:, : pr.navel].view(np.int64)), \
            "str: " + helpers.first_mismatch(fs.str, st.str[:, : pr.navel])
    f = helpers.output_files(fs.stress, fs.strintx, fs.strinty, fs.uvel, fs.vvel, pr.skipU)
    g = helpers.output_files(st.stress, st.strintx, st.strinty, st.uvel, st.vvel, pr.skipU)
    assert helpers.md5(f[0]) == helpers.md5(g[0])
    assert helpers.md5(f[1]) == helpers.md5(g[1])


@pytest.mark.parametrize("curvilinear", [False, True])
@pytest.mark.parametrize("nx,ny,seed,ndte", [(60, 40, 3, 20), (131, 77, 9, 13)])
def test_small_grids_bitwise(oracle_mod, nx, ny, seed, ndte, curvilinear):
    pr = synth.to_1d(synth.make_grid(nx, ny, seed=seed, ndte=ndte, curvilinear=curvilinear))
    assert_same(gpu_run(pr, ndte), oracle_run(oracle_mod, pr, ndte), pr)


def test_grid400x300_full_md5(oracle_mod):
    """400 x 300 synthetic grid, ndte = 120: md5-identical output files."""
    pr = synth.make_problem("grid400x300")
    assert_same(gpu_run(pr, pr.ndte, want_str=False), oracle_run(oracle_mod, pr, pr.ndte),
                pr, check_str=False)


def test_two_calls_carry_state(oracle_mod):
    """Two dyn_evp1d_run calls in a row: the second starts from the first's
    stresses and velocities."""
    pr = synth.make_problem("grid400x300", nx=80, ny=60, ndte=10)
    fs = gpu_run(pr, 10, calls=2)
    st = oracle_run(oracle_mod, pr, 10)
    pr2 = pr.copy()
    pr2.stress[:] = st.stress
    pr2.uvel[:] = st.uvel[: pr.navel]
    pr2.vvel[:] = st.vvel[: pr.navel]
    pr2.strintx[:], pr2.strinty[:], pr2.Cb[:] = st.strintx, st.strinty, st.Cb
    # the second call's uvel_init defaults to its starting velocity
    pr2.f["uvel_init"] = st.uvel[: pr.na].copy()
    pr2.f["vvel_init"] = st.vvel[: pr.na].copy()
    assert_same(fs, oracle_run(oracle_mod, pr2, 10), pr2)


def test_standalone_closed_form():
    """Integration smoke-test state with strength = 0: stress = stress0 *
    denom1**ndte exactly."""
    ndte = 4
    pr = helpers.standalone_problem(ndte=ndte)
    fs = gpu_run(pr, ndte)
    p = evp1d.set_evp_parameters(ndte)
    want = pr.stress.copy()
    for _ in range(ndte):
        want = want * p.denom1
    assert np.array_equal(fs.stress, want)
    assert np.all(fs.Cb == 0)


def test_standalone_with_strength(oracle_mod):
    pr = helpers.standalone_problem(ndte=3, strength=2.5e4)
    assert_same(gpu_run(pr, 3), oracle_run(oracle_mod, pr, 3), pr)


def test_every_parameter_path(oracle_mod):
    """Revised EVP with explicit uvel_init, basal stress, turning angle,
    tensile strength and capping = 0: every term of stress/stepu is live."""
    g = synth.make_grid(70, 50, seed=21, ndte=15, curvilinear=True)
    rng = np.random.default_rng(5)
    g.f["Tbu"] = np.asfortranarray(rng.uniform(0.0, 5.0, g.f["Tbu"].shape))
    g.f["fm"] = np.asfortranarray(g.f["fm"] * np.where(rng.random(g.f["fm"].shape) < 0.3, -1, 1))
    pr = synth.to_1d(g)
    pr.f["uvel_init"] = pr.f["uvel_init"] + rng.normal(0, 0.01, pr.na)
    p = evp1d.set_evp_parameters(15)
    p.revp, p.Ktens, p.capping = 1.0, 0.2, 0.0
    p.cosw, p.sinw = np.cos(0.4), np.sin(0.4)
    fs = gpu_run(pr, 15, params=p, explicit_init=True)
    assert_same(fs, oracle_run(oracle_mod, pr, 15, params=p), pr)
    assert np.any(fs.Cb != 0)


def test_halo_velocity_read_as_given(oracle_mod):
    """Halo slots of uvel/vvel are inputs (src/vars.F90:2108 reads
    uvel(1:navel)); nonzero halo values feed the stress gathers."""
    pr = synth.make_problem("grid400x300", nx=50, ny=40, ndte=6)
    rng = np.random.default_rng(2)
    pr.uvel[pr.na:] = rng.normal(0, 0.05, pr.navel - pr.na)
    pr.vvel[pr.na:] = rng.normal(0, 0.05, pr.navel - pr.na)
    fs = gpu_run(pr, 6)
    assert_same(fs, oracle_run(oracle_mod, pr, 6), pr)
    assert np.array_equal(fs.uvel[pr.na:], pr.uvel[pr.na:])


@pytest.mark.parametrize("which", ["allT", "allU", "none"])
def test_skip_patterns(oracle_mod, which):
    pr = synth.make_problem("grid400x300", nx=40, ny=30, ndte=5)
    if which == "allT":
        pr.skipT[:] = 1
    elif which == "allU":
        pr.skipU[:] = 1
    else:
        pr.skipT[:] = 0
        pr.skipU[:] = 0
    assert_same(gpu_run(pr, 5), oracle_run(oracle_mod, pr, 5), pr)


def test_empty_problem():
    p = evp1d.set_evp_parameters(5)
    z = np.zeros(0, np.int32)
    zd = np.zeros(0)
    with evp1d.EVP1D(0, 0, ee=z, ne=z, se=z, nw=z, sw=z, sse=z, dxT=zd, dyT=zd,
                     HTE=zd, HTN=zd, HTEm1=zd, HTNm1=zd, uarear=zd, params=p) as s:
        fs = evp1d.FieldSet(0, 0, skipT=z, skipU=z, stress=np.zeros((12, 0)),
                            uvel=zd, vvel=zd, strintx=zd, strinty=zd, Cb=zd,
                            **{k: zd for k in evp1d.FieldSet.DYN})
        s.run(5, fs)
        s.stress_only(3)
        s.stepu_only(3)


def test_lindividual_loops(oracle_mod):
    """stress alone n times, then stepu alone n times (src/evp_v2b.F90:127-155)."""
    pr = synth.make_problem("grid400x300", nx=60, ny=45, ndte=4)
    fs = evp1d.FieldSet.from_problem(pr, want_str=True)
    st = oracle_mod.State1D(pr)
    op = oracle_mod.params(4)
    with evp1d.EVP1D.from_problem(pr, ndte=4) as s:
        s.upload(fs)
        s.stress_only(3)
        s.stepu_only(2)
        s.download(fs)
    oracle_mod.run_1d(pr, 3, p=op, mode="stress", state=st)
    oracle_mod.run_1d(pr, 2, p=op, mode="stepu", state=st)
    assert_same(fs, st, pr)


def test_error_paths_on_device():
    pr = synth.make_problem("grid400x300", nx=30, ny=20, ndte=3)
    with evp1d.EVP1D.from_problem(pr, ndte=3) as s:
        with pytest.raises(evp1d.EVP1DError) as e:
            s.subcycles(3)  # nothing uploaded
        assert e.value.code == -7
        with pytest.raises(evp1d.EVP1DError) as e:
            s.subcycles(-1)
        assert e.value.code == -1
        fs = evp1d.FieldSet.from_problem(pr)
        fs.c.strength = None
        with pytest.raises(evp1d.EVP1DError) as e:
            s.upload(fs)
        assert e.value.code == -1
    with pytest.raises(evp1d.EVP1DError) as e:
        evp1d.EVP1D.from_problem(pr, ndte=3, device=4096)
    assert e.value.code == -1


def test_launch_count_is_native():
    pr = synth.make_problem("grid400x300", nx=30, ny=20, ndte=7)
    fs = evp1d.FieldSet.from_problem(pr)
    with evp1d.EVP1D.from_problem(pr, ndte=7) as s:
        s.launch_count(reset=True)
        s.run(7, fs)
        assert s.launch_count() > 0


def test_shuffled_list_order(oracle_mod):
    """A list in random order: the solver rebuilds the grid tiles from the
    neighbour graph; results stay bitwise equal."""
    pr = helpers.shuffle_problem(synth.make_problem("grid400x300", nx=90, ny=70, ndte=9), 7)
    assert_same(gpu_run(pr, 9), oracle_run(oracle_mod, pr, 9), pr)


def test_tiles_at_the_halo_cap(oracle_mod):
    """Tiles cut at the forward-halo cap: 64 recomputed halo points fill both
    halo warps and the halo arrays of a stage."""
    pr = helpers.halo_limited_problem(3000, 50, 7)
    assert evp1d.plan_stats(pr.na, pr.navel, pr.idx)["max_halo"] == 64
    assert_same(gpu_run(pr, pr.ndte), oracle_run(oracle_mod, pr, pr.ndte), pr)


@pytest.mark.parametrize("na,nhalo,seed", [(5000, 300, 0), (777, 5, 1)])
def test_irregular_graph(oracle_mod, na, nhalo, seed):
    """Random neighbour slots (no grid): consecutive-point tiles whose halo
    is split to fit; results stay bitwise equal."""
    pr = helpers.random_graph_problem(na, nhalo, seed)
    assert_same(gpu_run(pr, 5), oracle_run(oracle_mod, pr, 5), pr)


@pytest.mark.parametrize("ndte", [1, 2, 49, 50, 51, 101])
def test_graph_chunk_boundaries(oracle_mod, ndte):
    """Subcycle counts around the captured-graph chunk (50) and both
    ping-pong parities."""
    pr = synth.make_problem("grid400x300", nx=40, ny=30, ndte=ndte)
    assert_same(gpu_run(pr, ndte), oracle_run(oracle_mod, pr, ndte), pr)


@pytest.mark.parametrize("path", ["fused", "tma"])
def test_kernel_paths(oracle_mod, monkeypatch, path):
    """Both subcycle kernels (plain loads and TMA-fed) are bitwise equal to
    the oracle; EVP1D_PATH selects the kernel at evp1d_init."""
    if path == "fused":
        monkeypatch.setenv("EVP1D_PATH", "fused")
    else:
        monkeypatch.delenv("EVP1D_PATH", raising=False)
    pr = synth.make_problem("grid400x300", nx=150, ny=110, ndte=11)
    fs = evp1d.FieldSet.from_problem(pr, want_str=True)
    with evp1d.EVP1D.from_problem(pr, ndte=11) as s:
        assert s.path == ("fused-tile" if path == "fused" else "fused-tile-tma")
        s.run(11, fs)
    assert_same(fs, oracle_run(oracle_mod, pr, 11), pr)


def assert_same_nan_aware(fs, st, pr):
    """Bitwise equality, except that NaN must meet NaN (GPU and x86 produce
    different NaN payloads)."""
    na = pr.na
    for name, a, b in (("stress", fs.stress, st.stress), ("uvel", fs.uvel[:na], st.uvel[:na]),
                       ("vvel", fs.vvel[:na], st.vvel[:na]), ("strintx", fs.strintx, st.strintx),
                       ("strinty", fs.strinty, st.strinty), ("Cb", fs.Cb, st.Cb)):
        a = np.asarray(a).reshape(-1)
        b = np.asarray(b).reshape(-1)
        assert np.array_equal(np.isnan(a), np.isnan(b)), f"{name}: NaN pattern differs"
        m = ~np.isnan(b)
        assert np.array_equal(a[m].view(np.int64), b[m].view(np.int64)), \
            f"{name}: {helpers.first_mismatch(a[m], b[m])}"


@pytest.mark.parametrize("u0", [5e-5, 0.0])
def test_shortcut_edges(oracle_mod, u0):
    """Inputs at the edges of the solver's exact shortcuts: signed zeros in
    Tbu and fm, negative drag factors, zero strength, zero cell area (no
    Delta floor), resting ice with u0 = 0 (0/0 in Cb)."""
    pr = synth.make_problem("grid400x300", nx=60, ny=44, seed=13, ndte=7)
    rng = np.random.default_rng(9)
    n = pr.na
    pick = lambda f: rng.random(n) < f
    pr.f["Tbu"] = np.where(pick(0.3), -0.0, np.where(pick(0.3), 0.0, rng.uniform(0, 3, n)))
    pr.f["fm"] = np.where(pick(0.2), -0.0, np.where(pick(0.2), 0.0, pr.f["fm"]))
    pr.f["aiu"] = np.where(pick(0.1), -pr.f["aiu"], pr.f["aiu"])
    pr.f["strength"] = np.where(pick(0.1), 0.0, np.where(pick(0.05), -0.0, pr.f["strength"]))
    pr.f["dxT"] = np.where(pick(0.03), 0.0, pr.f["dxT"])
    rest = pick(0.1)
    pr.uvel[:n] = np.where(rest, 0.0, pr.uvel[:n])
    pr.vvel[:n] = np.where(rest, 0.0, pr.vvel[:n])
    pr.f["uvel_init"], pr.f["vvel_init"] = pr.uvel[:n].copy(), pr.vvel[:n].copy()
    p = evp1d.set_evp_parameters(7)
    p.u0 = u0
    fs = gpu_run(pr, 7, params=p)
    assert_same_nan_aware(fs, oracle_run(oracle_mod, pr, 7, params=p), pr)


def test_nonfinite_inputs(oracle_mod):
    """Non-finite and extreme inputs take the straight-line stress's fallback
    (NaN strain rates, strength at or above 1e300*DminArea) and propagate as
    the reference does: NaN velocities at some points, infinite and huge
    strength at others; NaNs are compared by position."""
    pr = synth.make_problem("grid400x300", nx=60, ny=44, seed=17, ndte=5)
    rng = np.random.default_rng(21)
    n = pr.na
    pick = lambda f: rng.random(n) < f
    pr.uvel[:n] = np.where(pick(0.01), np.nan, pr.uvel[:n])
    pr.vvel[:n] = np.where(pick(0.01), np.inf, pr.vvel[:n])
    pr.f["uvel_init"], pr.f["vvel_init"] = pr.uvel[:n].copy(), pr.vvel[:n].copy()
    pr.f["strength"] = np.where(pick(0.01), np.inf, np.where(pick(0.01), 1e305, pr.f["strength"]))
    fs = gpu_run(pr, 5)
    assert_same_nan_aware(fs, oracle_run(oracle_mod, pr, 5), pr)


@pytest.mark.parametrize("case", ["signed_zeros", "tbu_minus_zero", "tbu_nonzero",
                                  "uinit_inf", "revp_minus_zero", "compact_off"])
def test_short_stepu_part_edges(oracle_mod, monkeypatch, case):
    """The subcycle kernel copies a stepu part without Tbu, uinit and vinit
    when every Tbu of the call is +0 and every uinit, vinit is finite (with
    revp == 0): Tbu is then +0 and revp*uinit a zero with uinit's sign.
    Explicit uvel_init/vvel_init of both signs and signed zeros, velocities
    that are -0 (so brlx*uold + revp*uinit is a sum of two zeros), revp = -0,
    and fields that rule the short part out (Tbu = -0 or 1e-3 at one point,
    an infinite uinit): every case gives the oracle's bits."""
    if case == "compact_off":
        monkeypatch.setenv("EVP1D_COMPACT", "0")
    pr = synth.make_problem("grid400x300", nx=64, ny=40, seed=29, ndte=6)
    rng = np.random.default_rng(33)
    n = pr.na
    ui = rng.normal(0, 0.05, n)
    vi = rng.normal(0, 0.05, n)
    z = rng.random(n)
    ui = np.where(z < 0.1, 0.0, np.where(z < 0.2, -0.0, ui))
    vi = np.where(z > 0.9, -0.0, np.where(z > 0.8, 0.0, vi))
    pr.f["uvel_init"], pr.f["vvel_init"] = ui, vi
    w = rng.random(n)
    pr.uvel[:n] = np.where(w < 0.15, -0.0, pr.uvel[:n])
    pr.vvel[:n] = np.where(w > 0.85, -0.0, pr.vvel[:n])
    p = evp1d.set_evp_parameters(6)
    if case == "revp_minus_zero":
        p.revp = -0.0
    k = n // 3
    if case == "tbu_minus_zero":
        pr.f["Tbu"] = pr.f["Tbu"].copy()
        pr.f["Tbu"][k] = -0.0
    elif case == "tbu_nonzero":
        pr.f["Tbu"] = pr.f["Tbu"].copy()
        pr.f["Tbu"][k] = 1e-3
    elif case == "uinit_inf":
        pr.f["uvel_init"][k] = np.inf
    fs = gpu_run(pr, 6, params=p, explicit_init=True)
    assert_same_nan_aware(fs, oracle_run(oracle_mod, pr, 6, params=p), pr)


def test_params_change_between_calls_bitwise(oracle_mod):
    """One handle runs a call with the default parameters (revp = 0, Tbu = 0:
    the short stepu part, captured in graphs), then, after evp1d_set_params,
    a call with revised EVP (revp = 1), whose stepu needs uvel_init; then the
    defaults again.  Each call gives the oracle's bits for its parameters."""
    pr = synth.to_1d(synth.make_grid(120, 90, seed=81, ndte=120, curvilinear=True))
    rng = np.random.default_rng(8)
    pr.f["uvel_init"] = pr.f["uvel_init"] + rng.normal(0, 0.01, pr.na)
    p0 = evp1d.set_evp_parameters(120)
    p1 = evp1d.set_evp_parameters(120)
    p1.revp = 1.0
    with evp1d.EVP1D.from_problem(pr, ndte=120, params=p0) as s:
        for p in (p0, p1, p0):
            s.set_params(p)
            # uvel_init given explicitly, as the oracle reads it from the fields
            fs = evp1d.FieldSet.from_problem(pr, explicit_init=True)
            s.run(120, fs)
            assert_same(fs, oracle_run(oracle_mod, pr, 120, params=p), pr, check_str=False)


def test_concurrent_handles_bitwise(oracle_mod):
    """Three handles on their own streams, their calls issued back to back
    without waiting (each call's subcycle launches overlap the launch before
    them on the same stream, and the streams run side by side): every
    handle's results are the oracle's bits."""
    probs = [synth.to_1d(synth.make_grid(nx, ny, seed=70 + i, ndte=120, curvilinear=True))
             for i, (nx, ny) in enumerate([(90, 70), (150, 110), (60, 40)])]
    handles = [evp1d.EVP1D.from_problem(pr, ndte=120) for pr in probs]
    try:
        sets = [evp1d.FieldSet.from_problem(pr) for pr in probs]
        for h, fs in zip(handles, sets):
            h.upload(fs)
        for h in handles:
            h.subcycles(120)
        for h, fs in zip(handles, sets):
            h.download(fs)
    finally:
        for h in handles:
            h.finalize()
    for pr, fs in zip(probs, sets):
        assert_same(fs, oracle_run(oracle_mod, pr, 120), pr, check_str=False)


@pytest.mark.parametrize("points", [128, 200])
def test_smaller_tiles_bitwise(oracle_mod, points):
    """Plans with a smaller largest tile (evp1d_set_tile_points) give the same
    bits: the tile size is a performance choice only."""
    pr = synth.to_1d(synth.make_grid(131, 77, seed=9, ndte=13, curvilinear=True))
    old = evp1d.get_tile_points()
    try:
        evp1d.set_tile_points(points)
        assert evp1d.plan_stats(pr.na, pr.navel, pr.idx)["max_tile"] <= points
        fs = gpu_run(pr, 13)
    finally:
        evp1d.set_tile_points(old)
    assert_same(fs, oracle_run(oracle_mod, pr, 13), pr)


@pytest.mark.parametrize("strip_w,runs", [(1, 148), (7, 3), (48, 1), (48, 148), (128, 17)])
def test_plan_shapes_bitwise(oracle_mod, monkeypatch, strip_w, runs):
    """Strip widths and run counts (EVP1D_STRIP_W, EVP1D_RUNS) move the run
    boundaries, where a tile loses its previous table, and the share of
    points recomputed as forward halo: one-column strips recompute every
    nw/sw neighbour, one run chains every tile to its predecessor.  The bits
    stay the oracle's."""
    pr = synth.to_1d(synth.make_grid(131, 77, seed=9, ndte=7, curvilinear=True))
    monkeypatch.setenv("EVP1D_STRIP_W", str(strip_w))
    monkeypatch.setenv("EVP1D_RUNS", str(runs))
    assert_same(gpu_run(pr, 7), oracle_run(oracle_mod, pr, 7), pr)


@pytest.mark.parametrize("persist,pdl", [("0", "1"), ("0", "0"), ("1", "1")])
@pytest.mark.parametrize("ndte", [1, 2, 3, 49, 50, 51, 101])
def test_launch_modes_bitwise(oracle_mod, monkeypatch, persist, pdl, ndte):
    """A call's subcycles in one multi-subcycle launch (CTAs resident, per-tile
    counters between subcycles) or one launch per subcycle in graphs of 50,
    each launch after the first of a call or chunk a programmatic dependent
    of the one before (pdl) or not: the same bits, for odd and even counts
    and around the graph chunk."""
    monkeypatch.setenv("EVP1D_PERSIST", persist)
    monkeypatch.setenv("EVP1D_PDL", pdl)
    pr = synth.to_1d(synth.make_grid(97, 61, seed=31, ndte=ndte, curvilinear=True))
    assert_same(gpu_run(pr, ndte, calls=1), oracle_run(oracle_mod, pr, ndte), pr)


@pytest.mark.parametrize("strip_w,runs", [(64, 3), (48, 148), (8, 20)])
def test_multi_subcycle_launch_halo_gathers(oracle_mod, monkeypatch, strip_w, runs):
    """The multi-subcycle launch gathers the forward halo and the extra
    velocities with coherent loads, each gather lane issuing a batch before it
    stores any: wide strips (a run's first tile recomputes a whole row above
    it, up to 64 halo points, several batches per lane) and narrow ones (many
    halo points in every tile), the same bits as the oracle."""
    monkeypatch.setenv("EVP1D_PERSIST", "1")
    monkeypatch.setenv("EVP1D_STRIP_W", str(strip_w))
    monkeypatch.setenv("EVP1D_RUNS", str(runs))
    pr = synth.to_1d(synth.make_grid(131, 77, seed=9, ndte=9, curvilinear=True))
    assert_same(gpu_run(pr, 9, calls=1), oracle_run(oracle_mod, pr, 9), pr)


def test_tile_size_tuner():
    """evp1d.tune_tile_points times each candidate on the caller's problem
    (single and batched) and leaves the fastest set."""
    old = evp1d.get_tile_points()
    try:
        pr = synth.make_problem("grid400x300", nx=120, ny=90, ndte=4)
        best, times = evp1d.tune_tile_points(pr, candidates=(256, 128), nsub=4)
        assert set(times) == {256, 128} and best in times and evp1d.get_tile_points() == best
        assert all(t > 0 for t in times.values())
        members = [synth.make_problem("grid400x300", nx=nx, ny=ny, seed=60 + i, ndte=4)
                   for i, (nx, ny) in enumerate([(40, 30), (70, 55)])]
        best, times = evp1d.tune_tile_points(synth.concat(members), candidates=(192, 256), nsub=4)
        assert set(times) == {192, 256} and evp1d.get_tile_points() == best
    finally:
        evp1d.set_tile_points(old)


def test_golden_fixture_md5():
    """The CUDA path reproduces the committed fixture's md5s and arrays."""
    import golden_io
    pr, out, exp = golden_io.load()
    fs = gpu_run(pr, pr.ndte)
    f1, f2 = helpers.output_files(fs.stress, fs.strintx, fs.strinty, fs.uvel, fs.vvel, pr.skipU)
    assert helpers.md5(f1) == exp["md5_stress_v2"]
    assert helpers.md5(f2) == exp["md5_stepu_v2"]
    assert np.array_equal(fs.str.view(np.int64), out["str"].view(np.int64))


@pytest.mark.parametrize("tbu_member", [None, 3])
def test_batched_ensemble_matches_members(oracle_mod, tbu_member):
    """Uneven members solved in one handle give, member by member, bitwise the
    single-member results (and the oracle's); with basal stress in one
    member, the whole batch takes the full stepu part."""
    members = [synth.make_problem("grid400x300", nx=nx, ny=ny, seed=40 + i, ndte=8)
               for i, (nx, ny) in enumerate([(30, 20), (75, 41), (12, 9), (50, 60), (90, 17)])]
    if tbu_member is not None:
        m = members[tbu_member]
        m.f["Tbu"] = np.random.default_rng(7).uniform(0.0, 5.0, m.na)
    ens = synth.concat(members)
    fs = evp1d.FieldSet.from_problem(ens.combined, want_str=True)
    with evp1d.EVP1D.batched(ens, ndte=8) as s:
        s.run(8, fs)
    for m, pr in enumerate(members):
        st = oracle_run(oracle_mod, pr, 8)
        one = evp1d.FieldSet(pr.na, pr.navel, skipT=pr.skipT, skipU=pr.skipU,
                             stress=ens.split_points(fs.stress)[m],
                             uvel=ens.split_slots(fs.uvel)[m], vvel=ens.split_slots(fs.vvel)[m],
                             strintx=ens.split_points(fs.strintx)[m],
                             strinty=ens.split_points(fs.strinty)[m], Cb=ens.split_points(fs.Cb)[m],
                             want_str=True, **{k: pr.f[k] for k in evp1d.FieldSet.DYN})
        one.str[:] = ens.split_slots(fs.str)[m]
        assert_same(one, st, pr)


def _empty_member(like):
    z = np.zeros(0)
    zi = np.zeros(0, np.int32)
    return synth.Problem1D(na=0, navel=0, ndte=like.ndte, idx={k: zi.copy() for k in like.idx},
                           skipT=zi.copy(), skipU=zi.copy(), f={k: z.copy() for k in like.f},
                           stress=np.zeros((12, 0)), uvel=z.copy(), vvel=z.copy(),
                           strintx=z.copy(), strinty=z.copy(), Cb=z.copy())


def test_batched_ensemble_with_empty_and_one_point_members(oracle_mod):
    """Members without ice (na = 0: first, in the middle, last) and a member
    of one point whose neighbours are all halo slots sit beside ordinary
    members; every member still gets its own result bit for bit."""
    a = synth.make_problem("grid400x300", nx=40, ny=30, seed=61, ndte=6)
    b = synth.make_problem("grid400x300", nx=55, ny=25, seed=62, ndte=6)
    one = helpers.random_graph_problem(1, 6, 3)
    one.idx = {k: np.array([2 + i], np.int32) for i, k in enumerate(("ee", "ne", "se", "nw", "sw", "sse"))}
    one.navel = 7
    one.uvel = np.concatenate([one.uvel[:1], np.zeros(6)])
    one.vvel = np.concatenate([one.vvel[:1], np.zeros(6)])
    one.skipT[:] = 0
    one.skipU[:] = 0
    one.ndte = 6
    members = [_empty_member(a), a, _empty_member(a), one, b, _empty_member(a)]
    ens = synth.concat(members)
    fs = evp1d.FieldSet.from_problem(ens.combined)
    with evp1d.EVP1D.batched(ens, ndte=6) as s:
        s.run(6, fs)
    for m, pr in enumerate(members):
        if pr.na == 0:
            continue
        st = oracle_run(oracle_mod, pr, 6)
        got = evp1d.FieldSet(pr.na, pr.navel, skipT=pr.skipT, skipU=pr.skipU,
                             stress=ens.split_points(fs.stress)[m],
                             uvel=ens.split_slots(fs.uvel)[m], vvel=ens.split_slots(fs.vvel)[m],
                             strintx=ens.split_points(fs.strintx)[m],
                             strinty=ens.split_points(fs.strinty)[m],
                             Cb=ens.split_points(fs.Cb)[m],
                             **{k: pr.f[k] for k in evp1d.FieldSet.DYN})
        assert_same(got, st, pr)


def test_autotune_keeps_state(oracle_mod):
    pr = synth.make_problem("grid400x300", nx=120, ny=90, ndte=12)
    fs = evp1d.FieldSet.from_problem(pr, want_str=True)
    with evp1d.EVP1D.from_problem(pr, ndte=12) as s:
        s.upload(fs)
        choice = s.autotune(6)
        assert "us/subcycle" in choice
        s.subcycles(12)
        s.download(fs)
    assert_same(fs, oracle_run(oracle_mod, pr, 12), pr)


def test_reference_file_case_on_gpu(tmp_path):
    """A case in the reference's file formats, run on the GPU, reproduces the
    golden fixture's md5 sums (python -m evp1d.io)."""
    import golden_io
    from evp1d import io as evio
    pr, _, exp = golden_io.load()
    p = evp1d.set_evp_parameters(pr.ndte)
    evio.write_inputs(str(tmp_path), pr, dict(capping=p.capping, e_factor=p.e_factor,
                                              epp2i=p.epp2i, deltaminEVP=p.deltaminEVP))
    h = evio.run_case(str(tmp_path), pr.na, pr.navel, pr.ndte)
    assert h == (exp["md5_stress_v2"], exp["md5_stepu_v2"])


@pytest.mark.parametrize("curvilinear", [False, True])
def test_dyn2d_adapter_matches_v0(oracle_mod, curvilinear):
    """The 2D adapter (list = every ocean point, skip flags from the ice masks,
    as dyn_evp1d_init/run) against the oracle's v0 2D kernels (upstream CICE
    form): bitwise equal stresses, velocities and internal stress divergence."""
    from evp1d import dyn
    g = synth.make_grid(64, 50, seed=17, ndte=9, curvilinear=curvilinear)
    p = evp1d.set_evp_parameters(9)
    F = dyn.fields_from_grid(g)
    with dyn.Dyn2D(g.tmask, g.f["dyT"], g.f["dxT"], g.f["uarear"], g.f["HTE"],
                   g.f["HTN"], p) as d:
        na, navel = d.sizes
        assert na == int(g.tmask.sum())
        d.run(9, F, g.iceT, g.iceU)
    V = oracle_mod.run_v0(g, 9)
    for k in dyn.STRESS:
        assert np.array_equal(F[k].view(np.int64), V[k].view(np.int64)), k
    for mine, ref in (("uvel", "uvel"), ("vvel", "vvel"), ("strintxU", "strintx"),
                      ("strintyU", "strinty")):
        assert np.array_equal(F[mine].view(np.int64), V[ref].view(np.int64)), mine


def test_dyn2d_adapter_keeps_cells_outside_the_list(oracle_mod):
    """Cells outside the 1D list (land) keep whatever the caller passed, and
    a second call continues from the first call's state, as v0 does."""
    from evp1d import dyn
    g = synth.make_grid(48, 40, seed=19, ndte=6, curvilinear=True)
    p = evp1d.set_evp_parameters(6)
    F = dyn.fields_from_grid(g)
    land = ~np.asarray(g.tmask, dtype=bool)
    assert land.any()
    marks = {k: np.float64(1234.5 + i) for i, k in enumerate(list(dyn.STRESS) + ["uvel", "vvel", "strintxU"])}
    for k, v in marks.items():
        F[k][land] = v
    with dyn.Dyn2D(g.tmask, g.f["dyT"], g.f["dxT"], g.f["uarear"], g.f["HTE"],
                   g.f["HTN"], p) as d:
        d.run(6, F, g.iceT, g.iceU)
        d.run(6, F, g.iceT, g.iceU)
    for k, v in marks.items():
        assert np.all(F[k][land] == v), k
    G = dyn.fields_from_grid(g)
    with dyn.Dyn2D(g.tmask, g.f["dyT"], g.f["dxT"], g.f["uarear"], g.f["HTE"],
                   g.f["HTN"], p) as d:
        d.run(6, G, g.iceT, g.iceU)
        d.run(6, G, g.iceT, g.iceU)
    sea = ~land
    for k in list(dyn.STRESS) + ["uvel", "vvel", "strintxU", "strintyU", "Cb"]:
        assert np.array_equal(F[k][sea].view(np.int64), G[k][sea].view(np.int64)), k


def test_sharded_run_single_rank_gpu(oracle_mod):
    """The ensemble driver on one rank (no process group) solves its members
    on the GPU with the same summaries as the oracle."""
    from evp1d import ensemble
    members = [synth.make_problem("grid400x300", nx=nx, ny=25, seed=90 + i, ndte=5)
               for i, nx in enumerate([20, 47, 33])]
    got = ensemble.sharded_run(members, 5)
    for i, pr in enumerate(members):
        st = oracle_run(oracle_mod, pr, 5)
        want = ensemble.summarize(dict(stress=st.stress, uvel=st.uvel[: pr.navel],
                                       vvel=st.vvel[: pr.navel], strintx=st.strintx,
                                       strinty=st.strinty, Cb=st.Cb), pr.na)
        assert got[i] == want


def test_pinned_host_arrays_same_results(oracle_mod):
    """Fields in page-locked host memory (evp1d_host_alloc) give the same bits
    as pageable arrays, over two calls with a refill in between."""
    pr = synth.make_problem("grid400x300", nx=70, ny=55, ndte=9)
    a = evp1d.FieldSet.from_problem(pr, want_str=False)
    b = evp1d.FieldSet.from_problem(pr, want_str=False, pinned=True)
    with evp1d.EVP1D.from_problem(pr) as s:
        for _ in range(2):
            s.run(pr.ndte, a)
            s.run(pr.ndte, b)
            for x, y in ((a.stress, b.stress), (a.uvel, b.uvel), (a.vvel, b.vvel),
                         (a.strintx, b.strintx), (a.Cb, b.Cb)):
                assert np.array_equal(x.view(np.int64), y.view(np.int64))
        b.refill(pr)
        s.run(pr.ndte, b)
    assert_same(b, oracle_run(oracle_mod, pr, pr.ndte), pr, check_str=False)
