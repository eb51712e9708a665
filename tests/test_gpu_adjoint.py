"""GPU tests of the adjoint (evp1d_run_checkpointed + evp1d_adjoint) through
the C-ABI, against the taped FP64 torch restatement (oracle/evp_tape.py) and
central finite differences of the bit-exact GPU forward.

Tolerances: gradients agree with the tape to 1e-9 relative (max-norm over
the field; the two differ only by rounding order); directional derivatives
agree with central differences (step 1e-6 relative) to 1e-6 relative;
checkpointed and full-tape sweeps agree bit for bit; an ensemble member's
gradients agree with the member solved alone to 1e-10 relative.
"""
import numpy as np
import pytest

import evp1d
from evp1d import synth

pytestmark = pytest.mark.gpu

FIELDS = ("strength", "Cw", "forcex", "forcey")


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def small(seed=41, nx=60, ny=45, ndte=15, curvilinear=True):
    return synth.to_1d(synth.make_grid(nx, ny, seed=seed, ndte=ndte, curvilinear=curvilinear))


def gpu_grads(pr, ndte, uobs, vobs, interval=0, stress=False, lam_stress=None):
    fs = evp1d.FieldSet.from_problem(pr)
    with evp1d.EVP1D.from_problem(pr, ndte=ndte) as s:
        s.run_checkpointed(ndte, fs, interval)
        na = pr.na
        lu = 2.0 * (fs.uvel[:na] - uobs)
        lv = 2.0 * (fs.vvel[:na] - vobs)
        g = s.adjoint(lu, lv, lam_stress=lam_stress, stress=stress)
        info = s.adjoint_info()
    return g, fs, info


@pytest.mark.parametrize("curvilinear", [False, True])
@pytest.mark.parametrize("interval", [0, 4, 15, 40])
def test_adjoint_matches_tape(oracle_mod, curvilinear, interval):
    import evp_tape
    pr = small(curvilinear=curvilinear)
    ndte = pr.ndte
    uobs, vobs = synth.observations(pr.na, seed=77)
    p = evp1d.set_evp_parameters(ndte)
    g, fs, info = gpu_grads(pr, ndte, uobs, vobs, interval=interval, stress=True)
    assert info["valid"] == 1
    # interval mode tapes the last segment; the rest is checkpointed
    k = min(interval, ndte)
    assert info["tape_subcycles"] == (ndte if interval == 0 else ndte - k * ((ndte - 1) // k))
    assert info["checkpoints"] == (0 if interval == 0 else (ndte - 1) // k)
    t = evp_tape.gradient(pr, ndte, p, uobs, vobs)
    for k in FIELDS:
        assert rel(g[k], t[k]) < 1e-9, (k, rel(g[k], t[k]))
    assert rel(g["uvel"], t["uvel0"]) < 1e-9
    assert rel(g["vvel"], t["vvel0"]) < 1e-9
    assert rel(g["stress"], t["stress0"]) < 1e-9


def test_checkpointed_forward_is_the_forward(oracle_mod):
    """run_checkpointed returns exactly evp1d_run's outputs, in both modes."""
    pr = small(seed=43, ndte=23)
    ref = evp1d.FieldSet.from_problem(pr, want_str=True)
    with evp1d.EVP1D.from_problem(pr) as s:
        s.run(pr.ndte, ref)
    for interval in (0, 5, 50):
        fs = evp1d.FieldSet.from_problem(pr, want_str=True)
        with evp1d.EVP1D.from_problem(pr) as s:
            s.run_checkpointed(pr.ndte, fs, interval)
        for a, b in ((fs.stress, ref.stress), (fs.uvel, ref.uvel), (fs.vvel, ref.vvel),
                     (fs.strintx, ref.strintx), (fs.strinty, ref.strinty), (fs.Cb, ref.Cb),
                     (fs.str, ref.str)):
            assert np.array_equal(a.view(np.int64), b.view(np.int64))


def test_checkpoint_and_tape_sweeps_agree_bitwise():
    pr = small(seed=45, ndte=31)
    uobs, vobs = synth.observations(pr.na, seed=3)
    ga, _, ia = gpu_grads(pr, pr.ndte, uobs, vobs, interval=0)
    for interval in (1, 7, 31, 100):
        gb, _, ib = gpu_grads(pr, pr.ndte, uobs, vobs, interval=interval)
        # every interval but the last segment, which is taped
        assert ib["checkpoints"] == (pr.ndte - 1) // min(interval, pr.ndte)
        for k in ga:
            assert np.array_equal(ga[k].view(np.int64), gb[k].view(np.int64)), (interval, k)


def test_recordings_on_one_handle_and_constant_slots(oracle_mod):
    """Velocities at skipU points stay at their starting value through the
    call and enter the stress of neighbouring T points; with them nonzero,
    recordings of different layouts in a row on one handle (full tape, then
    checkpoints, then the tape again) give each mode's fresh-handle gradients
    bit for bit, and these match the tape oracle."""
    import evp_tape
    pr = small(seed=44, ndte=24)
    rng = np.random.default_rng(2)
    su = pr.skipU != 0
    assert su.any()
    pr.uvel[: pr.na][su] = rng.normal(0, 0.05, su.sum())
    pr.vvel[: pr.na][su] = rng.normal(0, 0.05, su.sum())
    pr.f["uvel_init"] = pr.uvel[: pr.na].copy()
    pr.f["vvel_init"] = pr.vvel[: pr.na].copy()
    uobs, vobs = synth.observations(pr.na, seed=9)
    fresh = {iv: gpu_grads(pr, pr.ndte, uobs, vobs, interval=iv)[0] for iv in (0, 5)}
    t = evp_tape.gradient(pr, pr.ndte, evp1d.set_evp_parameters(pr.ndte), uobs, vobs,
                          wrt=FIELDS)
    for k in FIELDS:
        assert rel(fresh[0][k], t[k]) < 1e-9, k
    with evp1d.EVP1D.from_problem(pr) as s:
        for iv in (0, 5, 0, 5):
            fs = evp1d.FieldSet.from_problem(pr)
            s.run_checkpointed(pr.ndte, fs, iv)
            g = s.adjoint(2 * (fs.uvel[: pr.na] - uobs), 2 * (fs.vvel[: pr.na] - vobs))
            for k in g:
                assert np.array_equal(g[k].view(np.int64), fresh[iv][k].view(np.int64)), (iv, k)


def test_memory_sized_recording_with_a_small_budget():
    """A budget halfway between the least a recording needs (checkpoints at
    the memory-minimising interval plus one segment of recompute space) and
    the full tape: the first subcycles are checkpointed and recomputed, the
    final ones taped; the forward outputs and the gradients are those of the
    full tape, bit for bit, and a second sweep of the same recording (whose
    segment recompute must not overwrite the taped tail) gives them again.
    The least recording (checkpoints only) gives the same gradients too."""
    pr = small(seed=46, ndte=60)
    uobs, vobs = synth.observations(pr.na, seed=4)
    ga, fa, ia = gpu_grads(pr, pr.ndte, uobs, vobs, interval=0)
    assert ia["tape_subcycles"] == pr.ndte
    full = ia["store_bytes"]
    with evp1d.EVP1D.from_problem(pr) as s:
        s.set_adjoint_budget(1)  # below the minimum: gets the minimum
        fl = evp1d.FieldSet.from_problem(pr)
        s.run_checkpointed(pr.ndte, fl, 0)
        least = s.adjoint_info()
        # every segment recomputed; only the last one's end state is not
        # stored already (no taped tail), so it alone is recomputed in full
        gl = s.adjoint(2 * (fl.uvel[: pr.na] - uobs), 2 * (fl.vvel[: pr.na] - vobs))
    assert least["tape_subcycles"] == 0 and least["checkpoints"] > 0, least
    for k in ga:
        assert np.array_equal(ga[k].view(np.int64), gl[k].view(np.int64)), k
    budget = (least["store_bytes"] + full) // 2
    fs = evp1d.FieldSet.from_problem(pr)
    with evp1d.EVP1D.from_problem(pr) as s:
        s.set_adjoint_budget(budget)
        s.run_checkpointed(pr.ndte, fs, 0)
        info = s.adjoint_info()
        g = s.adjoint(2 * (fs.uvel[: pr.na] - uobs), 2 * (fs.vvel[: pr.na] - vobs))
        g2 = s.adjoint(2 * (fs.uvel[: pr.na] - uobs), 2 * (fs.vvel[: pr.na] - vobs))
    assert 0 < info["tape_subcycles"] < pr.ndte and info["checkpoints"] > 0, info
    assert info["store_bytes"] <= budget
    for a, b in ((fs.uvel, fa.uvel), (fs.vvel, fa.vvel), (fs.stress, fa.stress)):
        assert np.array_equal(a.view(np.int64), b.view(np.int64))
    for k in ga:
        assert np.array_equal(ga[k].view(np.int64), g[k].view(np.int64)), k
        assert np.array_equal(g2[k].view(np.int64), g[k].view(np.int64)), k


def central_difference(run, pr, field, d, h, uobs, vobs):
    """(J(p + h d) - J(p - h d)) / 2h for J = sum (u-u_obs)^2 + (v-v_obs)^2,
    summed point by point as (u+ - u-)(u+ + u- - 2 u_obs) so that the
    difference does not cancel against the size of J."""
    prp, prm = pr.copy(), pr.copy()
    prp.f[field] = pr.f[field] + h * d
    prm.f[field] = pr.f[field] - h * d
    up, vp = run(prp)
    um, vm = run(prm)
    return float(np.sum((up - um) * (up + um - 2 * uobs) + (vp - vm) * (vp + vm - 2 * vobs))) / (2 * h)


def test_adjoint_matches_finite_differences():
    """grid400x300-sized grid (400 x 300), ndte = 120: directional derivatives of J
    along 8 random directions per field against central differences of the
    GPU forward, step 1e-6 relative."""
    pr = synth.make_problem("grid400x300")
    ndte = pr.ndte
    uobs, vobs = synth.observations(pr.na, seed=404)
    g, fs0, _ = gpu_grads(pr, ndte, uobs, vobs, interval=synth.ADJOINT_INTERVAL)
    na = pr.na
    rng = np.random.default_rng(8)
    h = 1e-6
    with evp1d.EVP1D.from_problem(pr, ndte=ndte) as s:
        def run(prx):
            fs = evp1d.FieldSet.from_problem(prx)
            s.run(ndte, fs)
            return fs.uvel[:na].copy(), fs.vvel[:na].copy()
        worst = {}
        for k in FIELDS:
            for _ in range(8):
                d = pr.f[k] * rng.standard_normal(na)
                fd = central_difference(run, pr, k, d, h, uobs, vobs)
                ad = float(np.dot(g[k], d))
                err = abs(fd - ad) / max(abs(ad), 1e-300)
                worst[k] = max(worst.get(k, 0.0), err)
                assert err <= 1e-6, (k, fd, ad)
    print("worst FD relative error per field", {k: f"{v:.1e}" for k, v in worst.items()})


def test_adjoint_is_linear_in_the_seed_and_reusable():
    pr = small(seed=47, ndte=12)
    fs = evp1d.FieldSet.from_problem(pr)
    rng = np.random.default_rng(1)
    a = rng.normal(size=(2, pr.na))
    b = rng.normal(size=(2, pr.na))
    with evp1d.EVP1D.from_problem(pr) as s:
        s.run_checkpointed(pr.ndte, fs, 5)
        ga = s.adjoint(a[0], a[1])
        gb = s.adjoint(b[0], b[1])
        gab = s.adjoint(a[0] + b[0], a[1] + b[1])
        ga2 = s.adjoint(a[0], a[1])
    for k in ga:
        assert rel(gab[k], ga[k] + gb[k]) < 1e-12, k
        assert np.array_equal(ga[k], ga2[k]), k


def test_adjoint_explicit_uvel_init(oracle_mod):
    """With uvel_init given, its gradient is reported apart (revp = 1 makes
    it nonzero) and matches the tape."""
    import evp_tape
    pr = small(seed=49, ndte=9)
    p = evp1d.set_evp_parameters(pr.ndte)
    p.revp = 1.0
    uobs, vobs = synth.observations(pr.na, seed=5)
    fs = evp1d.FieldSet.from_problem(pr, explicit_init=True)
    with evp1d.EVP1D.from_problem(pr, params=p) as s:
        s.run_checkpointed(pr.ndte, fs, 0)
        g = s.adjoint(2 * (fs.uvel[: pr.na] - uobs), 2 * (fs.vvel[: pr.na] - vobs), init=True)
    t = evp_tape.gradient(pr, pr.ndte, p, uobs, vobs,
                          wrt=("forcex", "uvel0", "vvel0", "uvel_init", "vvel_init"))
    assert np.abs(g["uvel_init"]).max() > 0
    assert rel(g["uvel_init"], t["uvel_init"]) < 1e-9
    assert rel(g["vvel_init"], t["vvel_init"]) < 1e-9
    assert rel(g["uvel"], t["uvel0"]) < 1e-9
    assert rel(g["forcex"], t["forcex"]) < 1e-9


def test_batched_adjoint_matches_members():
    members = [small(seed=51 + m, nx=30 + 17 * m, ny=28, ndte=20) for m in range(3)]
    ens = synth.concat(members)
    ndte = 20
    obs = [synth.observations(m.na, seed=600 + i) for i, m in enumerate(members)]
    uobs = np.concatenate([o[0] for o in obs])
    vobs = np.concatenate([o[1] for o in obs])
    fs = evp1d.FieldSet.from_problem(ens.combined)
    with evp1d.EVP1D.batched(ens, ndte=ndte) as s:
        s.run_checkpointed(ndte, fs, 0)
        # list-point velocities of the member-major layout
        u_list = np.concatenate([u[: m.na] for u, m in zip(ens.split_slots(fs.uvel), members)])
        v_list = np.concatenate([v[: m.na] for v, m in zip(ens.split_slots(fs.vvel), members)])
        g = s.adjoint(2 * (u_list - uobs), 2 * (v_list - vobs))
    off = 0
    for i, m in enumerate(members):
        gm, _, _ = gpu_grads(m, ndte, obs[i][0], obs[i][1], interval=0)
        for k in FIELDS:
            assert rel(g[k][off: off + m.na], gm[k]) <= 1e-10, (i, k)
        off += m.na


def test_adjoint_state_errors():
    pr = small(seed=53, ndte=4)
    fs = evp1d.FieldSet.from_problem(pr)
    z = np.zeros(pr.na)
    with evp1d.EVP1D.from_problem(pr) as s:
        with pytest.raises(evp1d.EVP1DError) as e:
            s.adjoint(z, z)
        assert e.value.code == -7
        s.run_checkpointed(pr.ndte, fs, 2)
        s.adjoint(z, z)
        s.upload(fs)  # new inputs drop the recording
        with pytest.raises(evp1d.EVP1DError) as e:
            s.adjoint(z, z)
        assert e.value.code == -7


def test_autograd_function_gradcheck():
    """torch.autograd.gradcheck of the library's adjoint (through the
    autograd binding) on a small problem: the full Jacobian of the final
    velocities with respect to the four fields against torch's numerical
    Jacobian of the GPU forward."""
    import torch
    from evp1d.autograd import evp_velocities
    pr = small(seed=55, nx=13, ny=11, ndte=6)
    with evp1d.EVP1D.from_problem(pr) as s:
        ins = tuple(torch.tensor(pr.f[k], dtype=torch.float64, requires_grad=True)
                    for k in ("strength", "Cw", "forcex", "forcey"))
        # relative perturbations: scale each input to order one
        scale = [float(np.abs(pr.f[k]).max()) or 1.0 for k in ("strength", "Cw", "forcex", "forcey")]
        xs = tuple((t / c).detach().requires_grad_(True) for t, c in zip(ins, scale))

        def f(a, b, c, d):
            return evp_velocities(s, pr, pr.ndte, a * scale[0], b * scale[1], c * scale[2],
                                  d * scale[3], interval=2)
        assert torch.autograd.gradcheck(f, xs, eps=1e-6, atol=1e-7, rtol=1e-4)


def test_autograd_function_matches_tape(oracle_mod):
    import torch
    import evp_tape
    from evp1d.autograd import evp_velocities
    pr = small(seed=57, ndte=10)
    uobs, vobs = synth.observations(pr.na, seed=11)
    with evp1d.EVP1D.from_problem(pr) as s:
        ins = [torch.tensor(pr.f[k], dtype=torch.float64, requires_grad=True) for k in FIELDS]
        u, v = evp_velocities(s, pr, pr.ndte, *ins)
        J = ((u - torch.from_numpy(uobs)) ** 2 + (v - torch.from_numpy(vobs)) ** 2).sum()
        J.backward()
    t = evp_tape.gradient(pr, pr.ndte, evp1d.set_evp_parameters(pr.ndte), uobs, vobs, wrt=FIELDS)
    for k, x in zip(FIELDS, ins):
        assert rel(x.grad.numpy(), t[k]) < 1e-9, k


@pytest.mark.parametrize("na,nhalo,seed", [(3000, 200, 4), (700, 9, 5)])
def test_adjoint_irregular_graph_matches_tape(oracle_mod, na, nhalo, seed):
    """Random (non-grid) neighbour vectors: points are read by several
    neighbours, so the transposed lists have many entries (the general gather
    path); gradients still match the tape."""
    import evp_tape
    import helpers
    pr = helpers.random_graph_problem(na, nhalo, seed)
    uobs, vobs = synth.observations(pr.na, seed=seed + 10)
    g, _, _ = gpu_grads(pr, pr.ndte, uobs, vobs, interval=2, stress=True)
    t = evp_tape.gradient(pr, pr.ndte, evp1d.set_evp_parameters(pr.ndte), uobs, vobs)
    for k in FIELDS:
        assert rel(g[k], t[k]) < 1e-9, (k, rel(g[k], t[k]))
    assert rel(g["uvel"], t["uvel0"]) < 1e-9
    assert rel(g["stress"], t["stress0"]) < 1e-9


def test_adjoint_general_parameters_match_tape(oracle_mod):
    """Every parameter branch at once (capping = 0, Ktens != 0, revised EVP,
    a turning angle) with a nonzero seabed stress: gradients match the tape."""
    import evp_tape
    pr = small(seed=59, ndte=8)
    rng = np.random.default_rng(9)
    pr.f["Tbu"] = np.where(rng.uniform(size=pr.na) < 0.5, 0.0, rng.uniform(0.0, 2.0, pr.na))
    p = evp1d.set_evp_parameters(pr.ndte)
    p.capping, p.Ktens, p.revp = 0.0, 0.3, 1.0
    p.cosw, p.sinw = float(np.cos(0.4)), float(np.sin(0.4))
    uobs, vobs = synth.observations(pr.na, seed=12)
    fs = evp1d.FieldSet.from_problem(pr)
    with evp1d.EVP1D.from_problem(pr, params=p) as s:
        s.run_checkpointed(pr.ndte, fs, 3)
        g = s.adjoint(2 * (fs.uvel[: pr.na] - uobs), 2 * (fs.vvel[: pr.na] - vobs), stress=True)
    t = evp_tape.gradient(pr, pr.ndte, p, uobs, vobs)
    for k in FIELDS:
        assert rel(g[k], t[k]) < 1e-9, (k, rel(g[k], t[k]))
    assert rel(g["uvel"], t["uvel0"]) < 1e-9
    assert rel(g["stress"], t["stress0"]) < 1e-9


@pytest.mark.parametrize("interval,persist", [(0, "0"), (3, "0"), (3, "1")])
def test_adjoint800x600_grid_matches_tape(oracle_mod, monkeypatch, interval, persist):
    """The adjoint benchmark's own grid (800 x 600, 294,541 points) at a
    reduced ndte, against the taped FP64 restatement: the gradients the bench
    differentiates are the tape's to 1e-9, so its finite-difference residuals
    are finite-difference error, not adjoint error.  interval = 3 recomputes
    checkpointed segments of three subcycles; with EVP1D_PERSIST=1 each
    segment, and the taped tail, is one multi-subcycle launch writing a tape
    entry per subcycle."""
    import evp_tape
    monkeypatch.setenv("EVP1D_PERSIST", persist)
    ndte = 7
    pr = synth.make_problem("adjoint800x600", ndte=ndte)
    assert pr.na > 250_000
    uobs, vobs = synth.observations(pr.na, seed=synth.CONFIGS["adjoint800x600"]["seed"] + 500)
    p = evp1d.set_evp_parameters(ndte)
    g, fs, info = gpu_grads(pr, ndte, uobs, vobs, interval=interval)
    assert info["valid"] == 1
    t = evp_tape.gradient(pr, ndte, p, uobs, vobs)
    for k in FIELDS:
        assert rel(g[k], t[k]) < 1e-9, (k, rel(g[k], t[k]))
