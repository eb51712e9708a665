"""CPU checks of the adjoint's checkers: the taped torch restatement
(oracle/evp_tape.py) reproduces the bit-exact C oracle's forward to rounding,
and its autograd gradient matches central finite differences of the C
oracle's forward.  The GPU adjoint is compared with both in
test_gpu_adjoint.py."""
import numpy as np
import pytest

from evp1d import synth

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def tape():
    import evp_tape
    return evp_tape


def small_problem(seed=21, nx=34, ny=26, ndte=12, curvilinear=True):
    return synth.to_1d(synth.make_grid(nx, ny, seed=seed, ndte=ndte, curvilinear=curvilinear))


def oracle_J(oracle_mod, pr, ndte, uobs, vobs):
    st = oracle_mod.run_1d(pr, ndte)
    na = pr.na
    return float(np.sum((st.uvel[:na] - uobs) ** 2 + (st.vvel[:na] - vobs) ** 2)), st


@pytest.mark.parametrize("curvilinear", [False, True])
def test_tape_forward_matches_oracle(oracle_mod, tape, curvilinear):
    pr = small_problem(curvilinear=curvilinear)
    p = oracle_mod.params(pr.ndte)
    st = oracle_mod.run_1d(pr, pr.ndte, p=p)
    with torch.no_grad():
        u, v, S = tape.forward(pr, pr.ndte, p)
    scale = max(np.abs(st.uvel[: pr.na]).max(), 1e-30)
    assert np.abs(u.numpy() - st.uvel[: pr.na]).max() <= 1e-11 * scale
    assert np.abs(v.numpy() - st.vvel[: pr.na]).max() <= 1e-11 * scale
    sscale = max(np.abs(st.stress).max(), 1e-30)
    assert np.abs(S.numpy() - st.stress).max() <= 1e-11 * sscale


def test_tape_gradient_matches_finite_differences(oracle_mod, tape):
    """Directional derivatives of J along 6 random directions per field,
    central differences with a step of 1e-6 relative: agreement <= 1e-6."""
    pr = small_problem(seed=23, ndte=10)
    ndte = pr.ndte
    p = oracle_mod.params(ndte)
    uobs, vobs = synth.observations(pr.na, seed=99)
    g = tape.gradient(pr, ndte, p, uobs, vobs)
    rng = np.random.default_rng(5)
    h = 1e-6
    for field in ("strength", "Cw", "forcex", "forcey"):
        base = pr.f[field]
        for _ in range(6):
            r = rng.standard_normal(pr.na)
            d = base * r if np.any(base != 0) else r
            prp, prm = pr.copy(), pr.copy()
            prp.f[field] = base + h * d
            prm.f[field] = base - h * d
            Jp, _ = oracle_J(oracle_mod, prp, ndte, uobs, vobs)
            Jm, _ = oracle_J(oracle_mod, prm, ndte, uobs, vobs)
            fd = (Jp - Jm) / (2 * h)
            ad = float(np.dot(g[field], d))
            assert abs(fd - ad) <= 1e-6 * max(abs(ad), 1e-12 * abs(g["J"])), (field, fd, ad)


def test_tape_branches_and_zero_sqrt(oracle_mod, tape):
    """Zero initial velocities (every Delta and |u| start at 0) give finite
    gradients: a square root of 0 has derivative 0."""
    pr = small_problem(seed=25, ndte=4)
    pr.uvel[:] = 0.0
    pr.vvel[:] = 0.0
    p = oracle_mod.params(pr.ndte)
    uobs, vobs = synth.observations(pr.na, seed=7)
    g = tape.gradient(pr, pr.ndte, p, uobs, vobs)
    for k in ("strength", "Cw", "forcex", "forcey", "uvel0", "vvel0", "stress0"):
        assert np.all(np.isfinite(g[k])), k
