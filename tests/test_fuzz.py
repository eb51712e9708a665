"""Property-based tests on CPU (hypothesis, derandomized: the same examples
on every run).

- Tile plans of random ice masks verify (evp1d_plan_check): every index the
  kernels gather through is what the neighbour vectors say.  The masks range
  from noise of any density to stripes, checkerboards and isolated points,
  with the list in the reference's order or shuffled, and any tile size.
- A state split into bands gives the single-domain oracle run bit for bit,
  on random grids with any number of bands.
"""
import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

import evp1d
from evp1d import synth

NB = ("ee", "ne", "se", "nw", "sw", "sse")


def _mask(nx, ny, kind, density, seed):
    rng = np.random.default_rng(seed)
    if kind == "noise":
        m = rng.random((nx, ny)) < density
    elif kind == "stripes":
        m = np.zeros((nx, ny), bool)
        m[:, :: 2] = True
    elif kind == "checker":
        m = (np.add.outer(np.arange(nx), np.arange(ny)) % 2) == 0
    else:  # isolated points
        m = np.zeros((nx, ny), bool)
        m[:: 3, :: 3] = True
    m[0, :] = m[-1, :] = False  # ghost ring, as the reference's padding
    m[:, 0] = m[:, -1] = False
    return m


def _shuffled(ix, seed):
    """The same graph with the list points relabelled (halo slots keep their
    numbers)."""
    rng = np.random.default_rng(seed)
    na = ix.na
    perm = rng.permutation(na)
    inv = np.empty(na, np.int64)
    inv[perm] = np.arange(na)
    out = {}
    for k in NB:
        v = ix.nb[k].astype(np.int64)[inv]
        lst = v <= na
        v[lst] = perm[v[lst] - 1] + 1
        out[k] = v.astype(np.int32)
    return out


@settings(max_examples=60, deadline=None, derandomize=True,
          suppress_health_check=[HealthCheck.too_slow])
@given(nx=st.integers(3, 90), ny=st.integers(3, 90),
       kind=st.sampled_from(["noise", "stripes", "checker", "isolated"]),
       density=st.floats(0.02, 1.0), seed=st.integers(0, 2**31 - 1),
       points=st.sampled_from([32, 64, 100, 200, 256]), shuffle=st.booleans())
def test_random_mask_plans_verify(nx, ny, kind, density, seed, points, shuffle):
    ix = synth.build_index(_mask(nx, ny, kind, density, seed))
    idx = _shuffled(ix, seed) if shuffle else ix.nb
    old = evp1d.get_tile_points()
    try:
        evp1d.set_tile_points(points)
        evp1d.plan_check(ix.na, ix.navel, idx)
    finally:
        evp1d.set_tile_points(old)


@settings(max_examples=25, deadline=None, derandomize=True,
          suppress_health_check=[HealthCheck.too_slow])
@given(nx=st.integers(5, 45), ny=st.integers(5, 45), seed=st.integers(0, 10**6),
       curvilinear=st.booleans(), nbands=st.integers(1, 7))
def test_random_band_splits_match_the_single_domain_run(nx, ny, seed, curvilinear, nbands):
    import oracle
    from test_bands import _same, solve_in_process
    pr = synth.to_1d(synth.make_grid(nx, ny, seed=seed, ndte=3, curvilinear=curvilinear))
    if pr.na == 0:
        return
    _, res = solve_in_process(pr, nbands, 3)
    _same(res, oracle.run_1d(pr, 3), pr)
