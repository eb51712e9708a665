"""CPU tests of the fused solver's tile plan (evp1d_plan_stats): grid tiles
are rebuilt from the neighbour graph whatever the list order, irregular
graphs fall back to consecutive points, and no tile exceeds its limits."""
import numpy as np
import pytest

import evp1d
from evp1d import synth
import helpers


TILE = 256  # kTileOwned (csrc/evp_tiles.h)


def stats(pr):
    return evp1d.plan_stats(pr.na, pr.navel, pr.idx)


def test_grid400x300_plan_uses_full_compact_tiles():
    pr = synth.make_problem("grid400x300")
    s = stats(pr)
    # Hilbert-curve runs of TILE points: tiles nearly full, forward halo small
    assert s["from_coords"] and s["max_halo"] <= 64 and s["max_tile"] <= TILE
    assert pr.na / s["tiles"] > 0.9 * TILE
    assert s["halo"] < 0.2 * s["slots"]


def test_shuffled_list_still_finds_grid():
    pr = synth.make_problem("grid400x300", nx=90, ny=70)
    a = stats(pr)
    b = stats(helpers.shuffle_problem(pr, 4))
    assert b["from_coords"]
    assert (a["tiles"], a["halo"]) == (b["tiles"], b["halo"])


@pytest.mark.parametrize("na,nhalo,seed", [(5000, 300, 0), (777, 5, 1), (1, 1, 2)])
def test_random_graph_falls_back(na, nhalo, seed):
    pr = helpers.random_graph_problem(na, nhalo, seed)
    s = stats(pr)
    assert s["max_halo"] <= 64 and s["max_tile"] <= TILE
    if na > 10:
        assert not s["from_coords"]


def test_standalone_plan():
    s = stats(helpers.standalone_problem())
    # 441 points in runs of TILE: two tiles
    assert s["from_coords"] and s["tiles"] == 2 and s["slots"] >= 441


def test_empty_plan():
    z = np.zeros(0, np.int32)
    s = evp1d.plan_stats(0, 0, {k: z for k in ("ee", "ne", "se", "nw", "sw", "sse")})
    assert s["tiles"] == 0 and s["slots"] == 0


def test_caps_are_reached_and_kept():
    """The two per-tile caps of the TMA kernel's shared-memory arrays: the
    forward halo (64 points) binds for a graph whose stress neighbours are a
    few shared slots, the extra velocities (128) for a random graph and for
    a grid; neither is exceeded."""
    pr = helpers.halo_limited_problem(3000, 50, 7)
    s = evp1d.plan_stats(pr.na, pr.navel, pr.idx)
    assert s["max_halo"] == 64 and s["max_extras"] <= 128, s
    pr = helpers.random_graph_problem(5000, 300, 0)
    s = evp1d.plan_stats(pr.na, pr.navel, pr.idx)
    assert s["max_extras"] == 128 and s["max_halo"] <= 64, s


def test_tile_points_setting():
    """evp1d_set_tile_points bounds the tiles of later plans; values outside
    32..256 are refused; 256 is the default."""
    pr = synth.make_problem("grid400x300", nx=80, ny=60, ndte=3)
    old = evp1d.get_tile_points()
    try:
        assert old == TILE
        for n in (128, 200):
            evp1d.set_tile_points(n)
            s = evp1d.plan_stats(pr.na, pr.navel, pr.idx)
            assert s["max_tile"] <= n and s["max_halo"] <= 64, (n, s)
        for bad in (0, 31, 257):
            with pytest.raises(evp1d.EVP1DError):
                evp1d.set_tile_points(bad)
        assert evp1d.get_tile_points() == 200
    finally:
        evp1d.set_tile_points(old)


# ---- the plan verifier (evp1d_plan_check) ------------------------------------

def _check(pr):
    evp1d.plan_check(pr.na, pr.navel, pr.idx)


@pytest.mark.parametrize("points", [256, 200, 128, 37])
def test_plan_check_passes_on_grids(points):
    old = evp1d.get_tile_points()
    try:
        evp1d.set_tile_points(points)
        _check(synth.to_1d(synth.make_grid(131, 77, seed=9, ndte=2, curvilinear=True)))
        _check(helpers.shuffle_problem(synth.make_problem("grid400x300", nx=90, ny=70, ndte=2), 3))
    finally:
        evp1d.set_tile_points(old)


def test_plan_check_passes_on_a_large_grid():
    """4.4 M points (3000 x 2400, 17,619 tiles, runs of up to 120 tiles):
    every packed index and range still decodes to what the neighbour
    vectors say, and the caps hold."""
    pr = synth.to_1d(synth.make_grid(3000, 2400, seed=5, ndte=2))
    st = stats(pr)
    assert pr.na > 4_000_000 and st["from_coords"]
    assert st["max_tile"] <= TILE and st["max_halo"] <= 64 and st["max_extras"] <= 128
    assert st["halo"] < 0.02 * pr.na
    evp1d.plan_check(pr.na, pr.navel, pr.idx)


def test_plan_check_passes_on_the_reference_shaped_problems():
    _check(synth.make_problem("grid400x300"))
    _check(helpers.standalone_problem())
    for na, nhalo, seed in ((5000, 300, 0), (777, 5, 1), (1, 1, 2)):
        _check(helpers.random_graph_problem(na, nhalo, seed))
    evp1d.plan_check(0, 0, {k: np.zeros(0, np.int32) for k in ("ee", "ne", "se", "nw", "sw", "sse")})


def test_plan_check_passes_on_band_problems():
    """The local problems of a state split into bands (ring points, ghost
    halo slots, partial rows)."""
    from evp1d import bands
    pr = synth.to_1d(synth.make_grid(131, 77, seed=9, ndte=2, curvilinear=True))
    for nb in (2, 5, pr.na // 40):
        for b in bands.split(pr, nb):
            _check(b.local)


@pytest.fixture(scope="module")
def plan_shim(tmp_path_factory):
    import ctypes as C
    import os
    import subprocess
    from conftest import PKG, ROOT
    out = str(tmp_path_factory.mktemp("plan") / "plan_check_shim.so")
    csrc = os.path.join(PKG, "csrc")
    subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-I", csrc,
                    os.path.join(csrc, "evp_tiles.cpp"), os.path.join(csrc, "evp_plan_check.cpp"),
                    os.path.join(ROOT, "tests", "native", "plan_check_shim.cpp"), "-o", out],
                   check=True)
    L = C.CDLL(out)
    L.shim_kinds.restype = C.c_int
    L.shim_plan_check.restype = C.c_longlong
    L.shim_plan_check.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_void_p), C.c_int, C.c_int,
                                  C.c_char_p, C.c_int]
    return L


@pytest.mark.parametrize("max_tile", [256, 128])
def test_plan_check_catches_planted_mistakes(plan_shim, max_tile):
    """One wrong index of each kind, planted in a plan on the host, is caught
    (the verifier is not vacuous)."""
    import ctypes as C
    pr = synth.to_1d(synth.make_grid(90, 60, seed=12, ndte=2, curvilinear=True))
    arrs = [np.ascontiguousarray(pr.idx[k], dtype=np.int32) for k in ("ee", "ne", "se", "nw", "sw", "sse")]
    ptrs = (C.c_void_p * 6)(*[a.ctypes.data for a in arrs])
    msg = C.create_string_buffer(256)
    assert plan_shim.shim_plan_check(pr.na, pr.navel, ptrs, max_tile, 0, msg, 256) == 0
    for kind in range(1, plan_shim.shim_kinds() + 1):
        n = plan_shim.shim_plan_check(pr.na, pr.navel, ptrs, max_tile, kind, msg, 256)
        assert n > 0, (kind, n)
        assert msg.value, kind
