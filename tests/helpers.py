"""Test helpers: small workloads and output comparison."""
from __future__ import annotations

import hashlib

import numpy as np

from evp1d import synth


def standalone_grid(ndte: int = 1, strength: float = 0.0) -> synth.Grid2D:
    """The integration smoke-test state (integration/ice_dyn_evp1d_standalone.F90:
    60-79, 108-115): a 100 x 120 block (ghosts included), a 21 x 21 ocean/ice
    square at i, j = 20..40, umassdti = 1, aiu = 0.9, dxT = dyT = 1,
    uarear = 2, HTE = HTN = 1, uvel = 0.3, vvel = -0.3, stressp_1..4 = 1..4,
    stressm_1..4 = 5..8.  Fields the reference leaves unset are 0 here; the
    strength is a parameter (0 gives the closed-form answer of
    stress_k(n) = stress_k(0) * denom1**n)."""
    nxt, nyt = 100, 120
    g = synth.Grid2D(nx=nxt - 2, ny=nyt - 2, nghost=1, ndte=ndte, dt=1800.0)
    sq = np.zeros((nxt, nyt), dtype=bool)
    sq[19:40, 19:40] = True
    g.tmask, g.iceT, g.iceU = sq, sq.copy(), sq.copy()
    z = lambda: np.zeros((nxt, nyt), order="F")
    f = {k: z() for k in synth.STRESS_NAMES}
    for k in range(4):
        f[synth.STRESS_NAMES[k]][:] = 1.0 + k
        f[synth.STRESS_NAMES[4 + k]][:] = 5.0 + k
    for k in ("strength", "Cw", "uocn", "vocn", "waterx", "watery", "forcex",
              "forcey", "fm", "Tbu", "strintx", "strinty", "Cb"):
        f[k] = z()
    f["strength"][:] = strength
    f["umassdti"] = z() + 1.0
    f["aiu"] = z() + 0.9
    f["dxT"] = z() + 1.0
    f["dyT"] = z() + 1.0
    f["uarear"] = z() + 2.0
    f["HTE"] = z() + 1.0
    f["HTN"] = z() + 1.0
    f["uvel"] = z() + 0.3
    f["vvel"] = z() - 0.3
    g.f = f
    return g


def standalone_problem(ndte: int = 1, strength: float = 0.0) -> synth.Problem1D:
    """1D form of :func:`standalone_grid`; halo velocities are 0 as the adapter
    sets them (integration/ice_dyn_evp1d.F90:880-881)."""
    return synth.to_1d(standalone_grid(ndte, strength))


def output_files(stress, strintx, strinty, uvel, vvel, skipU):
    """The two output files of the reference (src/vars.F90:2233-2304)."""
    na = stress.shape[1]
    keep = np.asarray(skipU[:na]) == 0
    f1 = np.ascontiguousarray(stress, dtype="<f8").tobytes()
    f2 = b"".join(np.ascontiguousarray(np.asarray(a)[:na][keep], dtype="<f8").tobytes()
                  for a in (strintx, strinty, uvel, vvel))
    return f1, f2


def md5(b: bytes) -> str:
    return hashlib.md5(b).hexdigest()


def first_mismatch(a: np.ndarray, b: np.ndarray) -> str:
    """Describe the first bitwise difference of two float64 arrays."""
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    b = np.asarray(b, dtype=np.float64).reshape(-1)
    if a.shape != b.shape:
        return f"shape {a.shape} vs {b.shape}"
    ne = np.nonzero(a.view(np.int64) != b.view(np.int64))[0]
    if ne.size == 0:
        return "identical"
    i = ne[0]
    rel = np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))
    return f"{ne.size} differ; first at {i}: {a[i]!r} vs {b[i]!r}; max rel {rel:.3e}"


def shuffle_problem(pr: synth.Problem1D, seed: int) -> synth.Problem1D:
    """Relabel the list points in a random order (halo slots keep their
    numbers).  Every point computes the same values, so results are the
    original ones permuted; the solver must rebuild the grid from the graph."""
    rng = np.random.default_rng(seed)
    na = pr.na
    perm = rng.permutation(na)          # new position of old point p
    inv = np.empty(na, np.int64)
    inv[perm] = np.arange(na)           # old point at new position q
    q = pr.copy()
    def remap(v):
        v = v.astype(np.int64)
        out = v.copy()
        m = v <= na
        out[m] = perm[v[m] - 1] + 1
        return out.astype(np.int32)
    q.idx = {k: remap(v)[inv] for k, v in pr.idx.items()}
    q.skipT, q.skipU = pr.skipT[inv], pr.skipU[inv]
    q.f = {k: v[inv] for k, v in pr.f.items()}
    q.stress = pr.stress[:, inv]
    q.uvel = np.concatenate([pr.uvel[:na][inv], pr.uvel[na:]])
    q.vvel = np.concatenate([pr.vvel[:na][inv], pr.vvel[na:]])
    q.strintx, q.strinty, q.Cb = pr.strintx[inv], pr.strinty[inv], pr.Cb[inv]
    q.indxti = q.indxtj = None
    return q


def random_graph_problem(na: int, nhalo: int, seed: int) -> synth.Problem1D:
    """A 1D problem whose neighbour vectors are random slots: no grid layout
    exists, which exercises the consecutive-point tiling and halo splitting."""
    rng = np.random.default_rng(seed)
    navel = na + nhalo
    base = synth.make_problem("grid400x300", nx=60, ny=50, seed=seed, ndte=5)
    reps = -(-na // base.na)
    f = {k: np.tile(v, reps)[:na].copy() for k, v in base.f.items()}
    idx = {k: rng.integers(1, navel + 1, na).astype(np.int32)
           for k in ("ee", "ne", "se", "nw", "sw", "sse")}
    skipT = (rng.random(na) < 0.1).astype(np.int32)
    skipU = (rng.random(na) < 0.1).astype(np.int32)
    uvel = np.concatenate([rng.normal(0, 0.05, na), np.zeros(nhalo)])
    vvel = np.concatenate([rng.normal(0, 0.05, na), np.zeros(nhalo)])
    f["uvel_init"], f["vvel_init"] = uvel[:na].copy(), vvel[:na].copy()
    return synth.Problem1D(na=na, navel=navel, ndte=5, idx=idx, skipT=skipT,
                           skipU=skipU, f=f, stress=np.zeros((12, na)),
                           uvel=uvel, vvel=vvel, strintx=np.zeros(na),
                           strinty=np.zeros(na), Cb=np.zeros(na))


def halo_limited_problem(na: int, nhalo: int, seed: int, nshared: int = 2) -> synth.Problem1D:
    """A random-graph problem whose stress neighbours (ee, ne, se) all point at
    `nshared` slots while the stepu neighbours (nw, sw, sse) stay random: each
    point brings three new forward-halo points but almost no extra velocities,
    so the tile plan cuts its tiles at the forward-halo cap (64 points)."""
    pr = random_graph_problem(na, nhalo, seed)
    rng = np.random.default_rng(seed + 1000)
    shared = rng.integers(1, pr.navel + 1, nshared).astype(np.int32)
    for k in ("ee", "ne", "se"):
        pr.idx[k] = rng.choice(shared, pr.na).astype(np.int32)
    return pr
