"""Seeded synthetic sea-ice states for the EVP-1D solver.

The reference's own inputs (DMI operational fields, read by
src/vars.F90:2101-2135) are not distributed, so every workload here is built
from seeded random fields with the shapes and value ranges of the benchmark
configurations:

* a 2D B-grid of ``nx x ny`` T cells plus a one-cell ghost ring (land);
* land from smoothed Gaussian noise thresholded at its 20 % quantile;
* ice concentration ``aice = clip(0.5 + 0.5 * n, 0, 1)`` from a second smoothed
  field; an ice T cell is ocean with ``aice > 0.15``;
* the U point of T cell (i, j) is its north-east corner; it is an ice U point
  when the four T cells around it are ocean and their mean concentration
  exceeds 0.15;
* thickness ``h ~ U(0.1, 4)``, ``strength = 2.75e4 h exp(-20 (1 - aice))``,
  velocities ``~ N(0, 0.05)`` on ice U points (0 elsewhere), ocean currents
  ``~ N(0, 0.2)``, wind stress ``~ N(0, 0.1)``, ``Cw = 5.5e-3``,
  ``mass = 917 h aiu``, ``fm = 1.46e-4 mass``, ``umassdti = mass ndte / dt``,
  ``Tbu = 0``, all stresses 0.

The 1D list is every point that is an ice T point or an ice U point, in the
reference's j-outer / i-inner order (integration/ice_dyn_evp1d.F90:559-589);
``skipT``/``skipU`` mark the points that are not ice T / ice U points
(set_skipMe, integration/ice_dyn_evp1d.F90:521-537).  Neighbour indices and
halo slots follow convert_2d_1d_init (integration/ice_dyn_evp1d.F90:743-816).

All 2D arrays are Fortran-ordered ``[nx + 2, ny + 2]`` so that element
``a[i - 1, j - 1]`` is the reference's ``a(i, j)``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

STRESS_NAMES = (
    "stressp_1", "stressp_2", "stressp_3", "stressp_4",
    "stressm_1", "stressm_2", "stressm_3", "stressm_4",
    "stress12_1", "stress12_2", "stress12_3", "stress12_4",
)
# per-point inputs of stepu (src/bench_v2b.F90:444-458), in C-ABI order
STEPU_NAMES = (
    "Cw", "aiu", "uocn", "vocn", "waterx", "watery", "forcex", "forcey",
    "umassdti", "fm", "uarear", "Tbu",
)
STATIC_T_NAMES = ("dxT", "dyT", "HTE", "HTN", "HTEm1", "HTNm1")


def _smooth_noise(rng: np.random.Generator, shape, sigma: float) -> np.ndarray:
    """White noise low-passed by a Gaussian of width ``sigma`` cells,
    normalised to zero mean and unit variance."""
    white = rng.standard_normal(shape)
    kx = np.fft.fftfreq(shape[0])[:, None]
    ky = np.fft.rfftfreq(shape[1])[None, :]
    filt = np.exp(-2.0 * (np.pi * sigma) ** 2 * (kx * kx + ky * ky))
    f = np.fft.irfft2(np.fft.rfft2(white) * filt, s=shape)
    f -= f.mean()
    sd = f.std()
    return f / sd if sd > 0 else f


@dataclass
class Grid2D:
    """One sea-ice state on the 2D B-grid (Fortran order, ghost ring incl.)."""

    nx: int                 # interior T cells in x
    ny: int                 # interior T cells in y
    nghost: int
    ndte: int
    dt: float
    f: dict = field(default_factory=dict)  # name -> [nx+2g, ny+2g] float64 F-order
    tmask: np.ndarray = None  # ocean
    iceT: np.ndarray = None
    iceU: np.ndarray = None

    @property
    def nxt(self) -> int:
        return self.nx + 2 * self.nghost

    @property
    def nyt(self) -> int:
        return self.ny + 2 * self.nghost


def make_grid(nx: int, ny: int, seed: int, ndte: int = 120, dt: float = 1800.0,
              sigma: float = 6.0, land_frac: float = 0.2,
              curvilinear: bool = False, strength_scale: float = 1.0,
              forcing_sd: float = 0.0) -> Grid2D:
    """Build one synthetic state.

    ``curvilinear`` replaces the constant 10 km grid by per-cell edge lengths
    in [8, 12] km so that every geometric term of the stress kernel is
    non-zero (the constant grid makes dxhy = dyhx = 0).
    ``strength_scale`` and ``forcing_sd`` are the ensemble perturbations
    (strength x U(0.8, 1.2), wind stress + N(0, 0.02)).
    """
    g = 1
    nxt, nyt = nx + 2 * g, ny + 2 * g
    rng = np.random.default_rng(seed)
    land_noise = _smooth_noise(rng, (nxt, nyt), sigma)
    ice_noise = _smooth_noise(rng, (nxt, nyt), sigma)
    ocean = np.zeros((nxt, nyt), dtype=bool)
    interior = land_noise[g:nxt - g, g:nyt - g]
    thr = np.quantile(interior, land_frac)
    ocean[g:nxt - g, g:nyt - g] = interior >= thr
    aice = np.clip(0.5 + 0.5 * ice_noise, 0.0, 1.0) * ocean

    iceT = ocean & (aice > 0.15)
    # U point (i, j) = NE corner of T (i, j); its four T cells are
    # (i, j), (i+1, j), (i, j+1), (i+1, j+1).
    oc4 = np.zeros_like(ocean)
    oc4[:-1, :-1] = ocean[:-1, :-1] & ocean[1:, :-1] & ocean[:-1, 1:] & ocean[1:, 1:]
    aiu = np.zeros_like(aice)
    aiu[:-1, :-1] = 0.25 * (aice[:-1, :-1] + aice[1:, :-1] + aice[:-1, 1:] + aice[1:, 1:])
    iceU = oc4 & (aiu > 0.15)

    shp = (nxt, nyt)
    h = rng.uniform(0.1, 4.0, shp)
    fld = {}
    if curvilinear:
        fld["HTE"] = rng.uniform(8e3, 12e3, shp)
        fld["HTN"] = rng.uniform(8e3, 12e3, shp)
        fld["dxT"] = rng.uniform(8e3, 12e3, shp)
        fld["dyT"] = rng.uniform(8e3, 12e3, shp)
        fld["uarear"] = 1.0 / (fld["dxT"] * fld["dyT"])
    else:
        d = 1e4
        for k in ("HTE", "HTN", "dxT", "dyT"):
            fld[k] = np.full(shp, d)
        fld["uarear"] = np.full(shp, 1.0 / (d * d))
    fld["strength"] = strength_scale * 2.75e4 * h * np.exp(-20.0 * (1.0 - aice))
    u = rng.normal(0.0, 0.05, shp)
    v = rng.normal(0.0, 0.05, shp)
    fld["uvel"] = np.where(iceU, u, 0.0)
    fld["vvel"] = np.where(iceU, v, 0.0)
    fld["waterx"] = rng.normal(0.0, 0.2, shp)
    fld["watery"] = rng.normal(0.0, 0.2, shp)
    fld["uocn"] = fld["waterx"].copy()
    fld["vocn"] = fld["watery"].copy()
    fld["forcex"] = rng.normal(0.0, 0.1, shp)
    fld["forcey"] = rng.normal(0.0, 0.1, shp)
    if forcing_sd > 0:
        fld["forcex"] += rng.normal(0.0, forcing_sd, shp)
        fld["forcey"] += rng.normal(0.0, forcing_sd, shp)
    fld["Cw"] = np.full(shp, 5.5e-3)
    fld["aiu"] = aiu
    mass = 917.0 * h * aiu
    fld["umassdti"] = mass * ndte / dt
    fld["fm"] = 1.46e-4 * mass
    fld["Tbu"] = np.zeros(shp)
    for k in STRESS_NAMES:
        fld[k] = np.zeros(shp)
    fld["strintx"] = np.zeros(shp)
    fld["strinty"] = np.zeros(shp)
    fld["Cb"] = np.zeros(shp)
    fld = {k: np.asfortranarray(a, dtype=np.float64) for k, a in fld.items()}
    return Grid2D(nx=nx, ny=ny, nghost=g, ndte=ndte, dt=dt, f=fld,
                  tmask=ocean, iceT=iceT, iceU=iceU)


@dataclass
class Index1D:
    """The adapter's 1D index space (integration/ice_dyn_evp1d.F90:743-816)."""

    na: int
    navel: int
    indxti: np.ndarray   # [na] 1-based i
    indxtj: np.ndarray   # [na] 1-based j
    indxtij: np.ndarray  # [navel] 1-based linear index i + (j-1) nx
    nb: dict             # 'ee','ne','se','nw','sw','sse' -> [na] int32, 1-based


def build_index(mask: np.ndarray, nghost: int = 1) -> Index1D:
    """Vectorised restatement of calc_2d_indices_init + calc_navel +
    convert_2d_1d_init (integration/ice_dyn_evp1d.F90:559-589, 743-797,
    1047-1087): points in j-outer / i-inner order from ``1 + nghost``, halo
    slots sorted by linear index after the ``na`` list points, neighbour
    vectors as 1-based positions."""
    nx, ny = mask.shape
    sub = np.asarray(mask[nghost:, nghost:], dtype=bool)
    # Fortran order flatten: i fastest
    jj, ii = np.nonzero(sub.T)
    i = (ii + 1 + nghost).astype(np.int64)
    j = (jj + 1 + nghost).astype(np.int64)
    na = i.size
    lin = i + (j - 1) * nx
    offs = {
        "ee": lin - 1, "ne": lin - 1 - nx, "se": lin - nx,
        "nw": lin + 1, "sw": lin + 1 + nx, "sse": lin + nx,
    }
    allv = np.unique(np.concatenate([lin] + list(offs.values())))
    halo = np.setdiff1d(allv, lin, assume_unique=True)
    indxtij = np.concatenate([lin, halo])
    navel = indxtij.size
    order = np.argsort(indxtij, kind="stable")
    sorted_vals = indxtij[order]
    nb = {}
    for k, x in offs.items():
        pos = np.searchsorted(sorted_vals, x)
        assert np.all(sorted_vals[pos] == x)
        nb[k] = (order[pos] + 1).astype(np.int32)
    return Index1D(na=na, navel=navel, indxti=i.astype(np.int32),
                   indxtj=j.astype(np.int32), indxtij=indxtij.astype(np.int32),
                   nb=nb)


@dataclass
class Problem1D:
    """One EVP-1D problem in the reference's v2 layout (src/vars.F90:2054-2135).

    ``stress`` holds the 12 stress components [12, na]; ``uvel``/``vvel`` are
    [navel] with halo slots 0; every other per-point field is [na]."""

    na: int
    navel: int
    ndte: int
    idx: dict          # neighbour vectors, 1-based int32 [na]
    skipT: np.ndarray  # int32 [na]
    skipU: np.ndarray  # int32 [na]
    f: dict            # per-point float64 fields [na]
    stress: np.ndarray  # [12, na]
    uvel: np.ndarray   # [navel]
    vvel: np.ndarray   # [navel]
    strintx: np.ndarray
    strinty: np.ndarray
    Cb: np.ndarray
    indxti: np.ndarray = None
    indxtj: np.ndarray = None

    def copy(self) -> "Problem1D":
        return Problem1D(
            na=self.na, navel=self.navel, ndte=self.ndte,
            idx={k: v.copy() for k, v in self.idx.items()},
            skipT=self.skipT.copy(), skipU=self.skipU.copy(),
            f={k: v.copy() for k, v in self.f.items()},
            stress=self.stress.copy(), uvel=self.uvel.copy(),
            vvel=self.vvel.copy(), strintx=self.strintx.copy(),
            strinty=self.strinty.copy(), Cb=self.Cb.copy(),
            indxti=None if self.indxti is None else self.indxti.copy(),
            indxtj=None if self.indxtj is None else self.indxtj.copy())

    @property
    def n_active(self) -> int:
        """Points that are not both skipT and skipU (the unit of work)."""
        return int(np.count_nonzero((self.skipT == 0) | (self.skipU == 0)))


def to_1d(grid: Grid2D) -> Problem1D:
    """2D -> 1D conversion of one state (convert_2d_1d_init / _dyn,
    integration/ice_dyn_evp1d.F90:743-882)."""
    mask = grid.iceT | grid.iceU
    ix = build_index(mask, grid.nghost)
    i0 = ix.indxti - 1
    j0 = ix.indxtj - 1
    F = grid.f
    f = {}
    for k in ("dxT", "dyT", "HTE", "HTN", "strength") + STEPU_NAMES:
        f[k] = np.ascontiguousarray(F[k][i0, j0])
    f["HTEm1"] = np.ascontiguousarray(F["HTE"][i0 - 1, j0])
    f["HTNm1"] = np.ascontiguousarray(F["HTN"][i0, j0 - 1])
    f["uvel_init"] = np.ascontiguousarray(F["uvel"][i0, j0])
    f["vvel_init"] = np.ascontiguousarray(F["vvel"][i0, j0])
    stress = np.stack([F[k][i0, j0] for k in STRESS_NAMES]).astype(np.float64)
    uvel = np.zeros(ix.navel)
    vvel = np.zeros(ix.navel)
    uvel[: ix.na] = F["uvel"][i0, j0]
    vvel[: ix.na] = F["vvel"][i0, j0]
    return Problem1D(
        na=ix.na, navel=ix.navel, ndte=grid.ndte, idx=ix.nb,
        skipT=(~grid.iceT[i0, j0]).astype(np.int32),
        skipU=(~grid.iceU[i0, j0]).astype(np.int32),
        f=f, stress=np.ascontiguousarray(stress), uvel=uvel, vvel=vvel,
        strintx=np.ascontiguousarray(F["strintx"][i0, j0]),
        strinty=np.ascontiguousarray(F["strinty"][i0, j0]),
        Cb=np.ascontiguousarray(F["Cb"][i0, j0]),
        indxti=ix.indxti, indxtj=ix.indxtj)


# Benchmark configurations (shapes of the reference's evaluation cases).
CONFIGS = {
    "grid400x300": dict(nx=400, ny=300, seed=1, ndte=120),
    "grid1600x1200": dict(nx=1600, ny=1200, seed=2, ndte=1000),
    # adjoint workload: 800 x 600, ndte = 500, checkpoints every 50 subcycles
    "adjoint800x600": dict(nx=800, ny=600, seed=4, ndte=500),
}

ADJOINT_INTERVAL = 50


def observations(na: int, seed: int) -> tuple:
    """u_obs, v_obs ~ N(0, 0.1) m/s at the list points (a seed of their own)
    for the misfit J = sum (u-u_obs)^2 + (v-v_obs)^2."""
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, 0.1, na), rng.normal(0.0, 0.1, na)


def make_problem(name: str = "grid400x300", **over) -> Problem1D:
    kw = dict(CONFIGS[name])
    kw.update(over)
    return to_1d(make_grid(**kw))


def make_ensemble(n_members: int, ny: int, nx_lo: int, nx_hi: int, seed: int,
                  ndte: int) -> list:
    """Ensemble members with uneven domains: nx ~ U(nx_lo, nx_hi), per-member
    seed = seed + m, strength x U(0.8, 1.2), wind stress + N(0, 0.02)."""
    rng = np.random.default_rng(seed)
    nxs = rng.integers(nx_lo, nx_hi + 1, size=n_members)
    scales = rng.uniform(0.8, 1.2, size=n_members)
    out = []
    for m in range(n_members):
        g = make_grid(int(nxs[m]), ny, seed + 1 + m, ndte=ndte,
                      strength_scale=float(scales[m]), forcing_sd=0.02)
        out.append(to_1d(g))
    return out


@dataclass
class Ensemble:
    """Members concatenated member-major, the layout of evp1d_init_batched:
    per-point arrays back to back, u/v with each member's halo slots after its
    own list points, neighbour vectors 1-based within each member."""

    members: list
    combined: Problem1D   # na = sum(na), navel = sum(navel); idx member-local
    na: np.ndarray        # [nmembers] int32
    navel: np.ndarray     # [nmembers] int32

    def split_points(self, a: np.ndarray) -> list:
        """Per-member views of a concatenated per-point array ([..., sum(na)])."""
        o = np.concatenate([[0], np.cumsum(self.na)])
        return [a[..., o[m]:o[m + 1]] for m in range(len(self.members))]

    def split_slots(self, a: np.ndarray) -> list:
        """Per-member views of a concatenated u/v/str array ([..., sum(navel)])."""
        o = np.concatenate([[0], np.cumsum(self.navel)])
        return [a[..., o[m]:o[m + 1]] for m in range(len(self.members))]


def concat(members: list) -> Ensemble:
    na = np.array([m.na for m in members], dtype=np.int32)
    navel = np.array([m.navel for m in members], dtype=np.int32)
    cat = lambda xs: np.concatenate(xs) if xs else np.zeros(0)
    f = {k: cat([m.f[k] for m in members]) for k in members[0].f}
    idx = {k: cat([m.idx[k] for m in members]).astype(np.int32) for k in members[0].idx}
    comb = Problem1D(
        na=int(na.sum()), navel=int(navel.sum()), ndte=members[0].ndte, idx=idx,
        skipT=cat([m.skipT for m in members]).astype(np.int32),
        skipU=cat([m.skipU for m in members]).astype(np.int32), f=f,
        stress=np.concatenate([m.stress for m in members], axis=1),
        uvel=cat([m.uvel for m in members]), vvel=cat([m.vvel for m in members]),
        strintx=cat([m.strintx for m in members]), strinty=cat([m.strinty for m in members]),
        Cb=cat([m.Cb for m in members]))
    return Ensemble(members=members, combined=comb, na=na, navel=navel)


# Ensemble configurations (uneven member domains).
ENSEMBLES = {
    "ens64": dict(n_members=64, ny=300, nx_lo=100, nx_hi=1300, seed=3, ndte=500),
    # batched adjoint: gradients of the misfit with respect to forcex, forcey
    "adjoint_ens32": dict(n_members=32, ny=600, nx_lo=300, nx_hi=1300, seed=5, ndte=1000),
}
