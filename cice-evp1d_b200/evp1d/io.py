"""The reference's 1D file formats (stream binary, native little-endian, no
record markers), so that cases prepared for the Fortran benchmark run here:

* ``input_double_1d_v2.bin``  -- src/vars.F90:2104-2117 (readin_1d_v2):
  strength[na], uvel[navel], vvel[navel], dxt, dyt, uarear, cdn_ocn, aiu,
  uocn, vocn, waterxU, wateryU, forcexU, forceyU, umassdti, fmU, strintxU,
  strintyU, Tbu, stressp_1..4, stressm_1..4, stress12_1..4 [na each], the
  scalars capping, e_factor, epp2i, deltaminEVP, then HTE, HTN, HTEm1, HTNm1;
* ``input_integer_1d.bin``    -- ee, ne, se, nw, sw, sse [na each, int32]
  (src/vars.F90:2122-2124);
* ``input_logical_1d.bin``    -- skipUcell1d, skipTcell1d [na each, 4-byte
  logicals, nonzero = .true.] (src/vars.F90:2132-2134);
* ``output_stress_<id>_1d.bin`` / ``output_stepu_<id>_1d.bin`` --
  src/vars.F90:2233-2304 (writeout_1d): the 12 stresses [na each]; then
  strintx, strinty, uvel, vvel compacted over the points that are not skipU.

``python -m evp1d.io <dir> [--ndte N] [--id b200] [--stats]`` runs a case
directory on the GPU the way src/evp_v2b.F90:57-123 does, writes its two
output files and, with --stats, prints the reference's output statistics.
"""
from __future__ import annotations

import argparse
import hashlib
import os

import numpy as np

from .synth import Problem1D

_DBL_NA_1 = ("strength",)
_DBL_NA_2 = ("dxT", "dyT", "uarear", "Cw", "aiu", "uocn", "vocn", "waterx", "watery",
             "forcex", "forcey", "umassdti", "fm", "strintx", "strinty", "Tbu")
_HT = ("HTE", "HTN", "HTEm1", "HTNm1")
_SCAL = ("capping", "e_factor", "epp2i", "deltaminEVP")
_NB = ("ee", "ne", "se", "nw", "sw", "sse")


def write_inputs(path: str, pr: Problem1D, scalars: dict) -> None:
    """Write the three input files of problem `pr`; `scalars` gives capping,
    e_factor, epp2i and deltaminEVP."""
    os.makedirs(path, exist_ok=True)
    f = dict(pr.f)
    f["strintx"], f["strinty"] = pr.strintx, pr.strinty
    parts = [pr.f["strength"], pr.uvel, pr.vvel]
    parts += [f[k] for k in _DBL_NA_2]
    parts += [pr.stress[k] for k in range(12)]
    parts += [np.array([scalars[k] for k in _SCAL])]
    parts += [pr.f[k] for k in _HT]
    with open(os.path.join(path, "input_double_1d_v2.bin"), "wb") as fh:
        for a in parts:
            fh.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
    with open(os.path.join(path, "input_integer_1d.bin"), "wb") as fh:
        for k in _NB:
            fh.write(np.ascontiguousarray(pr.idx[k], dtype="<i4").tobytes())
    with open(os.path.join(path, "input_logical_1d.bin"), "wb") as fh:
        fh.write(np.ascontiguousarray(pr.skipU != 0, dtype="<i4").tobytes())
        fh.write(np.ascontiguousarray(pr.skipT != 0, dtype="<i4").tobytes())


def read_inputs(path: str, na: int, navel: int, ndte: int = 1):
    """Read a case written in the reference's v2 layout.  Returns the
    Problem1D (uvel_init = uvel, as src/vars.F90:2119-2120) and the dict of the
    four scalars the file carries."""
    d = np.fromfile(os.path.join(path, "input_double_1d_v2.bin"), dtype="<f8")
    want = na * (1 + len(_DBL_NA_2) + 12 + len(_HT)) + 2 * navel + len(_SCAL)
    if d.size != want:
        raise ValueError(f"input_double_1d_v2.bin holds {d.size} doubles, expected {want} "
                         f"for na={na}, navel={navel}")
    o = 0

    def take(n):
        nonlocal o
        a = d[o:o + n].copy()
        o += n
        return a
    f = {"strength": take(na)}
    uvel, vvel = take(navel), take(navel)
    for k in _DBL_NA_2:
        f[k] = take(na)
    stress = np.stack([take(na) for _ in range(12)])
    scal = dict(zip(_SCAL, take(len(_SCAL)).tolist()))
    for k in _HT:
        f[k] = take(na)
    ints = np.fromfile(os.path.join(path, "input_integer_1d.bin"), dtype="<i4")
    if ints.size != 6 * na:
        raise ValueError("input_integer_1d.bin has the wrong size")
    idx = {k: ints[i * na:(i + 1) * na].astype(np.int32) for i, k in enumerate(_NB)}
    logi = np.fromfile(os.path.join(path, "input_logical_1d.bin"), dtype="<i4")
    if logi.size != 2 * na:
        raise ValueError("input_logical_1d.bin has the wrong size")
    skipU = (logi[:na] != 0).astype(np.int32)
    skipT = (logi[na:] != 0).astype(np.int32)
    strintx, strinty = f.pop("strintx"), f.pop("strinty")
    f["uvel_init"], f["vvel_init"] = uvel[:na].copy(), vvel[:na].copy()
    pr = Problem1D(na=na, navel=navel, ndte=ndte, idx=idx, skipT=skipT, skipU=skipU,
                   f=f, stress=stress, uvel=uvel, vvel=vvel, strintx=strintx,
                   strinty=strinty, Cb=np.zeros(na))
    return pr, scal


def output_bytes(stress, strintx, strinty, uvel, vvel, skipU) -> tuple:
    """The contents of the two output files (writeout_1d, src/vars.F90:2233-2304)."""
    na = np.asarray(stress).shape[1]
    keep = np.asarray(skipU[:na]) == 0
    a = np.ascontiguousarray(stress, dtype="<f8").tobytes()
    b = b"".join(np.ascontiguousarray(np.asarray(x)[:na][keep], dtype="<f8").tobytes()
                 for x in (strintx, strinty, uvel, vvel))
    return a, b


def write_outputs(path: str, ident: str, stress, strintx, strinty, uvel, vvel, skipU) -> tuple:
    """Write output_stress_<id>_1d.bin and output_stepu_<id>_1d.bin; returns
    their md5 sums (the reference's correctness check, README.md:44-127)."""
    a, b = output_bytes(stress, strintx, strinty, uvel, vvel, skipU)
    names = (f"output_stress_{ident}_1d.bin", f"output_stepu_{ident}_1d.bin")
    for n, x in zip(names, (a, b)):
        with open(os.path.join(path, n), "wb") as fh:
            fh.write(x)
    return hashlib.md5(a).hexdigest(), hashlib.md5(b).hexdigest()


_STRESS_LABELS = ([f" stressp_{k}:" for k in range(1, 5)] + [f" stressm_{k}:" for k in range(1, 5)]
                  + [f"stress12_{k}:" for k in range(1, 5)])


def output_statistics(stress, strs, strintx, strinty, uvel, vvel) -> list:
    """The lines of the reference's output statistics (stat_out_1d,
    src/vars.F90:2209-2232): label, min, max and sum of the 12 stresses [na],
    str1..str8 [navel] (when given), strintx, strinty [na] and uvel, vvel
    [navel], in Fortran's a11,3f25.8 layout.  The sums are numpy's, whose
    summation order is not Fortran's, so they agree to rounding only: a
    diagnostic, not a bitwise check."""
    def line(label, a):
        a = np.asarray(a, dtype=np.float64)
        return f"{label:>11}{a.min():25.8f}{a.max():25.8f}{a.sum():25.8f}"
    out = [line(lab, stress[k]) for k, lab in enumerate(_STRESS_LABELS)]
    if strs is not None:
        out += [line(f"str{k + 1}:", strs[k]) for k in range(8)]
    out += [line("strintx:", strintx), line("strinty:", strinty),
            line("uvel:", uvel), line("vvel:", vvel)]
    return out


def run_case(path: str, na: int, navel: int, ndte: int, ident: str = "b200",
             device: int = 0, stats: bool = False) -> tuple:
    """Read a case, run ndte subcycles on the GPU with set_evp_parameters(ndte)
    overridden by the file's four scalars (src/evp_v2b.F90:63, 68), write the
    outputs, return their md5 sums (and, with stats, the output statistics
    lines of output_statistics)."""
    import evp1d
    pr, scal = read_inputs(path, na, navel, ndte)
    p = evp1d.set_evp_parameters(ndte)
    for k, v in scal.items():
        setattr(p, k, v)
    fs = evp1d.FieldSet.from_problem(pr, explicit_init=True, want_str=stats)
    with evp1d.EVP1D.from_problem(pr, params=p, device=device) as s:
        s.run(ndte, fs)
    sums = write_outputs(path, ident, fs.stress, fs.strintx, fs.strinty, fs.uvel,
                         fs.vvel, pr.skipU)
    if not stats:
        return sums
    return sums + (output_statistics(fs.stress, fs.str, fs.strintx, fs.strinty,
                                     fs.uvel, fs.vvel),)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("dir")
    ap.add_argument("--na", type=int, required=True)
    ap.add_argument("--navel", type=int, required=True)
    ap.add_argument("--ndte", type=int, default=1)
    ap.add_argument("--id", default="b200")
    ap.add_argument("--stats", action="store_true",
                    help="print the reference's output statistics (stat_out_1d)")
    a = ap.parse_args(argv)
    res = run_case(a.dir, a.na, a.navel, a.ndte, a.id, stats=a.stats)
    if a.stats:
        print("\n".join(res[2]))
    print(f"{res[0]}  output_stress_{a.id}_1d.bin\n{res[1]}  output_stepu_{a.id}_1d.bin")


if __name__ == "__main__":
    main()
