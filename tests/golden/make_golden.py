"""Regenerate the golden fixtures of the EVP-1D parity tests.

    python tests/golden/make_golden.py

Writes, next to this script:
  evp1d_small.npz    a 36 x 28 curvilinear synthetic problem in the 1D layout
                     (inputs) and the oracle's results after NDTE subcycles;
  expected.json      md5 of the two reference output files
                     (output_stress_*_1d.bin, output_stepu_*_1d.bin, layout of
                     src/vars.F90:2233-2304) from the oracle's v2 (1D) form and
                     from its v0 (2D) form -- equal, which is the reference's
                     own acceptance criterion (README.md:63-104) -- plus the
                     closed-form answer of the integration smoke-test state.

The reference's published md5 pair pins DMI input files that are not
distributed, so these fixtures pin the oracle (and through it the CUDA path)
on seeded synthetic input instead.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "cice-evp1d_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from evp1d import synth  # noqa: E402
import oracle  # noqa: E402
import helpers  # noqa: E402

NX, NY, SEED, NDTE = 36, 28, 101, 10


def problem():
    g = synth.make_grid(NX, NY, seed=SEED, ndte=NDTE, curvilinear=True)
    return g, synth.to_1d(g)


def main():
    oracle.build()
    g, pr = problem()
    st = oracle.run_1d(pr, NDTE)
    f1, f2 = helpers.output_files(st.stress, st.strintx, st.strinty, st.uvel, st.vvel, pr.skipU)
    F = oracle.run_v0(g, NDTE)
    g1, g2 = oracle.v0_output_files(g, F, pr)
    assert (f1, f2) == (g1, g2), "v0 and v2 forms disagree"
    arrays = {f"idx_{k}": v for k, v in pr.idx.items()}
    arrays.update({f"f_{k}": v for k, v in pr.f.items()})
    arrays.update(skipT=pr.skipT, skipU=pr.skipU, stress=pr.stress, uvel=pr.uvel,
                  vvel=pr.vvel, strintx=pr.strintx, strinty=pr.strinty, Cb=pr.Cb,
                  out_stress=st.stress, out_uvel=st.uvel[: pr.navel], out_vvel=st.vvel[: pr.navel],
                  out_strintx=st.strintx, out_strinty=st.strinty, out_Cb=st.Cb,
                  out_str=st.str[:, : pr.navel], na=np.int64(pr.na), navel=np.int64(pr.navel),
                  ndte=np.int64(NDTE))
    np.savez_compressed(os.path.join(HERE, "evp1d_small.npz"), **arrays)

    sa = helpers.standalone_problem(ndte=3, strength=0.0)
    sst = oracle.run_1d(sa, 3)
    exp = {
        "problem": {"nx": NX, "ny": NY, "seed": SEED, "ndte": NDTE, "curvilinear": True,
                    "na": pr.na, "navel": pr.navel},
        "md5_stress_v2": hashlib.md5(f1).hexdigest(),
        "md5_stepu_v2": hashlib.md5(f2).hexdigest(),
        "md5_stress_v0": hashlib.md5(g1).hexdigest(),
        "md5_stepu_v0": hashlib.md5(g2).hexdigest(),
        "standalone_ndte3_strength0": {
            "na": sa.na, "navel": sa.navel,
            "stressp_1": float(sst.stress[0, 0]), "stressm_4": float(sst.stress[7, 0]),
            "md5_stress": hashlib.md5(np.ascontiguousarray(sst.stress).tobytes()).hexdigest(),
        },
    }
    with open(os.path.join(HERE, "expected.json"), "w") as f:
        json.dump(exp, f, indent=1)
    print(json.dumps(exp, indent=1))


if __name__ == "__main__":
    main()
