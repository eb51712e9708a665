"""Load the committed golden fixture (tests/golden/evp1d_small.npz) as a
Problem1D plus the oracle's recorded results."""
import json
import os

import numpy as np

from evp1d import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load():
    z = np.load(os.path.join(GOLDEN, "evp1d_small.npz"))
    exp = json.load(open(os.path.join(GOLDEN, "expected.json")))
    na, navel, ndte = int(z["na"]), int(z["navel"]), int(z["ndte"])
    idx = {k[4:]: z[k] for k in z.files if k.startswith("idx_")}
    f = {k[2:]: z[k] for k in z.files if k.startswith("f_")}
    pr = synth.Problem1D(na=na, navel=navel, ndte=ndte, idx=idx, skipT=z["skipT"],
                         skipU=z["skipU"], f=f, stress=z["stress"], uvel=z["uvel"],
                         vvel=z["vvel"], strintx=z["strintx"], strinty=z["strinty"],
                         Cb=z["Cb"])
    out = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return pr, out, exp
