"""Generates the golden fixtures of tests/golden/ with the FP64 oracle.

The reference ships no test vectors and cannot be built here (Fortran with an
un-vendored PoisFFT module), so these fixtures pin the oracle itself: a
regression in the oracle or in the CUDA path shows up as a mismatch.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from gpu_elmm_b200.config import grid_of, make_config  # noqa: E402
from gpu_elmm_b200.workloads import interiors, log_profile_state  # noqa: E402
from oracle import Oracle  # noqa: E402

CASES = {
    # name: (make_config kwargs, steps)
    "channel_16x12x8": (dict(Prnx=16, Prny=12, Prnz=8), 2),
    "stretched_16x12x10": (dict(Prnx=16, Prny=12, Prnz=10,
                                zW=np.concatenate([[0.0], np.cumsum(0.5 * 1.04 ** np.arange(10))])), 2),
}


def run_case(kw, steps):
    kw = dict(kw)
    n = (kw.pop("Prnx"), kw.pop("Prny"), kw.pop("Prnz"))
    cfg = make_config(*n, **kw)
    g = grid_of(cfg)
    zW = kw.get("zW")
    st = log_profile_state(g, seed=0, zW=zW)
    o = Oracle(cfg)
    o.set_state(*st)
    o.project(1.0)
    proj = [a.copy() for a in interiors(g, *o.state())]
    o.step(steps)
    out = [a.copy() for a in interiors(g, *o.state())]
    return cfg, st, proj, out


def main():
    for name, (kw, steps) in CASES.items():
        _, st, proj, out = run_case(kw, steps)
        np.savez_compressed(os.path.join(HERE, name + ".npz"),
                            U0=st[0], V0=st[1], W0=st[2],
                            Up=proj[0], Vp=proj[1], Wp=proj[2], Pp=proj[3],
                            U=out[0], V=out[1], W=out[2], P=out[3], steps=steps)
        print("wrote", name)


if __name__ == "__main__":
    main()
