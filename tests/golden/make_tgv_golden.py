"""Writes tests/golden/tgv_1024.json: the FP64 C oracle's vortex amplitude of
the 2-level periodic Taylor-Green vortex (mblbm.tgv_geometry(n=1024,
patch=256, u0=0.01, tau=0.6, levels=2), initial state mblbm.tgv_init) after
the listed coarse steps.  The reference has no periodic boundary, so the
oracle's own ghost fill is the checker; about 2 minutes on 8 cores.

    python tests/golden/make_tgv_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(REPO, "multi-block-lbm-gpu_b200"), os.path.join(REPO, "oracle")]

import mblbm  # noqa: E402
import oracle  # noqa: E402

STEPS = (1000, 5000)


def main():
    g = mblbm.tgv_geometry(n=1024, patch=256, u0=0.01, tau=0.6, levels=2)
    o = oracle.Oracle(g)
    o.init()
    mblbm.tgv_init(o, g)
    out = {"n": 1024, "patch": 256, "u0": 0.01, "tau": 0.6, "levels": 2,
           "a0": mblbm.tgv_amplitude(o, g), "amplitude": {}}
    done = 0
    for t in STEPS:
        o.evolution(t - done)
        done = t
        out["amplitude"][str(t)] = mblbm.tgv_amplitude(o, g)
        print(t, out["amplitude"][str(t)], flush=True)
    with open(os.path.join(HERE, "tgv_1024.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
