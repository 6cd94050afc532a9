"""Generates tests/golden/cube6_ot_5steps.npz from the reference built from
its own sources (oracle/_ref): the static inputs, grid cell centres, the
step-0 state and derived fields, and the state after 5 steps of a periodic
6^3 curvilinear cube (the periodic Orszag-Tang cube at a small size).

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mercury_oracle as mo  # noqa: E402

N, STEPS = 6, 5


def main():
    d = mo.cube_run(n=N, steps=STEPS, dump_at=[0, STEPS])
    out = {"meta|n": np.full((1, 1, 1, 1), N), "meta|steps": np.full((1, 1, 1, 1), STEPS)}
    for (name, block), r in d.items():
        if block != 0:
            continue
        if name.startswith("step"):
            tag, fld = name.split(":", 1)
            if tag != "step0" and fld not in mo.STATE_FIELDS:
                continue
            if fld in mo.WORK_FIELDS and tag == "step0":
                pass
            key = tag + ":|" + fld
        elif name.startswith("static:"):
            key = "static:|" + name[len("static:"):]
        elif name.startswith("dual_"):
            key = "|" + name
        else:
            continue
        out[key] = r.data
        out[key + "__lohi"] = np.array(list(r.lo) + list(r.hi))
    np.savez_compressed(os.path.join(HERE, f"cube{N}_ot_{STEPS}steps.npz"), **out)


if __name__ == "__main__":
    main()
