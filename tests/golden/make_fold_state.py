"""Generates tests/golden/sheet256_fold_state.npz: the state of the 256x256
self-contact fold (config 1 scene, seed 1) after PHASE_START steps of the CUDA
step, stored as float32 positions/velocities (the bench and the reference arm
both start from these exact bytes, widened to float64).

Run on a GPU machine:  python tests/golden/make_fold_state.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

PHASE_START = 200


def main(out=os.path.join(os.path.dirname(os.path.abspath(__file__)), "sheet256_fold_state.npz")):
    from clothcraft_b200 import scenes
    from clothcraft_b200.vbd import VbdSolver

    sc = scenes.config1()
    st = sc.settings.to_c()
    s = VbdSolver(sc)
    s.set_state(sc.x0, sc.v0, 0.0)
    for _ in range(PHASE_START):
        s.step_resident(st)
    x, v, t = s.get_state()
    np.savez_compressed(out, x=x.astype(np.float32), v=v.astype(np.float32), time=np.float64(t),
                        steps=np.int64(PHASE_START), scene=np.array("config1 seed 1"))
    # the widened state must be a valid start for a fresh solver
    xs = x.astype(np.float32).astype(np.float64)
    vs = v.astype(np.float32).astype(np.float64)
    VbdSolver(scenes.config1()).step(xs, vs, float(t), st)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
