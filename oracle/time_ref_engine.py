"""Times the reference's own CUDA engine on a synthetic disk (GPU).

TEST INFRASTRUCTURE: runs oracle/_ref/libref_engine.so -- src/physics/BHTree.cu,
Integrator.cu and Perturber.cu of the reference compiled unchanged for
sm_100a -- through the launcher sequence of src/main.cu:101-139 (no file
I/O), and prints one JSON line with its particle-steps/s.  This is the
"reference engine on the same B200" figure that the plain path is compared
with.  Before the GPU sees the input, the CPU restatement (oracle/port.c)
checks that the reference build keeps every body (no 128-level or node
overflow loss) and that its 20 summarize passes reach the root.

    python oracle/time_ref_engine.py [--n 1048576] [--steps 3] [--theta 0.5]
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--theta", type=float, default=0.5)
    ap.add_argument("--r-min", type=float, default=0.3)
    ap.add_argument("--r-max", type=float, default=30.0)
    ap.add_argument("--mass", type=float, default=1e-9)
    ap.add_argument("--eps", type=float, default=5e-4)
    ap.add_argument("--dt", type=float, default=0.002)
    a = ap.parse_args()
    import oracle
    nb = importlib.import_module("nbody-sim_b200")
    d = nb.make_disk(a.n, a.r_min, a.r_max, 0.01, 0.005, 1.0, 0)
    st = {k: v.astype(np.float32) for k, v in d.items()}
    st["m"] = np.full(a.n, a.mass, np.float32)
    port = oracle.Port()
    t = port.build_tree(st["x"], st["y"], st["z"], st["m"])
    info = port.tree_info(t)
    port.free_tree(t)
    if info.lost_bodies or info.unsummarized or info.height > 20:
        print(json.dumps({"unsafe_input": True, "lost": info.lost_bodies,
                          "unsummarized": info.unsummarized, "height": info.height}))
        return 1
    eng = oracle.RefEngine(a.n)
    eng.set_state(st)
    eng.build()
    eng.force(a.theta, a.eps, 1.0)
    eng.steps(0, 1, a.dt, a.theta, a.eps, 1.0, 0.0, 0.0, 0.0)  # warm-up step
    ms = eng.steps(1, a.steps, a.dt, a.theta, a.eps, 1.0, 0.0, 0.0, 0.0)
    eng.close()
    out = {"engine": "reference src/physics/*.cu @ sm_100a", "n": a.n, "steps": a.steps,
           "theta": a.theta, "ms_per_step": ms / a.steps,
           "particle_steps_per_s": a.n * a.steps / (ms * 1e-3), "tree_height": info.height}
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
