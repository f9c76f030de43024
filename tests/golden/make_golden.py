"""Golden vectors from the reference's own engine.

Runs the reference's Engine (engine.cu/kernels.cu/config.cu compiled from its
sources into oracle/_ref/libref_engine.so by `make -C oracle ref`) on small
seeded scenes and saves its inputs and outputs as compressed .npz fixtures
beside this script.  The reference is CUDA-only, so this needs a GPU:

    python tests/golden/make_golden.py

Each fixture holds the config text, the 26-plane buffer handed to
Engine::init, the triangles handed to Engine::initSDF, and after `substeps`
calls of Engine::step(): the state (getBuffer), the grid planes (getGrid),
the SDF, the positions export (changeFormat), plus the Morton keys and sort
permutation of the first substep (setKeys + thrust::sort_by_key).
tests/test_golden.py checks the CPU oracle against them without a GPU.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "water-sim-cuda_b200"))
sys.path.insert(0, ROOT)

# name: (grid size, particles, seed, obstacle, substeps, physics overrides)
CASES = {
    "free16": ((16, 16, 16), 800, 31, False, 1, {}),
    "obstacle24": ((24, 16, 32), 1200, 32, True, 1, {}),
    "obstacle24_x3": ((24, 16, 32), 1200, 32, True, 3, {}),
    "tait16": ((16, 16, 16), 800, 33, False, 1,
               {"gamma": -2.0, "gravity": 9.81, "compression": 200.0, "dt": 0.01, "padding": 2}),
}


def make_case(ref, name, size, n, seed, obstacle, substeps, physics):
    from mpm_b200 import scenes
    cfg, st, tris = scenes.small_scene(n, size, seed=seed, obstacle=obstacle, **physics)
    with tempfile.TemporaryDirectory() as d:
        ref.create(cfg, st, tris, os.path.join(d, "config.txt"))
    start = ref.state()
    keys = ref.keys()
    ref.step(1)
    perm = ref.perm()
    if substeps > 1:
        ref.step(substeps - 1)
    out = dict(config=np.array(cfg.to_text()), state_in=st, triangles=np.asarray(tris, np.float32),
               start=start, keys=keys, perm=perm, state=ref.state(), grid=ref.grid(), sdf=ref.sdf(),
               positions=ref.positions(), substeps=np.int32(substeps))
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: n={n} grid={size} substeps={substeps} -> {os.path.getsize(path)} bytes")


def main():
    from oracle.oracle import RefEngine
    ref = RefEngine()
    try:
        for name, args in CASES.items():
            make_case(ref, name, *args)
    finally:
        ref.destroy()


if __name__ == "__main__":
    main()
