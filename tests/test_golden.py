"""The CPU oracle against golden vectors made by the reference's own engine.

tests/golden/*.npz were written by tests/golden/make_golden.py, which runs the
reference's Engine (engine.cu/kernels.cu compiled from its sources) on small
seeded scenes on a B200.  These tests need no GPU: they pin the oracle that
the GPU parity tests use as their checker.

Tolerances (the parity rules of tests/parity.py):
  * initial state after Engine::init (initFMatrices): bit-exact;
  * Morton keys and sort permutation: bit-exact;
  * SDF: 1e-4 cell widths at nodes whose winding number is not within 1e-3 of
    the 0.5 threshold;
  * state after one substep: 1e-5 relative (normwise; positions on the
    displacement), after three substeps 1e-4; grid mass and velocity 1e-5;
  * the positions export equals the state's positions bit for bit.
"""
import glob
import os

import numpy as np
import pytest

from parity import assert_normwise, assert_state_close

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def _load(path, mpm):
    g = dict(np.load(path))
    cfg = mpm.parse_config_string(str(g["config"]))
    return g, cfg


def test_fixtures_present():
    names = {os.path.basename(p)[:-4] for p in FIXTURES}
    assert {"free16", "obstacle24", "obstacle24_x3", "tait16"} <= names


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_reference_engine(path, mpm, oracle64):
    g, cfg = _load(path, mpm)
    st0 = oracle64.init_particles(cfg, g["state_in"])
    assert np.array_equal(st0.astype(np.float32), g["start"]), "initFMatrices rules differ"
    keys = oracle64.morton_keys(g["start"])
    assert np.array_equal(keys, g["keys"]), "Morton keys differ from setKeys"
    assert np.array_equal(oracle64.sort_perm(keys), g["perm"]), "permutation differs from thrust::sort_by_key"

    sdf = g["sdf"].astype(np.float64)
    if g["triangles"].size:
        want, wn = oracle64.make_sdf(cfg, g["triangles"].astype(np.float64))
        ok = np.abs(wn - 0.5) >= 1e-3
        assert ok.mean() > 0.999
        assert np.abs(sdf - want)[ok].max() <= 1e-4
    else:
        assert np.all(g["sdf"] == np.sqrt(np.float32(1e30)))

    s = g["start"].astype(np.float64)
    nsub = int(g["substeps"])
    for _ in range(nsub):
        s, grid, _, _ = oracle64.substep(cfg, s, sdf)
    rtol = 1e-5 if nsub == 1 else 1e-4
    assert_state_close(g["state"], s, g["start"], rtol=rtol)
    assert_normwise("grid mass", g["grid"][0], grid[0], rtol=rtol)
    assert_normwise("grid velocity", g["grid"][1:4], grid[1:4], rtol=rtol)
    assert np.array_equal(g["positions"], g["state"][0:3].T)


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[:-4])
def test_fp32_restatement_near_reference(path, mpm, oracle32):
    """The timed CPU baseline (FP32 restatement) tracks the reference's FP32
    results to a few ulp-level differences per substep."""
    g, cfg = _load(path, mpm)
    s = oracle32.init_particles(cfg, g["state_in"])
    for _ in range(int(g["substeps"])):
        s = oracle32.substep(cfg, s, g["sdf"])[0]
    assert_state_close(s, g["state"].astype(np.float64), g["start"], rtol=1e-4)
