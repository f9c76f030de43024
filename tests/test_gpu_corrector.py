"""The learned large-step corrector (no counterpart in the reference; it
sits beside the plain substep): the tensor-core MLP against a PyTorch fp32
reference, the training kernel's gradient against autograd, training, the
collection probe, and the large step against the FP64 oracle at RATIO x DT.

Tolerances: MLP outputs within 2e-2 of the output scale (bf16 operands; the
hardware tanh of the GELU differs from torch's by ~1e-3 relative, which can
move a bf16 rounding by one step); gradients within 2e-2 relative (normwise
per parameter block); the uncorrected large step within the substep's 1e-5
of the oracle run at DT x RATIO."""
import dataclasses

import numpy as np
import pytest
import torch

import mlp_ref
from parity import assert_state_close

pytestmark = pytest.mark.gpu


def _features(n, seed):
    rng = np.random.default_rng(seed)
    f = rng.normal(0, 1, (n, 16)).astype(np.float32)
    f[:, 0:9] *= 0.3          # C
    f[:, 9:12] *= 2.0         # velocity
    f[:, 12] = rng.normal(0.1, 0.4, n)   # density - 1
    f[:, 13:16] *= 0.5        # folded SDF
    return f


def test_forward_matches_torch(gpu_ok, mpm):
    feats = _features(4099, 1)  # not a multiple of 32: idle lanes of the last warp
    targs = np.random.default_rng(2).normal(0, 0.3, (4099, 3)).astype(np.float32)
    w = mlp_ref.random_params(3, feats, targs)
    with mpm.Corrector(16) as c:
        c.set_params(w)
        got = c.forward(feats)
    want = mlp_ref.forward(torch.tensor(w), torch.tensor(feats)).detach().numpy()
    scale = np.sqrt((want ** 2).mean(0))
    err = np.abs(got - want).max(0) / scale
    assert (err < 2e-2).all(), err
    # every output column is wired to its own row: permuting rows permutes outputs
    with mpm.Corrector(16) as c:
        c.set_params(w)
        got2 = c.forward(feats[::-1].copy())
    assert np.abs(got2[::-1] - got).max() <= 1e-6 * np.abs(got).max()


@pytest.mark.parametrize("kernel", ["tcgen05", "fp32"])
@pytest.mark.parametrize("n", [1024, 64, 192])
def test_gradient_matches_autograd(gpu_ok, mpm, kernel, n):
    """1024 samples: 8 full tiles of the tcgen05 kernel; 64 and 192: a
    half-filled last tile (its rows beyond the batch are masked)."""
    feats = _features(1024, 4)
    targs = (np.tanh(feats[:, 9:12]) * 0.5 + 0.1 * feats[:, 0:3]).astype(np.float32)
    w = mlp_ref.random_params(5, feats, targs)
    idx = np.random.default_rng(n).permutation(1024)[:n]
    with mpm.Corrector(1024) as c:
        c.add_data(feats, targs)
        c.set_params(w)
        c.set_train_kernel(kernel)
        g, loss = c.gradient(idx)
    want_loss, want_g = mlp_ref.loss_and_grad(w, feats[idx], targs[idx])
    assert abs(loss - want_loss) <= 1e-2 * want_loss
    for name in ("W1", "b1", "W2", "b2", "W3", "b3"):
        o, k = mlp_ref.OFF[name]
        a, b = g[o:o + k], want_g[o:o + k]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert rel < 2e-2, (name, rel)
    # normalisation entries are not trained
    assert not g[:35].any()


def test_train_kernels_agree(gpu_ok, mpm):
    """The same Adam steps with either gradient kernel end at nearby parameters."""
    n = 50_000
    feats = _features(n, 8)
    targs = (np.tanh(feats[:, 9:12]) + 0.3 * feats[:, 0:3]).astype(np.float32)
    out = {}
    for kernel in ("tcgen05", "fp32"):
        with mpm.Corrector(n) as c:
            c.add_data(feats, targs)
            c.init(seed=3)
            c.set_train_kernel(kernel)
            out[kernel] = (c.train(40, batch=8192, lr=1e-3, seed=4), c.get_params())
    (la, wa), (lb, wb) = out["tcgen05"], out["fp32"]
    assert abs(la - lb) <= 2e-2 * lb, (la, lb)
    for name in ("W1", "W2", "W3"):
        o, k = mlp_ref.OFF[name]
        rel = np.linalg.norm(wa[o:o + k] - wb[o:o + k]) / np.linalg.norm(wb[o:o + k])
        assert rel < 2e-2, (name, rel)


def test_training_fits_a_smooth_map(gpu_ok, mpm):
    n = 200_000
    feats = _features(n, 6)
    targs = (np.tanh(feats[:, 9:12]) + 0.5 * feats[:, 0:3] * feats[:, 12:13]).astype(np.float32)
    with mpm.Corrector(n) as c:
        c.add_data(feats, targs)
        c.init(seed=7)
        first = c.train(20, batch=4096, lr=2e-3, seed=1)
        last = c.train(600, batch=4096, lr=2e-3, seed=2)
        last = c.train(50, batch=4096, lr=5e-4, seed=3)
        w = c.get_params()
    assert last < 0.1 * first, (first, last)
    pred = mlp_ref.forward(torch.tensor(w), torch.tensor(feats[:5000])).detach().numpy()
    rel = np.sqrt(((pred - targs[:5000]) ** 2).mean() / (targs[:5000] ** 2).mean())
    assert rel < 0.2, rel


def _small(mpm, n=3000, obstacle=False, seed=11, **kw):
    from mpm_b200 import scenes
    return scenes.small_scene(n, (32, 32, 32), seed=seed, obstacle=obstacle, **kw)


@pytest.mark.parametrize("ratio", [1, 4])
def test_uncorrected_large_step_is_substep_at_ratio_dt(gpu_ok, mpm, oracle64, ratio):
    """Velocity, C and F: the substep at RATIO x DT.  Positions: advected
    with v_old + (R + 1) / (2R) (v_new - v_old) (R = 1: the plain substep)."""
    cfg, st, tris = _small(mpm, obstacle=False)
    with mpm.Engine(cfg) as e:
        e.init(st)
        start = e.get_buffer()
        sdf = e.get_sdf()
        e.set_corrector(None, ratio=ratio)
        stats = e.step_learned(1)
        got = e.get_buffer()
        assert stats["large_steps"] == 1 and stats["fallbacks"] == 0
    dt = float(np.float32(cfg.dt) * ratio)
    big = dataclasses.replace(cfg, dt=dt)
    want, _, _, _ = oracle64.substep(big, start.astype(np.float64), sdf.astype(np.float64))
    blend = (ratio + 1) / (2 * ratio)
    v0 = start[3:6].astype(np.float64)
    want[0:3] = start[0:3] + dt * (v0 + blend * (want[3:6] - v0))
    assert_state_close(got, want, start)


def test_zero_correction_and_bias_wiring(gpu_ok, mpm):
    cfg, st, tris = _small(mpm)
    w = mlp_ref.random_params(8)
    p = mlp_ref.split(w)
    p["W3"][:] = 0
    p["b3"][:] = 0
    outs = {}
    for tag, b3 in (("none", None), ("zero", (0.0, 0.0, 0.0)), ("bias", (0.05, -0.1, 0.15))):
        with mpm.Engine(cfg) as e:
            e.init(st)
            if b3 is None:
                e.set_corrector(None, ratio=4)
            else:
                p["b3"][:] = b3
                e.set_corrector(w, ratio=4, max_density_change=-1.0)
            e.step_learned(1)
            outs[tag] = e.get_buffer()
    a, z, b = outs["none"], outs["zero"], outs["bias"]
    assert np.abs(z[0:6] - a[0:6]).max() < 1e-4
    dv = np.array([0.05, -0.1, 0.15], np.float32)[:, None]
    dt = np.float32(cfg.dt) * 4
    blend = 5.0 / 8.0
    assert np.abs((b[3:6] - a[3:6]) - dv).max() < 1e-4
    assert np.abs((b[0:3] - a[0:3]) - dt * blend * dv).max() < 1e-4 * max(1.0, float(dt))


def test_fallback_runs_plain_substeps(gpu_ok, mpm):
    cfg, st, tris = _small(mpm, obstacle=True, seed=12)
    w = mlp_ref.random_params(9)
    with mpm.Engine(cfg) as e:
        e.init(st)
        e.init_sdf(tris)
        e.step(4)
        plain = e.get_buffer()
    with mpm.Engine(cfg) as e:
        e.init(st)
        e.init_sdf(tris)
        e.set_corrector(w, ratio=4, max_density_change=0.0)
        stats = e.step_learned(1)
        got = e.get_buffer()
        assert stats["fallbacks"] == 1 and stats["large_steps"] == 0
        assert stats["last_density_change"] > 0
        assert e.stats()["substeps"] == 4
    assert_state_close(got, plain.astype(np.float64), st, rtol=1e-4)


def test_collect_records_the_probe(gpu_ok, mpm):
    cfg, st, tris = _small(mpm, n=2000, seed=13)
    ratio, samples = 4, 600
    with mpm.Engine(cfg) as e:
        e.init(st)
        e.step(3)
        s0 = e.get_buffer()
        e.step(ratio)
        plain = e.get_buffer()
    with mpm.Engine(cfg) as e:
        e.init(st)
        e.set_state(s0)
        e.set_corrector(None, ratio=ratio)
        e.step_learned(1)
        large = e.get_buffer()
    with mpm.Engine(cfg) as e, mpm.Corrector(10_000) as c:
        e.init(st)
        e.set_state(s0)
        e.set_corrector(None, ratio=ratio)
        c.collect(e, samples, seed=5)
        after = e.get_buffer()
        assert c.size == samples
        feats, targs = c.get_data()
    # the engine continues the plain trajectory
    assert_state_close(after, plain.astype(np.float64), s0, rtol=1e-4)
    # each row is some particle r: features (C, v) of the large step, target v_plain - v_large
    key = np.concatenate([large[6:15].T, large[3:6].T], axis=1)          # C row-major, v
    tgt = (plain[3:6] - large[3:6]).T
    fk = feats[:, 0:12]
    d = np.abs(fk[:, None, :] - key[None, :, :]).max(-1)
    r = d.argmin(1)
    scale = max(1.0, float(np.abs(key).max()))
    assert (d[np.arange(samples), r] < 1e-4 * scale).all()
    assert np.abs(targs - tgt[r]).max() < 1e-3 * max(1.0, float(np.abs(tgt).max()))
    assert len(np.unique(r)) > samples // 2  # drawn across the scene
    # density feature: interpolated mass over the seeding density, minus 1, is > -1
    assert (feats[:, 12] > -1).all()
    assert not feats[:, 13:16].any()  # no obstacle: the folded SDF is zero


def test_forward_tcgen05_matches(gpu_ok, mpm):
    """The tcgen05 / TMEM MLP against the torch reference and the mma.sync path
    (both round the same operands to bf16; only fp32 summation order differs)."""
    n = 4099  # 17 CTAs of 256 rows, the last one ragged
    feats = _features(n, 11)
    targs = np.random.default_rng(12).normal(0, 0.3, (n, 3)).astype(np.float32)
    w = mlp_ref.random_params(13, feats, targs)
    with mpm.Corrector(16) as c:
        c.set_params(w)
        tc = c.forward(feats, tcgen05=True)
        ms = c.forward(feats)
    want = mlp_ref.forward(torch.tensor(w), torch.tensor(feats)).detach().numpy()
    scale = np.sqrt((want ** 2).mean(0))
    assert (np.abs(tc - want).max(0) / scale < 2e-2).all()
    assert (np.abs(tc - ms).max(0) / scale < 1e-2).all()


def test_learned_step_tcgen05_matches_mma_sync(gpu_ok, mpm):
    """The learned large step with the MLP on tcgen05 (default) and on
    mma.sync: the same corrections up to fp32 summation order."""
    cfg, st, tris = _small(mpm, n=5000, obstacle=True, seed=14)
    feats = _features(2000, 15)
    w = mlp_ref.random_params(16, feats)
    mlp_ref.split(w)["out_std"][:] = 0.05
    out = {}
    for tc in (True, False):
        with mpm.Engine(cfg) as e:
            e.init(st)
            e.init_sdf(tris)
            e.set_corrector(w, ratio=4, max_density_change=-1.0)
            e.set_corrector_kernel(tcgen05=tc)
            e.step_learned(2)
            out[tc] = e.get_buffer()
    a, b = out[True], out[False]
    assert np.abs(a[3:6] - b[3:6]).max() < 2e-3 * max(1.0, float(np.abs(b[3:6]).max()))
    assert np.abs(a[0:3] - b[0:3]).max() < 2e-3


@pytest.mark.parametrize("threshold", [0.0, 1e9])
def test_device_decided_fallback_matches_host(gpu_ok, mpm, threshold):
    """The checked large step decided on the device (one graph per step: the
    large step, the decision kernel and a conditional node whose body is the
    fallback) against the same steps decided on the host, over three large
    steps: every step rejected (threshold 0) or every one accepted (1e9).
    Counters, statistics and states agree (to the rounding of the float
    atomics, whose order differs between runs)."""
    cfg, st, tris = _small(mpm, obstacle=True, seed=21, randomize=False)
    w = mlp_ref.random_params(10)
    out = {}
    for on_device in (False, True):
        with mpm.Engine(cfg) as e:
            e.init(st)
            e.init_sdf(tris)
            e.set_corrector(w, ratio=4, max_density_change=threshold)
            e.set_fallback_on_device(on_device)
            stats = e.step_learned(2)
            stats = e.step_learned(1)
            out[on_device] = (stats, e.learned_statistics(), e.get_buffer(), e.stats()["substeps"], e.get_positions())
    (sh, lh, bh, nh, ph), (sd, ld, bd, nd, pd) = out[False], out[True]
    assert sh["large_steps"] == sd["large_steps"] and sh["fallbacks"] == sd["fallbacks"]
    assert (sd["fallbacks"], sd["large_steps"]) == ((3, 0) if threshold == 0.0 else (0, 3))
    assert nh == nd == (12 if threshold == 0.0 else 0)
    for k in lh:
        assert ld[k] == pytest.approx(lh[k], rel=1e-3, abs=1e-6)
    assert np.isfinite(bd).all()
    assert np.abs(bd.astype(np.float64) - bh).max() <= 1e-4 * max(1.0, np.abs(bh).max())
    assert np.array_equal(pd, bd[0:3].T)
