"""Training and evaluation of the learned large-step corrector.

The corrector (include/mpm_b200.h, "Learned large step") lets one substep of
RATIO x DT stand in for RATIO plain substeps.  This module:

  * builds seeded variants of the 128^3 dam-break scene (water-box extents
    +-20 %, torus position +-15 cells);
  * runs plain trajectories on them and, every few substeps, the collection
    probe (one uncorrected large step vs RATIO plain substeps from the same
    state), filling the corrector's dataset on the device;
  * trains the MLP with the library's fused training kernel (Adam);
  * evaluates a learned run against the plain run from the same state:
    simulated time per second of each, the fallback count, the grid-density
    error and the particle-position divergence.

Density error: sum over nodes of |m_learned - m_plain| / sum of m_plain, with
m the B-spline node mass of the particle positions (the P2G mass field).
Divergence: mean distance in cells between a particle's two positions.

Run `python -m mpm_b200.learned train --out FILE` to train and save the
parameters, `python -m mpm_b200.learned evaluate --params FILE` to measure.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import time

import numpy as np

from . import Corrector, Engine, scenes

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_PARAMS = os.path.join(HERE, "corrector_dam_break.npz")
PHYSICAL_PARAMS = os.path.join(HERE, "corrector_dam_break_physical.npz")


def dam_break_variant(seed: int, physical: bool = False):
    """The 2M dam break with seeded box extents (+-20 %) and torus position
    (+-15 cells).  physical=True flips GRAVITY and GAMMA to the orientation in
    which gravity pulls -y and the Tait law resists compression."""
    rng = np.random.default_rng(seed)
    cfg = scenes._cfg((128, 128, 128))
    f = rng.uniform(0.8, 1.2, size=3)
    hi = np.minimum(4.0 + np.array([56.0, 37.0, 120.0]) * f, 124.0)
    pos = scenes.seed_box((4.0, 4.0, 4.0), hi, cfg.resolution, rng)
    c = np.array([80.0, 30.0, 64.0]) + rng.uniform(-15, 15, size=3)
    c[0] = min(c[0], 128 - 3 - 34.0)
    tris = scenes.torus(25.0, 8.0, tuple(c), 48, 24)
    if physical:
        cfg = physical_config(cfg)
    return cfg, scenes.pack_state(pos), tris


def physical_config(cfg):
    return dataclasses.replace(cfg, gravity=-cfg.gravity, gamma=-cfg.gamma)


def collect(corr: Corrector, seeds, substeps: int, probe_every: int, samples: int, ratio: int = 4,
            physical: bool = False, log=print, policy=None):
    """Trajectories of `substeps` substeps on dam_break_variant(seed), with the
    collection probe every `probe_every` substeps.  Between probes the
    trajectory advances with plain substeps, or, given `policy` parameters,
    with learned large steps (no fallback): the probes then sample the states
    a learned rollout visits (dataset aggregation)."""
    for k, seed in enumerate(seeds):
        cfg, st, tris = dam_break_variant(seed, physical)
        with Engine(cfg) as e:
            e.init(st)
            e.init_sdf(tris)
            done = 0
            probe = 0
            while done + ratio <= substeps:
                if done % probe_every == 0:
                    e.set_corrector(None, ratio=ratio)
                    corr.collect(e, samples, seed=seed * 100003 + probe)
                    probe += 1
                    done += ratio
                else:
                    step = min(probe_every - done % probe_every, substeps - done)
                    if policy is not None and step % ratio == 0:
                        e.set_corrector(policy, ratio=ratio, max_density_change=-1.0)
                        e.step_learned(step // ratio)
                    else:
                        e.step(step)
                    done += step
        log(f"variant {k + 1}/{len(seeds)} seed {seed}: {corr.size} samples")


def train(corr: Corrector, steps: int, batch: int = 65536, lr: float = 1e-3, seed: int = 0, log=print,
          chunk: int = 1000):
    """Adam with a cosine learning-rate decay, in chunks of `chunk` steps."""
    corr.init(seed)
    losses = []
    done = 0
    t0 = time.perf_counter()
    while done < steps:
        k = min(chunk, steps - done)
        frac = (done + 0.5 * k) / steps
        cur = lr * (0.05 + 0.95 * 0.5 * (1 + np.cos(np.pi * frac)))
        losses.append(corr.train(k, batch=batch, lr=float(cur), seed=seed * 7919 + done))
        done += k
        log(f"step {done}/{steps}: loss {losses[-1]:.5f} lr {cur:.2e} ({time.perf_counter() - t0:.1f} s)")
    return losses, time.perf_counter() - t0


def density_field(pos: np.ndarray, cfg, device="cuda"):
    """B-spline node mass of unit-mass particles (the P2G mass field), as a
    torch tensor on `device`."""
    import torch
    x = torch.as_tensor(pos, dtype=torch.float32, device=device)
    base = torch.floor(x - 0.5)
    fx = x - base
    w = torch.stack([0.5 * (1.5 - fx) ** 2, 0.75 - (fx - 1.0) ** 2, 0.5 * (fx - 0.5) ** 2], 0)  # (3, n, 3)
    size = torch.tensor([cfg.size_x, cfg.size_y, cfg.size_z], device=device)
    g = torch.zeros(cfg.size_x * cfg.size_y * cfg.size_z, dtype=torch.float64, device=device)
    bi = base.long()
    for a in range(3):
        for b in range(3):
            for c in range(3):
                node = bi + torch.tensor([a, b, c], device=device)
                ok = ((node >= 0) & (node < size)).all(1)
                idx = (node[:, 2] * cfg.size_y + node[:, 1]) * cfg.size_x + node[:, 0]
                wt = w[a, :, 0] * w[b, :, 1] * w[c, :, 2]
                g.index_add_(0, idx[ok], wt[ok].double())
    return g


def compare(cfg, pos_learned: np.ndarray, pos_plain: np.ndarray) -> dict:
    import torch
    ml, mp = density_field(pos_learned, cfg), density_field(pos_plain, cfg)
    rho0 = 1.0 / float(cfg.resolution) ** 3
    occ = mp > 0.5 * rho0
    d = np.linalg.norm(pos_learned.astype(np.float64) - pos_plain, axis=1)
    return {
        "density_err": float((ml - mp).abs().sum() / mp.sum()),
        "density_err_occupied": float(((ml - mp).abs()[occ] / rho0).mean()) if bool(occ.any()) else 0.0,
        "divergence_cells": float(d.mean()),
        "divergence_p95_cells": float(np.percentile(d, 95)),
    }


def _timed(fn):
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = fn()
    torch.cuda.synchronize()
    return out, time.perf_counter() - t0


def evaluate(cfg, st, tris, params, nlarge: int = 100, ratio: int = 4, max_density_change: float = 0.02,
             checkpoints=(10, 25, 50, 100), perturb: float = 1e-4, rule: str = "density_change",
             on_device: bool = True, per_step_stats: bool = False) -> dict:
    """Plain (ratio * nlarge substeps) vs learned (nlarge large steps) vs the
    uncorrected large step, from the same state; metrics at each checkpoint
    (in large steps) and at the end.  "perturbed" is the plain run from
    positions moved by N(0, perturb) cells: its distance from the plain run
    is the chaos floor of the scene, what no large step can undercut.
    rule: the fallback statistic (Engine.set_fallback_rule); on_device: the
    fallback decided on the device (Engine.set_fallback_on_device); the learned
    run also reports the mean of each statistic, over every checked large step
    with per_step_stats (one call per step), else over the last step before
    each checkpoint."""
    marks = sorted(set([c for c in checkpoints if c <= nlarge] + [nlarge]))
    res = {"ratio": ratio, "large_steps": nlarge, "max_density_change": max_density_change, "rule": rule}
    runs = {}
    st_p = st.copy()
    st_p[0:3] += np.random.default_rng(99).normal(0, perturb, st_p[0:3].shape).astype(np.float32)
    for tag in ("plain", "perturbed", "learned", "uncorrected"):
        with Engine(cfg) as e:
            e.init(st_p if tag == "perturbed" else st)
            e.init_sdf(tris)
            if tag == "learned":
                e.set_corrector(params, ratio=ratio, max_density_change=max_density_change)
                e.set_fallback_rule(rule)
                e.set_fallback_on_device(on_device)
            elif tag == "uncorrected":
                e.set_corrector(None, ratio=ratio)
            pos, total, prev, stats = {}, 0.0, 0, {}
            seen = {"density_change": [], "rest_density": [], "rest_density_before": []}
            for m in marks:
                k = m - prev
                if tag in ("plain", "perturbed"):
                    _, dt = _timed(lambda: e.step(k * ratio))
                elif tag == "learned" and max_density_change >= 0 and per_step_stats:
                    # One call per large step, to record each step's statistics.
                    dt = 0.0
                    for _ in range(k):
                        stats, d = _timed(lambda: e.step_learned(1))
                        dt += d
                        for key, v in e.learned_statistics().items():
                            seen[key].append(v)
                else:
                    stats, dt = _timed(lambda: e.step_learned(k))
                    if tag == "learned" and max_density_change >= 0:
                        for key, v in e.learned_statistics().items():
                            seen[key].append(v)
                total += dt
                prev = m
                pos[m] = e.get_positions().copy()
            sim_time = nlarge * ratio * float(cfg.dt)
            runs[tag] = pos
            res[tag] = {"seconds": total, "sim_time_per_s": sim_time / total,
                        "particle_substeps_per_s": e.get_number() * nlarge * ratio / total}
            if tag == "learned":
                res[tag].update(stats)
                if seen["density_change"]:
                    res[tag]["mean_statistics"] = {key: float(np.mean(v)) for key, v in seen.items()}
    for tag in ("perturbed", "learned", "uncorrected"):
        for m in marks:
            res[tag][f"at_{m}"] = compare(cfg, runs[tag][m], runs["plain"][m])
    res["speedup_sim_time"] = res["learned"]["sim_time_per_s"] / res["plain"]["sim_time_per_s"]
    return res


def save_params(path: str, params: np.ndarray, meta: dict):
    """path (.npz: parameters and training record) and the raw little-endian
    float32 parameters beside it (.bin, what `mpm_run --corrector` reads)."""
    np.savez_compressed(path, params=params.astype(np.float32), meta=json.dumps(meta))
    params.astype("<f4").tofile(os.path.splitext(path)[0] + ".bin")


def load_params(path: str = DEFAULT_PARAMS):
    z = np.load(path)
    return z["params"], json.loads(str(z["meta"]))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--variants", type=int, default=200)
    t.add_argument("--first-seed", type=int, default=5000)
    t.add_argument("--substeps", type=int, default=1000)
    t.add_argument("--probe-every", type=int, default=40)
    t.add_argument("--samples", type=int, default=20000)
    t.add_argument("--steps", type=int, default=50000)
    t.add_argument("--batch", type=int, default=65536)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--ratio", type=int, default=4)
    t.add_argument("--physical", action="store_true")
    t.add_argument("--out", default=DEFAULT_PARAMS)
    t.add_argument("--dagger", default=None, help="parameters whose learned rollouts add probes")
    t.add_argument("--dagger-variants", type=int, default=100)
    ev = sub.add_parser("evaluate")
    ev.add_argument("--params", default=DEFAULT_PARAMS)
    ev.add_argument("--large-steps", type=int, default=250)
    ev.add_argument("--threshold", type=float, default=0.02)
    ev.add_argument("--physical", action="store_true")
    ev.add_argument("--seed", type=int, default=1235)
    ev.add_argument("--alpha", type=float, default=1.0, help="scale of the applied correction")
    ev.add_argument("--rule", choices=["density_change", "rest_density", "rest_density_excess"],
                    default="density_change", help="the fallback statistic")
    ev.add_argument("--host-decision", action="store_true", help="decide the fallback on the host")
    ev.add_argument("--per-step-stats", action="store_true", help="record every large step's statistics")
    pr = sub.add_parser("probe", help="a few learned large steps on a thinned dam break (a small case to profile)")
    pr.add_argument("--params", default=PHYSICAL_PARAMS)
    pr.add_argument("--thin", type=int, default=5, help="keep every THIN-th particle")
    pr.add_argument("--large-steps", type=int, default=4)
    pr.add_argument("--kernel", choices=["tcgen05", "mma_sync"], default="tcgen05")
    tt = sub.add_parser("train-timing", help="wall-clock time per Adam step of each training kernel")
    tt.add_argument("--samples", type=int, default=1_000_000)
    tt.add_argument("--batch", type=int, default=65536)
    tt.add_argument("--warmup", type=int, default=20)
    tt.add_argument("--steps", type=int, default=200)
    a = ap.parse_args(argv)
    if a.cmd == "probe":
        params, meta = load_params(a.params)
        cfg, st, tris = scenes.dam_break(seed=1235)
        if meta.get("physical"):
            cfg = physical_config(cfg)
        st = np.ascontiguousarray(st[:, ::a.thin])
        with Engine(cfg) as e:
            e.init(st)
            e.init_sdf(tris)
            e.set_corrector(params, ratio=int(meta.get("ratio", 4)), max_density_change=-1.0)
            e.set_corrector_kernel(a.kernel == "tcgen05")
            _, dt = _timed(lambda: e.step_learned(a.large_steps))
        print(json.dumps({"particles": int(st.shape[1]), "large_steps": a.large_steps, "kernel": a.kernel,
                          "seconds": dt}))
        return
    if a.cmd == "train-timing":
        rng = np.random.default_rng(17)
        feats = rng.normal(0, 1, (a.samples, 16)).astype(np.float32)
        targs = (np.tanh(feats[:, 9:12]) + 0.1 * rng.normal(0, 1, (a.samples, 3))).astype(np.float32)
        out = {}
        with Corrector(a.samples) as c:
            c.add_data(feats, targs)
            for kind in ("tcgen05", "fp32", "tcgen05"):
                c.init(seed=1)
                c.set_train_kernel(kind)
                c.train(a.warmup, batch=a.batch, lr=1e-3, seed=3)
                loss, dt = _timed(lambda: c.train(a.steps, batch=a.batch, lr=1e-3, seed=5))
                out[kind] = {"ms_per_step": 1e3 * dt / a.steps, "loss": float(loss)}
        print(json.dumps({"samples": a.samples, "batch": a.batch, "steps": a.steps} | out))
        return
    if a.cmd == "train":
        seeds = list(range(a.first_seed, a.first_seed + a.variants))
        probes = a.substeps // a.probe_every
        extra = a.dagger_variants if a.dagger else 0
        cap = (a.variants + extra) * (probes + 1) * a.samples
        t0 = time.perf_counter()
        with Corrector(cap) as c:
            collect(c, seeds, a.substeps, a.probe_every, a.samples, a.ratio, a.physical)
            if a.dagger:
                policy, _ = load_params(a.dagger)
                dseeds = list(range(a.first_seed + 100000, a.first_seed + 100000 + extra))
                collect(c, dseeds, a.substeps, a.probe_every, a.samples, a.ratio, a.physical, policy=policy)
            t_collect = time.perf_counter() - t0
            losses, t_train = train(c, a.steps, a.batch, a.lr)
            params = c.get_params()
            meta = {"variants": a.variants, "first_seed": a.first_seed, "substeps": a.substeps,
                    "probe_every": a.probe_every, "samples_per_probe": a.samples, "dataset": c.size,
                    "steps": a.steps, "batch": a.batch, "lr": a.lr, "ratio": a.ratio, "physical": a.physical,
                    "dagger": os.path.basename(a.dagger) if a.dagger else None, "dagger_variants": extra,
                    "losses": losses, "collect_s": t_collect, "train_s": t_train}
        save_params(a.out, params, meta)
        print(json.dumps({k: v for k, v in meta.items() if k != "losses"} | {"final_loss": losses[-1]}))
    else:
        params, meta = load_params(a.params)
        params = params.copy()
        params[32:35] *= a.alpha  # output scale (MPM_CORRECTOR_PARAMS layout)
        cfg, st, tris = scenes.dam_break(seed=a.seed)
        if a.physical:
            cfg = physical_config(cfg)
        res = evaluate(cfg, st, tris, params, nlarge=a.large_steps, ratio=int(meta.get("ratio", 4)),
                       max_density_change=a.threshold, rule=a.rule, on_device=not a.host_decision,
                       per_step_stats=a.per_step_stats)
        res["alpha"] = a.alpha
        print(json.dumps(res))


if __name__ == "__main__":
    main()
