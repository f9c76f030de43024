#!/usr/bin/env python3
"""Throughput of the MLS-MPM substep engine: particle-substeps per second.

Workload (default `dam_break_2M`): water box x in [4,60), y in [4,41),
z in [4,124) of a 128^3 grid at RESOLUTION 0.5 (1,989,120 particles, seeded
sub-cell jitter), a torus obstacle (R 25, r 8, 48x24 segments, 2,304
triangles) at (80,30,64), PADDING 3, GRAVITY -0.3, DT 0.1, GAMMA 7,
COMPRESSION 10, SUBSTEPS 4.  One bench step is one frame of the reference's
Simulation::run loop: SUBSTEPS calls of Engine::step() (keys, stable sort,
clear, P2G, grid update, G2P) plus the position export.  Inputs are synthetic.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

K defaults to 1000 frames, the dam break's whole run: the fluid spreads and
compresses over it and P2G slows, so the first frames alone overstate the
steady throughput.

Engine arm (default): `value` is device time (CUDA events on the engine's
stream) of K frames with the state resident in HBM; `e2e` is the whole job
through the C ABI with host buffers: upload of the scene from pinned memory
(mpm_init_particles), then K x (mpm_step + positions read back to pinned
memory), host wall time.  A second, instrumented pass of the same K frames,
restarted from the state the timed frames started from, records CUDA events
between the stages of every substep for the per-kernel roofline.  Rank 0 at
N=1 also times the FP32 OpenMP CPU restatement on a bounded sample.
Under torchrun each rank simulates an independent replica of the scene on its
own GPU (no collective on the data path; weak scaling), timing is the max over
ranks.

Reference arm: the reference's own Engine (engine.cu/kernels.cu compiled from
its sources into oracle/_ref) on the same scene, K frames, device time.  The
reference implementation of this path is CUDA, so this arm runs on the GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "water-sim-cuda_b200"))
sys.path.insert(0, ROOT)

# The headline metric as quoted for this workload: plain particle-substeps/s at 2M particles on
# a 128^3 grid, with the learned 4xDT path reported beside it ("learned" in the JSON line).
METRIC = "particle-substeps/s at 2M pcl, 128^3; learned 4xDT vs plain at <=2% density err"
UNIT = "particle-substeps/s"
FALLBACK_HBM_GBS = 6650.0
SEEDS = {"dam_break_2M": 1235, "dam_break_5M": 1235, "sphere_drop": 1234, "scale_256": 1236, "batched_64": 1237}
# Frames (steps of SUBSTEPS substeps) of each workload's whole run.
WHOLE_RUN = {"dam_break_2M": 1000, "dam_break_5M": 1000, "sphere_drop": 500, "scale_256": 200, "batched_64": 300}
# Algorithmic bytes per unit (FP32 reference state): per particle and per grid
# node of each stage, from the hot-path scope table of this project.
ALGO_BYTES = {"sort": (16, 0), "p2g": (108, 16), "grid": (0, 48), "g2p": (148, 12)}


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000,
                    help="timed frames (each = SUBSTEPS substeps); default: the dam break's 1000 steps")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned 4xDT leg")
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--workload", choices=sorted(SEEDS), default="dam_break_2M")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU-baseline sample budget (0: skip)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--advance", type=int, default=0,
                    help="substeps simulated before the warm-up, to measure a later state of the scene")
    ap.add_argument("--no-whole-run", action="store_true",
                    help="skip the leg that times the workload's whole run from its initial state")
    ap.add_argument("--compare-stages", action="store_true",
                    help="instead of the bench line: per-stage device times of the reference engine and of this "
                         "engine on the workload (K frames after the warm-up), the SDF build and the sort")
    return ap.parse_args(argv)


def make_scene(workload: str, rank: int = 0):
    from mpm_b200 import scenes
    seed = SEEDS[workload] + 1000 * rank
    if workload == "sphere_drop":
        return scenes.sphere_drop(seed)
    if workload == "scale_256":
        return scenes.scale_scene(seed)
    if workload == "batched_64":
        return scenes.batched_scenes(64, seed)
    return scenes.dam_break(seed, literal_extent=(workload == "dam_break_5M"))


def workload_config(workload, cfg, n, t, advance=0):
    grid = f"{cfg.size_x}x{cfg.size_y}x{cfg.size_z}"
    if workload == "batched_64":
        grid = "64 independent scenes, 32-96 nodes per axis each, one launch per stage"
    return {"workload": workload, "grid": grid, "particles": n,
            "advanced_substeps": advance,
            "triangles": t, "substeps_per_step": cfg.substeps,
            "physics": {"padding": cfg.padding, "gravity": cfg.gravity, "dt": cfg.dt, "gamma": cfg.gamma,
                        "compression": cfg.compression, "resolution": cfg.resolution},
            "l2": "inputs larger than L2: particle state 96 B x N per buffer (192 MB at 2M) vs 126 MB L2"}


# ---------------------------------------------------------------- clocks ----
_REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
            0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
            0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}


class ClockSampler:
    """Samples SM clock and clock-event reasons via NVML during a timed region."""

    def __init__(self, cuda_index: int):
        self.samples, self.reasons, self.max_mhz, self.err = [], 0, None, None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml
            self.nv = pynvml
            pynvml.nvmlInit()
            self._h = self._handle(cuda_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # noqa: BLE001 - clocks are reported, not required
            self.err = f"nvml unavailable: {e}"

    def _handle(self, cuda_index):
        pynvml = self.nv
        try:
            import torch
            p = torch.cuda.get_device_properties(cuda_index)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:  # noqa: BLE001
            return pynvml.nvmlDeviceGetHandleByIndex(cuda_index)

    def _reason_bits(self):
        f = getattr(self.nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            getattr(self.nv, "nvmlDeviceGetCurrentClocksThrottleReasons")
        return int(f(self._h))

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self._h, self.nv.NVML_CLOCK_SM))
                self.reasons |= self._reason_bits()
            except Exception as e:  # noqa: BLE001
                self.err = str(e)
            self._stop.wait(0.05)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._h is not None:
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "note": self.err}
        s = sorted(self.samples)
        names = [v for k, v in _REASONS.items() if self.reasons & k and k != 0x1]
        return {"sm_mhz": s[len(s) // 2], "sm_max_mhz": self.max_mhz, "reasons": names, "samples": len(s)}


# ------------------------------------------------------------ distributed ----
class Dist:
    """Barrier and max-over-ranks for the timing; no data-path collective.
    backend "nccl" on GPUs (one rank per GPU), "gloo" for CPU tests."""

    def __init__(self, world: int, local: int, backend: str = "nccl"):
        self.world, self.local, self.backend, self.pg = world, local, backend, None
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
            self.pg = dist

    def barrier(self):
        if self.pg:
            if self.backend == "nccl":
                self.pg.barrier(device_ids=[self.local])
            else:
                self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return FALLBACK_HBM_GBS, "fallback"


def load_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` from a committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)[workload][kernel]["bytes_per_launch"]
    except Exception:  # noqa: BLE001
        return None


def kernel_rooflines(per_sub, n, g_active, peak, peak_kind):
    """Achieved HBM bandwidth of each stage from its average time per substep
    and its algorithmic bytes (ALGO_BYTES), as a fraction of the peak."""
    out = {}
    for k, (bpp, bpn) in ALGO_BYTES.items():
        if per_sub.get(k, 0) <= 0:
            continue
        algo = bpp * n + bpn * g_active
        ach = algo / (per_sub[k] / 1e3) / 1e9
        out[k] = {"ms": round(per_sub[k], 5), "achieved_gbs": round(ach, 1), "frac": round(ach / peak, 4),
                  "algorithmic_bytes": algo}
    out["peak_gbs"] = peak
    out["peak_source"] = f"hbm_gbs of {peak_kind}"
    return out


def whole_run_leg(eng, st0, frames, sub, n, cfg, stream):
    """The workload's whole run (`frames` frames) from its initial state st0:
    device time on the engine's stream, then the same frames again with
    stage events for the per-stage times."""
    import numpy as np
    import torch
    eng.set_state(st0)
    eng.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(frames):
        eng.step_async(sub)
    e1.record(stream)
    eng.synchronize()
    ms = e0.elapsed_time(e1)
    g_end = int(np.count_nonzero(eng.get_grid()[0] > 0))
    eng.set_state(st0)
    eng.set_stage_timing(frames * sub)
    for _ in range(frames):
        eng.step_async(sub)
    stage_ms, cnt = eng.stage_times()
    eng.set_stage_timing(0)
    per_sub = {k: v / max(cnt, 1) for k, v in stage_ms.items()}
    peak, peak_kind = load_peaks()
    return {"frames": frames, "substeps": frames * sub, "value": n * sub * frames / (ms / 1e3), "unit": UNIT,
            "ms_per_step": ms / frames,
            "stage_ms_per_substep": {k: round(v, 5) for k, v in per_sub.items()},
            "roofline_by_kernel": kernel_rooflines(per_sub, n, g_end, peak, peak_kind),
            "active_nodes_at_end": g_end,
            "note": "from the initial state over the workload's whole run; node terms use the active nodes at "
                    "the end of the run"}


# -------------------------------------------------------------- CPU leg ----
CPU_SNIPPET = r"""
import json, os, sys, time
sys.path.insert(0, os.path.join(sys.argv[1], "water-sim-cuda_b200")); sys.path.insert(0, sys.argv[1])
import numpy as np
from bench import make_scene
from oracle.oracle import Oracle
cfg, st, tris = make_scene(sys.argv[2], 0)
o = Oracle(32)
st = o.init_particles(cfg, st)
sdf = np.load(sys.argv[4]).astype(np.float32)  # the SDF the engine built
budget = float(sys.argv[3]); done = 0; t0 = time.perf_counter()
while True:
    st = o.substep(cfg, st, sdf)[0]
    done += 1
    el = time.perf_counter() - t0
    if el >= budget:
        break
model = ""
try:
    for line in open("/proc/cpuinfo"):
        if line.startswith("model name"):
            model = line.split(":", 1)[1].strip()
            break
except OSError:
    pass
print(json.dumps({"substeps": done, "seconds": el, "n": int(st.shape[1]), "threads": o.threads(),
                  "cpu_model": model, "logical_cpus": os.cpu_count()}))
"""


def cpu_baseline(workload: str, seconds: float, sdf):
    """FP32 OpenMP restatement of Engine::step timed on the host cores, in a
    fresh process (no CUDA in it), on the engine's SDF."""
    import tempfile

    import numpy as np
    with tempfile.NamedTemporaryFile(suffix=".npy", delete=False) as f:
        np.save(f, sdf)
        sdf_path = f.name
    try:
        r = subprocess.run([sys.executable, "-c", CPU_SNIPPET, ROOT, workload, str(seconds), sdf_path],
                           capture_output=True, text=True, timeout=900)
    finally:
        os.unlink(sdf_path)
    if r.returncode != 0:
        return {"value": None, "unit": UNIT, "cores": None, "kind": "port", "sample": "failed: " + r.stderr[-300:]}
    d = json.loads(r.stdout.strip().splitlines()[-1])
    return {"value": d["n"] * d["substeps"] / d["seconds"], "unit": UNIT, "cores": d["threads"], "kind": "port",
            "cpu_model": d["cpu_model"], "logical_cpus": d["logical_cpus"],
            "sample": f"{d['substeps']} substeps of the full {d['n']}-particle scene from its initial state (SDF "
                      f"build excluded), FP32 OpenMP restatement of Engine::step on {d['threads']} threads, "
                      f"{d['seconds']:.1f} s"}


# ----------------------------------------------------------- engine arm ----
def run_engine(args, rank, world, local):
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    dist = Dist(world, local)
    import mpm_b200

    scene = make_scene(args.workload, rank)
    batched = isinstance(scene, list)
    if batched:
        cfgs = [c for c, _, _ in scene]
        states = [x for _, x, _ in scene]
        tri_sets = [t for _, _, t in scene]
        cfg, st, tris = cfgs[0], None, np.concatenate(tri_sets)
        n, sub = sum(x.shape[1] for x in states), cfg.substeps

        def make_engine(state_list):
            e = mpm_b200.Batch(cfgs, device=local)
            e.init_all(state_list)
            for k, t in enumerate(tri_sets):
                if len(t):
                    e.init_scene_sdf(k, t)
            return e
        eng = make_engine(states)
    else:
        cfg, st, tris = scene
        n, sub = st.shape[1], cfg.substeps
        eng = mpm_b200.Engine(cfg, device=local)
        eng.init(st)
        eng.init_sdf(tris)
    st0 = None if batched else eng.get_buffer()  # the initial state (initFMatrices applied)
    if args.advance > 0:
        eng.step(args.advance)
    stream = torch.cuda.ExternalStream(eng.stream(), device=local)

    for _ in range(max(args.warmup, 3)):
        eng.step_async(sub)
    eng.synchronize()
    # Launch shapes: the engine's autotuner, timed on these particles (it
    # does not advance the state).
    tuning = None if args.no_autotune else eng.autotune(3)

    # The state the timed frames start from: the instrumented repeat below
    # restarts from it, so that its stage times cover the same frames.
    snap = [eng.scene_buffer(k) for k in range(len(cfgs))] if batched else eng.get_buffer()

    # Timed region: K frames, device time on the engine's stream.
    launches0 = eng.stats()["kernel_launches"]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            eng.step_async(sub)
        e1.record(stream)
        eng.synchronize()
        torch.cuda.synchronize()
        dist.barrier()
    launches = eng.stats()["kernel_launches"] - launches0
    ms = dist.max(e0.elapsed_time(e1))
    value = world * n * sub * args.steps / (ms / 1e3)

    # Instrumented repeat of the same K frames from the same starting state:
    # CUDA events between the stages of every substep.
    if batched:
        eng.init_all(snap)
    else:
        eng.set_state(snap)
    del snap
    eng.set_stage_timing(args.steps * sub)
    for _ in range(args.steps):
        eng.step_async(sub)
    stage_ms, cnt = eng.stage_times()
    eng.set_stage_timing(0)
    per_sub = {k: v / max(cnt, 1) for k, v in stage_ms.items()}
    if batched:
        g_dense = sum(c.grid_number for c in cfgs)
        g_active = sum(int(np.count_nonzero(eng.scene_grid(k)[0] > 0)) for k in range(len(cfgs)))
    else:
        g_dense = cfg.grid_number
        g_active = int(np.count_nonzero(eng.get_grid()[0] > 0))
    peak, peak_kind = load_peaks()
    dom = max(("p2g", "g2p", "grid", "sort"), key=lambda k: per_sub[k])
    bpp, bpn = ALGO_BYTES[dom]
    algo = bpp * n + bpn * g_active
    achieved = algo / (per_sub[dom] / 1e3) / 1e9
    roof = {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": f"hbm_gbs of {peak_kind}",
            "traffic": load_traffic(dom, args.workload),
            "algorithmic_bytes_per_launch": algo, "avg_launch_ms": round(per_sub[dom], 5),
            "units": f"{bpp} B x {n} particles + {bpn} B x {g_active} active nodes (dense grid {g_dense})"}
    by_kernel = kernel_rooflines(per_sub, n, g_active, peak, peak_kind)
    whole = None
    if not batched and not args.no_whole_run and world == 1:
        whole = whole_run_leg(eng, st0, WHOLE_RUN[args.workload], sub, n, cfg, stream)

    # End to end through the C ABI with host buffers (pinned).
    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        if batched:
            st_pins = [pin(x) for x in states]
            pos_pins = [torch.empty((x.shape[1], 3), dtype=torch.float32).pin_memory().numpy() for x in states]
            eng2 = make_engine(st_pins)
            init2 = lambda: eng2.init_all(st_pins)

            def read_positions():
                for k, buf in enumerate(pos_pins):
                    lib.mpm_scene_get_positions(eng2._h, k, buf.ctypes.data)
        else:
            st_pin = pin(st)
            # Two pinned position buffers: frame k is read back (on the
            # engine's copy stream) while frame k + 1 computes.
            pos_pins = [torch.empty((n, 3), dtype=torch.float32).pin_memory().numpy() for _ in range(2)]
            eng2 = mpm_b200.Engine(cfg, device=local)
            eng2.init_sdf(tris)
            init2 = lambda: eng2.init(st_pin)
            frame = [0]

            def read_positions():
                eng2.get_positions_async(pos_pins[frame[0] % 2])
                frame[0] += 1
        lib = mpm_b200.lib
        init2()  # warm the allocation path once
        if tuning:
            eng2.set_tuning(tuning["p2g_ctas_per_sm"], tuning["g2p_block"], tuning["grid_block"],
                            tuning["p2g_cell_cap"])
        eng2.step(sub)
        dist.barrier()
        marks = [time.perf_counter()]
        init2()
        marks.append(time.perf_counter())
        for _ in range(args.steps):
            eng2.step_async(sub)
            read_positions()
            marks.append(time.perf_counter())
        eng2.synchronize()
        eng2.positions_wait()
        marks[-1] = time.perf_counter()
        t0, t1 = marks[0], marks[-1]
        dist.barrier()
        e2e_s = dist.max(t1 - t0)
        frames = [1e3 * (b - a) for a, b in zip(marks[1:-1], marks[2:])]
        e2e = {"value": world * n * sub * args.steps / e2e_s, "unit": UNIT,
               # mpm_init_particles copies the 21 planes its import reads (not
               # F's diagonal, VOL or MASS, which the init rules set)
               "h2d_bytes_per_step": int(21 * 4 * n / args.steps), "d2h_bytes_per_step": 12 * n,
               "timed": "mpm_init_particles(pinned host state) + K x (mpm_step_async(SUBSTEPS) + "
                        "positions read back to pinned memory: mpm_get_positions_async, one frame's copy "
                        "overlapping the next frame's substeps) + the final synchronisation; host wall "
                        "clock, max over ranks",
               "init_ms": round(1e3 * (marks[1] - marks[0]), 3),
               "frame_ms": {"min": round(min(frames), 3), "median": round(sorted(frames)[len(frames) // 2], 3),
                            "max": round(max(frames), 3)}}
        eng2.close()

    cpu = None
    if rank == 0 and world == 1 and args.cpu_seconds > 0 and not batched:
        cpu = cpu_baseline(args.workload, args.cpu_seconds, eng.get_sdf())
    learned = None
    if not args.no_learned and args.workload == "dam_break_2M" and not batched:
        learned = learned_leg(cfg, st, tris, local)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": dict(workload_config(args.workload, cfg, n, len(tris), args.advance), parallelism=f"replicas{world}"),
            "tuning": None if tuning is None else
                      {k: (round(v, 5) if isinstance(v, float) else v) for k, v in tuning.items()},
            "e2e": e2e, "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu,
            "clocks": clk.summary(), "stage_ms_per_substep": {k: round(v, 5) for k, v in per_sub.items()},
            "roofline_by_kernel": by_kernel, "whole_run": whole,
            "impl": "engine"}
    if learned is not None:
        line["learned"] = learned
    eng.close()
    dist.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def learned_leg(cfg, st, tris, device):
    """The learned 4xDT path beside the plain engine on the same scene: both
    from the same state, plain for 4 x 100 substeps, learned for 100 large
    steps, simulated time per second of each (host wall clock around
    synchronous calls: a checked large step reads its fallback statistic), and
    the learned state's distance from the plain one; "perturbed" is the plain
    run from positions moved by 1e-4 cells, the scene's chaos floor.  Fallback
    rules (Engine.set_fallback_rule) at 2 %: "rest_density" (the predicted
    density's deviation from rest density), "density_change" (the density
    change the step predicts), and none."""
    from mpm_b200 import learned as L
    out = {}
    legs = {"literal": (("density_change_2pct", "density_change", 0.02), ("no_fallback", "density_change", -1.0)),
            "physical": (("rest_density_2pct", "rest_density", 0.02),
                         ("density_change_2pct", "density_change", 0.02), ("no_fallback", "density_change", -1.0))}
    for name, path, phys in (("literal", L.DEFAULT_PARAMS, False), ("physical", L.PHYSICAL_PARAMS, True)):
        if not os.path.exists(path):
            out[name] = {"unavailable": f"no trained corrector parameters ({os.path.basename(path)})"}
            continue
        params, meta = L.load_params(path)
        c = L.physical_config(cfg) if phys else cfg
        v = {"config": "GRAVITY and GAMMA as configured" if not phys else
             "physical orientation: GRAVITY and GAMMA negated (gravity pulls -y, pressure resists compression)"}
        for key, rule, thr in legs[name]:
            res = L.evaluate(c, st, tris, params, nlarge=100, ratio=int(meta.get("ratio", 4)),
                             max_density_change=thr, checkpoints=(10, 25, 100), rule=rule)
            r = {"rule": rule if thr >= 0 else None, "threshold": thr if thr >= 0 else None,
                 "speedup_sim_time": round(res["speedup_sim_time"], 3),
                 "sim_time_per_s": {k: round(res[k]["sim_time_per_s"], 2) for k in ("plain", "learned", "uncorrected")},
                 "fallbacks": res["learned"].get("fallbacks"),
                 "mean_statistics": {k: round(x, 5) for k, x in res["learned"].get("mean_statistics", {}).items()}}
            for tag in ("learned", "uncorrected", "perturbed"):
                r[tag] = {m: {k: round(val, 4) for k, val in res[tag][f"at_{m}"].items()} for m in (10, 25, 100)}
            v[key] = r
        v["trained_on"] = {k: meta.get(k) for k in ("variants", "dataset", "steps", "batch")}
        out[name] = v
    out["ratio"] = 4
    out["large_steps"] = 100
    return out


# -------------------------------------------------------- reference arm ----
def run_reference(args, rank, world, local):
    if rank != 0:
        return
    from oracle.oracle import REF_LIB, RefEngine
    if not os.path.exists(REF_LIB):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_engine.so was not built "
                          "(the reference sources were absent at build time)"}))
        return
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    scene = make_scene(args.workload, 0)
    # The reference runs one scene per process (a __constant__ config); a
    # batch is timed scene after scene, over the scenes whose grid it can run
    # (its grid kernels have no bounds check: node count a multiple of 256).
    runs = scene if isinstance(scene, list) else [scene]
    runs = [r for r in runs if r[0].grid_number % 256 == 0]
    cfg, tris = runs[0][0], np.concatenate([r[2] for r in runs])
    sub = cfg.substeps
    n, ms = 0, 0.0
    ref = RefEngine()
    with ClockSampler(local) as clk:
        for c, st, t in runs:
            ref.create(c, st, t, f"/tmp/ref_bench_config_{os.getpid()}.txt")
            ref.step(args.advance + max(args.warmup, 3) * sub)
            ms += ref.time_steps(args.steps * sub)
            n += st.shape[1]
    ref.destroy()
    value = n * sub * args.steps / (ms / 1e3)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": dict(workload_config(args.workload, cfg, n, len(tris), args.advance), parallelism="replicas1"),
            "reference_scenes": len(runs),
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": f"{args.steps} frames x {sub} Engine::step() of the reference's own CUDA "
                                       "engine compiled from its sources for sm_100a; the reference implements "
                                       "this path only in CUDA, so it runs on the GPU driven by 1 host thread"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def compare_stages(args, local):
    """Per-stage device times (CUDA events) of the reference's engine and of
    this engine on the same scene and frames, plus the one-time SDF build and
    the bit-exact sort on their own.  One JSON line."""
    import numpy as np
    import torch
    from oracle.oracle import REF_LIB, RefEngine
    import mpm_b200
    torch.cuda.set_device(local)
    cfg, st, tris = make_scene(args.workload, 0)
    n, sub, K = st.shape[1], cfg.substeps, args.steps
    out = {"workload": args.workload, "particles": n, "frames": K, "substeps": K * sub, "advanced": args.advance}
    if os.path.exists(REF_LIB) and cfg.grid_number % 256 == 0:
        ref = RefEngine()
        ref.create(cfg, st, tris, f"/tmp/ref_stages_config_{os.getpid()}.txt")
        ref.step(args.advance + max(args.warmup, 3) * sub)
        r = ref.time_stages(K * sub)
        out["reference_ms_per_substep"] = {k: round(v / (K * sub), 5) for k, v in r.items()}
        out["reference_make_sdf_ms"] = round(ref.time_make_sdf(tris), 3)
        out["reference_sort_ms"] = round(ref.time_sort(10), 4)
        ref.destroy()
    with mpm_b200.Engine(cfg, device=local) as eng:
        eng.init(st)
        stream = torch.cuda.ExternalStream(eng.stream(), device=local)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        eng.init_sdf(tris)  # warm
        ev[0].record(stream)
        eng.init_sdf(tris)
        ev[1].record(stream)
        torch.cuda.synchronize()
        out["sdf_build_ms"] = round(ev[0].elapsed_time(ev[1]), 3)
        eng.step(args.advance + max(args.warmup, 3) * sub)
        eng.autotune(3)
        eng.set_stage_timing(K * sub)
        for _ in range(K):
            eng.step_async(sub)
        ms, cnt = eng.stage_times()
        eng.set_stage_timing(0)
        out["engine_ms_per_substep"] = {k: round(v / max(cnt, 1), 5) for k, v in ms.items()}
        out["engine_tuning"] = eng.tuning()
        # The bit-exact Morton sort on the same positions (caller-owned buffers).
        cur = eng.get_buffer()
        d = torch.from_numpy(np.ascontiguousarray(cur[0:3])).cuda()
        keys = torch.empty(n, dtype=torch.int32, device="cuda")
        perm = torch.empty(n, dtype=torch.int32, device="cuda")
        cs = torch.cuda.current_stream()
        args_ = (d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), n, keys.data_ptr(), perm.data_ptr(),
                 cs.cuda_stream)
        mpm_b200.sort_particles_device(*args_)
        ev[0].record(cs)
        for _ in range(10):
            mpm_b200.sort_particles_device(*args_)
        ev[1].record(cs)
        torch.cuda.synchronize()
        out["engine_sort_ms"] = round(ev[0].elapsed_time(ev[1]) / 10, 4)
    print(json.dumps(out), flush=True)


def main(argv=None):
    args = parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.compare_stages:
        if rank == 0:
            compare_stages(args, local)
    elif args.impl == "reference":
        run_reference(args, rank, world, local)
    else:
        run_engine(args, rank, world, local)


if __name__ == "__main__":
    main()
