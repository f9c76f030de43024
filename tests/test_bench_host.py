"""Host logic of bench.py: arguments, replica seeding, and the N>1 timing
reduction run as two gloo ranks on the CPU (the GPU run uses NCCL with the
same code)."""
import json
import os
import socket

import numpy as np
import pytest


def test_defaults():
    import bench
    a = bench.parse_args([])
    assert (a.gpus, a.warmup, a.impl, a.workload) == (1, 3, "engine", "dam_break_2M")
    assert a.steps >= 1


def test_replica_scenes_differ_per_rank():
    import bench
    c0, s0, t0 = bench.make_scene("sphere_drop", 0)
    c1, s1, t1 = bench.make_scene("sphere_drop", 1)
    assert s0.shape[1] == s1.shape[1] and not np.array_equal(s0[0:3], s1[0:3])


def test_algorithmic_bytes_table():
    import bench
    assert bench.ALGO_BYTES["p2g"] == (108, 16) and bench.ALGO_BYTES["g2p"] == (148, 12)
    # 288 B per particle-substep = keys 16 (fused into G2P here) + sort 16 + P2G 108 + G2P 148
    assert 16 + sum(v[0] for v in bench.ALGO_BYTES.values()) == 288


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench
    d = bench.Dist(world, rank, backend="gloo")
    d.barrier()
    got = d.max(10.0 + rank)
    d.barrier()
    d.close()
    with open(out, "w") as f:
        json.dump({"rank": rank, "max": got}, f)


def test_two_rank_max_over_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    outs = [str(tmp_path / f"r{r}.json") for r in range(2)]
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, outs[r])) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for o in outs:
        assert json.load(open(o))["max"] == 11.0


def test_reference_arm_without_library(tmp_path, monkeypatch, capsys):
    import bench
    import oracle.oracle as oo
    monkeypatch.setattr(oo, "REF_LIB", str(tmp_path / "nothing.so"))
    bench.run_reference(bench.parse_args(["--impl", "reference"]), 0, 1, 0)
    line = json.loads(capsys.readouterr().out.strip())
    assert line["impl"] == "reference" and "unavailable" in line


def test_reference_arm_other_ranks_exit(capsys):
    import bench
    bench.run_reference(bench.parse_args(["--impl", "reference"]), 1, 2, 1)
    assert capsys.readouterr().out == ""
