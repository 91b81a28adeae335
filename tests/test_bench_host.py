"""CPU tests of bench.py's host logic: argument defaults, the max-over-ranks
timing reduction on world_size 2 (gloo), mask packing and the reference arm."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_defaults_finish_quickly():
    a = bench.parse_args([])
    assert a.gpus == 1 and a.warmup >= 3 and a.steps >= 1
    assert a.impl == "ours"


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    v = bench.max_over_ranks(float(10 + rank * 5), world, device="cpu")
    bench.barrier(world)
    q.put((rank, v))
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    got = sorted(q.get() for _ in range(2))
    assert got == [(0, 15.0), (1, 15.0)]


def test_pack_mask_torch_matches_numpy():
    from cudf_b200.column import pack_mask

    rng = np.random.default_rng(0)
    for n in (1, 31, 32, 33, 1000, 4097):
        v = rng.random(n) > 0.3
        got = bench.pack_mask_torch(torch.from_numpy(v)).numpy()
        want = pack_mask(v)
        assert np.array_equal(got[: len(want)], want[: len(got)])


def test_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--cpu-sample-rows", "20000", "--cards", "100,10000"],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "rows/s"
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0


def test_gpus_must_match_world_size():
    env = dict(os.environ, WORLD_SIZE="3", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--impl", "reference"],
                       capture_output=True, text=True, timeout=120, cwd=ROOT, env=env)
    assert r.returncode == 2
    assert "does not match WORLD_SIZE=3" in r.stderr


def test_replica_command_runs_n_ranks_on_loopback():
    cmd = bench.replica_command(4, ["--gpus", "4", "--steps", "2"], 29555)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-4:] == ["--gpus", "4", "--steps", "2"]
