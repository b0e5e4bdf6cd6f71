"""Host-side logic of multi-GPU bench runs, on CPU with world_size-2 gloo ranks.

`bench.py --gpus N` runs N independent replicas of the MD workload, one rank per
GPU; the ranks meet only at barriers and at one MAX all-reduce of their timings,
and rank 0 alone prints.  These tests run that host logic (the reduction, the
whole-job rate, the reference arm's rank-0-only rule) without a GPU.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch
    import bench

    torch.distributed.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                         world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # per-rank step time, FP64 step time and inverse end-to-end rate: rank 1 is slower on
        # the first two, rank 0 on the third
        mine = [100.0 + 50.0 * rank, 300.0 - 10.0 * rank, 1e-6 * (2 - rank)]
        torch.distributed.barrier()
        got = bench.max_over_ranks(torch, mine, world, "cpu")
        rate = bench.whole_job_rate(1000, world, 20, got[0])
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"max": got, "rate": rate}, f)
    finally:
        torch.distributed.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_gloo(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    # every rank sees the same maxima: the slowest rank's value of each entry
    for r in res:
        assert r["max"] == pytest.approx([150.0, 300.0, 2e-6], rel=0, abs=1e-15)
        # 2 ranks x 1000 atoms x 20 steps in the slowest rank's 150 ms
        assert r["rate"] == pytest.approx(2 * 1000 * 20 / 0.150, rel=1e-12)


def test_single_rank_needs_no_process_group():
    import torch
    import bench

    assert not torch.distributed.is_initialized()
    assert bench.max_over_ranks(torch, [1.5, 0.0, 3.0], 1, "cpu") == [1.5, 0.0, 3.0]
    assert bench.whole_job_rate(1_024_000, 1, 200, 360.0) == pytest.approx(1_024_000 * 200 / 0.36)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


def test_reference_arm_rank0_prints_one_line():
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    p = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    lines = [l for l in p.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "atom-step/s"
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "atom-step/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
