"""The multi-GPU form of bench.py on CPU ranks (gloo, world size 2).

bench.py runs one replica per GPU: every rank corrects its own series, with
no collective on the data path.  What the ranks share is the timing: the
job lasts as long as its slowest rank (max over ranks of the device-timed
steps and of the end-to-end time), and the whole-job rate counts the
registrations of every rank.  Under torchrun the reference arm runs on rank
0 alone, and the other ranks exit 0 without work.  These tests run the
same functions on two gloo ranks on 127.0.0.1; the NCCL form differs only
in the tensor's device."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r's step time and end-to-end time; the slowest of each is
        # rank 1's step (12 ms) and rank 0's end-to-end (9 ms)
        ms, e2e_ms = 10.0 + 2.0 * rank, 9.0 - 3.0 * rank
        got = bench.max_over_ranks([ms, e2e_ms], world, torch.device("cpu"))
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(got, f)
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        with open(tmp_path / f"rank{r}.json") as f:
            assert json.load(f) == [12.0, 9.0]


def test_one_rank_keeps_its_own_times():
    assert bench.max_over_ranks([1.5, 2.5], 1, None) == [1.5, 2.5]


def test_whole_job_rate_counts_every_replica():
    # 2 replicas x 3 steps x (T - 1) registrations in the slowest rank's 12 ms
    assert bench.whole_job_rate(2, 3, 12.0) == pytest.approx(2 * 3 * (bench.T - 1) / 0.012)
    assert bench.whole_job_rate(1, 3, 12.0) == pytest.approx(bench.whole_job_rate(2, 3, 12.0) / 2)


def test_replicas_register_their_own_series(monkeypatch):
    monkeypatch.setattr(bench, "T", 4)
    a0, _ = bench.make_series(0)
    a1, _ = bench.make_series(1)
    b1, _ = bench.make_series(1)
    assert a0.shape == a1.shape == (4,) + bench.SHAPE
    assert (a1 == b1).all()          # seeded by the rank: the same series on every run
    assert not (a0 == a1).all()      # and a different one on each rank


def test_reference_arm_idles_on_ranks_other_than_zero():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
