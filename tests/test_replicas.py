"""The multi-GPU path of bench.py is independent replicas (the hot path does not shard):
every rank builds its own seeded box and reports its step time; rank 0 prints the maximum
over the ranks.  Checked here with two gloo ranks on the CPU: the maximum reaches every rank,
the ranks' boxes differ only in their seed, and the reference arm runs on rank 0 alone."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        r, w, _ = bench.dist_env()
        v = bench.max_over_ranks(1.5 + r, w, device="cpu")
        _, box, cfg = bench.build_inputs(r)
        out[r] = (v, cfg["seed"] + r, float(box.x[0]), box.nm, box.box)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas():
    world = 2
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 2.5          # the slower rank's time on every rank
    assert res[0][1] != res[1][1]                  # a seed per rank
    assert res[0][2] != res[1][2]                  # hence a different box
    assert res[0][3:] == res[1][3:]                # of the same size


def test_reference_arm_runs_on_rank_zero_only(capsys, monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        steps, warmup, gpus = 1, 0, 2
    assert bench.run_reference(Args()) is None
    assert capsys.readouterr().out == ""
