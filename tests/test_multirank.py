"""The multi-rank host logic of bench.py on CPU: two gloo ranks, as torchrun would start them.

Cells are independent, so ranks share nothing on the data path: each draws its own shard, the job's
rate is (ranks x cells x steps) over the slowest rank's time, and the reference arm runs on rank 0
only.  The GPU path is the same code with the NCCL backend.
"""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, str(ROOT))
    import json

    import numpy as np
    import torch.distributed as dist

    import bench

    args = bench.parse_args(["--gpus", str(world), "--steps", "3", "--warmup", "3", "--impl", "reference"])
    w, r, _ = bench.dist_setup(args)
    assert (w, r) == (world, rank) and dist.get_backend() == "gloo"
    # the slowest rank sets the job time
    rate, t = bench.weak_rate(w, 4096, 10, 1.0 + rank)
    # each rank's shard of cells is its own draw, same shape
    cells = bench.make_cells(4, 4, 64, seed=bench.rank_seed(args.seed, r))
    # the reference arm: rank 0 alone does the work and prints
    ref = bench.run_reference(args) if r != 0 else "skipped on rank 0 (CPU time)"
    bench.dist_barrier(w)
    res = {"rate": rate, "t": t, "cells_digest": float(np.abs(cells).sum()), "shape": list(cells.shape),
           "ref": ref}
    Path(out_dir, f"rank{rank}.json").write_text(json.dumps(res))
    dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import json

    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r in res:
        assert r["t"] == pytest.approx(2.0)  # max over ranks of 1.0, 2.0
        assert r["rate"] == pytest.approx(2 * 4096 * 10 / 2.0)
        assert r["shape"] == [64, 4, 25]
    assert res[0]["cells_digest"] != res[1]["cells_digest"]  # different shards
    assert res[1]["ref"] is None  # non-zero ranks of the reference arm exit without work

