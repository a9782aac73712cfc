"""The multi-rank logic of bench.py on CPU: two gloo ranks, each tracking its
own shard (a different seeded pair, no data-path collective) with the CPU
oracle as the per-rank step, then the max-over-ranks timing reduction."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str):
    import importlib
    import time

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    import bind
    wl = importlib.import_module("p-tracker_b200.workloads")
    pair = wl.make_pair("tiny", seed=bench.rank_seed(rank))
    opts = wl.tracker_options(pair["params"])
    t = bind.setup(bind.Port, pair, threads=1, zones=opts["zones"], params={"rescue_level": 0, "iraz": 100})
    t0 = time.perf_counter()
    t.track_frame(1)
    ms = (time.perf_counter() - t0) * 1e3 + 5.0 * rank  # rank 1 is the slow one
    red = bench.reduce_max([ms, float(rank)], world)
    n = pair["rec"].shape[0]
    np.save(Path(out_dir) / f"rank{rank}.npy", np.array([ms, red[0], red[1], n,
                                                          bench.aggregate_rate(n, world, red[0]),
                                                          pair["rec"][:, 0].sum()]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce(tmp_path, oracle, wl):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0 = np.load(tmp_path / "rank0.npy")
    r1 = np.load(tmp_path / "rank1.npy")
    # both ranks agree on the reduced (max) time and it is the slower rank's
    assert r0[1] == r1[1] == max(r0[0], r1[0])
    assert r0[2] == r1[2] == 1.0
    # whole-job rate = all ranks' grains over the slowest rank's time
    assert abs(r0[4] - (r0[3] * 2) / (r0[1] * 1e-3)) < 1e-6 * r0[4]
    # shards differ (own seed per rank)
    assert r0[5] != r1[5]
