"""Multi-GPU form of the tracer: independent replicas (rays and bundles
share nothing, so there is no data-path collective).  The host logic of
`bench.py --gpus N` runs here as world_size-2 gloo ranks on the CPU: every rank
gets the slowest rank's time from one all-reduce, the whole-job value is all
ranks' rays over that time, and each rank's environment is read the way
torchrun sets it."""
import json
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime

    import torch.distributed as dist

    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        ws, r, local = bench.dist_env()
        own_ms = 100.0 + 25.0 * rank  # rank 1 is the slow one
        slowest = bench.max_over_ranks(own_ms, ws, "cpu")
        value = bench.replica_value(4_194_304, ws, 5, slowest)
        dist.barrier()
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"ws": ws, "rank": r, "local": local, "slowest": slowest, "value": value}, f)


def test_two_replicas_report_the_slowest_rank(tmp_path):
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for r, d in enumerate(res):
        assert (d["ws"], d["rank"], d["local"]) == (2, r, r)
        assert d["slowest"] == 125.0
        assert d["value"] == pytest.approx(2 * 4_194_304 * 5 / 0.125 / 1e6)
