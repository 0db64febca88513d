"""The multi-GPU path of this solver is replicas only: each rank solves its own slabs
(disjoint seeds), the job's time is the slowest rank's, and rank 0 alone reports. These
tests run that host logic of bench.py on two gloo ranks on the CPU (rendezvous on
127.0.0.1); no GPU is involved."""

import io
import os
import socket
import sys
from contextlib import redirect_stdout
from pathlib import Path

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        res = {}
        # the job's time is the slowest rank's
        res["max"] = bench.max_over_ranks(10.0 + 5.0 * rank, world, torch.device("cpu"))
        # disjoint per-rank workloads: the ranks' batch slabs differ
        probs = bench.batch_problems(dict(bench.WORKLOADS["cfg3"], batch=4), seed=bench.rank_seed(1000, rank))
        key = torch.tensor([float(p.geometry.M * 1000 + p.geometry.N_z) + p.omega for p in probs],
                           dtype=torch.float64)
        keys = [torch.empty_like(key) for _ in range(world)]
        dist.all_gather(keys, key)
        res["disjoint"] = not torch.equal(keys[0], keys[1])
        # the reference arm: rank 0 alone runs and prints; the others exit 0 without work
        args = bench.argparse.Namespace(warmup=0, steps=0, gpus=world, workload="cfg1")
        buf = io.StringIO()
        if rank != 0:
            with redirect_stdout(buf):
                res["ref_rc"] = bench.run_reference(args, bench.WORKLOADS["cfg1"], rank, world)
            res["ref_out"] = buf.getvalue()
        dist.barrier()
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_replicas_on_two_gloo_ranks():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0]["max"] == res[1]["max"] == 15.0
    assert res[0]["disjoint"] and res[1]["disjoint"]
    assert res[1]["ref_rc"] == 0 and res[1]["ref_out"] == ""
