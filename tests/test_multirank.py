"""bench.py's multi-GPU path on CPU: world_size 2 over gloo.  Each rank runs an
independent replica (the single-mesh path does not shard), the job time is
the max over ranks and the rate aggregates the ranks' iterations; the
reference arm runs on rank 0 only."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = [12.0, 15.0][rank]                      # rank 1 is the slow replica
    m = bench.reduce_max(ms, dist, "cpu")
    out[rank] = (m, bench.aggregate_rate(world, 10, m))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_aggregate_rate():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    assert out[0] == out[1]
    m, rate = out[0]
    assert m == 15.0
    assert abs(rate - 2 * 10 / 0.015) < 1e-9


def test_reference_arm_only_on_rank0(monkeypatch, capsys):
    import argparse
    import bench
    args = argparse.Namespace(n=8, steps=2, warmup=1, gpus=2, impl="reference")
    bench.run_reference(args, rank=1)
    assert capsys.readouterr().out == ""


def _shard_worker(rank, world, port, out):
    # each rank takes its share of the 64-case ensemble (as bench.py --ensemble
    # does); the whole-job cell count is the only collective
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    from flowsolversourcecode_b200 import ensemble as E
    specs = E.make_specs(64, seed=0)
    mine = E.shard([s.cells for s in specs], world)[rank]
    cells = torch.tensor([float(sum(specs[q].cells for q in mine))], dtype=torch.float64)
    dist.all_reduce(cells)
    got = [None] * world
    dist.all_gather_object(got, mine)
    out[rank] = (cells.item(), got)
    dist.barrier()
    dist.destroy_process_group()


def test_ensemble_shards_over_ranks():
    from flowsolversourcecode_b200 import ensemble as E
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_shard_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    specs = E.make_specs(64, seed=0)
    total, parts = out[0]
    assert out[1][0] == total == float(sum(s.cells for s in specs))
    assert sorted(q for p in parts for q in p) == list(range(64))
    assert not set(parts[0]) & set(parts[1])


def _solve_shard(specs, idx, iters=4):
    """Outer iterations of the cases `idx` on the CPU restatement (the stand-in
    for a GPU rank's work here): per case the final stop metric and u."""
    import numpy as np
    import oracle
    from flowsolversourcecode_b200 import ensemble as E
    out = {}
    for q, (mesh, case) in zip(idx, E.build_cases([specs[q] for q in idx], workers=1, solver_cont="bicgs",
                                                     batched_momentum=False)):
        o = oracle.Oracle(mesh, case)
        src = [o.simple_iteration() for _ in range(iters)]
        out[q] = (src[-1], float(np.abs(o.get("u")).sum()))
    return out


def _solve_worker(rank, world, port, out):
    # each rank solves its shard of a small ensemble end to end; the results and
    # the per-rank time meet only in the final gather and max-reduce
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import time
    import bench
    from flowsolversourcecode_b200 import ensemble as E
    specs = E.make_specs(6, seed=3, edges=(4, 7))
    mine = E.shard([s.cells for s in specs], world)[rank]
    t0 = time.perf_counter()
    res = _solve_shard(specs, mine)
    ms = bench.reduce_max((time.perf_counter() - t0) * 1e3, dist, "cpu")
    got = [None] * world
    dist.all_gather_object(got, res)
    out[rank] = (ms, got)
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_ensemble_solves_match_single_process(oracle_lib):
    from flowsolversourcecode_b200 import ensemble as E
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_solve_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    specs = E.make_specs(6, seed=3, edges=(4, 7))
    ref = _solve_shard(specs, list(range(len(specs))))
    assert out[0][0] == out[1][0] > 0.0                       # the job time is the max over ranks
    merged = {}
    for part in out[0][1]:
        assert not set(part) & set(merged)                   # every case on exactly one rank
        merged.update(part)
    assert sorted(merged) == list(range(len(specs)))
    for q in ref:
        assert merged[q] == ref[q], q                        # same iterates, bit for bit
