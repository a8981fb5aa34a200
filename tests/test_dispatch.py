"""The multi-GPU case dispatch of the batching and serving forms (no collective on
the data path: every case runs whole on one GPU, the GPUs of a node split one
case list).  Host logic only: two gloo ranks on the CPU derive their shares of
the list, gather them, and merge their time-to-converge records as the bench
does at N > 1."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from myjoe_b200 import serve


def _specs():
    return serve.case_specs(24, 5000, 500000, seed=1000)


def test_partition_is_complete_disjoint_and_balanced():
    specs = _specs()
    for world in (1, 2, 3, 4, 8):
        shares = [serve.partition_cases(specs, world, r) for r in range(world)]
        ids = sorted(id(s) for sh in shares for s in sh)
        assert ids == sorted(id(s) for s in specs)   # every case on exactly one GPU
        loads = [sum(serve.spec_cells(s) for s in sh) for sh in shares]
        biggest = max(serve.spec_cells(s) for s in specs)
        assert max(loads) - min(loads) <= biggest    # longest-first greedy bound
        for sh in shares:                             # list order kept within a share
            pos = [specs.index(s) for s in sh]
            assert pos == sorted(pos)
    assert serve.partition_cases(specs, 1, 0) == specs
    with pytest.raises(ValueError):
        serve.partition_cases(specs, 2, 2)


def test_merge_adds_solves_and_takes_the_ratio_of_sums():
    a = {"solves_per_hour": 100.0, "cases": 12, "cells_total": 10, "plain_fp64": {"solves_per_hour": 50.0}}
    b = {"solves_per_hour": 300.0, "cases": 12, "cells_total": 30, "plain_fp64": {"solves_per_hour": 150.0}}
    m = serve.merge_rank_results([a, b])
    assert m["solves_per_hour"] == 400.0 and m["ratio_vs_plain_fp64"] == 2.0
    assert m["cases"] == 24 and m["cells_total"] == 40 and m["gpus"] == 2


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = serve.partition_cases(_specs(), world, rank)
        got = [None] * world
        dist.all_gather_object(got, [(s["nx"], s["ny"], s["seed"]) for s in mine])
        rec = {"solves_per_hour": float(len(mine)), "cases": len(mine), "cells_total": 1,
               "plain_fp64": {"solves_per_hour": 0.5 * len(mine)}}
        recs = [None] * world
        dist.all_gather_object(recs, rec)
        if rank == 0:
            out.put((got, serve.merge_rank_results(recs)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_one_case_list():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    allcases = [(s["nx"], s["ny"], s["seed"]) for s in _specs()]
    assert sorted(got[0] + got[1]) == sorted(allcases) and not set(got[0]) & set(got[1])
    assert merged["cases"] == 24 and merged["gpus"] == 2 and merged["ratio_vs_plain_fp64"] == 2.0
