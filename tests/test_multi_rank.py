"""The N > 1 host logic on CPU: two gloo ranks (127.0.0.1), max-over-ranks timing,
summed throughput and the LPT packing of ensemble members onto ranks."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from openpfc_b200 import parallel_plan as pp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, members, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mine = pp.members_for_rank(members, rank, world)
        ms = 10.0 + 5.0 * rank  # a rank-dependent "timing"
        mx = pp.max_over_ranks(ms)
        cells = sum(m["n"][0] * m["n"][1] * m["n"][2] for m in mine)
        tot = pp.sum_over_ranks(cells)
        dist.barrier()
        out[rank] = (mx, tot, [m["id"] for m in mine])
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    members = [{"n": (s, s, s), "id": i} for i, s in enumerate([32, 96, 48, 64, 80, 96, 32, 48])]
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, _free_port(), members, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0
    total = sum(m["n"][0] ** 3 for m in members)
    assert res[0][1] == res[1][1] == total
    ids = sorted(res[0][2] + res[1][2])
    assert ids == list(range(len(members)))
    assert not set(res[0][2]) & set(res[1][2])


def test_lpt_balance():
    costs = [pp.member_cost((s, s, s)) for s in [32, 48, 64, 80, 96] * 20]
    parts, loads = pp.lpt_partition(costs, 8)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    # LPT is within 4/3 of optimal; the mean load bounds optimal from below
    assert max(loads) <= (4.0 / 3.0) * (sum(loads) / 8) + max(costs)
    with pytest.raises(ValueError):
        pp.lpt_partition(costs, 0)


def test_single_process_identity():
    assert pp.max_over_ranks(3.5) == 3.5
    assert pp.sum_over_ranks(2.0) == 2.0
    _ = torch
