"""LPT placement of ensemble boxes on ranks, and a world-size-2 gloo run in which each rank
builds its share independently and the shares cover every box exactly once."""
import os

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from astr_gpu_b200.fields import ensemble_specs
from astr_gpu_b200.shard import box_cost, lpt_partition


def test_lpt_covers_and_balances():
    specs = ensemble_specs(48, 48)
    costs = [box_cost(s.n) for s in specs]
    for n in (1, 2, 3, 4, 8):
        parts = lpt_partition(costs, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(48))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: max load <= 4/3 of the optimum, and the optimum >= max(mean, largest box)
        lower = max(sum(costs) / n, max(costs))
        assert max(loads) <= 4.0 / 3.0 * lower + 1e-9


def test_lpt_deterministic_and_edge_cases():
    assert lpt_partition([], 3) == [[], [], []]
    assert lpt_partition([5, 5, 5], 3) == [[0], [1], [2]]
    assert lpt_partition([1, 2, 3], 1) == [[0, 1, 2]]
    with pytest.raises(ValueError):
        lpt_partition([1], 0)


def _worker(rank, ws, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    specs = ensemble_specs(48, 48)
    mine = lpt_partition([box_cost(s.n) for s in specs], ws)[rank]
    got = [None] * ws
    dist.all_gather_object(got, mine)
    out[rank] = got
    dist.destroy_process_group()


def test_gloo_two_ranks_partition_agrees():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn")
    a, b = out[0], out[1]
    assert a == b
    assert sorted(a[0] + a[1]) == list(range(48))
    assert not set(a[0]) & set(a[1])


def test_ensemble_specs_seeded():
    from astr_gpu_b200.fields import tgv_q
    a, b = ensemble_specs(), ensemble_specs()
    assert a == b and len(a) == 48
    assert {s.n for s in a} <= {32, 48, 64, 96, 128}
    assert all(0.1 <= s.mach <= 0.5 and 400 <= s.reynolds <= 3200 for s in a)
    assert sum(s.kind == "tgv" for s in a) == 24
    q = tgv_q(8, 0.1)
    assert q.shape == (9, 9, 9, 5) and q.flags["F_CONTIGUOUS"]
