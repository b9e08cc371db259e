"""The sharded patch run on two ranks (gloo, CPU): the dealing of `batch.deal` and the two
collectives of `batch.reduce_totals` that `bench.py --workload patches --gpus N` uses.

Each rank runs in its own process, deals the same seeded patch sizes, reports which patches it
owns, its cell load, and the reductions of its fake device time and cells x iterations.  The parent
checks that every patch is owned exactly once, that the loads differ by no more than the largest
patch, and that the reductions equal the max and the sum taken on one rank.
"""
import os
import socket

import pytest

from fluidisim_b200 import batch

WORLD = 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _sizes(n=61, seed=5):
    import numpy as np
    rng = np.random.default_rng(seed)
    sides = (8 * np.round(np.exp(rng.uniform(np.log(16), np.log(96), size=(n, 3))) / 8)).astype(int)
    return [int(a * b * c) for a, b, c in sides]


def _iterations(i: int) -> int:
    return 7 + (i * 13) % 11


def _rank_main(rank, world, port, out_dir):
    import json

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cells = _sizes()
        mine = batch.deal(cells, world, rank)
        my_ci = sum(cells[i] * _iterations(i) for i in mine)
        my_ms = 10.0 + 3.5 * rank
        ms, ci = batch.reduce_totals(my_ms, my_ci, world)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"mine": mine, "load": sum(cells[i] for i in mine), "ms": ms, "ci": ci}, f)
    finally:
        dist.destroy_process_group()


def test_snake_order():
    assert [batch.snake_owner(k, 3) for k in range(9)] == [0, 1, 2, 2, 1, 0, 0, 1, 2]
    assert all(batch.snake_owner(k, 1) == 0 for k in range(5))


def test_one_rank_keeps_everything():
    cells = _sizes(17)
    assert batch.deal(cells, 1, 0) == sorted(range(17), key=lambda i: (-cells[i], i))
    assert batch.reduce_totals(4.0, 12.0, 1) == (4.0, 12.0)


@pytest.mark.parametrize("world", [2, 3, 4, 8])
def test_dealing_partitions_and_balances(world):
    cells = _sizes()
    owned = [batch.deal(cells, world, r) for r in range(world)]
    flat = sorted(i for o in owned for i in o)
    assert flat == list(range(len(cells)))
    loads = [sum(cells[i] for i in o) for o in owned]
    assert max(loads) - min(loads) <= max(cells)


def test_two_gloo_ranks_deal_and_reduce(tmp_path):
    import json

    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(WORLD, port, str(tmp_path)), nprocs=WORLD, join=True, start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(WORLD)]
    cells = _sizes()
    owned = [set(r["mine"]) for r in res]
    assert owned[0].isdisjoint(owned[1])
    assert owned[0] | owned[1] == set(range(len(cells)))
    assert abs(res[0]["load"] - res[1]["load"]) <= max(cells)
    total_ci = sum(c * _iterations(i) for i, c in enumerate(cells))
    for r in res:
        assert r["ci"] == float(total_ci)  # the gathered count equals the one-rank sum
        assert r["ms"] == 10.0 + 3.5 * (WORLD - 1)  # the slowest rank's time
