"""Multi-rank sharding of independent systems, on CPU: the LPT plan
(cm3d_b200.shard) and a world-size-2 gloo run in which each rank steps its
share of an ensemble with the CPU oracle and the ranks gather their results
-- the data path of a multi-GPU run without a GPU."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cm3d_b200 import configs, setup
from cm3d_b200.shard import imbalance, partition, system_cost


def test_partition_is_a_balanced_exact_cover():
    rng = np.random.default_rng(3)
    costs = np.exp(rng.uniform(0, 5, 1024))
    for nr in (1, 2, 3, 8):
        parts = partition(costs, nr)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(1024))
        assert imbalance(costs, parts) < 1.01
    assert partition([5.0, 1.0, 1.0, 1.0, 1.0, 1.0], 2) == [[0], [1, 2, 3, 4, 5]]


def test_cost_model_orders_systems():
    small = setup.build_system(configs.lj_box(64, 0.8, 1.0, 1))
    big = setup.build_system(configs.lj_box(2048, 0.8, 1.0, 1))
    charged = setup.build_system(configs.lj_box(2048, 0.8, 1.0, 1, charged=True))
    assert system_cost(small) < system_cost(big) < system_cost(charged)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import Oracle
        wls = configs.ensemble(8, seed=5, nmax=300)
        systems = [setup.build_system(w) for w in wls]
        parts = partition([system_cost(s) for s in systems], world)
        mine = {}
        for k in parts[rank]:
            o = Oracle(systems[k], nocell_all=1)
            o.step_init()
            o.step(1, 5)
            mine[k] = float(o.energies()["poter"])
        gathered = [None] * world
        dist.all_gather_object(gathered, (rank, parts[rank], mine))
        if rank == 0:
            out.put(gathered)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_rank_gloo_run_covers_every_system_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    seen = {}
    for rank, part, res in gathered:
        assert sorted(res) == sorted(part)
        for k, v in res.items():
            assert k not in seen
            seen[k] = v
    assert sorted(seen) == list(range(8))
    # each rank's result is the system's own: the same as a single-process run
    from oracle import Oracle
    wls = configs.ensemble(8, seed=5, nmax=300)
    for k in (0, 7):
        o = Oracle(setup.build_system(wls[k]), nocell_all=1)
        o.step_init()
        o.step(1, 5)
        assert seen[k] == float(o.energies()["poter"])
