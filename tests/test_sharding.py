"""Independent LPs across ranks (noaidi_b200/prima/sharding.py), on CPU.

The device solve is stood in for by the oracle here (no GPU): what is under
test is the partition and the gather, run as two gloo ranks on 127.0.0.1."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from noaidi_b200.prima import PdhgParams
from noaidi_b200.prima import generators as G
from noaidi_b200.prima.sharding import instance_size, shard, solve_sharded
from tests import lp_fixtures as F

P = PdhgParams(eps_abs=1e-6, eps_rel=1e-6, max_iterations=50_000)


def test_shard_covers_every_instance_once():
    rng = np.random.default_rng(0)
    sizes = rng.integers(1, 10_000, size=257).tolist()
    for world in (1, 2, 3, 8):
        parts = shard(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        # longest-processing-time: no rank exceeds the mean by more than the largest item
        assert max(loads) <= sum(sizes) / world + max(sizes)


def test_shard_is_deterministic_and_breaks_ties_low():
    assert shard([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]
    assert shard([1, 2, 3], 1) == [[0, 1, 2]]
    assert shard([], 4) == [[], [], [], []]
    with pytest.raises(ValueError):
        shard([1], 0)


def problems():
    out = [i.problem for i in F.optimal()]
    out += [G.dc_lopf(seed=k, buses=30 + 10 * k, lines=45 + 15 * k, generators=15 + 5 * k, snapshots=2)
            for k in range(3)]
    return out


def oracle_solve(ps):
    from oracle import oracle as O
    return [(s.status.value, s.objective_value, s.iterations) for s in (O.solve(p, P) for p in ps)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res, mine = solve_sharded(problems(), oracle_solve, rank=rank, world=world)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array(res, dtype=object), allow_pickle=True)
        np.save(os.path.join(out_dir, f"m{rank}.npy"), np.array(mine))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_the_single_process_results(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    single, _ = solve_sharded(problems(), oracle_solve)
    mines = [set(np.load(tmp_path / f"m{r}.npy").tolist()) for r in range(world)]
    assert mines[0].isdisjoint(mines[1]) and len(mines[0] | mines[1]) == len(problems())
    for r in range(world):
        got = np.load(tmp_path / f"r{r}.npy", allow_pickle=True).tolist()
        assert [tuple(g) for g in got] == [tuple(s) for s in single]


def test_sizes_follow_the_problem():
    p = F.economic_dispatch().problem
    assert instance_size(p) == p.constraint_matrix.nnz + p.num_variables + p.num_constraints
