"""Sharding of the batched-serving cases across ranks: the LPT partition on its own, and the
multi-rank path as two gloo processes on the CPU (disjoint, covering shares; max over ranks;
gathered metrics)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from flowpro_v2_b200 import meshgen, sharding


def test_lpt_partition_is_disjoint_covering_and_balanced():
    cases = meshgen.serving_cases(256, seed=1)
    costs = [sharding.case_cost(2 * c["nx"] * c["ny"], c["order"]) for c in cases]
    for n in (1, 2, 4, 8):
        parts = sharding.lpt_partition(costs, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(cases)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: max load <= mean load + largest single cost
        assert max(loads) <= sum(costs) / n + max(costs) + 1e-9
    assert sharding.lpt_partition(costs, 4) == sharding.lpt_partition(costs, 4)


def test_serving_cases_follow_the_configuration():
    cases = meshgen.serving_cases(256, seed=1)
    n_el = np.array([2 * c["nx"] * c["ny"] for c in cases])
    assert 1500 < n_el.min() and n_el.max() < 70000
    assert {c["order"] for c in cases} == {2, 3, 4}
    assert all(0.3 <= c["mach"] <= 0.7 and 0.05 <= c["height"] <= 0.12 for c in cases)
    assert cases == meshgen.serving_cases(256, seed=1)


def _worker(rank, world, port, result_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    cases = meshgen.serving_cases(64, seed=3, min_elements=100, max_elements=1000)
    costs = [sharding.case_cost(2 * c["nx"] * c["ny"], c["order"]) for c in cases]
    mine = sharding.lpt_partition(costs, world)[rank]
    t_max = sharding.max_over_ranks(1.0 + rank)
    metrics = sharding.gather_metrics({"rank": rank, "cases": mine, "cost": sum(costs[i] for i in mine)})
    with open(os.path.join(result_dir, f"r{rank}.txt"), "w") as f:
        f.write(repr((t_max, metrics)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_share_the_cases(tmp_path):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    res = [eval(open(tmp_path / f"r{r}.txt").read()) for r in range(2)]
    for t_max, metrics in res:
        assert t_max == 2.0
        assert [m["rank"] for m in metrics] == [0, 1]
        shares = [set(m["cases"]) for m in metrics]
        assert shares[0].isdisjoint(shares[1]) and shares[0] | shares[1] == set(range(64))
    assert res[0][1] == res[1][1]
