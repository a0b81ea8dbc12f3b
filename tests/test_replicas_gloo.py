"""Host logic of the multi-GPU replica path on CPU: the cost-balanced split of an
ensemble across ranks, and the two collectives it uses (max-over-ranks timing,
the gather of per-replica results), run as two gloo ranks."""
import json
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "dav-qed2d_b200"))

from qed2d.replicas import gather_by_replica, partition_by_cost, rank_share, replica_cost, slowest  # noqa: E402


def ensemble_sizes():
    from qed2d.cases import ensemble_config
    return ensemble_config(512, 2024)[0]


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_partition_is_complete_disjoint_and_balanced(world):
    sizes = ensemble_sizes()
    costs = [replica_cost(a, b) for a, b in sizes]
    parts = partition_by_cost(costs, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(sizes)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) / (sum(loads) / world) < 1.02
    assert parts == partition_by_cost(costs, world)   # deterministic


def test_partition_edge_cases():
    assert partition_by_cost([], 3) == [[], [], []]
    assert partition_by_cost([5.0], 2) == [[0], []]
    with pytest.raises(ValueError):
        partition_by_cost([1.0], 0)


def _worker(rank, world, port, outdir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        sizes = ensemble_sizes()
        mine = rank_share(sizes, rank, world)
        results = [{"replica": i, "L": sizes[i][0], "rank": rank} for i in mine]
        everything = gather_by_replica(mine, results, len(sizes))
        t = slowest(1.0 + rank)
        with open(os.path.join(outdir, f"rank{rank}.json"), "w") as fh:
            json.dump({"mine": mine, "all": everything, "slowest": t}, fh)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    out = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    sizes = ensemble_sizes()
    assert sorted(out[0]["mine"] + out[1]["mine"]) == list(range(len(sizes)))
    for o in out:
        assert o["slowest"] == 2.0
        assert [e["replica"] for e in o["all"]] == list(range(len(sizes)))
        assert all(e["L"] == sizes[e["replica"]][0] for e in o["all"])
        assert all(e["replica"] in out[e["rank"]]["mine"] for e in o["all"])
