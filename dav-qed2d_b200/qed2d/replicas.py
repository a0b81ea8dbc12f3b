"""Replica chains over several GPUs: one process per GPU, independent Markov
chains, no exchange on the data path.

The replicas of an ensemble are split across ranks by cost (sites x expected
CG work; the larger lattices need both more sites and more iterations), each
rank advances its share as one batch, and the per-replica results are gathered
at the end.  Timings are taken on each rank's device and reduced to the
slowest rank, so an aggregate rate is (all replicas' trajectories) / (slowest
rank's time).  The functions take a torch.distributed process group, so the
same code runs over NCCL on GPUs and over gloo on CPU (the tests).
"""
import heapq


def replica_cost(L1, L2):
    """Relative cost of one trajectory of an L1 x L2 replica: sites times the
    CG iteration growth with the lattice extent (iterations of a hot start grow
    slowly with L at fixed mass; a linear proxy in log L suffices for balance)."""
    import math
    V = L1 * L2
    return V * (1.0 + 0.25 * math.log2(max(L1, L2)))


def partition_by_cost(costs, world):
    """Longest-processing-time split of replicas across `world` ranks.  Returns
    one sorted index list per rank; deterministic (ties broken by index)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def rank_share(sizes, rank, world):
    """Indices of the replicas (sizes = [(L1, L2), ...]) that `rank` advances."""
    return partition_by_cost([replica_cost(a, b) for a, b in sizes], world)[rank]


def slowest(seconds, group=None, device=None):
    """Max over ranks of a per-rank device time (seconds); the value itself
    when torch.distributed is not initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(seconds)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_by_replica(local_indices, local_results, n, group=None):
    """All ranks' per-replica results, ordered by replica index (list of n)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        out = [None] * n
        for i, r in zip(local_indices, local_results):
            out[i] = r
        return out
    everything = [None] * dist.get_world_size(group)
    dist.all_gather_object(everything, (list(local_indices), list(local_results)), group=group)
    out = [None] * n
    for idx, res in everything:
        for i, r in zip(idx, res):
            out[i] = r
    return out
