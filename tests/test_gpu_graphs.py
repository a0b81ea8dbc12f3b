"""CUDA-graph replay of the MD integration (qed2d_ctx_set_graphs,
qed2d_batch_set_graphs).  A chain of trajectories run with graphs on -- the
first direct, the second captured, the rest replayed -- must end bitwise where
the same chain with graphs off ends: same links, same Delta H, same accept /
reject, same CG iteration counts.  Both chains run on the same context or batch,
so they use the same tuned solver schedules."""
import numpy as np
import pytest

from helpers import hot_links, to_dev, to_host

pytestmark = pytest.mark.gpu

NTRAJ = 4


@pytest.fixture(scope="module")
def q():
    import qed2d
    yield qed2d
    qed2d.set_precision("f64")


def _chain(q, prm, U0, run, graphs):
    q.set_graphs(prm, graphs)
    U = to_dev(U0)
    out = [run(U, 7000 + t) for t in range(NTRAJ)]
    return to_host(U), [(i.accepted, i.dH, i.hini, i.qtop, i.cg_iterations) for i in out]


def _check_same(q, prm, U0, run):
    Ua, ia = _chain(q, prm, U0, run, False)
    s0 = q.graph_stats(prm)
    Ub, ib = _chain(q, prm, U0, run, True)
    s1 = q.graph_stats(prm)
    assert s1["on"] and s1["failures"] == 0, s1
    assert s1["captures"] - s0["captures"] == 1, (s0, s1)
    assert s1["replays"] - s0["replays"] == NTRAJ - 1, (s0, s1)   # the first trajectory runs directly
    assert ia == ib
    assert np.array_equal(Ua, Ub)


@pytest.mark.parametrize("integ", ["omf4", "leapfrog"])
def test_graph_pure_gauge_bitwise(q, integ):
    L1, L2 = 128, 96
    prm = q.LattParm((L1, L2), 11.25)
    integrator = q.OMF4() if integ == "omf4" else q.Leapfrog()
    q.seed(77)
    _check_same(q, prm, hot_links(L1, L2, 5),
                lambda U, ctr: q.HMC_(U, 0.05, 10, [], prm, None, integrator=integrator, counter=ctr))


@pytest.mark.parametrize("prec,integ", [("mixed", "leapfrog"), ("f64", "leapfrog"), ("mixed", "omf4")])
def test_graph_nf2_bitwise(q, prec, integ):
    L1, L2 = 64, 48
    prm = q.LattParm((L1, L2), 4.0)
    q.set_precision(prec)
    integrator = q.OMF4() if integ == "omf4" else q.Leapfrog()
    q.seed(78)
    ns = 3 if integ == "omf4" else 8
    _check_same(q, prm, hot_links(L1, L2, 6),
                lambda U, ctr: q.HMC_(U, 0.2, 0.1, ns, [], 10000, 1e-24, prm, None, integrator=integrator,
                                      counter=ctr))
    q.set_precision("f64")


@pytest.mark.parametrize("prec", ["mixed", "f64"])
def test_graph_rhmc_bitwise(q, prec):
    L1, L2 = 32, 32
    prm = q.LattParm((L1, L2), 4.0)
    q.set_precision(prec)
    rp = [q.get_rhmc_params(6, 0.05, 3.0), q.get_rhmc_params(6, 0.06, 3.0)]
    q.seed(79)
    _check_same(q, prm, hot_links(L1, L2, 7),
                lambda U, ctr: q.HMC_(U, [0.2, 0.3], 0.1, 5, [], 10000, 1e-24, prm, None, rp, counter=ctr))
    q.set_precision("f64")


def test_graph_plain_precision_runs_directly(q):
    """The reference-structured solver reads scalars back every iteration: its
    trajectories are never captured."""
    L1, L2 = 32, 32
    prm = q.LattParm((L1, L2), 4.0)
    q.set_precision("plain")
    q.set_graphs(prm, True)
    s0 = q.graph_stats(prm)
    U = to_dev(hot_links(L1, L2, 8))
    for t in range(3):
        q.HMC_(U, 0.2, 0.1, 4, [], 10000, 1e-24, prm, None, counter=8000 + t)
    s1 = q.graph_stats(prm)
    assert s1["captures"] == s0["captures"] and s1["replays"] == s0["replays"]
    q.set_precision("f64")


@pytest.mark.parametrize("sizes", [None, [(32, 32), (48, 40), (64, 64), (40, 24)]])
def test_graph_batch_bitwise(q, sizes):
    if sizes is None:
        nrep, L1, L2 = 4, 64, 48
        b = q.Batch(nrep, L1, L2, [3.0, 4.0, 5.0, 4.5])
        U0 = [hot_links(L1, L2, 900 + r) for r in range(nrep)]
    else:
        nrep = len(sizes)
        b = q.Batch.ragged(sizes, [3.0, 4.0, 5.0, 4.5])
        U0 = [hot_links(l1, l2, 900 + r) for r, (l1, l2) in enumerate(sizes)]
    am0s = [0.2, 0.25, 0.3, 0.35]
    seeds = [11, 12, 13, 14]

    def chain(graphs):
        b.graphs = graphs
        U = b.field()
        for r in range(nrep):
            b.replica(U, r).copy_(to_dev(U0[r]))
        res = []
        for t in range(NTRAJ):
            infos = b.hmc_nf2(U, am0s, 0.1, 6, 10000, 1e-24, seeds, 9000 + t)
            res.append([(i.accepted, i.dH, i.hini, i.qtop, i.cg_iterations) for i in infos])
        return U.cpu().numpy(), res

    Ua, ra = chain(False)
    s0 = b.graphs
    Ub, rb = chain(True)
    s1 = b.graphs
    assert s1["on"] and s1["failures"] == 0, s1
    assert s1["captures"] - s0["captures"] == 1 and s1["replays"] - s0["replays"] == NTRAJ - 1, (s0, s1)
    assert ra == rb
    assert np.array_equal(Ua, Ub)


def test_graph_dropped_when_arguments_change(q):
    """A new step size is a new graph: the trajectory after the change runs
    directly, the next one captures again."""
    L1, L2 = 64, 64
    prm = q.LattParm((L1, L2), 11.25)
    q.set_graphs(prm, True)
    U = to_dev(hot_links(L1, L2, 9))
    s0 = q.graph_stats(prm)
    for eps in (0.05, 0.05, 0.05, 0.04, 0.04):
        q.HMC_(U, eps, 5, [], prm, None, counter=int(eps * 1000))
    s1 = q.graph_stats(prm)
    assert s1["captures"] - s0["captures"] == 2
    assert s1["replays"] - s0["replays"] == 3
