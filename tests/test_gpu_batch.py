"""Batched replicas: each replica of a batch trajectory reproduces the
single-lattice Nf=2 HMC step (mixed solver) with the same seed and counter, and
the oracle replaying the same draws.  Tolerances (each about 10x the error
measured on a B200, recorded through helpers.bound): links 1e-12 (batch vs
single lattice) and 5e-12 (vs the oracle) relative, Delta H 1e-10 / 5e-10
absolute, identical accept/reject."""
import numpy as np
import pytest

from helpers import bound, cgauss, hot_links, rel, to_dev, to_host
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L1,L2", [(32, 24), (40, 36)])
def test_batch_matches_single_and_oracle(L1, L2):
    import torch

    import qed2d
    nrep = 3
    betas = [4.0, 3.0, 5.0]
    am0s = [0.3, 0.25, 0.4]
    seeds = [11, 12, 13]
    counter = 7
    U0 = [hot_links(L1, L2, 100 + r) for r in range(nrep)]
    b = qed2d.Batch(nrep, L1, L2, betas)
    Ub = b.field()
    for r in range(nrep):
        Ub[r] = to_dev(U0[r])
    infos = b.hmc_nf2(Ub, am0s, 0.1, 5, 10000, 1e-24, seeds, counter)
    qed2d.set_precision("mixed")
    for r in range(nrep):
        prm = qed2d.LattParm((L1, L2), betas[r])
        Ud = to_dev(U0[r])
        qed2d.seed(seeds[r])
        single = qed2d.HMC_(Ud, am0s[r], 0.1, 5, [], 10000, 1e-24, prm, None, counter=counter)
        bound("batch vs single-lattice dH abs", abs(single.dH - infos[r].dH), 1e-10)
        assert single.accepted == infos[r].accepted
        bound("batch vs single-lattice links", rel(to_host(Ub[r]), to_host(Ud)), 1e-12)
    qed2d.set_precision("f64")
    # replica 1 against the oracle replaying its draws
    r = 1
    o = Oracle(L1, L2, betas[r])
    mom0 = Oracle.normal(2 * L1 * L2, seeds[r], 1, counter).reshape(2, L2, L1)
    noise = cgauss(L1, L2, seeds[r], 16, counter)
    st, Uo, acc, hi, hf, _ = o.hmc_nf2(U0[r], am0s[r], 0.1, 5, 10000, 1e-24, mom0, noise,
                                        Oracle.uniform(seeds[r], 3, counter))
    assert st == 0 and acc == infos[r].accepted
    bound("batch vs oracle dH abs", abs(infos[r].dH - (hf - hi)), 5e-10)
    bound("batch vs oracle links", rel(to_host(Ub[r]), Uo), 5e-12)


def test_batch_rejects_bad_shape():
    import qed2d
    b = qed2d.Batch(2, 16, 16, 4.0)
    import torch
    with pytest.raises(ValueError):
        b.hmc_nf2(torch.zeros((3, 2, 16, 16), dtype=torch.complex128, device="cuda"), 0.3, 0.1, 2, 100, 1e-20,
                  [1, 2], 0)


def test_batch_cg_matches_single_cg():
    """qed2d_batch_cg: replica r's solution equals the single-lattice mixed solve (1e-9)."""
    import torch

    import qed2d
    nrep, L1, L2 = 4, 48, 40
    am0s = [0.2, 0.3, 0.4, 0.5]
    b = qed2d.Batch(nrep, L1, L2, 4.0)
    U, src, x = b.field(), b.field(), b.field()
    for r in range(nrep):
        U[r] = to_dev(hot_links(L1, L2, 200 + r))
        src[r] = to_dev(cgauss(L1, L2, 300 + r, 2))
    its, upd = b.cg(x, U, src, am0s, 20000, 1e-24)
    qed2d.set_precision("mixed")
    prm = qed2d.LattParm((L1, L2), 4.0)
    for r in range(nrep):
        xs = qed2d.cfield(L1, L2)
        it = qed2d.CG(xs, U[r].contiguous(), src[r].contiguous(), am0s[r], 20000, 1e-24,
                      qed2d.gamm5Dw_sqr_msq, prm, None)
        bound("batched CG vs single-lattice CG", rel(to_host(x[r]), to_host(xs)), 1e-12)
        assert abs(its[r] - it) <= max(3, it // 20) and upd[r] >= 1
    qed2d.set_precision("f64")


RAGGED = [(32, 24), (16, 16), (40, 36), (64, 8), (24, 40), (33, 17)]


def test_ragged_batch_matches_single_and_oracle():
    """Replicas of uneven sizes (partial 32x8 tiles included) in one batch: each
    reproduces the single-lattice trajectory with its own beta, mass and seed."""
    import qed2d
    n = len(RAGGED)
    betas = [4.0, 3.0, 5.0, 2.5, 4.5, 3.5]
    am0s = [0.3, 0.25, 0.4, 0.2, 0.35, 0.3]
    seeds = [21, 22, 23, 24, 25, 26]
    counter = 3
    b = qed2d.Batch.ragged(RAGGED, betas)
    assert b.offsets[-1] == sum(l1 * l2 for l1, l2 in RAGGED)
    Ub = b.field()
    U0 = [hot_links(l1, l2, 500 + r) for r, (l1, l2) in enumerate(RAGGED)]
    for r in range(n):
        b.replica(Ub, r).copy_(to_dev(U0[r]))
    infos = b.hmc_nf2(Ub, am0s, 0.1, 5, 10000, 1e-24, seeds, counter)
    qed2d.set_precision("mixed")
    for r, (l1, l2) in enumerate(RAGGED):
        prm = qed2d.LattParm((l1, l2), betas[r])
        Ud = to_dev(U0[r])
        qed2d.seed(seeds[r])
        single = qed2d.HMC_(Ud, am0s[r], 0.1, 5, [], 10000, 1e-24, prm, None, counter=counter)
        bound("ragged batch vs single-lattice dH abs", abs(single.dH - infos[r].dH), 1e-10)  # r
        assert single.accepted == infos[r].accepted, r
        bound("ragged batch vs single-lattice links", rel(to_host(b.replica(Ub, r)), to_host(Ud)), 1e-12)  # r
    qed2d.set_precision("f64")
    r = 5   # the odd-sized replica against the oracle replaying its draws
    l1, l2 = RAGGED[r]
    o = Oracle(l1, l2, betas[r])
    mom0 = Oracle.normal(2 * l1 * l2, seeds[r], 1, counter).reshape(2, l2, l1)
    noise = cgauss(l1, l2, seeds[r], 16, counter)
    st, Uo, acc, hi, hf, _ = o.hmc_nf2(U0[r], am0s[r], 0.1, 5, 10000, 1e-24, mom0, noise,
                                        Oracle.uniform(seeds[r], 3, counter))
    assert st == 0 and acc == infos[r].accepted
    bound("ragged batch vs oracle dH abs", abs(infos[r].dH - (hf - hi)), 1e-10)
    bound("ragged batch vs oracle links", rel(to_host(b.replica(Ub, r)), Uo), 5e-12)


def test_ragged_batch_cg_matches_single_and_is_deterministic():
    import qed2d
    n = len(RAGGED)
    am0s = [0.2, 0.3, 0.4, 0.5, 0.25, 0.35]
    b = qed2d.Batch.ragged(RAGGED, [4.0] * n)
    U, src, x, x2 = b.field(), b.field(), b.field(), b.field()
    for r, (l1, l2) in enumerate(RAGGED):
        b.replica(U, r).copy_(to_dev(hot_links(l1, l2, 700 + r)))
        b.replica(src, r).copy_(to_dev(cgauss(l1, l2, 800 + r, 2)))
    its, upd = b.cg(x, U, src, am0s, 20000, 1e-24)
    its2, _ = b.cg(x2, U, src, am0s, 20000, 1e-24)
    assert its == its2 and bool((x == x2).all())   # fixed-order reductions: bit-identical
    qed2d.set_precision("mixed")
    for r, (l1, l2) in enumerate(RAGGED):
        prm = qed2d.LattParm((l1, l2), 4.0)
        xs = qed2d.cfield(l1, l2)
        it = qed2d.CG(xs, b.replica(U, r).contiguous(), b.replica(src, r).contiguous(), am0s[r], 20000, 1e-24,
                      qed2d.gamm5Dw_sqr_msq, prm, None)
        bound("ragged batched CG vs single-lattice CG", rel(to_host(b.replica(x, r)), to_host(xs)), 1e-12)  # r
        assert abs(its[r] - it) <= max(3, it // 20) and upd[r] >= 1, r
    qed2d.set_precision("f64")


def test_ragged_rejects_bad_sizes():
    import qed2d
    with pytest.raises(qed2d.Qed2dError):
        qed2d.Batch.ragged([(16, 16), (1, 16)], [4.0, 4.0])
    with pytest.raises(ValueError):
        qed2d.Batch.ragged([(16, 16), (16, 8)], [4.0])


def test_many_replicas_global_state_cg():
    """More than 64 replicas keep the solver records in global memory: solutions
    still equal the single-lattice solves and repeat bit for bit."""
    import qed2d
    rng = np.random.default_rng(77)
    n = 80
    sizes = [(int(a), int(b)) for a, b in zip(rng.choice([8, 16, 24, 40], n), rng.choice([4, 8, 12, 16], n))]
    am0s = rng.uniform(0.1, 0.5, n).tolist()
    b = qed2d.Batch.ragged(sizes, [4.0] * n)
    U, src, x, x2 = b.field(), b.field(), b.field(), b.field()
    for r, (l1, l2) in enumerate(sizes):
        b.replica(U, r).copy_(to_dev(hot_links(l1, l2, 900 + r)))
        b.replica(src, r).copy_(to_dev(cgauss(l1, l2, 1000 + r, 2)))
    its, _ = b.cg(x, U, src, am0s, 20000, 1e-24)
    its2, _ = b.cg(x2, U, src, am0s, 20000, 1e-24)
    assert its == its2 and bool((x == x2).all())
    qed2d.set_precision("mixed")
    for r in (0, 1, 41, n - 1):
        l1, l2 = sizes[r]
        prm = qed2d.LattParm((l1, l2), 4.0)
        xs = qed2d.cfield(l1, l2)
        qed2d.CG(xs, b.replica(U, r).contiguous(), b.replica(src, r).contiguous(), am0s[r], 20000, 1e-24,
                 qed2d.gamm5Dw_sqr_msq, prm, None)
        bound("80-replica batched CG vs single-lattice CG", rel(to_host(b.replica(x, r)), to_host(xs)), 1e-12)  # r
    qed2d.set_precision("f64")


def test_batch_reduction_schedules_give_identical_bits():
    """Equal-size batches: the three schedules of the batched solver (two grid
    reduction schedules; independent replicas with a barrier each, whose blocks
    leave as their replica converges) give bitwise identical solutions and
    per-replica iteration counts; the first solve tunes the schedule."""
    import qed2d
    nrep, L1, L2 = 3, 64, 48
    b = qed2d.Batch(nrep, L1, L2, 4.0)
    assert b.schedule == -1
    U, src = b.field(), b.field()
    for r in range(nrep):
        U[r] = to_dev(hot_links(L1, L2, 40 + r))
        src[r] = to_dev(cgauss(L1, L2, 50 + r, 2))
    x = b.field()
    b.cg(x, U, src, [0.2, 0.3, 0.25], 20000, 1e-24)
    assert b.schedule in (0, 1, 4, 5, 8, 9)
    res = []
    for sched in (0, 1, 4, 5):
        b.schedule = sched
        x = b.field()
        its, _ = b.cg(x, U, src, [0.2, 0.3, 0.25], 20000, 1e-24)
        res.append((list(its), to_host(x)))
    assert len(set(res[0][0])) == 3   # the replicas converge at different iterations
    for i in (1, 2, 3):
        assert res[0][0] == res[i][0] and np.array_equal(res[0][1], res[i][1])
    assert qed2d.Batch.ragged([(16, 16), (32, 8)], [4.0, 4.0]).schedule == -1


@pytest.mark.parametrize("L1,L2", [(64, 48), (96, 40), (100, 37)])
def test_batch_tile_heights(L1, L2):
    """The equal-size solver's tile heights (tiles of 32 x 4, 8, 16 sites; 100 x 37
    has a partial column tile and a partial last tile row): within a height the
    four schedules give identical bits; across heights the block partials are
    grouped differently, so the bits differ: solutions agree to 1e-13 relative
    (measured on a B200: 2.6e-16) and iteration counts within 5%.  The first
    solve tunes height and schedule together."""
    import qed2d
    nrep = 3
    b = qed2d.Batch(nrep, L1, L2, 4.0)
    assert b.tile_rows == -1
    U, src = b.field(), b.field()
    for r in range(nrep):
        U[r] = to_dev(hot_links(L1, L2, 140 + r))
        src[r] = to_dev(cgauss(L1, L2, 150 + r, 2))
    am0 = [0.2, 0.3, 0.25]
    b.cg(b.field(), U, src, am0, 20000, 1e-24)
    assert b.tile_rows in (4, 8, 16) and b.schedule in (0, 1, 4, 5, 8, 9)
    res = {}
    for rows in (8, 4, 16):
        b.tile_rows = rows
        per = []
        for sched in (0, 1, 4, 5):
            b.schedule = sched
            x = b.field()
            its, _ = b.cg(x, U, src, am0, 20000, 1e-24)
            per.append((list(its), to_host(x)))
        for i in (1, 2, 3):
            assert per[0][0] == per[i][0] and np.array_equal(per[0][1], per[i][1]), (rows, i)
        res[rows] = per[0]
    for rows in (4, 16):
        bound("tile height vs 32x8 solution rel", rel(res[rows][1], res[8][1]), 1e-13)
        for r in range(nrep):
            assert abs(res[rows][0][r] - res[8][0][r]) <= max(3, res[8][0][r] // 20), (rows, r)
    b.tile_rows = -1
    assert b.tile_rows == -1
    with pytest.raises(qed2d.Qed2dError):
        b.tile_rows = 12


@pytest.mark.parametrize("nrep", [6, 80])
def test_ragged_cluster_solver_matches_grid_solver(nrep):
    """Uneven batches have two solvers: one launch over all replicas with grid
    barriers (schedule 2) and one thread-block cluster per replica (schedule 3;
    schedule 6 is 3 with the first phase's stencil on r).  They group their sums
    differently: solutions agree to the solver's accuracy and with the
    single-lattice solve; the first solve tunes the choice."""
    import qed2d
    rng = np.random.default_rng(123 + nrep)
    sizes = [(int(a), int(b)) for a, b in zip(rng.choice([8, 16, 33, 64, 96], nrep), rng.choice([4, 8, 17, 40], nrep))]
    am0s = rng.uniform(0.1, 0.5, nrep).tolist()
    b = qed2d.Batch.ragged(sizes, [4.0] * nrep)
    U, src = b.field(), b.field()
    for r, (l1, l2) in enumerate(sizes):
        b.replica(U, r).copy_(to_dev(hot_links(l1, l2, 60 + r)))
        b.replica(src, r).copy_(to_dev(cgauss(l1, l2, 90 + r, 2)))
    x = b.field()
    b.cg(x, U, src, am0s, 20000, 1e-24)
    assert b.schedule in (2, 3, 6)
    res = {}
    for sched in (2, 3, 6):
        b.schedule = sched
        x = b.field()
        its, upd = b.cg(x, U, src, am0s, 20000, 1e-24)
        res[sched] = (its, to_host(x))
        x2 = b.field()
        b.cg(x2, U, src, am0s, 20000, 1e-24)
        assert np.array_equal(to_host(x2), res[sched][1])   # each solver is deterministic
    bound("cluster-per-replica vs grid solver", rel(res[3][1], res[2][1]), 2e-12)
    bound("cluster-per-replica, stencil on r, vs grid solver", rel(res[6][1], res[2][1]), 2e-12)
    for r in range(nrep):
        bound("cluster-per-replica vs grid iterations", abs(res[3][0][r] - res[2][0][r]), 2)  # r
        bound("cluster-per-replica, stencil on r, vs grid iterations", abs(res[6][0][r] - res[2][0][r]), 2)  # r
    qed2d.set_precision("mixed")
    for r in (0, nrep - 1):
        l1, l2 = sizes[r]
        prm = qed2d.LattParm((l1, l2), 4.0)
        xs = qed2d.cfield(l1, l2)
        qed2d.CG(xs, b.replica(U, r).contiguous(), b.replica(src, r).contiguous(), am0s[r], 20000, 1e-24,
                 qed2d.gamm5Dw_sqr_msq, prm, None)
        bound("cluster-per-replica vs single-lattice CG", rel(to_host(b.replica(x2, r)), to_host(xs)), 1e-12)  # r
    qed2d.set_precision("f64")


@pytest.mark.parametrize("nrep,L1,L2", [(3, 64, 48), (2, 128, 64), (4, 64, 32)])
def test_tma_schedule_same_bits_as_lean(nrep, L1, L2):
    """Batch schedule 7 (the stencil operands of every tile staged into shared
    memory by TMA one tile ahead) runs the arithmetic of schedule 5 in the same
    order: identical iterations and solutions, bit for bit, at both tile
    heights it supports; then two batched Nf=2 trajectories from the same start
    give identical dH and links."""
    import qed2d
    b = qed2d.Batch(nrep, L1, L2, 4.0)
    U, src = b.field(), b.field()
    for r in range(nrep):
        U[r] = to_dev(hot_links(L1, L2, 160 + r))
        src[r] = to_dev(cgauss(L1, L2, 170 + r, 2))
    am0 = [0.15 + 0.05 * r for r in range(nrep)]
    for rows in (8, 16):
        b.tile_rows = rows
        out = []
        for sched in (5, 7):
            b.schedule = sched
            x = b.field()
            its, _ = b.cg(x, U, src, am0, 20000, 1e-24)
            out.append((list(its), to_host(x)))
        assert out[0][0] == out[1][0], rows
        assert np.array_equal(out[0][1], out[1][1]), rows
    traj = []
    for sched in (5, 7):
        bt = qed2d.Batch(nrep, L1, L2, 4.0)
        bt.tile_rows, bt.schedule = 16, sched
        Ut = bt.field()
        for r in range(nrep):
            Ut[r] = to_dev(hot_links(L1, L2, 180 + r))
        infos = [bt.hmc_nf2(Ut, am0, 0.1, 4, 20000, 1e-24, [950 + r for r in range(nrep)], c) for c in (0, 1)]
        traj.append(([(i.dH, i.cg_iterations) for inf in infos for i in inf], to_host(Ut)))
    assert traj[0][0] == traj[1][0]
    assert np.array_equal(traj[0][1], traj[1][1])


@pytest.mark.parametrize("L1,L2,rows", [(100, 37, 8), (96, 40, 16), (64, 48, 4)])
def test_tma_schedule_refuses_partial_tiles(L1, L2, rows):
    """Schedule 7 needs whole tiles (L1 a multiple of 32, L2 of the tile height
    8 or 16): otherwise the solve returns QED2D_ERR_UNSUPPORTED without
    launching, and the batch still solves under its other schedules."""
    import qed2d
    b = qed2d.Batch(2, L1, L2, 4.0)
    U, src = b.field(), b.field()
    for r in range(2):
        U[r] = to_dev(hot_links(L1, L2, 190 + r))
        src[r] = to_dev(cgauss(L1, L2, 195 + r, 2))
    b.tile_rows, b.schedule = rows, 7
    with pytest.raises(qed2d.Qed2dError) as e:
        b.cg(b.field(), U, src, 0.2, 20000, 1e-24)
    assert e.value.status == qed2d._lib.UNSUPPORTED
    b.schedule = 5
    its, _ = b.cg(b.field(), U, src, 0.2, 20000, 1e-24)
    assert min(its) > 0


def test_independent_replica_schedule_trajectories():
    """Batched Nf=2 trajectories under the grid schedule (1) and the independent-
    replica schedule (4) from the same start: identical dH, iterations and links."""
    import qed2d
    nrep, L = 4, 64
    out = []
    for sched in (1, 4, 5):
        b = qed2d.Batch(nrep, L, L, 4.0)
        b.tile_rows = 8   # heights group the sums differently: fix it for a bitwise comparison
        b.schedule = sched
        U = b.field()
        for r in range(nrep):
            U[r] = to_dev(hot_links(L, L, 70 + r))
        seeds = [900 + r for r in range(nrep)]
        am0 = [0.1 + 0.05 * r for r in range(nrep)]   # replicas converge at different iterations
        infos = [b.hmc_nf2(U, am0, 0.1, 5, 20000, 1e-24, seeds, c) for c in (0, 1)]
        out.append(([(i.dH, i.cg_iterations) for inf in infos for i in inf], to_host(U)))
    for i in (1, 2):
        assert out[0][0] == out[i][0]
        assert np.array_equal(out[0][1], out[i][1])


@pytest.mark.parametrize("maxiter", [7, 8])
def test_capped_solves_agree_across_solvers(maxiter):
    """A solve capped at `maxiter` iterations returns the FP64 iterate x_k of
    every mixed solver: the single-lattice solver with one x update per iteration
    (one-cluster schedule) and with the update deferred to every second iteration
    for two directions (grid schedule), the equal-size batched solver under its
    schedules, and both uneven-batch solvers.  The cap forces a final reliable
    update, which has to fold a deferred update in (odd and even caps); a lost one
    would move x by alpha_k p_k, orders of magnitude above the FP32 spread
    between the solvers."""
    import qed2d
    L, am0 = 64, 0.15
    prm = qed2d.LattParm((L, L), 4.0)
    U, b = to_dev(hot_links(L, L, 81)), to_dev(cgauss(L, L, 82, 2))

    def capped(fn):
        try:
            fn()
        except qed2d.Qed2dError:
            pass   # not converged at the cap, as intended

    ref = {}
    qed2d.set_precision("mixed")
    try:
        for sched in (2, 1):
            qed2d.set_schedule(prm, sched, "mixed")
            x = qed2d.cfield(L, L)
            capped(lambda: qed2d.CG(x, U, b, am0, maxiter, 1e-24, qed2d.gamm5Dw_sqr_msq, prm, None))
            ref[sched] = to_host(x)
    finally:
        qed2d.set_schedule(prm, -1, "mixed")
        qed2d.set_precision("f64")
    assert np.abs(ref[2]).max() > 0
    bound("capped solve, x paired vs one update per iteration", rel(ref[1], ref[2]), 1e-6)
    bt = qed2d.Batch(2, L, L, 4.0)
    Ub, bb = bt.field(), bt.field()
    for r in range(2):
        Ub[r], bb[r] = U, b
    for sched in (1, 4, 5, 8):
        bt.schedule = sched
        x = bt.field()
        capped(lambda: bt.cg(x, Ub, bb, [am0, am0], maxiter, 1e-24))
        for r in range(2):
            bound("capped batched solve vs single-lattice", rel(to_host(x[r]), ref[2]), 1e-6)  # (sched, r)
    rb = qed2d.Batch.ragged([(L, L), (32, 32)], [4.0, 4.0])
    Ur, br = rb.field(), rb.field()
    rb.replica(Ur, 0).copy_(U)
    rb.replica(br, 0).copy_(b)
    rb.replica(Ur, 1).copy_(to_dev(hot_links(32, 32, 83)))
    rb.replica(br, 1).copy_(to_dev(cgauss(32, 32, 84, 2)))
    for sched in (2, 3, 6):
        rb.schedule = sched
        x = rb.field()
        capped(lambda: rb.cg(x, Ur, br, [am0, am0], maxiter, 1e-24))
        bound("capped ragged solve vs single-lattice", rel(to_host(rb.replica(x, 0)), ref[2]), 1e-6)  # sched


@pytest.mark.parametrize("L1,L2,rows", [(64, 48, 8), (100, 37, 16), (96, 40, 4)])
def test_rstencil_schedule_matches_lean(L1, L2, rows):
    """Batch schedule 8 (phase A applies the stencil to r and carries t = g5Dw r +
    beta t_old) runs the same CG recurrences as schedule 5 with t rounded along
    its own recurrence: both stop on the same FP64 true residual, so solutions
    agree to the solver's accuracy and iteration counts within 5%."""
    import qed2d
    nrep = 3
    b = qed2d.Batch(nrep, L1, L2, 4.0)
    U, src = b.field(), b.field()
    for r in range(nrep):
        U[r] = to_dev(hot_links(L1, L2, 240 + r))
        src[r] = to_dev(cgauss(L1, L2, 250 + r, 2))
    am0 = [0.2, 0.3, 0.25]
    b.tile_rows = rows
    res = {}
    for sched in (5, 8):
        b.schedule = sched
        x = b.field()
        its, upd = b.cg(x, U, src, am0, 20000, 1e-24)
        res[sched] = (list(its), to_host(x))
    bound("schedule 8 vs schedule 5 solution rel", rel(res[8][1], res[5][1]), 1e-11)
    for r in range(nrep):
        assert abs(res[8][0][r] - res[5][0][r]) <= max(3, res[5][0][r] // 20), (r, res[8][0], res[5][0])
    # the solution satisfies the reference's stop rule on the FP64 operator
    prm = qed2d.LattParm((L1, L2), 4.0)
    for r in range(nrep):
        ax, tmp = qed2d.cfield(L1, L2), qed2d.cfield(L1, L2)
        xr = to_dev(res[8][1][r])
        qed2d.gamm5Dw_sqr_msq(ax, tmp, U[r].contiguous(), xr, am0[r], prm, None)
        bh = to_host(src[r])
        rr = np.linalg.norm(to_host(ax) - bh) / np.linalg.norm(bh)
        bound("schedule 8 true relative residual |b - A x| / |b|", rr, 1.01e-12)


@pytest.mark.parametrize("sched", [8, 9])
def test_rstencil_schedule_trajectories_vs_oracle(sched):
    """Batched Nf=2 trajectories under schedule 8 (the first stencil on r) and 9
    (the same with the links staged in shared memory) against the oracle
    replaying the same draws (as under the other schedules: links 5e-12
    relative, Delta H 5e-10 absolute, same accept/reject)."""
    import qed2d
    nrep, L1, L2 = 2, 48, 40
    betas, am0s, seeds = [4.0, 4.0], [0.2, 0.3], [31, 32]
    b = qed2d.Batch(nrep, L1, L2, betas)
    b.schedule = sched
    U0 = [hot_links(L1, L2, 330 + r) for r in range(nrep)]
    U = b.field()
    for r in range(nrep):
        U[r] = to_dev(U0[r])
    counter = 5
    infos = b.hmc_nf2(U, am0s, 0.1, 5, 10000, 1e-24, seeds, counter)
    assert b.schedule == sched
    for r in range(nrep):
        o = Oracle(L1, L2, betas[r])
        mom0 = Oracle.normal(2 * L1 * L2, seeds[r], 1, counter).reshape(2, L2, L1)
        noise = cgauss(L1, L2, seeds[r], 16, counter)
        st, Uo, acc, hi, hf, _ = o.hmc_nf2(U0[r], am0s[r], 0.1, 5, 10000, 1e-24, mom0, noise,
                                            Oracle.uniform(seeds[r], 3, counter))
        assert st == 0 and acc == infos[r].accepted
        bound("schedule 8/9 batch vs oracle dH abs", abs(infos[r].dH - (hf - hi)), 5e-10)  # sched
        bound("schedule 8/9 batch vs oracle links", rel(to_host(U[r]), Uo), 5e-12)  # sched


@pytest.mark.parametrize("nrep,L1,L2,rows", [(3, 64, 48, 8), (3, 100, 37, 16), (2, 96, 40, 4), (4, 128, 128, 16)])
def test_staged_links_schedule_matches(nrep, L1, L2, rows):
    """Batch schedule 9 (schedule 8 with the FP32 links of every block's tiles
    staged once per solve in shared memory) reads the same link values from
    another memory; the compiler contracts the stencil's products into FMAs
    differently around shared-memory loads, so results agree with schedule 8 to
    rounding (measured on a B200: same iteration counts and reliable updates),
    for solves and for trajectories."""
    import qed2d
    b = qed2d.Batch(nrep, L1, L2, 4.0)
    U, src = b.field(), b.field()
    for r in range(nrep):
        U[r] = to_dev(hot_links(L1, L2, 440 + r))
        src[r] = to_dev(cgauss(L1, L2, 450 + r, 2))
    am0 = [0.2 + 0.05 * r for r in range(nrep)]
    b.tile_rows = rows
    res = {}
    for sched in (8, 9):
        b.schedule = sched
        x = b.field()
        its, upd = b.cg(x, U, src, am0, 20000, 1e-24)
        res[sched] = (list(its), list(upd), to_host(x))
    for r in range(nrep):
        assert abs(res[8][0][r] - res[9][0][r]) <= 2, (res[8][0], res[9][0])
    bound("schedule 9 vs schedule 8 solution rel", rel(res[9][2], res[8][2]), 1e-12)
    out = {}
    for sched in (8, 9):
        b.schedule = sched
        Ut = U.clone()
        infos = b.hmc_nf2(Ut, am0, 0.1, 4, 20000, 1e-24, [60 + r for r in range(nrep)], 3)
        out[sched] = (infos, to_host(Ut))
    for r in range(nrep):
        assert out[8][0][r].accepted == out[9][0][r].accepted
        bound("schedule 9 vs schedule 8 trajectory dH abs", abs(out[8][0][r].dH - out[9][0][r].dH), 1e-10)
    bound("schedule 9 vs schedule 8 trajectory links rel", rel(out[9][1], out[8][1]), 1e-12)
