"""The benchmark's headline step pinned to the oracle.

* Four 512x512 Nf=2 replica chains advanced by batched trajectories exactly as
  bench.py times them: the same thermalised start (seeded hot start + 10
  pure-gauge trajectories), beta=4, m0=0.1, leapfrog ns=20, eps=0.05, every CG
  to |r|^2 < 1e-24 |b|^2, the equal-size batched mixed solver under the
  schedule its tuner picks.  Each replica's trajectory is replayed on the
  oracle (FP64 reference CG, src/QED2dHMC.jl:64-113, :426-481) with the same
  Philox draws from the same start field.
* Single-lattice CG at 512^2 and 2048^2 (fused FP64 and mixed solvers) against
  the oracle's CG (src/QED2dSolver.jl:3-46) on a thermalised field.

Bounds are stated per quantity below; every achieved error is recorded through
helpers.bound.  H_ini and H_fin are O(beta V) sums (~1e6 here): they are
compared relative to |H|, dH absolutely.  H_fin is evaluated on the field and
momenta at the end of the molecular dynamics, before the Metropolis step, so it
pins the MD evolution even when the trajectory is rejected and the links
restored."""
import numpy as np
import pytest

import bench
from helpers import bound, cgauss, note, rel, to_dev, to_host
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

NREP = 4


@pytest.fixture(scope="module")
def thermalised():
    """bench.py's start field: hot start, 10 pure-gauge trajectories on the GPU."""
    import qed2d
    L = bench.L
    prm = qed2d.LattParm((L, L), bench.BETA)
    U1 = to_dev(bench.hot_start(L, L, bench.SEED))
    qed2d.seed(bench.SEED + 1)
    for _ in range(bench.THERM_TRAJ):
        qed2d.HMC_(U1, 0.1, 10, [], prm, None)
    return U1


def test_headline_batched_trajectories_vs_oracle(thermalised):
    import qed2d
    L = bench.L
    V = L * L
    b = qed2d.Batch(NREP, L, L, bench.BETA)
    U = b.field()
    for r in range(NREP):
        U[r] = thermalised
    seeds = [bench.SEED + 101 * r for r in range(NREP)]   # rank 0's replica seeds in bench.py
    o = Oracle(L, L, bench.BETA)
    accepted = 0
    for counter in (0, 1):
        U_start = [to_host(U[r]) for r in range(NREP)]
        infos = b.hmc_nf2(U, bench.AM0, bench.EPS, bench.NS, bench.MAXITER, bench.TOL, seeds, counter)
        assert b.schedule in (0, 1, 4, 5, 8, 9)
        note("batched solver schedule, tile rows", [b.schedule, b.tile_rows])
        for r in range(NREP):
            mom0 = Oracle.normal(2 * V, seeds[r], 1, counter).reshape(2, L, L)
            noise = cgauss(L, L, seeds[r], 16, counter)
            st, Uo, acc, hi, hf, ito = o.hmc_nf2(U_start[r], bench.AM0, bench.EPS, bench.NS, bench.MAXITER,
                                                  bench.TOL, mom0, noise, Oracle.uniform(seeds[r], 3, counter))
            assert st == 0
            i = infos[r]
            assert i.accepted == acc, (counter, r, i.dH, hf - hi)
            accepted += acc
            bound("H_ini rel (4x512^2 batched)", abs(i.hini - hi) / abs(hi), 5e-15)
            bound("H_fin rel (4x512^2 batched)", abs(i.hfin - hf) / abs(hf), 1e-14)
            bound("dH abs (4x512^2 batched)", abs(i.dH - (hf - hi)), 1e-8)
            bound("final links rel (4x512^2 batched)", rel(to_host(U[r]), Uo), 1e-11)
            # 21 solves per trajectory; the FP32 inner iterations may differ from FP64 by one here and there
            bound("CG iterations rel diff (4x512^2 batched mixed vs oracle FP64)",
                  abs(i.cg_iterations - ito) / ito, 2e-3)
            note("dH (4x512^2 batched)", i.dH)
    note("accepted of 8 (4x512^2 batched)", accepted)


@pytest.mark.parametrize("prec", ["f64", "mixed"])
@pytest.mark.parametrize("L", [512, 2048])
def test_cg_large_vs_oracle(thermalised, prec, L):
    """Single-lattice CG at the headline size and at 2048^2 (the 512^2 start
    field unfolded 2x2 twice, as the master-field driver grows lattices, then
    thermalised by 5 pure-gauge trajectories).  Both solutions meet the
    relative residual 1e-12; they differ by the residual difference amplified
    by at most the condition number, which is recorded beside the error."""
    import qed2d
    qed2d.set_precision(prec)
    try:
        prm0 = qed2d.LattParm((512, 512), bench.BETA)
        U = thermalised
        Ls = 512
        while Ls < L:
            U = qed2d.unfold_fld_(U, qed2d.LattParm((Ls, Ls), bench.BETA))
            Ls *= 2
        prm = qed2d.LattParm((L, L), bench.BETA)
        if L != 512:
            qed2d.seed(77)
            for _ in range(5):
                qed2d.HMC_(U, 0.1, 10, [], prm, None)
        del prm0
        Uh = to_host(U)
        b = cgauss(L, L, 4242, 2)
        o = Oracle(L, L, bench.BETA)
        st, xo, ito, _ = o.cg(Uh, b, bench.AM0, bench.MAXITER, bench.TOL)
        assert st == 0
        x = qed2d.cfield(L, L)
        it = qed2d.CG(x, U, to_dev(b), bench.AM0, bench.MAXITER, bench.TOL, qed2d.gamm5Dw_sqr_msq, prm, None)
        xg = to_host(x)
        nb = np.linalg.norm(b)
        res_g = np.linalg.norm(b - o.g5dw_sqr(Uh, xg, bench.AM0)) / nb
        res_o = np.linalg.norm(b - o.g5dw_sqr(Uh, xo, bench.AM0)) / nb
        err = np.linalg.norm(xg - xo) / np.linalg.norm(xo)
        # the residual the reference's stop rule asks for, evaluated by the oracle in FP64
        bound(f"CG {prec} {L}^2 oracle-evaluated |b-Ax|/|b|", res_g, 1.0e-12)
        # solution difference, L2-relative; the amplification err / (res_g + res_o) is at most kappa
        bound(f"CG {prec} {L}^2 |x-x_o|/|x_o|", err, 1e-14 if prec == "f64" else 1e-13)
        note(f"CG {prec} {L}^2 amplification err/(res_g+res_o)", err / (res_g + res_o))
        note(f"CG {prec} {L}^2 max-abs rel", rel(xg, xo))
        if prec == "f64":
            bound(f"CG f64 {L}^2 iterations |it-it_o|", abs(it - ito), 1)
        else:
            bound(f"CG mixed {L}^2 iterations rel diff", abs(it - ito) / ito, 0.01)
        note(f"CG {prec} {L}^2 iterations (gpu, oracle)", [it, ito])
    finally:
        qed2d.set_precision("f64")
