"""Single-kernel cases for profiling (ncu) and bandwidth sweeps.

    python -m qed2d.cases <case> --L 2048 [--maxiter 100] [--repeat 3]

cases: g5dw (FP64 gamm5Dw apply), cg_mixed / cg_f64 (one persistent CG launch
capped at --maxiter iterations), force (gamm5Dw + tr_dQwdU), updt (link update),
gauge (krnl_force!, updt_fld!, tr_dQwdU, plaquette! and one pure-gauge OMF4
step),
bcg (one batched mixed CG launch over --batch replicas of L x L), ens (one
batched mixed CG over the 512-replica ensemble of uneven sizes), ms (MultiCG
with 12 Zolotarev poles on [0.9 lambda_min, 1.1 lambda_max] from 300 power
iterations, as the RHMC 128^2 configuration; --schedule 3 for the FP32-inner
form), rhmc (--repeat one-flavour RHMC trajectories of that configuration, ns
20, eps 0.05, after 10 pure-gauge thermalisation trajectories).  Seeded
hot-start links and Gaussian sources; prints the per-launch time of the last
repeat.
"""
import argparse
import sys

import numpy as np
import torch

import qed2d

ENSEMBLE_SIZES = (32, 48, 64, 96, 128, 256)


def ensemble_config(n=512, seed=2024):
    """The replica ensemble: n Nf=2 lattices with sizes drawn from the seed over
    {32, 48, 64, 96, 128, 256}^2, beta ~ U[2, 6], m0 ~ U[0.05, 0.3]; returns
    (sizes, betas, masses)."""
    rng = np.random.default_rng(seed)
    sizes = [(int(s), int(s)) for s in rng.choice(ENSEMBLE_SIZES, n)]
    return sizes, rng.uniform(2.0, 6.0, n).tolist(), rng.uniform(0.05, 0.3, n).tolist()


def hot_batch_field(batch, seed):
    """A hot start (link angles uniform in [-pi, pi)) for every replica of a batch."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    n = 2 * batch.sites
    th = (torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1) * np.pi
    U = torch.polar(torch.ones(n, dtype=torch.float64, device="cuda"), th)
    return U.view(batch.field().shape) if batch.uniform else U


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["g5dw", "cg_mixed", "cg_f64", "force", "updt", "bcg", "ens", "ms", "rhmc", "gauge"])
    ap.add_argument("--schedule", type=int, default=-1, help="ms: multishift schedule (-1 tuned)")
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--L", type=int, default=2048)
    ap.add_argument("--maxiter", type=int, default=100)
    ap.add_argument("--repeat", type=int, default=3)
    a = ap.parse_args(argv)
    L = a.L
    prm = qed2d.LattParm((L, L), 4.0)
    g = torch.Generator(device="cuda").manual_seed(1234)
    U = torch.polar(torch.ones(2, L, L, dtype=torch.float64, device="cuda"),
                    (torch.rand(2, L, L, dtype=torch.float64, device="cuda", generator=g) * 2 - 1) * np.pi)
    si = torch.randn(2, L, L, dtype=torch.complex128, device="cuda", generator=g)
    so = torch.zeros_like(si)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if a.case == "bcg":
        bt = qed2d.Batch(a.batch, L, L, 4.0)
        Ub, bb, xb = bt.field(), bt.field(), bt.field()
        for r in range(a.batch):
            Ub[r] = U
            bb[r] = torch.randn(2, L, L, dtype=torch.complex128, device="cuda", generator=g)
    if a.case == "ens":
        sizes, betas, am0s = ensemble_config(512, 2024)
        bt = qed2d.Batch.ragged(sizes, betas)
        Ub = hot_batch_field(bt, 2024)
        bb = torch.randn(2 * bt.sites, dtype=torch.complex128, device="cuda", generator=g)
        xb = torch.zeros_like(bb)
    if a.case == "rhmc":
        for _ in range(10):
            qed2d.HMC_(U, 0.1, 10, [], prm, None)
    if a.case in ("ms", "rhmc"):
        lmin, lmax = qed2d.power_method(U, 0.1, prm, None, iter=300)
        rp = qed2d.get_rhmc_params(12, np.sqrt(0.9 * lmin), np.sqrt(1.1 * lmax))
        qed2d.set_schedule(prm, a.schedule, "multishift")
    for _ in range(a.repeat):
        ev0.record()
        if a.case == "g5dw":
            qed2d.gamm5Dw(so, U, si, 0.1, prm)
        elif a.case in ("cg_mixed", "cg_f64"):
            qed2d.set_precision("mixed" if a.case == "cg_mixed" else "f64")
            try:
                qed2d.CG(so, U, si, 0.1, a.maxiter, 1e-24, qed2d.gamm5Dw_sqr_msq, prm, None)
            except qed2d.Qed2dError:
                pass   # capped iteration count, as intended
        elif a.case == "force":
            g5 = torch.empty_like(si)
            qed2d.gamm5Dw(g5, U, si, 0.1, prm)
            f = torch.zeros(2, L, L, dtype=torch.float64, device="cuda")
            qed2d.tr_dQwdU(f, U, si, g5, prm)
        elif a.case in ("bcg", "ens"):
            try:
                it = bt.cg(xb, Ub, bb, 0.1 if a.case == "bcg" else am0s, a.maxiter, 1e-24)
            except qed2d.Qed2dError:
                it = "capped"
        elif a.case == "ms":
            try:
                it = qed2d.MultiCG(so, U, si, 0.1, a.maxiter, 1e-24, qed2d.gamm5Dw_sqr_msq, rp, prm)
            except qed2d.Qed2dError:
                it = "capped"
        elif a.case == "rhmc":
            it = qed2d.HMC_(U, [0.1], 0.05, 20, [], 10000, 1e-24, prm, None, [rp])
        elif a.case == "gauge":
            f1 = torch.empty(2, L, L, dtype=torch.float64, device="cuda")
            f2 = torch.empty_like(f1)
            mom = torch.randn(2, L, L, dtype=torch.float64, device="cuda", generator=g) * 1e-12
            plx = torch.empty(L, L, dtype=torch.float64, device="cuda")
            qed2d.krnl_force_(f1, f2, U, prm)
            qed2d.updt_fld_(U, mom, 1.0)
            qed2d.tr_dQwdU(f1, U, si, so, prm)
            qed2d.plaquette_(plx, U, prm)
            qed2d.OMF4_(mom, U, 1e-3, 1, prm, None)
        elif a.case == "updt":
            mom = torch.randn(2, L, L, dtype=torch.float64, device="cuda", generator=g)
            qed2d.updt_fld_(U, mom, 0.01)
        ev1.record()
        torch.cuda.synchronize()
    it = qed2d.last_solve(prm) if a.case.startswith("cg") else (it if a.case in ("bcg", "ens", "ms", "rhmc") else None)
    print(f"{a.case} L={L}: {ev0.elapsed_time(ev1):.3f} ms  solve={it}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
