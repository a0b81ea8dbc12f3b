"""Command-line drivers with the inputs and outputs of the reference's main/ scripts.

    python -m qed2d.drivers mc           -i run.in                          # main/MC.jl
    python -m qed2d.drivers hmc-nf2      -i run.in --savedir d/ --cont 0    # main/hmc-nf2.jl
    python -m qed2d.drivers rhmc         -i run.in --savedir d/ --cont 0    # main/rhmc.jl
    python -m qed2d.drivers master-field -i run.in                          # main/master_field.jl

Inputs are the reference's JSON files (sections Run, Lattice, HMC, RHMC; keys as in
its README and extra/*.in).  Outputs:
  * hmc-nf2 / rhmc: `<savedir>statistics.txt` (CSV, the reference's columns),
    `<savedir>log.txt`, checkpoints `<savedir>configs/config_<L1>_<L2>_b<beta>_m<mass>_n<i>`
    in the reference's text format every 100 (hmc-nf2) / 10 (rhmc) trajectories, and
    `--cont n` resumes from checkpoint n (main/hmc-nf2.jl:93-145, main/rhmc.jl:100-160);
  * mc / master-field: `<Run.name>.log` with the per-trajectory lines of HMC!
    (src/QED2dHMC.jl:53-57) and the measurements, and `<Run.name>.bdio` with the
    records the reference writes (qed2d/bdio.py; the BDIO container is restated
    from its published format, byte compatibility with BDIO.jl unverified):
      1 the input file (ASC_GENERIC), 2 F64LE [L1, L2, beta, n] (n = ntraj for mc,
      measurements for master-field), then for mc 3 / 4 the plaquette / Q series of
      the measured trajectories -- written L1 times over, as main/MC.jl:140-152
      does -- and for master-field, at every measurement, 3 / 4 the per-site
      plaquette / arg-plaquette densities in rows of fixed i1
      (main/master_field.jl:105-131); every record long and followed by its MD5.
"""
import argparse
import json
import logging
import os
import random
import sys

from . import bdio
from . import io as qio


def _julia(x):
    return qio.julia_float(x) if isinstance(x, float) else str(x)


def _logger(path):
    log = logging.getLogger(f"qed2d.driver.{path}")
    log.setLevel(logging.INFO)
    log.handlers[:] = []
    h = logging.FileHandler(path, mode="a")
    h.setFormatter(logging.Formatter("[ Info: %(message)s"))
    log.addHandler(h)
    return log


def _hmc_line(info, acc):
    tag = "ACCEPT" if info.accepted else "REJECT"
    rate = sum(acc) / len(acc) if acc else 0.0
    return (f"    {tag}: Energy [inital: {_julia(info.hini)}; final: {_julia(info.hfin)}; "
            f"difference: {_julia(info.dH)}]; Pacc = {_julia(float(rate))}")


def read_input(fname):
    with open(fname) as fh:
        s = json.load(fh)
    return s


def _seed(s, fixed=None):
    if fixed is not None:
        return fixed
    seed = int(s["Run"].get("seed", 0))
    return seed if seed != 0 else random.SystemRandom().randint(1, 2**62)


def _config_name(savedir, L1, L2, beta, mass, i):
    return os.path.join(savedir, "configs", f"config_{L1}_{L2}_b{_julia(float(beta))}_m{_julia(mass)}_n{i}")


# ---------------------------------------------------------------------------
def _bdio_title(beta, L1, L2):
    # the protocol text both drivers give BDIO_open (main/MC.jl:87-88, main/master_field.jl:87-88)
    return f"Data from Master field simulation in QED [2d]; beta = {_julia(beta)}; {L1} x {L2}"


def run_mc(args):
    """main/MC.jl: pure-gauge HMC (OMF4); seeds are fixed to 1234 as in MC.jl:70-71."""
    import numpy as np
    import torch

    import qed2d
    s = read_input(args.i)
    name = s["Run"]["name"]
    L1, L2 = s["Lattice"]["size"]
    beta = float(s["Lattice"]["beta"])
    eps, ns = float(s["HMC"]["eps"]), int(s["HMC"]["ns"])
    nthm, nt, qzero = int(s["HMC"]["nthm"]), int(s["HMC"]["ntraj"]), bool(s["HMC"]["Qzero"])
    log = _logger(name + ".log")
    qed2d.seed(1234)
    prm = qed2d.LattParm((L1, L2), beta)
    log.info(f"MONTE CARLO SIMULATION AT BETA = {_julia(beta)}; LATTICE SIZE: {L1} x {L2}")
    log.info(f"  MD PARAMETER eps      = {_julia(eps)}")
    log.info(f"  TRAJECTORY tau        = {_julia(eps * ns)}")
    log.info(f"  THERMALIZATION MDU's  = {_julia(eps * ns * nthm)}")
    fb = bdio.open_run_file(name, s, args.i, _bdio_title(beta, L1, L2), nt)
    U = torch.ones((2, L2, L1), dtype=torch.complex128, device="cuda")   # cold start, MC.jl:119
    acc = []
    for i in range(1, nthm + 1):
        log.info(f" # THERMALIZATION Trajectory {i} / {nthm} [{L1} x {L2}]")
        info = qed2d.HMC_(U, eps, ns, acc, prm, None, qzero=qzero)
        log.info(_hmc_line(info, acc))
        log.info(f"   Plaquette: {_julia(qed2d.Plaquette(U, prm))}")
        log.info(f"   Qtop:      {_julia(qed2d.Qtop(U, prm))}")
    acc, pl, qt = [], [], []
    for j in range(1, nt + 1):
        log.info(f" # MEASUREMENT Trajectory {j} / {nt} [{L1} x {L2}]")
        info = qed2d.HMC_(U, eps, ns, acc, prm, None, qzero=qzero)
        log.info(_hmc_line(info, acc))
        pl.append(qed2d.Plaquette(U, prm))
        qt.append(qed2d.Qtop(U, prm))
        log.info(f"   Plaquette: {_julia(pl[-1])}")
        log.info(f"   Qtop:      {_julia(qt[-1])}")
    for uinfo, series in ((3, pl), (4, qt)):
        fb.start_record(bdio.BIN_F64LE, uinfo, True)
        for _ in range(L1):
            fb.write(np.asarray(series, dtype=np.float64))
        fb.write_hash()
    fb.close()
    return pl, qt


# ---------------------------------------------------------------------------
def run_hmc_nf2(args):
    """main/hmc-nf2.jl: Nf=2 HMC (leapfrog); CGmaxiter 10000, CGtol 1e-16 (:101-103)."""
    import torch

    import qed2d
    s = read_input(args.i)
    savedir, cont = args.savedir, int(args.cont)
    seed = _seed(s, args.seed)
    qed2d.seed(seed)
    if args.precision:
        qed2d.set_precision(args.precision)
    tau, ns = float(s["HMC"]["tau"]), int(s["HMC"]["ns"])
    ntraj, qzero, am0 = int(s["HMC"]["ntraj"]), bool(s["HMC"]["Qzero"]), s["HMC"]["mass"]
    L1, L2 = s["Lattice"]["size"]
    beta = float(s["Lattice"]["beta"])
    prm = qed2d.LattParm((L1, L2), beta)
    U = torch.ones((2, L2, L1), dtype=torch.complex128, device="cuda")
    if cont != 0:
        qed2d.load_gauge(U, _config_name(savedir, L1, L2, beta, am0, cont), prm)
    eps = tau / ns
    CGmaxiter, CGtol = args.cg_maxiter, args.cg_tol
    stat, logf = os.path.join(savedir, "statistics.txt"), os.path.join(savedir, "log.txt")
    if cont == 0:
        os.makedirs(os.path.join(savedir, "configs"), exist_ok=True)
        with open(stat, "w") as fh:
            fh.write("step,accepted,plaquette,top_charge,acc_rate\n")
        with open(logf, "w") as fh:
            fh.write(f"Start HMC run in QED2d with beta = {_julia(beta)}; {L1} x {L2}; mass = {_julia(am0)}; "
                     f"ntraj = {ntraj}; seed = {seed}, nsteps={ns}, tau={_julia(tau)}\n")
    else:
        with open(logf, "a") as fh:
            fh.write(f"Continue HMC run from n={cont} with beta = {_julia(beta)}; {L1} x {L2}; mass = "
                     f"{_julia(am0)}; ntraj = {ntraj}; seed = {seed}, nsteps={ns}, tau={_julia(tau)}\n")
    acc = []
    for i in range(1 + cont, ntraj + cont + 1):
        qed2d.HMC_(U, float(am0), eps, ns, acc, CGmaxiter, CGtol, prm, None, qzero=False)
        plaq, qtop = qed2d.Plaquette(U, prm), qed2d.Qtop(U, prm)
        with open(stat, "a") as fh:
            fh.write(f"{i},{acc[-1]},{_julia(plaq)},{_julia(qtop)},{_julia(sum(acc) / len(acc))}\n")
        if i % 100 == 0:
            qed2d.save_gauge(U, _config_name(savedir, L1, L2, beta, am0, i), prm)
    return U


# ---------------------------------------------------------------------------
def run_rhmc(args):
    """main/rhmc.jl: RHMC, one pseudofermion per flavour; after each trajectory the
    reweighting factor and power-method spectral bounds (iter=5000, :147-148)."""
    import torch

    import qed2d
    s = read_input(args.i)
    savedir, cont = args.savedir, int(args.cont)
    seed = _seed(s, args.seed)
    qed2d.seed(seed)
    if args.precision:
        qed2d.set_precision(args.precision)
    tau, ns = float(s["HMC"]["tau"]), int(s["HMC"]["ns"])
    ntraj = int(s["HMC"]["ntraj"])
    am0 = [float(m) for m in s["RHMC"]["masses"]]
    n_rhmc = [int(n) for n in s["RHMC"]["n_rhmc"]]
    r_a = [float(x) ** 0.5 for x in s["RHMC"]["r_a_g5Dw_sqr"]]
    r_b = [float(x) ** 0.5 for x in s["RHMC"]["r_b_g5Dw_sqr"]]
    L1, L2 = s["Lattice"]["size"]
    beta = float(s["Lattice"]["beta"])
    prm = qed2d.LattParm((L1, L2), beta)
    U = torch.ones((2, L2, L1), dtype=torch.complex128, device="cuda")
    if cont != 0:
        qed2d.load_gauge(U, _config_name(savedir, L1, L2, beta, am0[0], cont), prm)
    rprm = qed2d.get_rhmc_params(n_rhmc, r_a, r_b)
    eps = tau / ns
    CGmaxiter, CGtol = args.cg_maxiter, args.cg_tol
    stat, logf = os.path.join(savedir, "statistics.txt"), os.path.join(savedir, "log.txt")
    if cont == 0:
        os.makedirs(os.path.join(savedir, "configs"), exist_ok=True)
        with open(stat, "w") as fh:
            fh.write("step,accepted,plaquette,top_charge,reweight_factor,lambda_min,lambda_max,acc_rate\n")
        with open(logf, "w") as fh:
            fh.write(f"Start RHMC run in QED2d with beta = {_julia(beta)}; {L1} x {L2}; masses = {am0}; "
                     f"n_rhmc = {n_rhmc}, r_a = {r_a}, r_b = {r_b}; ntraj = {ntraj}; seed = {seed}, "
                     f"nsteps={ns}, tau={_julia(tau)}\n")
    acc = []
    for i in range(1 + cont, ntraj + cont + 1):
        qed2d.HMC_(U, am0, eps, ns, acc, CGmaxiter, CGtol, prm, None, rprm, qzero=False)
        plaq, qtop = qed2d.Plaquette(U, prm), qed2d.Qtop(U, prm)
        w = qed2d.reweighting_factor(U, am0, CGmaxiter, CGtol, prm, None, rprm)
        lmin, lmax = qed2d.power_method(U, am0[0], prm, None, iter=args.power_iter)
        with open(stat, "a") as fh:
            fh.write(f"{i},{acc[-1]},{_julia(plaq)},{_julia(qtop)},{_julia(w)},{_julia(lmin)},{_julia(lmax)},"
                     f"{_julia(sum(acc) / len(acc))}\n")
        if i % 10 == 0:
            qed2d.save_gauge(U, _config_name(savedir, L1, L2, beta, am0[0], i), prm)
    return U


def _err_avg(dfoo):
    """err_avg (main/master_field.jl:41-56): mean and error of the per-site density
    dfoo[i1, i2] from its averages over 16 x 16 blocks (std with Bessel's correction / 16)."""
    import numpy as np
    l1, l2 = dfoo.shape[0] // 16, dfoo.shape[1] // 16
    blks = dfoo[:16 * l1, :16 * l2].reshape(16, l1, 16, l2).sum(axis=(1, 3)) / (l1 * l2)
    return float(blks.mean()), float(blks.std(ddof=1) / 16)


# ---------------------------------------------------------------------------
def run_master_field(args):
    """main/master_field.jl: thermalise 16x16, unfold 2x2 until the target size,
    then `measurements` times store per-site plaquette / arg-plaquette densities."""
    import numpy as np
    import torch

    import qed2d
    s = read_input(args.i)
    name = s["Run"]["name"]
    Lt1, Lt2 = s["Lattice"]["size"]
    beta = float(s["Lattice"]["beta"])
    eps, ns = float(s["HMC"]["eps"]), int(s["HMC"]["ns"])
    nt, qzero = int(s["HMC"]["ntraj"]), bool(s["HMC"]["Qzero"])
    nmsm = int(s["Run"].get("measurements", 1))
    log = _logger(name + ".log")
    fb = bdio.open_run_file(name, s, args.i, _bdio_title(beta, Lt1, Lt2), nmsm)
    qed2d.seed(1234)
    l1 = l2 = 16
    U = torch.ones((2, l2, l1), dtype=torch.complex128, device="cuda")
    acc = []
    while True:
        prm = qed2d.LattParm((l1, l2), beta)
        log.info(f" ## DOUBLING Lattice size: {l1} x {l2}")
        for i in range(1, nt + 1):
            info = qed2d.HMC_(U, eps, ns, acc, prm, None, qzero=qzero)
            log.info(_hmc_line(info, acc))
        if 2 * l1 > Lt1:
            break
        U = qed2d.unfold_fld_(U, prm)
        l1, l2 = 2 * l1, 2 * l2
    prm = qed2d.LattParm((l1, l2), beta)
    plx = torch.empty((l2, l1), dtype=torch.float64, device="cuda")

    def save_msm(j):
        # rows of fixed i1 (Julia's dfoo[i, :]): the (L2, L1) density transposed
        for uinfo, kernel in ((3, qed2d.plaquette_), (4, qed2d.qtop_)):
            kernel(plx, U, prm)
            dens = plx.cpu().numpy()
            fb.start_record(bdio.BIN_F64LE, uinfo, True)
            for i1 in range(l1):
                fb.write(dens[:, i1])
            fb.write_hash()
            if uinfo == 3:
                pavg, perr = _err_avg(dens.T)
                log.info(f" MEASUREMENT {j} of {nmsm}")
                log.info(f"   Plaquette and error: {_julia(pavg)} +/- {_julia(perr)}")

    for j in range(1, nmsm + 1):
        save_msm(j)
        for i in range(1, nt + 1):
            info = qed2d.HMC_(U, eps, ns, acc, prm, None, qzero=qzero)
            log.info(_hmc_line(info, acc))
    save_msm(nmsm + 1)
    fb.close()
    return U


def main(argv=None):
    ap = argparse.ArgumentParser(prog="qed2d.drivers")
    ap.add_argument("driver", choices=["mc", "hmc-nf2", "rhmc", "master-field"])
    ap.add_argument("-i", required=True, help="input file")
    ap.add_argument("--savedir", default="./", help="directory for configurations and logs")
    ap.add_argument("--cont", type=int, default=0, help="continue from configuration number; 0 if new run")
    ap.add_argument("--seed", type=int, default=None, help="override Run.seed")
    ap.add_argument("--precision", choices=["f64", "mixed", "plain"], default=None)
    ap.add_argument("--cg-maxiter", type=int, default=10000)
    ap.add_argument("--cg-tol", type=float, default=1e-16)
    ap.add_argument("--power-iter", type=int, default=5000)
    a = ap.parse_args(argv)
    if not a.savedir.endswith(os.sep):
        a.savedir += os.sep
    {"mc": run_mc, "hmc-nf2": run_hmc_nf2, "rhmc": run_rhmc, "master-field": run_master_field}[a.driver](a)
    return 0


if __name__ == "__main__":
    sys.exit(main())
