#!/usr/bin/env python
"""Headline benchmark: Nf=2 HMC trajectories/s on 512x512 lattices.

    python bench.py [--gpus N --steps K --warmup W] [--batch B] [--impl reference]

Workload: Nf=2 Wilson fermions, beta=4.0, m0=0.1, leapfrog ns=20, eps=0.05
(tau=1), every CG solved to |r|/|b| < 1e-12 (the reference's stop rule with
eps=1e-24), mixed FP32-inner/FP64-reliable-update solver, B replica chains per
GPU advanced together ("batched"); one "step" = one batched trajectory = B
trajectories.  Synthetic data: a seeded hot start thermalised by 10 untimed
pure-gauge trajectories, copied to every replica (distinct seeds).  L2 is
flushed (256 MiB write) between timed steps.

Prints one JSON line (rank 0).  Under torchrun every rank runs an independent
replica chain (no collective on the data path): value = all ranks' trajectories
/ the slowest rank's time.

--impl reference times the reference's algorithm on the host CPU cores: the C
restatement in oracle/ (the reference itself is Julia/CUDA.jl with no CPU
path, and Julia is not installed).  Each of its steps is one full trajectory of
replica chain 0 -- the same thermalised start and the same draws as the GPU
arm's replica 0 at that step -- so its CG iteration counts match the GPU arm's.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (REPO, os.path.join(REPO, "dav-qed2d_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "HMC traj/s Nf=2 512²: mixed+batched vs FP64 at CG res 1e-12; Dslash HBM GB/s"
L, BETA, AM0, NS, EPS, TOL, MAXITER = 512, 4.0, 0.1, 20, 0.05, 1e-24, 200000
SEED = 1234
WORKLOAD = (f"Nf=2 HMC trajectory, {L}x{L}, beta={BETA}, m0={AM0}, leapfrog ns={NS} eps={EPS}, "
            f"CG to |r|/|b|<1e-12 (eps=1e-24)")
THERM_TRAJ = 10
# algorithmic bytes per site of the solver phases (FP32 packed spinors and links)
# FP32 fused iteration: phase A 80 B + phase B 96 B on average -- the mixed solvers
# update x every second iteration for two directions (phase B 64 B, then 128 B)
B_MIXED_ITER = 176.0
B_MIXED_UPDATE = 400.0   # one FP64 reliable update (4 phases)
B_MIXED_SETUP = 112.0    # |b|^2, x=0, r32 = b/|b|, x32 = 0
B_F64_ITER = 384.0       # FP64 fused iteration: phase A 160 B + phase B 224 B
B_DSLASH_F64 = 96.0      # g5Dw apply, FP64: spinor in 32 + links 32 + out 32
B_DSLASH_C64 = 48.0      # g5Dw apply on complex64 fields: spinor in 16 + links 16 + out 16
B_KRNL_FORCE = 64.0      # krnl_force!: links in 32 + frc1, frc2 out 16 + 16
B_UPDT_FLD = 80.0        # updt_fld!: momenta in 16 + links in and out 32 + 32
B_TR_DQWDU = 112.0       # tr_dQwdU: links 32 + X 32 + g5Dw X 32 in, force out 16
B_PLAQ_FIELD = 40.0      # plaquette!: links in 32 + per-site plaquette out 8
B_OMF4_STEP = 6 * 64.0 + 5 * 80.0   # one pure-gauge OMF4 step as the reference's kernels move it: 6 kicks
                                    # (links 32 + momenta r/w 32), 5 link updates (the fused passes move 544)
# Roofline units of the headline kernel.  Algorithmic bytes per site of one CG
# iteration on (g5Dw)^2: 256 B in FP32 (two applies at 48 B + ten vector passes
# at 16 B), 512 B in FP64 -- an FP64 reliable update is counted as one FP64
# iteration.  (The fused solver moves 176 B per FP32 iteration by design; that
# figure is reported beside.)
B_ITER_F32 = 256.0
B_ITER_F64 = 512.0
# Measured traffic per site-iteration of k_u_cg_mixed at 4 x 512^2, from one ncu
# capture of a 100-iteration launch of the tuned kernel (independent replicas,
# lean reduction, phase-A stencil on r, links staged in shared memory, 32 x 16
# tiles): DRAM read + write (5.391 GB over 1,048,576 sites x 100) and L1 <-> L2
# (13.29 GB read + 6.56 GB written); both grow in proportion to the iterations
# at fixed size
U_DRAM_PER_SITE_ITER = 51.4
U_L2_PER_SITE_ITER = 189.3
U_L2_THROUGHPUT = 0.360   # lts__throughput.avg.pct_of_peak_sustained_elapsed of the same capture
ENS_NS, ENS_EPS = 10, 0.1   # replica ensemble: leapfrog ns=10, eps=0.1
CPU_TRAJ = 2                # trajectories of the GPU arm's CPU-baseline sample


def l2_copy_peak(torch, dev):
    """L2 bandwidth probe in this run (CUDA events): the best of three streaming
    passes over buffers that stay in L2 (126 MB) -- a copy (24 MiB in, 24 MiB
    out), an in-place add (two 16 MiB reads, one write) and a sum (48 MiB read) --
    counting the bytes each moves.  Reported beside the headline kernel's L2
    rate; these simple kernels do not reach the L2's peak, so the L2 fraction
    itself is ncu's for the kernel."""
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def rate(fn, nbytes, reps=200):
        for _ in range(10):
            fn()
        best = 0.0
        for _ in range(3):
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            best = max(best, nbytes * reps / (e0.elapsed_time(e1) / 1e3) / 1e9)
        return best

    a = torch.ones(24 * 2**20 // 4, dtype=torch.float32, device=dev)
    b = torch.empty_like(a)
    c = torch.ones(16 * 2**20 // 4, dtype=torch.float32, device=dev)
    d = torch.ones_like(c)
    e = torch.ones(48 * 2**20 // 4, dtype=torch.float32, device=dev)
    out = torch.empty((), dtype=torch.float32, device=dev)
    return max(rate(lambda: b.copy_(a), 2 * a.numel() * 4),
               rate(lambda: c.add_(d), 3 * c.numel() * 4),
               rate(lambda: torch.sum(e, dim=0, out=out), e.numel() * 4))


def load_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.index)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def hot_start(L1, L2, seed):
    import numpy as np
    rng = np.random.default_rng(seed)
    return np.exp(1j * rng.uniform(-np.pi, np.pi, (2, L2, L1)))


# ---------------------------------------------------------------------------
# reference arm / CPU baseline: the oracle (C restatement of the reference)
def oracle_trajectory(o, U, seed, counter):
    """One full Nf=2 trajectory of the workload (HMC! with leapfrog: momenta and
    pseudofermion draws, ns+1 force evaluations each with a CG solve to 1e-24,
    Metropolis) on the host cores, with the draws replica chain `seed` makes at
    trajectory `counter` on the GPU.  Returns (seconds, new field, CG iterations)."""
    import numpy as np
    from oracle import oracle as O
    mom0 = O.Oracle.normal(2 * L * L, seed, 1, counter).reshape(2, L, L)
    z = O.Oracle.normal(4 * L * L, seed, 16, counter)
    noise = ((z[0::2] + 1j * z[1::2]) / np.sqrt(2.0)).reshape(2, L, L)
    u = O.Oracle.uniform(seed, 3, counter)
    t0 = time.perf_counter()
    st, U, acc, hi, hf, it = o.hmc_nf2(U, AM0, EPS, NS, MAXITER, TOL, mom0, noise, u)
    dt = time.perf_counter() - t0
    if st != 0:
        raise RuntimeError("oracle CG did not converge")
    return dt, U, it


def oracle_thermalised_field():
    """The same thermalisation as the GPU arm, replayed on the oracle."""
    from oracle import oracle as O
    o = O.Oracle(L, L, BETA)
    U = hot_start(L, L, SEED)
    for t in range(THERM_TRAJ):
        mom0 = O.Oracle.normal(2 * L * L, SEED + 1, 1, t).reshape(2, L, L)
        st, U, acc, hi, hf = o.hmc_gauge(U, 0.1, 10, mom0, O.Oracle.uniform(SEED + 1, 3, t))
    return U


def run_reference(args):
    """The reference's algorithm on the host cores: one step = one full trajectory
    of replica chain 0 (seed SEED, counter = step index), from the same
    thermalised start as the GPU arm, i.e. the trajectory the GPU arm's replica 0
    runs at the same step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    U = oracle_thermalised_field()
    o = O.Oracle(L, L, BETA)
    times, iters = [], []
    for k in range(args.warmup + args.steps):
        dt, U, it = oracle_trajectory(o, U, SEED, k)
        if k >= args.warmup:
            times.append(dt)
            iters.append(it)
    t_traj = statistics.mean(times)
    value = 1.0 / t_traj
    cores = O.num_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "traj/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_traj, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "solver": "reference CG (FP64, host)", "chains": 1},
        "cpu_baseline": {"value": value, "unit": "traj/s", "cores": cores, "kind": "port",
                         "sample": f"per step one full {L}x{L} trajectory (HMC! Nf=2, leapfrog ns={NS}) of replica "
                                   f"chain 0 from the thermalised start, the draws of the GPU arm's replica 0 "
                                   f"at the same step; mean CG iterations per trajectory "
                                   f"{statistics.mean(iters):.0f}"},
        "e2e": {"value": value, "unit": "traj/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def run_configs(qed2d, torch, dev):
    """Trajectories/s of the benchmark configurations on one GPU (timed with
    CUDA events after warm-up; each a bounded number of trajectories):
    C1 pure gauge 128^2 (OMF4 ns=10 eps=0.15), C2 Nf=2 64^2 (leapfrog ns=20
    eps=0.05; mixed, fused FP64 and plain FP64 solvers), C3 Nf=1 RHMC 128^2 with
    12 Zolotarev poles on the power-method interval (ns=20 eps=0.05), C5 master
    field pure gauge 8192^2 (OMF4 ns=20 eps=0.025)."""
    import numpy as np

    def timed(fn, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return n / (e0.elapsed_time(e1) / 1e3)

    out = {}
    qed2d.seed(SEED)
    # C1
    p1 = qed2d.LattParm((128, 128), 11.25)
    U = torch.from_numpy(hot_start(128, 128, 1234)).to(dev)
    step = lambda: qed2d.HMC_(U, 0.15, 10, [], p1, None, integrator=qed2d.OMF4())
    for _ in range(20):
        step()
    out["C1_pure_gauge_128_omf4"] = {"value": timed(step, 100), "unit": "traj/s", "trajectories": 100}
    # C2
    p2 = qed2d.LattParm((64, 64), 4.0)
    U2 = torch.from_numpy(hot_start(64, 64, 64)).to(dev)
    for _ in range(10):
        qed2d.HMC_(U2, 0.1, 10, [], p2, None)   # pure-gauge thermalisation
    c2, sched = {}, {}
    names = {0: "grid, last block publishes", 1: "grid, every block sums", 2: "one thread-block cluster"}
    names.update({k + 4: v + "; stencil on r, links in shared memory" for k, v in list(names.items())})
    for prec in ("mixed", "f64", "plain"):
        qed2d.set_precision(prec)
        Uc = U2.clone()
        st = lambda: qed2d.HMC_(Uc, 0.1, 0.05, 20, [], MAXITER, TOL, p2, None)
        st()
        c2[prec] = timed(st, 10)
        if prec != "plain":
            sched[prec] = names.get(qed2d.get_schedule(p2, prec), "untuned")
    qed2d.set_precision("f64")
    out["C2_nf2_64_leapfrog"] = {"unit": "traj/s", "mixed": c2["mixed"], "f64_fused": c2["f64"], "plain_f64": c2["plain"],
                                 "mixed_vs_plain": c2["mixed"] / c2["plain"], "trajectories": 10,
                                 "solver_schedule": sched}
    # C3
    p3 = qed2d.LattParm((128, 128), 4.0)
    U3 = torch.from_numpy(hot_start(128, 128, 128)).to(dev)
    for _ in range(10):
        qed2d.HMC_(U3, 0.1, 10, [], p3, None)
    lmin, lmax = qed2d.power_method(U3, 0.1, p3, None, iter=300)
    rp = [qed2d.get_rhmc_params(12, np.sqrt(0.9 * lmin), np.sqrt(1.1 * lmax))]
    st3 = lambda: qed2d.HMC_(U3, [0.1], 0.05, 20, [], MAXITER, TOL, p3, None, rp)
    st3()
    out["C3_rhmc_128_12_poles"] = {"value": timed(st3, 10), "unit": "traj/s", "solver": "FP64 multi-shift, one launch for all poles",
                                   "solver_schedule": names.get(qed2d.get_schedule(p3, "multishift"), "untuned"),
                                   "solver_layout": {0: "32x8 tiles, one thread per site", 1: "32x8 tiles, two threads per site",
                                                     2: "32x4 tiles, four threads per site",
                                                     3: "32x4 tiles, two threads per site"}.get(
                                       qed2d.get_multishift_layout(p3), "untuned"),
                                   "trajectories": 10}
    del U, U2, U3
    # C5
    p5 = qed2d.LattParm((8192, 8192), 11.25)
    U5 = torch.polar(torch.ones(2, 8192, 8192, dtype=torch.float64, device=dev),
                     (torch.rand(2, 8192, 8192, dtype=torch.float64, device=dev) * 2 - 1) * np.pi)
    st5 = lambda: qed2d.HMC_(U5, 0.025, 20, [], p5, None, integrator=qed2d.OMF4())
    st5()
    out["C5_master_field_8192_omf4"] = {"value": timed(st5, 2), "unit": "traj/s", "trajectories": 2}
    del U5
    torch.cuda.empty_cache()
    return out


def run_ours(args):
    import numpy as np
    import torch

    import qed2d
    from qed2d import _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    Lb = _lib.lib()
    B = args.batch
    prm = qed2d.LattParm((L, L), BETA)
    seed0 = SEED + 7919 * rank
    seeds = [seed0 + 101 * r for r in range(B)]

    # --- set-up (untimed): hot start, pure-gauge thermalisation, copied to every replica
    U1 = torch.from_numpy(hot_start(L, L, SEED)).to(dev)
    qed2d.seed(SEED + 1)
    for _ in range(THERM_TRAJ):
        qed2d.HMC_(U1, 0.1, 10, [], prm, None)
    batch = qed2d.Batch(B, L, L, BETA)
    U = batch.field()
    for r in range(B):
        U[r] = U1
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    counter = [0]

    def step():
        flush.fill_(1.0)
        c = counter[0]
        counter[0] += 1
        return batch.hmc_nf2(U, AM0, EPS, NS, MAXITER, TOL, seeds, c)

    for _ in range(args.warmup):
        step()
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    n0 = Lb.qed2d_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    infos = [step() for _ in range(args.steps)]
    ev1.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = Lb.qed2d_launch_count() - n0
    clk = clocks.stop()
    elapsed = ev0.elapsed_time(ev1) / 1e3
    if dist:
        t = torch.tensor([elapsed], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    value = world * B * args.steps / elapsed
    flat = [i for step_infos in infos for i in step_infos]

    # --- e2e: the same step through the C ABI with host buffers: H2D of the
    # links from pinned memory, the batched trajectory, D2H of links + results
    U_host = U.cpu().pin_memory()
    res = (_lib.HmcResult * B)()
    am = (C.c_double * B)(*([AM0] * B))
    sd = (C.c_uint64 * B)(*seeds)
    Lb.qed2d_batch_set_stream(batch.h, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(args.steps):
        U.copy_(U_host, non_blocking=True)
        st = Lb.qed2d_batch_hmc_nf2(batch.h, C.c_void_p(U.data_ptr()), am, EPS, NS, MAXITER, TOL, 0, sd,
                                    50000 + k, res)
        _lib.check(st, "batch_hmc_nf2")
        U_host.copy_(U, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_t = e0.elapsed_time(e1) / 1e3
    if dist:
        t = torch.tensor([e2e_t], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_t = float(t.item())
    e2e = {"value": world * B * args.steps / e2e_t, "unit": "traj/s",
           "h2d_bytes_per_step": U.numel() * 16, "d2h_bytes_per_step": U.numel() * 16 + C.sizeof(res)}

    # --- replica ensemble: 512 Nf=2 lattices of uneven sizes; under torchrun
    # each rank advances its cost-balanced share (no exchange), timed as the
    # slowest rank
    ensemble = None
    if not args.skip_ensemble:
        from qed2d.cases import ensemble_config, hot_batch_field
        from qed2d.replicas import gather_by_replica, rank_share, slowest
        sizes, betas, am0s = ensemble_config(512, 2024)
        mine = rank_share(sizes, rank, world)
        eb = qed2d.Batch.ragged([sizes[i] for i in mine], [betas[i] for i in mine])
        Ue = hot_batch_field(eb, 2024 + rank)
        em, es = [am0s[i] for i in mine], [9000 + i for i in mine]
        eb.hmc_nf2(Ue, em, ENS_EPS, ENS_NS, MAXITER, TOL, es, 0)   # warm-up
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n_traj = 2
        e0.record()
        einfos = [eb.hmc_nf2(Ue, em, ENS_EPS, ENS_NS, MAXITER, TOL, es, 1 + t) for t in range(n_traj)]
        e1.record()
        torch.cuda.synchronize()
        t_e = slowest(e0.elapsed_time(e1) / 1e3, device=dev if dist else None)
        per_rep = gather_by_replica(mine, [(sum(st[j].cg_iterations for st in einfos),
                                            sum(st[j].accepted for st in einfos)) for j in range(len(mine))],
                                    len(sizes))
        ensemble = {"replicas": len(sizes), "sites": sum(a * b for a, b in sizes),
                    "sizes": "32..256 squared, drawn from seed 2024", "beta": "U[2,6]", "m0": "U[0.05,0.3]",
                    "ns": ENS_NS, "eps": ENS_EPS, "start": "hot", "ranks": world,
                    "value": len(sizes) * n_traj / t_e, "unit": "traj/s", "ms_per_batched_traj": 1e3 * t_e / n_traj,
                    "cg_iterations_per_traj_mean": sum(p[0] for p in per_rep) / (n_traj * len(sizes)),
                    "accepted": sum(p[1] for p in per_rep), "of": n_traj * len(sizes),
                    "timed": f"{n_traj} batched trajectories after 1 warm-up",
                    "solver": {2: "one launch over all replicas, grid barriers",
                               3: "one thread-block cluster per replica",
                               6: "one thread-block cluster per replica, phase-A stencil on r"}.get(eb.schedule,
                                                                                                    "untuned")}
        del eb, Ue
        torch.cuda.empty_cache()

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    # --- roofline of the dominant kernel: one batched mixed CG launch solving
    # every replica's (g5Dw)^2 x = b at the workload's fields, CUDA events
    peak, peak_kind = load_peaks()
    src = (torch.randn(U.shape, dtype=torch.complex128, device=dev) / np.sqrt(2.0)).contiguous()
    xs = torch.zeros_like(src)
    kern = []
    for _ in range(3):
        flush.fill_(1.0)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        its, upd = batch.cg(xs, U, src, AM0, MAXITER, TOL)
        a1.record()
        torch.cuda.synchronize()
        kern.append((a0.elapsed_time(a1) / 1e3, its, upd))
    t_k, its, upd = min(kern[1:], key=lambda z: z[0])
    V = L * L
    bytes_k = V * sum(i * B_ITER_F32 + u * B_ITER_F64 for i, u in zip(its, upd))
    fused_k = V * sum(B_MIXED_SETUP + i * B_MIXED_ITER + u * B_MIXED_UPDATE for i, u in zip(its, upd))
    achieved = bytes_k / t_k / 1e9
    traffic = V * sum(its) * U_DRAM_PER_SITE_ITER
    l2_bytes = V * sum(its) * U_L2_PER_SITE_ITER
    l2_peak = l2_copy_peak(torch, dev)
    roofline = {"kernel": "k_u_cg_mixed", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                "dram_achieved": traffic / t_k / 1e9, "dram_frac": traffic / t_k / 1e9 / peak,
                "fused_model_achieved": fused_k / t_k / 1e9,
                "l2": {"achieved": l2_bytes / t_k / 1e9, "unit": "GB/s", "frac": U_L2_THROUGHPUT,
                       "frac_kind": "ncu lts__throughput of this kernel, fraction of the L2 peak",
                       "probe_GBs": l2_peak,
                       "probe_kind": "best of a copy, an add and a sum on L2-resident buffers in this run "
                                     "(torch kernels; below what the L2 sustains for this kernel's mix)"},
                "launch_us": t_k * 1e6,
                "schedule": {0: "last block publishes the sums", 1: "every block sums",
                             4: "independent replicas (a barrier per replica)",
                             5: "independent replicas, lean reduction",
                             7: "independent replicas, lean reduction, TMA-staged stencil operands",
                             8: "independent replicas, lean reduction, phase-A stencil on r",
                             9: "independent replicas, lean reduction, phase-A stencil on r, links in shared "
                                "memory"}.get(
                                 batch.schedule, "untuned"),
                "tile_rows": batch.tile_rows,
                "note": f"one launch = one solve of all {B} replicas: per replica iterations {min(its)}-{max(its)} "
                        f"x {B_ITER_F32:.0f} B/site + reliable updates {min(upd)}-{max(upd)} x {B_ITER_F64:.0f} "
                        f"B/site (algorithmic); the {B} x {L}^2 FP32 working set is mostly L2-resident, so the "
                        f"algorithmic rate exceeds the DRAM copy bandwidth; traffic = ncu DRAM bytes per "
                        f"site-iteration x the solve's site-iterations (dram_achieved = traffic / time); l2 = "
                        f"ncu L1<->L2 bytes per site-iteration x site-iterations against an L2-resident copy "
                        f"measured in this run; neither is saturated: the kernel is latency- and barrier-bound"}

    # --- single-chain baselines on the same field and draws as replica 0's first
    # timed step: mixed (no batching), fused FP64, and the plain FP64 GPU path
    base = {}
    if not args.skip_baselines:
        for prec in ("mixed", "f64", "plain"):
            qed2d.set_precision(prec)
            Ub = U1.clone()
            qed2d.seed(seeds[0])
            qed2d.HMC_(Ub.clone(), AM0, EPS, NS, [], MAXITER, TOL, prm, None, counter=args.warmup)   # warm-up
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            info = qed2d.HMC_(Ub, AM0, EPS, NS, [], MAXITER, TOL, prm, None, counter=args.warmup)
            torch.cuda.synchronize()
            base[prec] = (time.perf_counter() - t0, info.cg_iterations)
        qed2d.set_precision("f64")

    # --- Dslash / CG-iteration HBM bandwidth at 8192^2 (working set >> L2)
    dslash = None
    if not args.skip_sweep:
        del batch, U, xs, src
        torch.cuda.empty_cache()
        Lbig = 8192
        pb = qed2d.LattParm((Lbig, Lbig), BETA)
        Ub = torch.polar(torch.ones(2, Lbig, Lbig, dtype=torch.float64, device=dev),
                         (torch.rand(2, Lbig, Lbig, dtype=torch.float64, device=dev) * 2 - 1) * np.pi)
        si = torch.randn(2, Lbig, Lbig, dtype=torch.complex128, device=dev)
        so = torch.empty_like(si)
        for _ in range(3):
            qed2d.gamm5Dw(so, Ub, si, AM0, pb)
        n_ap = 20
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        for _ in range(n_ap):
            qed2d.gamm5Dw(so, Ub, si, AM0, pb)
        a1.record()
        torch.cuda.synchronize()
        t_ap = a0.elapsed_time(a1) / 1e3 / n_ap
        Vb = Lbig * Lbig
        f64_gbs = B_DSLASH_F64 * Vb / t_ap / 1e9
        # the same apply on complex64 spinors and links
        U64, si64 = Ub.to(torch.complex64), si.to(torch.complex64)
        so64 = torch.empty_like(si64)
        for _ in range(3):
            qed2d.gamm5Dw(so64, U64, si64, AM0, pb)
        a0.record()
        for _ in range(n_ap):
            qed2d.gamm5Dw(so64, U64, si64, AM0, pb)
        a1.record()
        torch.cuda.synchronize()
        t_ap32 = a0.elapsed_time(a1) / 1e3 / n_ap
        c64_gbs = B_DSLASH_C64 * Vb / t_ap32 / 1e9
        apply_err = float(((so64.to(torch.complex128) - so).abs().max() / so.abs().max()).item())
        del U64, si64, so64

        def kernel_gbs(fn, nbytes):
            for _ in range(3):
                fn()
            a0.record()
            for _ in range(n_ap):
                fn()
            a1.record()
            torch.cuda.synchronize()
            t = a0.elapsed_time(a1) / 1e3 / n_ap
            return {"GBs": nbytes * Vb / t / 1e9, "frac": nbytes * Vb / t / 1e9 / peak, "us": t * 1e6}
        # the gauge-field kernels of the reference's interface, each on its own
        frc1 = torch.empty(2, Lbig, Lbig, dtype=torch.float64, device=dev)
        frc2 = torch.empty_like(frc1)
        mom = torch.randn(2, Lbig, Lbig, dtype=torch.float64, device=dev) * 1e-12   # keeps U near its start
        plx = torch.empty(Lbig, Lbig, dtype=torch.float64, device=dev)
        gauge_kernels = {
            "krnl_force": kernel_gbs(lambda: qed2d.krnl_force_(frc1, frc2, Ub, pb), B_KRNL_FORCE),
            "updt_fld": kernel_gbs(lambda: qed2d.updt_fld_(Ub, mom, 1.0), B_UPDT_FLD),
            "tr_dQwdU": kernel_gbs(lambda: qed2d.tr_dQwdU(frc1, Ub, si, so, pb), B_TR_DQWDU),
            "plaquette_field": kernel_gbs(lambda: qed2d.plaquette_(plx, Ub, pb), B_PLAQ_FIELD),
            # two steps per call (an even number of fused update+kick passes: no copy back), per step
            "omf4_step_pure_gauge": kernel_gbs(lambda: qed2d.OMF4_(mom, Ub, 1e-3, 2, pb, None), 2 * B_OMF4_STEP),
            "bytes_per_site": {"krnl_force": B_KRNL_FORCE, "updt_fld": B_UPDT_FLD, "tr_dQwdU": B_TR_DQWDU,
                               "plaquette_field": B_PLAQ_FIELD, "omf4_step_pure_gauge": B_OMF4_STEP},
        }
        gauge_kernels["omf4_step_pure_gauge"]["us"] /= 2   # per step
        del frc1, frc2, mom, plx
        qed2d.set_precision("mixed")
        xb = torch.zeros_like(si)
        cg_runs = []
        for _ in range(2):
            a0.record()
            try:
                qed2d.CG(xb, Ub, si, AM0, 60, TOL, qed2d.gamm5Dw_sqr_msq, pb, None)
            except qed2d.Qed2dError:
                pass
            a1.record()
            torch.cuda.synchronize()
            it, _, up = qed2d.last_solve(pb)
            cg_runs.append((a0.elapsed_time(a1) / 1e3, it, up))
        # FP32-inner vs FP64 solution at the reference's stop rule
        sols = {}
        for prec in ("mixed", "f64"):
            qed2d.set_precision(prec)
            xs_ = torch.zeros_like(si)
            qed2d.CG(xs_, Ub, si, AM0, MAXITER, TOL, qed2d.gamm5Dw_sqr_msq, pb, None)
            sols[prec] = (xs_, qed2d.last_solve(pb))
        sol_err = float(((sols["mixed"][0] - sols["f64"][0]).abs().max() / sols["f64"][0].abs().max()).item())
        sol_its = {k: v[1][0] for k, v in sols.items()}
        del sols
        qed2d.set_precision("f64")
        t_cg, it_cg, upd_cg = cg_runs[-1]
        cg_gbs = Vb * (B_MIXED_SETUP + it_cg * B_MIXED_ITER + upd_cg * B_MIXED_UPDATE) / t_cg / 1e9
        dslash = {"lattice": f"{Lbig}x{Lbig}", "g5dw_f64_GBs": f64_gbs, "g5dw_f64_frac": f64_gbs / peak,
                  "g5dw_f64_us": t_ap * 1e6, "g5dw_c64_GBs": c64_gbs, "g5dw_c64_frac": c64_gbs / peak,
                  "g5dw_c64_us": t_ap32 * 1e6, "g5dw_c64_vs_f64_rel_err": apply_err,
                  "cg_solution_mixed_vs_f64_rel_err": sol_err, "cg_solution_iterations": sol_its,
                  "cg_mixed_GBs": cg_gbs, "cg_mixed_frac": cg_gbs / peak,
                  "cg_mixed_iters": it_cg, "cg_mixed_updates": upd_cg, "gauge_kernels": gauge_kernels,
                  "peak_GBs": peak, "peak_kind": peak_kind}
        del Ub, si, so, xb
        torch.cuda.empty_cache()

    # --- throughput of the other benchmark configurations (C1, C2, C3, C5)
    configs = None if args.skip_configs else run_configs(qed2d, torch, dev)

    # --- CPU baseline: the oracle on the host cores, bounded sample
    cpu = None
    if not args.skip_cpu:
        from oracle import oracle as O
        Uc = oracle_thermalised_field()
        o = O.Oracle(L, L, BETA)
        t_cpu, its_cpu = [], []
        for k in range(CPU_TRAJ):
            dt, Uc, it = oracle_trajectory(o, Uc, SEED, k)
            t_cpu.append(dt)
            its_cpu.append(it)
        cpu = {"value": CPU_TRAJ / sum(t_cpu), "unit": "traj/s", "cores": O.num_threads(), "kind": "port",
               "sample": f"the first {CPU_TRAJ} trajectories of replica chain 0 (the GPU arm's draws, "
                         f"{'/'.join(str(i) for i in its_cpu)} CG iterations) from the thermalised start, one chain"}

    line = {
        "metric": METRIC, "value": value, "unit": "traj/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": f"synthetic: seeded hot start thermalised by {THERM_TRAJ} pure-gauge trajectories, copied to "
                f"{B} replica chains with distinct seeds",
        "config": {"workload": WORKLOAD, "replicas_per_gpu": B, "L1": L, "L2": L, "beta": BETA, "m0": AM0, "ns": NS,
                   "eps": EPS, "cg_tol_sq": TOL,
                   "solver": "batched mixed FP32 inner / FP64 reliable updates, FP64 stop rule",
                   "step": f"one batched trajectory = {B} trajectories (one per replica chain)",
                   "l2": f"flushed between steps (256 MiB write); working set {B} x ~60 MB",
                   "parallelism": f"replicas x{world * B}"},
        "e2e": e2e,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": int(launches),
        "trajectories": {"cg_iterations_per_trajectory_mean": statistics.mean(i.cg_iterations for i in flat),
                         "accepted": sum(i.accepted for i in flat), "of": len(flat),
                         "dH_replica0": [round(st[0].dH, 6) for st in infos]},
        "baselines": None if not base else {
            "single_chain_mixed_traj_s": 1.0 / base["mixed"][0],
            "f64_fused_gpu_traj_s": 1.0 / base["f64"][0], "f64_fused_cg_iterations": base["f64"][1],
            "plain_f64_gpu_traj_s": 1.0 / base["plain"][0], "plain_f64_cg_iterations": base["plain"][1],
            "batched_vs_plain": value / world / (1.0 / base["plain"][0]),
            "batched_vs_f64_fused": value / world / (1.0 / base["f64"][0])},
        "dslash_hbm": dslash,
        "ensemble": ensemble,
        "configs": configs,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=4, help="replica chains per GPU advanced together")
    ap.add_argument("--skip-sweep", action="store_true", help="skip the 8192^2 Dslash bandwidth sweep")
    ap.add_argument("--skip-cpu", action="store_true", help="skip the oracle CPU baseline")
    ap.add_argument("--skip-ensemble", action="store_true", help="skip the 512-replica ensemble measurement")
    ap.add_argument("--skip-configs", action="store_true", help="skip the C1/C2/C3/C5 throughput measurements")
    ap.add_argument("--skip-baselines", action="store_true",
                    help="skip the plain-FP64 and fused-FP64 GPU trajectories")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
