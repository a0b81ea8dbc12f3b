"""Parity cases at the sizes of the benchmark configurations.

* Nf=1 RHMC at 128x128 with 12 Zolotarev poles on [lambda_min, lambda_max] from
  the power method (src/QED2dHMC.jl:116-195, test/rhmc_pf_forcetest.jl:29-32):
  one trajectory against the oracle replaying the same draws.
* Master field at 8192x8192 built the reference's way (main/master_field.jl:
  148-167: thermalise a small lattice, unfold it 2x2 repeatedly): checked through
  size-independent properties -- OMF4 reversibility of the FP64 link and momentum
  masters, a finite small Delta H, and Sum arg P / 2 pi equal to an integer.
* Nf=2 at 64x64 with the mixed solver against the FP64 path and the oracle."""
import numpy as np
import pytest

from helpers import bound, cgauss, hot_links, rel, to_dev, to_host
from oracle.oracle import Oracle, zolotarev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q():
    import qed2d
    yield qed2d
    qed2d.set_precision("f64")


def test_rhmc_128_twelve_poles_vs_oracle(q):
    L, beta, am0 = 128, 4.0, [0.3]
    prm = q.LattParm((L, L), beta)
    o = Oracle(L, L, beta)
    U0 = hot_links(L, L, 77)
    Ud = to_dev(U0)
    q.seed(5)
    lmin, lmax = q.power_method(Ud, am0[0], prm, None, iter=300)
    rp = [q.get_rhmc_params(12, np.sqrt(0.9 * lmin), np.sqrt(1.1 * lmax))]
    ro = [zolotarev(12, np.sqrt(0.9 * lmin), np.sqrt(1.1 * lmax))]
    info = q.HMC_(Ud, am0, 0.05, 4, [], 20000, 1e-24, prm, None, rp)
    ctr = info.counter
    mom0 = Oracle.normal(2 * L * L, 5, 1, ctr).reshape(2, L, L)
    noise = [cgauss(L, L, 5, 16, ctr)]
    st, Uo, acc, hi, hf, _ = o.hmc_rhmc(U0, am0, 0.05, 4, 20000, 1e-24, ro, mom0, noise, Oracle.uniform(5, 3, ctr))
    assert st == 0
    bound("RHMC 128^2 x 12 poles H_ini rel vs oracle", abs(info.hini - hi) / abs(hi), 1e-14)
    bound("RHMC 128^2 x 12 poles dH abs vs oracle", abs(info.dH - (hf - hi)), 1e-10)
    assert info.accepted == acc
    bound("RHMC 128^2 x 12 poles links vs oracle", rel(to_host(Ud), Uo), 1e-12)


def test_master_field_8192(q):
    import torch
    beta = 11.25
    L = 16
    U = torch.ones((2, L, L), dtype=torch.complex128, device="cuda")
    q.seed(1234)
    while True:
        prm = q.LattParm((L, L), beta)
        for _ in range(3):
            q.HMC_(U, 0.1, 10, [], prm, None)
        if L == 8192:
            break
        U = q.unfold_fld_(U, prm)
        L *= 2
    prm = q.LattParm((L, L), beta)
    # integer topological charge of the unfolded field
    Q = q.Qtop(U, prm)
    bound("master field 8192^2 |Q - round(Q)|", abs(Q - round(Q)), 1e-12)
    # OMF4 reversibility at 8192^2 (ns=20, eps=0.025 as the master-field config)
    U0 = U.clone()
    mom = torch.randn((2, L, L), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    H0 = q.Hamiltonian(mom, U, prm)
    q.OMF4_(mom, U, 0.025, 20, prm, None)
    H1 = q.Hamiltonian(mom, U, prm)
    bound("master field 8192^2 OMF4 |H1 - H0| (energy error, not parity)", abs(H1 - H0), 0.5)
    mom.neg_()
    q.OMF4_(mom, U, 0.025, 20, prm, None)
    bound("master field 8192^2 reversibility max |U - U0|", float((U - U0).abs().max()), 1e-11)
    bound("master field 8192^2 reversibility |H - H0| / |H0|", abs(q.Hamiltonian(mom, U, prm) - H0) / abs(H0), 1e-12)


def test_nf2_64_mixed_vs_f64_and_oracle(q):
    L, beta, am0 = 64, 4.0, 0.1
    prm = q.LattParm((L, L), beta)
    U0 = hot_links(L, L, 31)
    out = {}
    for prec in ("f64", "mixed"):
        q.set_precision(prec)
        Ud = to_dev(U0)
        q.seed(64)
        out[prec] = (q.HMC_(Ud, am0, 0.05, 20, [], 20000, 1e-24, prm, None), to_host(Ud))
    q.set_precision("f64")
    info = out["f64"][0]
    o = Oracle(L, L, beta)
    mom0 = Oracle.normal(2 * L * L, 64, 1, info.counter).reshape(2, L, L)
    noise = cgauss(L, L, 64, 16, info.counter)
    st, Uo, acc, hi, hf, _ = o.hmc_nf2(U0, am0, 0.05, 20, 20000, 1e-24, mom0, noise,
                                        Oracle.uniform(64, 3, info.counter))
    assert st == 0
    for prec in ("f64", "mixed"):
        i, Uh = out[prec]
        bound(f"Nf=2 64^2 {prec} dH abs vs oracle", abs(i.dH - (hf - hi)), 5e-10)  # prec
        assert i.accepted == acc, prec
        bound(f"Nf=2 64^2 {prec} links vs oracle", rel(Uh, Uo), 5e-12)  # prec


def test_ensemble_512_ragged_replicas(q):
    """512 Nf=2 replicas with sizes drawn from {32, 48, 64, 96, 128, 256}^2, beta in
    [2, 6], m0 in [0.05, 0.3], hot starts, leapfrog ns=10 eps=0.1: one batched
    trajectory, then one replica of each size (and the last one) against the
    single-lattice mixed path."""
    from qed2d.cases import ensemble_config, hot_batch_field
    n = 512
    sizes, betas, am0s = ensemble_config(n, 2024)
    seeds = [9000 + r for r in range(n)]
    counter = 1
    b = q.Batch.ragged(sizes, betas)
    U = hot_batch_field(b, 2024)
    U0 = U.clone()
    infos = b.hmc_nf2(U, am0s, 0.1, 10, 20000, 1e-24, seeds, counter)
    assert all(np.isfinite(i.dH) for i in infos)
    picks = sorted({sizes.index(s) for s in set(sizes)} | {n - 1})
    q.set_precision("mixed")
    for r in picks:
        prm = q.LattParm(sizes[r], betas[r])
        Ud = b.replica(U0, r).clone()
        q.seed(seeds[r])
        single = q.HMC_(Ud, am0s[r], 0.1, 10, [], 20000, 1e-24, prm, None, counter=counter)
        bound("512-replica ensemble vs single-lattice dH abs", abs(single.dH - infos[r].dH), 1e-10)  # r
        assert single.accepted == infos[r].accepted, r
        bound("512-replica ensemble vs single-lattice links", rel(to_host(b.replica(U, r)), to_host(Ud)), 5e-12)  # r
    q.set_precision("f64")
