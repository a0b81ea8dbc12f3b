"""GPU parity of the integrators and HMC steps against the CPU oracle.  The
library draws momenta, pseudofermion noise and the Metropolis uniform from
Philox streams (seed, stream, counter); the same draws are replayed into the
oracle, so both run the same trajectory.  Tolerances (each about 10x the error
measured on a B200, recorded through helpers.bound): final links 1e-12 to 1e-13
relative, H_ini 1e-14 relative, Delta H 5e-11 to 1e-10 absolute, identical
accept/reject, CG iteration counts within one per solve."""
import numpy as np
import pytest

from helpers import bound, cgauss, hot_links, rel, to_dev, to_host
from oracle.oracle import LEAPFROG as O_LEAPFROG, OMF4 as O_OMF4, Oracle, zolotarev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q():
    import qed2d
    yield qed2d
    qed2d.set_precision("f64")


def draws(L1, L2, seed, ctr, nf=1):
    mom0 = Oracle.normal(2 * L1 * L2, seed, 1, ctr).reshape(2, L2, L1)
    noise = [cgauss(L1, L2, seed, 16 + j, ctr) for j in range(nf)]
    return mom0, noise, Oracle.uniform(seed, 3, ctr)


@pytest.mark.parametrize("integ", ["omf4", "leapfrog"])
def test_hmc_gauge(q, integ):
    L1, L2, beta = 128, 96, 11.25
    prm = q.LattParm((L1, L2), beta)
    o = Oracle(L1, L2, beta)
    U0 = hot_links(L1, L2, 1)
    Ud = to_dev(U0)
    q.seed(1234)
    Uo = U0
    for t in range(3):
        acc = []
        integrator = q.OMF4() if integ == "omf4" else q.Leapfrog()
        info = q.HMC_(Ud, 0.05, 10, acc, prm, None, integrator=integrator)
        mom0, _, u = draws(L1, L2, 1234, info.counter)
        st, Uo, acco, hi, hf = o.hmc_gauge(Uo, 0.05, 10, mom0, u,
                                            integrator=O_OMF4 if integ == "omf4" else O_LEAPFROG)
        bound("HMC! gauge H_ini rel vs oracle", abs(info.hini - hi) / abs(hi), 1e-14)
        bound("HMC! gauge dH abs vs oracle", abs(info.dH - (hf - hi)), 2e-9)
        assert info.accepted == acco == acc[0]
        bound("HMC! gauge links vs oracle", rel(to_host(Ud), Uo), 1e-12)
        bound("HMC! gauge Qtop abs vs oracle", abs(info.qtop - o.qtop(Uo)), 1e-12)


def test_omf4_gauge_reversible(q):
    L = 64
    prm = q.LattParm((L, L), 4.0)
    U0 = hot_links(L, L, 2)
    Ud = to_dev(U0)
    mom = to_dev(np.random.default_rng(1).standard_normal((2, L, L)))
    q.OMF4_(mom, Ud, 0.1, 10, prm, None)
    mom.neg_()
    q.OMF4_(mom, Ud, 0.1, 10, prm, None)
    bound("OMF4! gauge reversibility (links)", rel(to_host(Ud), U0), 1e-13)


@pytest.mark.parametrize("integ", ["leapfrog", "omf4"])
def test_hmc_nf2(q, integ):
    q.set_precision("f64")
    L1, L2, beta, am0 = 32, 24, 4.0, 0.3
    prm = q.LattParm((L1, L2), beta)
    o = Oracle(L1, L2, beta)
    U0 = hot_links(L1, L2, 3)
    Ud = to_dev(U0)
    q.seed(99)
    acc = []
    ns = 6 if integ == "leapfrog" else 2
    integrator = q.Leapfrog() if integ == "leapfrog" else q.OMF4()
    info = q.HMC_(Ud, am0, 0.1, ns, acc, 10000, 1e-24, prm, None, integrator=integrator)
    mom0, noise, u = draws(L1, L2, 99, info.counter)
    st, Uo, acco, hi, hf, ito = o.hmc_nf2(U0, am0, 0.1, ns, 10000, 1e-24, mom0, noise[0], u,
                                           integrator=O_LEAPFROG if integ == "leapfrog" else O_OMF4)
    assert st == 0
    bound(f"HMC! Nf=2 {integ} H_ini rel vs oracle", abs(info.hini - hi) / abs(hi), 1e-14)
    bound(f"HMC! Nf=2 {integ} dH abs vs oracle", abs(info.dH - (hf - hi)), 5e-11)
    assert info.accepted == acco
    bound(f"HMC! Nf=2 {integ} links vs oracle", rel(to_host(Ud), Uo), 1e-13)
    # one iteration of slack per solve (ns+1 solves, 6 per step for OMF4)
    bound(f"HMC! Nf=2 {integ} CG iterations vs oracle", abs(info.cg_iterations - ito),
          (ns + 1) * (6 if integ == "omf4" else 1))


def test_hmc_nf2_mixed_matches_f64(q):
    """The mixed FP32/FP64 solver reproduces the FP64 trajectory: every solve
    meets the same FP64 residual, so Delta H agrees to ~1e-8."""
    L, beta, am0 = 64, 4.0, 0.2
    prm = q.LattParm((L, L), beta)
    U0 = hot_links(L, L, 8)
    res = {}
    for prec in ("f64", "mixed"):
        q.set_precision(prec)
        Ud = to_dev(U0)
        q.seed(5)
        info = q.HMC_(Ud, am0, 0.05, 10, [], 10000, 1e-24, prm, None)
        res[prec] = (info, to_host(Ud))
    q.set_precision("f64")
    bound("HMC! Nf=2 mixed vs f64 dH abs", abs(res["f64"][0].dH - res["mixed"][0].dH), 1e-10)
    bound("HMC! Nf=2 mixed vs f64 links", rel(res["mixed"][1], res["f64"][1]), 1e-12)
    assert res["f64"][0].accepted == res["mixed"][0].accepted


@pytest.mark.parametrize("prec", ["f64", "plain"])
def test_hmc_rhmc(q, prec):
    q.set_precision(prec)
    L, beta = 12, 6.05
    am0 = [0.6, 1.2]
    prm = q.LattParm((L, L), beta)
    o = Oracle(L, L, beta)
    U0 = hot_links(L, L, 6)
    rp = [q.get_rhmc_params(4, np.sqrt(0.1), np.sqrt(26.0)) for _ in am0]
    ro = [zolotarev(4, np.sqrt(0.1), np.sqrt(26.0)) for _ in am0]
    Ud = to_dev(U0)
    q.seed(31)
    info = q.HMC_(Ud, am0, 0.1, 5, [], 10000, 1e-24, prm, None, rp)
    mom0, noise, u = draws(L, L, 31, info.counter, nf=2)
    st, Uo, acco, hi, hf, _ = o.hmc_rhmc(U0, am0, 0.1, 5, 10000, 1e-24, ro, mom0, noise, u)
    assert st == 0
    bound(f"HMC! RHMC {prec} H_ini rel vs oracle", abs(info.hini - hi) / abs(hi), 1e-14)
    bound(f"HMC! RHMC {prec} dH abs vs oracle", abs(info.dH - (hf - hi)), 5e-11)
    assert info.accepted == acco
    bound(f"HMC! RHMC {prec} links vs oracle", rel(to_host(Ud), Uo), 1e-12)
    q.set_precision("f64")


def test_leapfrog_and_update_momenta_api(q):
    """leapfrog!/update_momenta! called directly (src/QED2dHMC.jl:426-481)."""
    q.set_precision("f64")
    L, beta, am0 = 24, 4.0, 0.4
    prm = q.LattParm((L, L), beta)
    o = Oracle(L, L, beta)
    U0 = hot_links(L, L, 12)
    X0 = cgauss(L, L, 3, 5)
    F0 = o.g5dw(U0, X0, am0)
    mom0 = np.random.default_rng(2).standard_normal((2, L, L))
    Ud, mom, X, F, G = to_dev(U0), to_dev(mom0), q.cfield(L, L), to_dev(F0), q.cfield(L, L)
    q.leapfrog_(mom, Ud, X, F, G, am0, 0.1, 4, 10000, 1e-24, prm, None)
    import ctypes as C
    from oracle.oracle import _p
    Uo, momo, Xo, Go = U0.copy(), mom0.copy(), o.cfield(), o.cfield()
    it = C.c_int(0)
    st = o.L.o_leapfrog_nf2(o._pp, _p(momo), _p(Uo), _p(Xo), _p(F0), _p(Go), am0, 0.1, 4, 10000, 1e-24,
                            C.byref(it))
    assert st == 0
    bound("leapfrog! links vs oracle", rel(to_host(Ud), Uo), 1e-12)
    bound("leapfrog! momenta vs oracle", rel(to_host(mom), momo), 1e-12)
    bound("leapfrog! X vs oracle", rel(to_host(X), Xo), 1e-12)
    bound("leapfrog! g5Dw X vs oracle", rel(to_host(G), Go), 1e-12)
