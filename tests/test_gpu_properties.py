"""The reference's own assertions (test/*.jl) and force checks (tests/*.jl), run
on the GPU library through the C ABI at the reference's parameters."""
import numpy as np
import pytest

from helpers import bound, cgauss, hot_links, to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q():
    import qed2d
    yield qed2d
    qed2d.set_precision("f64")


def test_pf_generation_identity(q):
    """test/rhmc_pf_generation.jl:56-57: |sum xi^dag phi - sum X^dag X| < 1e-10."""
    L, beta, am0 = 10, 6.05, [0.02, 1.2]
    prm = q.LattParm((L, L), beta)
    U = to_dev(cgauss(L, L, 1234, 1))
    rp = q.get_rhmc_params([1, 1], [np.sqrt(0.1)] * 2, [np.sqrt(26.0)] * 2)
    hini = hfin = 0.0
    Fs = []
    for j, m in enumerate(am0):
        X = to_dev(cgauss(L, L, 1234, 10 + j))
        hini += float((X.abs() ** 2).sum())
        F = q.cfield(L, L)
        q.generate_pseudofermion_(F, U, X, m, 10000, 1e-25, prm, None, rp[j])
        Fs.append(F)
    for j, m in enumerate(am0):
        xi = q.cfield(L, L)
        q.MultiCG(xi, U, Fs[j], m, 10000, 1e-25, q.gamm5Dw_sqr_musq, rp[j], prm)
        hfin += float((xi.conj() * Fs[j]).sum().real)
    bound("abs(hfin - hini)", abs(hfin - hini), 1e-10)


def test_rhmc_force_vs_finite_difference(q):
    """test/rhmc_pf_forcetest.jl:92-93 (link (2,5,1), Deps = 1e-6)."""
    L, beta, am0 = 10, 6.05, 10.0
    prm = q.LattParm((L, L), beta)
    Uh = cgauss(L, L, 1234, 1)
    U = to_dev(Uh)
    q.seed(1234)
    lmin, lmax = q.power_method(U, am0, prm, None)
    rp = q.get_rhmc_params(5, np.sqrt(lmin), np.sqrt(lmax))
    X = to_dev(cgauss(L, L, 1234, 20))
    Sini = float((X.abs() ** 2).sum())
    F = q.cfield(L, L)
    q.generate_pseudofermion_(F, U, X, am0, 10000, 1e-25, prm, None, rp)
    frc, frc_i, G, Xi = q.rfield(L, L), q.rfield(L, L), q.cfield(L, L), q.cfield(L, L)
    for i in range(rp.n):
        q.CG(Xi, U, F, am0, rp.mu[i], 10000, 1e-25, q.gamm5Dw_sqr_musq, prm, None)
        q.gamm5Dw(G, U, Xi, am0, prm)
        q.tr_dQwdU(frc_i, U, Xi, G, prm)
        frc += rp.rho[i] * frc_i
    Frc_i = float(frc[0, 4, 1])
    Deps = 1e-6
    U2h = Uh.copy()
    U2h[0, 4, 1] *= complex(np.cos(Deps), np.sin(Deps))
    xi = q.cfield(L, L)
    q.MultiCG(xi, to_dev(U2h), F, am0, 10000, 1e-25, q.gamm5Dw_sqr_musq, rp, prm)
    Sfin = float((xi.conj() * F).sum().real)
    bound("abs(Frc_i + (Sfin - Sini) / Deps)", abs(Frc_i + (Sfin - Sini) / Deps), 1e-5)


@pytest.mark.parametrize("prec", ["f64", "plain"])
def test_rhmc_reversibility(q, prec):
    """test/rhmc_hmc_reversibility.jl:46-50: |Delta S_gauge| < 1e-10."""
    q.set_precision(prec)
    L, beta, am0 = 10, 6.05, [10.0]
    prm = q.LattParm((L, L), beta)
    U = to_dev(cgauss(L, L, 1234, 1))
    q.seed(1234)
    lmin, lmax = q.power_method(U, am0[0], prm, None)
    rp = q.get_rhmc_params([5], [np.sqrt(lmin)], [np.sqrt(lmax)])
    Sini = q.Action(U, prm)
    q.HMC_(U, am0, 0.01, 100, [], 10000, 1e-25, prm, None, rp, reversibility_test=True)
    bound("abs(q.Action(U, prm) - Sini)", abs(q.Action(U, prm) - Sini), 1e-10)
    q.set_precision("f64")


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_nf2_md_reversibility(q, prec):
    """Nf=2 leapfrog forward then with negated momenta back: the FP64 link and
    momentum masters return to the start (mixed: solves meet the FP64 residual)."""
    q.set_precision(prec)
    L, beta, am0 = 32, 4.0, 0.2
    prm = q.LattParm((L, L), beta)
    U0 = hot_links(L, L, 4)
    U = to_dev(U0)
    X = to_dev(cgauss(L, L, 8, 1))
    F = q.cfield(L, L)
    q.gamm5Dw(F, U, X, am0, prm)
    mom = to_dev(np.random.default_rng(3).standard_normal((2, L, L)))
    G, Y = q.cfield(L, L), q.cfield(L, L)
    q.leapfrog_(mom, U, Y, F, G, am0, 0.05, 20, 10000, 1e-26, prm, None)
    mom.neg_()
    q.leapfrog_(mom, U, Y, F, G, am0, 0.05, 20, 10000, 1e-26, prm, None)
    dS = abs(q.Action(U, prm) - q.Action(to_dev(U0), prm))
    assert dS < 1e-10
    q.set_precision("f64")


def test_gauge_and_nf2_force_vs_finite_difference(q):
    """tests/gauge_forcetest.jl and tests/fermion_forcetest.jl on the GPU."""
    L, beta, am0 = 12, 4.0, 0.5
    prm = q.LattParm((L, L), beta)
    Uh = hot_links(L, L, 9)
    U = to_dev(Uh)
    f1, f2 = q.rfield(L, L), q.rfield(L, L)
    q.krnl_force_(f1, f2, U, prm)
    F = q.cfield(L, L)
    q.gamm5Dw(F, U, to_dev(cgauss(L, L, 4, 1)), am0, prm)
    X, G, ff = q.cfield(L, L), q.cfield(L, L), q.rfield(L, L)
    q.CG(X, U, F, am0, 10000, 1e-28, q.gamm5Dw_sqr_msq, prm, None)
    q.gamm5Dw(G, U, X, am0, prm)
    q.tr_dQwdU(ff, U, X, G, prm)

    def S(Uc):
        Ud = to_dev(Uc)
        Y = q.cfield(L, L)
        q.CG(Y, Ud, F, am0, 10000, 1e-28, q.gamm5Dw_sqr_msq, prm, None)
        return q.Action(Ud, prm), float((F.conj() * Y).sum().real)

    for (i1, i2, mu) in ((0, 0, 0), (5, 7, 1), (11, 3, 0)):
        d = 1e-6
        Up, Um = Uh.copy(), Uh.copy()
        Up[mu, i2, i1] *= np.exp(1j * d)
        Um[mu, i2, i1] *= np.exp(-1j * d)
        (gp, fp), (gm, fm) = S(Up), S(Um)
        bound("abs(float((f1 + f2)[mu, i2, i1]) + (gp - gm) / (2 * d))", abs(float((f1 + f2)[mu, i2, i1]) + (gp - gm) / (2 * d)), 1e-7)
        bound("abs(float(ff[mu, i2, i1]) + (fp - fm) / (2 * d))", abs(float(ff[mu, i2, i1]) + (fp - fm) / (2 * d)), 1e-6 * max(1.0, abs((fp - fm) / (2 * d))))


@pytest.mark.slow
def test_zolotarev_bounds(q):
    """test/rhmc_zolovarev_bound.jl:42,65,84."""
    L, beta, am0 = 20, 5.0, 0.2
    prm = q.LattParm((L, L), beta)
    V = L * L
    U = to_dev(cgauss(L, L, 1234, 1))
    q.seed(4321)
    lmin, lmax = q.power_method(U, am0, prm, None, iter=10000)
    r_a, r_b = np.sqrt(lmin * 0.99), np.sqrt(lmax * 1.01)
    rp = q.get_rhmc_params(5, r_a, r_b)
    X = to_dev(cgauss(L, L, 1234, 3))
    F, tmp = q.cfield(L, L), q.cfield(L, L)
    q.R(F, U, X, am0, 10000, 1e-25, q.gamm5Dw_sqr_musq, rp, prm)
    tmp.copy_(F)
    q.R(F, U, tmp, am0, 10000, 1e-25, q.gamm5Dw_sqr_musq, rp, prm)
    Xf, t2 = q.cfield(L, L), q.cfield(L, L)
    q.gamm5Dw(t2, U, F, am0, prm)
    q.gamm5Dw(Xf, U, t2, am0, prm)
    d = rp.delta
    assert float((X - Xf).norm() / X.norm()) < d * (2 + d)
    rp10 = q.get_rhmc_params(10, r_a, r_b)
    tmp.copy_(X)
    Z = q.cfield(L, L)
    for p in range(1, 11):
        q.LuscherZ(Z, U, tmp, am0, 100000, 1e-25, rp10, prm)
        bound("abs(float((X.conj() * Z).sum().real))", abs(float((X.conj() * Z).sum().real)), 2 * V * (2 * rp10.delta) ** p)
        tmp.copy_(Z)
    for n in range(1, 11):
        r = q.get_rhmc_params(n, r_a, r_b)
        W = q.reweighting_factor(U, am0, 100000, 1e-25, prm, None, r)
        assert np.exp(-2 * V * r.delta) < W < np.exp(2 * V * r.delta)


def test_energy_sums_are_compensated(q):
    """The sums behind Action/Plaquette/Hamiltonian (and so Delta H) are
    compensated: at 2048^2 they equal the correctly rounded sum of the site terms
    (math.fsum) to within one ulp, where a plain FP64 sum drifts by many."""
    import math
    import torch
    L = 2048
    V = L * L   # a power of two: Plaquette * V is the raw sum
    rng = np.random.default_rng(5)
    U = np.exp(1j * 0.3 * rng.uniform(-1, 1, (2, L, L)))
    U1, U2 = U[0], U[1]
    P = (U1 * np.roll(U2, -1, axis=1)) * np.conj(np.roll(U1, -1, axis=0) * U2)
    exact = math.fsum(P.real.ravel().tolist())
    Ud = to_dev(U)
    got = q.Plaquette(Ud, q.LattParm((L, L), 4.0)) * V
    bound("abs(got - exact)", abs(got - exact), np.spacing(exact))  # (got - exact) / np.spacing(exact)
    mom = rng.normal(size=(2, L, L))
    exact_m = math.fsum((mom[0] ** 2 + mom[1] ** 2).ravel().tolist()) / 2
    H = q.Hamiltonian(torch.from_numpy(mom).cuda(), Ud, q.LattParm((L, L), 0.0))
    bound("abs(H - exact_m)", abs(H - exact_m), np.spacing(exact_m))  # (H - exact_m) / np.spacing(exact_m)
