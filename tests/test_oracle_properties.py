"""The reference's own assertions (test/*.jl) and force-vs-finite-difference
checks (tests/*.jl), run on the CPU oracle at the reference's parameters.  The
same properties are checked on the GPU in test_gpu_properties.py."""
import numpy as np
import pytest

from oracle.oracle import Oracle, zolotarev


def cgauss(L1, L2, seed, stream):
    """(randn + i randn)/sqrt(2) on an L1 x L2 lattice, from the shared Philox stream."""
    z = Oracle.normal(4 * L1 * L2, seed, stream, 0)
    return ((z[0::2] + 1j * z[1::2]) / np.sqrt(2.0)).reshape(2, L2, L1)


def test_pf_generation_identity():
    """test/rhmc_pf_generation.jl: |sum xi^dag phi - sum X^dag X| < 1e-10."""
    L, beta = 10, 6.05
    am0 = [0.02, 1.2]
    o = Oracle(L, L, beta)
    U = cgauss(L, L, 1234, 1)
    rprm = [zolotarev(1, np.sqrt(0.1), np.sqrt(26.0)) for _ in am0]
    hini = hfin = 0.0
    Fs = []
    for j, m in enumerate(am0):
        X = cgauss(L, L, 1234, 10 + j)
        hini += np.vdot(X, X).real
        st, F, _ = o.pf_generate(U, X, m, 10000, 1e-25, rprm[j])
        assert st == 0
        Fs.append(F)
    for j, m in enumerate(am0):
        st, xi, _ = o.multi_cg(U, Fs[j], m, 10000, 1e-25, rprm[j])
        assert st == 0
        hfin += np.vdot(xi, Fs[j]).real
    assert abs(hfin - hini) < 1e-10


def rhmc_force_fd(o, U, am0, rprm, link, seed):
    """test/rhmc_pf_forcetest.jl:84-143 on the oracle."""
    X = cgauss(o.L1, o.L2, seed, 20)
    Sini = np.vdot(X, X).real
    st, F, _ = o.pf_generate(U, X, am0, 10000, 1e-25, rprm)
    assert st == 0
    frc = np.zeros((2, o.L2, o.L1))
    for i in range(rprm.n):
        st, Xi, _, _ = o.cg(U, F, am0, 10000, 1e-25, mu=rprm.mu[i])
        assert st == 0
        g5DX = o.g5dw(U, Xi, am0)
        frc = frc + rprm.rho[i] * o.fermion_force(U, Xi, g5DX)
    i1, i2, mu = link
    Deps = 1e-6
    U2 = U.copy()
    U2[mu, i2, i1] = complex(np.cos(Deps), np.sin(Deps)) * U2[mu, i2, i1]
    st, xi, _ = o.multi_cg(U2, F, am0, 10000, 1e-25, rprm)
    Sfin = np.vdot(xi, F).real
    return frc[mu, i2, i1], (Sfin - Sini) / Deps


def test_rhmc_force_vs_finite_difference():
    """test/rhmc_pf_forcetest.jl: |F_analytic + dS/dtheta| < 1e-5 at link (2,5,1)."""
    L, beta, am0 = 10, 6.05, 10.0
    o = Oracle(L, L, beta)
    U = cgauss(L, L, 1234, 1)
    lmin, lmax = o.power_method(U, am0, 1000, cgauss(L, L, 1234, 2))
    rprm = zolotarev(5, np.sqrt(lmin), np.sqrt(lmax))
    fa, fn = rhmc_force_fd(o, U, am0, rprm, (1, 4, 0), 1234)
    assert abs(fa + fn) < 1e-5


def test_rhmc_reversibility():
    """test/rhmc_hmc_reversibility.jl: |Delta S_gauge| < 1e-10 after MD forward + backward."""
    L, beta, am0 = 10, 6.05, [10.0]
    o = Oracle(L, L, beta)
    U = cgauss(L, L, 1234, 1)
    lmin, lmax = o.power_method(U, am0[0], 1000, cgauss(L, L, 1234, 2))
    rprm = [zolotarev(5, np.sqrt(lmin), np.sqrt(lmax))]
    Sini = o.action(U)
    mom0 = Oracle.normal(2 * L * L, 1234, 3, 0).reshape(2, L, L)
    noise = [cgauss(L, L, 1234, 30)]
    st, U2, acc, hi, hf, _ = o.hmc_rhmc(U, am0, 0.01, 100, 10000, 1e-25, rprm, mom0, noise, 0.5,
                                         reversibility=True)
    assert st == 0
    assert abs(o.action(U2) - Sini) < 1e-10


def test_nf2_force_vs_finite_difference():
    """tests/fermion_forcetest.jl: Nf=2 force tr_dQwdU against dS/dtheta of
    S = F^dag ((g5Dw)^2)^-1 F."""
    L, beta, am0 = 8, 4.0, 0.5
    o = Oracle(L, L, beta)
    rng = np.random.default_rng(7)
    U = np.exp(1j * rng.uniform(-np.pi, np.pi, (2, L, L)))
    F = o.g5dw(U, cgauss(L, L, 99, 1), am0)

    def S(Uc):
        st, X, _, _ = o.cg(Uc, F, am0, 10000, 1e-28)
        return np.vdot(F, X).real, X

    S0, X = S(U)
    frc = o.fermion_force(U, X, o.g5dw(U, X, am0))
    for (i1, i2, mu) in ((0, 0, 0), (3, 5, 1), (7, 2, 0)):
        d = 1e-6
        Up, Um = U.copy(), U.copy()
        Up[mu, i2, i1] *= np.exp(1j * d)
        Um[mu, i2, i1] *= np.exp(-1j * d)
        fd = (S(Up)[0] - S(Um)[0]) / (2 * d)
        assert abs(frc[mu, i2, i1] + fd) < 1e-6 * max(1.0, abs(fd))


def test_gauge_force_vs_finite_difference():
    """tests/gauge_forcetest.jl: krnl_force! frc1+frc2 against -dS_gauge/dtheta."""
    L, beta = 6, 4.0
    o = Oracle(L, L + 2, beta)
    rng = np.random.default_rng(5)
    U = np.exp(1j * rng.uniform(-np.pi, np.pi, (2, L + 2, L)))
    f1, f2 = o.gauge_force(U)
    f = f1 + f2
    for (i1, i2, mu) in ((0, 0, 0), (5, 7, 1), (2, 3, 0), (4, 1, 1)):
        d = 1e-6
        Up, Um = U.copy(), U.copy()
        Up[mu, i2, i1] *= np.exp(1j * d)
        Um[mu, i2, i1] *= np.exp(-1j * d)
        fd = (o.action(Up) - o.action(Um)) / (2 * d)
        assert abs(f[mu, i2, i1] + fd) < 1e-7


@pytest.mark.slow
def test_zolotarev_bounds():
    """test/rhmc_zolovarev_bound.jl: the delta bound of R, the Z^p bound and the
    W_1 bound (Luscher, hep-lat/0406022, eqs. 4.3-4.6)."""
    L, beta, am0 = 20, 5.0, 0.2
    o = Oracle(L, L, beta)
    V = L * L
    U = cgauss(L, L, 1234, 1)
    lmin, lmax = o.power_method(U, am0, 10000, cgauss(L, L, 1234, 2))
    r_a, r_b = np.sqrt(lmin * 0.99), np.sqrt(lmax * 1.01)
    rprm = zolotarev(5, r_a, r_b)
    X = cgauss(L, L, 1234, 3)
    st, F, _ = o.rational(U, X, am0, 10000, 1e-25, rprm)
    st, F, _ = o.rational(U, F, am0, 10000, 1e-25, rprm)
    Xf = o.g5dw(U, o.g5dw(U, F, am0), am0)
    dX = np.linalg.norm(X - Xf) / np.linalg.norm(X)
    d = rprm.delta
    assert dX < d * (2 + d)
    rprm10 = zolotarev(10, r_a, r_b)
    tmp = X.copy()
    for p in range(1, 11):
        st, Z = o.luscher_z(U, tmp, am0, 100000, 1e-25, rprm10)
        assert st == 0
        assert abs(np.vdot(X, Z).real) < 2 * V * (2 * rprm10.delta) ** p
        tmp = Z
    for n in range(1, 11):
        r = zolotarev(n, r_a, r_b)
        st, W = o.reweighting_factor(U, am0, 100000, 1e-25, r, cgauss(L, L, 1234, 40 + n)[None])
        assert st == 0
        assert np.exp(-2 * V * r.delta) < W < np.exp(2 * V * r.delta)
