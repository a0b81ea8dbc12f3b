"""Generate the golden fixtures in tests/golden/ (run: python tests/golden/make_golden.py).

The reference (Julia + CUDA.jl) cannot run here and ships no golden vectors, so
the fixtures come from a second, independent restatement of the reference
formulas written with NumPy array shifts (no code shared with the C oracle),
plus dense linear algebra and 50-digit mpmath arithmetic:

* ``kernels_<L1>x<L2>.npz`` -- seeded non-unitary random links (the reference's
  own tests use non-unitary Gaussian links, e.g. test/rhmc_pf_generation.jl:19)
  and spinors, with the outputs of gamm5Dw, Dw, gamm5Dw_sqr, gamm5Dw_sqr_musq,
  tr_dQwdU, plaquette!, qtop!, krnl_force!, updt_fld!, unfold/reflect and the
  exact solution of (g5 Dw)^2 x = b from a dense solve.
* ``zolotarev.json`` -- Zolotarev coefficients (src/QED2dRHMC.jl:1-121) with K,
  sn, cn evaluated by mpmath at 50 digits for several (n, r_a, r_b).
"""
import json
import os

import mpmath as mp
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def fwd(a, axis):
    """a(x + mu_hat) on arrays shaped (..., L2, L1): axis 1 -> i1, axis 2 -> i2."""
    return np.roll(a, -1, axis=-1 if axis == 1 else -2)


def bwd(a, axis):
    return np.roll(a, 1, axis=-1 if axis == 1 else -2)


def g5dw(U, s, m0):
    """src/QED2dDirac.jl:2-33 with array shifts."""
    U1, U2 = U[0], U[1]
    s1, s2 = s[0], s[1]
    s1p1, s2p1 = fwd(s1, 1), fwd(s2, 1)
    s1m1, s2m1 = bwd(s1, 1), bwd(s2, 1)
    s1p2, s2p2 = fwd(s1, 2), fwd(s2, 2)
    s1m2, s2m2 = bwd(s1, 2), bwd(s2, 2)
    U1m1, U2m2 = bwd(U1, 1), bwd(U2, 2)
    A = 0.5 * (U1 * (s1p1 - s2p1) + np.conj(U1m1) * (s1m1 + s2m1))
    B = 0.5 * (U2 * (s1p2 + 1j * s2p2) + np.conj(U2m2) * (s1m2 - 1j * s2m2))
    A2 = 0.5 * (U1 * (s1p1 - s2p1) - np.conj(U1m1) * (s1m1 + s2m1))
    B2 = 0.5 * (U2 * (-s2p2 + 1j * s1p2) - np.conj(U2m2) * (s2m2 + 1j * s1m2))
    return np.stack([(2.0 + m0) * s1 - A - B, -(2.0 + m0) * s2 - A2 - B2])


def plaq(U):
    U1, U2 = U[0], U[1]
    return U1 * fwd(U2, 1) * np.conj(fwd(U1, 2) * U2)


def gauge_force(U, beta):
    """krnl_force! (src/QED2dAction.jl:34-53): frc1 local, frc2 scattered."""
    v = beta * np.imag(plaq(U))
    f1 = np.stack([-v, v])
    f2 = np.stack([bwd(v, 2), bwd(-v, 1)])   # frc2[x+2,1] = v, frc2[x+1,2] = -v
    return f1, f2


def fermion_force(U, X, G):
    """tr_dQwdU (src/QED2dDirac.jl:172-199)."""
    U1, U2 = U[0], U[1]
    X1, X2, G1, G2 = X[0], X[1], G[0], G[1]
    z1 = (np.conj(U1) * (np.conj(fwd(X1, 1)) * (G1 + G2) - np.conj(fwd(X2, 1)) * (G1 + G2))
          - U1 * (np.conj(X1) * (fwd(G1, 1) - fwd(G2, 1)) + np.conj(X2) * (fwd(G1, 1) - fwd(G2, 1))))
    z2 = (np.conj(U2) * (np.conj(fwd(X1, 2)) * (G1 - 1j * G2) - np.conj(fwd(X2, 2)) * (1j * G1 + G2))
          - U2 * (np.conj(X1) * (fwd(G1, 2) + 1j * fwd(G2, 2)) + np.conj(X2) * (1j * fwd(G1, 2) - fwd(G2, 2))))
    return np.stack([np.real(1j * z1), np.real(1j * z2)])


def unfold(U, reflect):
    c = np.conj(U) if reflect else U
    top = np.concatenate([U, c], axis=2)
    bot = np.concatenate([c, U], axis=2)
    return np.concatenate([top, bot], axis=1)


def dense_operator(U, m0):
    _, L2, L1 = U.shape
    n = 2 * L1 * L2
    M = np.zeros((n, n), np.complex128)
    for j in range(n):
        e = np.zeros(n, np.complex128)
        e[j] = 1.0
        M[:, j] = g5dw(U, e.reshape(2, L2, L1), m0).ravel()
    return M


def kernels_fixture(L1, L2, seed):
    rng = np.random.default_rng(seed)
    cshape = (2, L2, L1)

    def cgauss():
        return (rng.standard_normal(cshape) + 1j * rng.standard_normal(cshape)) / np.sqrt(2.0)

    U = cgauss()
    Uu = np.exp(1j * rng.uniform(-np.pi, np.pi, cshape))     # unitary links as well
    si = cgauss()
    X = cgauss()
    mom = rng.standard_normal(cshape)
    m0, mu, beta, eps = 0.3, 0.7, 4.0, 0.13
    out = dict(L1=L1, L2=L2, m0=m0, mu=mu, beta=beta, eps=eps, U=U, Uu=Uu, si=si, X=X, mom=mom)
    out["g5dw"] = g5dw(U, si, m0)
    g = g5dw(U, si, m0)
    out["dw"] = np.stack([g[0], -g[1]])
    out["g5dw_sqr"] = g5dw(U, g, m0)
    out["g5dw_sqr_musq"] = out["g5dw_sqr"] + mu * mu * si
    G = g5dw(U, X, m0)
    out["g5dw_X"] = G
    out["fermion_force"] = fermion_force(U, X, G)
    out["plaq_field"] = np.real(plaq(Uu))
    out["qtop_field"] = np.angle(plaq(Uu))
    f1, f2 = gauge_force(Uu, beta)
    out["frc1"], out["frc2"] = f1, f2
    out["update_links"] = np.exp(1j * eps * mom) * Uu
    out["unfold"] = unfold(Uu, False)
    out["reflect"] = unfold(Uu, True)
    M = dense_operator(U, m0)
    A = M @ M
    out["cg_solution"] = np.linalg.solve(A, si.ravel()).reshape(cshape)
    out["cg_solution_musq"] = np.linalg.solve(A + mu * mu * np.eye(A.shape[0]), si.ravel()).reshape(cshape)
    ev = np.linalg.eigvalsh(A)
    out["eig_min"], out["eig_max"] = ev[0], ev[-1]
    Mu = dense_operator(Uu, m0)
    evu = np.linalg.eigvalsh(Mu @ Mu)
    out["eig_min_unitary"], out["eig_max_unitary"] = evu[0], evu[-1]
    out["action_unitary"] = beta * (L1 * L2 - np.sum(np.real(plaq(Uu))))
    return out


def zolo_mp(n, r_a, r_b):
    """src/QED2dRHMC.jl:1-121 in 50-digit arithmetic (m = k^2 parameter)."""
    mp.mp.dps = 50
    r_a, r_b = mp.mpf(r_a), mp.mpf(r_b)
    eps = (r_a / r_b) ** 2
    k = mp.sqrt(1 - eps)
    m = k ** 2
    v = mp.ellipk(m) / (2 * n + 1)

    def sn(u):
        return mp.ellipfun("sn", u, m=m)

    def cn(u):
        return mp.ellipfun("cn", u, m=m)

    def a_r(r):
        return cn(r * v) ** 2 / sn(r * v) ** 2

    def c_r(r):
        return sn(r * v) ** 2

    mu = [r_b * mp.sqrt(a_r(2 * j)) for j in range(1, n + 1)]
    nu = [r_b * mp.sqrt(a_r(2 * j - 1)) for j in range(1, n + 1)]
    rho = []
    for j in range(n):
        res = nu[j] ** 2 - mu[j] ** 2
        for mm in range(n):
            if mm != j:
                res *= (nu[mm] ** 2 - mu[j] ** 2) / (mu[mm] ** 2 - mu[j] ** 2)
        rho.append(res)
    d = k ** (2 * n + 1)
    for i in range(1, 2 * n + 2, 2):
        d *= c_r(i) ** 2
    delta = d ** 2 / (1 + mp.sqrt(1 - d ** 2)) ** 2
    A = 2 / (1 + mp.sqrt(1 - d ** 2))
    for i in range(1, 2 * n, 2):
        A *= c_r(i)
    for i in range(2, 2 * n + 1, 2):
        A /= c_r(i)
    f = lambda xs: [float(x) for x in xs]
    return dict(n=n, r_a=float(r_a), r_b=float(r_b), eps=float(eps), A=float(A), delta=float(delta),
                mu=f(mu), nu=f(nu), rho=f(rho))


def elliptic_points():
    mp.mp.dps = 50
    pts = []
    for m in (0.1, 0.5, 0.9, 0.99, 0.9999, 1 - 1e-6):
        K = mp.ellipk(m)
        for frac in (0.05, 0.3, 0.7, 0.95):
            u = frac * K
            pts.append(dict(m=m, u=float(u), K=float(K), sn=float(mp.ellipfun("sn", u, m=m)),
                            cn=float(mp.ellipfun("cn", u, m=m))))
    return pts


def main():
    for (L1, L2, seed) in ((6, 4, 11), (5, 7, 12)):
        fx = kernels_fixture(L1, L2, seed)
        np.savez_compressed(os.path.join(HERE, f"kernels_{L1}x{L2}.npz"), **fx)
    zs = [zolo_mp(n, ra, rb) for (n, ra, rb) in (
        (1, 0.1 ** 0.5, 26 ** 0.5), (5, 0.1 ** 0.5, 26 ** 0.5), (4, 0.05 ** 0.5, 20 ** 0.5),
        (12, 0.01 ** 0.5, 30.0 ** 0.5), (10, 0.3, 4.0))]
    with open(os.path.join(HERE, "zolotarev.json"), "w") as fh:
        json.dump(dict(zolotarev=zs, elliptic=elliptic_points()), fh, indent=1)


if __name__ == "__main__":
    main()
