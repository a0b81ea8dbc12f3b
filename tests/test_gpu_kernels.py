"""GPU parity of the site kernels and observables, called through the C ABI
(libqed2d via the qed2d host mirror), against the golden fixtures and the CPU
oracle.  Tolerances (each about 10x the error measured on a B200, recorded
through helpers.bound): FP64 site kernels 1e-15 to 2e-15 relative (only the
order of floating-point operations differs); energies 1e-14 to 1e-15 relative;
the complex64 apply 5e-7 against the FP64 apply of the same inputs; the
rounded topological charge is exact."""
import os

import numpy as np
import pytest

from helpers import bound, cgauss, hot_links, rel, to_dev, to_host
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def q():
    import qed2d
    return qed2d


def load(tag):
    return dict(np.load(os.path.join(GOLD, f"kernels_{tag}.npz")))


@pytest.mark.parametrize("tag", ["6x4", "5x7"])
def test_kernels_golden(q, tag):
    import torch
    g = load(tag)
    L1, L2 = int(g["L1"]), int(g["L2"])
    prm = q.LattParm((L1, L2), float(g["beta"]))
    m0, mu = float(g["m0"]), float(g["mu"])
    U, si, X = to_dev(g["U"]), to_dev(g["si"]), to_dev(g["X"])
    so = q.cfield(L1, L2)
    q.gamm5Dw(so, U, si, m0, prm)
    bound("g5dw vs golden", rel(to_host(so), g["g5dw"]), 1e-15)
    q.Dw(so, U, si, m0, prm)
    bound("Dw vs golden", rel(to_host(so), g["dw"]), 1e-15)
    q.gamm5Dw_sqr(so, U, si, m0, prm)
    bound("g5dw_sqr vs golden", rel(to_host(so), g["g5dw_sqr"]), 1e-15)
    q.gamm5Dw_sqr_musq(so, None, U, si, m0, mu, prm)
    bound("g5dw_sqr_musq vs golden", rel(to_host(so), g["g5dw_sqr_musq"]), 1e-15)
    G = q.cfield(L1, L2)
    q.gamm5Dw(G, U, X, m0, prm)
    frc = q.rfield(L1, L2)
    q.tr_dQwdU(frc, U, X, G, prm)
    bound("tr_dQwdU vs golden", rel(to_host(frc), g["fermion_force"]), 2e-15)
    Uu = to_dev(g["Uu"])
    plx = torch.zeros((L2, L1), dtype=torch.float64, device="cuda")
    q.plaquette_(plx, Uu, prm)
    bound("plaquette! vs golden", rel(to_host(plx), g["plaq_field"]), 1e-15)
    q.qtop_(plx, Uu, prm)
    bound("qtop! vs golden", rel(to_host(plx), g["qtop_field"]), 1e-15)
    f1, f2 = q.rfield(L1, L2), q.rfield(L1, L2)
    q.krnl_force_(f1, f2, Uu, prm)
    bound("krnl_force! frc1 vs golden", rel(to_host(f1), g["frc1"]), 1e-15)
    bound("krnl_force! frc2 vs golden", rel(to_host(f2), g["frc2"]), 1e-15)
    U2 = Uu.clone()
    q.updt_fld_(U2, to_dev(g["mom"]), float(g["eps"]))
    bound("updt_fld! vs golden", rel(to_host(U2), g["update_links"]), 1e-15)
    assert np.array_equal(to_host(q.unfold_fld_(Uu, prm)), g["unfold"])
    assert np.array_equal(to_host(q.unfold_reflect_(Uu, prm)), g["reflect"])
    bound("Action rel vs golden", abs(q.Action(Uu, prm) - float(g["action_unitary"])) / abs(float(g["action_unitary"])),
          1e-14)


def test_free_field_eigenvalue(q):
    """Known answer of tests/Dw-eigenvalues.jl: D plane wave = lambda plane wave."""
    L, am0 = 20, 10.0
    prm = q.LattParm((L, L), 6.05)
    import torch
    U = torch.ones((2, L, L), dtype=torch.complex128, device="cuda")
    k1 = k2 = 2 * np.pi * 5 / 20
    b = q.cfield(L, L)
    q.plwv(b, (k1, k2), prm)
    Db = q.cfield(L, L)
    q.Dw(Db, U, b, am0, prm)
    bh, Dh = to_host(b), to_host(Db)
    o = Oracle(L, L, 6.05)
    bound("plwv vs oracle", rel(bh, o.plane_wave(k1, k2)), 2e-14)
    lam = np.vdot(bh, Dh) / np.vdot(bh, bh)
    re = am0 + 2 * (np.sin(k1 / 2) ** 2 + np.sin(k2 / 2) ** 2)
    im = np.sqrt(np.sin(k1) ** 2 + np.sin(k2) ** 2)
    assert min(abs(lam - (re + 1j * im)), abs(lam - (re - 1j * im))) < 1e-12
    assert np.max(np.abs(Dh / lam - bh)) < 1e-12


@pytest.mark.parametrize("L1,L2", [(64, 48), (100, 36), (256, 256)])
def test_kernels_vs_oracle(q, L1, L2):
    prm = q.LattParm((L1, L2), 4.0)
    o = Oracle(L1, L2, 4.0)
    U = cgauss(L1, L2, 7, 1)
    si = cgauss(L1, L2, 7, 2)
    Ud, sd = to_dev(U), to_dev(si)
    so = q.cfield(L1, L2)
    q.gamm5Dw(so, Ud, sd, 0.1, prm)
    bound("g5dw vs oracle", rel(to_host(so), o.g5dw(U, si, 0.1)), 1e-15)
    q.gamm5Dw_sqr_sqr(so, Ud, sd, 0.1, prm)
    bound("g5dw_sqr_sqr vs oracle", rel(to_host(so), o.g5dw_sqr_sqr(U, si, 0.1)), 2e-15)
    q.gamm5Dw_sqr_sqr_musq(so, None, Ud, sd, 0.1, 0.4, prm)
    bound("g5dw_sqr_sqr_musq vs oracle", rel(to_host(so), o.g5dw_sqr_sqr_musq(U, si, 0.1, 0.4)), 2e-15)
    G = o.g5dw(U, si, 0.1)
    frc = q.rfield(L1, L2)
    q.tr_dQwdU(frc, Ud, sd, to_dev(G), prm)
    bound("tr_dQwdU vs oracle", rel(to_host(frc), o.fermion_force(U, si, G)), 2e-15)


@pytest.mark.parametrize("L1,L2", [(64, 64), (96, 40), (1024, 512)])
def test_observables_vs_oracle(q, L1, L2):
    prm = q.LattParm((L1, L2), 4.0)
    o = Oracle(L1, L2, 4.0)
    U = hot_links(L1, L2, 3)
    Ud = to_dev(U)
    mom = np.random.default_rng(4).standard_normal((2, L2, L1))
    bound("Action rel vs oracle", abs(q.Action(Ud, prm) - o.action(U)) / abs(o.action(U)), 1e-14)
    bound("Plaquette abs vs oracle", abs(q.Plaquette(Ud, prm) - o.plaquette(U)), 1e-16)
    Qg, Qo = q.Qtop(Ud, prm), o.qtop(U)
    bound("Qtop abs vs oracle", abs(Qg - Qo), 5e-12)
    assert q.Qtop_rounded(Ud, prm) == int(np.rint(Qo))
    H = q.Hamiltonian(to_dev(mom), Ud, prm)
    bound("Hamiltonian rel vs oracle", abs(H - o.hamiltonian(mom, U)) / abs(H), 1e-15)


def test_random_streams_match_oracle(q):
    prm = q.LattParm((16, 8), 1.0)
    for (n, seed, stream, ctr) in [(1001, 1234, 1, 0), (4096, 2**40 + 5, 17, 3), (7, 0, 64, 2**31)]:
        g = to_host(q.random_normal(n, seed, stream, ctr, prm=prm))
        c = Oracle.normal(n, seed, stream, ctr)
        assert np.max(np.abs(g - c)) < 1e-13
    from qed2d import _lib
    assert _lib.lib().qed2d_random_uniform(99, 3, 7) == Oracle.uniform(99, 3, 7)


def test_topological_charge_exact_on_large_hot_field(q):
    """round(Q) bit-exact against the oracle on a 2048^2 hot start."""
    L = 2048
    prm = q.LattParm((L, L), 11.25)
    U = hot_links(L, L, 11)
    assert q.Qtop_rounded(to_dev(U), prm) == int(np.rint(Oracle(L, L, 11.25).qtop(U)))


@pytest.mark.parametrize("L1,L2", [(64, 48), (333, 77)])
def test_g5dw_complex64_vs_f64(q, L1, L2):
    """The FP32 apply on complex64 fields against the FP64 apply of the same
    (rounded) inputs: relative error at FP32 rounding, below 1e-6."""
    import torch
    prm = q.LattParm((L1, L2), 4.0)
    U = to_dev(hot_links(L1, L2, 41)).to(torch.complex64)
    si = to_dev(cgauss(L1, L2, 42, 2)).to(torch.complex64)
    so = torch.empty_like(si)
    q.gamm5Dw(so, U, si, 0.1, prm)
    ref = q.cfield(L1, L2)
    q.gamm5Dw(ref, U.to(torch.complex128), si.to(torch.complex128), 0.1, prm)
    bound("g5dw complex64 vs FP64 apply", rel(to_host(so).astype(np.complex128), to_host(ref)), 5e-7)
    with pytest.raises(ValueError):   # mixed precisions are rejected
        q.gamm5Dw(so, U.to(torch.complex128), si, 0.1, prm)
