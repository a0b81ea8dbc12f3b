"""Pin the CPU oracle against the golden fixtures (tests/golden/make_golden.py):
an independent NumPy restatement of the reference formulas, dense solves and
50-digit mpmath Zolotarev coefficients.  CPU only."""
import json
import os

import numpy as np
import pytest

from oracle.oracle import Oracle, ellip_K, ellip_sncn, zolotarev

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SIZES = ["6x4", "5x7"]


def load(tag):
    return dict(np.load(os.path.join(GOLD, f"kernels_{tag}.npz")))


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("tag", SIZES)
def test_dirac_kernels(tag):
    g = load(tag)
    o = Oracle(int(g["L1"]), int(g["L2"]), float(g["beta"]))
    m0, mu = float(g["m0"]), float(g["mu"])
    assert rel(o.g5dw(g["U"], g["si"], m0), g["g5dw"]) < 1e-14
    assert rel(o.dw(g["U"], g["si"], m0), g["dw"]) < 1e-14
    assert rel(o.g5dw_sqr(g["U"], g["si"], m0), g["g5dw_sqr"]) < 1e-14
    assert rel(o.g5dw_sqr_musq(g["U"], g["si"], m0, mu), g["g5dw_sqr_musq"]) < 1e-14
    assert rel(o.fermion_force(g["U"], g["X"], g["g5dw_X"]), g["fermion_force"]) < 1e-14


@pytest.mark.parametrize("tag", SIZES)
def test_gauge_kernels(tag):
    g = load(tag)
    o = Oracle(int(g["L1"]), int(g["L2"]), float(g["beta"]))
    Uu = g["Uu"]
    assert rel(o.plaquette_field(Uu), g["plaq_field"]) < 1e-14
    assert rel(o.qtop_field(Uu), g["qtop_field"]) < 1e-14
    f1, f2 = o.gauge_force(Uu)
    assert rel(f1, g["frc1"]) < 1e-14 and rel(f2, g["frc2"]) < 1e-14
    assert rel(o.update_links(Uu, g["mom"], float(g["eps"])), g["update_links"]) < 1e-14
    assert np.array_equal(o.unfold(Uu, False), g["unfold"])
    assert np.array_equal(o.unfold(Uu, True), g["reflect"])
    assert abs(o.action(Uu) - float(g["action_unitary"])) < 1e-12 * abs(float(g["action_unitary"]))


@pytest.mark.parametrize("tag", SIZES)
def test_cg_against_dense_solve(tag):
    g = load(tag)
    o = Oracle(int(g["L1"]), int(g["L2"]), float(g["beta"]))
    m0, mu = float(g["m0"]), float(g["mu"])
    st, x, it, _ = o.cg(g["U"], g["si"], m0, 10000, 1e-26)
    assert st == 0 and it > 0
    assert rel(x, g["cg_solution"]) < 1e-9
    st, x, it, _ = o.cg(g["U"], g["si"], m0, 10000, 1e-26, mu=mu)
    assert st == 0
    assert rel(x, g["cg_solution_musq"]) < 1e-10


@pytest.mark.parametrize("tag", SIZES)
def test_power_method_against_dense_spectrum(tag):
    g = load(tag)
    o = Oracle(int(g["L1"]), int(g["L2"]), float(g["beta"]))
    rng = np.random.default_rng(3)
    shape = (2, int(g["L2"]), int(g["L1"]))
    b0 = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2)
    lmin, lmax = o.power_method(g["Uu"], float(g["m0"]), 4000, b0)
    assert abs(lmax - float(g["eig_max_unitary"])) < 1e-6 * float(g["eig_max_unitary"])
    assert abs(lmin - float(g["eig_min_unitary"])) < 1e-3 * float(g["eig_max_unitary"])


def test_elliptic_functions():
    data = json.load(open(os.path.join(GOLD, "zolotarev.json")))
    for p in data["elliptic"]:
        assert abs(ellip_K(p["m"]) - p["K"]) < 1e-14 * p["K"]
        s, c = ellip_sncn(p["u"], p["m"])
        assert abs(s - p["sn"]) < 5e-15 and abs(c - p["cn"]) < 5e-14


def test_zolotarev_coefficients():
    data = json.load(open(os.path.join(GOLD, "zolotarev.json")))
    for z in data["zolotarev"]:
        r = zolotarev(z["n"], z["r_a"], z["r_b"]).as_dict()
        assert r["n"] == z["n"]
        assert abs(r["A"] - z["A"]) < 1e-12 * abs(z["A"])
        assert abs(r["delta"] - z["delta"]) < 1e-9 * abs(z["delta"]) + 1e-300
        for key in ("mu", "nu", "rho"):
            a, b = np.array(r[key]), np.array(z[key])
            assert np.max(np.abs(a - b) / np.abs(b)) < 1e-11, key


def test_free_field_plane_wave_eigenvalue():
    """Known answer of tests/Dw-eigenvalues.jl:15-35 (U = 1, k = 2 pi 5/20)."""
    L, am0 = 20, 10.0
    o = Oracle(L, L, 6.05)
    U = np.ones((2, L, L), np.complex128)
    k1 = k2 = 2 * np.pi * 5 / 20
    b = o.plane_wave(k1, k2)
    Db = o.dw(U, b, am0)
    lam = np.vdot(b, Db) / np.vdot(b, b)
    re = am0 + 2 * (np.sin(k1 / 2) ** 2 + np.sin(k2 / 2) ** 2)
    im = np.sqrt(np.sin(k1) ** 2 + np.sin(k2) ** 2)
    assert min(abs(lam - (re + 1j * im)), abs(lam - (re - 1j * im))) < 1e-12
    assert np.max(np.abs(Db / lam - b)) < 1e-12


def test_philox_known_answer():
    """Philox4x32-10 known-answer vectors published with Random123 (kat_vectors)."""
    import ctypes as C
    from oracle.oracle import lib
    out = (C.c_uint32 * 4)()
    cases = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in cases:
        c = (C.c_uint32 * 4)(*ctr)
        k = (C.c_uint32 * 2)(*key)
        lib().o_philox4x32_10(c, k, out)
        assert tuple(out) == want
