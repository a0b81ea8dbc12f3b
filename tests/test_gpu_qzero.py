"""The fixed-topology veto of HMC! (qzero = true; src/QED2dHMC.jl:31-39, 84-92,
174-182): when the field at the end of the molecular dynamics has |Q| > 0.1
the acceptance probability is 0, the Metropolis uniform is still drawn and the
links are restored; otherwise Metropolis decides as usual.

Chains start cold (Q = 0) at beta = 2 on 12x12, where the charge moves in most
trajectories.  Every trajectory is replayed on the oracle with the same draws,
with the veto (the chain that must match) and without it (to count the
trajectories the veto alone rejected).  Seeds and lengths are chosen so that
both cases occur: trajectories vetoed although Metropolis would have accepted
them, and Q = 0 trajectories accepted through Metropolis."""
import numpy as np
import pytest

from helpers import bound, cgauss, rel, to_dev, to_host
from oracle.oracle import OMF4 as O_OMF4, Oracle

pytestmark = pytest.mark.gpu

L, BETA, EPS, NS, SEED = 12, 2.0, 0.1, 4, 4321


def test_qzero_pure_gauge_chain():
    import torch

    import qed2d
    prm = qed2d.LattParm((L, L), BETA)
    o = Oracle(L, L, BETA)
    Ud = torch.ones((2, L, L), dtype=torch.complex128, device="cuda")
    Uo = np.ones((2, L, L), np.complex128)
    qed2d.seed(SEED)
    vetoed = accepted = 0
    for t in range(30):
        acc = []
        info = qed2d.HMC_(Ud, EPS, NS, acc, prm, None, integrator=qed2d.OMF4(), qzero=True)
        assert info.counter == t
        mom0 = Oracle.normal(2 * L * L, SEED, 1, t).reshape(2, L, L)
        u = Oracle.uniform(SEED, 3, t)
        _, Uq, aq, hi, hf = o.hmc_gauge(Uo, EPS, NS, mom0, u, integrator=O_OMF4, qzero=True)
        _, Un, an, _, _ = o.hmc_gauge(Uo, EPS, NS, mom0, u, integrator=O_OMF4, qzero=False)
        assert info.accepted == aq == acc[0], t
        bound("qzero gauge dH abs", abs(info.dH - (hf - hi)), 5e-12)
        bound("qzero gauge links rel", rel(to_host(Ud), Uq), 5e-13)
        if an and not aq:
            vetoed += 1
            assert abs(o.qtop(Un)) > 0.1
            assert np.array_equal(Uq, Uo)   # restored exactly
        accepted += aq
        assert qed2d.Qtop_rounded(Ud, prm) == 0   # the chain never leaves Q = 0
        Uo = Uq
    assert vetoed >= 5 and accepted >= 5, (vetoed, accepted)


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_qzero_nf2_chain(prec):
    import torch

    import qed2d
    am0 = 0.3
    prm = qed2d.LattParm((L, L), BETA)
    o = Oracle(L, L, BETA)
    qed2d.set_precision(prec)
    try:
        Ud = torch.ones((2, L, L), dtype=torch.complex128, device="cuda")
        Uo = np.ones((2, L, L), np.complex128)
        qed2d.seed(SEED)
        vetoed = accepted = 0
        for t in range(12):
            info = qed2d.HMC_(Ud, am0, EPS, NS, [], 10000, 1e-24, prm, None, qzero=True)
            mom0 = Oracle.normal(2 * L * L, SEED, 1, t).reshape(2, L, L)
            noise = cgauss(L, L, SEED, 16, t)
            u = Oracle.uniform(SEED, 3, t)
            _, Uq, aq, hi, hf, _ = o.hmc_nf2(Uo, am0, EPS, NS, 10000, 1e-24, mom0, noise, u, qzero=True)
            _, Un, an, _, _, _ = o.hmc_nf2(Uo, am0, EPS, NS, 10000, 1e-24, mom0, noise, u, qzero=False)
            assert info.accepted == aq, t
            bound(f"qzero nf2 {prec} dH abs", abs(info.dH - (hf - hi)), 1e-9 if prec == "mixed" else 2e-10)
            bound(f"qzero nf2 {prec} links rel", rel(to_host(Ud), Uq), 5e-11 if prec == "mixed" else 2e-12)
            if an and not aq:
                vetoed += 1
                assert np.array_equal(Uq, Uo)
            accepted += aq
            assert qed2d.Qtop_rounded(Ud, prm) == 0
            Uo = Uq
        assert vetoed >= 2 and accepted >= 4, (vetoed, accepted)
    finally:
        qed2d.set_precision("f64")


def test_qzero_batched_replicas():
    """The batched trajectory applies the veto per replica: two replicas of the
    same cold start with different seeds, each replayed on the oracle."""
    import qed2d
    am0 = 0.3
    seeds = [SEED, SEED + 1]
    b = qed2d.Batch(2, L, L, BETA)
    U = b.field()
    U.fill_(1.0)
    o = Oracle(L, L, BETA)
    Uo = [np.ones((2, L, L), np.complex128) for _ in seeds]
    vetoed = accepted = 0
    for t in range(12):
        infos = b.hmc_nf2(U, am0, EPS, NS, 10000, 1e-24, seeds, t, qzero=True)
        for r, s in enumerate(seeds):
            mom0 = Oracle.normal(2 * L * L, s, 1, t).reshape(2, L, L)
            noise = cgauss(L, L, s, 16, t)
            u = Oracle.uniform(s, 3, t)
            _, Uq, aq, hi, hf, _ = o.hmc_nf2(Uo[r], am0, EPS, NS, 10000, 1e-24, mom0, noise, u, qzero=True)
            _, _, an, _, _, _ = o.hmc_nf2(Uo[r], am0, EPS, NS, 10000, 1e-24, mom0, noise, u, qzero=False)
            assert infos[r].accepted == aq, (t, r)
            bound("qzero batched dH abs", abs(infos[r].dH - (hf - hi)), 1e-9)
            bound("qzero batched links rel", rel(to_host(U[r]), Uq), 5e-11)
            vetoed += int(an and not aq)
            accepted += aq
            Uo[r] = Uq
    assert vetoed >= 2 and accepted >= 4, (vetoed, accepted)
