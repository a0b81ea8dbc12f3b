"""Batched replicas: each replica of a batch trajectory reproduces the
single-lattice Nf=2 HMC step (mixed solver) with the same seed and counter, and
the oracle replaying the same draws.  Tolerances as test_gpu_hmc.py: links 1e-9
relative, Delta H 1e-8 absolute, identical accept/reject."""
import numpy as np
import pytest

from helpers import cgauss, hot_links, rel, to_dev, to_host
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L1,L2", [(32, 24), (40, 36)])
def test_batch_matches_single_and_oracle(L1, L2):
    import torch

    import qed2d
    nrep = 3
    betas = [4.0, 3.0, 5.0]
    am0s = [0.3, 0.25, 0.4]
    seeds = [11, 12, 13]
    counter = 7
    U0 = [hot_links(L1, L2, 100 + r) for r in range(nrep)]
    b = qed2d.Batch(nrep, L1, L2, betas)
    Ub = b.field()
    for r in range(nrep):
        Ub[:, r] = to_dev(U0[r])
    infos = b.hmc_nf2(Ub, am0s, 0.1, 5, 10000, 1e-24, seeds, counter)
    qed2d.set_precision("mixed")
    for r in range(nrep):
        prm = qed2d.LattParm((L1, L2), betas[r])
        Ud = to_dev(U0[r])
        qed2d.seed(seeds[r])
        single = qed2d.HMC_(Ud, am0s[r], 0.1, 5, [], 10000, 1e-24, prm, None, counter=counter)
        assert abs(single.dH - infos[r].dH) < 1e-8
        assert single.accepted == infos[r].accepted
        assert rel(to_host(Ub[:, r]), to_host(Ud)) < 1e-9
    qed2d.set_precision("f64")
    # replica 1 against the oracle replaying its draws
    r = 1
    o = Oracle(L1, L2, betas[r])
    mom0 = Oracle.normal(2 * L1 * L2, seeds[r], 1, counter).reshape(2, L2, L1)
    noise = cgauss(L1, L2, seeds[r], 16, counter)
    st, Uo, acc, hi, hf, _ = o.hmc_nf2(U0[r], am0s[r], 0.1, 5, 10000, 1e-24, mom0, noise,
                                        Oracle.uniform(seeds[r], 3, counter))
    assert st == 0 and acc == infos[r].accepted
    assert abs(infos[r].dH - (hf - hi)) < 1e-8
    assert rel(to_host(Ub[:, r]), Uo) < 1e-9


def test_batch_rejects_bad_shape():
    import qed2d
    b = qed2d.Batch(2, 16, 16, 4.0)
    import torch
    with pytest.raises(ValueError):
        b.hmc_nf2(torch.zeros((2, 3, 16, 16), dtype=torch.complex128, device="cuda"), 0.3, 0.1, 2, 100, 1e-20,
                  [1, 2], 0)


def test_batch_cg_matches_single_cg():
    """qed2d_batch_cg: replica r's solution equals the single-lattice mixed solve (1e-9)."""
    import torch

    import qed2d
    nrep, L1, L2 = 4, 48, 40
    am0s = [0.2, 0.3, 0.4, 0.5]
    b = qed2d.Batch(nrep, L1, L2, 4.0)
    U, src, x = b.field(), b.field(), b.field()
    for r in range(nrep):
        U[:, r] = to_dev(hot_links(L1, L2, 200 + r))
        src[:, r] = to_dev(cgauss(L1, L2, 300 + r, 2))
    its, upd = b.cg(x, U, src, am0s, 20000, 1e-24)
    qed2d.set_precision("mixed")
    prm = qed2d.LattParm((L1, L2), 4.0)
    for r in range(nrep):
        xs = qed2d.cfield(L1, L2)
        it = qed2d.CG(xs, U[:, r].contiguous(), src[:, r].contiguous(), am0s[r], 20000, 1e-24,
                      qed2d.gamm5Dw_sqr_msq, prm, None)
        assert rel(to_host(x[:, r]), to_host(xs)) < 1e-9
        assert abs(its[r] - it) <= max(3, it // 20) and upd[r] >= 1
    qed2d.set_precision("f64")
