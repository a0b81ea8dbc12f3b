"""Failure detection on the GPU without a fault.  Every grid-barrier wait in the
persistent kernels is bounded: a block that never arrives makes the others give
up after a poll limit, record QED2D_ERR_TIMEOUT and leave, and the host reads the
status.  The self-test entry point runs one kernel whose barrier can never
complete (its second member does not exist), with a small poll limit, through
the C ABI; afterwards the same context must solve as usual."""
import pytest

from helpers import bound, cgauss, hot_links, rel, to_dev, to_host
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def test_barrier_wait_gives_up_and_context_stays_usable():
    import qed2d
    from qed2d import _lib
    L1, L2, am0 = 32, 24, 0.3
    prm = qed2d.LattParm((L1, L2), 4.0)
    lib = _lib.lib()
    for polls in (1000, 20000):   # twice: the error does not stick to the context
        assert lib.qed2d_selftest_barrier_timeout(qed2d._c(prm), polls) == _lib.TIMEOUT
    assert lib.qed2d_selftest_barrier_timeout(qed2d._c(prm), 0) == _lib.BAD_ARG
    Uh, bh = hot_links(L1, L2, 31), cgauss(L1, L2, 32, 2)
    st, xo, _, _ = Oracle(L1, L2, 4.0).cg(Uh, bh, am0, 20000, 1e-24)
    assert st == 0
    qed2d.set_precision("f64")
    x = qed2d.cfield(L1, L2)
    qed2d.CG(x, to_dev(Uh), to_dev(bh), am0, 20000, 1e-24, qed2d.gamm5Dw_sqr_msq, prm, None)
    bound("CG after a barrier timeout vs oracle", rel(to_host(x), xo), 1e-13)
