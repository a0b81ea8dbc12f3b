"""qed2d_cg_noalloc: the allocation-free CG entry point.

It exists for callers that must not allocate device memory while they run (a loop
whose device memory belongs to its own pool allocator, or one that cannot take
the implicit device synchronisation of cudaMalloc).  It runs the same FP64 CG as
qed2d_cg but keeps its scratch in one static device array, so it is limited to
lattices of at most QED2D_NOALLOC_MAX_SITES sites.

Checked through the C ABI: two calls in a row (with different sources, since the
calls share the static scratch) agree with qed2d_cg within the solver tolerance
used by the other CG tests, and an oversized lattice is rejected.  This file is
collected last (its name) so that a run stopping at the first failure has run
every other test before it; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from helpers import cgauss, hot_links, rel, to_dev, to_host

pytestmark = pytest.mark.gpu


def _cg_reference(q, U, b, am0, L1, L2):
    prm = q.LattParm((L1, L2), 4.0)
    x = q.cfield(L1, L2)
    it = q.CG(x, U, b, am0, 20000, 1e-24, q.gamm5Dw_sqr_msq, prm, None)
    return x, it


def _cg_noalloc(U, b, am0, L1, L2, torch):
    from qed2d import _lib
    x = torch.full((2, L2, L1), float("nan"), dtype=torch.complex128, device="cuda")   # garbage in the output
    it = C.c_int(-1)
    st = _lib.lib().qed2d_cg_noalloc(L1, L2, C.c_void_p(x.data_ptr()), C.c_void_p(U.data_ptr()),
                                     C.c_void_p(b.data_ptr()), am0, 20000, 1e-24,
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream), C.byref(it))
    assert st == _lib.OK, _lib.lib().qed2d_last_error()
    return x, it.value


@pytest.mark.parametrize("L1,L2,unitary", [(64, 48, False), (128, 128, True)])
def test_noalloc_cg_matches_cg_twice(L1, L2, unitary):
    import torch

    import qed2d
    qed2d.set_precision("f64")
    am0 = 0.25
    U = to_dev(hot_links(L1, L2, 21) if unitary else cgauss(L1, L2, 21, 1))
    for call in range(2):   # two calls in a row, different sources
        b = to_dev(cgauss(L1, L2, 40 + call, 2))
        x_ref, it_ref = _cg_reference(qed2d, U, b, am0, L1, L2)
        x, it = _cg_noalloc(U, b, am0, L1, L2, torch)
        torch.cuda.synchronize()
        # qed2d_cg may run its tuned one-cluster schedule, whose sums are grouped
        # differently from the cooperative grid this entry point always uses
        assert abs(it - it_ref) <= 2
        assert rel(to_host(x), to_host(x_ref)) < 1e-9


def test_noalloc_cg_rejects_oversized_lattice():
    import torch

    from qed2d import _lib
    L1, L2 = 129, 128   # one row more than 128x128 = QED2D_NOALLOC_MAX_SITES
    assert L1 * L2 > _lib.NOALLOC_MAX_SITES
    U = torch.ones((2, L2, L1), dtype=torch.complex128, device="cuda")
    b = torch.ones_like(U)
    x = torch.zeros_like(U)
    it = C.c_int(0)
    st = _lib.lib().qed2d_cg_noalloc(L1, L2, C.c_void_p(x.data_ptr()), C.c_void_p(U.data_ptr()),
                                     C.c_void_p(b.data_ptr()), 0.2, 100, 1e-24, None, C.byref(it))
    assert st == _lib.BAD_ARG
    assert b"exceeds the static scratch limit" in _lib.lib().qed2d_last_error()
    # an output that overlaps the links is rejected before anything runs
    L1 = 64
    U = torch.ones((2, L2, L1), dtype=torch.complex128, device="cuda")
    b = torch.ones_like(U)
    st = _lib.lib().qed2d_cg_noalloc(L1, L2, C.c_void_p(U.data_ptr()), C.c_void_p(U.data_ptr()),
                                     C.c_void_p(b.data_ptr()), 0.2, 100, 1e-24, None, C.byref(it))
    assert st == _lib.BAD_ARG
