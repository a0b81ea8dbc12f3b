"""A NumPy model of the mixed FP32/FP64 CG (the library's recurrences: FP32
iterations, FP64 reliable updates when |r|^2 dropped by delta^2 or looks
converged, FP32 fields rescaled to unit norm at every update, the FP64 stop rule)
in its two direction updates:

  * stencil on p:  p = r + beta p_old, t = g5Dw p            (first form);
  * stencil on r:  t = g5Dw r + beta t_old, p = r + beta p_old (batch schedules
    8 and 9, the mixed CG's schedules 4 to 6).

g5Dw is linear, so both carry t = g5Dw p; the second rounds t along its own
recurrence.  On hot lattices at small masses both forms need the same number of
iterations and reach the same FP64 residual -- the property the GPU solvers'
second form relies on (the GPU tests compare them directly)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_golden import g5dw  # noqa: E402  (the NumPy restatement of gamm5Dw)


def mixed_cg(U, b, m0, stencil_on_r, delta=0.01, eps=1e-24, maxiter=5000):
    U32 = U.astype(np.complex64)
    D32 = lambda v: g5dw(U32, v, np.float32(m0)).astype(np.complex64)   # noqa: E731
    D64 = lambda v: g5dw(U, v, m0)                                       # noqa: E731
    x = np.zeros_like(b)
    bb = np.vdot(b, b).real
    tol = eps * bb
    s = 1.0 / np.sqrt(bb)
    r = (s * b).astype(np.complex64)
    x32 = np.zeros_like(r)
    rr = np.vdot(r, r).real
    maxrr = rr
    p = np.zeros_like(r)
    t = np.zeros_like(r)
    beta, first = 0.0, True
    for k in range(1, maxiter + 1):
        bf = np.float32(beta)
        if stencil_on_r:
            w = D32(r)
            p = r.copy() if first else (r + bf * p).astype(np.complex64)
            t = w if first else (w + bf * t).astype(np.complex64)
        else:
            p = r.copy() if first else (r + bf * p).astype(np.complex64)
            t = D32(p)
        alpha = np.float32(rr / np.vdot(t, t).real)
        x32 = (x32 + alpha * p).astype(np.complex64)
        r = (r - alpha * D32(t)).astype(np.complex64)
        rn = np.vdot(r, r).real
        maxrr = max(maxrr, rn)
        first = False
        if rn < delta ** 2 * maxrr or rn < tol * s * s:   # reliable update
            x = x + x32.astype(np.complex128) / s
            x32[:] = 0
            r64 = b - D64(D64(x))
            rr64 = np.vdot(r64, r64).real
            if rr64 < tol:
                return k, x, rr64 / bb
            s_new = 1.0 / np.sqrt(rr64)
            beta = (rr64 * s * s / rr) * (s_new / s)   # the rescaled beta of the library's record
            s = s_new
            r = (s * r64).astype(np.complex64)
            rr = np.vdot(r, r).real
            maxrr = rr
        else:
            beta = rn / rr
            rr = rn
    raise AssertionError("not converged")


@pytest.mark.parametrize("L,m0,seed", [(32, 0.05, 1), (48, 0.05, 2), (32, 0.3, 3)])
def test_direction_updates_need_the_same_iterations(L, m0, seed):
    rng = np.random.default_rng(seed)
    U = np.exp(1j * rng.uniform(-np.pi, np.pi, (2, L, L)))
    b = (rng.standard_normal((2, L, L)) + 1j * rng.standard_normal((2, L, L))) / np.sqrt(2.0)
    k_p, x_p, res_p = mixed_cg(U, b, m0, stencil_on_r=False)
    k_r, x_r, res_r = mixed_cg(U, b, m0, stencil_on_r=True)
    assert abs(k_r - k_p) <= 2, (k_p, k_r)
    assert res_p < 1e-24 and res_r < 1e-24
    assert np.max(np.abs(x_r - x_p)) / np.max(np.abs(x_p)) < 1e-10
