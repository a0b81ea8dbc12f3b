"""ctypes bindings for the CPU oracle (oracle/qed2d_oracle.c).

Test infrastructure only: the checker the CUDA library is compared against, and
the timed CPU baseline.  The product path never imports this module.

Arrays use the reference's memory layout.  A Julia ``ComplexF64[L1, L2, 2]``
(column-major) is a NumPy ``complex128`` array of shape ``(2, L2, L1)``
(row-major); ``Float64[L1, L2, 2]`` is ``float64`` of shape ``(2, L2, L1)`` and a
per-site ``Float64[L1, L2]`` is ``(L2, L1)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libqed2d_oracle.so")
MAXPOLES = 32

O_OK, O_NOT_CONVERGED, O_BAD_ARG = 0, 1, 3
OP_SQR, OP_SQR_MUSQ = 0, 1
LEAPFROG, OMF4 = 0, 1


class OLatt(C.Structure):
    _fields_ = [("L1", C.c_int), ("L2", C.c_int), ("beta", C.c_double)]


class ORhmc(C.Structure):
    _fields_ = [
        ("r_b", C.c_double), ("n", C.c_int), ("eps", C.c_double), ("A", C.c_double),
        ("rho", C.c_double * MAXPOLES), ("mu", C.c_double * MAXPOLES), ("nu", C.c_double * MAXPOLES),
        ("delta", C.c_double), ("reweighting_N", C.c_int), ("reweighting_Taylor", C.c_int),
    ]

    def as_dict(self):
        n = self.n
        return {
            "r_b": self.r_b, "n": n, "eps": self.eps, "A": self.A,
            "rho": list(self.rho[:n]), "mu": list(self.mu[:n]), "nu": list(self.nu[:n]),
            "delta": self.delta, "reweighting_N": self.reweighting_N,
            "reweighting_Taylor": self.reweighting_Taylor,
        }


def build():
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


P = C.c_void_p
I = C.c_int
D = C.c_double


def _declare(L):
    sig = {
        "o_fill_normal": (None, [P, C.c_int64, C.c_uint64, C.c_uint32, C.c_uint32]),
        "o_uniform": (D, [C.c_uint64, C.c_uint32, C.c_uint32]),
        "o_philox4x32_10": (None, [P, P, P]),
        "o_plaquette_field": (None, [P, P, P]),
        "o_qtop_field": (None, [P, P, P]),
        "o_gauge_force": (None, [P, P, P, P]),
        "o_update_links": (None, [P, P, P, D]),
        "o_g5dw": (None, [P, P, P, P, D]),
        "o_g5": (None, [P, P, P]),
        "o_dw": (None, [P, P, P, P, D]),
        "o_g5dw_sqr": (None, [P, P, P, P, D]),
        "o_g5dw_sqr_sqr": (None, [P, P, P, P, D]),
        "o_g5dw_sqr_musq": (None, [P, P, P, P, D, D]),
        "o_g5dw_sqr_sqr_musq": (None, [P, P, P, P, D, D]),
        "o_fermion_force": (None, [P, P, P, P, P]),
        "o_unfold": (None, [I, I, P, P, I]),
        "o_plane_wave": (None, [P, P, D, D]),
        "o_action": (D, [P, P]),
        "o_plaquette": (D, [P, P]),
        "o_qtop": (D, [P, P]),
        "o_hamiltonian": (D, [P, P, P]),
        "o_norm2": (D, [C.c_int64, P]),
        "o_cg": (I, [P, P, P, P, D, D, I, I, D, I, P, P]),
        "o_multi_cg": (I, [P, P, P, P, D, I, D, P, P]),
        "o_rational": (I, [P, P, P, P, D, I, D, P, P]),
        "o_ellip_K": (D, [D]),
        "o_ellip_sncn": (None, [D, D, P, P]),
        "o_zolotarev": (I, [I, D, D, P]),
        "o_pf_generate": (I, [P, P, P, P, D, I, D, P, P]),
        "o_power_method": (None, [P, P, D, I, P, P, P]),
        "o_luscher_z": (I, [P, P, P, P, D, I, D, P]),
        "o_reweighting_factor": (I, [P, P, D, I, D, P, P, P]),
        "o_omf4_gauge": (None, [P, P, P, D, I]),
        "o_update_momenta_nf2": (I, [P, P, P, P, P, P, D, D, I, D, P]),
        "o_leapfrog_nf2": (I, [P, P, P, P, P, P, D, D, I, I, D, P]),
        "o_omf4_nf2": (I, [P, P, P, P, P, P, D, D, I, I, D, P]),
        "o_hmc_gauge": (I, [P, P, D, I, I, I, P, D, P, P, P]),
        "o_hmc_nf2": (I, [P, P, D, D, I, I, I, D, I, P, P, D, P, P, P, P]),
        "o_hmc_rhmc": (I, [P, P, I, P, D, I, I, D, P, I, I, P, P, D, P, P, P, P]),
        "o_num_threads": (I, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _c(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a


def _r(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    """The reference API restated on the CPU for an L1 x L2 lattice."""

    def __init__(self, L1, L2, beta=0.0):
        self.L1, self.L2, self.beta = int(L1), int(L2), float(beta)
        self.V = self.L1 * self.L2
        self.prm = OLatt(self.L1, self.L2, self.beta)
        self._pp = C.byref(self.prm)
        self.L = lib()

    # shapes
    def cfield(self):
        return np.zeros((2, self.L2, self.L1), np.complex128)

    def rfield(self):
        return np.zeros((2, self.L2, self.L1), np.float64)

    # ---- random numbers (same stream layout as the CUDA library) ----
    @staticmethod
    def normal(n, seed, stream, counter):
        out = np.empty(int(n), np.float64)
        lib().o_fill_normal(_p(out), int(n), int(seed), int(stream), int(counter))
        return out

    @staticmethod
    def uniform(seed, stream, counter):
        return lib().o_uniform(int(seed), int(stream), int(counter))

    # ---- site kernels ----
    def plaquette_field(self, U):
        out = np.empty((self.L2, self.L1))
        self.L.o_plaquette_field(self._pp, _p(out), _p(_c(U)))
        return out

    def qtop_field(self, U):
        out = np.empty((self.L2, self.L1))
        self.L.o_qtop_field(self._pp, _p(out), _p(_c(U)))
        return out

    def gauge_force(self, U):
        f1, f2 = self.rfield(), self.rfield()
        self.L.o_gauge_force(self._pp, _p(f1), _p(f2), _p(_c(U)))
        return f1, f2

    def update_links(self, U, mom, eps):
        U = _c(U).copy()
        self.L.o_update_links(self._pp, _p(U), _p(_r(mom)), float(eps))
        return U

    def _op(self, name, U, si, *args):
        so = self.cfield()
        getattr(self.L, name)(self._pp, _p(so), _p(_c(U)), _p(_c(si)), *[float(a) for a in args])
        return so

    def g5dw(self, U, si, am0):
        return self._op("o_g5dw", U, si, am0)

    def dw(self, U, si, am0):
        return self._op("o_dw", U, si, am0)

    def g5dw_sqr(self, U, si, am0):
        return self._op("o_g5dw_sqr", U, si, am0)

    def g5dw_sqr_sqr(self, U, si, am0):
        return self._op("o_g5dw_sqr_sqr", U, si, am0)

    def g5dw_sqr_musq(self, U, si, am0, mu):
        return self._op("o_g5dw_sqr_musq", U, si, am0, mu)

    def g5dw_sqr_sqr_musq(self, U, si, am0, mu):
        return self._op("o_g5dw_sqr_sqr_musq", U, si, am0, mu)

    def g5(self, si):
        so = self.cfield()
        self.L.o_g5(self._pp, _p(so), _p(_c(si)))
        return so

    def fermion_force(self, U, X, g5X):
        f = self.rfield()
        self.L.o_fermion_force(self._pp, _p(f), _p(_c(U)), _p(_c(X)), _p(_c(g5X)))
        return f

    def unfold(self, U, reflect=False):
        out = np.zeros((2, 2 * self.L2, 2 * self.L1), np.complex128)
        self.L.o_unfold(self.L1, self.L2, _p(out), _p(_c(U)), int(bool(reflect)))
        return out

    def plane_wave(self, k1, k2):
        so = self.cfield()
        self.L.o_plane_wave(self._pp, _p(so), float(k1), float(k2))
        return so

    # ---- observables ----
    def action(self, U):
        return self.L.o_action(self._pp, _p(_c(U)))

    def plaquette(self, U):
        return self.L.o_plaquette(self._pp, _p(_c(U)))

    def qtop(self, U):
        return self.L.o_qtop(self._pp, _p(_c(U)))

    def hamiltonian(self, mom, U):
        return self.L.o_hamiltonian(self._pp, _p(_r(mom)), _p(_c(U)))

    # ---- solvers ----
    def cg(self, U, si, am0, maxiter, tol, mu=None, guess=None):
        """Reference CG: method 1 when mu is None, else method 2 with shift mu."""
        so = self.cfield() if guess is None else _c(guess).copy()
        it = C.c_int(0)
        err = C.c_double(0)
        op = OP_SQR if mu is None else OP_SQR_MUSQ
        st = self.L.o_cg(self._pp, _p(so), _p(_c(U)), _p(_c(si)), float(am0), float(mu or 0.0), op,
                         int(maxiter), float(tol), int(guess is not None), C.byref(it), C.byref(err))
        return st, so, it.value, err.value

    def multi_cg(self, U, si, am0, maxiter, tol, rhmc):
        so = self.cfield()
        it = C.c_int(0)
        st = self.L.o_multi_cg(self._pp, _p(so), _p(_c(U)), _p(_c(si)), float(am0), int(maxiter),
                               float(tol), C.byref(rhmc), C.byref(it))
        return st, so, it.value

    def rational(self, U, si, am0, maxiter, tol, rhmc):
        so = self.cfield()
        it = C.c_int(0)
        st = self.L.o_rational(self._pp, _p(so), _p(_c(U)), _p(_c(si)), float(am0), int(maxiter),
                               float(tol), C.byref(rhmc), C.byref(it))
        return st, so, it.value

    def pf_generate(self, U, X, am0, maxiter, tol, rhmc):
        F = self.cfield()
        it = C.c_int(0)
        st = self.L.o_pf_generate(self._pp, _p(F), _p(_c(U)), _p(_c(X)), float(am0), int(maxiter),
                                  float(tol), C.byref(rhmc), C.byref(it))
        return st, F, it.value

    def power_method(self, U, am0, iters, b0):
        lmin, lmax = C.c_double(0), C.c_double(0)
        self.L.o_power_method(self._pp, _p(_c(U)), float(am0), int(iters), _p(_c(b0)),
                              C.byref(lmin), C.byref(lmax))
        return lmin.value, lmax.value

    def luscher_z(self, U, Xin, am0, maxiter, tol, rhmc):
        Z = self.cfield()
        st = self.L.o_luscher_z(self._pp, _p(Z), _p(_c(U)), _p(_c(Xin)), float(am0), int(maxiter),
                                float(tol), C.byref(rhmc))
        return st, Z

    def reweighting_factor(self, U, am0, maxiter, tol, rhmc, noise):
        W = C.c_double(0)
        st = self.L.o_reweighting_factor(self._pp, _p(_c(U)), float(am0), int(maxiter), float(tol),
                                         C.byref(rhmc), _p(_c(noise)), C.byref(W))
        return st, W.value

    # ---- integrators / HMC ----
    def omf4_gauge(self, mom, U, eps, ns):
        mom, U = _r(mom).copy(), _c(U).copy()
        self.L.o_omf4_gauge(self._pp, _p(mom), _p(U), float(eps), int(ns))
        return mom, U

    def hmc_gauge(self, U, eps, ns, mom0, r_unif, integrator=OMF4, qzero=False):
        U = _c(U).copy()
        acc, hi, hf = C.c_int(0), C.c_double(0), C.c_double(0)
        st = self.L.o_hmc_gauge(self._pp, _p(U), float(eps), int(ns), int(integrator), int(bool(qzero)),
                                _p(_r(mom0)), float(r_unif), C.byref(acc), C.byref(hi), C.byref(hf))
        return st, U, acc.value, hi.value, hf.value

    def hmc_nf2(self, U, am0, eps, ns, maxiter, tol, mom0, noise, r_unif, integrator=LEAPFROG, qzero=False):
        U = _c(U).copy()
        acc, hi, hf, it = C.c_int(0), C.c_double(0), C.c_double(0), C.c_int(0)
        st = self.L.o_hmc_nf2(self._pp, _p(U), float(am0), float(eps), int(ns), int(integrator), int(maxiter),
                              float(tol), int(bool(qzero)), _p(_r(mom0)), _p(_c(noise)), float(r_unif),
                              C.byref(acc), C.byref(hi), C.byref(hf), C.byref(it))
        return st, U, acc.value, hi.value, hf.value, it.value

    def hmc_rhmc(self, U, am0s, eps, ns, maxiter, tol, rhmcs, mom0, noises, r_unif, qzero=False,
                 reversibility=False):
        U = _c(U).copy()
        nf = len(am0s)
        am = np.ascontiguousarray(am0s, np.float64)
        rarr = (ORhmc * nf)(*rhmcs)
        noise = _c(np.stack([_c(x) for x in noises]))
        acc, hi, hf, it = C.c_int(0), C.c_double(0), C.c_double(0), C.c_int(0)
        st = self.L.o_hmc_rhmc(self._pp, _p(U), nf, _p(am), float(eps), int(ns), int(maxiter), float(tol),
                               rarr, int(bool(qzero)), int(bool(reversibility)), _p(_r(mom0)), _p(noise),
                               float(r_unif), C.byref(acc), C.byref(hi), C.byref(hf), C.byref(it))
        return st, U, acc.value, hi.value, hf.value, it.value


def zolotarev(n, r_a, r_b):
    out = ORhmc()
    st = lib().o_zolotarev(int(n), float(r_a), float(r_b), C.byref(out))
    if st != O_OK:
        raise ValueError("bad Zolotarev arguments")
    return out


def ellip_K(m):
    return lib().o_ellip_K(float(m))


def ellip_sncn(u, m):
    s, c = C.c_double(0), C.c_double(0)
    lib().o_ellip_sncn(float(u), float(m), C.byref(s), C.byref(c))
    return s.value, c.value


def num_threads():
    return lib().o_num_threads()
