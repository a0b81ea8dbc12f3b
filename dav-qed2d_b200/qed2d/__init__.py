"""qed2d -- Python host API of libqed2d, mirroring the reference's Julia module
``QED2d`` (src/QED2d.jl:27-54) name for name.

Conventions
* Fields are CUDA ``torch`` tensors in the reference's memory layout: a Julia
  ``CuArray{ComplexF64}(L1, L2, 2)`` is a contiguous ``complex128`` tensor of
  shape ``(2, L2, L1)``; ``Float64(L1, L2, 2)`` is ``float64`` ``(2, L2, L1)`` and
  a per-site ``Float64(L1, L2)`` is ``(L2, L1)``.
* Julia's mutating ``f!`` is Python's ``f_`` (``HMC!`` -> ``HMC_``,
  ``plaquette!`` -> ``plaquette_``).  Kernels the reference launches with
  ``CUDA.@cuda threads= blocks= f(args)`` are plain calls ``f(args)`` here;
  ``KernelParm`` is accepted everywhere and ignored (launch geometry is chosen
  by the library).
* Errors: CG non-convergence raises ``Qed2dError`` (the reference calls
  ``error``, src/QED2dSolver.jl:39-43, 98-102).
* Random numbers: the reference draws from CURAND's and Julia's global
  generators.  Here every draw comes from Philox4x32-10 keyed by the module's
  seed (``seed(s)``, the role of ``Random.seed!``) and a counter that advances
  once per HMC step / power method / reweighting call.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Sequence

import torch

from . import _lib
from ._lib import Qed2dError, check, lib

__all__ = [
    "LattParm", "KernelParm", "RHMCParm", "Integrators", "Leapfrog", "OMF4",
    "plaquette_", "qtop_", "updt_fld_", "krnl_force_",
    "HMC_", "Hamiltonian", "Action", "Plaquette", "Qtop", "OMF4_", "leapfrog_", "update_momenta_",
    "unfold_fld_", "unfold_reflect_",
    "gamm5Dw", "gamm5Dw_sqr", "gamm5Dw_sqr_msq", "tr_dQwdU", "gamm5Dw_sqr_musq", "gamm5Dw_sqr_sqr_musq",
    "gamm5Dw_sqr_sqr", "gamm5", "Dw", "CG", "save_gauge", "load_gauge", "get_rhmc_params", "power_method",
    "reweighting_factor", "R", "MultiCG", "generate_pseudofermion_", "plwv", "LuscherZ", "LuscherZp",
    "k", "v", "a_r", "c_r", "mu", "nu", "rho_mu", "rho_nu", "P", "d", "A", "delta", "error",
    "seed", "set_precision", "set_schedule", "get_schedule", "set_multishift_layout", "get_multishift_layout", "Qed2dError", "cfield", "rfield", "context",
]


# ---------------------------------------------------------------------------
# parameter types (src/QED2d.jl:5-26, src/integrators/integrators.jl:1-3)
@dataclass(frozen=True)
class LattParm:
    iL: tuple
    beta: float


@dataclass(frozen=True)
class KernelParm:
    threads: tuple = (1, 1)
    blocks: tuple = (1, 1)


@dataclass
class RHMCParm:
    r_b: float
    n: int
    eps: float
    A: float
    rho: List[float]
    mu: List[float]
    nu: List[float]
    delta: float
    reweighting_N: int = 1
    reweighting_Taylor: int = 5

    def to_c(self) -> _lib.RhmcParams:
        p = _lib.RhmcParams()
        p.r_b, p.n, p.eps, p.A, p.delta = self.r_b, self.n, self.eps, self.A, self.delta
        p.reweighting_N, p.reweighting_Taylor = self.reweighting_N, self.reweighting_Taylor
        for i in range(self.n):
            p.rho[i], p.mu[i], p.nu[i] = self.rho[i], self.mu[i], self.nu[i]
        return p

    @staticmethod
    def from_c(p: _lib.RhmcParams) -> "RHMCParm":
        n = p.n
        return RHMCParm(p.r_b, n, p.eps, p.A, list(p.rho[:n]), list(p.mu[:n]), list(p.nu[:n]), p.delta,
                        p.reweighting_N, p.reweighting_Taylor)


class Integrators:
    pass


class Leapfrog(Integrators):
    code = _lib.LEAPFROG


class OMF4(Integrators):
    code = _lib.OMF4


# ---------------------------------------------------------------------------
# contexts, RNG state, precision
_ctx = {}
_rng = {"seed": 1234, "counter": 0}
_precision = {"value": _lib.PREC_F64}


def seed(s: int) -> None:
    """Random.seed! for the library's draws: reset the Philox key and counter."""
    _rng["seed"] = int(s) & 0xFFFFFFFFFFFFFFFF
    _rng["counter"] = 0


def _next_counter() -> int:
    c = _rng["counter"]
    _rng["counter"] = (c + 1) & 0xFFFFFFFF
    return c


def set_precision(p) -> None:
    """Solver path of every CG: "f64" (default), "mixed" (FP32 inner, FP64
    reliable updates, FP64 stop rule) or "plain" (reference-structured)."""
    m = {"f64": _lib.PREC_F64, "mixed": _lib.PREC_MIXED, "plain": _lib.PREC_PLAIN}
    _precision["value"] = m[p] if isinstance(p, str) else int(p)
    for h in _ctx.values():
        check(lib().qed2d_ctx_set_precision(h, _precision["value"]))


def context(L1: int, L2: int, beta: float = 0.0):
    """The library context of an L1 x L2 lattice on the current device (cached)."""
    dev = torch.cuda.current_device()
    key = (int(L1), int(L2), dev)
    h = _ctx.get(key)
    if h is None:
        hp = C.c_void_p()
        check(lib().qed2d_ctx_create(int(L1), int(L2), float(beta), C.byref(hp)), "ctx_create")
        h = hp.value
        check(lib().qed2d_ctx_set_precision(h, _precision["value"]))
        _ctx[key] = h
    L = lib()
    check(L.qed2d_ctx_set_beta(h, float(beta)))
    check(L.qed2d_ctx_set_stream(h, C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return h


def _c(prm: LattParm):
    return context(prm.iL[0], prm.iL[1], prm.beta)


def cfield(L1, L2, device="cuda"):
    """A zero complex field (spinor or links), Julia CuArray{ComplexF64}(L1, L2, 2)."""
    return torch.zeros((2, L2, L1), dtype=torch.complex128, device=device)


def rfield(L1, L2, device="cuda"):
    """A zero real field (momenta, forces), Julia CuArray{Float64}(L1, L2, 2)."""
    return torch.zeros((2, L2, L1), dtype=torch.float64, device=device)


def _ptr(t: torch.Tensor, prm: LattParm, dtype, shape=None, name="array"):
    L1, L2 = prm.iL
    want = shape or (2, L2, L1)
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name}: expected a CUDA tensor")
    if t.dtype != dtype or tuple(t.shape) != tuple(want) or not t.is_contiguous():
        raise ValueError(f"{name}: expected contiguous {dtype} of shape {want}, got {t.dtype} {tuple(t.shape)}")
    return C.c_void_p(t.data_ptr())


def _cp(t, prm, name="field"):
    return _ptr(t, prm, torch.complex128, name=name)


def _rp(t, prm, name="field"):
    return _ptr(t, prm, torch.float64, name=name)


def _prm_of(U: torch.Tensor, beta=0.0) -> LattParm:
    return LattParm((U.shape[2], U.shape[1]), beta)


# ---------------------------------------------------------------------------
# gauge kernels (src/QED2dAction.jl)
def plaquette_(plx, U, prm: LattParm):
    """plaquette! (src/QED2dAction.jl:2-16)."""
    h = _c(prm)
    check(lib().qed2d_plaquette_field(h, _ptr(plx, prm, torch.float64, (prm.iL[1], prm.iL[0]), "plx"),
                                      _cp(U, prm, "U")))


def qtop_(plx, U, prm: LattParm):
    """qtop! (src/QED2dAction.jl:18-32)."""
    h = _c(prm)
    check(lib().qed2d_qtop_field(h, _ptr(plx, prm, torch.float64, (prm.iL[1], prm.iL[0]), "plx"),
                                 _cp(U, prm, "U")))


def krnl_force_(frc1, frc2, U, prm: LattParm):
    """krnl_force! (src/QED2dAction.jl:34-53)."""
    h = _c(prm)
    check(lib().qed2d_krnl_force(h, _rp(frc1, prm), _rp(frc2, prm), _cp(U, prm, "U")))


def updt_fld_(U, mom, eps):
    """updt_fld! (src/QED2dAction.jl:55-65)."""
    prm = _prm_of(U)
    h = _c(prm)
    check(lib().qed2d_updt_fld(h, _cp(U, prm, "U"), _rp(mom, prm, "mom"), float(eps)))


# ---------------------------------------------------------------------------
# Dirac operator (src/QED2dDirac.jl)
def gamm5Dw(so, U, si, am0, prm: LattParm, kprm=None):
    """gamm5Dw (src/QED2dDirac.jl:2-33).  complex64 fields (so, U, si all
    complex64) run the FP32 apply; complex128 the FP64 one."""
    if isinstance(so, torch.Tensor) and so.dtype == torch.complex64:
        c64 = torch.complex64
        check(lib().qed2d_gamm5dw_c64(_c(prm), _ptr(so, prm, c64, name="so"), _ptr(U, prm, c64, name="U"),
                                      _ptr(si, prm, c64, name="si"), float(am0)), "gamm5Dw (complex64)")
        return
    check(lib().qed2d_gamm5dw(_c(prm), _cp(so, prm), _cp(U, prm), _cp(si, prm), float(am0)), "gamm5Dw")


def gamm5(so, si, am0, prm: LattParm, kprm=None):
    """gamm5 (src/QED2dDirac.jl:130-146)."""
    check(lib().qed2d_gamm5(_c(prm), _cp(so, prm), _cp(si, prm)), "gamm5")


def Dw(so, U, si, am0, prm: LattParm, kprm=None):
    """Dw (src/QED2dDirac.jl:157-169)."""
    check(lib().qed2d_dw(_c(prm), _cp(so, prm), _cp(U, prm), _cp(si, prm), float(am0)), "Dw")


def gamm5Dw_sqr(so, U, si, am0, prm: LattParm, kprm=None):
    """gamm5Dw_sqr (src/QED2dDirac.jl:35-46)."""
    check(lib().qed2d_gamm5dw_sqr(_c(prm), _cp(so, prm), _cp(U, prm), _cp(si, prm), float(am0)), "gamm5Dw_sqr")


def gamm5Dw_sqr_sqr(so, U, si, am0, prm: LattParm, kprm=None):
    """gamm5Dw_sqr_sqr (src/QED2dDirac.jl:48-67)."""
    check(lib().qed2d_gamm5dw_sqr_sqr(_c(prm), _cp(so, prm), _cp(U, prm), _cp(si, prm), float(am0)))


def gamm5Dw_sqr_msq(so, tmp, U, si, am0, prm: LattParm, kprm=None):
    """gamm5Dw_sqr_msq (src/QED2dDirac.jl:69-81): (g5Dw)^2, no mass term; tmp unused."""
    gamm5Dw_sqr(so, U, si, am0, prm)


def gamm5Dw_sqr_musq(so, tmp, U, si, am0, mu_j, prm: LattParm, kprm=None):
    """gamm5Dw_sqr_musq (src/QED2dDirac.jl:83-95); tmp unused."""
    check(lib().qed2d_gamm5dw_sqr_musq(_c(prm), _cp(so, prm), _cp(U, prm), _cp(si, prm), float(am0),
                                       float(mu_j)))


def gamm5Dw_sqr_sqr_musq(so, tmp, U, si, am0, mu_j, prm: LattParm, kprm=None):
    """gamm5Dw_sqr_sqr_musq (src/QED2dDirac.jl:97-117); tmp unused."""
    check(lib().qed2d_gamm5dw_sqr_sqr_musq(_c(prm), _cp(so, prm), _cp(U, prm), _cp(si, prm), float(am0),
                                           float(mu_j)))


def tr_dQwdU(frc, U, X, g5DwX, prm: LattParm):
    """tr_dQwdU (src/QED2dDirac.jl:172-199)."""
    check(lib().qed2d_tr_dqwdu(_c(prm), _rp(frc, prm), _cp(U, prm), _cp(X, prm), _cp(g5DwX, prm)))


# ---------------------------------------------------------------------------
# CG (src/QED2dSolver.jl): both reference methods, dispatched on the arguments
#   CG(so, U, si, am0, maxiter, eps, A, prm, kprm)                    method 1
#   CG(so, U, si, am0, mu, maxiter, eps, A, prm, kprm; so_as_guess)   method 2
def CG(so, U, si, am0, *args, so_as_guess=False):
    if len(args) == 5:
        maxiter, eps, A, prm, kprm = args
        if A not in (gamm5Dw_sqr_msq, gamm5Dw_sqr):
            raise ValueError("CG method 1 supports A = gamm5Dw_sqr_msq")
        it = C.c_int(0)
        st = lib().qed2d_cg(_c(prm), _cp(so, prm), _cp(U, prm), _cp(si, prm), float(am0), int(maxiter),
                            float(eps), C.byref(it))
        if st == _lib.NOT_CONVERGED:
            raise Qed2dError(st, f"CG not converged after {maxiter} iterationss")
        check(st, "CG")
        return it.value
    if len(args) == 6:
        mu, maxiter, eps, A, prm, kprm = args
        if A is not gamm5Dw_sqr_musq:
            raise ValueError("CG method 2 supports A = gamm5Dw_sqr_musq")
        it = C.c_int(0)
        st = lib().qed2d_cg_shift(_c(prm), _cp(so, prm), _cp(U, prm), _cp(si, prm), float(am0), float(mu),
                                  int(maxiter), float(eps), int(bool(so_as_guess)), C.byref(it))
        if st == _lib.NOT_CONVERGED:
            raise Qed2dError(st, f"CG not converged after {maxiter} iterationss")
        check(st, "CG")
        return it.value
    raise TypeError("CG: unsupported argument list")


_PRECS = {"f64": _lib.PREC_F64, "mixed": _lib.PREC_MIXED, "multishift": _lib.MULTISHIFT}


def set_schedule(prm: LattParm, schedule: int, precision="mixed") -> None:
    """Fix a persistent solver's reduction schedule on this lattice's context:
    0 (last block publishes the sums), 1 (every block sums), 2 (one
    thread-block cluster, small lattices), or -1 to tune again on the next
    solve.  0 and 1 give the same bits.  `precision` selects the solver:
    "f64" or "mixed" (CG), "multishift" (the RHMC shifted solves; its schedule
    3 is the FP32 shared Krylov space with every shift refined by the mixed CG,
    the untuned choice from 2^22 sites on).  The mixed CG also has 4, 5, 6:
    0, 1, 2 with the first stencil applied to r and the links staged in shared
    memory (agrees with 0, 1, 2 to the solver's accuracy; small lattices)."""
    check(lib().qed2d_ctx_set_schedule(_c(prm), _PRECS[precision], int(schedule)), "set_schedule")


def set_multishift_layout(prm: LattParm, layout: int) -> None:
    """Fix the layout of the FP64 multishift kernel on this lattice's context:
    0 (32 x 8 tiles, one thread per site), 1 (32 x 8 tiles, two threads per
    site), 2 (32 x 4 tiles, four threads per site), 3 (32 x 4 tiles, two
    threads per site), or -1 to tune it with the schedule on the next solve.
    Layouts that split the lattice into the same blocks give the same bits."""
    check(lib().qed2d_ctx_set_multishift_layout(_c(prm), int(layout)), "set_multishift_layout")


def get_multishift_layout(prm: LattParm) -> int:
    """The multishift kernel's layout on this lattice (-1 until tuned)."""
    v = C.c_int(0)
    check(lib().qed2d_ctx_get_multishift_layout(_c(prm), C.byref(v)), "get_multishift_layout")
    return v.value


def get_schedule(prm: LattParm, precision="mixed") -> int:
    """The solver's reduction schedule on this lattice (-1 until the first solve tunes it)."""
    v = C.c_int(0)
    check(lib().qed2d_ctx_get_schedule(_c(prm), _PRECS[precision], C.byref(v)), "get_schedule")
    return v.value


def set_graphs(prm: LattParm, on: bool) -> None:
    """Turn CUDA-graph replay of the MD integration of HMC_ on or off for this
    lattice's context (on by default): the first trajectory with given
    arguments runs its launches directly, the second captures them into a
    graph, later ones replay it.  Results are bitwise those of direct launches."""
    check(lib().qed2d_ctx_set_graphs(_c(prm), 1 if on else 0), "set_graphs")


def _stats(fn, h):
    on, cap, rep, fail = C.c_int(0), C.c_int64(0), C.c_int64(0), C.c_int64(0)
    check(fn(h, C.byref(on), C.byref(cap), C.byref(rep), C.byref(fail)), "graph_stats")
    return {"on": bool(on.value), "captures": cap.value, "replays": rep.value, "failures": fail.value}


def graph_stats(prm: LattParm) -> dict:
    """{"on", "captures", "replays", "failures"} of this lattice's MD graph."""
    return _stats(lib().qed2d_ctx_graph_stats, _c(prm))


def last_solve(prm: LattParm):
    """(iterations, |r|^2/|b|^2, reliable updates) of the most recent solve on this lattice."""
    it, rel, upd = C.c_int64(0), C.c_double(0), C.c_int64(0)
    check(lib().qed2d_last_solve(_c(prm), C.byref(it), C.byref(rel), C.byref(upd)))
    return it.value, rel.value, upd.value


def multishift_CG(sos: Sequence[torch.Tensor], U, si, am0, mus, maxiter, eps, prm: LattParm):
    """All shifted solves ((g5Dw)^2 + mu_i^2) so_i = si in one Krylov space."""
    n = len(mus)
    ptrs = (C.c_void_p * n)(*[_cp(s, prm).value for s in sos])
    mu = (C.c_double * n)(*[float(m) for m in mus])
    it = C.c_int(0)
    check(lib().qed2d_multishift_cg(_c(prm), ptrs, _cp(U, prm), _cp(si, prm), float(am0), mu, n, int(maxiter),
                                    float(eps), C.byref(it)), "multishift CG")
    return it.value


# ---------------------------------------------------------------------------
# observables (src/QED2dHMC.jl:198-237)
def Action(U, prm: LattParm, kprm=None) -> float:
    v = C.c_double(0)
    check(lib().qed2d_action(_c(prm), _cp(U, prm), C.byref(v)))
    return v.value


def Plaquette(U, prm: LattParm, kprm=None) -> float:
    v = C.c_double(0)
    check(lib().qed2d_plaquette(_c(prm), _cp(U, prm), C.byref(v)))
    return v.value


def Qtop(U, prm: LattParm, kprm=None) -> float:
    v = C.c_double(0)
    check(lib().qed2d_qtop(_c(prm), _cp(U, prm), C.byref(v), None))
    return v.value


def Qtop_rounded(U, prm: LattParm) -> int:
    q = C.c_int64(0)
    check(lib().qed2d_qtop(_c(prm), _cp(U, prm), None, C.byref(q)))
    return q.value


def Hamiltonian(mom, U, prm: LattParm, kprm=None) -> float:
    v = C.c_double(0)
    check(lib().qed2d_hamiltonian(_c(prm), _rp(mom, prm), _cp(U, prm), C.byref(v)))
    return v.value


# ---------------------------------------------------------------------------
# fields and utilities
def unfold_fld_(Uin, prm: LattParm, kprm=None):
    """unfold_fld! (src/QED2dFields.jl:2-10): returns the (2 L1) x (2 L2) field."""
    L1, L2 = prm.iL
    Uout = torch.ones((2, 2 * L2, 2 * L1), dtype=torch.complex128, device=Uin.device)
    check(lib().qed2d_unfold(_c(prm), C.c_void_p(Uout.data_ptr()), _cp(Uin, prm), 0))
    return Uout


def unfold_reflect_(Uin, prm: LattParm, kprm=None):
    """unfold_reflect! (src/QED2dFields.jl:27-35)."""
    L1, L2 = prm.iL
    Uout = torch.ones((2, 2 * L2, 2 * L1), dtype=torch.complex128, device=Uin.device)
    check(lib().qed2d_unfold(_c(prm), C.c_void_p(Uout.data_ptr()), _cp(Uin, prm), 1))
    return Uout


def plwv(so, k, prm: LattParm):
    """plwv (src/QED2dUtils.jl:2-11)."""
    check(lib().qed2d_plwv(_c(prm), _cp(so, prm), float(k[0]), float(k[1])))


def random_normal(n, seed_, stream, counter, device="cuda", prm: LattParm = None):
    """n N(0,1) numbers of Philox stream (seed, stream, counter), as the library draws them."""
    out = torch.empty(int(n), dtype=torch.float64, device=device)
    h = _c(prm) if prm is not None else context(2, 2)
    check(lib().qed2d_random_normal(h, C.c_void_p(out.data_ptr()), int(n), int(seed_), int(stream), int(counter)))
    return out


def save_gauge(U, file: str, prm: LattParm):
    """save_gauge (src/QED2dLoadSave.jl:1-10): one 'Re<TAB>Im' line per link,
    i1 fastest, then i2, then mu (the reference's writedlm of reshape(U, 2V))."""
    from . import io
    io.save_gauge_text(U.detach().cpu().numpy(), file)


def load_gauge(U, file: str, prm: LattParm):
    """load_gauge (src/QED2dLoadSave.jl:12-19)."""
    from . import io
    arr = io.load_gauge_text(file, prm.iL[0], prm.iL[1])
    U.copy_(torch.from_numpy(arr).to(U.device))


# ---------------------------------------------------------------------------
# RHMC (src/QED2dRHMC.jl)
def get_rhmc_params(n_rhmc, r_a_rhmc, r_b_rhmc, reweighting_N=1, reweighting_Taylor=5):
    """get_rhmc_params (:93-121); list arguments give a list of RHMCParm."""
    if isinstance(n_rhmc, (list, tuple)):
        # the reference's array method forwards no keyword arguments (:112-121)
        return [get_rhmc_params(n, a, b) for n, a, b in zip(n_rhmc, r_a_rhmc, r_b_rhmc)]
    p = _lib.RhmcParams()
    check(lib().qed2d_get_rhmc_params(int(n_rhmc), float(r_a_rhmc), float(r_b_rhmc), C.byref(p)), "get_rhmc_params")
    r = RHMCParm.from_c(p)
    r.reweighting_N, r.reweighting_Taylor = int(reweighting_N), int(reweighting_Taylor)
    return r


# Zolotarev helpers exported by the reference (src/QED2dRHMC.jl:2-89), written on
# the library's Elliptic.K and Jacobi sn/cn (the reference calls Elliptic.jl).
# Host scalars; no device work.
def _ellip_K(m):
    K = C.c_double(0)
    check(lib().qed2d_ellip_K(float(m), C.byref(K)), "Elliptic.K")
    return K.value


def _sncn(u, m):
    s, c = C.c_double(0), C.c_double(0)
    check(lib().qed2d_ellip_sncn(float(u), float(m), C.byref(s), C.byref(c)), "Jacobi.sn/cn")
    return s.value, c.value


def k(eps):
    """k(eps) = sqrt(1 - eps) (:2)."""
    return math.sqrt(1.0 - eps)


def v(n, eps):
    """v(n, eps) = K(k^2) / (2n + 1) (:3)."""
    return _ellip_K(k(eps) ** 2) / (2.0 * n + 1.0)


def a_r(r, n, eps):
    """a_r = cn^2 / sn^2 at r v(n, eps) (:4)."""
    s, c = _sncn(r * v(n, eps), k(eps) ** 2)
    return c * c / (s * s)


def c_r(r, n, eps):
    """c_r = sn^2 at r v(n, eps) (:5)."""
    return _sncn(r * v(n, eps), k(eps) ** 2)[0] ** 2


def mu(j, n, eps, r_b):
    """mu_j = r_b sqrt(a_{2j}) (:8)."""
    return r_b * math.sqrt(a_r(2 * j, n, eps))


def nu(j, n, eps, r_b):
    """nu_j = r_b sqrt(a_{2j-1}) (:9)."""
    return r_b * math.sqrt(a_r(2 * j - 1, n, eps))


def rho_mu(j, k_, l, n, eps, r_b):
    """Residue of the pole at -mu_j^2, Luscher eq. (3.5) (:11-25)."""
    if j < k_ or j > l:
        raise ValueError("j is not between k and l")
    res = nu(j, n, eps, r_b) ** 2 - mu(j, n, eps, r_b) ** 2
    for m in range(k_, l + 1):
        if m != j:
            res *= (nu(m, n, eps, r_b) ** 2 - mu(j, n, eps, r_b) ** 2) / \
                   (mu(m, n, eps, r_b) ** 2 - mu(j, n, eps, r_b) ** 2)
    return res


def rho_nu(j, k_, l, n, eps, r_b):
    """Luscher eq. (3.9) (:27-41)."""
    if j < k_ or j > l:
        raise ValueError("j is not between k and l")
    res = mu(j, n, eps, r_b) - nu(j, n, eps, r_b)
    for m in range(k_, l + 1):
        if m != j:
            res *= (mu(m, n, eps, r_b) - nu(j, n, eps, r_b)) / (nu(m, n, eps, r_b) - nu(j, n, eps, r_b))
    return res


def P(k_, l, n, eps, r_b, Y):
    """P_{k,l}(Y) = 1 + sum_j rho_j (Y + mu_j^2)^-1, Luscher eq. (3.4) (:43-57); Y a
    scalar or a square matrix, the result a matrix (the reference also prints it)."""
    import numpy as np
    Y = np.atleast_2d(np.asarray(Y, dtype=float))
    eye = np.eye(Y.shape[1])
    res = eye.copy()
    if k_ != 0 and l != 0:
        for j in range(k_, l + 1):
            res = res + rho_mu(j, k_, l, n, eps, r_b) * np.linalg.inv(Y + mu(j, n, eps, r_b) ** 2 * eye)
    return res


def d(n, eps):
    """d(n, eps) (:60-68)."""
    res = k(eps) ** (2 * n + 1)
    for i in range(1, 2 * n + 2, 2):
        res *= c_r(i, n, eps) ** 2
    return res


def delta(n, eps):
    """Maximal relative error of the approximation (:70)."""
    dd = d(n, eps)
    return dd ** 2 / (1 + math.sqrt(1 - dd ** 2)) ** 2


def A(n, eps):
    """Normalisation A(n, eps) (:72-84)."""
    res = 2 / (1 + math.sqrt(1 - d(n, eps) ** 2))
    for i in range(1, 2 * n, 2):
        res *= c_r(i, n, eps)
    for i in range(2, 2 * n + 1, 2):
        res *= 1 / c_r(i, n, eps)
    return res


def error(Y, Yapprox):
    """|1 - sqrt(Y) Yapprox[1]| (:87-89), Yapprox[1] its first element."""
    import numpy as np
    return abs(1 - math.sqrt(Y) * np.asarray(Yapprox).flat[0])


def MultiCG(so, U, si, am0, maxiter, eps, A, rprm: RHMCParm, prm: LattParm, kprm=None):
    """MultiCG (:281-290)."""
    it = C.c_int(0)
    rp = rprm.to_c()
    check(lib().qed2d_multi_cg(_c(prm), _cp(so, prm), _cp(U, prm), _cp(si, prm), float(am0), int(maxiter),
                               float(eps), C.byref(rp), C.byref(it)), "MultiCG")
    return it.value


def R(so, U, si, am0, maxiter, eps, A, rprm: RHMCParm, prm: LattParm, kprm=None):
    """R (:261-271)."""
    it = C.c_int(0)
    rp = rprm.to_c()
    check(lib().qed2d_rational(_c(prm), _cp(so, prm), _cp(U, prm), _cp(si, prm), float(am0), int(maxiter),
                               float(eps), C.byref(rp), C.byref(it)), "R")
    return it.value


def generate_pseudofermion_(F, U, X, am0, CGmaxiter, CGtol, prm: LattParm, kprm, rprm: RHMCParm):
    """generate_pseudofermion! (:298-319)."""
    it = C.c_int(0)
    rp = rprm.to_c()
    check(lib().qed2d_generate_pseudofermion(_c(prm), _cp(F, prm), _cp(U, prm), _cp(X, prm), float(am0),
                                             int(CGmaxiter), float(CGtol), C.byref(rp), C.byref(it)),
          "generate_pseudofermion!")
    return it.value


def power_method(U, am0, prm: LattParm, kprm=None, iter: int = 1000):
    """power_method (:135-170): (lambda_min, lambda_max) of (g5Dw)^2."""
    lmin, lmax = C.c_double(0), C.c_double(0)
    check(lib().qed2d_power_method(_c(prm), _cp(U, prm), float(am0), int(iter), _rng["seed"], _next_counter(),
                                   C.byref(lmin), C.byref(lmax)), "power_method")
    return lmin.value, lmax.value


def LuscherZ(Z, U, X_in, am0, CGmaxiter, CGtol, rprm: RHMCParm, prm: LattParm, kprm=None):
    """LuscherZ (:174-186)."""
    rp = rprm.to_c()
    check(lib().qed2d_luscher_z(_c(prm), _cp(Z, prm), _cp(U, prm), _cp(X_in, prm), float(am0), int(CGmaxiter),
                                float(CGtol), C.byref(rp)), "LuscherZ")


def LuscherZp(Z, p: int, U, X_in, am0, CGmaxiter, CGtol, rprm: RHMCParm, prm: LattParm, kprm=None):
    """LuscherZp (:189-202): Z = ((g5Dw)^2 R^2 - 1)^p X_in, p applications of LuscherZ."""
    tmp = X_in.clone()
    for _ in range(int(p)):
        LuscherZ(Z, U, tmp, am0, CGmaxiter, CGtol, rprm, prm, kprm)
        tmp.copy_(Z)


def reweighting_factor(U, am0, CGmaxiter, CGtol, prm: LattParm, kprm, rprm):
    """reweighting_factor (:210-251); list arguments give the product over flavours."""
    if isinstance(am0, (list, tuple)):
        w = 1.0
        for m, r in zip(am0, rprm):
            w *= reweighting_factor(U, m, CGmaxiter, CGtol, prm, kprm, r)
        return w
    W = C.c_double(0)
    rp = rprm.to_c()
    check(lib().qed2d_reweighting_factor(_c(prm), _cp(U, prm), float(am0), int(CGmaxiter), float(CGtol),
                                         C.byref(rp), _rng["seed"], _next_counter(), C.byref(W)),
          "reweighting_factor")
    return W.value


# ---------------------------------------------------------------------------
# molecular dynamics (src/QED2dHMC.jl)
def OMF4_(mom, U, *args):
    """OMF4! -- pure gauge (:239-305): OMF4_(mom, U, eps, ns, prm, kprm);
    Nf=2 (:307-422): OMF4_(mom, U, X, F, g5DX, am0, eps, ns, maxiter, tol, prm, kprm)."""
    if len(args) == 4:
        eps, ns, prm, kprm = args
        check(lib().qed2d_omf4_gauge(_c(prm), _rp(mom, prm), _cp(U, prm), float(eps), int(ns)), "OMF4!")
        return None
    X, F, g5DX, am0, eps, ns, maxiter, tol, prm, kprm = args
    it = C.c_int64(0)
    check(lib().qed2d_omf4_nf2(_c(prm), _rp(mom, prm), _cp(U, prm), _cp(X, prm), _cp(F, prm), _cp(g5DX, prm),
                               float(am0), float(eps), int(ns), int(maxiter), float(tol), C.byref(it)), "OMF4!")
    return it.value


def _rhmc_arrays(F, am0, rprm):
    nf = len(am0)
    fp = (C.c_void_p * nf)(*[C.c_void_p(f.data_ptr()).value for f in F])
    am = (C.c_double * nf)(*[float(a) for a in am0])
    rp = (_lib.RhmcParams * nf)(*[r.to_c() for r in rprm])
    return nf, fp, am, rp


def leapfrog_(mom, U, X, F, g5DX, am0, eps, ns, CGmaxiter, tol, prm: LattParm, kprm=None, rprm=None):
    """leapfrog! -- Nf=2 (:426-449) or RHMC when rprm is given (:485-513)."""
    it = C.c_int64(0)
    if rprm is None:
        check(lib().qed2d_leapfrog_nf2(_c(prm), _rp(mom, prm), _cp(U, prm), _cp(X, prm), _cp(F, prm),
                                       _cp(g5DX, prm), float(am0), float(eps), int(ns), int(CGmaxiter), float(tol),
                                       C.byref(it)), "leapfrog!")
        return it.value
    nf, fp, am, rp = _rhmc_arrays(F, am0, rprm)
    check(lib().qed2d_leapfrog_rhmc(_c(prm), _rp(mom, prm), _cp(U, prm), _cp(X, prm), fp, _cp(g5DX, prm), nf, am,
                                    float(eps), int(ns), int(CGmaxiter), float(tol), rp, C.byref(it)), "leapfrog!")
    return it.value


def update_momenta_(mom, U, X, F, g5DX, am0, eps, ns, maxiter, tol, prm: LattParm, kprm=None, rprm=None):
    """update_momenta! -- Nf=2 (:452-481) or RHMC when rprm is given (:516-557)."""
    it = C.c_int64(0)
    if rprm is None:
        check(lib().qed2d_update_momenta_nf2(_c(prm), _rp(mom, prm), _cp(U, prm), _cp(X, prm), _cp(F, prm),
                                             _cp(g5DX, prm), float(am0), float(eps), int(maxiter), float(tol),
                                             C.byref(it)), "update_momenta!")
        return it.value
    nf, fp, am, rp = _rhmc_arrays(F, am0, rprm)
    check(lib().qed2d_update_momenta_rhmc(_c(prm), _rp(mom, prm), _cp(U, prm), _cp(X, prm), fp, _cp(g5DX, prm),
                                          nf, am, float(eps), int(maxiter), float(tol), rp, C.byref(it)),
          "update_momenta!")
    return it.value


@dataclass
class HMCInfo:
    accepted: int
    hini: float
    hfin: float
    dH: float
    qtop: float
    cg_iterations: int
    counter: int


def HMC_(U, *args, integrator: Integrators = None, qzero=False, reversibility_test=False, counter=None):
    """HMC! with the reference's three methods (src/QED2dHMC.jl:19-195):
        HMC_(U, eps, ns, acc, prm, kprm)                                   pure gauge (OMF4)
        HMC_(U, am0, eps, ns, acc, CGmaxiter, tol, prm, kprm)              Nf=2 (Leapfrog)
        HMC_(U, am0_list, eps, ns, acc, CGmaxiter, tol, prm, kprm, rprm)   RHMC (Leapfrog)
    Appends 1/0 to `acc` like the reference and returns an HMCInfo."""
    L = lib()
    res = _lib.HmcResult()
    ctr = _next_counter() if counter is None else int(counter)
    sd = _rng["seed"]
    if len(args) == 5:
        eps, ns, acc, prm, kprm = args
        integ = (integrator or OMF4()).code
        st = L.qed2d_hmc_gauge(_c(prm), _cp(U, prm), float(eps), int(ns), integ, int(bool(qzero)), sd, ctr,
                               C.byref(res))
    elif len(args) == 8:
        am0, eps, ns, acc, CGmaxiter, tol, prm, kprm = args
        integ = (integrator or Leapfrog()).code
        st = L.qed2d_hmc_nf2(_c(prm), _cp(U, prm), float(am0), float(eps), int(ns), integ, int(CGmaxiter),
                             float(tol), int(bool(qzero)), sd, ctr, C.byref(res))
    elif len(args) == 9:
        am0, eps, ns, acc, CGmaxiter, tol, prm, kprm, rprm = args
        nf = len(am0)
        am = (C.c_double * nf)(*[float(a) for a in am0])
        rp = (_lib.RhmcParams * nf)(*[r.to_c() for r in rprm])
        st = L.qed2d_hmc_rhmc(_c(prm), _cp(U, prm), nf, am, float(eps), int(ns), int(CGmaxiter), float(tol), rp,
                              int(bool(qzero)), int(bool(reversibility_test)), sd, ctr, C.byref(res))
    else:
        raise TypeError("HMC!: unsupported argument list")
    if st == _lib.NOT_CONVERGED:
        raise Qed2dError(st, "CG not converged")
    check(st, "HMC!")
    if not reversibility_test:
        acc.append(int(res.accepted))
    return HMCInfo(res.accepted, res.hini, res.hfin, res.dH, res.qtop, res.cg_iterations, ctr)


# ---------------------------------------------------------------------------
# batched replicas (no single reference counterpart; include/qed2d.h)
def _per_rep(v, n, name):
    if isinstance(v, (list, tuple)):
        if len(v) != n:
            raise ValueError(f"{name}: expected {n} values, got {len(v)}")
        return [float(x) for x in v]
    return [float(v)] * n


class Batch:
    """Independent replica lattices advanced together: Batch(nrep, L1, L2, beta)
    for nrep lattices of L1 x L2 sites, Batch.ragged([(L1, L2), ...], betas) for
    lattices of uneven sizes.  A batch field is replica-major: replica r's field
    is an ordinary reference-layout array at complex element 2*offsets[r].  For
    an equal-size batch field() has shape (nrep, 2, L2, L1) and field[r] is
    replica r; replica(t, r) gives that (2, L2_r, L1_r) view for every batch.
    Every replica follows HMC! Nf=2 with leapfrog (src/QED2dHMC.jl:64-113) using
    the mixed solver; replica r draws exactly as a single-lattice HMC_ with seed
    seeds[r]."""

    def __init__(self, nrep, L1, L2, beta, _sizes=None):
        self.sizes = list(_sizes) if _sizes is not None else [(int(L1), int(L2))] * int(nrep)
        self.nrep = len(self.sizes)
        self.uniform = len(set(self.sizes)) == 1
        self.L1, self.L2 = self.sizes[0]
        self.beta = _per_rep(beta, self.nrep, "beta")
        h = C.c_void_p()
        arr = (C.c_double * self.nrep)(*self.beta)
        if _sizes is None:
            check(lib().qed2d_batch_create(self.nrep, self.L1, self.L2, arr, C.byref(h)), "batch_create")
        else:
            l1 = (C.c_int * self.nrep)(*[s[0] for s in self.sizes])
            l2 = (C.c_int * self.nrep)(*[s[1] for s in self.sizes])
            check(lib().qed2d_batch_create_ragged(self.nrep, l1, l2, arr, C.byref(h)), "batch_create_ragged")
        self.h = h.value
        offs = (C.c_int64 * (self.nrep + 1))()
        check(lib().qed2d_batch_layout(self.h, offs), "batch_layout")
        self.offsets = list(offs)
        self.sites = self.offsets[-1]

    @classmethod
    def ragged(cls, sizes, beta):
        return cls(None, None, None, beta, _sizes=[(int(a), int(b)) for a, b in sizes])

    @property
    def schedule(self) -> int:
        """Schedule of the batched solver: -1 untuned; equal-size batches of at
        most 64 replicas 0/1 (reduction schedules), 4 (independent replicas, a
        barrier per replica), 5 (the same with a leaner reduction) or 7 (5 with
        the stencil operands staged by TMA; replicas of whole 32 x 8 or 32 x 16
        tiles), all with the same bits, or 8 (5 with the first phase's stencil
        applied to r, t = g5Dw r + beta t_old; agrees with 5 to solver
        accuracy) or 9 (8 with the links staged in shared memory once per
        solve; agrees with 8 to rounding); other batches 2 (one launch with grid barriers), 3 (one
        thread-block cluster per replica) or 6 (3 with the first phase's stencil
        on r)."""
        v = C.c_int(0)
        check(lib().qed2d_batch_get_schedule(self.h, C.byref(v)), "batch_get_schedule")
        return v.value

    @schedule.setter
    def schedule(self, s: int) -> None:
        check(lib().qed2d_batch_set_schedule(self.h, int(s)), "batch_set_schedule")

    @property
    def tile_rows(self) -> int:
        """Tile height of the equal-size solver (tiles of 32 x rows sites): 4, 8
        or 16, tuned with the schedule on the first solve (-1 until then)."""
        v = C.c_int(0)
        check(lib().qed2d_batch_get_tile_rows(self.h, C.byref(v)), "batch_get_tile_rows")
        return v.value

    @tile_rows.setter
    def tile_rows(self, rows: int) -> None:
        check(lib().qed2d_batch_set_tile_rows(self.h, int(rows)), "batch_set_tile_rows")

    @property
    def graphs(self) -> dict:
        """{"on", "captures", "replays", "failures"} of the batch's MD graph
        (CUDA-graph replay of the leapfrog inside hmc_nf2, on by default)."""
        return _stats(lib().qed2d_batch_graph_stats, self.h)

    @graphs.setter
    def graphs(self, on: bool) -> None:
        check(lib().qed2d_batch_set_graphs(self.h, 1 if on else 0), "batch_set_graphs")

    def field(self, dtype=torch.complex128):
        if self.uniform:
            return torch.zeros((self.nrep, 2, self.L2, self.L1), dtype=dtype, device="cuda")
        return torch.zeros(2 * self.sites, dtype=dtype, device="cuda")

    def replica(self, t, r):
        """(2, L2_r, L1_r) view of replica r of a batch field t."""
        L1, L2 = self.sizes[r]
        o = self.offsets[r]
        return t.reshape(-1)[2 * o: 2 * (o + L1 * L2)].view(2, L2, L1)

    def _check(self, t, name):
        if t.numel() != 2 * self.sites or t.dtype != torch.complex128 or not t.is_contiguous() or not t.is_cuda:
            raise ValueError(f"{name}: expected a contiguous CUDA complex128 batch field of {2 * self.sites} elements")

    def cg(self, x, U, b, am0, maxiter, eps):
        """Every replica's CG method 1 in one launch; returns (iterations, reliable updates) per replica."""
        for t, n in ((x, "x"), (U, "U"), (b, "b")):
            self._check(t, n)
        ams = _per_rep(am0, self.nrep, "am0")
        its, upd = (C.c_int * self.nrep)(), (C.c_int * self.nrep)()
        L = lib()
        check(L.qed2d_batch_set_stream(self.h, C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        st = L.qed2d_batch_cg(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(U.data_ptr()), C.c_void_p(b.data_ptr()),
                              (C.c_double * self.nrep)(*ams), int(maxiter), float(eps), its, upd)
        if st == _lib.NOT_CONVERGED:
            raise Qed2dError(st, "CG not converged")
        check(st, "batch CG")
        return list(its), list(upd)

    def hmc_nf2(self, U, am0, eps, ns, CGmaxiter, tol, seeds, counter, qzero=False):
        self._check(U, "U")
        ams = _per_rep(am0, self.nrep, "am0")
        if len(seeds) != self.nrep:
            raise ValueError(f"seeds: expected {self.nrep} values")
        res = (_lib.HmcResult * self.nrep)()
        L = lib()
        check(L.qed2d_batch_set_stream(self.h, C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        st = L.qed2d_batch_hmc_nf2(self.h, C.c_void_p(U.data_ptr()), (C.c_double * self.nrep)(*ams), float(eps),
                                   int(ns), int(CGmaxiter), float(tol), int(bool(qzero)),
                                   (C.c_uint64 * self.nrep)(*[int(s) for s in seeds]), int(counter), res)
        check(st, "batch HMC!")
        return [HMCInfo(r.accepted, r.hini, r.hfin, r.dH, r.qtop, r.cg_iterations, int(counter)) for r in res]

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().qed2d_batch_destroy(self.h)
        except Exception:
            pass
