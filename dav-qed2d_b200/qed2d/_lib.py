"""ctypes binding of libqed2d.so (include/qed2d.h).

The library is built in-tree by dav-qed2d_b200/build.py.  There is no fallback:
if the shared library is missing or fails to load, every call raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libqed2d.so")

MAXPOLES = 32
NOALLOC_MAX_SITES = 16384
OK, NOT_CONVERGED, TIMEOUT, BAD_ARG, CUDA_ERR, NO_MEMORY, UNSUPPORTED = range(7)
PREC_F64, PREC_MIXED, PREC_PLAIN = 0, 1, 2
MULTISHIFT = 3   # schedule selector of the multishift solver (QED2D_MULTISHIFT)
LEAPFROG, OMF4 = 0, 1
STREAM_MOMENTA, STREAM_METROPOLIS, STREAM_POWER, STREAM_NOISE, STREAM_REWEIGHT = 1, 3, 4, 16, 64


class RhmcParams(C.Structure):
    """qed2d_rhmc_params == RHMCParm (src/QED2d.jl:15-26)."""
    _fields_ = [
        ("r_b", C.c_double), ("n", C.c_int32), ("eps", C.c_double), ("A", C.c_double),
        ("rho", C.c_double * MAXPOLES), ("mu", C.c_double * MAXPOLES), ("nu", C.c_double * MAXPOLES),
        ("delta", C.c_double), ("reweighting_N", C.c_int32), ("reweighting_Taylor", C.c_int32),
    ]


class HmcResult(C.Structure):
    _fields_ = [("accepted", C.c_int32), ("hini", C.c_double), ("hfin", C.c_double), ("dH", C.c_double),
                ("qtop", C.c_double), ("cg_iterations", C.c_int64)]


P, D, I, I64, U64, U32 = C.c_void_p, C.c_double, C.c_int, C.c_int64, C.c_uint64, C.c_uint32
PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int)
PI64 = C.POINTER(C.c_int64)
PR = C.POINTER(RhmcParams)
PH = C.POINTER(HmcResult)
PP = C.POINTER(C.c_void_p)

SIGNATURES = {
    "qed2d_ctx_create": (I, [I, I, D, C.POINTER(C.c_void_p)]),
    "qed2d_ctx_destroy": (I, [P]),
    "qed2d_ctx_set_beta": (I, [P, D]),
    "qed2d_ctx_set_stream": (I, [P, P]),
    "qed2d_ctx_set_precision": (I, [P, I]),
    "qed2d_ctx_get_dims": (I, [P, PI, PI]),
    "qed2d_ctx_set_schedule": (I, [P, I, I]),
    "qed2d_ctx_get_schedule": (I, [P, I, PI]),
    "qed2d_ctx_set_multishift_layout": (I, [P, I]),
    "qed2d_ctx_get_multishift_layout": (I, [P, PI]),
    "qed2d_ctx_set_graphs": (I, [P, I]),
    "qed2d_ctx_graph_stats": (I, [P, PI, PI64, PI64, PI64]),
    "qed2d_last_solve": (I, [P, PI64, PD, PI64]),
    "qed2d_selftest_barrier_timeout": (I, [P, I64]),
    "qed2d_status_string": (C.c_char_p, [I]),
    "qed2d_last_error": (C.c_char_p, []),
    "qed2d_launch_count": (I64, []),
    "qed2d_plaquette_field": (I, [P, P, P]),
    "qed2d_qtop_field": (I, [P, P, P]),
    "qed2d_krnl_force": (I, [P, P, P, P]),
    "qed2d_updt_fld": (I, [P, P, P, D]),
    "qed2d_gamm5dw": (I, [P, P, P, P, D]),
    "qed2d_gamm5dw_c64": (I, [P, P, P, P, D]),
    "qed2d_gamm5": (I, [P, P, P]),
    "qed2d_dw": (I, [P, P, P, P, D]),
    "qed2d_gamm5dw_sqr": (I, [P, P, P, P, D]),
    "qed2d_gamm5dw_sqr_sqr": (I, [P, P, P, P, D]),
    "qed2d_gamm5dw_sqr_musq": (I, [P, P, P, P, D, D]),
    "qed2d_gamm5dw_sqr_sqr_musq": (I, [P, P, P, P, D, D]),
    "qed2d_tr_dqwdu": (I, [P, P, P, P, P]),
    "qed2d_unfold": (I, [P, P, P, I]),
    "qed2d_plwv": (I, [P, P, D, D]),
    "qed2d_random_normal": (I, [P, P, I64, U64, U32, U32]),
    "qed2d_random_uniform": (D, [U64, U32, U32]),
    "qed2d_action": (I, [P, P, PD]),
    "qed2d_plaquette": (I, [P, P, PD]),
    "qed2d_qtop": (I, [P, P, PD, PI64]),
    "qed2d_hamiltonian": (I, [P, P, P, PD]),
    "qed2d_cg": (I, [P, P, P, P, D, I, D, PI]),
    "qed2d_cg_shift": (I, [P, P, P, P, D, D, I, D, I, PI]),
    "qed2d_multishift_cg": (I, [P, PP, P, P, D, PD, I, I, D, PI]),
    "qed2d_cg_noalloc": (I, [I, I, P, P, P, D, I, D, P, PI]),
    "qed2d_get_rhmc_params": (I, [I, D, D, PR]),
    "qed2d_ellip_K": (I, [D, PD]),
    "qed2d_ellip_sncn": (I, [D, D, PD, PD]),
    "qed2d_multi_cg": (I, [P, P, P, P, D, I, D, PR, PI]),
    "qed2d_rational": (I, [P, P, P, P, D, I, D, PR, PI]),
    "qed2d_generate_pseudofermion": (I, [P, P, P, P, D, I, D, PR, PI]),
    "qed2d_power_method": (I, [P, P, D, I, U64, U32, PD, PD]),
    "qed2d_luscher_z": (I, [P, P, P, P, D, I, D, PR]),
    "qed2d_reweighting_factor": (I, [P, P, D, I, D, PR, U64, U32, PD]),
    "qed2d_omf4_gauge": (I, [P, P, P, D, I]),
    "qed2d_update_momenta_nf2": (I, [P, P, P, P, P, P, D, D, I, D, PI64]),
    "qed2d_leapfrog_nf2": (I, [P, P, P, P, P, P, D, D, I, I, D, PI64]),
    "qed2d_omf4_nf2": (I, [P, P, P, P, P, P, D, D, I, I, D, PI64]),
    "qed2d_update_momenta_rhmc": (I, [P, P, P, P, PP, P, I, PD, D, I, D, PR, PI64]),
    "qed2d_leapfrog_rhmc": (I, [P, P, P, P, PP, P, I, PD, D, I, I, D, PR, PI64]),
    "qed2d_hmc_gauge": (I, [P, P, D, I, I, I, U64, U32, PH]),
    "qed2d_hmc_nf2": (I, [P, P, D, D, I, I, I, D, I, U64, U32, PH]),
    "qed2d_hmc_rhmc": (I, [P, P, I, PD, D, I, I, D, PR, I, I, U64, U32, PH]),
    "qed2d_batch_create": (I, [I, I, I, PD, C.POINTER(C.c_void_p)]),
    "qed2d_batch_create_ragged": (I, [I, PI, PI, PD, C.POINTER(C.c_void_p)]),
    "qed2d_batch_layout": (I, [P, C.POINTER(C.c_int64)]),
    "qed2d_batch_set_schedule": (I, [P, I]),
    "qed2d_batch_get_schedule": (I, [P, PI]),
    "qed2d_batch_set_tile_rows": (I, [P, I]),
    "qed2d_batch_get_tile_rows": (I, [P, PI]),
    "qed2d_batch_set_graphs": (I, [P, I]),
    "qed2d_batch_graph_stats": (I, [P, PI, PI64, PI64, PI64]),
    "qed2d_batch_destroy": (I, [P]),
    "qed2d_batch_set_stream": (I, [P, P]),
    "qed2d_batch_cg": (I, [P, P, P, P, PD, I, D, PI, PI]),
    "qed2d_batch_hmc_nf2": (I, [P, P, PD, D, I, I, D, I, C.POINTER(C.c_uint64), U32, PH]),
}

_lib = None


class Qed2dError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


def lib():
    """Load libqed2d.so (raises if it is missing: there is no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libqed2d.so not built ({LIB_PATH}); run python dav-qed2d_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status, what=""):
    if status != OK:
        L = lib()
        msg = L.qed2d_last_error().decode() or L.qed2d_status_string(status).decode()
        raise Qed2dError(status, f"{what}: {msg}" if what else msg)
    return status
