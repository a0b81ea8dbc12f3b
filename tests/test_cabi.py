"""CPU checks of the drop-in boundary: libqed2d.so loads, exports every entry
point that include/qed2d.h declares, the Python mirror binds all of them, the
host-only entry points work without a GPU, and the checkpoint text format
round-trips."""
import os
import re
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "qed2d.h")
LIB = os.path.join(REPO, "dav-qed2d_b200", "lib", "libqed2d.so")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(qed2d_[A-Za-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def built():
    if not os.path.exists(LIB):
        subprocess.run(["python", os.path.join(REPO, "dav-qed2d_b200", "build.py")], check=True)
    return LIB


def test_library_exports_every_declared_symbol(built):
    out = subprocess.check_output(["nm", "-D", "--defined-only", built]).decode()
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    missing = [s for s in declared() if s not in exported]
    assert not missing, missing


def test_python_mirror_binds_every_symbol(built):
    from qed2d import _lib
    L = _lib.lib()
    assert set(declared()) == set(_lib.SIGNATURES)
    for s in declared():
        assert getattr(L, s) is not None


def test_host_entry_points_without_gpu(built):
    import ctypes as C
    from qed2d import _lib
    from oracle.oracle import Oracle, zolotarev
    L = _lib.lib()
    # Metropolis uniform: same Philox stream as the oracle
    for args in [(1234, 3, 0), (2**63 + 17, 3, 99), (0, 1, 2**32 - 1)]:
        assert L.qed2d_random_uniform(*args) == Oracle.uniform(*args)
    # Zolotarev coefficients: host code, compared with the oracle
    p = _lib.RhmcParams()
    assert L.qed2d_get_rhmc_params(12, 0.1, 5.0, C.byref(p)) == 0
    r = zolotarev(12, 0.1, 5.0)
    for k in range(12):
        assert abs(p.mu[k] - r.mu[k]) < 1e-13 * r.mu[k]
        assert abs(p.rho[k] - r.rho[k]) < 1e-12 * abs(r.rho[k])
    assert L.qed2d_get_rhmc_params(0, 0.1, 5.0, C.byref(p)) == _lib.BAD_ARG
    assert L.qed2d_get_rhmc_params(3, 5.0, 0.1, C.byref(p)) == _lib.BAD_ARG
    # NULL context is rejected, not dereferenced
    assert L.qed2d_ctx_set_beta(None, 1.0) == _lib.BAD_ARG
    assert L.qed2d_status_string(_lib.NOT_CONVERGED) == b"CG not converged"


def test_gauge_checkpoint_roundtrip(tmp_path):
    from qed2d.io import julia_float, load_gauge_text, save_gauge_text
    assert julia_float(1.0) == "1.0" and julia_float(1e-5) == "1.0e-5" and julia_float(-0.25) == "-0.25"
    assert julia_float(1.5e20) == "1.5e20"
    U = np.exp(1j * np.random.default_rng(0).uniform(-np.pi, np.pi, (2, 3, 4)))
    f = tmp_path / "config_4_3_b4.0_m0.1_n100"
    save_gauge_text(U, str(f))
    lines = f.read_text().splitlines()
    assert len(lines) == 24 and all(len(l.split("\t")) == 2 for l in lines)
    # Julia column-major order: first lines are U[1,1,1], U[2,1,1], ...
    assert float(lines[1].split("\t")[0]) == U[0, 0, 1].real
    assert np.array_equal(load_gauge_text(str(f), 4, 3), U)


def prototypes():
    """{name: number of parameters} of every prototype in include/qed2d.h."""
    txt = re.sub(r"/\*.*?\*/", " ", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(qed2d_[A-Za-z0-9_]+)\s*\(([^;{]*?)\)\s*;", txt):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_python_signatures_match_header_arity(built):
    """Every ctypes signature of the Python mirror passes as many arguments as the
    header's prototype declares (a dropped or extra argument would shift every
    later one)."""
    from qed2d import _lib
    protos = prototypes()
    assert set(protos) == set(declared())
    wrong = {s: (len(_lib.SIGNATURES[s][1]), n) for s, n in protos.items() if len(_lib.SIGNATURES[s][1]) != n}
    assert not wrong, wrong


def test_graph_entry_points_reject_null_handles(built):
    """The CUDA-graph controls reject a NULL context or batch without touching a GPU."""
    from qed2d import _lib
    L = _lib.lib()
    assert L.qed2d_ctx_set_graphs(None, 1) == _lib.BAD_ARG
    assert L.qed2d_ctx_graph_stats(None, None, None, None, None) == _lib.BAD_ARG
    assert L.qed2d_batch_set_graphs(None, 0) == _lib.BAD_ARG
    assert L.qed2d_batch_graph_stats(None, None, None, None, None) == _lib.BAD_ARG
