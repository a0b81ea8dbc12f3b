"""Host-side file formats of the reference drivers.

* Gauge checkpoints of save_gauge/load_gauge (src/QED2dLoadSave.jl:1-19): a
  ``writedlm`` text file of 2*L1*L2 lines ``Re<TAB>Im``, links in Julia
  column-major order (i1 fastest, then i2, then the direction), floats printed
  the way Julia prints a Float64 (shortest round-trip digits, ``1.0e-5`` style
  exponents).
"""
import numpy as np


def julia_float(x: float) -> str:
    """Float64 text as Julia's `print` writes it (shortest round trip)."""
    x = float(x)
    if x != x:
        return "NaN"
    if x in (float("inf"), float("-inf")):
        return "Inf" if x > 0 else "-Inf"
    s = repr(x)
    if "e" in s or "E" in s:
        mant, exp = s.lower().split("e")
        if "." not in mant:
            mant += ".0"
        return f"{mant}e{int(exp)}"
    if "." not in s:
        s += ".0"
    return s


def save_gauge_text(U: np.ndarray, path: str) -> None:
    """U: complex128 array of shape (2, L2, L1) (the reference layout)."""
    flat = np.ascontiguousarray(U).reshape(-1)
    with open(path, "w") as fh:
        for z in flat:
            fh.write(f"{julia_float(z.real)}\t{julia_float(z.imag)}\n")


def load_gauge_text(path: str, L1: int, L2: int) -> np.ndarray:
    data = np.loadtxt(path, dtype=np.float64, ndmin=2)
    if data.shape != (2 * L1 * L2, 2):
        raise ValueError(f"{path}: expected {2 * L1 * L2} rows of (Re, Im), got {data.shape}")
    return (data[:, 0] + 1j * data[:, 1]).reshape(2, L2, L1)
