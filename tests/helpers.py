"""Shared helpers for the parity tests: NumPy <-> CUDA tensors in the reference
layout, seeded inputs drawn from the Philox stream the library uses, and the
bound check that records every achieved error."""
import json
import os

import numpy as np

from oracle.oracle import Oracle


def bound(quantity, err, limit):
    """Assert err <= limit.  With QED2D_PARITY_LOG set, append the achieved
    error, the bound and the test id as one JSON line to that file, so every
    parity case reports what it measured, not only that it passed."""
    err = float(err)
    path = os.environ.get("QED2D_PARITY_LOG")
    if path:
        test = os.environ.get("PYTEST_CURRENT_TEST", "?").split(" ")[0]
        with open(path, "a") as fh:
            fh.write(json.dumps({"test": test, "quantity": quantity, "err": err, "bound": float(limit)}) + "\n")
    assert err <= limit, f"{quantity}: {err:.3e} > {limit:.1e}"


def note(quantity, value):
    """Record an informational figure (no assertion) beside the bounds."""
    path = os.environ.get("QED2D_PARITY_LOG")
    if path:
        test = os.environ.get("PYTEST_CURRENT_TEST", "?").split(" ")[0]
        with open(path, "a") as fh:
            fh.write(json.dumps({"test": test, "quantity": quantity, "value": value}) + "\n")


def cgauss(L1, L2, seed, stream, counter=0):
    """(randn + i randn)/sqrt(2), shape (2, L2, L1), from the shared Philox stream."""
    z = Oracle.normal(4 * L1 * L2, seed, stream, counter)
    return ((z[0::2] + 1j * z[1::2]) / np.sqrt(2.0)).reshape(2, L2, L1)


def hot_links(L1, L2, seed):
    rng = np.random.default_rng(seed)
    return np.exp(1j * rng.uniform(-np.pi, np.pi, (2, L2, L1)))


def to_dev(a):
    import torch
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a).cuda()


def to_host(t):
    return t.detach().cpu().numpy()


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
