"""Shared helpers for the parity tests: NumPy <-> CUDA tensors in the reference
layout and seeded inputs drawn from the Philox stream the library uses."""
import numpy as np

from oracle.oracle import Oracle


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
