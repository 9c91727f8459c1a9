"""Shared helpers for the tests (seeded inputs, error norms)."""
import numpy as np


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    dt = np.complex128 if (np.iscomplexobj(a) or np.iscomplexobj(b)) else np.float64
    a = a.astype(dt)
    b = b.astype(dt)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def phantom_stack(S, n, seed=0):
    from oracle import oracle as O
    return np.stack([O.ellipse_phantom(n, 10, seed + s) for s in range(S)]).astype(np.float32)
