"""Shared helpers for the parity tests (tests only)."""
import numpy as np


def to_original(solver, name):
    """Per-particle field of a pbf_b200 Solver in original particle order, xyz only."""
    a = solver.fetch_original(name)
    return a[:, :3] if a.ndim == 2 else a


def oracle_original(orc, name):
    """Oracle field (reorder mode: slot order) in original particle order."""
    a = orc.get(name)
    perm = orc.get("perm")
    out = np.empty_like(a)
    out[perm] = a
    return out


def bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def mismatch(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    bad = a.view(np.uint32) != b.view(np.uint32)
    return int(bad.sum()), float(np.abs(a.astype(np.float64) - b).max()) if a.size else 0.0
