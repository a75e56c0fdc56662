"""Shared comparison helpers for the parity tests."""
import numpy as np


def max_rel(a, b):
    """Largest relative difference per column, where each column is scaled by
    the larger of |b| and 1e-3 of the column's largest |b|: prim velocity
    components pass through zero, density and pressure do not."""
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    a2 = a.reshape(a.shape[0], -1)
    b2 = b.reshape(b.shape[0], -1)
    floor = 1e-3 * np.max(np.abs(b2), axis=0)
    scale = np.maximum(np.abs(b2), np.maximum(floor, 1e-300))
    return float(np.max(np.abs(a2 - b2) / scale))


def max_scaled(a, b, floor=1e-4):
    """max over columns of |a-b| / max(max|b| of that column, floor): for
    arrays whose entries pass through zero (dq, flux_res) or vanish."""
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    a2 = a.reshape(a.shape[0], -1)
    b2 = b.reshape(b.shape[0], -1)
    scale = np.maximum(np.max(np.abs(b2), axis=0), floor)
    return float(np.max(np.abs(a2 - b2) / scale))
