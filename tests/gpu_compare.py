"""Comparison helpers of the GPU parity tests (CUDA path vs CPU oracle)."""
import numpy as np


def interior(a, dims, ngg=2):
    mx, my, mz = dims
    return a.reshape(a.shape[0], mz + 2 * ngg, my + 2 * ngg, mx + 2 * ngg)[:, ngg:-ngg, ngg:-ngg, ngg:-ngg].reshape(
        a.shape[0], -1)


def group_errors(a, b, groups):
    """Max |a-b| / scale per named group of rows; the scale of a group is the
    largest |b| over all its rows (so an all-zero transverse velocity is
    measured against the velocity magnitude)."""
    out = {}
    for name, rows in groups.items():
        if len(rows) == 0:
            continue
        ref = b[rows]
        scale = max(float(np.abs(ref).max()), 1e-300)
        out[name] = float(np.abs(a[rows] - ref).max() / scale)
    return out


def bv_groups():
    return {"rho": [0], "vel": [1, 2, 3], "p": [4], "T": [5]}


def cv_groups(ns):
    g = {"rho": [0], "mom": [1, 2, 3], "rhoE": [4]}
    if ns:
        g["rhoY"] = list(range(5, 5 + ns))
    return g


def l2_rel(a, b):
    """Relative L2 error per row: ||a-b||_2 / ||b||_2."""
    return np.linalg.norm(a - b, axis=-1) / np.maximum(np.linalg.norm(b, axis=-1), 1e-300)
