"""Shared helpers for the parity tests (CPU oracle vs the CUDA library)."""
import numpy as np


def rel_force_err(g, gref):
    """per-particle |dg| / |g_ref| (the reference's compute_error metric, src/output.cpp:33-35)"""
    return np.linalg.norm(g - gref, axis=1) / np.maximum(np.linalg.norm(gref, axis=1), 1e-300)


def leaf_members(nodes, perm):
    """{boxid: sorted caller indices} for every non-empty leaf"""
    out = {}
    for i in np.nonzero(nodes["child0"] < 0)[0]:
        b, e = nodes["pbegin"][i], nodes["pend"][i]
        if e > b:
            out[int(nodes["boxid"][i])] = np.sort(perm[b:e])
    return out
