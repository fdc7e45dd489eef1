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


# The FP32 parity bound: per particle, the path may be no further from the
# FP64 evaluation of the same interaction lists than the reference's own FP32
# arithmetic is (in either of two summation orders), plus 1e-5 of the force.
# A force well below the rms force is the cancellation of larger partial
# sums, whose FP32 rounding sets its error in any summation order (at 128^3,
# theta 0.7, the reference's kernels and their restatement, which differ only
# in order, deviate by 7e-6 and 2.8e-5 of |g| = 0.12 g_rms at one particle;
# the FP32 path here, whose M2L sums stay in FP32 where the reference sums
# them in FP64, by 1.5e-5 of |g| = 0.35 g_rms at another), so the 1e-5
# applies to max(|g|, g_rms / 2).  The potential takes 1e-5 of |phi| with a
# floor of 1e-6 of the rms potential (periodic potentials cross zero).
ARBITER_REL = 1e-5
ARBITER_G_FLOOR = 0.5
ARBITER_PHI_FLOOR = 1e-6


def arbiter_excess(g, g_ref, g64, phi=None, phi_ref=None, phi64=None, g_alt=None, phi_alt=None):
    """Largest violation of |x - x64| <= |x_ref - x64| + tol over the particles,
    in units of the tolerance term (<= 0 everywhere: the bound holds).
    g_alt / phi_alt: the reference's arithmetic summed in another order (the
    oracle's restatement); the reference's own FP32 deviation at a particle is
    then the larger of the two orders' (FP32 rounding makes it depend on the
    order of the sums: at 128^3, theta 0.7, 4.3e-6 and 1.3e-5 of |g| at one
    particle).  Returns (force excess, potential excess or None)."""
    n64 = np.linalg.norm(g64, axis=1)
    scale = np.maximum(n64, ARBITER_G_FLOOR * np.sqrt(np.mean(n64 ** 2)))
    lhs = np.linalg.norm(g - g64, axis=1)
    dev = np.linalg.norm(g_ref - g64, axis=1)
    if g_alt is not None:
        dev = np.maximum(dev, np.linalg.norm(g_alt - g64, axis=1))
    rhs = dev + ARBITER_REL * scale
    fx = float(np.max((lhs - rhs) / np.maximum(ARBITER_REL * scale, 1e-300)))
    if phi is None:
        return fx, None
    tol = ARBITER_REL * np.abs(phi64) + ARBITER_PHI_FLOOR * np.sqrt(np.mean(phi64 ** 2))
    pdev = np.abs(phi_ref - phi64)
    if phi_alt is not None:
        pdev = np.maximum(pdev, np.abs(phi_alt - phi64))
    px = float(np.max((np.abs(phi - phi64) - pdev - tol) / tol))
    return fx, px
