"""Differentiation of the leapfrog through the tree forces (tg_forward /
tg_backward / tg_tidal) against central finite differences of the FP64
forward path.

The reference has no adjoint; the checks follow the workload that the task
states for it: 64^3 clustered particles (seed 5), L = sum_i w_i . x_i(T) with
w_i ~ N(0, 1) (seed 6), 8 leapfrog steps at dt = 1e-3, central differences
with h = 1e-4 in box units on 32 sampled coordinates (seed 7).  A tree force
is only piecewise smooth: a sample whose +h and -h runs produce different
interaction lists is not a derivative and is skipped (counted).
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P32 = 4294967296.0


def _p2d(x):
    return np.asarray(x, np.int32).astype(np.float64) / P32 + 0.5


def test_tidal_matches_fd_of_direct_forces():
    """theta = 0.1 on 4096 particles: every interaction is a PP pair (direct +
    Ewald), so J u must match the central difference of the forces."""
    import tigergrav_b200 as tg
    from tigergrav_b200 import ics
    x = ics.uniform(4096, 1)
    n = len(x)
    u = np.random.default_rng(11).standard_normal((n, 3))
    eps = 1e-6
    with tg.GravitySolver(n, theta=0.1, ewald=True, leaf_max=64, precision="f64") as s:
        xd = _p2d(x)
        xp = ics.double_to_pos((xd + eps * u) % 1.0)
        xm = ics.double_to_pos((xd - eps * u) % 1.0)
        ueff = (((_p2d(xp) - xd + 0.5) % 1.0 - 0.5) - ((_p2d(xm) - xd + 0.5) % 1.0 - 0.5)) / (2 * eps)
        s.set_particles(xp).solve_gravity()
        _, gp = s.get_forces()
        s.set_particles(xm).solve_gravity()
        _, gm = s.get_forces()
        fd = (gp - gm) / (2 * eps)
        s.set_particles(x).solve_gravity()
        ju = s.tidal(ueff)
    err = np.linalg.norm(ju - fd) / np.linalg.norm(fd)
    assert err < 1e-4, err


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_adjoint_matches_central_fd(precision):
    import torch
    import tigergrav_b200 as tg
    from tigergrav_b200 import ics
    x0 = ics.clustered(64, 5)
    n = len(x0)
    w = np.random.default_rng(6).standard_normal((n, 3))
    dt, steps, h = 1e-3, 8, 1e-4
    with tg.GravitySolver(n, theta=0.7, ewald=True, leaf_max=64, precision=precision) as s:
        s.set_particles(x0)
        s.forward(dt, steps)
        s.set_particles(x0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.forward(dt, steps)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        gx0, _ = s.backward(w)
        t2 = time.perf_counter()
    assert (t2 - t1) <= 3.0 * (t1 - t0), ((t2 - t1), (t1 - t0))
    xd0 = _p2d(x0)
    fds = tg.GravitySolver(n, theta=0.7, ewald=True, leaf_max=64, precision="f64")

    def loss(xpos):
        fds.set_particles(xpos).solve_gravity()
        sig = []
        for _ in range(steps):
            fds.kick(0.5 * dt)
            fds.drift(dt)
            fds.solve_gravity()
            fds.kick(0.5 * dt)
            sig.append(tuple(fds.stats()["counts"].values()))
        xt, _ = fds.get_particles()
        disp = (_p2d(xt) - xd0 + 0.5) % 1.0 - 0.5
        return float(np.sum(w * (xd0 + disp))), tuple(sig)

    rng = np.random.default_rng(7)
    idx = rng.choice(n, 32, replace=False)
    dims = rng.integers(0, 3, 32)

    def central(hstep, samples):
        errs, nonid, skipped = [], [], 0
        for i, d in samples:
            xp, xm = x0.copy(), x0.copy()
            xp[i, d] = ics.double_to_pos(np.array([xd0[i, d] + hstep]))[0]
            xm[i, d] = ics.double_to_pos(np.array([xd0[i, d] - hstep]))[0]
            hh = ((_p2d(xp[i, d]) - _p2d(xm[i, d]) + 0.5) % 1.0) - 0.5
            (lp, sp), (lm, sm) = loss(xp), loss(xm)
            if sp != sm:
                skipped += 1
                continue
            fd = (lp - lm) / hh
            errs.append(abs(gx0[i, d] - fd) / abs(fd))
            nonid.append(abs((gx0[i, d] - w[i, d]) - (fd - w[i, d])) / abs(fd - w[i, d]))
        return np.array(errs), np.array(nonid), skipped

    errs, _, skipped = central(h, list(zip(idx, dims)))
    assert skipped <= 8
    assert np.median(errs) <= 1e-4, np.median(errs)
    assert np.percentile(errs, 90) <= 1e-3, np.percentile(errs, 90)
    # The force term alone: dL/dx0 - w is ~2e-4 |w|, the size of the
    # fixed-point requantisation noise of the difference at h = 1e-4 (every
    # drift rounds to 2^-32); at h = 1e-3 that noise is 10x smaller and the
    # non-identity part is judged on its own (measured median 6% here, 2% at
    # 16^3, where the tree approximation of J and the noise are both smaller).
    _, nonid, skipped = central(1e-3, list(zip(idx, dims))[:16])
    fds.close()
    assert skipped <= 6
    assert np.median(nonid) <= 0.15, np.median(nonid)
