"""The FP64 reference gradient of the oracle (oracle/adjoint.py) and the
library's adjoint against it.

CPU: the analytic pair Hessians (softened direct force and Ewald correction)
against central differences of the same FP64 forces in continuous
coordinates.  GPU: tg_backward (FP64 path) on an all-pairs configuration
(theta 0.1: every interaction is PP direct + PP Ewald) against the reference
gradient of the oracle's FP64 stepper, on the whole gradient and on its
non-identity part (the gradient minus w)."""
import numpy as np
import pytest

import adjoint as oadj


def test_pair_hessians_match_differences():
    rng = np.random.default_rng(3)
    n = 24
    x = rng.random((n, 3))
    x[1] = x[0] + np.array([1e-3, -4e-4, 2e-4])   # inside the softening length
    x[2] = x[0] + np.array([0.006, 0.002, -0.001])  # in the spline's outer branch
    m, h = 1.0 / n, 0.01
    u = rng.standard_normal((n, 3))
    ju = oadj.jvp(oadj.pair_hessians(x, m, h), u)
    # the differences' truncation error falls as eps^2 (2.3e-5 at 1e-5,
    # 2.4e-9 at 1e-7: the close pairs' third derivatives)
    eps = 1e-7
    fd = (oadj.forces(x + eps * u, m, h) - oadj.forces(x - eps * u, m, h)) / (2 * eps)
    err = np.linalg.norm(ju - fd) / np.linalg.norm(fd)
    assert err < 1e-7, err
    # the Ewald part is the oracle's FP64 correction (the reference's green_ewald)
    import oracle
    d = oadj.nearest(x[3] - x[5])
    assert np.allclose(oadj.ewald_force_hessian(d[None])[0][0], oracle.ewald_corr_f64(d)[1:], rtol=1e-12, atol=0)


def test_lattice_sizes():
    assert len(oadj.REAL) == 305  # the reference's real-space index set (|n|^2 <= 17)
    assert len(oadj.FOUR) == 122  # |h|^2 <= 9 without h = 0


@pytest.mark.gpu
@pytest.mark.parametrize("ewald", [True, False])
def test_backward_matches_fp64_reference_gradient(oracle_mod, ewald):
    import tigergrav_b200 as tg
    from tigergrav_b200 import ics
    x0 = ics.clustered(6, 3)  # 216 particles
    n = len(x0)
    w = np.random.default_rng(6).standard_normal((n, 3))
    dt, steps = 1e-3, 3
    with tg.GravitySolver(n, theta=0.1, ewald=ewald, precision="f64") as s:
        s.set_particles(x0).forward(dt, steps)
        gx0, gv0 = s.backward(w)
    rx, rv = oadj.reference_gradient(oracle_mod, x0, w, dt, steps, theta=0.1, ewald=ewald)
    assert np.linalg.norm(gx0 - rx) / np.linalg.norm(rx) < 1e-9
    # the non-identity part (the force term), on its own scale
    assert np.linalg.norm((gx0 - w) - (rx - w)) / np.linalg.norm(rx - w) < 1e-6
    assert np.linalg.norm(gv0 - rv) / np.linalg.norm(rv) < 1e-6
