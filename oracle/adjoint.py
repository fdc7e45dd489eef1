"""Oracle (test infrastructure only): an FP64 reference gradient of the
leapfrog through all-pairs periodic gravity, for checking tg_backward.

The library's adjoint (tg_forward / tg_backward) differentiates kick-drift-
kick steps through the tree forces.  Where every interaction is a pair
(theta small enough that all lists are PP direct + PP Ewald), the forces are
g_i = sum_j m G(x_i - x_j) with

  G(d) = -d f(|d|)               the spline-softened direct force of
                                 gravity_PP_direct (src/gravity.cpp:231-256),
                                 d the nearest image (periodic) or the plain
                                 difference (free space)
       + e(d)  (periodic only)   the Ewald correction of gravity_PP_ewald
                                 (src/gravity.cpp:491-614, tigergrav/green.hpp
                                 189-286): the real-space images |n|^2 <= 17
                                 cut at 3.6, erfc(2r); the reciprocal vectors
                                 |h|^2 <= 9; the nearest image's 1/r removed

and the Jacobian is J u_i = sum_j m H(x_i - x_j) (u_i - u_j), H = dG/dd,
written here analytically in FP64 (numpy), independently of the CUDA code.
`reference_gradient` runs the oracle's FP64 stepper (restated kick / drift,
FP64 kernels) forward, keeping the positions where forces are evaluated, and
the reverse-mode recursion of one KDK step backward:

  lx += dt/2 G J(x_1) lv;  lv += dt lx;  lx += dt/2 G J(x_0) lv

(J is symmetric for pair forces).  The fixed-point requantisation of each
drift is treated as the identity, as the library's adjoint does.
"""
import numpy as np

SQRT_PI = np.sqrt(np.pi)


def _lattice(n2max):
    k = int(np.sqrt(n2max)) + 1
    r = np.arange(-k, k + 1)
    g = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
    return g[(g * g).sum(1) <= n2max].astype(np.float64)


REAL = _lattice(17)          # 305 lattice vectors (tigergrav/green.hpp ewald_indices)
FOUR = _lattice(9)
FOUR = FOUR[(FOUR * FOUR).sum(1) > 0]  # the h = 0 term carries nothing


def nearest(d):
    """nearest-image separation in the unit box"""
    return d - np.round(d)


def direct_force_hessian(d, h):
    """d: (M, 3) nearest-image separations.  Returns (G, H) of the softened
    direct force G(d) = -d f(r) (per unit source mass) and H = dG/dd."""
    r = np.sqrt((d * d).sum(1))
    x = np.minimum(r / h, 1.0)
    # the spline of src/gravity.cpp:231-256 and its r-derivative
    f1 = 1.0 / np.maximum(r, 1e-300) ** 3
    df1 = -3.0 / np.maximum(r, 1e-300) ** 4
    P = (((-32.0 / 3.0 * x + 192.0 / 5.0) * x - 48.0) * x + 64.0 / 3.0) * x ** 3 - 1.0 / 15.0
    dP = ((-64.0 * x + 192.0) * x - 192.0) * x ** 3 + 64.0 * x * x  # dP/dx
    rc = np.maximum(r, 0.5 * h)
    f2 = P / rc ** 3
    df2 = dP / h / rc ** 3 - 3.0 * P / rc ** 4
    f3 = (32.0 * x ** 3 - 192.0 / 5.0 * x * x + 32.0 / 3.0) / h ** 3
    df3 = (96.0 * x * x - 384.0 / 5.0 * x) / h ** 4
    far, near = r > h, r < 0.5 * h
    f = np.where(far, f1, np.where(near, f3, f2))
    df = np.where(far, df1, np.where(near, df3, df2))
    G = -d * f[:, None]
    rr = np.maximum(r, 1e-300)[:, None, None]
    H = -np.eye(3)[None] * f[:, None, None] - (d[:, :, None] * d[:, None, :]) * (df[:, None, None] / rr)
    H[r == 0] = 0.0
    return G, H


def ewald_force_hessian(d):
    """The Ewald correction e(d) of the reference (d nearest image, |d| >= 1e-6)
    and its derivative de/dd, FP64."""
    M = len(d)
    G = np.zeros((M, 3))
    H = np.zeros((M, 3, 3))
    for n in REAL:
        dd = d - n
        r = np.sqrt((dd * dd).sum(1))
        use = r < 3.6
        r_ = np.where(use, r, 1.0)
        erfc = _erfc(2.0 * r_)
        e = np.exp(-4.0 * r_ * r_)
        F = (4.0 / SQRT_PI * r_ * e + erfc) / r_ ** 3
        dF = -32.0 / SQRT_PI * e / r_ - 3.0 * F / r_
        F = np.where(use, F, 0.0)
        dF = np.where(use, dF, 0.0)
        G -= dd * F[:, None]
        H -= np.eye(3)[None] * F[:, None, None] + (dd[:, :, None] * dd[:, None, :]) * (dF / r_)[:, None, None]
    for hv in FOUR:
        h2 = (hv * hv).sum()
        c0 = np.exp(-np.pi ** 2 * h2 / 4.0) / h2
        om = 2.0 * np.pi * (d @ hv)
        G -= 2.0 * c0 * np.sin(om)[:, None] * hv[None]
        H -= (4.0 * np.pi * c0 * np.cos(om))[:, None, None] * (hv[:, None] * hv[None, :])[None]
    r = np.sqrt((d * d).sum(1))
    G += d / r[:, None] ** 3
    H += np.eye(3)[None] / r[:, None, None] ** 3 - 3.0 * (d[:, :, None] * d[:, None, :]) / r[:, None, None] ** 5
    return G, H


def _erfc(x):
    from scipy.special import erfc
    return erfc(x)


def pair_hessians(x, m, h, ewald=True):
    """m H(x_i - x_j) for every pair i != j, as a dense (N, N, 3, 3) array
    (zero on the diagonal)."""
    n = len(x)
    i, j = np.nonzero(~np.eye(n, dtype=bool))
    d = nearest(x[i] - x[j]) if ewald else x[i] - x[j]  # free space: the plain difference
    _, H = direct_force_hessian(d, h)
    if ewald:
        H = H + ewald_force_hessian(d)[1]
    out = np.zeros((n, n, 3, 3))
    out[i, j] = m * H
    return out


def jvp(Hp, u):
    """J u with J_i = sum_j Hp[i, j] (u_i - u_j) (Hp from pair_hessians)"""
    return np.einsum("ijab,ib->ia", Hp, u) - np.einsum("ijab,jb->ia", Hp, u)


def forces(x, m, h, ewald=True):
    """g_i = sum_j m G(x_i - x_j) (FP64; for checking the Hessians by differences)"""
    n = len(x)
    i, j = np.nonzero(~np.eye(n, dtype=bool))
    d = nearest(x[i] - x[j]) if ewald else x[i] - x[j]
    G, _ = direct_force_hessian(d, h)
    if ewald:
        G = G + ewald_force_hessian(d)[0]
    out = np.zeros((n, 3))
    np.add.at(out, i, m * G)
    return out


def reference_gradient(oracle_mod, x0, w, dt, steps, theta=0.1, G=1.0, ewald=True):
    """dL/dx(0) for L = sum w . x(T) after `steps` KDK steps of the oracle's FP64
    stepper (positions x0 as int32 fixed point, zero initial velocity)."""
    n = len(x0)
    m, h = 1.0 / n, 0.02 * n ** (-1.0 / 3.0)
    o = oracle_mod.Oracle(theta=theta, ewald=ewald).set_particles(x0)
    o.build().multipoles().walk().evaluate(fp64=True)
    xs = [oracle_mod_pos(o)]
    for _ in range(steps):
        o.kick(0.5 * dt)
        o.drift(dt)
        o.build().multipoles().walk().evaluate(fp64=True)
        o.kick(0.5 * dt)
        xs.append(oracle_mod_pos(o))
    lx = np.array(w, np.float64)
    lv = np.zeros_like(lx)
    for s in range(steps, 0, -1):
        lx = lx + 0.5 * dt * G * jvp(pair_hessians(xs[s], m, h, ewald), lv)
        lv = lv + dt * lx
        lx = lx + 0.5 * dt * G * jvp(pair_hessians(xs[s - 1], m, h, ewald), lv)
    return lx, lv


def oracle_mod_pos(o):
    x, _ = o.particles()
    return x.astype(np.float64) / 4294967296.0 + 0.5
