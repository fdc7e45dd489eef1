"""Seeded synthetic particle sets in the reference's fixed-point format.

Positions are int32 with x = i * 2^-32 + 0.5 (tigergrav/position.hpp:13-37);
``double_to_pos`` reproduces the reference's quantisation (std::lround, ties
away from zero, with the wrap at 2^31).  The reference ships no generator for
these workloads (its ``cosmos`` problem draws from ``rand()``,
src/initialize.cpp:20-27), so these are this project's own:

* ``uniform(n, seed)``     -- i.i.d. U[0,1)^3 from numpy's PCG64(seed).
* ``batch(nboxes, seed)`` -- the uneven-box batch (see its docstring).
* ``clustered(nside, seed)`` -- an nside^3 lattice displaced by the Zel'dovich
  displacement of a Gaussian random density field with P(k) ~ k^-2 (white
  noise from PCG64(seed), FFT on the nside^3 grid), scaled so that the rms
  displacement vector length is ``rms`` mean spacings (default 0.5), wrapped
  into the periodic unit box.
"""
from __future__ import annotations

import numpy as np

POS_MAX = 4294967296.0


def double_to_pos(x: np.ndarray) -> np.ndarray:
    """Vectorised tigergrav/position.hpp:30-37 (lround ties away from zero)."""
    v = (np.asarray(x, np.float64) - 0.5) * POS_MAX
    f = np.floor(v)
    frac = v - f
    z = f + (frac > 0.5) + ((frac == 0.5) & (v >= 0))
    z = np.where(z >= POS_MAX / 2.0, z - POS_MAX, z)
    return z.astype(np.int64).astype(np.int32)


def pos_to_double(x: np.ndarray) -> np.ndarray:
    """tigergrav/position.hpp:18-20."""
    return np.asarray(x, np.int32).astype(np.float64) / POS_MAX + 0.5


def uniform(n: int, seed: int = 1) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return double_to_pos(rng.random((n, 3)))


def clustered(nside: int, seed: int = 2, rms: float = 0.5) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    w = rng.standard_normal((nside, nside, nside))
    W = np.fft.rfftn(w)
    del w
    k1 = 2.0 * np.pi * np.fft.fftfreq(nside, d=1.0 / nside)
    kz = 2.0 * np.pi * np.fft.rfftfreq(nside, d=1.0 / nside)
    kx = k1[:, None, None]
    ky = k1[None, :, None]
    kzz = kz[None, None, :]
    k2 = kx * kx + ky * ky + kzz * kzz
    k2[0, 0, 0] = 1.0
    # delta(k) = W(k) sqrt(P(k)), P ~ k^-2 ; psi(k) = i k delta(k) / k^2
    amp = W / np.sqrt(k2) / k2
    amp[0, 0, 0] = 0.0
    psi = np.empty((3, nside, nside, nside), np.float64)
    for d, kd in enumerate((kx, ky, kzz)):
        psi[d] = np.fft.irfftn(1j * kd * amp, s=(nside, nside, nside), axes=(0, 1, 2))
    del amp, W
    cur = np.sqrt(np.mean(np.sum(psi * psi, axis=0)))
    psi *= (rms / nside) / cur
    g = np.arange(nside, dtype=np.float64) / nside
    X = np.empty((nside, nside, nside, 3), np.float64)
    X[..., 0] = g[:, None, None] + psi[0]
    X[..., 1] = g[None, :, None] + psi[1]
    X[..., 2] = g[None, None, :] + psi[2]
    X = np.mod(X.reshape(-1, 3), 1.0)
    X[X >= 1.0] = 0.0
    return double_to_pos(X)


def halos(n: int, seed: int = 5, frac: float = 0.6, nmin: int = 10, core: float = 0.1) -> np.ndarray:
    """A group-finding workload: frac of the n particles in Plummer spheres
    (sizes from a Pareto law, at least nmin, at most n/50; scale radius
    core n^(-1/3) N_h^(1/3), cut at 10 scale radii) at uniform random centres,
    the rest uniform; caller order shuffled.  The displaced-lattice workload
    above has no pairs closer than a fifth of the mean spacing, so it holds no
    friends-of-friends groups."""
    rng = np.random.Generator(np.random.PCG64(seed))
    want = int(frac * n)
    sizes = []
    tot = 0
    cap = max(nmin, n // 50)
    while tot < want:
        k = int(min(cap, nmin * (1.0 + rng.pareto(1.0))))
        k = min(k, want - tot)
        sizes.append(k)
        tot += k
    sizes = np.array(sizes, np.int64)
    nh = len(sizes)
    hid = np.repeat(np.arange(nh), sizes)
    centre = rng.random((nh, 3))
    a = core * n ** (-1.0 / 3.0) * sizes.astype(np.float64) ** (1.0 / 3.0)
    umax = 1000.0 / 101.0 ** 1.5  # enclosed fraction of a Plummer sphere inside 10 a
    u = rng.random(tot) * umax
    r = a[hid] / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    d = rng.standard_normal((tot, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    X = np.empty((n, 3))
    X[:tot] = centre[hid] + r[:, None] * d
    X[tot:] = rng.random((n - tot, 3))
    X = np.mod(X[rng.permutation(n)], 1.0)
    X[X >= 1.0] = 0.0
    return double_to_pos(X)


def samples(n: int, count: int = 4096, seed: int = 3) -> np.ndarray:
    """Seeded sample of particle indices for error measurement."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.sort(rng.choice(n, size=min(count, n), replace=False)).astype(np.int64)


def batch_sizes(nboxes: int = 64, seed: int = 4, lo: float = 12.0, hi: float = 18.0) -> np.ndarray:
    """Box particle counts N = round(2^U[lo,hi])."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.round(2.0 ** rng.uniform(lo, hi, size=nboxes)).astype(np.int64)


def batch(nboxes: int = 64, seed: int = 4):
    """The batching workload: box counts from batch_sizes(nboxes, seed); even
    boxes uniform (PCG64 seed 1000 + b), odd boxes clustered on the nearest
    cube lattice (nside = round(N^(1/3)), seed 2000 + b).  Returns (counts,
    positions of all boxes concatenated in box order)."""
    sizes = batch_sizes(nboxes, seed)
    counts, xs = [], []
    for b, n in enumerate(sizes):
        if b % 2 == 0:
            x = uniform(int(n), 1000 + b)
        else:
            x = clustered(max(2, int(round(float(n) ** (1.0 / 3.0)))), 2000 + b)
        counts.append(len(x))
        xs.append(x)
    return np.array(counts, np.int64), np.concatenate(xs)


def default_soft_len(n: int) -> float:
    """soft_len default 0.02 N^-1/3 (src/options.cpp:86-88)."""
    return 0.02 * float(n) ** (-1.0 / 3.0)
