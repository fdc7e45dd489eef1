"""The algebra behind the FP32 path's reciprocal-space sums per sink
(tigergrav_b200/csrc/tg_ewald_sep.cuh, k_node_ewald_recip): for any
coefficient table of the M2P / M2L contractions (src/gravity.cpp:26-169) and
any set of sources, summing m_k cos/sin(2 pi h.X_j) per sink and evaluating
the terms once at the sink equals contracting each source's multipole with
the reciprocal part of green_ewald (tigergrav/green.hpp:237-264) one
interaction at a time.  numpy, FP64; the CUDA kernels themselves are checked
against the oracle's forces by the GPU tests."""
import itertools

import numpy as np

PI = np.pi
S = [-1 / PI, 2.0, 4 * PI, -8 * PI ** 2, -16 * PI ** 3]
T3 = sorted(set(tuple(sorted(t)) for t in itertools.product(range(3), repeat=3)))
T4 = sorted(set(tuple(sorted(t)) for t in itertools.product(range(3), repeat=4)))
P2 = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]


def I2(a, b):
    return P2.index(tuple(sorted((a, b))))


def I3(*t):
    return T3.index(tuple(sorted(t)))


def I4(*t):
    return T4.index(tuple(sorted(t)))


E0 = 0


def E1(a):
    return 1 + a


def E2(a, b):
    return 4 + I2(a, b)


def E3(a, b, c):
    return 10 + I3(a, b, c)


def E4(a, b, c, d):
    return 20 + I4(a, b, c, d)


def M2(a, b):
    return 1 + I2(a, b)


def M3(a, b, c):
    return 7 + I3(a, b, c)


def d_recip(x, hs, cs):
    """The reciprocal part of D (35 terms) at separation x, term by term."""
    D = np.zeros(35)
    for h, c in zip(hs, cs):
        th = 2 * PI * h.dot(x)
        co, si = np.cos(th), np.sin(th)
        D[E0] += c * S[0] * co
        for a in range(3):
            D[E1(a)] += c * S[1] * h[a] * si
            for b in range(a + 1):
                D[E2(a, b)] += c * S[2] * h[a] * h[b] * co
                for cc in range(b + 1):
                    D[E3(a, b, cc)] += c * S[3] * h[a] * h[b] * h[cc] * si
                    for d in range(cc + 1):
                        D[E4(a, b, cc, d)] += c * S[4] * h[a] * h[b] * h[cc] * h[d] * co
    return D


def m2p(M, D, f):
    """contract_M2P's loops (the potential's octupole sum runs a over all axes)."""
    phi = M[0] * D[E0]
    for a in range(3):
        for b in range(a, 3):
            phi += M[M2(a, b)] * D[E2(a, b)] * f[E2(a, b)]
    for a in range(3):
        for b in range(3):
            for c in range(b, 3):
                phi -= M[M3(a, b, c)] * D[E3(a, b, c)] * f[E3(a, b, c)]
    g = np.zeros(3)
    for a in range(3):
        ga = -M[0] * D[E1(a)]
        for b in range(3):
            for c in range(b, 3):
                ga -= M[M2(c, b)] * D[E3(a, b, c)] * f[E2(c, b)]
                for d in range(c, 3):
                    ga += M[M3(c, b, d)] * D[E4(a, b, c, d)] * f[E3(b, c, d)]
        g[a] = ga
    return phi, g


def m2l(M, D, f):
    L = np.zeros(35)
    L0 = M[0] * D[E0]
    for a in range(3):
        for b in range(a, 3):
            L0 += M[M2(a, b)] * D[E2(a, b)] * f[E2(a, b)]
            for c in range(b, 3):
                L0 -= M[M3(a, b, c)] * D[E3(a, b, c)] * f[E3(a, b, c)]
    L[E0] += L0
    for a in range(3):
        La = M[0] * D[E1(a)]
        for b in range(3):
            for c in range(b, 3):
                La += M[M2(c, b)] * D[E3(a, b, c)] * f[E2(c, b)]
                for d in range(c, 3):
                    La -= M[M3(b, c, d)] * D[E4(a, b, c, d)] * f[E3(b, c, d)]
        L[E1(a)] += La
    for a in range(3):
        for b in range(a, 3):
            Lab = M[0] * D[E2(a, b)]
            for c in range(3):
                for d in range(c, 3):
                    Lab += M[M2(c, d)] * D[E4(a, b, c, d)] * f[E2(c, d)]
            L[E2(a, b)] += Lab
    L[10:] += M[0] * D[10:]
    return L


def weights(h, f):
    """sep_q: the monomial weights of m_2, m_3 and the potential's m_3'."""
    q2, q3, q3p = np.zeros(6), np.zeros(10), np.zeros(10)
    for a in range(3):
        for b in range(a, 3):
            q2[I2(a, b)] = f[E2(a, b)] * h[a] * h[b]
            for c in range(b, 3):
                q3[I3(a, b, c)] = f[E3(a, b, c)] * h[a] * h[b] * h[c]
    for a in range(3):
        for b in range(3):
            for c in range(b, 3):
                q3p[I3(a, b, c)] += f[E3(a, b, c)] * h[a] * h[b] * h[c]
    return q2, q3, q3p


def _setup(seed):
    rng = np.random.default_rng(seed)
    f = rng.uniform(0.5, 3.0, 35)
    hs = [np.array(h, float) for h in [(1, 0, 0), (1, 2, -1), (0, 1, 3), (2, -1, 1), (0, 0, 1)]]
    cs = rng.uniform(0.1, 1.0, len(hs))
    srcs = [(rng.standard_normal(17), rng.random(3)) for _ in range(6)]
    return rng, f, hs, cs, srcs


def test_leaf_sink_sums_equal_m2p_per_interaction():
    rng, f, hs, cs, srcs = _setup(1)
    xi = rng.random(3)
    ref_phi, ref_g = 0.0, np.zeros(3)
    for M, X in srcs:
        p, g = m2p(M, d_recip(xi - X, hs, cs), f)
        ref_phi += p
        ref_g += g
    phi, g = 0.0, np.zeros(3)
    for h, c in zip(hs, cs):
        q2, q3, q3p = weights(h, f)
        A = np.zeros(8)
        for M, X in srcs:
            th = 2 * PI * h.dot(X)
            C, Sn = np.cos(th), np.sin(th)
            m2, m3, m3p = q2.dot(M[1:7]), q3.dot(M[7:17]), q3p.dot(M[7:17])
            A += [M[0] * C, M[0] * Sn, m2 * C, m2 * Sn, m3p * C, m3p * Sn, m3 * C, m3 * Sn]
        th = 2 * PI * h.dot(xi)
        C, Sn = np.cos(th), np.sin(th)
        ev0, od0 = C * A[0] + Sn * A[1], Sn * A[0] - C * A[1]
        ev2, od2 = C * A[2] + Sn * A[3], Sn * A[2] - C * A[3]
        od3p, ev3 = Sn * A[4] - C * A[5], C * A[6] + Sn * A[7]
        phi += c * (S[0] * ev0 + S[2] * ev2 - S[3] * od3p)
        g += c * (-S[1] * od0 - S[3] * od2 + S[4] * ev3) * h
    assert abs(phi - ref_phi) <= 1e-12 * max(1.0, abs(ref_phi))
    assert np.abs(g - ref_g).max() <= 1e-12 * max(1.0, np.abs(ref_g).max())


def test_node_sink_sums_equal_m2l_per_interaction():
    rng, f, hs, cs, srcs = _setup(2)
    Xs = rng.random(3)
    ref = np.zeros(35)
    for M, X in srcs:
        ref += m2l(M, d_recip(Xs - X, hs, cs), f)
    L = np.zeros(35)
    for h, c in zip(hs, cs):
        q2, q3, _ = weights(h, f)
        A = np.zeros(6)
        for M, X in srcs:
            th = 2 * PI * h.dot(X)
            C, Sn = np.cos(th), np.sin(th)
            m2, m3 = q2.dot(M[1:7]), q3.dot(M[7:17])
            A += [M[0] * C, M[0] * Sn, m2 * C, m2 * Sn, m3 * C, m3 * Sn]
        th = 2 * PI * h.dot(Xs)
        C, Sn = np.cos(th), np.sin(th)
        ev = [C * A[2 * k] + Sn * A[2 * k + 1] for k in range(3)]
        od = [Sn * A[2 * k] - C * A[2 * k + 1] for k in range(3)]
        v = [S[0] * ev[0] + S[2] * ev[1] - S[3] * od[2], S[1] * od[0] + S[3] * od[1] - S[4] * ev[2],
             S[2] * ev[0] + S[4] * ev[1], S[3] * od[0], S[4] * ev[0]]
        L[E0] += c * v[0]
        for a in range(3):
            L[E1(a)] += c * v[1] * h[a]
            for b in range(a + 1):
                L[E2(a, b)] += c * v[2] * h[a] * h[b]
                for cc in range(b + 1):
                    L[E3(a, b, cc)] += c * v[3] * h[a] * h[b] * h[cc]
                    for d in range(cc + 1):
                        L[E4(a, b, cc, d)] += c * v[4] * h[a] * h[b] * h[cc] * h[d]
    assert np.abs(L - ref).max() <= 1e-12 * np.abs(ref).max()


def test_fixed_point_phase_is_exact():
    """sep_cs: h.x mod 1 from the int32 coordinates, x = i 2^-32 + 1/2."""
    rng = np.random.default_rng(3)
    x = rng.integers(-2 ** 31, 2 ** 31, size=(200, 3), dtype=np.int64)
    for h in [(1, 0, 0), (1, 2, -1), (3, -3, 1), (0, 2, 2)]:
        P = x.dot(np.array(h, np.int64))
        u = (P % 2 ** 32 + (2 ** 31 if sum(h) % 2 else 0)) % 2 ** 32
        r = np.where(u >= 2 ** 31, u - 2 ** 32, u) / 2.0 ** 32
        exact = (x.astype(np.float64) / 2 ** 32 + 0.5).dot(np.array(h, float))
        d = (r - exact) % 1.0
        assert np.all(np.minimum(d, 1 - d) < 1e-9)
        assert np.all((r >= -0.5) & (r < 0.5))
