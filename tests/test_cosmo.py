"""Cosmological kick/drift factors (tg_cosmo_kdk, host code; no GPU) against
the oracle's restatement of src/cosmo.cpp and against Einstein-de Sitter; and
that restatement against the reference's own src/cosmo.cpp."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_matches_restatement_lcdm():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cosmo as oc
    from tigergrav_b200.solver import cosmo_kdk
    H0, om, ol = 0.1, 0.3, 0.7
    a0 = 1.0 / 51.0  # z = 50
    st = [a0, H0 * np.sqrt(om / a0 + ol * a0 ** 2), 0.0]  # da/dt from the Friedmann equation
    s_lib, s_or = list(st), list(st)
    for dt in (0.01, 0.02, 0.05):
        s_lib, f_lib = cosmo_kdk(s_lib, dt, H0, om, ol)
        s_or, f_or = oc.kdk_factors(s_or, dt, H0, om, ol)
        # the same operations in the same order: bit for bit
        assert list(s_lib) == list(s_or)
        assert list(f_lib) == list(f_or)


def test_einstein_de_sitter():
    """omega_m = 1: a = t^(2/3) with a(1) = 1 needs H0 = 2/3"""
    from tigergrav_b200.solver import cosmo_kdk
    st, f = cosmo_kdk([1.0, 2.0 / 3.0, 0.0], 0.1, 2.0 / 3.0, 1.0, 0.0)
    assert abs(st[0] - 1.1 ** (2.0 / 3.0)) < 1e-12
    assert abs(f[0] - 3 * (1.05 ** (1 / 3) - 1)) < 1e-12
    assert abs(f[1] - 3 * (1 - 1.1 ** (-1 / 3))) < 1e-12
    assert abs(f[2] - 3 * (1.1 ** (1 / 3) - 1.05 ** (1 / 3))) < 1e-12
    assert abs(st[2] - 3 * (1.1 ** (1 / 3) - 1)) < 1e-12  # tau = int dt / a


def test_rung_advance_factors():
    """the oracle's cosmo_advance for rung steps: kick_dt1 is filled only once
    the float time reaches a rung's step; the factors integrate 1/a over half
    steps (Einstein-de Sitter: closed forms)"""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cosmo as oc
    t_max = 0.25
    cs = oc.rung_state(1.0, 2.0 / 3.0)  # EdS, t = 1 at a = 1
    drift, k1, k2, a3inv = oc.rung_advance(cs, 0.0, t_max, 2.0 / 3.0, 1.0, 0.0)
    assert drift == 0.0 and k1[0] == -1.0 and a3inv == 1.0
    # kick ahead over half of rung 2's step (t_max / 4): int_1^{1+1/32} t^(-2/3) dt
    assert abs(k2[2] - 3 * ((1 + t_max / 8) ** (1 / 3) - 1)) < 1e-12
    drift, k1, k2, a3inv = oc.rung_advance(cs, t_max / 4, t_max, 2.0 / 3.0, 1.0, 0.0)
    assert float(cs["time"]) == t_max / 4
    assert k1[1] == 0.0 and k1[0] == -1.0  # rungs 0 and 1: time below their steps
    t1 = 1 + t_max / 4
    assert abs(k1[2] - 3 * (t1 ** (1 / 3) - (t1 - t_max / 8) ** (1 / 3))) < 1e-12
    assert abs(drift - 3 * (1 - t1 ** (-1 / 3))) < 1e-12
    assert abs(cs["a"] - t1 ** (2 / 3)) < 1e-12 and a3inv == 1.0


# ---- the restatement against the reference's own src/cosmo.cpp ------------
# (compiled into oracle/_ref/libtg_reftree.so; skipped where it was not built)

def _ref_tree():
    import ref_tree
    if not ref_tree.available():
        pytest.skip("oracle/_ref/libtg_reftree.so not built")
    return ref_tree


COSMO_CASES = [(1.0, 1.0, 0.3, 0.7), (0.5, 1.0, 0.3, 0.7), (1.0 / 51.0, 0.1, 1.0, 0.0), (0.25, 2.0, 0.3, 0.7)]


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-300)


@pytest.mark.parametrize("a0,H0,om,ol", COSMO_CASES)
def test_advance_to_time_matches_reference(a0, H0, om, ol):
    """cosmos::advance_to_time, forwards and backwards, from the reference's
    own build: the restatement to the last bit or two (the reference's build
    may contract products into FMAs)"""
    import cosmo as oc
    rt = _ref_tree()
    adot = H0 * a0 * np.sqrt(om / a0 ** 3 + ol)
    for t0 in (0.0, 1e-4, 1.0 / 64.0, -1.0 / 128.0, 0.3):
        rs, rd, rk = rt.cosmos_advance([a0, adot, 0.0], t0, H0, om, ol)
        os_, od, ok = oc.advance_to_time([a0, adot, 0.0], t0, H0, om, ol)
        assert _rel(rs + [rd, rk], os_ + [od, ok]).max() <= 1e-14, t0


@pytest.mark.parametrize("a0,H0,om,ol", COSMO_CASES)
def test_rung_advance_matches_reference(a0, H0, om, ol):
    """cosmo_advance step by step (src/cosmo.cpp:187-218): the scale factors,
    the float time, tau, the drift factor and kick_dt1 / kick_dt2 of every
    rung, against the reference's own build"""
    import cosmo as oc
    rt = _ref_tree()
    adot = H0 * a0 * np.sqrt(om / a0 ** 3 + ol)
    dts = [0.0, 1 / 64, 1 / 64, 1 / 32, 1 / 64, 1 / 128, 1 / 128, 1 / 16]
    ref = rt.cosmo_steps(a0, adot, dts, H0, om, ol)
    cs = oc.rung_state(a0, adot)
    for r, dt in zip(ref, dts):
        drift, k1, k2, _ = oc.rung_advance(cs, dt, 1.0, H0, om, ol)
        assert r["time"] == float(cs["time"])
        mine = [cs["a"], cs["a_last"], cs["tau"], drift] + list(k1) + list(k2)
        theirs = [r["a"], r["a_last"], r["tau"], r["drift"]] + list(r["kick1"]) + list(r["kick2"])
        assert _rel(theirs, mine).max() <= 1e-13, dt
