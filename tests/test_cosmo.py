"""Cosmological kick/drift factors (tg_cosmo_kdk, host code; no GPU) against
the oracle's restatement of src/cosmo.cpp and against Einstein-de Sitter."""
import os
import sys

import numpy as np

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
