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
        assert np.allclose(s_lib, s_or, rtol=1e-13, atol=0)
        assert np.allclose(f_lib, f_or, rtol=1e-13, atol=0)


def test_einstein_de_sitter():
    """omega_m = 1: a = t^(2/3) with a(1) = 1 needs H0 = 2/3"""
    from tigergrav_b200.solver import cosmo_kdk
    st, f = cosmo_kdk([1.0, 2.0 / 3.0, 0.0], 0.1, 2.0 / 3.0, 1.0, 0.0)
    assert abs(st[0] - 1.1 ** (2.0 / 3.0)) < 1e-12
    assert abs(f[0] - 3 * (1.05 ** (1 / 3) - 1)) < 1e-12
    assert abs(f[1] - 3 * (1 - 1.1 ** (-1 / 3))) < 1e-12
    assert abs(f[2] - 3 * (1.1 ** (1 / 3) - 1.05 ** (1 / 3))) < 1e-12
    assert abs(st[2] - 3 * (1.1 ** (1 / 3) - 1)) < 1e-12  # tau = int dt / a
