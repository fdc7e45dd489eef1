"""N-GenIC / Gadget-1 initial conditions (tg_load_gadget1, host code; no GPU)
against the oracle's restatement of src/load.cpp, on a file the oracle writes."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_gadget1_reader_matches_reference_semantics(tmp_path):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gadget
    from tigergrav_b200.solver import load_gadget1
    rng = np.random.default_rng(3)
    n = 4096
    pos = rng.random((n, 3)).astype(np.float32)
    pos[:5] = [[0.99, 0.999, 0.0], [1.0, 0.5, 0.25], [0.0, 0.0, 0.0], [0.9921875, 0.5, 0.5], [0.3, 0.6, 0.9]]
    vel = (rng.standard_normal((n, 3)) * 100).astype(np.float32)
    f = tmp_path / "ics.dat"
    gadget.write(str(f), pos, vel, redshift=49.0)
    hdr, x, v = load_gadget1(f)
    n_o, x_o, v_o = gadget.load(str(f))
    assert hdr["npart"] == n == n_o and abs(hdr["redshift"] - 49.0) < 1e-12
    assert abs(hdr["omega_m"] - 0.3) < 1e-12 and abs(hdr["omega_lambda"] - 0.7) < 1e-12
    assert np.array_equal(x, x_o)
    assert np.array_equal(v, v_o)


def test_gadget1_missing_file():
    import pytest
    from tigergrav_b200 import _lib
    from tigergrav_b200.solver import load_gadget1
    with pytest.raises(_lib.TGError):
        load_gadget1("/nonexistent/ics.dat")


def test_gadget1_oracle_matches_reference_load_particles(tmp_path):
    """the oracle's reader (and so tg_load_gadget1, bit-identical to it above)
    against the reference's own load_particles, bit for bit, including
    positions that wrap past 1 and ones exactly at the faces"""
    import pytest
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gadget
    import ref_tree
    if not ref_tree.available():
        pytest.skip("oracle/_ref/libtg_reftree.so not built")
    rng = np.random.default_rng(4)
    n = 4096
    pos = rng.random((n, 3)).astype(np.float32)
    pos[:6] = [[0.99, 0.999, 0.0], [1.0, 0.5, 0.25], [0.0, 0.0, 0.0], [0.9921875, 0.5, 0.5], [0.3, 0.6, 0.9],
               [0.99999994, 0.875, 0.125]]
    vel = (rng.standard_normal((n, 3)) * 100).astype(np.float32)
    f = tmp_path / "ics.dat"
    gadget.write(str(f), pos, vel, redshift=24.0)
    xr, vr = ref_tree.load_gadget1(f)
    n_o, x_o, v_o = gadget.load(str(f))
    assert len(xr) == n == n_o
    np.testing.assert_array_equal(xr, x_o)
    np.testing.assert_array_equal(vr, v_o)
