"""The reference's solver test (src/main.cpp:137-165) on the GPU path: error
against the theta = 1e-10 direct solution falls with theta."""
import pytest

pytestmark = pytest.mark.gpu


def test_theta_sweep_against_direct():
    from tigergrav_b200 import ics
    from tigergrav_b200.solver_test import run
    rows = run(ics.uniform(4096, 1), "f32", thetas=[1.0, 0.7, 0.5, 0.3, 0.2])
    err = {r["theta"]: r["error"] for r in rows}
    assert err[1.0] > err[0.7] > err[0.5] > err[0.3]
    assert err[0.2] < 1e-5 and err[0.3] < 1e-5     # all pairs direct at 4096 particles
    assert 1e-4 < err[0.7] < 1e-1
    for r in rows:
        assert r["time"] > 0 and r["gflops"] > 0
