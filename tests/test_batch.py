"""Batches of independent boxes (tg_batch_*): every box's forces equal a
single-box solve of the same particles with the same leaf size."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batch_equals_single_boxes():
    import tigergrav_b200 as tg
    from tigergrav_b200 import ics
    counts, x = ics.batch(8, seed=4)
    off = np.concatenate([[0], np.cumsum(counts)])
    with tg.GravityBatch(counts, theta=0.7, nstreams=4) as b:
        b.set_particles(x).solve()
        phi, g = b.get_forces()
        chosen = b.autotune((16, 64))
        assert set(chosen.tolist()) <= {16, 64}
        b.solve()
        phi2, g2 = b.get_forces()
    for k in range(len(counts)):
        n = int(counts[k])
        xs = x[off[k]:off[k + 1]]
        for leaf, (ph, gg) in ((64, (phi, g)), (int(chosen[k]), (phi2, g2))):
            with tg.GravitySolver(n, theta=0.7, leaf_max=leaf) as s:
                s.set_particles(xs).solve_gravity()
                p1, g1 = s.get_forces(dtype=np.float32)
            assert np.array_equal(p1, ph[off[k]:off[k + 1]])
            assert np.array_equal(g1, gg[off[k]:off[k + 1]])
