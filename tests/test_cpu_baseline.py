"""The CPU baseline machinery of bench.py (no GPU): per-kind host throughput
sampling with the reference's kernels and the extrapolated evaluation time,
and the seeded workload generators."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_kind_costs_and_extrapolation(oracle_mod, has_ref):
    sys.path.insert(0, ROOT)
    import bench
    from tigergrav_b200 import ics
    x = ics.clustered(16, 2)
    r = bench.cpu_reference(x, 0.7, 2, budget_s=0.05)
    assert r["kind"] == ("reference" if has_ref else "port")
    assert r["seconds"] > 0 and np.isfinite(r["seconds"])
    for k in bench.KINDS:
        if r["counts"][k] > 0:
            assert r["sampled_interactions"][k] > 0 and r["ns_per_interaction"][k] > 0, k
    line = bench.cpu_line(r, len(x), 2, 0.05)
    assert line["value"] > 0 and line["cores"] == 2 and "extrapolated" in line["sample"]


def test_kind_costs_match_a_full_evaluation(oracle_mod):
    """the sampled throughputs times the counts predict a full (restated-kernel)
    evaluation within a factor of 3 on one thread"""
    import time
    from tigergrav_b200 import ics
    x = ics.uniform(2048, 1)
    o = oracle_mod.Oracle(theta=0.7).set_particles(x)
    o.build().multipoles().walk()
    costs = o.kind_costs(use_ref=False, nthreads=1, budget_s=2.0)
    _, counts, _ = o.stats()
    pred = sum(counts[k] * costs[k][0] * 1e-9 for k in counts)
    t0 = time.perf_counter()
    o.evaluate(nthreads=1)
    t = time.perf_counter() - t0
    assert pred / 3 < t < 3 * pred, (t, pred)


def test_batch_workload():
    from tigergrav_b200 import ics
    c, x = ics.batch(6, seed=4)
    assert len(c) == 6 and x.shape == (c.sum(), 3) and x.dtype == np.int32
    s = ics.batch_sizes(6, seed=4)
    assert np.all(c[0::2] == s[0::2])                       # uniform boxes: exact N
    assert np.all(np.abs(c[1::2] / s[1::2] - 1) < 0.35)     # clustered: nearest cube
