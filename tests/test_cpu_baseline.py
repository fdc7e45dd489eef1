"""The CPU baseline machinery of bench.py (no GPU): the timed tree and
threaded walk, per-kind host throughput sampling with the reference's
kernels, the assembled evaluation time, a full evaluation with the
reference's kernels, and the seeded workload generators."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_kind_costs_and_estimate(oracle_mod, has_ref):
    sys.path.insert(0, ROOT)
    import bench
    from tigergrav_b200 import ics
    x = ics.clustered(16, 2)
    o, parts = bench.cpu_walk(x, 0.7, 2)
    assert parts["walk_s"] > 0 and parts["build_multipoles_s"] > 0
    r = bench.cpu_estimate(o, parts, 2, budget_s=0.05, seed=1)
    assert r["kind"] == ("reference" if has_ref else "port")
    assert r["seconds"] > 0 and np.isfinite(r["seconds"])
    _, counts, _ = o.stats()
    for k in bench.KINDS:
        if counts[k] > 0:
            assert r["sampled_interactions"][k] > 0 and r["ns_per_interaction"][k] > 0, k
    line = bench.cpu_line(r, len(x), 2, 0.05)
    assert line["value"] > 0 and line["cores"] == 2 and "walk (2 threads" in line["sample"]


def test_full_reference_evaluation(oracle_mod, has_ref):
    """The reference arm's measured full evaluation: the reference's kernels on
    the threaded walk's lists give the serial oracle's forces."""
    sys.path.insert(0, ROOT)
    import bench
    from tigergrav_b200 import ics
    x = ics.uniform(4096, 1)
    r = bench.cpu_full_eval(x, 0.7, 2)
    assert r["seconds"] > 0 and r["kind"] == ("reference" if has_ref else "port")
    a = oracle_mod.Oracle(theta=0.7).set_particles(x).build().multipoles().walk(nthreads=3)
    b = oracle_mod.Oracle(theta=0.7).set_particles(x).build().multipoles().walk()
    assert a.stats() == b.stats()
    a.evaluate(use_ref=has_ref, nthreads=3)
    b.evaluate(use_ref=has_ref, nthreads=1)
    assert np.array_equal(a.forces()[1], b.forces()[1])


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
