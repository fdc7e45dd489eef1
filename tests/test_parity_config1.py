"""Parity at the benchmarked 128^3 clustered workload: 2,097,152 particles on a
lattice displaced by a P(k) ~ k^-2 Gaussian field (seed 2), periodic, Ewald
on, leaf 64, at the literal theta 0.7 and at theta 0.2 (RMS force error
<= 1e-4 there).

  tree and lists  node set, box ids, ranges, centres of mass and radii, and
                  all eight interaction lists: identical to the oracle's
                  restatement of refine / kick_fmm (src/tree.cpp:122-635)
  forces          at 4096 seeded sample particles (theta 0.7; 64 of them at
                  theta 0.2, where the reference's Ewald kernels take ~6 us
                  per interaction on the host): per particle no further from
                  the FP64 evaluation of the same lists than the reference's
                  own arithmetic is (its kernels, src/gravity.cpp via
                  oracle/_ref, or their restatement summed in another order),
                  + 1e-5 of max(|g|, g_rms / 2) (helpers.arbiter_excess)
  evolution       10 kick-drift-kick steps at dt = 1e-3 (theta 0.7) against
                  the oracle stepper driving the reference's kernels
"""
import os

import numpy as np
import pytest

from helpers import arbiter_excess, rel_force_err

pytestmark = pytest.mark.gpu

NTH = os.cpu_count() or 1
_x = None


def particles():
    global _x
    if _x is None:
        from tigergrav_b200 import ics
        _x = ics.clustered(128, 2)
    return _x


def _leaves_of(nodes, perm, callers):
    """oracle leaf ids holding the given caller indices"""
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    pos = inv[callers]
    leaf = np.nonzero((nodes["child0"] < 0) & (nodes["pend"] > nodes["pbegin"]))[0]
    order = np.argsort(nodes["pbegin"][leaf])
    leaf = leaf[order]
    k = np.searchsorted(nodes["pbegin"][leaf], pos, side="right") - 1
    assert np.all(nodes["pend"][leaf[k]] > pos)
    return np.unique(leaf[k]).astype(np.int32)


def _box_of_particle(nodes, perm):
    """box id of the leaf holding each particle, by caller index"""
    leaf = np.nonzero(nodes["child0"] < 0)[0]
    cnt = nodes["pend"][leaf] - nodes["pbegin"][leaf]
    order = np.argsort(nodes["pbegin"][leaf])
    box_sorted = np.repeat(nodes["boxid"][leaf][order], cnt[order])
    out = np.empty(len(perm), np.uint64)
    out[perm] = box_sorted
    return out


@pytest.mark.parametrize("theta", [0.7, 0.2])
def test_config1_tree_and_lists(theta, oracle_mod):
    import tigergrav_b200 as tg
    x = particles()
    with tg.GravitySolver(len(x), theta=theta, leaf_max=64) as s:
        s.set_particles(x).solve_gravity()
        gn, gperm, gst = s.nodes(), s.perm(), s.stats()
        glists = {k: s.list(k) for k in ("CC_D", "CP_D", "CC_E", "CP_E", "PC_D", "PP_D", "PC_E", "PP_E")}
    o = oracle_mod.Oracle(theta=theta, ewald=True, leaf_max=64).set_particles(x)
    o.build().multipoles().walk(nthreads=NTH)
    on = o.nodes()
    assert len(gn["boxid"]) == len(on["boxid"])
    for k in ("boxid", "level", "child0", "parent", "pbegin", "pend"):
        np.testing.assert_array_equal(gn[k], on[k], err_msg=k)
    # leaf membership: every particle in the leaf of the same box id
    np.testing.assert_array_equal(_box_of_particle(gn, gperm), _box_of_particle(on, o.perm()))
    nonempty = on["pend"] > on["pbegin"]
    np.testing.assert_array_equal(gn["x"][nonempty], on["x"][nonempty])
    np.testing.assert_array_equal(gn["r"].view(np.int32), on["r"].view(np.int32))
    for k, (goff, gids) in glists.items():
        ooff, oids = o.list(k)
        np.testing.assert_array_equal(goff, ooff, err_msg=k)
        np.testing.assert_array_equal(gids, oids, err_msg=k)
    _, counts, _ = o.stats()
    assert gst["counts"] == counts


@pytest.mark.parametrize("theta,nsamples", [(0.7, 4096), (0.2, 64)])
def test_config1_forces_at_samples(theta, nsamples, oracle_mod, has_ref):
    import tigergrav_b200 as tg
    from tigergrav_b200 import ics
    x = particles()
    smp = ics.samples(len(x), 4096, 3)[:nsamples]
    with tg.GravitySolver(len(x), theta=theta, leaf_max=64) as s:
        s.set_particles(x).solve_gravity()
        phi, g = s.get_forces()
    o = oracle_mod.Oracle(theta=theta, ewald=True, leaf_max=64).set_particles(x)
    o.build().multipoles().walk(nthreads=NTH)
    sub = _leaves_of(o.nodes(), o.perm(), smp)
    o.evaluate(use_ref=has_ref, nthreads=NTH, leaf_subset=sub)
    rphi, rg = (a[smp] for a in o.forces())
    o.evaluate(nthreads=NTH, leaf_subset=sub)  # the reference's arithmetic, summed in the oracle's order
    sphi, sg = (a[smp] for a in o.forces())
    o.evaluate(fp64=True, nthreads=NTH, leaf_subset=sub)
    phi64, g64 = (a[smp] for a in o.forces())
    assert np.all(np.linalg.norm(g64, axis=1) > 0)
    fx, px = arbiter_excess(g[smp], rg, g64, phi[smp], rphi, phi64, g_alt=sg, phi_alt=sphi)
    assert fx <= 0.0, fx
    assert px <= 0.0, px
    # at the 99th percentile, no further from the FP64 evaluation than the
    # reference's own kernels are (measured at theta 0.7: the reference's
    # kernels 1.83e-5 from FP64, its arithmetic in the oracle's summation
    # order 1.06e-5 from its kernels: the FP32 spread of the reference itself)
    e = rel_force_err(g[smp], g64)
    e_ref = rel_force_err(rg, g64)
    assert np.percentile(e, 99) <= np.percentile(e_ref, 99), (np.percentile(e, 99), np.percentile(e_ref, 99))


def test_config1_ten_kdk_steps(oracle_mod, has_ref):
    """10 KDK steps at dt = 1e-3, theta 0.7, FP32 path, against the oracle's
    stepper (restated kick / drift, src/part_vect.cpp:341-540, with the
    reference's force kernels), compared at 4096 samples."""
    import tigergrav_b200 as tg
    from tigergrav_b200 import ics
    x = particles()
    n = len(x)
    dt, steps = 1e-3, 10
    smp = ics.samples(n, 4096, 3)
    with tg.GravitySolver(n, theta=0.7, leaf_max=64) as s:
        s.set_particles(x).leapfrog(dt, steps)
        xg, vg = s.get_particles()
    o = oracle_mod.Oracle(theta=0.7, ewald=True, leaf_max=64).set_particles(x)
    o.build().multipoles().walk(nthreads=NTH).evaluate(use_ref=has_ref, nthreads=NTH)
    for _ in range(steps):
        o.kick(0.5 * dt)
        o.drift(dt)
        o.build().multipoles().walk(nthreads=NTH).evaluate(use_ref=has_ref, nthreads=NTH)
        o.kick(0.5 * dt)
    xo, vo = o.particles()
    dxi = np.abs((xg[smp].astype(np.int64) - xo[smp].astype(np.int64) + 2 ** 31) % 2 ** 32 - 2 ** 31)
    dv = np.linalg.norm(vg[smp] - vo[smp], axis=1) / np.maximum(np.linalg.norm(vo[smp], axis=1), 1e-30)
    # positions in fixed-point units (2^-32 of the box).  Forces agree to
    # ~1e-6, which moves a particle by a few units in 10 steps; once two
    # positions differ by a unit, an opening test near its threshold can
    # change a list, so a few particles may differ by more
    assert np.percentile(dxi, 99) <= 4, (np.percentile(dxi, 99), dxi.max())
    assert dxi.max() <= 4096, dxi.max()
    # velocities start at zero, so their relative difference is that of the
    # accumulated forces (the FP32 path and the reference's kernels: ~1e-5)
    assert np.percentile(dv, 99) <= 3e-5, (np.percentile(dv, 99), dv.max())
    assert dv.max() <= 3e-4, dv.max()
