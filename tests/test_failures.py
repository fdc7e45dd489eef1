"""Failure detection, injected from the host.

The reference aborts on bad input (src/part_vect.cpp:58-66 under !NDEBUG) or
runs into FP traps; this library answers status codes instead.  Every fault
here is made on the host: a bad argument, a capacity set too small, a retry
limit of zero.  No test makes a kernel fault, trap or hang: kernels that run
out of room or attempts set a flag and return, and the host reads the flag.
"""
import ctypes as C

import numpy as np
import pytest

from tigergrav_b200 import _lib

gpu = pytest.mark.gpu


def _params(**kw):
    from tigergrav_b200.solver import make_params
    p = make_params(n=4096)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("field,value", [
    ("theta", 0.0), ("theta", -0.5), ("theta", float("inf")), ("theta", float("nan")),
    ("soft_len", 0.0), ("soft_len", float("nan")), ("m", 0.0), ("m", float("inf")), ("G", float("nan")),
    ("leaf_max", 0), ("leaf_max", 129), ("precision", 7),
])
def test_create_rejects_bad_parameters(field, value):
    """Parameters are validated before any device is touched (no GPU needed)."""
    h = C.c_void_p()
    rc = _lib.lib.tg_create(C.byref(_params(**{field: value})), C.byref(h))
    assert rc == _lib.TG_ERR_ARG
    assert not h.value


def test_null_handles_are_bad_arguments():
    for f in ("tg_build", "tg_multipoles", "tg_walk", "tg_forces", "tg_solve_gravity"):
        assert getattr(_lib.lib, f)(None, None) == _lib.TG_ERR_ARG, f
    assert _lib.lib.tg_set_walk_capacity(None, 0) == _lib.TG_ERR_ARG
    assert _lib.lib.tg_set_fof_retry_limit(None, 1) == _lib.TG_ERR_ARG


@gpu
def test_bad_particles_are_refused():
    from tigergrav_b200 import ics
    from tigergrav_b200.solver import GravitySolver
    x = ics.uniform(4096, 21)
    with GravitySolver(len(x)) as s:
        assert _lib.lib.tg_set_particles(s.h, C.c_void_p(x.ctypes.data), None, 0, _lib.TG_HOST,
                                         None) == _lib.TG_ERR_ARG
        assert _lib.lib.tg_set_particles(s.h, None, None, len(x), _lib.TG_HOST, None) == _lib.TG_ERR_ARG
        for bad in (np.nan, np.inf, -np.inf):
            v = np.zeros((len(x), 3), np.float32)
            v[1234, 1] = bad
            with pytest.raises(_lib.TGError) as e:
                s.set_particles(x, v)
            assert e.value.status == _lib.TG_ERR_ARG
            # nothing was loaded: the path answers "out of order" until valid particles arrive
            with pytest.raises(_lib.TGError) as e:
                s.solve_gravity()
            assert e.value.status == _lib.TG_ERR_STATE
        s.set_particles(x, np.zeros((len(x), 3), np.float32)).solve_gravity()
        assert np.all(np.isfinite(s.get_forces()[1]))
        # the walk's capacity knob refuses negative sizes
        assert _lib.lib.tg_set_walk_capacity(s.h, -1) == _lib.TG_ERR_ARG


@gpu
def test_coincident_particles_beyond_the_leaf_size():
    """More than leaf_max particles at one point cannot be split by any of the
    63 Morton levels: the build answers TG_ERR_DEPTH (the reference's refine
    would recurse without end)."""
    from tigergrav_b200 import ics
    from tigergrav_b200.solver import GravitySolver
    x = ics.uniform(2048, 22)
    x[100:165] = x[7]  # 65 copies of one position plus the original: 66 > 64
    with GravitySolver(len(x), leaf_max=64) as s:
        s.set_particles(x)
        with pytest.raises(_lib.TGError) as e:
            s.solve_gravity()
        assert e.value.status == _lib.TG_ERR_DEPTH
    x[100:164] = x[7]
    x[164] = x[8]  # now 65 at one point: still too many
    with GravitySolver(len(x), leaf_max=64) as s:
        s.set_particles(x)
        with pytest.raises(_lib.TGError) as e:
            s.solve_gravity()
        assert e.value.status == _lib.TG_ERR_DEPTH
    x[100:163] = x[7]
    x[163:165] = x[8:10]  # 64 at one point fit in one leaf
    with GravitySolver(len(x), leaf_max=64) as s:
        s.set_particles(x).solve_gravity()
        assert np.all(np.isfinite(s.get_forces()[1]))


@gpu
@pytest.mark.parametrize("cap", [16, 256, 5000])
def test_walk_regrowth_gives_the_same_lists(cap):
    """Pools far too small for the lists overflow on the device (no write out of
    bounds), regrow on the host to the totals the walk asked for, and rerun:
    the lists and forces end identical to a walk that never overflowed."""
    from tigergrav_b200 import ics
    from tigergrav_b200.solver import GravitySolver
    x = ics.clustered(16, 23)
    with GravitySolver(len(x), theta=0.5) as a, GravitySolver(len(x), theta=0.5) as b:
        a.set_particles(x).solve_gravity()
        a.solve_gravity()  # the pools keep the size the first walk grew them to
        assert a.stats()["walk_retries"] == 0
        b.set_walk_capacity(cap)
        b.set_particles(x).solve_gravity()
        assert b.stats()["walk_retries"] >= 1
        for kind in ("CC_D", "CP_D", "CC_E", "CP_E", "PC_D", "PP_D", "PC_E", "PP_E"):
            oa, ia = a.list(kind)
            ob, ib = b.list(kind)
            lens_a, lens_b = np.diff(oa), np.diff(ob)
            assert np.array_equal(lens_a, lens_b), kind
            for k in np.nonzero(lens_a)[0][:: max(1, len(lens_a) // 500)]:
                assert np.array_equal(ia[oa[k]:oa[k + 1]], ib[ob[k]:ob[k + 1]]), (kind, k)
        pa, ga = a.get_forces()
        pb, gb = b.get_forces()
        assert np.array_equal(ga, gb) and np.array_equal(pa, pb)
        # back to automatic sizing: once grown, the pools serve the next walks
        b.set_walk_capacity(0)
        b.solve_gravity()
        b.solve_gravity()
        assert b.stats()["walk_retries"] == 0


@gpu
def test_fof_union_find_gives_up_without_spinning():
    """A union-find hook limit of 0 makes every join fail at once: the kernel
    sets its flag and returns, tg_find_groups answers TG_ERR_TIMEOUT, and the
    same handle finds the groups once the limit is back."""
    from tigergrav_b200 import ics
    from tigergrav_b200.solver import GravitySolver
    x = ics.halos(4096, seed=24)
    with GravitySolver(len(x)) as s:
        s.set_particles(x)
        ref = s.find_groups(0.2)
        assert (ref >= 0).sum() > 100
        assert _lib.lib.tg_set_fof_retry_limit(s.h, 0) == _lib.TG_OK
        with pytest.raises(_lib.TGError) as e:
            s.find_groups(0.2)
        assert e.value.status == _lib.TG_ERR_TIMEOUT
        assert _lib.lib.tg_set_fof_retry_limit(s.h, -1) == _lib.TG_ERR_ARG
        assert _lib.lib.tg_set_fof_retry_limit(s.h, 65536) == _lib.TG_OK
        assert np.array_equal(s.find_groups(0.2), ref)
