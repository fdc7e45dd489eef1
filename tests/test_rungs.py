"""Hierarchical (rung) time steps (tg_rung_step, tg_get_rungs).

CPU: the oracle's integer time line against values that follow from
tigergrav/time.hpp:12-48 by hand, and its kick rules.  GPU: K rung steps of
the library against the oracle's stepper driven by the library's own full
solve (every particle a sink) and the oracle's drift: positions, velocities
and rungs bit-identical, which also shows that the walk restricted to active
sinks gives the active particles exactly the forces of a full solve."""
import numpy as np
import pytest

import rungs as orung


def test_time_line_by_hand():
    assert orung.min_rung(0) == 0
    assert orung.min_rung(1 << 30) == 1
    assert orung.min_rung(3 << 28) == 3
    assert orung.min_rung(1) == 31
    assert orung.inc(0, 3) == 1 << 28 and orung.inc(1 << 28, 3) == 1 << 29
    assert orung.inc(0, 0) == 1 << 31
    assert orung.time_to_double(1 << 30, 2.0) == 1.0
    assert orung.rung_to_dt(1.0, 4) == 1.0 / 16
    # the smallest rung whose step is <= dt
    assert orung.dt_to_rung(1.0, np.array([1.0, 0.5, 0.49, 0.25, 1e-3])).tolist() == [0, 1, 2, 2, 10]
    with pytest.raises(ValueError):
        orung.dt_to_rung(1.0, np.array([1e-12]))


def test_kick_rules():
    t_max, h, eta = 1.0, 1e-3, 0.1
    v = np.zeros((4, 3), np.float32)
    rung = np.array([0, 3, 8, 2], np.int8)
    g = np.array([[1e3, 0, 0], [1e-6, 0, 0], [1e-6, 0, 0], [1.0, 0, 0]], np.float32)
    mr = orung.kick(v, rung, g, 2, t_max, 0.5, eta, h)
    # particle 0 is below min_rung 2: untouched
    assert rung[0] == 0 and (v[0] == 0).all()
    # particle 1: tiny force -> dt_max -> rung 1, raised to min_rung 2; stored max(2, 3 - 1, 1)
    assert rung[1] == 2
    want = np.float32(np.float32(1e-6) * np.float32(0.5 / 8)) + np.float32(1e-6) * np.float32(0.5 / 4)
    assert v[1, 0] == want
    # particle 2: the stored rung drops by one per kick at most, though its new rung is 2
    assert rung[2] == 7
    # particle 3: dt = eta sqrt(h / 2.8) = 1.89e-3 -> rung 10 (2^-10 <= dt < 2^-9)
    assert rung[3] == 10
    assert mr == 10


# ---------------------------------------------------------------- GPU -------

T_MAX, DT_MAX, ETA = 1.0 / 64, 1.0 / 128, 0.2


def _stepper(x, soft_len, theta=0.7):
    import oracle
    from tigergrav_b200.solver import GravitySolver
    n = len(x)
    full = GravitySolver(n, theta=theta)
    o = oracle.Oracle(theta=theta)

    def forces(xx, vv):
        full.set_particles(xx, vv).solve_gravity()
        return full.get_forces(dtype=np.float32)[1]

    def drift(xx, vv, dt):
        o.set_particles(xx, vv)
        o.drift(dt)
        return o.particles()[0]

    return orung.Stepper(x, np.zeros((n, 3), np.float32), forces, drift, T_MAX, DT_MAX, ETA, soft_len), full


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_rung_steps_match_oracle(precision):
    from tigergrav_b200 import ics
    from tigergrav_b200.solver import GravitySolver
    x = ics.halos(4096, seed=3)
    n = len(x)
    with GravitySolver(n, theta=0.7, precision=precision) as s:
        h = s.params.soft_len
        ref, full = _stepper(x, h)
        if precision == "f64":
            full.close()
            full = GravitySolver(n, theta=0.7, precision="f64")
            ref.forces = lambda xx, vv: full.set_particles(xx, vv).solve_gravity().get_forces(dtype=np.float32)[1]
        s.set_particles(x)
        state = None
        actives = []
        for k in range(12):
            state = s.rung_step(state, t_max=T_MAX, dt_max=DT_MAX, eta=ETA)
            want = ref.step()
            actives.append(state["num_active"])
            assert state == pytest.approx(want), k
            xs, vs = s.get_particles()
            assert np.array_equal(s.rungs(), ref.rung), k
            assert np.array_equal(xs, ref.x), k
            assert np.array_equal(vs, ref.v), k
        full.close()
    assert len(set(np.bincount(ref.rung).nonzero()[0])) >= 3  # several rungs in use
    assert min(actives) < n // 2  # some steps had few sinks


@pytest.mark.gpu
def test_rung_steps_cosmo_match_oracle():
    """Cosmological rung steps (tg_rung_step_cosmo): the expansion, kick_dt1 /
    kick_dt2 per rung, the drift factor and the a^-3 rung choice against the
    oracle's restatement of cosmo_advance and part_vect_kick -- positions,
    velocities, rungs and the cosmology state bit-identical over 12 steps."""
    import cosmo as oc
    from tigergrav_b200 import ics
    from tigergrav_b200.solver import GravitySolver, cosmo_rung_state
    x = ics.halos(4096, seed=3)
    n = len(x)
    H0, om, ol = 2.0, 0.3, 0.7  # a grows by ~3% over t_max = 1/64
    a0, adot0 = 1.0, 2.0
    with GravitySolver(n, theta=0.7) as s:
        ref, full = _stepper(x, s.params.soft_len)
        ref.cosmo = dict(H0=H0, omega_m=om, omega_lambda=ol, state=oc.rung_state(a0, adot0))
        s.set_particles(x)
        cs = cosmo_rung_state(a0, adot0)
        state = None
        for k in range(12):
            state = s.rung_step_cosmo(state, cs, H0, om, ol, t_max=T_MAX, dt_max=DT_MAX, eta=ETA)
            want = ref.step()
            assert state == pytest.approx(want), k
            xs, vs = s.get_particles()
            assert np.array_equal(s.rungs(), ref.rung), k
            assert np.array_equal(xs, ref.x), k
            assert np.array_equal(vs, ref.v), k
            c = ref.cosmo["state"]
            assert (cs.a, cs.adot, cs.tau, cs.a_last) == (c["a"], c["adot"], c["tau"], c["a_last"]), k
            assert np.float32(cs.time) == c["time"] and list(cs.kick1) == c["kick1"], k
        full.close()
        assert cs.a > 1.001 * a0  # the expansion moved
        # the factors differ from the static ones: the same steps without cosmology end elsewhere
        with GravitySolver(n, theta=0.7) as s0:
            s0.set_particles(x)
            st0 = None
            for k in range(12):
                st0 = s0.rung_step(st0, t_max=T_MAX, dt_max=DT_MAX, eta=ETA)
            assert not np.array_equal(s0.get_particles()[1], ref.v)


@pytest.mark.gpu
def test_rung_step_forces_state():
    from tigergrav_b200 import _lib, ics
    from tigergrav_b200.solver import GravitySolver
    x = ics.halos(4096, seed=3)
    with GravitySolver(len(x), theta=0.7) as s, GravitySolver(len(x), theta=0.7) as full:
        s.set_particles(x)
        st = s.rung_step(None, t_max=T_MAX, dt_max=DT_MAX, eta=ETA)
        for _ in range(8):  # until a step with inactive particles
            st = s.rung_step(st, t_max=T_MAX, dt_max=DT_MAX, eta=ETA)
            if st["num_active"] < len(x):
                break
        assert st["num_active"] < len(x)
        # the lists of a gated step hold active sinks only: no call may serve
        # forces or lists from them until the next full solve
        with pytest.raises(_lib.TGError):
            s.get_forces()
        with pytest.raises(_lib.TGError):
            s.forces()
        with pytest.raises(_lib.TGError):
            s.tidal(np.zeros((len(x), 3)))
        with pytest.raises(Exception):
            s.list("PP_D")
        # with all_forces every particle is a sink: forces equal a full solve's
        st = s.rung_step(st, t_max=T_MAX, dt_max=DT_MAX, eta=ETA, all_forces=True)
        xs, vs = s.get_particles()
        full.set_particles(xs, vs).solve_gravity()
        assert np.array_equal(s.get_forces(dtype=np.float32)[1], full.get_forces(dtype=np.float32)[1])
        # a step far below t_max / 2^30 is refused before any kick: velocities
        # and rungs stay as they were (only the drift has happened)
        v_before, r_before = s.get_particles()[1], s.rungs()
        with pytest.raises(_lib.TGError):
            s.rung_step(st, t_max=T_MAX, dt_max=T_MAX * 1e-12, eta=ETA)
        assert np.array_equal(s.get_particles()[1], v_before)
        assert np.array_equal(s.rungs(), r_before)


def test_oracle_stepper_time_line():
    """The oracle's main loop with a fixed force field: particle k has |g| chosen
    for rung k + 1, so the steps follow the finest rung and each particle is
    active exactly when its step divides the integer time."""
    t_max, h, eta = 1.0, 1e-3, 0.1
    # dt = eta sqrt(h / 2.8 / a) = 2^-(k+1) exactly at a_k; take a little above it
    a = np.array([(eta / 2.0 ** -(k + 1)) ** 2 * h / 2.8 * 1.001 for k in range(4)])
    g = np.zeros((4, 3), np.float32)
    g[:, 0] = a
    x0 = np.zeros((4, 3), np.int32)

    def forces(x, v):
        return g

    def drift(x, v, dt):
        return x

    st = orung.Stepper(x0, np.zeros((4, 3), np.float32), forces, drift, t_max, 0.5, eta, h)
    first = st.step()
    assert first["itime"] == 0 and first["min_rung"] == 0 and first["num_active"] == 4
    assert st.rung.tolist() == [2, 3, 4, 5] and first["max_rung"] == 5
    seen = []
    for _ in range(32):
        s = st.step()
        seen.append((s["itime"], s["min_rung"], s["num_active"]))
        assert s["itime"] % (1 << (31 - 5)) == 0  # steps of the finest rung
    # particle k (rung k + 2) is active every 2^(5 - (k + 2)) steps
    counts = [sum(1 for _, m, _ in seen if m <= r) for r in (2, 3, 4, 5)]
    assert counts == [32 // 8, 32 // 4, 32 // 2, 32]


# ---- the restated kick and drift against the reference's own ---------------
# (src/part_vect.cpp compiled into oracle/_ref/libtg_reftree.so; skipped where
# it was not built)

def _ref_tree():
    import ref_tree
    if not ref_tree.available():
        pytest.skip("oracle/_ref/libtg_reftree.so not built")
    return ref_tree


@pytest.mark.parametrize("min_rung,do_out", [(0, 0), (0, 1), (1, 0), (1, 1), (3, 0), (3, 1)])
def test_kick_matches_reference_part_vect_kick(min_rung, do_out):
    """orung.kick (the rung choice and both half kicks of the active
    particles) bit for bit against part_vect_kick itself, on accelerations
    spanning six decades so that the particles spread over many rungs"""
    rt = _ref_tree()
    rng = np.random.default_rng(10 + min_rung)
    n = 3000
    x = rng.integers(-2 ** 31, 2 ** 31, size=(n, 3), dtype=np.int64).astype(np.int32)
    v = (rng.standard_normal((n, 3)) * 0.05).astype(np.float32)
    g = (rng.standard_normal((n, 3)) * 10 ** rng.uniform(-2, 4, (n, 1))).astype(np.float32)
    rung = np.zeros(n, np.int8) if min_rung == 0 else rng.integers(0, 7, n).astype(np.int8)
    h, dt_max, eta = 0.02 / 14, 1.0 / 16, 0.2
    vr, rr, mr = rt.kick(x, v, rung, g, min_rung, do_out, dt_max, eta, h)
    vo, ro = v.copy(), rung.copy()
    mo = orung.kick(vo, ro, g, min_rung, 1.0, dt_max, eta, h)
    np.testing.assert_array_equal(vr, vo)
    np.testing.assert_array_equal(rr, ro)
    assert len(np.unique(rr)) >= 8
    assert mr == mo


@pytest.mark.parametrize("mrung", [0, 1, 4, 9])
def test_drift_matches_reference_part_vect_drift(mrung, oracle_mod):
    """the oracle's drift (x += v dt in double, wrapped, back to fixed point)
    bit for bit against part_vect_drift itself, with velocities that wrap
    particles across the box"""
    rt = _ref_tree()
    rng = np.random.default_rng(20 + mrung)
    n = 5000
    x = rng.integers(-2 ** 31, 2 ** 31, size=(n, 3), dtype=np.int64).astype(np.int32)
    v = (rng.standard_normal((n, 3)) * 0.7).astype(np.float32)
    xr = rt.drift(x, v, mrung)
    o = oracle_mod.Oracle(theta=0.7).set_particles(x, v)
    o.drift(1.0 / (1 << mrung))
    xo, _ = o.particles()
    np.testing.assert_array_equal(xr, xo)
