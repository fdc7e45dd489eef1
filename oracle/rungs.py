"""Oracle (test infrastructure only): hierarchical (rung) time steps of the
reference, restated on the CPU.

* min_rung, inc, rung_to_dt, dt_to_rung, time_to_double -- tigergrav/time.hpp:12-48.
* kick       -- part_vect_kick for the active particles (src/part_vect.cpp:358-381):
                without cosmology the second half kick is 0.5 dt of the new
                rung (the reference tests opts.ewald where opts.cosmic is
                meant, src/part_vect.cpp:376); with cosmology the half kicks
                are kick_dt1 of the old rung and kick_dt2 of the stored rung,
                and the rung follows from |g G| / a^3.  Float arithmetic where
                the reference has vect<float>: the force, the velocity and
                vect<float> * scalar (the scalar rounded to float first); the
                step in double.
* Stepper    -- the main loop (src/main.cpp:253-313): (cosmo_advance, then)
                drift every particle by the largest rung's step (or the drift
                factor), advance the integer time, forces for the particles
                with rung >= min_rung(itime), kick them.
"""
import numpy as np

RUNG_MAX = 30


def min_rung(t):
    t = int(t)
    r = 31
    while (t & 1) == 0 and r != 0:
        r -= 1
        t >>= 1
    return r


def inc(t, max_rung):
    return (int(t) + (1 << (31 - max_rung))) & 0xFFFFFFFF


def rung_to_dt(t_max, rung):
    return t_max / float(1 << int(rung))


def time_to_double(t, t_max):
    return (float(t) / float(1 << 31)) * t_max


def dt_to_rung(t_max, dt):
    """Vectorised over dt (float64 array)."""
    dt = np.asarray(dt, np.float64)
    rung = np.zeros(dt.shape, np.int64)
    while True:
        step = t_max / np.array([float(1 << int(r)) for r in rung.ravel()]).reshape(rung.shape)
        more = step > dt
        if not more.any():
            return rung
        rung[more] += 1
        if rung.max() > RUNG_MAX:
            raise ValueError("time step below t_max / 2^30")


def kick(v, rung, g, mrung, t_max, dt_max, eta, h, G=1.0, cosmo=None):
    """In place on v (float32, n x 3) and rung (int8); g float32 (n x 3).
    cosmo: None, or (kick_dt1 per rung, kick_dt2 per rung, 1 / a^3).
    Returns the largest new rung of the active particles (0 if none)."""
    act = rung.astype(np.int64) >= mrung
    idx = np.nonzero(act)[0]
    if len(idx) == 0:
        return 0
    old = rung[idx].astype(np.int64)
    vv = v[idx].copy()
    gg = g[idx].astype(np.float32)
    for r in np.unique(old[old != 0]):
        k = old == r
        dt1 = cosmo[0][r] if cosmo else 0.5 * rung_to_dt(t_max, r)
        s = np.float32(dt1 * 1.0 * G)
        vv[k] = vv[k] + gg[k] * s
    gG = gg * np.float32(G)
    a2 = (gG[:, 0] * gG[:, 0] + gG[:, 1] * gG[:, 1]) + gG[:, 2] * gG[:, 2]
    a = np.sqrt(a2).astype(np.float64)
    if cosmo:
        a = a * cosmo[2]
    eps = 10.0 * np.finfo(np.float64).tiny
    dt = eta * np.sqrt(h * (1.0 / 2.8) / (a + eps))
    dt = np.where(dt < dt_max, dt, dt_max)
    new = np.maximum(dt_to_rung(t_max, dt), mrung)
    stored = np.maximum(np.maximum(new, old - 1), 1)
    second = stored if cosmo else new
    for r in np.unique(second):
        k = second == r
        dt2 = cosmo[1][r] if cosmo else 0.5 * rung_to_dt(t_max, r)
        s = np.float32(dt2 * 1.0 * G)
        vv[k] = vv[k] + gg[k] * s
    v[idx] = vv
    rung[idx] = stored.astype(np.int8)
    return int(new.max())


class Stepper:
    """forces(x, v) -> float32 (n x 3) accelerations per unit G, caller order;
    drift(x, v, dt) -> new int32 positions."""

    def __init__(self, x, v, forces, drift, t_max, dt_max, eta, h, G=1.0, cosmo=None):
        """cosmo: None, or dict(H0, omega_m, omega_lambda, state) with state
        from cosmo.rung_state (advanced in place)."""
        self.x = np.array(x, np.int32)
        self.v = np.array(v, np.float32)
        self.rung = np.zeros(len(self.x), np.int8)
        self.forces, self.drift = forces, drift
        self.t_max, self.dt_max, self.eta, self.h, self.G = t_max, dt_max, eta, h, G
        self.itime, self.max_rung, self.min_rung, self.num_active = 0, -1, 0, 0
        self.cosmo = cosmo

    def step(self):
        step = rung_to_dt(self.t_max, self.max_rung) if self.max_rung >= 0 else 0.0
        drift_dt, factors = step, None
        if self.cosmo is not None:
            import cosmo as oc
            c = self.cosmo
            drift_dt, k1, k2, a3inv = oc.rung_advance(c["state"], step, self.t_max, c["H0"], c["omega_m"],
                                                      c["omega_lambda"])
            factors = (k1, k2, a3inv)
        if self.max_rung >= 0:
            self.x = self.drift(self.x, self.v, drift_dt)
            self.itime = inc(self.itime, self.max_rung)
        mr = min_rung(self.itime)
        g = self.forces(self.x, self.v)
        self.num_active = int((self.rung.astype(np.int64) >= mr).sum())
        self.max_rung = kick(self.v, self.rung, g, mr, self.t_max, self.dt_max, self.eta, self.h, self.G,
                             cosmo=factors)
        self.min_rung = mr
        return dict(itime=self.itime, max_rung=self.max_rung, min_rung=mr, num_active=self.num_active,
                    t=time_to_double(self.itime, self.t_max))
