"""Oracle (test infrastructure): restatement of the reference's cosmology
integrator, cosmos::advance_to_time (src/cosmo.cpp:50-106), and of the KDK
factors cosmo_advance derives from it (src/cosmo.cpp:187-218)."""


def advance_to_time(state, t0, H0, omega_m, omega_lambda):
    """state = [a, adot, tau]; returns (new state, drift, kick) after t0."""
    a, adot, tau = state
    dadot = lambda a_: H0 * H0 * (-0.5 * omega_m / (a_ * a_) + a_ * omega_lambda)
    t, done = 0.0, False
    sgn = -1.0 if t0 < 0.0 else 1.0
    drift = kick = 0.0
    if t0 == 0.0:
        return [a, adot, tau], 0.0, 0.0
    while not done:
        dt = sgn * 1e-3 * a / adot
        if abs(t + dt) > abs(t0):
            done = True
            dt = abs(t0 - t) * sgn
        # each rate times dt, as the reference's lambdas give them: (1 / a) dt, ...
        dtau1, da1, dadot1, ddr1, dk1 = (1.0 / a) * dt, adot * dt, dadot(a) * dt, (1.0 / (a * a)) * dt, (1.0 / a) * dt
        a2, ad2 = a + 0.5 * da1, adot + 0.5 * dadot1
        dtau2, da2, dadot2 = (1.0 / a2) * dt, ad2 * dt, dadot(a2) * dt
        ddr2, dk2 = (1.0 / (a2 * a2)) * dt, (1.0 / a2) * dt
        a3, ad3 = a + 0.5 * da2, adot + 0.5 * dadot2
        dtau3, da3, dadot3 = (1.0 / a3) * dt, ad3 * dt, dadot(a3) * dt
        ddr3, dk3 = (1.0 / (a3 * a3)) * dt, (1.0 / a3) * dt
        a4, ad4 = a + da3, adot + dadot3
        dtau4, da4, dadot4 = (1.0 / a4) * dt, ad4 * dt, dadot(a4) * dt
        ddr4, dk4 = (1.0 / (a4 * a4)) * dt, (1.0 / a4) * dt
        tau += (dtau1 + 2.0 * (dtau2 + dtau3) + dtau4) / 6.0
        a += (da1 + 2.0 * (da2 + da3) + da4) / 6.0
        adot += (dadot1 + 2.0 * (dadot2 + dadot3) + dadot4) / 6.0
        drift += (ddr1 + 2.0 * (ddr2 + ddr3) + ddr4) / 6.0
        kick += (dk1 + 2.0 * (dk2 + dk3) + dk4) / 6.0
        t += dt
    return [a, adot, tau], drift, kick


def kdk_factors(state, dt, H0, omega_m, omega_lambda):
    """(new state, [kick over the first half, drift, kick over the second half])"""
    _, _, k1 = advance_to_time(state, 0.5 * dt, H0, omega_m, omega_lambda)
    new, drift, _ = advance_to_time(state, dt, H0, omega_m, omega_lambda)
    _, _, kb = advance_to_time(new, -0.5 * dt, H0, omega_m, omega_lambda)
    return new, [k1, drift, -kb]


def rung_advance(cs, dt, t_max, H0, omega_m, omega_lambda, rung_max=30):
    """cosmo_advance (src/cosmo.cpp:187-218) on a rung-step state
    cs = dict(a, adot, tau, a_last, time (float32), kick1 (list of 31)):
    returns (drift factor, kick_dt1 per rung, kick_dt2 per rung, 1 / a_last^3)."""
    import numpy as np
    last = [cs["a"], cs["adot"], cs["tau"]]
    cs["a_last"] = cs["a"]
    cs["time"] = np.float32(np.float64(cs["time"]) + dt)
    now, drift = last, 0.0
    if dt != 0.0:
        now, drift, _ = advance_to_time(last, dt, H0, omega_m, omega_lambda)
    k2 = []
    for i in range(rung_max + 1):
        dti = t_max / float(1 << i)
        if float(cs["time"]) >= dti:
            _, _, kb = advance_to_time(now, -0.5 * dti, H0, omega_m, omega_lambda)
            cs["kick1"][i] = -kb
        _, _, kf = advance_to_time(now, 0.5 * dti, H0, omega_m, omega_lambda)
        k2.append(kf)
    cs["a"], cs["adot"], cs["tau"] = now
    return drift, list(cs["kick1"]), k2, 1.0 / (cs["a_last"] * cs["a_last"] * cs["a_last"])


def rung_state(a, adot):
    """the reference's starting state: kick_dt1 = {-1, 0, ...} (src/cosmo.cpp:12)"""
    import numpy as np
    return dict(a=a, adot=adot, tau=0.0, a_last=a, time=np.float32(0.0), kick1=[-1.0] + [0.0] * 30)
