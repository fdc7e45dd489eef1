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
        dtau1, da1, dadot1, ddr1, dk1 = dt / a, adot * dt, dadot(a) * dt, dt / (a * a), dt / a
        a2, ad2 = a + 0.5 * da1, adot + 0.5 * dadot1
        dtau2, da2, dadot2, ddr2, dk2 = dt / a2, ad2 * dt, dadot(a2) * dt, dt / (a2 * a2), dt / a2
        a3, ad3 = a + 0.5 * da2, adot + 0.5 * dadot2
        dtau3, da3, dadot3, ddr3, dk3 = dt / a3, ad3 * dt, dadot(a3) * dt, dt / (a3 * a3), dt / a3
        a4, ad4 = a + da3, adot + dadot3
        dtau4, da4, dadot4, ddr4, dk4 = dt / a4, ad4 * dt, dadot(a4) * dt, dt / (a4 * a4), dt / a4
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
