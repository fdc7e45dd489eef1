/*
 * tg_cosmo.cu -- the cosmological kick and drift factors (cosmos::
 * advance_to_time and cosmo_advance, src/cosmo.cpp:50-106,187-218), host
 * code behind the C ABI.
 *
 * The expansion a(t) follows the Friedmann acceleration of the reference,
 * a'' = H0^2 (-omega_m / (2 a^2) + omega_lambda a), integrated with the same
 * fixed-step RK4 (steps of 1e-3 a / a'), which also accumulates
 * tau = int dt / a, the drift factor int dt / a^2 and the kick factor
 * int dt / a.  For one kick-drift-kick step of length dt from t:
 *   kick1 = int_t^{t+dt/2} dt'/a,  drift = int_t^{t+dt} dt'/a^2,
 *   kick2 = int_{t+dt/2}^{t+dt} dt'/a,
 * the factors cosmo_advance gives the reference's kick (kick_dt2, then
 * kick_dt1 of the next call) and drift.  They replace dt in tg_kick and
 * tg_drift; with cosmology off the factors are dt/2, dt, dt/2 (a clean KDK,
 * without the reference's zero second half-kick, src/part_vect.cpp:376).
 */
#include <cmath>

namespace tg {

struct Cosmos {
    double a, adot, tau, drift, kick;
};

/* cosmos::advance_to_time (src/cosmo.cpp:50-106) */
static void cosmo_advance_to(Cosmos &c, double t0, const tg_cosmo_params &p) {
    const double H0 = p.H0, om = p.omega_m, ol = p.omega_lambda;
    auto dadot = [&](double a) { return H0 * H0 * (-0.5 * om / (a * a) + a * ol); };
    double t = 0.0;
    bool done = false;
    const double sgn = t0 < 0.0 ? -1.0 : 1.0;
    c.kick = c.drift = 0.0;
    if (t0 == 0.0) return;
    do {
        double dt = sgn * 1e-3 * c.a / c.adot;
        if (std::abs(t + dt) > std::abs(t0)) {
            done = true;
            dt = std::abs(t0 - t) * sgn;
        }
        const double a = c.a, ad = c.adot;
        /* four stages of (tau, a, adot, drift, kick): each rate times dt, as
         * the reference's lambdas give them ((1 / a) dt, not dt / a) */
        auto stage = [&](double aa, double aad, double *k) {
            k[0] = (1.0 / aa) * dt;
            k[1] = aad * dt;
            k[2] = dadot(aa) * dt;
            k[3] = (1.0 / (aa * aa)) * dt;
            k[4] = (1.0 / aa) * dt;
        };
        double k1[5], k2[5], k3[5], k4[5];
        stage(a, ad, k1);
        stage(a + 0.5 * k1[1], ad + 0.5 * k1[2], k2);
        stage(a + 0.5 * k2[1], ad + 0.5 * k2[2], k3);
        stage(a + k3[1], ad + k3[2], k4);
        double d[5];
        for (int q = 0; q < 5; q++) d[q] = (k1[q] + 2.0 * (k2[q] + k3[q]) + k4[q]) / 6.0;
        c.tau += d[0];
        c.a += d[1];
        c.adot += d[2];
        c.drift += d[3];
        c.kick += d[4];
        t += dt;
    } while (!done);
}

} // namespace tg

extern "C" int tg_cosmo_kdk(const tg_cosmo_params *p, double *state, double dt, double *factors) {
    if (!p || !state || !factors || !std::isfinite(dt)) return TG_ERR_ARG;
    if (!(state[0] > 0.0) || !(state[1] > 0.0) || !std::isfinite(p->H0) || !(p->H0 > 0.0)) return TG_ERR_ARG;
    tg::Cosmos c{state[0], state[1], state[2], 0.0, 0.0};
    /* first half kick: from t to t + dt/2 */
    tg::Cosmos h = c;
    tg::cosmo_advance_to(h, 0.5 * dt, *p);
    factors[0] = h.kick;
    /* drift over the whole step, and the new state */
    tg::Cosmos e = c;
    tg::cosmo_advance_to(e, dt, *p);
    factors[1] = e.drift;
    /* second half kick: from t + dt to t + dt/2, backwards, negated */
    tg::Cosmos b = e;
    tg::cosmo_advance_to(b, -0.5 * dt, *p);
    factors[2] = -b.kick;
    state[0] = e.a;
    state[1] = e.adot;
    state[2] = e.tau;
    return TG_OK;
}

extern "C" int tg_leapfrog_cosmo(tg_solver *s, const tg_cosmo_params *p, double *state, double dt, int n_steps,
                                 void *stream) {
    if (!s || !p || !state || n_steps < 0) return TG_ERR_ARG;
    if (!s->S.have_forces) TG_TRY(tg_solve_gravity(s, stream));
    /* each step's closing kick fused with the next step's opening kick and drift */
    double close = 0.0;
    for (int k = 0; k < n_steps; k++) {
        double f[3];
        TG_TRY(tg_cosmo_kdk(p, state, dt, f));
        TG_TRY(tg_kick_drift(s, close, f[0], f[1], stream));
        TG_TRY(tg_solve_gravity(s, stream));
        close = f[2];
    }
    if (n_steps > 0) TG_TRY(tg_kick(s, close, stream));
    return TG_OK;
}
