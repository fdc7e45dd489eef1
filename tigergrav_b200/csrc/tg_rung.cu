/*
 * tg_rung.cu -- hierarchical (rung) time steps: the integer time line of
 * tigergrav/time.hpp:12-48, the step of the main loop (src/main.cpp:266-313)
 * and the rung kick of part_vect_kick (src/part_vect.cpp:340-381), with only
 * the active particles as sinks in the walk (src/tree.cpp:396, 603).
 *
 * Time is an integer in units of t_max / 2^31; rung r has step t_max / 2^r.
 * A step drifts every particle by the step of the largest rung the previous
 * kick produced, advances the integer time by that step, and solves gravity
 * for the particles with rung >= min_rung(time) (the lowest rung whose step
 * divides the time).  Each active particle then closes its previous step with
 * a half kick of its old rung (skipped on rung 0, the first call), takes the
 * rung of dt = min(dt_max, eta sqrt(h / 2.8 / |g G|)), at least min_rung,
 * and opens the next step with a half kick of that rung; its stored rung is
 * max(rung, old - 1, 1).  The second half kick is 0.5 dt(rung) without
 * cosmology: the reference tests opts.ewald where it means opts.cosmic
 * (src/part_vect.cpp:376), which zeroes it in a periodic non-cosmological
 * run; the intended test is used here.  Arithmetic follows the reference's
 * types: the force and velocity in float, vect<float> * scalar as a float
 * product, the time step in double.
 *
 * GPU form: an active flag per particle (sorted order) and its exclusive
 * scan give every node's active count in O(1) (nodes are particle ranges);
 * the walk gives nodes with no active particle no lists and leaves them out
 * of the leaf set, so the force kernels only visit active leaves.  The rung
 * kick is one thread per particle.  The rung is kept in vel[i].w, which the
 * tree build permutes with the velocity.
 */
#include <cub/cub.cuh>

namespace tg {

constexpr int RUNG_MAX = 30; /* tigergrav/time.hpp:10 */

/* min_rung (tigergrav/time.hpp:23-30) */
static int host_min_rung(uint32_t t) {
    int r = 31;
    while ((t & 1u) == 0u && r != 0) {
        r--;
        t >>= 1;
    }
    return r;
}

__host__ __device__ __forceinline__ double rung_dt(double t_max, int rung) {
    return t_max / (double)(1 << rung); /* rung_to_dt, tigergrav/time.hpp:32-35 */
}

__global__ void k_rung_flags(int64_t n, const float4 *__restrict__ vel, int min_rung, int32_t *__restrict__ flag) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    flag[i] = (i < n && (int)vel[i].w >= min_rung) ? 1 : 0;
}

__global__ void k_node_active(int64_t nn, const int32_t *__restrict__ pb, const int32_t *__restrict__ pe,
                              const int32_t *__restrict__ scan, int32_t *__restrict__ nact) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    nact[i] = scan[pe[i]] - scan[pb[i]];
}

/* the cosmological kick factors of one step, per rung (cosmo_kick_dt1 /
 * cosmo_kick_dt2, src/cosmo.cpp:19-25), and the 1 / a^3 of the rung choice */
struct RungCosmo {
    int cosmic;
    double a3inv;
    double k1[RUNG_MAX + 1], k2[RUNG_MAX + 1];
};

/* part_vect_kick for one active particle (src/part_vect.cpp:358-381).
 * WRITE = false only checks that every new rung is representable (err bit 8),
 * so a step that fails leaves velocities and rungs untouched.  Cosmological:
 * the first half kick uses kick_dt1 of the old rung, the acceleration of the
 * rung choice is |g G| / a^3, the second half kick kick_dt2 of the stored
 * rung; otherwise half a step of the old rung and of the new (unclamped) one. */
template <bool WRITE>
__global__ void k_rung_kick(int64_t n, float4 *__restrict__ vel, const float4 *__restrict__ acc,
                            const double *__restrict__ accd, int min_rung, double t_max, double dt_max, double eta,
                            double h, double G, RungCosmo CZ, int *__restrict__ max_rung, uint32_t *__restrict__ err) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = vel[i];
    const int old = (int)v.w;
    if (old < min_rung) return;
    float g[3];
    if (accd) {
        for (int d = 0; d < 3; d++) g[d] = __double2float_rn(accd[4 * i + 1 + d]);
    } else {
        const float4 a = acc[i];
        g[0] = a.y;
        g[1] = a.z;
        g[2] = a.w;
    }
    if (old != 0) { /* close the previous step: v += g (0.5 dt(old) G) */
        const double dt1 = CZ.cosmic ? CZ.k1[old] : __dmul_rn(0.5, rung_dt(t_max, old));
        const float s = __double2float_rn(__dmul_rn(dt1, G));
        v.x = __fadd_rn(v.x, __fmul_rn(g[0], s));
        v.y = __fadd_rn(v.y, __fmul_rn(g[1], s));
        v.z = __fadd_rn(v.z, __fmul_rn(g[2], s));
    }
    /* |g G| in float, then the step in double */
    const float fG = __double2float_rn(G);
    const float gx = __fmul_rn(g[0], fG), gy = __fmul_rn(g[1], fG), gz = __fmul_rn(g[2], fG);
    const float a2 = __fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)), __fmul_rn(gz, gz));
    const double a = CZ.cosmic ? __dmul_rn((double)__fsqrt_rn(a2), CZ.a3inv) : (double)__fsqrt_rn(a2);
    const double eps = 10.0 * 2.2250738585072014e-308;
    double dt = __dmul_rn(eta, __dsqrt_rn(__ddiv_rn(__dmul_rn(h, 1.0 / 2.8), __dadd_rn(a, eps))));
    dt = dt_max < dt ? dt_max : dt;
    int rung = 0;
    while (rung_dt(t_max, rung) > dt) { /* dt_to_rung (tigergrav/time.hpp:37-47) */
        if (++rung > RUNG_MAX) {
            atomicOr(err, 8u);
            rung = RUNG_MAX;
            break;
        }
    }
    if (!WRITE) return;
    rung = max(rung, min_rung);
    atomicMax(max_rung, rung);
    const int stored = max(max(rung, old - 1), 1);
    const double dt2 = CZ.cosmic ? CZ.k2[stored] : __dmul_rn(0.5, rung_dt(t_max, rung));
    const float s2 = __double2float_rn(__dmul_rn(dt2, G));
    v.x = __fadd_rn(v.x, __fmul_rn(g[0], s2));
    v.y = __fadd_rn(v.y, __fmul_rn(g[1], s2));
    v.z = __fadd_rn(v.z, __fmul_rn(g[2], s2));
    v.w = (float)stored;
    vel[i] = v;
}

__global__ void k_get_rungs(int64_t n, const int4 *__restrict__ pos, const float4 *__restrict__ vel,
                            int8_t *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[pos[i].w] = (int8_t)(int)vel[i].w;
}

/* gravity for the particles with rung >= min_rung (every particle a sink when all) */
static int solve_active(Solver &S, int min_rung, bool all, int64_t *num_active, cudaStream_t st) {
    const int64_t n = S.n;
    TG_TRY(tree_build(S, st));
    TG_TRY(tree_multipoles(S, st));
    const int64_t nn = S.nnodes;
    TG_TRY(ensure(S.rung_flag, n + 1));
    TG_TRY(ensure(S.rung_scan, n + 1));
    TG_TRY(ensure(S.rung_nact, nn));
    k_rung_flags<<<(int)((n + 256) / 256), 256, 0, st>>>(n, S.vel.p, min_rung, S.rung_flag.p);
    TG_TRY(launched(S));
    size_t tmp = 0;
    TG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, S.rung_flag.p, S.rung_scan.p, (int)(n + 1), st));
    TG_TRY(ensure(S.cub_tmp, tmp));
    TG_CUDA(cub::DeviceScan::ExclusiveSum(S.cub_tmp.p, tmp, S.rung_flag.p, S.rung_scan.p, (int)(n + 1), st));
    k_node_active<<<(int)((nn + 255) / 256), 256, 0, st>>>(nn, S.nd_pb.p, S.nd_pe.p, S.rung_scan.p, S.rung_nact.p);
    TG_TRY(launched(S));
    int32_t na = 0;
    TG_CUDA(cudaMemcpyAsync(&na, S.rung_scan.p + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    *num_active = na;
    S.walk_nact = all ? nullptr : S.rung_nact.p;
    const int rc = tree_walk(S, st);
    S.walk_nact = nullptr;
    TG_TRY(rc);
    TG_TRY(gravity_forces(S, st));
    if (!all) {
        /* forces of inactive leaves were not evaluated, and the lists hold
         * active sinks only: neither may serve tg_forces, tg_get_forces,
         * tg_tidal or tg_get_list */
        S.have_forces = false;
        S.have_lists = false;
    }
    return TG_OK;
}

static int rung_kick(Solver &S, const tg_rung_params &p, const RungCosmo &CZ, int min_rung, int *max_rung,
                     cudaStream_t st) {
    const int64_t n = S.n;
    const bool f64 = S.prm.precision == TG_PREC_F64;
    TG_CUDA(cudaMemsetAsync(S.dev_cnt.p, 0, sizeof(unsigned long long), st));
    TG_CUDA(cudaMemsetAsync(S.dev_err.p, 0, sizeof(uint32_t), st));
    const int nb = (int)((n + 255) / 256);
    /* check pass first: on a rung overflow nothing is kicked */
    k_rung_kick<false><<<nb, 256, 0, st>>>(n, S.vel.p, f64 ? nullptr : S.acc.p, f64 ? S.accd.p : nullptr, min_rung,
                                           p.t_max, p.dt_max, p.eta, S.prm.soft_len, S.prm.G, CZ, (int *)S.dev_cnt.p,
                                           S.dev_err.p);
    TG_TRY(launched(S));
    uint32_t err = 0;
    TG_TRY(read_err(S, st, &err));
    if (err) return TG_ERR_ARG; /* a step below t_max / 2^30 */
    k_rung_kick<true><<<nb, 256, 0, st>>>(n, S.vel.p, f64 ? nullptr : S.acc.p, f64 ? S.accd.p : nullptr, min_rung,
                                          p.t_max, p.dt_max, p.eta, S.prm.soft_len, S.prm.G, CZ, (int *)S.dev_cnt.p,
                                          S.dev_err.p);
    TG_TRY(launched(S));
    int mr = 0;
    TG_CUDA(cudaMemcpyAsync(&mr, S.dev_cnt.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    *max_rung = mr;
    return TG_OK;
}

/* cosmo_advance (src/cosmo.cpp:187-218) on the rung step's cosmology state:
 * last = now; time += dt (a float, as the reference's this_time); now advanced
 * by dt; per rung i with step dt_i: kick_dt1[i] = the kick back over dt_i / 2
 * (kept from earlier steps while time < dt_i), kick_dt2[i] = the kick ahead
 * over dt_i / 2; the drift factor over [last, now]. */
static void cosmo_rung_advance(tg_cosmo_rung_state &cs, const tg_cosmo_params &cp, double t_max, double dt,
                               RungCosmo &CZ, double *drift_dt) {
    const Cosmos last{cs.a, cs.adot, cs.tau, 0.0, 0.0};
    cs.a_last = cs.a;
    cs.time = (float)((double)cs.time + dt);
    Cosmos now = last;
    if (dt != 0.0) cosmo_advance_to(now, dt, cp);
    for (int i = 0; i <= RUNG_MAX; i++) {
        const double dti = rung_dt(t_max, i);
        if ((double)cs.time >= dti) {
            Cosmos c1 = now;
            cosmo_advance_to(c1, -0.5 * dti, cp);
            cs.kick1[i] = -c1.kick;
        }
        Cosmos c2 = now;
        cosmo_advance_to(c2, 0.5 * dti, cp);
        CZ.k2[i] = c2.kick;
        CZ.k1[i] = cs.kick1[i];
    }
    *drift_dt = now.drift;
    cs.a = now.a;
    cs.adot = now.adot;
    cs.tau = now.tau;
    /* the rung choice divides by a^3 at the start of the step (cosmo_scale().first) */
    CZ.cosmic = 1;
    CZ.a3inv = 1.0 / (cs.a_last * cs.a_last * cs.a_last);
}

static int rung_step(tg_solver *s, const tg_rung_params *p, tg_rung_state *state, const tg_cosmo_params *cp,
                     tg_cosmo_rung_state *cs, int all_forces, void *stream) {
    if (!s || !p || !state) return TG_ERR_ARG;
    if (!(p->t_max > 0.0) || !(p->dt_max > 0.0) || !(p->eta > 0.0) || !std::isfinite(p->t_max)) return TG_ERR_ARG;
    Solver &S = s->S;
    if (S.n <= 0) return TG_ERR_STATE;
    if (state->max_rung > RUNG_MAX) return TG_ERR_ARG;
    TG_CUDA(cudaSetDevice(S.dev));
    cudaStream_t st = (cudaStream_t)stream;
    /* the states change only when the whole step succeeds */
    uint32_t itime = state->itime;
    RungCosmo CZ{};
    tg_cosmo_rung_state cnext{};
    double step = state->max_rung >= 0 ? rung_dt(p->t_max, state->max_rung) : 0.0;
    double drift_dt = step;
    if (cp) {
        cnext = *cs;
        cosmo_rung_advance(cnext, *cp, p->t_max, step, CZ, &drift_dt); /* before the drift (src/main.cpp:266-268) */
    }
    if (state->max_rung >= 0) {
        /* drift by the step of the largest rung, advance the integer time (src/main.cpp:284-299) */
        TG_TRY(drift(S, drift_dt, st));
        itime += 1u << (31 - state->max_rung);
    }
    const int mr = host_min_rung(itime);
    int64_t na = 0;
    TG_TRY(solve_active(S, mr, all_forces != 0, &na, st));
    int max_rung = 0;
    TG_TRY(rung_kick(S, *p, CZ, mr, &max_rung, st));
    state->itime = itime;
    state->min_rung = mr;
    state->max_rung = max_rung;
    state->num_active = na;
    state->t = ((double)itime / 2147483648.0) * p->t_max; /* time_to_double */
    if (cp) *cs = cnext;
    return TG_OK;
}

} // namespace tg

extern "C" int tg_rung_step(tg_solver *s, const tg_rung_params *p, tg_rung_state *state, int all_forces,
                            void *stream) {
    return tg::rung_step(s, p, state, nullptr, nullptr, all_forces, stream);
}

extern "C" int tg_rung_step_cosmo(tg_solver *s, const tg_rung_params *p, tg_rung_state *state,
                                  const tg_cosmo_params *cp, tg_cosmo_rung_state *cs, int all_forces, void *stream) {
    if (!cp || !cs || !(cs->a > 0.0) || !(cs->adot > 0.0) || !(cp->H0 > 0.0) || !std::isfinite(cp->H0))
        return TG_ERR_ARG;
    return tg::rung_step(s, p, state, cp, cs, all_forces, stream);
}

extern "C" int tg_cosmo_rung_init(tg_cosmo_rung_state *cs, double a, double adot) {
    if (!cs || !(a > 0.0) || !(adot > 0.0)) return TG_ERR_ARG;
    *cs = tg_cosmo_rung_state{};
    cs->a = a;
    cs->adot = adot;
    cs->a_last = a;
    cs->kick1[0] = -1.0; /* the reference's initialiser, src/cosmo.cpp:12 */
    return TG_OK;
}

extern "C" int tg_get_rungs(tg_solver *s, int8_t *rung, int where, void *stream) {
    if (!s || !rung || (where != TG_HOST && where != TG_DEVICE)) return TG_ERR_ARG;
    tg::Solver &S = s->S;
    if (S.n <= 0) return TG_ERR_STATE;
    TG_CUDA(cudaSetDevice(S.dev));
    cudaStream_t st = (cudaStream_t)stream;
    int8_t *out = rung;
    if (where == TG_HOST) {
        TG_TRY(tg::ensure(S.rung_out, S.n));
        out = S.rung_out.p;
    }
    tg::k_get_rungs<<<(int)((S.n + 255) / 256), 256, 0, st>>>(S.n, S.pos.p, S.vel.p, out);
    TG_TRY(tg::launched(S));
    if (where == TG_HOST) TG_CUDA(cudaMemcpyAsync(rung, out, S.n, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    return TG_OK;
}
