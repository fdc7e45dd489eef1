/*
 * tg_adjoint.cu -- reverse-mode differentiation of the kick-drift-kick
 * leapfrog (part_vect_kick / part_vect_drift, src/part_vect.cpp:341-436,
 * 493-540, driven as in src/main.cpp:258-273) through the tree forces.
 *
 * Forward (forward_steps): K leapfrog steps; the particle state (positions
 * and velocities, caller order) is checkpointed before the first step and
 * after every step.
 *
 * Backward (backward_steps): with J(x) = dg/dx the Jacobian of the
 * accelerations and (lx, lv) the adjoints of (x, v) at the end,
 *     lx += dt/2 G J(x_K) lv
 *     for s = K-1 .. 0:   lv += dt lx;   lx += c_s G J(x_s) lv
 * with c_s = dt for s > 0 (the half kicks of steps s-1 and s share x_s) and
 * dt/2 for s = 0.  J is symmetric, so J^T lv = J lv.  Each J(x_s) lv
 * rebuilds the tree, multipoles, lists and local expansions at the
 * checkpoint x_s (recomputation instead of storing them) and then runs
 * k_tidal_leaf, which contracts with the upstream gradient u = lv:
 *   far field   the tidal tensor of the leaf's local expansion L at the
 *               particle (L2P differentiated once more), times u_i;
 *   PC (direct and Ewald)  the tidal tensor of each source multipole
 *               (monopole and quadrupole terms of M2P differentiated) times u_i;
 *   PP (direct and Ewald)  each pair's Hessian times (u_i - u_j): the exact
 *               derivative of the pair force with respect to both particles.
 * Not differentiated: how a source node's multipoles and a sink node's
 * local expansion move with the positions of the particles inside the
 * source node (the far field's source side) and the octupole term of the
 * PC tidal tensor.  For upstream gradients that do not vary smoothly across
 * the box these are small against the terms kept; the finite-difference
 * tests measure the result.
 */
#include "tg_solver.cuh"

namespace tg {

/* dg/d(dX) of the local expansion at dX (L2P's force differentiated once
 * more), as 6 values in I2 order */
__device__ __forceinline__ void L2T(const double *L, const double *dX, double *T6) {
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int e = a; e < 3; e++) {
            double v = L[E2(a, e)];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                v += L[E3(a, e, c)] * dX[c];
#pragma unroll
                for (int d = c; d < 3; d++) v += L[E4(a, e, c, d)] * dX[c] * dX[d] * factor<double>(E2(c, d));
            }
            T6[I2(a, e)] = -v;
        }
}

/* dg/dx_sink of M2P (contract_M2P) for the monopole and quadrupole terms */
template <class T>
__device__ __forceinline__ void M2T(const T *M, const T *D, T *T6) {
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int e = a; e < 3; e++) {
            T v = M[0] * D[E2(a, e)];
#pragma unroll
            for (int b = 0; b < 3; b++)
#pragma unroll
                for (int c = b; c < 3; c++) v += M[M2(c, b)] * D[E4(a, b, c, e)] * factor<T>(E2(c, b));
            T6[I2(a, e)] = -v;
        }
}

/* Hessian part of the softened pair force g -= m dX f(r) (pp_direct_pair):
 * d(dX f)/d(dX) = f I + dX dX^T f'(r)/r; returns f and f'(r)/r */
template <class T>
__device__ __forceinline__ void pp_pair_deriv(const GParams &P, T r2, T &f, T &fpr) {
    const T h = T(P.h);
    if (r2 > h * h) {
        const T rinv = t_rsqrt(r2);
        const T rinv2 = rinv * rinv;
        f = rinv2 * rinv;
        fpr = T(-3) * f * rinv2;
        return;
    }
    const T r = t_sqrt(r2);
    const T u = r / h;
    const T hinv = T(1) / h;
    if (r < T(0.5) * h) {
        /* f3 = (32 u^3 - 192/5 u^2 + 32/3) / h^3 */
        f = ((T(32) * u - T(192.0 / 5.0)) * u * u + T(32.0 / 3.0)) * hinv * hinv * hinv;
        fpr = (T(96) * u - T(384.0 / 5.0)) * hinv * hinv * hinv * hinv * hinv;
        return;
    }
    /* f2 = P(u) / r^3, P = -32/3 u^6 + 192/5 u^5 - 48 u^4 + 64/3 u^3 - 1/15 */
    const T u3 = u * u * u;
    const T Pu = ((((T(-32.0 / 3.0) * u + T(192.0 / 5.0)) * u - T(48)) * u + T(64.0 / 3.0)) * u3) - T(1.0 / 15.0);
    const T dPu = (((T(-64) * u + T(192)) * u - T(192)) * u + T(64)) * u * u;
    const T rinv = T(1) / r;
    const T rinv3 = rinv * rinv * rinv;
    f = Pu * rinv3;
    fpr = (dPu * hinv * rinv - T(3) * Pu * rinv * rinv) * rinv3;
}

template <class T>
__device__ __forceinline__ void sym_mul_add(const T *T6, const T *u, Acc<T> *o) {
    o[0].add(T6[I2(0, 0)] * u[0] + T6[I2(0, 1)] * u[1] + T6[I2(0, 2)] * u[2]);
    o[1].add(T6[I2(0, 1)] * u[0] + T6[I2(1, 1)] * u[1] + T6[I2(1, 2)] * u[2]);
    o[2].add(T6[I2(0, 2)] * u[0] + T6[I2(1, 2)] * u[1] + T6[I2(2, 2)] * u[2]);
}

/* U_B = sum over the node's particles of m u_j (the mass-weighted upstream
 * gradient, i.e. M_B times the first-order shift of its centre of mass):
 * one warp per node, u in sorted order */
__global__ void k_node_usum(int64_t nn, double m, const int32_t *__restrict__ pb, const int32_t *__restrict__ pe,
                            const double *__restrict__ u, double *__restrict__ U) {
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= nn) return;
    double s[3] = {0.0, 0.0, 0.0};
    for (int64_t q = pb[i] + lane; q < pe[i]; q += 32)
        for (int d = 0; d < 3; d++) s[d] += u[3 * q + d];
    for (int d = 0; d < 3; d++) {
        const double v = warp_sum(s[d]);
        if (lane == 0) U[3 * i + d] = m * v;
    }
}

/* The source side of the node stage: a source of mass M at X whose particles
 * move by u shifts its centre by U/M, which changes the acceleration it causes
 * at the sink by D2(X_sink - X) U (monopole order).  V_A sums this over the
 * CC and CP lists of node A (direct and Ewald), evaluated at A's centre.
 * One warp per node, lanes over sources. */
template <class T>
__global__ void __launch_bounds__(128) k_vfield_node(GParams P, int64_t nn, const int32_t *__restrict__ pb,
                                                     const int32_t *__restrict__ pe, const MSrc *__restrict__ ms,
                                                     const int4 *__restrict__ pos, ListView LV, EwaldTables E,
                                                     const double *__restrict__ U, const double *__restrict__ us,
                                                     double *__restrict__ V) {
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= nn) return;
    double acc[3] = {0.0, 0.0, 0.0};
    if (pe[i] > pb[i]) {
        const int32_t X[3] = {ms[i].x[0], ms[i].x[1], ms[i].x[2]};
        const bool per = P.ewald != 0;
        for (int ew = 0; ew < (per ? 2 : 1); ew++) {
            const int kcc = ew ? TG_CC_E : TG_CC_D, kcp = ew ? TG_CP_E : TG_CP_D;
            const int32_t *lcc = LV.pool[kcc] + LV.off[kcc][i];
            const int32_t ncc = LV.len[kcc][i];
            for (int32_t j = lane; j < ncc; j += 32) {
                const int32_t src = lcc[j];
                T dX[3], D[LP];
                for (int d = 0; d < 3; d++) dX[d] = sep<T>(X[d], ms[src].x[d], ew ? true : per);
                if (ew) green_ewald_full<T>(E, dX, D);
                else green_direct<T>(dX, D);
                const double Ub[3] = {U[3 * (int64_t)src], U[3 * (int64_t)src + 1], U[3 * (int64_t)src + 2]};
                for (int a = 0; a < 3; a++)
                    acc[a] += (double)D[E2(a, 0)] * Ub[0] + (double)D[E2(a, 1)] * Ub[1] + (double)D[E2(a, 2)] * Ub[2];
            }
            const int32_t *lcp = LV.pool[kcp] + LV.off[kcp][i];
            const int32_t ncp = LV.len[kcp][i];
            for (int32_t c = 0; c < ncp; c++) {
                const int32_t src = lcp[c];
                for (int32_t q = pb[src] + lane; q < pe[src]; q += 32) {
                    const int4 y = pos[q];
                    const int32_t yy[3] = {y.x, y.y, y.z};
                    T dX[3], D[LP];
                    for (int d = 0; d < 3; d++) dX[d] = sep<T>(X[d], yy[d], ew ? true : per);
                    if (ew) green_ewald_full<T>(E, dX, D);
                    else green_direct<T>(dX, D);
                    for (int a = 0; a < 3; a++)
                        acc[a] += P.m_d * ((double)D[E2(a, 0)] * us[3 * (int64_t)q] +
                                           (double)D[E2(a, 1)] * us[3 * (int64_t)q + 1] +
                                           (double)D[E2(a, 2)] * us[3 * (int64_t)q + 2]);
                }
            }
        }
    }
    for (int a = 0; a < 3; a++) {
        const double v = warp_sum(acc[a]);
        if (lane == 0) V[3 * i + a] = v;
    }
}

/* Vtot = V + Vtot(parent), one level, top-down */
__global__ void k_vfield_down(int64_t first, int64_t count, const int32_t *__restrict__ parent,
                              const double *__restrict__ V, double *__restrict__ Vtot) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int64_t i = first + k;
    const int32_t p = parent[i];
    for (int d = 0; d < 3; d++) Vtot[3 * i + d] = V[3 * i + d] + (p >= 0 ? Vtot[3 * (int64_t)p + d] : 0.0);
}

/* out_i = (J u)_i for the sinks of each leaf; u and out in sorted order
 * (3 doubles per particle).  One block per leaf, one thread per sink. */
template <class T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_tidal_leaf(GParams P, const int32_t *__restrict__ leaves, int32_t nleaves,
                                                      const int32_t *__restrict__ pb, const int32_t *__restrict__ pe,
                                                      const MSrc *__restrict__ ms, const int4 *__restrict__ pos,
                                                      ListView LV, EwaldTables E, const double *__restrict__ Lnode,
                                                      const double *__restrict__ U, const double *__restrict__ Vtot,
                                                      const double *__restrict__ u, double *__restrict__ out) {
    __shared__ int4 sy[BLOCK];
    __shared__ T su[BLOCK][3];
    __shared__ double sL[LP];
    const int tid = threadIdx.x;
    const bool per = P.ewald != 0;
    for (int32_t li = blockIdx.x; li < nleaves; li += gridDim.x) {
        const int32_t leaf = leaves[li];
        const int32_t b = pb[leaf], cnt = pe[leaf] - b;
        const bool active = tid < cnt;
        const int32_t i = b + (active ? tid : 0);
        const int4 xi4 = pos[i];
        const int32_t xi[3] = {xi4.x, xi4.y, xi4.z};
        const T ui[3] = {T(u[3 * (int64_t)i]), T(u[3 * (int64_t)i + 1]), T(u[3 * (int64_t)i + 2])};
        __syncthreads();
        if (tid < LP) sL[tid] = Lnode[35 * (int64_t)leaf + tid];
        __syncthreads();
        Acc<T> o[3];
        for (int d = 0; d < 3; d++) o[d].init(0.0);
        {
            /* far field: tidal tensor of L (dX through float as in L2P) */
            double dx[3], T6[6];
            for (int d = 0; d < 3; d++)
                dx[d] = (double)__double2float_rn(__dadd_rn(pos2d(xi[d]), -pos2d(ms[leaf].x[d])));
            L2T(sL, dx, T6);
            const double ud[3] = {(double)ui[0], (double)ui[1], (double)ui[2]};
            for (int a = 0; a < 3; a++)
                o[a].add(T(T6[I2(a, 0)] * ud[0] + T6[I2(a, 1)] * ud[1] + T6[I2(a, 2)] * ud[2] +
                           Vtot[3 * (int64_t)leaf + a]));
        }
        /* PC direct and Ewald: sink-side tidal tensors */
        for (int ew = 0; ew < (per ? 2 : 1); ew++) {
            const int kind = ew ? TG_PC_E : TG_PC_D;
            const int32_t *lst = LV.pool[kind] + LV.off[kind][leaf];
            const int32_t len = LV.len[kind][leaf];
            for (int32_t j = 0; j < len; j++) {
                const MSrc &s = ms[lst[j]];
                T dX[3], D[LP], M[MP], T6[6];
#pragma unroll
                for (int d = 0; d < 3; d++) dX[d] = sep<T>(xi[d], s.x[d], ew ? true : per);
#pragma unroll
                for (int q = 0; q < MP; q++) M[q] = T(s.m[q]);
                if (ew) green_ewald_full<T>(E, dX, D);
                else green_direct<T>(dX, D);
                M2T<T>(M, D, T6);
                sym_mul_add<T>(T6, ui, o);
                /* source side: the source's centre moves by U/M (monopole order) */
                const T Ub[3] = {T(U[3 * (int64_t)lst[j]]), T(U[3 * (int64_t)lst[j] + 1]), T(U[3 * (int64_t)lst[j] + 2])};
                for (int a = 0; a < 3; a++) o[a].add(D[E2(a, 0)] * Ub[0] + D[E2(a, 1)] * Ub[1] + D[E2(a, 2)] * Ub[2]);
            }
        }
        /* PP direct and Ewald: pair Hessians times (u_i - u_j) */
        const T m = T(P.m_d);
        for (int ew = 0; ew < (per ? 2 : 1); ew++) {
            const int kind = ew ? TG_PP_E : TG_PP_D;
            const int32_t *lst = LV.pool[kind] + LV.off[kind][leaf];
            const int32_t len = LV.len[kind][leaf];
            for (int32_t c = 0; c < len; c++) {
                const int32_t src = lst[c];
                const int32_t sb = pb[src], sn = pe[src] - sb;
                for (int32_t base = 0; base < sn; base += BLOCK) {
                    const int32_t nt = min(BLOCK, sn - base);
                    __syncthreads();
                    if (tid < nt) {
                        const int64_t q = sb + base + tid;
                        sy[tid] = pos[q];
                        for (int d = 0; d < 3; d++) su[tid][d] = T(u[3 * q + d]);
                    }
                    __syncthreads();
                    for (int32_t q = 0; q < nt; q++) {
                        const int4 y = sy[q];
                        const T du[3] = {ui[0] - su[q][0], ui[1] - su[q][1], ui[2] - su[q][2]};
                        if (!ew) {
                            const T dX[3] = {sep<T>(xi[0], y.x, per), sep<T>(xi[1], y.y, per),
                                             sep<T>(xi[2], y.z, per)};
                            const T r2 = dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2];
                            T f, fpr;
                            pp_pair_deriv<T>(P, r2, f, fpr);
                            const T s = (dX[0] * du[0] + dX[1] * du[1] + dX[2] * du[2]) * fpr;
                            for (int d = 0; d < 3; d++) o[d].add(-m * (f * du[d] + dX[d] * s));
                        } else {
                            T dX[3] = {wrap_sep_t<T>(xi[0], y.x), wrap_sep_t<T>(xi[1], y.y), wrap_sep_t<T>(xi[2], y.z)};
                            if (!(dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2] > T(1.0e-12))) continue;
                            T D[LP];
                            green_ewald_full<T>(E, dX, D);
                            for (int a = 0; a < 3; a++)
                                o[a].add(-m * (D[E2(a, 0)] * du[0] + D[E2(a, 1)] * du[1] + D[E2(a, 2)] * du[2]));
                        }
                    }
                }
            }
        }
        if (active)
            for (int d = 0; d < 3; d++) out[3 * (int64_t)i + d] = o[d].get();
    }
}

/* u_sorted[i] = u[caller index of i] */
__global__ void k_gather3(int64_t n, const int4 *__restrict__ pos, const double *__restrict__ u,
                          double *__restrict__ us) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t w = pos[i].w;
    for (int d = 0; d < 3; d++) us[3 * i + d] = u[3 * w + d];
}

/* y[caller index of i] += c * x_sorted[i] */
__global__ void k_scatter_axpy3(int64_t n, const int4 *__restrict__ pos, double c, const double *__restrict__ xs,
                                double *__restrict__ y) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t w = pos[i].w;
    for (int d = 0; d < 3; d++) y[3 * w + d] += c * xs[3 * i + d];
}

/* y += c * x (n x 3, caller order) */
__global__ void k_axpy3(int64_t n, double c, const double *__restrict__ x, double *__restrict__ y) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * n) return;
    y[i] += c * x[i];
}

/* acc += c J u (u, acc: n x 3 doubles in caller order, device) for the
 * particles and lists currently in S; runs the node stage for the local
 * expansions first */
int tidal_apply(Solver &S, const double *u, double *acc, double c, cudaStream_t st) {
    if (!S.have_lists) return TG_ERR_STATE;
    TG_TRY(ewald_tables(S, st));
    const int64_t n = S.n;
    const GParams P = make_gparams(S.prm);
    const EwaldTables E = tables(S);
    const ListView LV = listview(S);
    TG_TRY(node_stage(S, P, LV, E, st));
    TG_TRY(ensure(S.tid_u, 3 * n));
    TG_TRY(ensure(S.tid_o, 3 * n));
    const int64_t nn = S.nnodes;
    TG_TRY(ensure(S.tid_U, 3 * nn));
    TG_TRY(ensure(S.tid_V, 6 * nn));
    const int gn = (int)((n + 255) / 256);
    k_gather3<<<gn, 256, 0, st>>>(n, S.pos.p, u, S.tid_u.p);
    TG_TRY(launched(S));
    const bool f64n = S.prm.precision == TG_PREC_F64;
    const int gw = (int)((nn * 32 + 127) / 128);
    k_node_usum<<<gw, 128, 0, st>>>(nn, S.prm.m, S.nd_pb.p, S.nd_pe.p, S.tid_u.p, S.tid_U.p);
    TG_TRY(launched(S));
    double *V = S.tid_V.p, *Vtot = S.tid_V.p + 3 * nn;
    if (f64n)
        k_vfield_node<double><<<gw, 128, 0, st>>>(P, nn, S.nd_pb.p, S.nd_pe.p, S.nd_ms.p, S.pos.p, LV, E, S.tid_U.p,
                                                  S.tid_u.p, V);
    else
        k_vfield_node<float><<<gw, 128, 0, st>>>(P, nn, S.nd_pb.p, S.nd_pe.p, S.nd_ms.p, S.pos.p, LV, E, S.tid_U.p,
                                                 S.tid_u.p, V);
    TG_TRY(launched(S));
    for (int L = 0; L <= S.depth; L++) {
        const int64_t first = S.level_off[L], count = S.level_off[L + 1] - S.level_off[L];
        if (count <= 0) continue;
        k_vfield_down<<<(int)((count + 127) / 128), 128, 0, st>>>(first, count, S.nd_parent.p, V, Vtot);
        TG_TRY(launched(S));
    }
    const int32_t nleaves = (int32_t)S.st.leaves;
    if (nleaves > 0) {
        const bool f64 = S.prm.precision == TG_PREC_F64;
        if (S.prm.leaf_max <= 64) {
            if (f64)
                k_tidal_leaf<double, 64><<<nleaves, 64, 0, st>>>(P, S.idx.p, nleaves, S.nd_pb.p, S.nd_pe.p, S.nd_ms.p,
                                                                 S.pos.p, LV, E, S.nd_L.p, S.tid_U.p, Vtot, S.tid_u.p, S.tid_o.p);
            else
                k_tidal_leaf<float, 64><<<nleaves, 64, 0, st>>>(P, S.idx.p, nleaves, S.nd_pb.p, S.nd_pe.p, S.nd_ms.p,
                                                                S.pos.p, LV, E, S.nd_L.p, S.tid_U.p, Vtot, S.tid_u.p, S.tid_o.p);
        } else {
            if (f64)
                k_tidal_leaf<double, 128><<<nleaves, 128, 0, st>>>(P, S.idx.p, nleaves, S.nd_pb.p, S.nd_pe.p,
                                                                   S.nd_ms.p, S.pos.p, LV, E, S.nd_L.p, S.tid_U.p,
                                                                   Vtot, S.tid_u.p, S.tid_o.p);
            else
                k_tidal_leaf<float, 128><<<nleaves, 128, 0, st>>>(P, S.idx.p, nleaves, S.nd_pb.p, S.nd_pe.p,
                                                                  S.nd_ms.p, S.pos.p, LV, E, S.nd_L.p, S.tid_U.p,
                                                                  Vtot, S.tid_u.p, S.tid_o.p);
        }
        TG_TRY(launched(S));
    }
    k_scatter_axpy3<<<gn, 256, 0, st>>>(n, S.pos.p, c, S.tid_o.p, acc);
    TG_TRY(launched(S));
    return TG_OK;
}

} // namespace tg
