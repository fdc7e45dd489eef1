/*
 * tg_gravity.cu -- the interaction kernels of kick_fmm (src/tree.cpp:400-631)
 * and the eight kernel-level seams of tigergrav/gravity.hpp:39-46.
 *
 *   k_node   one warp per node, lanes over sources: CC/CP direct; lane
 *            sums are reduced in FP64 -> Lloc (35 doubles)
 *   k_node_ewald (tg_ewald_node.cuh)  CC/CP Ewald in balanced chunks, one
 *            warp per chunk, one source's whole green_ewald per lane
 *            (walking only the lattice images inside the real-space cut);
 *            chunk sums added to Lloc in order
 *   k_l2l    one thread per node of a level, top-down:
 *            L = (L_parent << (x - x_parent)) + Lloc          (FP64)
 *   k_leaf   one block per leaf, one thread per sink particle: L2P, then
 *            PC_direct, PP_direct (source leaves staged in shared memory),
 *            PC_ewald, PP_ewald; -phi_self once (src/gravity.cpp:295).
 *            The FP32 path with leaf_max <= 64 runs it without PP_direct
 *            (into an FP64 buffer) and then k_pp_leaf (tg_pp2.cuh), which adds
 *            PP_direct and phi_self and writes the float4 result.
 *
 * Precision: T = float (FP32 path: FP32 arithmetic, per-tile FP32 partial
 * sums folded into Kahan-compensated accumulators) or T = double (the plain
 * FP64 port).  Expansions L are FP64 in both.
 */
#include "tg_solver.cuh"

namespace tg {

struct GParams {
    float m_f;
    double m_d;
    double h;
    float H, halfH, Hinv, H3inv, H2;
    double phi_self; /* -315/128 m / h */
    int ewald;
};

static GParams make_gparams(const tg_params &p) {
    GParams g;
    g.m_f = (float)p.m;
    g.m_d = p.m;
    g.h = p.soft_len;
    g.H = (float)p.soft_len;
    g.halfH = (float)(0.5 * p.soft_len);
    g.Hinv = (float)(1.0 / p.soft_len);
    g.H3inv = (float)(1.0 / p.soft_len / p.soft_len / p.soft_len);
    g.H2 = (float)(p.soft_len * p.soft_len);
    g.phi_self = (-315.0 / 128.0) * p.m / p.soft_len;
    g.ewald = p.ewald ? 1 : 0;
    return g;
}

/* ---- accumulators ---- */
template <class T> struct Acc;
template <> struct Acc<float> {
    KahanF k;
    __device__ __forceinline__ void init(double v) { k.s = (float)v; k.c = 0.0f; }
    __device__ __forceinline__ void add(float v) { k.add(v); }
    __device__ __forceinline__ double get() const { return (double)k.s - (double)k.c; }
};
template <> struct Acc<double> {
    double s;
    __device__ __forceinline__ void init(double v) { s = v; }
    __device__ __forceinline__ void add(double v) { s += v; }
    __device__ __forceinline__ double get() const { return s; }
};

/* ---- PP direct pair (src/gravity.cpp:214-287), GADGET spline softening.
 * Returns f (force factor, g -= dX * m * f) and p (phi -= m * p). */
template <class T>
__device__ __forceinline__ void pp_direct_pair(const GParams &P, const T *dX, T &f, T &p) {
    const T r2 = dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2];
    if (r2 > T(P.h * P.h)) {
        const T rinv = t_rsqrt(r2);
        p = rinv;
        f = rinv * rinv * rinv;
        return;
    }
    const T H = T(P.h), halfH = T(0.5 * P.h), Hinv = T(1.0 / P.h), H3inv = T(1.0 / P.h / P.h / P.h);
    const T r = t_sqrt(r2);
    const T rinv = T(1) / (r > halfH ? r : halfH);
    const T rinv3 = rinv * rinv * rinv;
    const T sw1 = r > H ? T(1) : T(0);
    const T sw3 = r < halfH ? T(1) : T(0);
    const T sw2 = T(1) - sw1 - sw3;
    T roh = r * Hinv;
    roh = roh < T(1) ? roh : T(1);
    const T roh2 = roh * roh;
    const T roh3 = roh2 * roh;
    T f2 = T(-32.0 / 3.0);
    f2 = fma(f2, roh, T(192.0 / 5.0));
    f2 = fma(f2, roh, T(-48.0));
    f2 = fma(f2, roh, T(64.0 / 3.0));
    f2 = fma(f2, roh3, T(-1.0 / 15.0));
    f2 *= rinv3;
    T f3 = T(32.0);
    f3 = fma(f3, roh, T(-192.0 / 5.0));
    f3 = fma(f3, roh2, T(32.0 / 3.0));
    f3 *= H3inv;
    f = sw1 * rinv3 + sw2 * f2 + sw3 * f3;
    T p2 = T(32.0 / 15.0);
    p2 = fma(p2, roh, T(-48.0 / 5.0));
    p2 = fma(p2, roh, T(16.0));
    p2 = fma(p2, roh, T(-32.0 / 3.0));
    p2 = fma(p2, roh2, T(16.0 / 5.0));
    p2 = fma(p2, roh, T(-1.0 / 15.0));
    p2 *= rinv;
    T p3 = T(-32.0 / 5.0);
    p3 = fma(p3, roh, T(48.0 / 5.0));
    p3 = fma(p3, roh2, T(-16.0 / 3.0));
    p3 = fma(p3, roh2, T(14.0 / 5.0));
    p3 *= Hinv;
    p = sw1 * rinv + sw2 * p2 + sw3 * p3;
}

/* Nearest image (n = 0) of the real-space sum together with the removal of
 * the direct 1/r that the Ewald kernels perform (src/gravity.cpp:594-600):
 *   -erfc(2r)/r + 1/r = erf(2r)/r
 *   force factor (1 - erfc(2r) - (4r/sqrt(pi)) e^{-4r^2}) / r^3
 * written without the cancellation of the two large 1/r terms.  With x = 2r,
 * F(x) = erf(x) - (2x/sqrt(pi)) e^{-x^2} = (2/sqrt(pi)) sum_{k>=1} (-1)^{k+1} 2k x^{2k+1} / (k! (2k+1))
 * (Taylor series of erf and of x e^{-x^2}), used below x = 0.5. */
template <class T>
__device__ __forceinline__ void ewald_nearest(T r, T rinv, T &p0, T &f0) {
    const T x = T(2) * r;
    const T erfx = erf(x);
    p0 = erfx * rinv;
    if (x < T(0.5)) {
        const T y = x * x;
        T s = T(-1.0 / 42840.0);
        s = fma(s, y, T(1.0 / 5400.0));
        s = fma(s, y, T(-1.0 / 780.0));
        s = fma(s, y, T(1.0 / 132.0));
        s = fma(s, y, T(-1.0 / 27.0));
        s = fma(s, y, T(1.0 / 7.0));
        s = fma(s, y, T(-0.4));
        s = fma(s, y, T(2.0 / 3.0));
        f0 = T(8.0 * 1.1283791670955126) * s; /* F / r^3 = 8 F / x^3 */
    } else {
        const T F = erfx - T(1.1283791670955126) * x * exp(-x * x);
        f0 = F * rinv * rinv * rinv;
    }
}

/* ---- PP Ewald pair (src/gravity.cpp:533-603): phi and g of the periodic
 * correction per unit mass.  The n = 0 image is taken by ewald_nearest. */
template <class T>
__device__ __forceinline__ void pp_ewald_pair(const EwaldTables &E, const T *dX0, T &phi, T *g) {
    const T r2 = dX0[0] * dX0[0] + dX0[1] * dX0[1] + dX0[2] * dX0[2];
    if (!(r2 > T(1.0e-12))) { /* r <= rcut: phi0, no force */
        phi = T(EWALD_PHI0);
        g[0] = g[1] = g[2] = T(0);
        return;
    }
    T ph = T(0), gx = T(0), gy = T(0), gz = T(0);
    ewald_images<T>(dX0, [&](const T *d, T rr2, bool origin) {
        if (origin) return;
        const T dx = d[0], dy = d[1], dz = d[2];
        const T rinv = t_rsqrt(rr2);
        const T r = rr2 * rinv;
        T expfac;
        const T erfc = t_erfcexp(T(2) * r, &expfac);
        const T d0 = -erfc * rinv;
        const T expfactor = T(2.2567583341910252) * r * expfac;
        const T d1 = (expfactor + erfc) * rinv * rinv * rinv;
        ph += d0;
        gx -= dx * d1;
        gy -= dy * d1;
        gz -= dz * d1;
    }, ewald_rcut2_pp<T>());
    for (int t = 0; t < NFOUR_HALF; t++) {
        const float4 h = __ldg(&E.four[t]);
        const T hdotdx = dX0[0] * T(h.x) + dX0[1] * T(h.y) + dX0[2] * T(h.z);
        T s, c;
        t_sincos2pi(hdotdx, &s, &c);
        T H0, Hx, Hy, Hz;
        if (sizeof(T) == 4) {
            const float4 q = __ldg(&E.Pf[t]);
            H0 = T(q.x), Hx = T(q.y), Hy = T(q.z), Hz = T(q.w);
        } else {
            const double2 q0 = __ldg(&E.Pd[2 * t]), q1 = __ldg(&E.Pd[2 * t + 1]);
            H0 = T(q0.x), Hx = T(q0.y), Hy = T(q1.x), Hz = T(q1.y);
        }
        ph += H0 * c;
        gx -= Hx * s;
        gy -= Hy * s;
        gz -= Hz * s;
    }
    const T rinv = t_rsqrt(r2);
    T p0, f0;
    ewald_nearest<T>(r2 * rinv, rinv, p0, f0);
    phi = ph + (T(0.78539816339744831) + p0);
    g[0] = gx + dX0[0] * f0;
    g[1] = gy + dX0[1] * f0;
    g[2] = gz + dX0[2] * f0;
}

/* full green_ewald(dX) evaluated by one thread (tigergrav/green.hpp:189-286) */
template <class T>
__device__ __forceinline__ void green_ewald_full(const EwaldTables &E, const T *X, T *D) {
#pragma unroll
    for (int k = 0; k < LP; k++) D[k] = T(0);
    const T r2 = X[0] * X[0] + X[1] * X[1] + X[2] * X[2];
    if (!(r2 > T(1.0e-12))) {
        D[0] = T(EWALD_PHI0);
        return;
    }
    EwaldMom<T> mom;
    mom.init();
    if constexpr (sizeof(T) == 4) {
        /* FP32: the n = 0 image carries the removal of the direct 1/r */
        ewald_images<T>(X, [&](const T *d, T rr2, bool origin) {
            if (origin) ewald_origin_add(D, mom, d, rr2);
            else ewald_real_image<T>(D, mom, d, rr2);
        });
    } else {
        ewald_images<T>(X, [&](const T *d, T rr2, bool) { ewald_real_image<T>(D, mom, d, rr2); });
    }
    ewald_mom_finish<T>(D, mom);
    for (int t = 0; t < NFOUR_HALF; t++) {
        const T *H = (sizeof(T) == 4) ? (const T *)(E.Hf + HS * t) : (const T *)(E.Hd + HS * t);
        ewald_four_term<T>(D, X, __ldg(&E.four[t]), H);
    }
    if constexpr (sizeof(T) == 4) D[E0()] += T(0.78539816339744831); /* pi/4 (tigergrav/green.hpp:270) */
    else ewald_finish<T, T>(D, X);
}

/* green_ewald(dX) split over a warp: this lane's share of the real-space
 * candidates (every n that can fall inside the cut) and of the reciprocal
 * terms, plus, on lane 0, the final assembly.  The sum of the 32 partial
 * results is green_ewald; the M2L / P2L contractions are linear, so each lane
 * contracts its own part.  X must not be 0 (the caller handles r <= 1e-6). */
template <class T>
__device__ __forceinline__ void green_ewald_warp(const EwaldTables &E, const T *X, T *D, int lane) {
#pragma unroll
    for (int k = 0; k < LP; k++) D[k] = T(0);
    const int ncand = sizeof(T) == 4 ? NREAL_F32 : NREAL;
    EwaldMom<T> mom;
    mom.init();
    for (int t = lane; t < ncand; t += 32) {
        const float4 n = __ldg(&E.real[t]);
        const T dx[3] = {X[0] - T(n.x), X[1] - T(n.y), X[2] - T(n.z)};
        const T r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        if (r2 < ewald_rcut2<T>() && n.w <= 17.0f) {
            if constexpr (sizeof(T) == 4) {
                if (n.w == 0.0f) ewald_origin_add(D, mom, dx, r2);
                else ewald_real_image<T>(D, mom, dx, r2);
            } else {
                ewald_real_image<T>(D, mom, dx, r2);
            }
        }
    }
    ewald_mom_finish<T>(D, mom);
    for (int t = lane; t < NFOUR_HALF; t += 32) {
        const T *H = (sizeof(T) == 4) ? (const T *)(E.Hf + HS * t) : (const T *)(E.Hd + HS * t);
        ewald_four_term<T>(D, X, __ldg(&E.four[t]), H);
    }
    if (lane == 0) {
        if constexpr (sizeof(T) == 4) D[E0()] += T(0.78539816339744831);
        else ewald_finish<T, T>(D, X);
    }
}

/* CC/CP Ewald lists shorter than this are evaluated one source at a time by
 * the whole warp (green_ewald_warp); longer ones one source per lane */
constexpr int EWALD_WARP_LIST = 12;

struct ListView {
    int32_t *pool[NLIST];
    int64_t *off[NLIST];
    int32_t *len[NLIST];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

/* ---- node kernel: CC / CP, direct and Ewald -> Lloc ---- */
template <class T>
__global__ void __launch_bounds__(128) k_node(GParams P, int64_t nn, const int32_t *__restrict__ pb,
                                              const int32_t *__restrict__ pe, const MSrc *__restrict__ ms,
                                              const int4 *__restrict__ pos, ListView LV, EwaldTables E,
                                              double *__restrict__ Lloc) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nn; i += warps) {
        if (pe[i] == pb[i]) continue;
        const int32_t X[3] = {ms[i].x[0], ms[i].x[1], ms[i].x[2]};
        const bool per = P.ewald != 0;
        T L[LP];
#pragma unroll
        for (int k = 0; k < LP; k++) L[k] = T(0);
        /* CC direct (src/gravity.cpp:368-426) */
        {
            const int32_t *lst = LV.pool[TG_CC_D] + LV.off[TG_CC_D][i];
            const int32_t len = LV.len[TG_CC_D][i];
            for (int32_t j = lane; j < len; j += 32) {
                const MSrc &s = ms[lst[j]];
                T dX[3], D[LP], M[MP];
#pragma unroll
                for (int d = 0; d < 3; d++) dX[d] = sep<T>(X[d], s.x[d], per);
#pragma unroll
                for (int q = 0; q < MP; q++) M[q] = T(s.m[q]);
                green_direct<T>(dX, D);
                contract_M2L<T, T>(L, M, D);
            }
        }
        /* CP direct (src/gravity.cpp:428-486) */
        {
            const int32_t *lst = LV.pool[TG_CP_D] + LV.off[TG_CP_D][i];
            const int32_t len = LV.len[TG_CP_D][i];
            const T m = T(P.m_d);
            for (int32_t c = 0; c < len; c++) {
                const int32_t src = lst[c];
                for (int32_t q = pb[src] + lane; q < pe[src]; q += 32) {
                    const int4 y = pos[q];
                    const int32_t yy[3] = {y.x, y.y, y.z};
                    T dX[3], D[LP];
#pragma unroll
                    for (int d = 0; d < 3; d++) dX[d] = sep<T>(X[d], yy[d], per);
                    green_direct<T>(dX, D);
                    contract_P2L<T, T>(L, m, D);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < LP; k++) {
            const double v = warp_sum((double)L[k]);
            if (lane == 0) Lloc[35 * i + k] = v;
        }
    }
}

#include "tg_ewald_node.cuh"

/* ---- L2L, one level ---- */
__global__ void k_l2l(int64_t first, int64_t count, const int32_t *__restrict__ pb, const int32_t *__restrict__ pe,
                      const int32_t *__restrict__ parent, const MSrc *__restrict__ ms, const double *__restrict__ Lloc,
                      double *__restrict__ Lout) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int64_t i = first + k;
    if (pe[i] == pb[i]) return;
    double L[LP];
    double Lcom[3] = {0.5, 0.5, 0.5};
    const int32_t p = parent[i];
    if (p >= 0) {
#pragma unroll
        for (int q = 0; q < LP; q++) L[q] = Lout[35 * (int64_t)p + q];
        for (int d = 0; d < 3; d++) Lcom[d] = pos2d(ms[p].x[d]);
    } else {
#pragma unroll
        for (int q = 0; q < LP; q++) L[q] = 0.0;
    }
    double dx[3];
    for (int d = 0; d < 3; d++) dx[d] = __dadd_rn(pos2d(ms[i].x[d]), -Lcom[d]);
    L2L(L, dx);
#pragma unroll
    for (int q = 0; q < LP; q++) Lout[35 * i + q] = L[q] + Lloc[35 * i + q];
}

/* ---- leaf kernel ---- */
template <class T, int BLOCK, bool PP = true, bool EW = true>
__global__ void __launch_bounds__(BLOCK) k_leaf(GParams P, const int32_t *__restrict__ leaves, int32_t nleaves,
                                                const int32_t *__restrict__ pb, const int32_t *__restrict__ pe,
                                                const MSrc *__restrict__ ms, const int4 *__restrict__ pos, ListView LV,
                                                EwaldTables E, const double *__restrict__ Lnode,
                                                float4 *__restrict__ acc_f, double *__restrict__ acc_d) {
    __shared__ int4 sy[BLOCK];
    __shared__ double sL[LP];
    const int tid = threadIdx.x;
    for (int32_t li = blockIdx.x; li < nleaves; li += gridDim.x) {
        const int32_t leaf = leaves[li];
        const int32_t b = pb[leaf], cnt = pe[leaf] - b;
        const bool active = tid < cnt;
        const int4 xi4 = pos[b + (active ? tid : 0)];
        const int32_t xi[3] = {xi4.x, xi4.y, xi4.z};
        const bool per = P.ewald != 0;
        __syncthreads();
        if (tid < LP) sL[tid] = Lnode[35 * (int64_t)leaf + tid];
        __syncthreads();
        /* L2P (tigergrav/expansion.hpp:235-269; dX through float, src/tree.cpp:607) */
        Acc<T> aphi, ag[3];
        {
            double dx[3], ph, g[3];
            for (int d = 0; d < 3; d++)
                dx[d] = (double)__double2float_rn(__dadd_rn(pos2d(xi[d]), -pos2d(ms[leaf].x[d])));
            L2P<double>(sL, dx, ph, g);
            aphi.init(ph);
            for (int d = 0; d < 3; d++) ag[d].init(g[d]);
        }
        /* PC direct (src/gravity.cpp:302-366) */
        {
            const int32_t *lst = LV.pool[TG_PC_D] + LV.off[TG_PC_D][leaf];
            const int32_t len = LV.len[TG_PC_D][leaf];
            for (int32_t j = 0; j < len; j++) {
                const MSrc &s = ms[lst[j]];
                T dX[3], D[LP], M[MP];
#pragma unroll
                for (int d = 0; d < 3; d++) dX[d] = sep<T>(xi[d], s.x[d], per);
#pragma unroll
                for (int q = 0; q < MP; q++) M[q] = T(s.m[q]);
                green_direct<T>(dX, D);
                T ph, g[3];
                contract_M2P<T>(ph, g, M, D);
                aphi.add(ph);
                for (int d = 0; d < 3; d++) ag[d].add(g[d]);
            }
        }
        /* PP direct (src/gravity.cpp:171-300) */
        if (PP) {
            const int32_t *lst = LV.pool[TG_PP_D] + LV.off[TG_PP_D][leaf];
            const int32_t len = LV.len[TG_PP_D][leaf];
            const T m = T(P.m_d);
            for (int32_t c = 0; c < len; c++) {
                const int32_t src = lst[c];
                const int32_t sb = pb[src], sn = pe[src] - sb;
                for (int32_t base = 0; base < sn; base += BLOCK) {
                    const int32_t nt = min(BLOCK, sn - base);
                    __syncthreads();
                    if (tid < nt) sy[tid] = pos[sb + base + tid];
                    __syncthreads();
                    /* plain sums over groups of 8 pairs, folded into the compensated totals */
                    for (int32_t q0 = 0; q0 < nt; q0 += 8) {
                        T tp = T(0), tg0 = T(0), tg1 = T(0), tg2 = T(0);
                        const int32_t q1 = min(nt, q0 + 8);
                        for (int32_t q = q0; q < q1; q++) {
                            const int4 y = sy[q];
                            T dX[3] = {sep<T>(xi[0], y.x, per), sep<T>(xi[1], y.y, per), sep<T>(xi[2], y.z, per)};
                            T f, p;
                            pp_direct_pair<T>(P, dX, f, p);
                            tp += p;
                            tg0 += dX[0] * f;
                            tg1 += dX[1] * f;
                            tg2 += dX[2] * f;
                        }
                        aphi.add(-m * tp);
                        ag[0].add(-m * tg0);
                        ag[1].add(-m * tg1);
                        ag[2].add(-m * tg2);
                    }
                }
            }
        }
        if (EW && per) {
            /* PC Ewald (src/gravity.cpp:616-678) */
            const int32_t *lst = LV.pool[TG_PC_E] + LV.off[TG_PC_E][leaf];
            const int32_t len = LV.len[TG_PC_E][leaf];
            for (int32_t j = 0; j < len; j++) {
                const MSrc &s = ms[lst[j]];
                T dX[3], D[LP], M[MP];
#pragma unroll
                for (int d = 0; d < 3; d++) dX[d] = sep<T>(xi[d], s.x[d], true);
#pragma unroll
                for (int q = 0; q < MP; q++) M[q] = T(s.m[q]);
                green_ewald_full<T>(E, dX, D);
                T ph, g[3];
                contract_M2P<T>(ph, g, M, D);
                aphi.add(ph);
                for (int d = 0; d < 3; d++) ag[d].add(g[d]);
            }
            /* PP Ewald (src/gravity.cpp:491-614) */
            const int32_t *lpp = LV.pool[TG_PP_E] + LV.off[TG_PP_E][leaf];
            const int32_t npp = LV.len[TG_PP_E][leaf];
            const T m = T(P.m_d);
            for (int32_t c = 0; c < npp; c++) {
                const int32_t src = lpp[c];
                const int32_t sb = pb[src], sn = pe[src] - sb;
                for (int32_t base = 0; base < sn; base += BLOCK) {
                    const int32_t nt = min(BLOCK, sn - base);
                    __syncthreads();
                    if (tid < nt) sy[tid] = pos[sb + base + tid];
                    __syncthreads();
                    for (int32_t q = 0; q < nt; q++) {
                        const int4 y = sy[q];
                        T dX[3] = {wrap_sep_t<T>(xi[0], y.x), wrap_sep_t<T>(xi[1], y.y), wrap_sep_t<T>(xi[2], y.z)};
                        T ph, g[3];
                        pp_ewald_pair<T>(E, dX, ph, g);
                        aphi.add(m * ph);
                        for (int d = 0; d < 3; d++) ag[d].add(m * g[d]);
                    }
                }
            }
        }
        if (active) {
            const double phi = aphi.get() - (PP ? P.phi_self : 0.0);
            if (acc_f) acc_f[b + tid] = make_float4((float)phi, (float)ag[0].get(), (float)ag[1].get(), (float)ag[2].get());
            if (acc_d) {
                acc_d[4 * (int64_t)(b + tid) + 0] = phi;
                for (int d = 0; d < 3; d++) acc_d[4 * (int64_t)(b + tid) + 1 + d] = ag[d].get();
            }
        }
    }
}

/* ---- PP direct for the FP32 path (leaf_max <= 64) ----
 * Source positions are staged in split fixed point relative to the sink
 * leaf's centre Xr: for a = wrap(Y - Xr),
 *     hi = (a >> 16) 2^-16,   lo = (a & 0xffff) 2^-32
 * are exact in FP32, and dX = (hi_i - hi_j) + (lo_i - lo_j) is the correctly
 * rounded FP32 value of (X_i - Y_j) 2^-32 -- exactly the reference's dX
 * (src/gravity.cpp:223) -- from three FP32 additions and no integer-to-float
 * conversion per pair.  The identity needs |a_i - a_j| < 2^31, checked per
 * staged batch; otherwise that batch's pairs take the per-pair wrap. */
__device__ __forceinline__ void split_hl(int32_t a, float &h, float &l) {
    h = __int2float_rn(a >> 16) * 1.52587890625e-05f;
    l = __int2float_rn(a & 0xffff) * 2.3283064365386963e-10f;
}

__device__ __forceinline__ uint32_t warp_max_u(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

/* offset of Y from Xr: int32 wrap (periodic) or plain difference (free space);
 * mag accumulates the largest magnitude, saturated at 2^31 (a free-space
 * offset that does not fit an int32 reads as 2^31) */
__device__ __forceinline__ int32_t rel_off(int32_t Y, int32_t Xr, bool per, uint32_t &mag) {
    if (per) {
        const int32_t a = (int32_t)((uint32_t)Y - (uint32_t)Xr);
        mag = max(mag, a < 0 ? 0u - (uint32_t)a : (uint32_t)a);
        return a;
    }
    const long long a = (long long)Y - (long long)Xr;
    const unsigned long long aa = (unsigned long long)(a < 0 ? -a : a);
    mag = max(mag, aa >= (1ull << 31) ? (1u << 31) : (uint32_t)aa);
    return (int32_t)a;
}

#include "tg_pp.cuh"
#include "tg_pp2.cuh"
#include "tg_ewald_sep.cuh"
#include "tg_ewald_leaf.cuh"

/* ---------------- kernel-level seams ---------------- */

template <class T>
__global__ void k_seam_pp(GParams P, int kind_ewald, int do_phi, int64_t ngroups, const int64_t *__restrict__ sink_off,
                          const int32_t *__restrict__ sink_x, const int64_t *__restrict__ src_off,
                          const int32_t *__restrict__ src_x, EwaldTables E, double *__restrict__ f) {
    const bool per = P.ewald != 0;
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        for (int64_t i = sink_off[g] + threadIdx.x; i < sink_off[g + 1]; i += blockDim.x) {
            const int32_t xi[3] = {sink_x[3 * i], sink_x[3 * i + 1], sink_x[3 * i + 2]};
            double ph = 0, gg[3] = {0, 0, 0};
            for (int64_t j = src_off[g]; j < src_off[g + 1]; j++) {
                const int32_t *y = src_x + 3 * j;
                if (kind_ewald) {
                    T dX[3] = {wrap_sep_t<T>(xi[0], y[0]), wrap_sep_t<T>(xi[1], y[1]), wrap_sep_t<T>(xi[2], y[2])};
                    T p, g3[3];
                    pp_ewald_pair<T>(E, dX, p, g3);
                    ph += P.m_d * (double)p;
                    for (int d = 0; d < 3; d++) gg[d] += P.m_d * (double)g3[d];
                } else {
                    T dX[3] = {sep<T>(xi[0], y[0], per), sep<T>(xi[1], y[1], per), sep<T>(xi[2], y[2], per)};
                    T fk, p;
                    pp_direct_pair<T>(P, dX, fk, p);
                    if (do_phi) ph -= P.m_d * (double)p;
                    for (int d = 0; d < 3; d++) gg[d] -= P.m_d * (double)(dX[d] * fk);
                }
            }
            if (!kind_ewald) ph -= P.phi_self;
            f[4 * i] += ph;
            for (int d = 0; d < 3; d++) f[4 * i + 1 + d] += gg[d];
        }
    }
}

template <class T>
__global__ void k_seam_pc(GParams P, int kind_ewald, int64_t ngroups, const int64_t *__restrict__ sink_off,
                          const int32_t *__restrict__ sink_x, const int64_t *__restrict__ src_off,
                          const float *__restrict__ src_m, const int32_t *__restrict__ src_x, EwaldTables E,
                          double *__restrict__ f) {
    const bool per = kind_ewald || P.ewald != 0;
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        for (int64_t i = sink_off[g] + threadIdx.x; i < sink_off[g + 1]; i += blockDim.x) {
            const int32_t xi[3] = {sink_x[3 * i], sink_x[3 * i + 1], sink_x[3 * i + 2]};
            double ph = 0, gg[3] = {0, 0, 0};
            for (int64_t j = src_off[g]; j < src_off[g + 1]; j++) {
                T dX[3], D[LP], M[MP];
                for (int d = 0; d < 3; d++) dX[d] = sep<T>(xi[d], src_x[3 * j + d], per);
                for (int q = 0; q < MP; q++) M[q] = T(src_m[MP * j + q]);
                if (kind_ewald) green_ewald_full<T>(E, dX, D);
                else green_direct<T>(dX, D);
                T p, g3[3];
                contract_M2P<T>(p, g3, M, D);
                ph += (double)p;
                for (int d = 0; d < 3; d++) gg[d] += (double)g3[d];
            }
            f[4 * i] += ph;
            for (int d = 0; d < 3; d++) f[4 * i + 1 + d] += gg[d];
        }
    }
}

/* CC/CP seams: one warp per group, lanes over sources */
template <class T>
__global__ void k_seam_node(GParams P, int kind_ewald, int is_cc, int64_t ngroups, const int32_t *__restrict__ sink_x,
                            const int64_t *__restrict__ src_off, const float *__restrict__ src_m,
                            const int32_t *__restrict__ src_x, EwaldTables E, double *__restrict__ Lout) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const bool per = kind_ewald || P.ewald != 0;
    for (int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ngroups; g += warps) {
        const int32_t X[3] = {sink_x[3 * g], sink_x[3 * g + 1], sink_x[3 * g + 2]};
        T L[LP];
        for (int k = 0; k < LP; k++) L[k] = T(0);
        const int64_t b = src_off[g], e = src_off[g + 1];
        for (int64_t j = b + lane; j < e; j += 32) {
            T dX[3], D[LP];
            for (int d = 0; d < 3; d++) dX[d] = sep<T>(X[d], src_x[3 * j + d], per);
            if (kind_ewald) green_ewald_full<T>(E, dX, D);
            else green_direct<T>(dX, D);
            if (is_cc) {
                T M[MP];
                for (int q = 0; q < MP; q++) M[q] = T(src_m[MP * j + q]);
                contract_M2L<T, T>(L, M, D);
            } else {
                contract_P2L<T, T>(L, T(P.m_d), D);
            }
        }
        for (int k = 0; k < LP; k++) {
            const double v = warp_sum((double)L[k]);
            if (lane == 0) Lout[35 * g + k] += v;
        }
    }
}

static EwaldTables tables(Solver &S) {
    return EwaldTables{S.ew_real.p, S.ew_four.p, S.ew_Hf.p, S.ew_Hd.p, S.ew_Pf.p, S.ew_Pd.p};
}

static ListView listview(Solver &S) {
    ListView LV;
    for (int k = 0; k < NLIST; k++) {
        LV.pool[k] = S.pool[k].p;
        LV.off[k] = S.loff[k].p;
        LV.len[k] = S.llen[k].p;
    }
    return LV;
}

/* the node Ewald lists (CC_E, CP_E) of every node, in balanced chunks, added
 * to Lloc */
static int node_ewald(Solver &S, const GParams &P, const ListView &LV, const EwaldTables &E, bool f64,
                      cudaStream_t st) {
    const int64_t nn = S.nnodes;
    TG_TRY(ensure(S.ew_cnt, (size_t)nn + 1));
    TG_TRY(ensure(S.ew_off, (size_t)nn + 1));
    k_node_ewald_count<<<(int)((nn + 1 + 127) / 128), 128, 0, st>>>(nn, S.nd_pb.p, S.nd_pe.p, LV, S.ew_cnt.p);
    TG_TRY(launched(S));
    size_t stmp = 0;
    TG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, stmp, S.ew_cnt.p, S.ew_off.p, (int)(nn + 1), st));
    TG_TRY(ensure(S.cub_tmp, stmp));
    TG_CUDA(cub::DeviceScan::ExclusiveSum(S.cub_tmp.p, stmp, S.ew_cnt.p, S.ew_off.p, (int)(nn + 1), st));
    int32_t total = 0;
    TG_TRY(read_small(S, st, &total, S.ew_off.p + nn, sizeof(int32_t)));
    if (total <= 0) return TG_OK;
    TG_TRY(ensure(S.ew_part, (size_t)total * LP));
    const int g = (int)(((int64_t)total * 32 + 127) / 128);
    if (f64)
        k_node_ewald<double><<<g, 128, 0, st>>>(P, nn, total, S.ew_off.p, S.nd_pb.p, S.nd_pe.p, S.nd_ms.p, S.pos.p, LV,
                                                E, S.ew_part.p);
    else
        k_node_ewald<float><<<g, 128, 0, st>>>(P, nn, total, S.ew_off.p, S.nd_pb.p, S.nd_pe.p, S.nd_ms.p, S.pos.p, LV,
                                               E, S.ew_part.p);
    TG_TRY(launched(S));
    k_node_ewald_reduce<<<(int)((nn * LP + 255) / 256), 256, 0, st>>>(nn, S.ew_off.p, S.ew_part.p, S.nd_Lloc.p);
    TG_TRY(launched(S));
    return TG_OK;
}

/* the leaf Ewald lists (PP_E, PC_E) of every leaf, in balanced chunks, added
 * to the FP64 accumulators accd (leaf_max <= 64) */
static int leaf_ewald(Solver &S, const GParams &P, const ListView &LV, const EwaldTables &E, bool f64,
                      cudaStream_t st) {
    const int32_t nleaves = (int32_t)S.st.leaves;
    TG_TRY(ensure(S.ew_cnt, (size_t)nleaves + 1));
    TG_TRY(ensure(S.ew_off, (size_t)nleaves + 1));
    k_ewald_count<<<(nleaves + 1 + 127) / 128, 128, 0, st>>>(S.idx.p, nleaves, LV, S.ew_cnt.p);
    TG_TRY(launched(S));
    size_t stmp = 0;
    TG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, stmp, S.ew_cnt.p, S.ew_off.p, nleaves + 1, st));
    TG_TRY(ensure(S.cub_tmp, stmp));
    TG_CUDA(cub::DeviceScan::ExclusiveSum(S.cub_tmp.p, stmp, S.ew_cnt.p, S.ew_off.p, nleaves + 1, st));
    int32_t total = 0;
    TG_TRY(read_small(S, st, &total, S.ew_off.p + nleaves, sizeof(int32_t)));
    if (total <= 0) return TG_OK;
    TG_TRY(ensure(S.ew_part, (size_t)total * 64 * 4));
    float *tpart = nullptr;
    if (f64) {
        k_ewald_chunk<double, false><<<total, 64, 0, st>>>(P, S.idx.p, nleaves, S.ew_off.p, S.nd_pb.p, S.nd_pe.p,
                                                           S.nd_ms.p, S.pos.p, S.nd_aabb.p, LV, E, S.ew_part.p, nullptr,
                                                           nullptr, nullptr);
    } else {
        /* reciprocal terms per sink leaf: (cos, sin) tables per node, sums per leaf */
        const int64_t nn = S.nnodes;
        TG_TRY(ensure(S.ew_nt, (size_t)nn * NFOUR_HALF));
        TG_TRY(ensure(S.ew_sf, (size_t)nn * NFOUR_HALF));
        TG_TRY(ensure(S.ew_tpart, (size_t)total * NFOUR_HALF * EW_SEP_K));
        tpart = S.ew_tpart.p;
        k_ewald_sf<<<(int)((nn * 32 + 127) / 128), 128, 0, st>>>(nn, S.nd_pb.p, S.nd_pe.p, S.nd_child0.p, S.nd_ms.p,
                                                                S.pos.p, E, S.ew_nt.p, S.ew_sf.p);
        TG_TRY(launched(S));
        k_ewald_chunk<float, true><<<total, 64, 0, st>>>(P, S.idx.p, nleaves, S.ew_off.p, S.nd_pb.p, S.nd_pe.p,
                                                         S.nd_ms.p, S.pos.p, S.nd_aabb.p, LV, E, S.ew_part.p, S.ew_nt.p,
                                                         S.ew_sf.p, tpart);
    }
    TG_TRY(launched(S));
    k_ewald_reduce<<<nleaves, 64, 0, st>>>(S.idx.p, nleaves, S.ew_off.p, S.nd_pb.p, S.nd_pe.p, S.ew_part.p, S.accd.p,
                                           tpart, S.pos.p, E);
    TG_TRY(launched(S));
    return TG_OK;
}

/* the node stage: CC/CP (direct, then Ewald) into Lloc, then L2L top-down into nd_L */
static int node_stage(Solver &S, const GParams &P, const ListView &LV, const EwaldTables &E, cudaStream_t st) {
    const int64_t nn = S.nnodes;
    const bool f64 = S.prm.precision == TG_PREC_F64;
    TG_TRY(ensure(S.nd_Lloc, 35 * nn));
    TG_TRY(ensure(S.nd_L, 35 * nn));
    {
        const int TPB = 128;
        const int64_t want = (nn * 32 + TPB - 1) / TPB;
        const int g = (int)(want < 65535 * 8 ? want : 65535 * 8);
        if (f64)
            k_node<double><<<g, TPB, 0, st>>>(P, nn, S.nd_pb.p, S.nd_pe.p, S.nd_ms.p, S.pos.p, LV, E, S.nd_Lloc.p);
        else
            k_node<float><<<g, TPB, 0, st>>>(P, nn, S.nd_pb.p, S.nd_pe.p, S.nd_ms.p, S.pos.p, LV, E, S.nd_Lloc.p);
        TG_TRY(launched(S));
    }
    if (S.prm.ewald) TG_TRY(node_ewald(S, P, LV, E, f64, st));
    for (int L = 0; L <= S.depth; L++) {
        const int64_t first = S.level_off[L], count = S.level_off[L + 1] - S.level_off[L];
        if (count <= 0) continue;
        const int g = (int)((count + 127) / 128);
        k_l2l<<<g, 128, 0, st>>>(first, count, S.nd_pb.p, S.nd_pe.p, S.nd_parent.p, S.nd_ms.p, S.nd_Lloc.p, S.nd_L.p);
        TG_TRY(launched(S));
    }
    return TG_OK;
}

int gravity_forces(Solver &S, cudaStream_t st) {
    if (!S.have_lists) return TG_ERR_STATE;
    TG_TRY(ewald_tables(S, st));
    const int64_t nn = S.nnodes, n = S.n;
    const GParams P = make_gparams(S.prm);
    const EwaldTables E = tables(S);
    const ListView LV = listview(S);
    const bool f64 = S.prm.precision == TG_PREC_F64;
    (void)nn;
    const bool split_pp = !f64 && S.prm.leaf_max <= 64;
    if (f64 || split_pp) TG_TRY(ensure(S.accd, 4 * n));
    if (!f64) TG_TRY(ensure(S.acc, n));
    S.pp_timed = false;
    if (S.have_events) TG_CUDA(cudaEventRecord(S.ev[3], st));
    TG_TRY(node_stage(S, P, LV, E, st));
    if (S.have_events) TG_CUDA(cudaEventRecord(S.ev[4], st));
    const int32_t nleaves = (int32_t)S.st.leaves;
    if (nleaves > 0) {
        const int g = nleaves;
        if (S.prm.leaf_max <= 64) {
            /* L2P, PC direct (and for FP64 PP direct) per leaf; the Ewald lists as balanced chunks */
            if (f64)
                k_leaf<double, 64, true, false><<<g, 64, 0, st>>>(P, S.idx.p, nleaves, S.nd_pb.p, S.nd_pe.p, S.nd_ms.p,
                                                                  S.pos.p, LV, E, S.nd_L.p, nullptr, S.accd.p);
            else
                k_leaf<float, 64, false, false><<<g, 64, 0, st>>>(P, S.idx.p, nleaves, S.nd_pb.p, S.nd_pe.p,
                                                                  S.nd_ms.p, S.pos.p, LV, E, S.nd_L.p, nullptr,
                                                                  S.accd.p);
            TG_TRY(launched(S));
            if (S.prm.ewald) TG_TRY(leaf_ewald(S, P, LV, E, f64, st));
            if (!f64) {
                if (S.have_events) {
                    TG_CUDA(cudaEventRecord(S.ev[6], st));
                    S.pp_timed = true;
                }
                k_pp_leaf<<<g, PPB_T, 0, st>>>(P, S.idx.p, nleaves, S.nd_pb.p, S.nd_pe.p, S.nd_ms.p, S.nd_aabb.p,
                                               S.pos.p, LV, S.accd.p, S.acc.p);
            }
        } else {
            if (f64)
                k_leaf<double, 128><<<g, 128, 0, st>>>(P, S.idx.p, nleaves, S.nd_pb.p, S.nd_pe.p, S.nd_ms.p, S.pos.p, LV,
                                                       E, S.nd_L.p, nullptr, S.accd.p);
            else
                k_leaf<float, 128><<<g, 128, 0, st>>>(P, S.idx.p, nleaves, S.nd_pb.p, S.nd_pe.p, S.nd_ms.p, S.pos.p, LV,
                                                      E, S.nd_L.p, S.acc.p, nullptr);
        }
        TG_TRY(launched(S));
    }
    if (S.have_events) TG_CUDA(cudaEventRecord(S.ev[5], st));
    S.have_forces = true;
    return TG_OK;
}

/* seam drivers */
int seam_pp(Solver *Sopt, const tg_params &prm, int ewald_kind, int do_phi, int64_t ngroups, const int64_t *sink_off,
            const int32_t *sink_x, const int64_t *src_off, const int32_t *src_x, double *f, const EwaldTables &E,
            cudaStream_t st) {
    const GParams P = make_gparams(prm);
    const int g = (int)(ngroups < 65535 ? ngroups : 65535);
    if (g <= 0) return TG_OK;
    if (prm.precision == TG_PREC_F64)
        k_seam_pp<double><<<g, 128, 0, st>>>(P, ewald_kind, do_phi, ngroups, sink_off, sink_x, src_off, src_x, E, f);
    else
        k_seam_pp<float><<<g, 128, 0, st>>>(P, ewald_kind, do_phi, ngroups, sink_off, sink_x, src_off, src_x, E, f);
    TG_CUDA(cudaGetLastError());
    (void)Sopt;
    return TG_OK;
}

int seam_pc(const tg_params &prm, int ewald_kind, int64_t ngroups, const int64_t *sink_off, const int32_t *sink_x,
            const int64_t *src_off, const float *src_m, const int32_t *src_x, double *f, const EwaldTables &E,
            cudaStream_t st) {
    const GParams P = make_gparams(prm);
    const int g = (int)(ngroups < 65535 ? ngroups : 65535);
    if (g <= 0) return TG_OK;
    if (prm.precision == TG_PREC_F64)
        k_seam_pc<double><<<g, 128, 0, st>>>(P, ewald_kind, ngroups, sink_off, sink_x, src_off, src_m, src_x, E, f);
    else
        k_seam_pc<float><<<g, 128, 0, st>>>(P, ewald_kind, ngroups, sink_off, sink_x, src_off, src_m, src_x, E, f);
    TG_CUDA(cudaGetLastError());
    return TG_OK;
}

int seam_node(const tg_params &prm, int ewald_kind, int is_cc, int64_t ngroups, const int32_t *sink_x,
              const int64_t *src_off, const float *src_m, const int32_t *src_x, double *L, const EwaldTables &E,
              cudaStream_t st) {
    const GParams P = make_gparams(prm);
    const int64_t want = (ngroups * 32 + 127) / 128;
    const int g = (int)(want < 65535 ? want : 65535);
    if (g <= 0) return TG_OK;
    if (prm.precision == TG_PREC_F64)
        k_seam_node<double><<<g, 128, 0, st>>>(P, ewald_kind, is_cc, ngroups, sink_x, src_off, src_m, src_x, E, L);
    else
        k_seam_node<float><<<g, 128, 0, st>>>(P, ewald_kind, is_cc, ngroups, sink_x, src_off, src_m, src_x, E, L);
    TG_CUDA(cudaGetLastError());
    return TG_OK;
}

EwaldTables solver_tables(Solver &S) { return tables(S); }

} // namespace tg
