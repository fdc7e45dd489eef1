/*
 * tg_ewald_node.cuh -- the node-sink Ewald kernels (gravity_CC_ewald,
 * src/gravity.cpp:680-731; gravity_CP_ewald, :733-785) as balanced work
 * units.  Included by tg_gravity.cu after k_node.
 *
 * Each node's CC_E list is cut into chunks of EN_KCC source nodes and its
 * CP_E list into chunks of EN_KCP source leaves.  One warp evaluates one
 * chunk: lanes over the chunk's sources (a source's whole green_ewald per
 * lane); a chunk of fewer than EWALD_WARP_LIST sources is evaluated one
 * source at a time by the whole warp (green_ewald_warp).  The warp's FP64
 * sum of the 35 expansion terms goes to the chunk's slot of a scratch array,
 * and k_node_ewald_reduce adds a node's chunk sums, in chunk order, to its
 * Lloc.  Keeping the Ewald evaluation out of k_node leaves both kernels
 * fewer live registers, and long lists no longer make one warp the tail.
 */
#pragma once

constexpr int EN_KCC = 128; /* CC_E source nodes per chunk (4 per lane) */
constexpr int EN_KCP = 4;   /* CP_E source leaves per chunk */
#ifndef EN_MINB
#define EN_MINB 6 /* resident 128-thread blocks per SM the kernel is compiled for */
#endif

__global__ void k_node_ewald_count(int64_t nn, const int32_t *__restrict__ pb, const int32_t *__restrict__ pe,
                                   ListView LV, int32_t *__restrict__ cnt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > nn) return;
    if (i == nn || pe[i] == pb[i]) {
        cnt[i] = 0;
        return;
    }
    const int32_t ncc = LV.len[TG_CC_E][i], ncp = LV.len[TG_CP_E][i];
    cnt[i] = (ncc + EN_KCC - 1) / EN_KCC + (ncp + EN_KCP - 1) / EN_KCP;
}

constexpr int EN_SEP_K = 6; /* per h: (cos, sin) sums of m_0, m_2, m_3 over a chunk's sources */

/* FP32 (SEP): the reciprocal-space terms are left out of the per-source
 * green_ewald and summed per sink node instead (tg_ewald_sep.cuh): each chunk
 * writes its sources' sums per h to tpart, k_node_ewald_recip turns a node's
 * sums into expansion terms. */
template <class T, bool SEP>
__global__ void __launch_bounds__(128, EN_MINB) k_node_ewald(GParams P, int64_t nn, int32_t nchunks,
                                                    const int32_t *__restrict__ off, const int32_t *__restrict__ pb,
                                                    const int32_t *__restrict__ pe, const MSrc *__restrict__ ms,
                                                    const int4 *__restrict__ pos, ListView LV, EwaldTables E,
                                                    double *__restrict__ part, const float2 *__restrict__ nt,
                                                    const float2 *__restrict__ sf, float *__restrict__ tpart) {
    const int lane = threadIdx.x & 31;
    const int32_t c = (int32_t)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (c >= nchunks) return;
    int64_t lo = 0, hi = nn - 1; /* the node: largest i with off[i] <= c */
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (off[mid] <= c) lo = mid;
        else hi = mid - 1;
    }
    const int64_t i = lo;
    const int32_t k = c - off[i];
    const int32_t X[3] = {ms[i].x[0], ms[i].x[1], ms[i].x[2]};
    /* each lane's expansion sums live in shared memory (odd stride LP: no bank
     * conflicts), which leaves the registers to the green_ewald evaluation */
    __shared__ T sL[128 * LP];
    T *L = sL + threadIdx.x * LP;
#pragma unroll
    for (int q = 0; q < LP; q++) L[q] = T(0);
    const int32_t ncc = LV.len[TG_CC_E][i];
    const int32_t kcc = (ncc + EN_KCC - 1) / EN_KCC;
    if (k < kcc) {
        const int32_t *lst = LV.pool[TG_CC_E] + LV.off[TG_CC_E][i];
        const int32_t e0 = k * EN_KCC, e1 = min(ncc, e0 + EN_KCC);
        if (e1 - e0 >= EWALD_WARP_LIST) {
            for (int32_t j = e0 + lane; j < e1; j += 32) {
                const MSrc &s = ms[lst[j]];
                T dX[3], D[LP], M[MP];
#pragma unroll
                for (int d = 0; d < 3; d++) dX[d] = sep<T>(X[d], s.x[d], true);
#pragma unroll
                for (int q = 0; q < MP; q++) M[q] = T(s.m[q]);
                if constexpr (SEP) green_ewald_sep<false>(E, dX, D); /* r ~ 0 sources stay out of the sums */
                else green_ewald_full<T>(E, dX, D);
                contract_M2L<T, T>(L, M, D);
            }
        } else {
            for (int32_t j = e0; j < e1; j++) {
                const MSrc &s = ms[lst[j]];
                T dX[3], D[LP], M[MP];
#pragma unroll
                for (int d = 0; d < 3; d++) dX[d] = sep<T>(X[d], s.x[d], true);
                if (!(dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2] > T(1.0e-12))) {
                    /* the node itself: green_ewald(0) = phi0 only (tigergrav/green.hpp:279) */
                    if (lane == 0) L[E0()] += T(s.m[0]) * T(EWALD_PHI0);
                    continue;
                }
#pragma unroll
                for (int q = 0; q < MP; q++) M[q] = T(s.m[q]);
                green_ewald_warp<T, !SEP>(E, dX, D, lane);
                contract_M2L<T, T>(L, M, D);
            }
        }
    } else {
        const int32_t ncp = LV.len[TG_CP_E][i];
        const int32_t *lst = LV.pool[TG_CP_E] + LV.off[TG_CP_E][i];
        const int32_t e0 = (k - kcc) * EN_KCP, e1 = min(ncp, e0 + EN_KCP);
        const T m = T(P.m_d);
        for (int32_t e = e0; e < e1; e++) {
            const int32_t src = lst[e];
            for (int32_t q = pb[src] + lane; q < pe[src]; q += 32) {
                const int4 y = pos[q];
                const int32_t yy[3] = {y.x, y.y, y.z};
                T dX[3], D[LP];
#pragma unroll
                for (int d = 0; d < 3; d++) dX[d] = sep<T>(X[d], yy[d], true);
                if constexpr (SEP) green_ewald_sep(E, dX, D);
                else green_ewald_full<T>(E, dX, D);
                contract_P2L<T, T>(L, m, D);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < LP; q++) {
        const double v = warp_sum((double)L[q]);
        if (lane == 0) part[(int64_t)c * LP + q] = v;
    }
    if constexpr (SEP) {
        /* this chunk's sources' reciprocal-space sums: lane takes h_t, t = lane, lane + 32 */
        for (int t = lane; t < NFOUR_HALF; t += 32) {
            float a[EN_SEP_K];
#pragma unroll
            for (int q = 0; q < EN_SEP_K; q++) a[q] = 0.0f;
            if (k < kcc) {
                const int32_t *lst = LV.pool[TG_CC_E] + LV.off[TG_CC_E][i];
                const int32_t e0 = k * EN_KCC, e1 = min(ncc, e0 + EN_KCC);
                SepQ Q;
                sep_q(__ldg(&E.four[t]), Q);
                for (int32_t e = e0; e < e1; e++) {
                    const int32_t src = lst[e];
                    float dX[3];
#pragma unroll
                    for (int d = 0; d < 3; d++) dX[d] = sep<float>(X[d], ms[src].x[d], true);
                    if (!(dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2] > 1.0e-12f)) continue; /* phi0 only */
                    const float2 f = nt[(int64_t)src * NFOUR_HALF + t];
                    const float *M = ms[src].m;
                    float m2 = 0.0f, m3 = 0.0f;
#pragma unroll
                    for (int q = 0; q < 6; q++) m2 += Q.q2[q] * M[1 + q];
#pragma unroll
                    for (int q = 0; q < 10; q++) m3 += Q.q3[q] * M[7 + q];
                    a[0] += M[0] * f.x;
                    a[1] += M[0] * f.y;
                    a[2] += m2 * f.x;
                    a[3] += m2 * f.y;
                    a[4] += m3 * f.x;
                    a[5] += m3 * f.y;
                }
            } else {
                const int32_t ncp = LV.len[TG_CP_E][i];
                const int32_t *lst = LV.pool[TG_CP_E] + LV.off[TG_CP_E][i];
                const int32_t e0 = (k - kcc) * EN_KCP, e1 = min(ncp, e0 + EN_KCP);
                const float m = P.m_f;
                for (int32_t e = e0; e < e1; e++) {
                    const float2 f = sf[(int64_t)lst[e] * NFOUR_HALF + t];
                    a[0] += m * f.x;
                    a[1] += m * f.y;
                }
            }
            float *o = tpart + ((int64_t)c * NFOUR_HALF + t) * EN_SEP_K;
#pragma unroll
            for (int q = 0; q < EN_SEP_K; q++) o[q] = a[q];
        }
    }
}

/*
 * The reciprocal-space expansion terms of a node from its chunks' sums
 * (chunk order): with E_n = cos th A + sin th B (n even) or sin th A - cos th B
 * (n odd) at the node's centre, M2L's reciprocal part is, per h,
 *   L0 += c (s0 E0(m0) + s2 E2(m2) - s3 E3(m3))
 *   La += c h_a (s1 E1(m0) + s3 E3(m2) - s4 E4(m3))
 *   Lab += c h_a h_b (s2 E2(m0) + s4 E4(m2)),  L3 += c h^3 s3 E3(m0),  L4 += c h^4 s4 E4(m0)
 * (P2L of a particle source is the m0 column).  One warp per node, lanes over h.
 */
__global__ void k_node_ewald_recip(int64_t nn, const int32_t *__restrict__ off, const float *__restrict__ tpart,
                                   const MSrc *__restrict__ ms, EwaldTables E, double *__restrict__ Lloc) {
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= nn || off[i + 1] == off[i]) return;
    const double pi = 3.141592653589793;
    const double s0 = -1.0 / pi, s1 = 2.0, s2 = 4.0 * pi, s3 = -8.0 * pi * pi, s4 = -16.0 * pi * pi * pi;
    double L[LP];
#pragma unroll
    for (int q = 0; q < LP; q++) L[q] = 0.0;
    const int32_t X[3] = {ms[i].x[0], ms[i].x[1], ms[i].x[2]};
    for (int t = lane; t < NFOUR_HALF; t += 32) {
        double A[EN_SEP_K];
#pragma unroll
        for (int q = 0; q < EN_SEP_K; q++) A[q] = 0.0;
        for (int32_t c = off[i]; c < off[i + 1]; c++) {
            const float *p = tpart + ((int64_t)c * NFOUR_HALF + t) * EN_SEP_K;
#pragma unroll
            for (int q = 0; q < EN_SEP_K; q++) A[q] += (double)p[q];
        }
        const float4 hv = __ldg(&E.four[t]);
        const double ct = sep_ct(hv);
        const float2 cs = sep_cs(X[0], X[1], X[2], hv);
        const double C = cs.x, S = cs.y;
        const double ev0 = C * A[0] + S * A[1], od0 = S * A[0] - C * A[1];
        const double ev2 = C * A[2] + S * A[3], od2 = S * A[2] - C * A[3];
        const double ev3 = C * A[4] + S * A[5], od3 = S * A[4] - C * A[5];
        const double v0 = ct * (s0 * ev0 + s2 * ev2 - s3 * od3);
        const double v1 = ct * (s1 * od0 + s3 * od2 - s4 * ev3);
        const double v2 = ct * (s2 * ev0 + s4 * ev2);
        const double v3 = ct * s3 * od0;
        const double v4 = ct * s4 * ev0;
        const double h[3] = {hv.x, hv.y, hv.z};
        L[E0()] += v0;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            L[E1(a)] += v1 * h[a];
#pragma unroll
            for (int b = 0; b <= a; b++) {
                L[E2(a, b)] += v2 * h[a] * h[b];
#pragma unroll
                for (int cc = 0; cc <= b; cc++) {
                    L[E3(a, b, cc)] += v3 * h[a] * h[b] * h[cc];
#pragma unroll
                    for (int d = 0; d <= cc; d++) L[E4(a, b, cc, d)] += v4 * h[a] * h[b] * h[cc] * h[d];
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < LP; q++) {
        const double v = warp_sum(L[q]);
        if (lane == 0) Lloc[i * LP + q] += v;
    }
}

/* Lloc += the node's chunk sums, in chunk order: one thread per (node, term) */
__global__ void k_node_ewald_reduce(int64_t nn, const int32_t *__restrict__ off, const double *__restrict__ part,
                                    double *__restrict__ Lloc) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nn * LP) return;
    const int64_t i = t / LP;
    const int q = (int)(t - i * LP);
    if (off[i + 1] == off[i]) return;
    double v = 0.0;
    for (int32_t c = off[i]; c < off[i + 1]; c++) v += part[(int64_t)c * LP + q];
    Lloc[i * LP + q] += v;
}
