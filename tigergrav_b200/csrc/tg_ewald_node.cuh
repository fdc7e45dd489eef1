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

template <class T>
__global__ void __launch_bounds__(128, EN_MINB) k_node_ewald(GParams P, int64_t nn, int32_t nchunks,
                                                    const int32_t *__restrict__ off, const int32_t *__restrict__ pb,
                                                    const int32_t *__restrict__ pe, const MSrc *__restrict__ ms,
                                                    const int4 *__restrict__ pos, ListView LV, EwaldTables E,
                                                    double *__restrict__ part) {
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
                green_ewald_full<T>(E, dX, D);
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
                green_ewald_warp<T>(E, dX, D, lane);
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
                green_ewald_full<T>(E, dX, D);
                contract_P2L<T, T>(L, m, D);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < LP; q++) {
        const double v = warp_sum((double)L[q]);
        if (lane == 0) part[(int64_t)c * LP + q] = v;
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
