/*
 * tg_ewald_leaf.cuh -- the leaf-sink Ewald kernels (gravity_PC_ewald,
 * src/gravity.cpp:616-678; gravity_PP_ewald, :491-614) as balanced work
 * units.  Included by tg_gravity.cu.
 *
 * The Ewald lists of a leaf are very uneven: large leaves in voids fail the
 * Ewald self test and interact with every leaf within (r_a + r_b)/theta, so
 * at theta = 0.2 on a clustered box 1% of the leaves hold half the PP_Ewald
 * pairs (up to 9e6 for one leaf).  One block per leaf would leave a tail of a
 * few blocks running for most of the kernel.  Instead each leaf's PP_E list
 * is cut into chunks of EW_KPP source leaves and its PC_E list into chunks of
 * EW_KPC source nodes; one 64-thread block (a thread per sink) evaluates one
 * chunk and writes its sinks' partial sums to its own slot of a scratch
 * array; k_ewald_reduce then adds a leaf's chunk sums in chunk order to the
 * leaf's FP64 accumulators.  The result does not depend on scheduling.
 */
#pragma once

constexpr int EW_KPP = 32;  /* PP_E source leaves per chunk (<= 32 * 64 * 64 pairs) */
constexpr int EW_KPC = 128; /* PC_E source nodes per chunk */
#ifndef EW_MINB
#define EW_MINB 12 /* resident 64-thread blocks per SM the kernel is compiled for */
#endif

/* chunks per leaf; cnt[nleaves] = 0 so that an exclusive scan ends in the total */
__global__ void k_ewald_count(const int32_t *__restrict__ leaves, int32_t nleaves, ListView LV,
                              int32_t *__restrict__ cnt) {
    const int32_t li = blockIdx.x * blockDim.x + threadIdx.x;
    if (li > nleaves) return;
    if (li == nleaves) {
        cnt[li] = 0;
        return;
    }
    const int32_t leaf = leaves[li];
    const int32_t npp = LV.len[TG_PP_E][leaf], npc = LV.len[TG_PC_E][leaf];
    cnt[li] = (npp + EW_KPP - 1) / EW_KPP + (npc + EW_KPC - 1) / EW_KPC;
}

/* one chunk: PP_E entries [k EW_KPP, ...) or PC_E entries [(k - npp) EW_KPC, ...) of its leaf */
template <class T, bool SEP>
__global__ void __launch_bounds__(64, EW_MINB) k_ewald_chunk(GParams P, const int32_t *__restrict__ leaves, int32_t nleaves,
                                                    const int32_t *__restrict__ off, const int32_t *__restrict__ pb,
                                                    const int32_t *__restrict__ pe, const MSrc *__restrict__ ms,
                                                    const int4 *__restrict__ pos, const int32_t *__restrict__ aabb,
                                                    ListView LV, EwaldTables E, double *__restrict__ part,
                                                    const float2 *__restrict__ nt, const float2 *__restrict__ sf,
                                                    float *__restrict__ tpart) {
    __shared__ int4 sy[64];
    __shared__ float4 s_img[SEP ? EW_IMG_CAP : 1]; /* FP32: the block's image list per source */
    __shared__ int s_tmp[3];
    const int tid = threadIdx.x;
    const int64_t c = blockIdx.x;
    int32_t lo = 0, hi = nleaves - 1; /* the leaf: largest li with off[li] <= c */
    while (lo < hi) {
        const int32_t mid = (lo + hi + 1) >> 1;
        if ((int64_t)off[mid] <= c) lo = mid;
        else hi = mid - 1;
    }
    const int32_t li = lo, k = (int32_t)(c - off[li]);
    const int32_t leaf = leaves[li];
    const int32_t b = pb[leaf], cnt = pe[leaf] - b;
    const bool active = tid < cnt;
    const int4 xi4 = pos[b + (active ? tid : 0)];
    const int32_t xi[3] = {xi4.x, xi4.y, xi4.z};
    Acc<T> aphi, ag[3];
    aphi.init(0.0);
    for (int d = 0; d < 3; d++) ag[d].init(0.0);
    const int32_t lpp = LV.len[TG_PP_E][leaf];
    const int32_t npp = (lpp + EW_KPP - 1) / EW_KPP;
    if (k < npp) {
        const int32_t *lst = LV.pool[TG_PP_E] + LV.off[TG_PP_E][leaf];
        const int32_t e1 = min(lpp, (k + 1) * EW_KPP);
        const T m = T(P.m_d);
        for (int32_t e = k * EW_KPP; e < e1; e++) {
            const int32_t src = lst[e];
            const int32_t sb = pb[src], sn = pe[src] - sb;
            EwPairing Q;
            int nimg = 0, s0 = 0;
            if constexpr (SEP) {
                ew_pairing(aabb + 6 * leaf, aabb + 6 * leaf + 3, aabb + 6 * src, aabb + 6 * src + 3, 2.0f, Q);
                nimg = ew_image_set(Q.c, Q.rr, s_img, s_tmp, s0);
            }
            for (int32_t base = 0; base < sn; base += 64) {
                const int32_t nsy = min(64, sn - base);
                __syncthreads();
                if (tid < nsy) sy[tid] = pos[sb + base + tid];
                __syncthreads();
                for (int32_t q = 0; q < nsy; q++) {
                    const int4 y = sy[q];
                    T dX[3] = {wrap_sep_t<T>(xi[0], y.x), wrap_sep_t<T>(xi[1], y.y), wrap_sep_t<T>(xi[2], y.z)};
                    T ph, g[3];
                    if constexpr (SEP) {
                        ImgList L{s_img, nimg, s0, Q.wrap, 0.0f, 0.0f, 0.0f};
                        if (Q.wrap) { /* block-uniform */
                            L.k0 = ew_wrap_k(Q.C[0], xi[0], Q.a[0], y.x, Q.b[0]);
                            L.k1 = ew_wrap_k(Q.C[1], xi[1], Q.a[1], y.y, Q.b[1]);
                            L.k2 = ew_wrap_k(Q.C[2], xi[2], Q.a[2], y.z, Q.b[2]);
                        }
                        pp_ewald_pair_sep(E, dX, ph, g, L);
                    } else {
                        pp_ewald_pair<T>(E, dX, ph, g);
                    }
                    aphi.add(m * ph);
                    for (int d = 0; d < 3; d++) ag[d].add(m * g[d]);
                }
            }
        }
    } else {
        const int32_t lpc = LV.len[TG_PC_E][leaf];
        const int32_t *lst = LV.pool[TG_PC_E] + LV.off[TG_PC_E][leaf];
        const int32_t e0 = (k - npp) * EW_KPC, e1 = min(lpc, e0 + EW_KPC);
        for (int32_t e = e0; e < e1; e++) {
            const MSrc &s = ms[lst[e]];
            T dX[3], D[LP], M[MP];
#pragma unroll
            for (int d = 0; d < 3; d++) dX[d] = sep<T>(xi[d], s.x[d], true);
#pragma unroll
            for (int q = 0; q < MP; q++) M[q] = T(s.m[q]);
            if constexpr (SEP) {
                EwPairing Q;
                ew_pairing(aabb + 6 * leaf, aabb + 6 * leaf + 3, s.x, s.x, 2.1f, Q);
                int s0;
                const int nimg = ew_image_set(Q.c, Q.rr, s_img, s_tmp, s0);
                ImgList L{s_img, nimg, s0, Q.wrap, 0.0f, 0.0f, 0.0f};
                if (Q.wrap) { /* block-uniform */
                    L.k0 = ew_wrap_k(Q.C[0], xi[0], Q.a[0], s.x[0], Q.b[0]);
                    L.k1 = ew_wrap_k(Q.C[1], xi[1], Q.a[1], s.x[1], Q.b[1]);
                    L.k2 = ew_wrap_k(Q.C[2], xi[2], Q.a[2], s.x[2], Q.b[2]);
                }
                green_ewald_sep(E, dX, D, L);
            } else {
                green_ewald_full<T>(E, dX, D);
            }
            T ph, g[3];
            contract_M2P<T>(ph, g, M, D);
            aphi.add(ph);
            for (int d = 0; d < 3; d++) ag[d].add(g[d]);
        }
    }
    if (active) {
        double *o = part + 4 * (c * 64 + tid);
        o[0] = aphi.get();
        for (int d = 0; d < 3; d++) o[1 + d] = ag[d].get();
    }
    if constexpr (SEP) {
        /* this chunk's share of the leaf's reciprocal sums: thread t takes vector h_t */
        if (tid < NFOUR_HALF) {
            float a[EW_SEP_K];
#pragma unroll
            for (int q = 0; q < EW_SEP_K; q++) a[q] = 0.0f;
            if (k < npp) {
                const int32_t *lst = LV.pool[TG_PP_E] + LV.off[TG_PP_E][leaf];
                const int32_t e1 = min(lpp, (k + 1) * EW_KPP);
                const float m = P.m_f;
                for (int32_t e = k * EW_KPP; e < e1; e++) {
                    const float2 f = sf[(int64_t)lst[e] * NFOUR_HALF + tid];
                    a[0] += m * f.x;
                    a[1] += m * f.y;
                }
            } else {
                const int32_t lpc = LV.len[TG_PC_E][leaf];
                const int32_t *lst = LV.pool[TG_PC_E] + LV.off[TG_PC_E][leaf];
                const int32_t e0 = (k - npp) * EW_KPC, e1 = min(lpc, e0 + EW_KPC);
                SepQ Q;
                sep_q(__ldg(&E.four[tid]), Q);
                for (int32_t e = e0; e < e1; e++) {
                    const int32_t src = lst[e];
                    const float2 f = nt[(int64_t)src * NFOUR_HALF + tid];
                    const float *M = ms[src].m;
                    float m2 = 0.0f, m3 = 0.0f, m3p = 0.0f;
#pragma unroll
                    for (int i = 0; i < 6; i++) m2 += Q.q2[i] * M[1 + i];
#pragma unroll
                    for (int i = 0; i < 10; i++) {
                        m3 += Q.q3[i] * M[7 + i];
                        m3p += Q.q3p[i] * M[7 + i];
                    }
                    a[0] += M[0] * f.x;
                    a[1] += M[0] * f.y;
                    a[2] += m2 * f.x;
                    a[3] += m2 * f.y;
                    a[4] += m3p * f.x;
                    a[5] += m3p * f.y;
                    a[6] += m3 * f.x;
                    a[7] += m3 * f.y;
                }
            }
            float *o = tpart + (c * NFOUR_HALF + tid) * EW_SEP_K;
#pragma unroll
            for (int q = 0; q < EW_SEP_K; q++) o[q] = a[q];
        }
    }
}

/* add each leaf's chunk sums, in chunk order, to its FP64 accumulators; with
 * tpart, also the reciprocal part from the chunks' leaf sums (in chunk order) */
__global__ void __launch_bounds__(64) k_ewald_reduce(const int32_t *__restrict__ leaves, int32_t nleaves,
                                                     const int32_t *__restrict__ off, const int32_t *__restrict__ pb,
                                                     const int32_t *__restrict__ pe, const double *__restrict__ part,
                                                     double *__restrict__ acc, const float *__restrict__ tpart,
                                                     const int4 *__restrict__ pos, EwaldTables E) {
    __shared__ double sT[NFOUR_HALF * EW_SEP_K];
    __shared__ double sct[NFOUR_HALF];
    const int32_t li = blockIdx.x;
    const int tid = threadIdx.x;
    if (li >= nleaves) return;
    const int32_t leaf = leaves[li];
    const int32_t b = pb[leaf], cnt = pe[leaf] - b;
    if (off[li + 1] == off[li]) return;
    if (tpart) { /* block-uniform */
        for (int i = tid; i < NFOUR_HALF * EW_SEP_K; i += 64) {
            double s = 0.0;
            for (int64_t c = off[li]; c < off[li + 1]; c++) s += (double)tpart[c * NFOUR_HALF * EW_SEP_K + i];
            sT[i] = s;
        }
        for (int t = tid; t < NFOUR_HALF; t += 64) sct[t] = sep_ct(__ldg(&E.four[t]));
        __syncthreads();
    }
    if (tid >= cnt) return;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t c = off[li]; c < off[li + 1]; c++)
#pragma unroll
        for (int q = 0; q < 4; q++) v[q] += part[4 * (c * 64 + tid) + q];
    if (tpart) {
        const int4 p = pos[b + tid];
        sep_eval(E, sT, sct, p.x, p.y, p.z, v[0], v + 1);
    }
    double *o = acc + 4 * (int64_t)(b + tid);
#pragma unroll
    for (int q = 0; q < 4; q++) o[q] += v[q];
}
