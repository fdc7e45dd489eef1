/*
 * tg_pp.cuh -- PP direct (gravity_PP_direct, src/gravity.cpp:171-300) for the
 * FP32 path, leaf_max <= 64.  Included by tg_gravity.cu.
 *
 * One block of two warps per sink leaf, one warp per 32 sinks; a warp with
 * 16 or fewer sinks runs two copies of them over alternate sources.  Each
 * warp stages up to PP_STAGE source particles (several source leaves) in its
 * own shared memory -- no block barriers -- in the split fixed point of
 * split_hl, so dX is the reference's correctly rounded separation from three
 * FP32 additions.  Pairs go in groups of 8 with no branch: 1/r comes from
 * rsqrt(max(r^2, h^2)); a group whose smallest r^2 is <= h^2 (rare: the self
 * pair and softened neighbours) is then corrected pair by pair to the
 * reference's spline.  Group sums are folded into Kahan-compensated totals
 * every 16 pairs.
 */
#pragma once

constexpr int PP_STAGE = 128;

struct PPAcc {
    float tp, t0, t1, t2; /* plain partial sums */
    KahanF kp, k0, k1, k2;
    __device__ __forceinline__ void init() {
        tp = t0 = t1 = t2 = 0.0f;
        kp.init();
        k0.init();
        k1.init();
        k2.init();
    }
    __device__ __forceinline__ void fold(float m) {
        kp.add(-m * tp);
        k0.add(-m * t0);
        k1.add(-m * t1);
        k2.add(-m * t2);
        tp = t0 = t1 = t2 = 0.0f;
    }
};

__device__ __forceinline__ void pp_sep(const float *AH, const float *AL, const SrcHL &s, float &dx, float &dy,
                                       float &dz) {
    dx = (AH[0] - s.hx) + (AL[0] - s.lx);
    dy = (AH[1] - s.hy) + (AL[1] - s.ly);
    dz = (AH[2] - s.hz) + (AL[2] - s.lz);
}

/* pairs [q, q + n*STEP) with r^2 <= h^2: replace the clamped 1/r terms by the
 * reference's softened kernel */
template <int STEP>
__device__ __forceinline__ void pp_soft_fix(const GParams &P, float h2, const SrcHL *sy, int q, int n, const float *AH,
                                            const float *AL, PPAcc &a) {
    const float hinv = rsqrtf(h2);
    const float hinv3 = hinv * hinv * hinv;
    for (int u = 0; u < n; u++) {
        float dx, dy, dz;
        pp_sep(AH, AL, sy[q + u * STEP], dx, dy, dz);
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        if (r2 <= h2) {
            const float d[3] = {dx, dy, dz};
            float f, p;
            pp_direct_pair<float>(P, d, f, p);
            a.tp += p - hinv;
            a.t0 = fmaf(dx, f - hinv3, a.t0);
            a.t1 = fmaf(dy, f - hinv3, a.t1);
            a.t2 = fmaf(dz, f - hinv3, a.t2);
        }
    }
}

/* the staged batch [half, nst) in steps of STEP */
template <int STEP>
__device__ __forceinline__ void pp_batch(const GParams &P, float h2, float m, const SrcHL *sy, int half, int nst,
                                         const float *AH, const float *AL, PPAcc &a) {
    int q = half;
    int groups = 0;
    for (; q + 7 * STEP < nst; q += 8 * STEP) {
        float rmin = 3.0e38f;
#pragma unroll
        for (int u = 0; u < 8; u++) {
            float dx, dy, dz;
            pp_sep(AH, AL, sy[q + u * STEP], dx, dy, dz);
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            rmin = fminf(rmin, r2);
            const float rinv = rsqrtf(fmaxf(r2, h2));
            const float f = rinv * rinv * rinv;
            a.tp += rinv;
            a.t0 = fmaf(dx, f, a.t0);
            a.t1 = fmaf(dy, f, a.t1);
            a.t2 = fmaf(dz, f, a.t2);
        }
        if (rmin <= h2) pp_soft_fix<STEP>(P, h2, sy, q, 8, AH, AL, a);
        if (++groups & 1) continue;
        a.fold(m);
    }
    const int rest = (nst - q + STEP - 1) / STEP;
    if (rest > 0) {
        float rmin = 3.0e38f;
        for (int u = 0; u < rest; u++) {
            float dx, dy, dz;
            pp_sep(AH, AL, sy[q + u * STEP], dx, dy, dz);
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            rmin = fminf(rmin, r2);
            const float rinv = rsqrtf(fmaxf(r2, h2));
            const float f = rinv * rinv * rinv;
            a.tp += rinv;
            a.t0 = fmaf(dx, f, a.t0);
            a.t1 = fmaf(dy, f, a.t1);
            a.t2 = fmaf(dz, f, a.t2);
        }
        if (rmin <= h2) pp_soft_fix<STEP>(P, h2, sy, q, rest, AH, AL, a);
    }
    a.fold(m);
}

/* a staged batch whose offsets exceed the split identity's range: per-pair
 * wrap from the raw positions (the plain path, rare) */
__device__ __forceinline__ void pp_batch_wrap(const GParams &P, float m, const int4 *raw, int half, int step, int nst,
                                              const int32_t *xi, bool per, PPAcc &a) {
    for (int q = half; q < nst; q += step) {
        const int4 y = raw[q];
        const float d[3] = {sep<float>(xi[0], y.x, per), sep<float>(xi[1], y.y, per), sep<float>(xi[2], y.z, per)};
        float f, p;
        pp_direct_pair<float>(P, d, f, p);
        a.tp += p;
        a.t0 = fmaf(d[0], f, a.t0);
        a.t1 = fmaf(d[1], f, a.t1);
        a.t2 = fmaf(d[2], f, a.t2);
        a.fold(m);
    }
}

/* far: the FP64 sums (phi, g) of L2P, PC and the Ewald kernels from
 * k_leaf<float, 64, false>; acc receives far + PP_direct - phi_self. */
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 16)
    k_pp_f32(GParams P, const int32_t *__restrict__ leaves, int32_t nleaves, const int32_t *__restrict__ pb,
             const int32_t *__restrict__ pe, const MSrc *__restrict__ ms, const int4 *__restrict__ pos, ListView LV,
             const double *__restrict__ far, float4 *__restrict__ acc) {
    __shared__ SrcHL sy[WARPS][PP_STAGE];
    __shared__ int4 sraw[WARPS][PP_STAGE];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool per = P.ewald != 0;
    const float m = P.m_f;
    const float h2 = (float)(P.h * P.h);
    for (int32_t li = blockIdx.x; li < nleaves; li += gridDim.x) {
        const int32_t leaf = leaves[li];
        const int32_t b = pb[leaf], ns = pe[leaf] - b;
        const int k = min(32, ns - warp * 32);
        if (k <= 0) continue;
        const bool split = k <= 16;
        const int sidx = split ? (lane & 15) : lane;
        const int half = split ? (lane >> 4) : 0;
        const bool active = sidx < k;
        const int32_t i = b + warp * 32 + (active ? sidx : 0);
        const int32_t Xr[3] = {ms[leaf].x[0], ms[leaf].x[1], ms[leaf].x[2]};
        const int4 xi4 = pos[i];
        const int32_t xi[3] = {xi4.x, xi4.y, xi4.z};
        float AH[3], AL[3];
        uint32_t amag = 0;
#pragma unroll
        for (int d = 0; d < 3; d++) split_hl(rel_off(xi[d], Xr[d], per, amag), AH[d], AL[d]);
        const uint32_t A = warp_max_u(amag);
        PPAcc a;
        a.init();
        const int32_t *lst = LV.pool[TG_PP_D] + LV.off[TG_PP_D][leaf];
        const int32_t len = LV.len[TG_PP_D][leaf];
        int32_t c = 0;
        while (c < len) {
            /* stage whole source leaves while they fit */
            int nst = 0;
            uint32_t bmag = 0;
            __syncwarp();
            while (c < len) {
                const int32_t src = lst[c];
                const int32_t sb = pb[src], sn = pe[src] - sb;
                if (nst + sn > PP_STAGE) break;
                for (int q = lane; q < sn; q += 32) {
                    const int4 y = pos[sb + q];
                    SrcHL s;
                    split_hl(rel_off(y.x, Xr[0], per, bmag), s.hx, s.lx);
                    split_hl(rel_off(y.y, Xr[1], per, bmag), s.hy, s.ly);
                    split_hl(rel_off(y.z, Xr[2], per, bmag), s.hz, s.lz);
                    s.hpad = s.lpad = 0.0f;
                    sy[warp][nst + q] = s;
                    sraw[warp][nst + q] = y;
                }
                nst += sn;
                c++;
            }
            const uint32_t B = warp_max_u(bmag);
            __syncwarp();
            if ((unsigned long long)A + B < (1ull << 30)) {
                if (split) pp_batch<2>(P, h2, m, sy[warp], half, nst, AH, AL, a);
                else pp_batch<1>(P, h2, m, sy[warp], 0, nst, AH, AL, a);
            } else {
                pp_batch_wrap(P, m, sraw[warp], half, split ? 2 : 1, nst, xi, per, a);
            }
        }
        double v[4] = {(double)a.kp.s - (double)a.kp.c, (double)a.k0.s - (double)a.k0.c,
                       (double)a.k1.s - (double)a.k1.c, (double)a.k2.s - (double)a.k2.c};
        if (split) {
#pragma unroll
            for (int q = 0; q < 4; q++) v[q] += __shfl_xor_sync(0xffffffffu, v[q], 16);
        }
        if (active && half == 0) {
            const double *fr = far + 4 * (int64_t)i;
            acc[i] = make_float4((float)(fr[0] + v[0] - P.phi_self), (float)(fr[1] + v[1]), (float)(fr[2] + v[2]),
                                 (float)(fr[3] + v[3]));
        }
    }
}
