/*
 * tg_pp.cuh -- PP direct (gravity_PP_direct, src/gravity.cpp:171-300) for the
 * FP32 path, leaf_max <= 64.  Included by tg_gravity.cu.
 *
 * Work unit: one warp (a one-warp block) per (sink leaf, chunk of up to 32
 * sinks): sinks [0, 32) and [32, ns).  A chunk of k sinks runs C copies of
 * them (C = 4 for k <= 8, 3 for k <= 10, 2 for k <= 16, else 1); copy p takes
 * every C-th source pair starting at p, and the copies' totals are added in
 * a fixed order at the end, so results do not depend on scheduling.
 *
 * Sources are staged per warp (no block barriers) in shared memory, up to
 * PP_STAGE particles (several source leaves) at a time, as PAIRS of sources
 * in the split fixed point of split_hl (negated), so that one packed FP32x2
 * instruction (FADD2 / FMUL2 / FFMA2, sm_100) works on two pairs at once:
 *     dX = (hi_i - hi_j) + (lo_i - lo_j)
 * is the reference's correctly rounded FP32 separation for each of the two
 * (three roundings-free steps, then one rounding).  An odd batch is padded
 * with a source at 1e30 whose terms are exactly zero (r^2 = inf, 1/r = 0).
 * Pairs go in groups of 8 source pairs with no branch: 1/r comes from
 * rsqrt(max(r^2, h^2)); a group whose smallest r^2 is <= h^2 (rare: the self
 * pair and softened neighbours) is then corrected pair by pair to the
 * reference's spline.  Group sums are folded into Kahan-compensated totals
 * after each group (16 pairs).
 */
#pragma once

constexpr int PP_STAGE = 128;
/* resident one-warp blocks per SM the kernel is compiled for (register cap) */
#ifndef PP_MINB
#define PP_MINB 32
#endif

/* two staged sources (even, odd), negated split coordinates */
struct __align__(16) SrcPair {
    float2 hx, hy, hz;
    float2 lx, ly, lz;
};

struct PPAcc {
    float2 tp, t0, t1, t2; /* plain partial sums, even / odd sources */
    KahanF kp, k0, k1, k2;
    __device__ __forceinline__ void init() {
        tp = t0 = t1 = t2 = make_float2(0.0f, 0.0f);
        kp.init();
        k0.init();
        k1.init();
        k2.init();
    }
    __device__ __forceinline__ void fold(float m) {
        kp.add(-m * (tp.x + tp.y));
        k0.add(-m * (t0.x + t0.y));
        k1.add(-m * (t1.x + t1.y));
        k2.add(-m * (t2.x + t2.y));
        tp = t0 = t1 = t2 = make_float2(0.0f, 0.0f);
    }
};

/* the sink's split coordinates, replicated for the packed instructions */
struct SinkHL {
    float2 hx, hy, hz, lx, ly, lz;
};

__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }

/* separations of the sink from the two sources of a pair */
__device__ __forceinline__ void pp_sep2(const SinkHL &A, const SrcPair &s, float2 &dx, float2 &dy, float2 &dz) {
    dx = __fadd2_rn(__fadd2_rn(A.hx, s.hx), __fadd2_rn(A.lx, s.lx));
    dy = __fadd2_rn(__fadd2_rn(A.hy, s.hy), __fadd2_rn(A.ly, s.ly));
    dz = __fadd2_rn(__fadd2_rn(A.hz, s.hz), __fadd2_rn(A.lz, s.lz));
}

/* source pairs [q, q + n*C) with r^2 <= h^2: replace the clamped 1/r terms by
 * the reference's softened kernel */
template <int C>
__device__ __forceinline__ void pp_soft_fix(const GParams &P, float h2, const SrcPair *sy, int q, int n, const SinkHL &A,
                                         PPAcc &a) {
    const float hinv = rsqrtf(h2);
    const float hinv3 = hinv * hinv * hinv;
    for (int u = 0; u < n; u++) {
        float2 dx, dy, dz;
        pp_sep2(A, sy[q + u * C], dx, dy, dz);
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const float x = e ? dx.y : dx.x, y = e ? dy.y : dy.x, z = e ? dz.y : dz.x;
            const float r2 = fmaf(x, x, fmaf(y, y, z * z));
            if (r2 <= h2) {
                const float d[3] = {x, y, z};
                float f, p;
                pp_direct_pair<float>(P, d, f, p);
                a.tp.x += p - hinv;
                a.t0.x = fmaf(x, f - hinv3, a.t0.x);
                a.t1.x = fmaf(y, f - hinv3, a.t1.x);
                a.t2.x = fmaf(z, f - hinv3, a.t2.x);
            }
        }
    }
}

/* one source pair: 2 interactions in packed arithmetic */
__device__ __forceinline__ void pp_pair2(const SinkHL &A, const SrcPair &s, float h2, float &rmin, PPAcc &a) {
    float2 dx, dy, dz;
    pp_sep2(A, s, dx, dy, dz);
    const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
    rmin = fminf(rmin, fminf(r2.x, r2.y));
    const float2 rinv = make_float2(rsqrtf(fmaxf(r2.x, h2)), rsqrtf(fmaxf(r2.y, h2)));
    const float2 f = __fmul2_rn(__fmul2_rn(rinv, rinv), rinv);
    a.tp = __fadd2_rn(a.tp, rinv);
    a.t0 = __ffma2_rn(dx, f, a.t0);
    a.t1 = __ffma2_rn(dy, f, a.t1);
    a.t2 = __ffma2_rn(dz, f, a.t2);
}

/* the staged source pairs [phase, np) in steps of C */
template <int C>
__device__ __forceinline__ void pp_batch(const GParams &P, float h2, float m, const SrcPair *sy, int phase, int np,
                                         const SinkHL &A, PPAcc &a) {
    int q = phase;
    for (; q + 7 * C < np; q += 8 * C) {
        float rmin = 3.0e38f;
#pragma unroll
        for (int u = 0; u < 8; u++) pp_pair2(A, sy[q + u * C], h2, rmin, a);
        if (rmin <= h2) pp_soft_fix<C>(P, h2, sy, q, 8, A, a);
        a.fold(m);
    }
    const int rest = q < np ? (np - q + C - 1) / C : 0;
    if (rest > 0) {
        float rmin = 3.0e38f;
        for (int u = 0; u < rest; u++) pp_pair2(A, sy[q + u * C], h2, rmin, a);
        if (rmin <= h2) pp_soft_fix<C>(P, h2, sy, q, rest, A, a);
        a.fold(m);
    }
}

/* a staged batch whose offsets exceed the split identity's range: per-pair
 * wrap from the raw positions of the list entries [c0, c1) (the plain path,
 * rare), this copy's share of them */
__device__ __forceinline__ void pp_batch_wrap(const GParams &P, float m, const int32_t *lst, int32_t c0, int32_t c1,
                                           const int32_t *pb, const int32_t *pe, const int4 *pos, int phase, int C,
                                           const int32_t *xi, bool per, PPAcc &a) {
    int t = 0;
    for (int32_t c = c0; c < c1; c++) {
        const int32_t src = lst[c];
        for (int32_t q = pb[src]; q < pe[src]; q++, t++) {
            if (t % C != phase) continue;
            const int4 y = pos[q];
            const float d[3] = {sep<float>(xi[0], y.x, per), sep<float>(xi[1], y.y, per), sep<float>(xi[2], y.z, per)};
            float f, p;
            pp_direct_pair<float>(P, d, f, p);
            a.tp.x += p;
            a.t0.x = fmaf(d[0], f, a.t0.x);
            a.t1.x = fmaf(d[1], f, a.t1.x);
            a.t2.x = fmaf(d[2], f, a.t2.x);
            a.fold(m);
        }
    }
}

/* far: the FP64 sums (phi, g) of L2P, PC and the Ewald kernels from
 * k_leaf<float, 64, false>; acc receives far + PP_direct - phi_self.
 * Launch: one-warp blocks, grid = 2 * nleaves (block 2l + u = leaf l, chunk u). */
__global__ void __launch_bounds__(32, PP_MINB)
    k_pp_f32(GParams P, const int32_t *__restrict__ leaves, int32_t nleaves, const int32_t *__restrict__ pb,
             const int32_t *__restrict__ pe, const MSrc *__restrict__ ms, const int4 *__restrict__ pos, ListView LV,
             const double *__restrict__ far, float4 *__restrict__ acc) {
    __shared__ SrcPair sy[PP_STAGE / 2];
    __shared__ double red[32][4];
    const int lane = threadIdx.x;
    const bool per = P.ewald != 0;
    const float m = P.m_f;
    const float h2 = (float)(P.h * P.h);
    const int32_t li = blockIdx.x >> 1, chunk = blockIdx.x & 1;
    if (li >= nleaves) return;
    const int32_t leaf = leaves[li];
    const int32_t b = pb[leaf], ns = pe[leaf] - b;
    const int k = min(32, ns - chunk * 32);
    if (k <= 0) return;
    const int C = k <= 8 ? 4 : (k <= 10 ? 3 : (k <= 16 ? 2 : 1));
    const int sidx = lane % k;
    const int phase = lane / k; /* >= C: a spare lane, computes copy 0 and is discarded */
    const int ph = phase < C ? phase : 0;
    const int32_t i = b + chunk * 32 + sidx;
    const int32_t Xr[3] = {ms[leaf].x[0], ms[leaf].x[1], ms[leaf].x[2]};
    const int4 xi4 = pos[i];
    const int32_t xi[3] = {xi4.x, xi4.y, xi4.z};
    SinkHL A;
    uint32_t amag = 0;
    {
        float h, l;
        split_hl(rel_off(xi[0], Xr[0], per, amag), h, l);
        A.hx = f2(h), A.lx = f2(l);
        split_hl(rel_off(xi[1], Xr[1], per, amag), h, l);
        A.hy = f2(h), A.ly = f2(l);
        split_hl(rel_off(xi[2], Xr[2], per, amag), h, l);
        A.hz = f2(h), A.lz = f2(l);
    }
    const uint32_t amax = warp_max_u(amag);
    PPAcc a;
    a.init();
    const int32_t *lst = LV.pool[TG_PP_D] + LV.off[TG_PP_D][leaf];
    const int32_t len = LV.len[TG_PP_D][leaf];
    float *sf = reinterpret_cast<float *>(sy);
    int32_t c = 0;
    while (c < len) {
        /* stage whole source leaves (<= 64 particles each) while they fit */
        const int32_t c0 = c;
        int nst = 0;
        uint32_t bmag = 0;
        __syncwarp();
        while (c < len) {
            const int32_t src = lst[c];
            const int32_t sb = pb[src], sn = pe[src] - sb;
            if (nst + sn > PP_STAGE) break;
            for (int q = lane; q < sn; q += 32) {
                const int4 y = pos[sb + q];
                const int t = nst + q;
                float *e = sf + (t >> 1) * 12 + (t & 1); /* SrcPair p: hx.x hx.y hy.x ... lz.y */
                float h, l;
                split_hl(rel_off(y.x, Xr[0], per, bmag), h, l);
                e[0] = -h, e[6] = -l;
                split_hl(rel_off(y.y, Xr[1], per, bmag), h, l);
                e[2] = -h, e[8] = -l;
                split_hl(rel_off(y.z, Xr[2], per, bmag), h, l);
                e[4] = -h, e[10] = -l;
            }
            nst += sn;
            c++;
        }
        if ((nst & 1) && lane == 0) { /* pad: exactly zero terms */
            float *e = sf + (nst >> 1) * 12 + 1;
            e[0] = -1.0e30f;
            e[2] = e[4] = e[6] = e[8] = e[10] = 0.0f;
        }
        const uint32_t bmax = warp_max_u(bmag);
        __syncwarp();
        const int np = (nst + 1) >> 1;
        if ((unsigned long long)amax + bmax < (1ull << 30)) {
            switch (C) {
            case 1: pp_batch<1>(P, h2, m, sy, ph, np, A, a); break;
            case 2: pp_batch<2>(P, h2, m, sy, ph, np, A, a); break;
            case 3: pp_batch<3>(P, h2, m, sy, ph, np, A, a); break;
            default: pp_batch<4>(P, h2, m, sy, ph, np, A, a); break;
            }
        } else {
            pp_batch_wrap(P, m, lst, c0, c, pb, pe, pos, ph, C, xi, per, a);
        }
    }
    red[lane][0] = (double)a.kp.s - (double)a.kp.c;
    red[lane][1] = (double)a.k0.s - (double)a.k0.c;
    red[lane][2] = (double)a.k1.s - (double)a.k1.c;
    red[lane][3] = (double)a.k2.s - (double)a.k2.c;
    __syncwarp();
    if (lane < k) {
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int p = 0; p < C; p++)
#pragma unroll
            for (int q = 0; q < 4; q++) v[q] += red[lane + p * k][q];
        const double *fr = far + 4 * (int64_t)i;
        acc[i] = make_float4((float)(fr[0] + v[0] - P.phi_self), (float)(fr[1] + v[1]), (float)(fr[2] + v[2]),
                             (float)(fr[3] + v[3]));
    }
}
