/*
 * tg_pp2.cuh -- PP direct (gravity_PP_direct, src/gravity.cpp:171-300) for the
 * FP32 path, leaf_max <= 64.  Included by tg_gravity.cu after tg_pp.cuh.
 *
 * Work unit: one block of PPB_T threads per sink leaf.  A leaf of ns sinks
 * runs C = PPB_T / ns copies of them: thread t takes sink t % ns and copy
 * t / ns, copy p takes the p-th of C contiguous shares of each stage's
 * source pairs, and the copies' totals are added in a fixed order at the end
 * (results do not depend on scheduling).  All warps of the block share one staging area: the block
 * stages whole source leaves (up to PPB_STAGE particles, coalesced loads of
 * each leaf's consecutive particles) and every copy of every sink reads them.
 *
 * Two kinds of source leaves, told apart per leaf from the particle bounding
 * boxes (nearest image):
 *   near  -- a gap to the sink leaf's box below max(2 (its diagonal + 2), h):
 *            the split fixed point of split_hl (tg_gravity.cu), so that
 *            dX = (hi_i - hi_j) + (lo_i - lo_j) is the reference's correctly
 *            rounded FP32 separation (src/gravity.cpp:223), bit for bit;
 *            softened pairs corrected to the reference's spline.
 *   far   -- every pair at least max(2 |a_i|, h) apart (a_i: the sink's offset
 *            from its leaf centre): offsets from the sink leaf centre rounded
 *            to FP32 once, dX = a_i - b_j in one subtraction.  Its error is at
 *            most 2^-24 (|a_i| + |b_j| + |dX|) <= 1.5 2^-23 |dX| (3 ulp of dX;
 *            the reference's conversion gives 0.5 ulp), and no pair is
 *            softened, so neither the clamp nor the spline check is needed.
 * The far form costs one packed FP32x2 addition per axis for two pairs where
 * the split form costs three, and reads four sources per 16-byte load; at the 256^3 clustered workload nearly all PP
 * pairs are far.  Sums accumulate in FP32 over groups of 16 interactions
 * (near) or 32 (far), folded into Kahan-compensated totals.
 */
#pragma once

constexpr int PPB_T = 128;     /* threads per block (one sink leaf) */
constexpr int PPB_STAGE = 512; /* staged source particles per pass */
constexpr int PPB_META = 64;   /* staged source leaves per pass, at most */
#ifndef PPB_MINB
#define PPB_MINB 10
#endif

__device__ __forceinline__ uint32_t lanemask_lt_pp() {
    uint32_t r;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
    return r;
}

/* four staged sources in the far form: negated FP32 offsets, one 16-byte
 * load per axis for four interactions */
struct __align__(16) FarQuad {
    float4 x, y, z;
};

/* gap between the intervals [a0, a1] and [b0, b1] of fixed-point coordinates
 * (nearest image when periodic) */
__device__ __forceinline__ double ppb_axis_gap(int32_t a0, int32_t a1, int32_t b0, int32_t b1, bool per) {
    long long g = max(0ll, max((long long)b0 - a1, (long long)a0 - b1));
    if (per) {
        const long long P = 1ll << 32;
        g = min(g, max(0ll, max((long long)b0 + P - a1, (long long)a0 - ((long long)b1 + P))));
        g = min(g, max(0ll, max((long long)b0 - P - a1, (long long)a0 - ((long long)b1 - P))));
    }
    return (double)g;
}

/* two far sources (packed): 2 interactions, no softening possible */
__device__ __forceinline__ void ppb_far2(const float2 &ax, const float2 &ay, const float2 &az, float2 sx, float2 sy,
                                         float2 sz, PPAcc &a) {
    const float2 dx = __fadd2_rn(ax, sx), dy = __fadd2_rn(ay, sy), dz = __fadd2_rn(az, sz);
    const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
    const float2 rinv = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
    const float2 f = __fmul2_rn(__fmul2_rn(rinv, rinv), rinv);
    a.tp = __fadd2_rn(a.tp, rinv);
    a.t0 = __ffma2_rn(dx, f, a.t0);
    a.t1 = __ffma2_rn(dy, f, a.t1);
    a.t2 = __ffma2_rn(dz, f, a.t2);
}
__device__ __forceinline__ void ppb_far4(const float2 &ax, const float2 &ay, const float2 &az, const FarQuad &s,
                                         PPAcc &a) {
    const float4 x = s.x, y = s.y, z = s.z;
    ppb_far2(ax, ay, az, make_float2(x.x, x.y), make_float2(y.x, y.y), make_float2(z.x, z.y), a);
    ppb_far2(ax, ay, az, make_float2(x.z, x.w), make_float2(y.z, y.w), make_float2(z.z, z.w), a);
}

/* near source pairs [q, q + n) with r^2 <= h^2: the reference's softened
 * kernel in place of the clamped 1/r terms */
__device__ __noinline__ void ppb_soft_fix(const GParams &P, float h2, const SrcPair *sy, int q, int n, const SinkHL &A,
                                          PPAcc &a) {
    const float hinv = rsqrt_ftz(h2);
    const float hinv3 = hinv * hinv * hinv;
    for (int u = 0; u < n; u++) {
        float2 dx, dy, dz;
        pp_sep2(A, sy[q + u], dx, dy, dz);
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

/* the near (split) source pairs [q0, q1) of a stage: this copy's share */
__device__ __forceinline__ void ppb_near_stage(const GParams &P, float h2, float m, const SrcPair *sy, int q0, int q1,
                                               const SinkHL &A, PPAcc &a) {
    int q = q0;
    for (; q + 8 <= q1; q += 8) {
        float rmin = 3.0e38f;
#pragma unroll
        for (int u = 0; u < 8; u++) pp_pair2(A, sy[q + u], h2, rmin, a);
        if (rmin <= h2) ppb_soft_fix(P, h2, sy, q, 8, A, a);
        a.fold(m);
    }
    if (q < q1) {
        float rmin = 3.0e38f;
        for (int u = q; u < q1; u++) pp_pair2(A, sy[u], h2, rmin, a);
        if (rmin <= h2) ppb_soft_fix(P, h2, sy, q, q1 - q, A, a);
        a.fold(m);
    }
}

/* the far source quads [q0, q1) of a stage: this copy's share, folded into
 * the compensated totals every 8 quads (32 interactions) */
__device__ __forceinline__ void ppb_far_stage(float m, const FarQuad *sy, int q0, int q1, const float2 &ax,
                                              const float2 &ay, const float2 &az, PPAcc &a) {
    int q = q0;
    for (; q + 8 <= q1; q += 8) {
#pragma unroll
        for (int u = 0; u < 8; u++) ppb_far4(ax, ay, az, sy[q + u], a);
        a.fold(m);
    }
    if (q < q1) {
        for (; q < q1; q++) ppb_far4(ax, ay, az, sy[q], a);
        a.fold(m);
    }
}

/* a stage whose offsets exceed the range of the two forms above (sources
 * about half a box from the sink leaf, in small boxes at small theta): per
 * pair from the raw positions with the reference's int32 wrap, this copy's
 * share */
__device__ __noinline__ void ppb_wrap_stage(const GParams &P, float m, const int32_t *m_start, const int32_t *m_pb,
                                            int nmeta, const int4 *pos, int phase, int C, const int32_t *xi,
                                            bool per, PPAcc &a) {
    for (int k = 0; k < nmeta; k++) {
        for (int32_t q = m_start[k]; q < m_start[k + 1]; q++) {
            if (q % C != phase) continue;
            const int4 y = pos[m_pb[k] + (q - m_start[k])];
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
 * Launch: blocks of PPB_T threads, grid = nleaves. */
__global__ void __launch_bounds__(PPB_T, PPB_MINB)
    k_pp_leaf(GParams P, const int32_t *__restrict__ leaves, int32_t nleaves, const int32_t *__restrict__ pb,
              const int32_t *__restrict__ pe, const MSrc *__restrict__ ms, const int32_t *__restrict__ aabb,
              const int4 *__restrict__ pos, ListView LV, const double *__restrict__ far, float4 *__restrict__ acc) {
    __shared__ __align__(16) SrcPair stage[PPB_STAGE / 2]; /* the far form (FarQuad) uses the first half */
    __shared__ int32_t m_start[PPB_META + 1], m_pb[PPB_META];
    __shared__ int32_t s_nmeta, s_used, s_cursor;
    __shared__ uint32_t s_amag, s_bmag;
    __shared__ double red[PPB_T][4];
    const int t = threadIdx.x, lane = t & 31;
    const bool per = P.ewald != 0;
    const float m = P.m_f;
    const float h2 = (float)(P.h * P.h);
    if ((int32_t)blockIdx.x >= nleaves) return;
    const int32_t leaf = leaves[blockIdx.x];
    const int32_t b = pb[leaf], ns = pe[leaf] - b;
    if (ns <= 0) return;
    const int C = max(1, PPB_T / ns);
    const int sidx = t % ns, phase = t / ns;
    const bool active = phase < C;
    const int32_t i = b + sidx;
    const int32_t Xr[3] = {ms[leaf].x[0], ms[leaf].x[1], ms[leaf].x[2]};
    const int4 xi4 = pos[i];
    const int32_t xi[3] = {xi4.x, xi4.y, xi4.z};
    SinkHL A;
    float2 ax, ay, az;
    uint32_t amag = 0;
    {
        float h, l;
        int32_t o = rel_off(xi[0], Xr[0], per, amag);
        split_hl(o, h, l);
        A.hx = f2(h), A.lx = f2(l), ax = f2(__int2float_rn(o) * 2.3283064365386963e-10f);
        o = rel_off(xi[1], Xr[1], per, amag);
        split_hl(o, h, l);
        A.hy = f2(h), A.ly = f2(l), ay = f2(__int2float_rn(o) * 2.3283064365386963e-10f);
        o = rel_off(xi[2], Xr[2], per, amag);
        split_hl(o, h, l);
        A.hz = f2(h), A.lz = f2(l), az = f2(__int2float_rn(o) * 2.3283064365386963e-10f);
    }
    /* the sink leaf's box: a source leaf is far when its box is at least
     * max(2 (diagonal + 2), h + 2) away (fixed-point units) */
    int32_t bx[6];
#pragma unroll
    for (int d = 0; d < 6; d++) bx[d] = aabb[6 * leaf + d];
    double diag2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double e = (double)((long long)bx[3 + d] - bx[d]);
        diag2 += e * e;
    }
    const double hfix = P.h * 4294967296.0;
    const double gmin = fmax(2.0 * (sqrt(diag2) + 2.0), hfix + 2.0);
    const double gmin2 = gmin * gmin;
    if (t == 0) s_amag = 0u;
    __syncthreads();
    atomicMax(&s_amag, amag);

    PPAcc a;
    a.init();
    const int32_t *lst = LV.pool[TG_PP_D] + LV.off[TG_PP_D][leaf];
    const int32_t len = LV.len[TG_PP_D][leaf];
    float *sf = reinterpret_cast<float *>(stage);
    for (int pass = 0; pass < 2; pass++) { /* 0: near leaves (split form), 1: far leaves */
        if (t == 0) s_cursor = 0;
        __syncthreads();
        for (;;) {
            /* warp 0 picks the next whole source leaves of this kind that fit */
            if (t < 32) {
                int nmeta = 0, used = 0, cur = s_cursor;
                while (cur < len && nmeta + 32 <= PPB_META) {
                    const int e = cur + lane;
                    int sn = 0, sb = 0;
                    if (e < len) {
                        const int32_t src = lst[e];
                        sb = pb[src];
                        sn = pe[src] - sb;
                        if (sn > 0) {
                            double g2 = 0.0;
#pragma unroll
                            for (int d = 0; d < 3; d++) {
                                const double g = ppb_axis_gap(bx[d], bx[3 + d], aabb[6 * src + d], aabb[6 * src + 3 + d],
                                                              per);
                                g2 += g * g;
                            }
                            if ((g2 >= gmin2) != (pass == 1)) sn = 0;
                        }
                    }
                    int inc = sn;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int v = __shfl_up_sync(0xffffffffu, inc, o);
                        if (lane >= o) inc += v;
                    }
                    const int navail = min(32, len - cur);
                    const int take = min(__popc(__ballot_sync(0xffffffffu, used + inc <= PPB_STAGE)), navail);
                    const bool rec = lane < take && sn > 0;
                    const uint32_t rm = __ballot_sync(0xffffffffu, rec);
                    if (rec) {
                        const int k = nmeta + __popc(rm & lanemask_lt_pp());
                        m_start[k] = used + inc - sn;
                        m_pb[k] = sb;
                    }
                    nmeta += __popc(rm);
                    if (take > 0) used += __shfl_sync(0xffffffffu, inc, take - 1);
                    cur += take;
                    if (take < navail) break; /* the stage is full */
                }
                if (lane == 0) {
                    s_nmeta = nmeta;
                    s_used = used;
                    s_cursor = cur;
                    m_start[nmeta] = used;
                    s_bmag = 0u;
                }
            }
            __syncthreads();
            const int used = s_used, nmeta = s_nmeta;
            if (used == 0) break; /* the list is exhausted for this kind */
            /* warp w copies the source leaves w, w + 4, ...: its lanes take
             * consecutive particles of one leaf (coalesced loads) */
            uint32_t bmag = 0;
            for (int k = t >> 5; k < nmeta; k += PPB_T / 32)
                for (int q = m_start[k] + lane; q < m_start[k + 1]; q += 32) {
                    const int4 y = pos[m_pb[k] + (q - m_start[k])];
                    const int32_t o0 = rel_off(y.x, Xr[0], per, bmag);
                    const int32_t o1 = rel_off(y.y, Xr[1], per, bmag);
                    const int32_t o2 = rel_off(y.z, Xr[2], per, bmag);
                    if (pass == 0) {
                        float *e = sf + (q >> 1) * 12 + (q & 1); /* SrcPair: hx.x hx.y hy.x ... lz.y */
                        float h, l;
                        split_hl(o0, h, l);
                        e[0] = -h, e[6] = -l;
                        split_hl(o1, h, l);
                        e[2] = -h, e[8] = -l;
                        split_hl(o2, h, l);
                        e[4] = -h, e[10] = -l;
                    } else {
                        float *e = sf + (q >> 2) * 12 + (q & 3); /* FarQuad: x[4] y[4] z[4] */
                        e[0] = -__int2float_rn(o0) * 2.3283064365386963e-10f;
                        e[4] = -__int2float_rn(o1) * 2.3283064365386963e-10f;
                        e[8] = -__int2float_rn(o2) * 2.3283064365386963e-10f;
                    }
                }
            /* pad to a whole pair (near) or quad (far): a source at 1e30 gives exactly zero terms */
            if (pass == 0 && t == 0 && (used & 1)) {
                float *e = sf + (used >> 1) * 12 + 1;
                e[0] = -1.0e30f;
                e[2] = e[4] = e[6] = e[8] = e[10] = 0.0f;
            }
            if (pass == 1 && t < 3 && used + t < ((used + 3) & ~3)) {
                const int q = used + t;
                float *e = sf + (q >> 2) * 12 + (q & 3);
                e[0] = -1.0e30f;
                e[4] = e[8] = 0.0f;
            }
            atomicMax(&s_bmag, bmag);
            __syncthreads();
            const int np = pass == 0 ? (used + 1) >> 1 : (used + 3) >> 2; /* pairs (near) or quads (far) */
            const uint32_t amax = s_amag, bmax = s_bmag;
            if (active) {
                /* copy `phase` takes the contiguous source pairs or quads [q0, q1) */
                const int q0 = (np * phase) / C, q1 = (np * (phase + 1)) / C;
                /* both forms give the int32-wrapped (nearest image) separation
                 * when every |a_i - b_j| < 2^31 */
                const bool fits = (unsigned long long)amax + bmax < (1ull << 31);
                if (pass == 0 && fits)
                    ppb_near_stage(P, h2, m, stage, q0, q1, A, a);
                else if (pass == 1 && fits)
                    ppb_far_stage(m, reinterpret_cast<const FarQuad *>(stage), q0, q1, ax, ay, az, a);
                else
                    ppb_wrap_stage(P, m, m_start, m_pb, nmeta, pos, phase, C, xi, per, a);
            }
            __syncthreads(); /* the stage is rewritten next */
        }
    }
    red[t][0] = (double)a.kp.s - (double)a.kp.c;
    red[t][1] = (double)a.k0.s - (double)a.k0.c;
    red[t][2] = (double)a.k1.s - (double)a.k1.c;
    red[t][3] = (double)a.k2.s - (double)a.k2.c;
    __syncthreads();
    if (t < ns) {
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int p = 0; p < C; p++)
#pragma unroll
            for (int q = 0; q < 4; q++) v[q] += red[t + p * ns][q];
        const double *fr = far + 4 * (int64_t)i;
        acc[i] = make_float4((float)(fr[0] + v[0] - P.phi_self), (float)(fr[1] + v[1]), (float)(fr[2] + v[2]),
                             (float)(fr[3] + v[3]));
    }
}
