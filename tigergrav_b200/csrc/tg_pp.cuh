/*
 * tg_pp.cuh -- the packed FP32x2 pair arithmetic of PP direct
 * (gravity_PP_direct, src/gravity.cpp:171-300) in the split fixed point of
 * split_hl (tg_gravity.cu): two sources per packed instruction (FADD2 / FMUL2
 * / FFMA2, sm_100), the sink replicated in both halves.  The kernel that uses
 * it is k_pp_leaf (tg_pp2.cuh).  Included by tg_gravity.cu.
 *
 * For a pair of sources staged as negated split coordinates,
 *     dX = (hi_i - hi_j) + (lo_i - lo_j)
 * is the reference's correctly rounded FP32 separation for each of the two
 * (two exact additions, then one rounding).  1/r comes from
 * rsqrt(max(r^2, h^2)) with no branch; the caller corrects pairs with
 * r^2 <= h^2 to the reference's spline.  Sums go to plain FP32x2 partials
 * that the caller folds into Kahan-compensated totals.
 */
#pragma once

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

/* one source pair: 2 interactions in packed arithmetic */
__device__ __forceinline__ void pp_pair2(const SinkHL &A, const SrcPair &s, float h2, float &rmin, PPAcc &a) {
    float2 dx, dy, dz;
    pp_sep2(A, s, dx, dy, dz);
    const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
    rmin = fminf(rmin, fminf(r2.x, r2.y));
    const float2 rinv = make_float2(rsqrt_ftz(fmaxf(r2.x, h2)), rsqrt_ftz(fmaxf(r2.y, h2)));
    const float2 f = __fmul2_rn(__fmul2_rn(rinv, rinv), rinv);
    a.tp = __fadd2_rn(a.tp, rinv);
    a.t0 = __ffma2_rn(dx, f, a.t0);
    a.t1 = __ffma2_rn(dy, f, a.t1);
    a.t2 = __ffma2_rn(dz, f, a.t2);
}
