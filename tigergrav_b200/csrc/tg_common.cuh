/*
 * tg_common.cuh -- shared device code: fixed-point positions, symmetric
 * tensor storage, Green's-function derivatives, Ewald sums and the
 * multipole/expansion contractions of the periodic gravity path.
 *
 * Storage layouts are the reference's (so node multipoles and expansions are
 * interchangeable with it):
 *   multipole (17): M, M_ab (6), M_abc (10)        tigergrav/multipole.hpp:24,58-82
 *   expansion (35): L, L_a, L_ab, L_abc, L_abcd    tigergrav/expansion.hpp:28,77-137
 * Within an order the slots enumerate sorted index tuples lexicographically.
 */
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tg {

constexpr int MP = 17;
constexpr int LP = 35;
constexpr double POS_MAX = 4294967296.0;
constexpr double POS_INV = 1.0 / 4294967296.0;
constexpr int NREAL = 305;  /* |n|^2 <= 17 (tigergrav/green.hpp:3,8-28) */
constexpr int NREAL_F32 = 123; /* |n|^2 <= 9: every n that can lie within the FP32 cut 2.1 of |X| <= sqrt(3)/2 */
constexpr int NFOUR = 123;  /* |h|^2 <= 9 */
constexpr int NFOUR_HALF = 61; /* one of each pair +-h (h != 0) */
constexpr int HS = 36;         /* row stride of the coefficient tables (16-byte rows) */
constexpr float EWALD_RCUT = 1.0e-6f;
constexpr float EWALD_PHI0 = 2.8372975f; /* r -> 0 limit (tigergrav/green.hpp:272) */

/* ---- symmetric index arithmetic (constant-folded after unrolling) ---- */
__host__ __device__ constexpr int cmin(int a, int b) { return a < b ? a : b; }
__host__ __device__ constexpr int cmax(int a, int b) { return a < b ? b : a; }
/* index of sorted pair (p<=q) among sorted pairs of {0..n-1} */
__host__ __device__ constexpr int idx2n(int p, int q, int n) { return p * n - p * (p - 1) / 2 + q - p; }
/* number of sorted pairs of {k..n-1} summed over k < p */
__host__ __device__ constexpr int off3n(int p, int n) {
    return p == 0 ? 0 : (p == 1 ? n * (n + 1) / 2 : n * (n + 1) / 2 + (n - 1) * n / 2);
}
__host__ __device__ constexpr int idx3n(int p, int q, int r, int n) { return off3n(p, n) + idx2n(q - p, r - p, n - p); }
/* number of sorted triples of {k..2} summed over k < p (n = 3) */
__host__ __device__ constexpr int off4(int p) { return p == 0 ? 0 : (p == 1 ? 10 : 14); }

__host__ __device__ constexpr int I2(int a, int b) { return idx2n(cmin(a, b), cmax(a, b), 3); }
__host__ __device__ constexpr int I3(int a, int b, int c) {
    return idx3n(cmin(a, cmin(b, c)), a + b + c - cmin(a, cmin(b, c)) - cmax(a, cmax(b, c)), cmax(a, cmax(b, c)), 3);
}
__host__ __device__ constexpr int sort4_0(int a, int b, int c, int d) { return cmin(cmin(a, b), cmin(c, d)); }
__host__ __device__ constexpr int sort4_3(int a, int b, int c, int d) { return cmax(cmax(a, b), cmax(c, d)); }
__host__ __device__ constexpr int sort4_1(int a, int b, int c, int d) {
    /* second smallest */
    return cmin(cmax(cmin(a, b), cmin(c, d)), cmin(cmax(a, b), cmax(c, d)));
}
__host__ __device__ constexpr int I4(int a, int b, int c, int d) {
    return off4(sort4_0(a, b, c, d)) +
           idx3n(sort4_1(a, b, c, d) - sort4_0(a, b, c, d),
                 (a + b + c + d - sort4_0(a, b, c, d) - sort4_1(a, b, c, d) - sort4_3(a, b, c, d)) - sort4_0(a, b, c, d),
                 sort4_3(a, b, c, d) - sort4_0(a, b, c, d), 3 - sort4_0(a, b, c, d));
}
__host__ __device__ constexpr int E0() { return 0; }
__host__ __device__ constexpr int E1(int a) { return 1 + a; }
__host__ __device__ constexpr int E2(int a, int b) { return 4 + I2(a, b); }
__host__ __device__ constexpr int E3(int a, int b, int c) { return 10 + I3(a, b, c); }
__host__ __device__ constexpr int E4(int a, int b, int c, int d) { return 20 + I4(a, b, c, d); }
__host__ __device__ constexpr int M2(int a, int b) { return 1 + I2(a, b); }
__host__ __device__ constexpr int M3(int a, int b, int c) { return 7 + I3(a, b, c); }

/* expansion_factors (tigergrav/expansion.hpp:162-182): multiplicity / k!,
 * accumulated in the working type exactly as the reference does; filled on
 * the host by init_constants(); the library is one translation unit. */
__constant__ float c_factor_f[LP];
__constant__ double c_factor_d[LP];
template <class T> __device__ __forceinline__ T factor(int i);
template <> __device__ __forceinline__ float factor<float>(int i) { return c_factor_f[i]; }
template <> __device__ __forceinline__ double factor<double>(int i) { return c_factor_d[i]; }

/* ---- fixed point (tigergrav/position.hpp:18-37) ---- */
__device__ __forceinline__ double pos2d(int32_t x) { return __dadd_rn(__dmul_rn((double)x, POS_INV), 0.5); }
__device__ __forceinline__ int32_t d2pos(double x) {
    const double y = __dadd_rn(x, -0.5);
    long long z = llround(__dmul_rn(y, POS_MAX));
    if ((double)z >= POS_MAX / 2.0) z -= (long long)POS_MAX;
    return (int32_t)(uint32_t)(unsigned long long)z;
}
/* minimum-image separation of two fixed-point coordinates, in box units:
 * (float)(int32)(X - Y) * 2^-32 (src/gravity.cpp:223) */
__device__ __forceinline__ float wrap_sep_f(int32_t X, int32_t Y) {
    return __int2float_rn((int32_t)((uint32_t)X - (uint32_t)Y)) * 2.3283064365386963e-10f;
}
__device__ __forceinline__ double wrap_sep_d(int32_t X, int32_t Y) {
    return (double)(int32_t)((uint32_t)X - (uint32_t)Y) * POS_INV;
}
/* non-periodic separation (src/gravity.cpp:228) */
__device__ __forceinline__ float free_sep_f(int32_t X, int32_t Y) {
    return __ll2float_rn((long long)X - (long long)Y) * 2.3283064365386963e-10f;
}
__device__ __forceinline__ double free_sep_d(int32_t X, int32_t Y) {
    return (double)((long long)X - (long long)Y) * POS_INV;
}
template <class T> __device__ __forceinline__ T sep(int32_t X, int32_t Y, bool periodic);
template <> __device__ __forceinline__ float sep<float>(int32_t X, int32_t Y, bool periodic) {
    return periodic ? wrap_sep_f(X, Y) : free_sep_f(X, Y);
}
template <> __device__ __forceinline__ double sep<double>(int32_t X, int32_t Y, bool periodic) {
    return periodic ? wrap_sep_d(X, Y) : free_sep_d(X, Y);
}

template <class T> __device__ __forceinline__ T wrap_sep_t(int32_t X, int32_t Y);
template <> __device__ __forceinline__ float wrap_sep_t<float>(int32_t X, int32_t Y) { return wrap_sep_f(X, Y); }
template <> __device__ __forceinline__ double wrap_sep_t<double>(int32_t X, int32_t Y) { return wrap_sep_d(X, Y); }

/* ---- per-type math ---- */
/* The hardware approximations of PTX (rsqrt / rcp / ex2 .approx) in their
 * .ftz form: subnormal inputs and results flush to zero, which spares the
 * scaling that the IEEE-subnormal forms need; every input here is a normal
 * number (r^2 >= h^2 or >= 1e-12, 1 + 0.33 x >= 1, exponents >= -26). */
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_ftz(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2_ftz(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float t_rsqrt(float x) { return rsqrt_ftz(x); }
__device__ __forceinline__ double t_rsqrt(double x) { return 1.0 / sqrt(x); }
__device__ __forceinline__ float t_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double t_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float t_rcp(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double t_rcp(double x) { return 1.0 / x; }

/* erfc(x) and exp(-x^2).  FP32: the Abramowitz & Stegun 7.1.26 rational
 * approximation that the reference uses (tigergrav/simd.hpp:676-692), with
 * expf; FP64: the double-precision erfc and exp. */
__device__ __forceinline__ float t_erfcexp(float x, float *e) {
    const float t1 = rcp_ftz(fmaf(0.3275911f, x, 1.0f));
    *e = ex2_ftz(x * x * -1.4426950408889634f); /* e^-x^2 = 2^(-x^2 log2 e) */
    const float poly = t1 * (0.254829592f + t1 * (-0.284496736f + t1 * (1.421413741f + t1 * (-1.453152027f + t1 * 1.061405429f))));
    return poly * *e;
}
__device__ __forceinline__ double t_erfcexp(double x, double *e) {
    *e = exp(-x * x);
    return erfc(x);
}

/* ---- Green's function derivatives ---- */

/* green_deriv_direct (tigergrav/green.hpp:62-117): set D from radial factors */
template <class T>
__device__ __forceinline__ void green_deriv_set(T *D, T d0, T d1, T d2, T d3, T d4, const T *dx) {
    D[E0()] = d0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        D[E1(a)] = dx[a] * d1;
#pragma unroll
        for (int b = 0; b <= a; b++) {
            const T dxadxb = dx[a] * dx[b];
            D[E2(a, b)] = dxadxb * d2;
#pragma unroll
            for (int c = 0; c <= b; c++) {
                const T dxadxbdxc = dxadxb * dx[c];
                D[E3(a, b, c)] = dxadxbdxc * d3;
#pragma unroll
                for (int d = 0; d <= c; d++) D[E4(a, b, c, d)] = dxadxbdxc * dx[d] * d4;
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        D[E2(a, a)] += d1;
        D[E3(a, a, a)] = fma(dx[a], d2, D[E3(a, a, a)]);
        D[E4(a, a, a, a)] = fma(dx[a] * dx[a], d3, D[E4(a, a, a, a)]);
        D[E4(a, a, a, a)] = fma(T(2), d2, D[E4(a, a, a, a)]);
#pragma unroll
        for (int b = 0; b <= a; b++) {
            const T dxadxb = dx[a] * dx[b];
            D[E3(a, a, b)] = fma(dx[b], d2, D[E3(a, a, b)]);
            D[E3(a, b, b)] = fma(dx[a], d2, D[E3(a, b, b)]);
            D[E4(a, a, a, b)] = fma(dxadxb, d3, D[E4(a, a, a, b)]);
            D[E4(a, b, b, b)] = fma(dxadxb, d3, D[E4(a, b, b, b)]);
            D[E4(a, a, b, b)] += d2;
#pragma unroll
            for (int c = 0; c <= b; c++) {
                D[E4(a, a, b, c)] = fma(dx[b], dx[c] * d3, D[E4(a, a, b, c)]);
                D[E4(a, b, c, c)] = fma(dxadxb, d3, D[E4(a, b, c, c)]);
                D[E4(a, b, b, c)] = fma(dx[a], dx[c] * d3, D[E4(a, b, b, c)]);
            }
        }
    }
}

/* green_deriv_ewald (tigergrav/green.hpp:119-165): accumulate into D */
template <class T, class A>
__device__ __forceinline__ void green_deriv_add(A *D, T d0, T d1, T d2, T d3, T d4, const T *dx) {
    D[E0()] += d0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        D[E1(a)] += dx[a] * d1;
        D[E2(a, a)] += d1;
        D[E3(a, a, a)] += dx[a] * d2;
        D[E4(a, a, a, a)] += dx[a] * dx[a] * d3;
        D[E4(a, a, a, a)] += T(2) * d2;
#pragma unroll
        for (int b = 0; b <= a; b++) {
            const T dxadxb = dx[a] * dx[b];
            D[E2(a, b)] += dxadxb * d2;
            D[E3(a, a, b)] += dx[b] * d2;
            D[E3(a, b, b)] += dx[a] * d2;
            D[E4(a, a, a, b)] += dxadxb * d3;
            D[E4(a, b, b, b)] += dxadxb * d3;
            D[E4(a, a, b, b)] += d2;
#pragma unroll
            for (int c = 0; c <= b; c++) {
                const T dxadxbdxc = dxadxb * dx[c];
                D[E3(a, b, c)] += dxadxbdxc * d3;
                D[E4(a, a, b, c)] += dx[b] * dx[c] * d3;
                D[E4(a, b, c, c)] += dxadxb * d3;
                D[E4(a, b, b, c)] += dx[a] * dx[c] * d3;
#pragma unroll
                for (int d = 0; d <= c; d++) D[E4(a, b, c, d)] += dxadxbdxc * dx[d] * d4;
            }
        }
    }
}

/* green_direct (tigergrav/green.hpp:167-186) */
template <class T>
__device__ __forceinline__ void green_direct(const T *dX, T *D) {
    const T r2 = dX[0] * dX[0] + dX[1] * dX[1] + dX[2] * dX[2];
    const T rinv = (r2 > T(1.0e-18)) ? t_rsqrt(r2) : T(0);
    const T r2inv = rinv * rinv;
    const T d0 = -rinv;
    const T d1 = -d0 * r2inv;
    const T d2 = T(-3) * d1 * r2inv;
    const T d3 = T(-5) * d2 * r2inv;
    const T d4 = T(-7) * d3 * r2inv;
    green_deriv_set(D, d0, d1, d2, d3, d4, dX);
}

/* Ewald tables (tigergrav/green.hpp:8-59), generated in FP64 on the device. */
struct EwaldTables {
    const float4 *real; /* NREAL lattice vectors n by increasing |n|^2 (w = |n|^2) */
    const float4 *four; /* NFOUR_HALF reciprocal vectors h, first non-zero component > 0 (w unused) */
    const float *Hf;    /* NFOUR_HALF rows of HS: 2 x periodic_parts coefficients, float */
    const double *Hd;   /* NFOUR_HALF rows of HS, double */
    const float4 *Pf;   /* NFOUR_HALF x (H0, Hx, Hy, Hz): the potential and force terms, float */
    const double2 *Pd;  /* NFOUR_HALF x 2, double */
};

/* Real-space cut of the Ewald sum.  The reference masks images at r >= 3.6
 * (tigergrav/green.hpp:220); the FP64 path keeps that.  The FP32 path stops
 * at r = 2.1 (~39 images instead of ~200): an image there adds 3e-9 to D0 and
 * 1.1e-8 to the force factor d1 (erfc(4.2) = 3e-9, exp(-17.6) times the
 * derivative polynomials) -- below the error of the reference's own erfc
 * (A&S 7.1.26, 1.5e-7 absolute) -- and its higher derivatives (d4 <= 1e-5)
 * enter forces only through multipole moments and expansion offsets of leaf
 * size. */
template <class T> __device__ __forceinline__ T ewald_rcut2();
template <> __device__ __forceinline__ float ewald_rcut2<float>() { return 4.41f; }
template <> __device__ __forceinline__ double ewald_rcut2<double>() { return 12.96; }
/* PP Ewald needs only the potential and force factors d0, d1: an image at
 * r >= 2 adds at most 8e-9 to d0 and 6e-8 to d1, so the FP32 path stops at 2
 * there (~34 images) */
template <class T> __device__ __forceinline__ T ewald_rcut2_pp() { return sizeof(T) == 4 ? T(4.0) : ewald_rcut2<T>(); }

/* Sums over the real-space images that green_ewald's derivative tensors are
 * built from (tigergrav/green.hpp:62-117 applied per image, 212-236): with
 * radial factors d0..d4 of each image at separation x,
 *   D0 = S d0,  D_a = S d1 x_a,  D_ab = S d2 x_a x_b + delta_ab S d1,
 *   D_abc = S d3 x_a x_b x_c + (delta_ab S d2 x_c + 2 perms),
 *   D_abcd = S d4 x_a x_b x_c x_d + (delta_ab S d3 x_c x_d + 5 perms)
 *            + (delta_ab delta_cd + 2 perms) S d2.
 * The pure products accumulate straight into D; the four delta sums below
 * are folded in once per evaluation by ewald_mom_finish -- the same tensor as
 * adding each image's full derivative set, at half the work per image. */
template <class T> struct EwaldMom {
    T s3[6]; /* S d3 x_a x_b, slot I2(a, b) */
    T t2[3]; /* S d2 x_a */
    T u1;    /* S d1 */
    T s2;    /* S d2 */
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int k = 0; k < 6; k++) s3[k] = T(0);
        t2[0] = t2[1] = t2[2] = T(0);
        u1 = s2 = T(0);
    }
};

/* add one image's radial factors d0..d4 at separation dx to the sums */
template <class T>
__device__ __forceinline__ void ewald_radial_add(T *D, EwaldMom<T> &m, const T *dx, T d0, T d1, T d2, T d3, T d4) {
    D[E0()] += d0;
    m.u1 += d1;
    m.s2 += d2;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        D[E1(a)] = fma(d1, dx[a], D[E1(a)]);
        m.t2[a] = fma(d2, dx[a], m.t2[a]);
        const T d2a = d2 * dx[a], d3a = d3 * dx[a], d4a = d4 * dx[a];
#pragma unroll
        for (int b = a; b < 3; b++) {
            D[E2(a, b)] = fma(d2a, dx[b], D[E2(a, b)]);
            m.s3[I2(a, b)] = fma(d3a, dx[b], m.s3[I2(a, b)]);
            const T d3ab = d3a * dx[b], d4ab = d4a * dx[b];
#pragma unroll
            for (int c = b; c < 3; c++) {
                D[E3(a, b, c)] = fma(d3ab, dx[c], D[E3(a, b, c)]);
                const T d4abc = d4ab * dx[c];
#pragma unroll
                for (int d = c; d < 3; d++) D[E4(a, b, c, d)] = fma(d4abc, dx[d], D[E4(a, b, c, d)]);
            }
        }
    }
}

/* radial factors of one real-space image, -erfc(2r)/r and (1/r d/dr)^k of it
 * (tigergrav/green.hpp:212-236), alpha = 2 */
template <class T>
__device__ __forceinline__ void ewald_image_factors(T r2, T &d0, T &d1, T &d2, T &d3, T &d4) {
    const T rinv = t_rsqrt(r2);
    const T r = r2 * rinv;
    const T r2inv = rinv * rinv;
    const T r3inv = r2inv * rinv;
    const T r5inv = r2inv * r3inv;
    const T r7inv = r2inv * r5inv;
    const T r9inv = r2inv * r7inv;
    const T r4 = r2 * r2;
    T expfac;
    const T erfc = t_erfcexp(T(2) * r, &expfac);
    const T expfactor = T(2.2567583341910252) * r * expfac; /* 4/sqrt(pi) */
    d0 = -erfc * rinv;
    d1 = (expfactor + erfc) * r3inv;
    d2 = -fma(expfactor, fma(T(8), r2, T(3)), T(3) * erfc) * r5inv;
    d3 = fma(expfactor, (T(15) + fma(T(40), r2, T(64) * r4)), T(15) * erfc) * r7inv;
    d4 = -fma(expfactor, fma(T(8) * r2, (T(35) + fma(T(56), r2, T(64) * r4)), T(105)), T(105) * erfc) * r9inv;
}

/* One real-space image (tigergrav/green.hpp:212-236) at separation dx with
 * |dx|^2 = r2 inside the cut. */
template <class T>
__device__ __forceinline__ void ewald_real_image(T *D, EwaldMom<T> &m, const T *dx, T r2) {
    T d0, d1, d2, d3, d4;
    ewald_image_factors<T>(r2, d0, d1, d2, d3, d4);
    ewald_radial_add<T>(D, m, dx, d0, d1, d2, d3, d4);
}

/* Taylor coefficients of (1/r d/dr)^k [erf(2r)/r] in u = r^2 (k = 0..4):
 * erf(2r)/r = (4/sqrt(pi)) sum_n (-4u)^n / (n! (2n+1)), and (1/r d/dr) = 2 d/du,
 * so row k holds 2^k a_{m+k} (m+k)!/m! for m = 0..13 (from the series of erf). */
constexpr int EO_TERMS = 14;
__constant__ float c_eo_f[5][EO_TERMS] = {
    {2.256758334e+00f, -3.009011112e+00f, 3.610813335e+00f, -3.438869843e+00f, 2.674676544e+00f, -1.750697374e+00f,
     9.875728779e-01f, -4.890837109e-01f, 2.157722254e-01f, -8.580415981e-02f, 3.105293403e-02f, -1.031006505e-02f,
     3.161753283e-03f, -9.007844111e-04f},
    {-6.018022225e+00f, 1.444325334e+01f, -2.063321906e+01f, 2.139741235e+01f, -1.750697374e+01f, 1.185087453e+01f,
     -6.847171953e+00f, 3.452355607e+00f, -1.544474877e+00f, 6.210586806e-01f, -2.268214312e-01f, 7.588207879e-02f,
     -2.342039469e-02f, 6.709290786e-03f},
    {2.888650668e+01f, -8.253287622e+01f, 1.283844741e+02f, -1.400557900e+02f, 1.185087453e+02f, -8.216606344e+01f,
     4.833297849e+01f, -2.471159803e+01f, 1.117905625e+01f, -4.536428623e+00f, 1.669405733e+00f, -5.620894725e-01f,
     1.744415604e-01f, -5.021146653e-02f},
    {-1.650657524e+02f, 5.135378965e+02f, -8.403347397e+02f, 9.480699628e+02f, -8.216606344e+02f, 5.799957419e+02f,
     -3.459623724e+02f, 1.788649000e+02f, -8.165571522e+01f, 3.338811467e+01f, -1.236596840e+01f, 4.186597450e+00f,
     -1.305498130e+00f, 3.773467787e-01f},
    {1.027075793e+03f, -3.361338959e+03f, 5.688419777e+03f, -6.573285075e+03f, 5.799957419e+03f, -4.151548468e+03f,
     2.504108600e+03f, -1.306491443e+03f, 6.009860640e+02f, -2.473193679e+02f, 9.210514391e+01f, -3.133195511e+01f,
     9.811016247e+00f, -2.846272845e+00f},
};

/* FP32: the n = 0 image together with the removal of the direct 1/r that
 * green_ewald's final assembly performs (tigergrav/green.hpp:265-285):
 * radial factors of erf(2r)/r.  In the reference's form the two parts cancel
 * to a factor r^(2k+1) in the k-th derivative (9 decimal digits of D4 at
 * r = 0.1, more than FP32 holds); below r = 0.6 the Taylor series above is
 * used instead, above it the difference of the closed forms loses < 35x. */
__device__ __forceinline__ void ewald_origin_add(float *D, EwaldMom<float> &m, const float *dx, float r2) {
    float c[5];
    if (r2 < 0.36f) {
#pragma unroll
        for (int k = 0; k < 5; k++) {
            float v = c_eo_f[k][EO_TERMS - 1];
#pragma unroll
            for (int q = EO_TERMS - 2; q >= 0; q--) v = fmaf(v, r2, c_eo_f[k][q]);
            c[k] = v;
        }
    } else {
        ewald_image_factors<float>(r2, c[0], c[1], c[2], c[3], c[4]);
        const float rinv = rsqrt_ftz(r2), r2inv = rinv * rinv;
        float dd = -rinv; /* direct: -1/r and its (1/r d/dr)^k: 1/r^3, -3/r^5, 15/r^7, -105/r^9 */
        c[0] -= dd;
        dd = rinv * r2inv;
        c[1] -= dd;
        dd *= -3.0f * r2inv;
        c[2] -= dd;
        dd *= -5.0f * r2inv;
        c[3] -= dd;
        dd *= -7.0f * r2inv;
        c[4] -= dd;
    }
    ewald_radial_add<float>(D, m, dx, c[0], c[1], c[2], c[3], c[4]);
}

/* fold the delta terms of the image sums into D (once per evaluation) */
template <class T>
__device__ __forceinline__ void ewald_mom_finish(T *D, const EwaldMom<T> &m) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
        D[E2(a, a)] += m.u1;
#pragma unroll
        for (int b = a; b < 3; b++)
#pragma unroll
            for (int c = b; c < 3; c++) {
                T v = T(0);
                if (a == b) v += m.t2[c];
                if (a == c) v += m.t2[b];
                if (b == c) v += m.t2[a];
                D[E3(a, b, c)] += v;
#pragma unroll
                for (int d = c; d < 3; d++) {
                    T w = T(0);
                    if (a == b) w += m.s3[I2(c, d)];
                    if (a == c) w += m.s3[I2(b, d)];
                    if (a == d) w += m.s3[I2(b, c)];
                    if (b == c) w += m.s3[I2(a, d)];
                    if (b == d) w += m.s3[I2(a, c)];
                    if (c == d) w += m.s3[I2(a, b)];
                    const int pairs = (a == b && c == d) + (a == c && b == d) + (a == d && b == c);
                    D[E4(a, b, c, d)] += w + T(pairs) * m.s2;
                }
            }
    }
}

/* Visit the lattice images n of the reference's set (|n|^2 <= 17,
 * tigergrav/green.hpp:3,8-28) with |X - n|^2 < ewald_rcut2, walking the
 * integer ranges that the cut allows instead of testing all 305 vectors.
 * The three nested ranges are flattened into one loop that advances each
 * lane to its next image, so a warp whose lanes hold different X runs the
 * image body together (about 39 images per lane in FP32, in lockstep) instead of
 * diverging at every level of the nest.  fn(dx, r2, is_origin) is called
 * once per image.  Caller guarantees |X| > 1e-6 (the reference's zmask = 1). */
template <class T, class F>
__device__ __forceinline__ void ewald_images(const T *X, F &&fn, T R2 = ewald_rcut2<T>()) {
    const T R = t_sqrt(R2);
    int nx = (int)ceil(X[0] - R) - 1;
    const int nx1 = (int)floor(X[0] + R);
    int ny = 0, ny1 = -1, nz = 0, nz1 = -1;
    T dx = T(0), dy = T(0), rx = T(0);
    for (;;) {
        /* advance to the next (nx, ny, nz) inside the cut; columns and rows
         * that the cut leaves empty are skipped here */
        nz++;
        bool done = false;
        while (nz > nz1) {
            ny++;
            while (ny > ny1) {
                nx++;
                if (nx > nx1) {
                    done = true;
                    break;
                }
                dx = X[0] - T(nx);
                rx = R2 - dx * dx;
                if (rx > T(0)) {
                    const T ry = t_sqrt(rx);
                    ny = (int)ceil(X[1] - ry);
                    ny1 = (int)floor(X[1] + ry);
                } else {
                    ny = 1;
                    ny1 = 0;
                }
            }
            if (done) break;
            dy = X[1] - T(ny);
            const T rxy = rx - dy * dy;
            if (rxy > T(0)) {
                const T rz = t_sqrt(rxy);
                nz = (int)ceil(X[2] - rz);
                nz1 = (int)floor(X[2] + rz);
            } else {
                nz = 1;
                nz1 = 0;
            }
        }
        if (done) break;
        if (nx * nx + ny * ny + nz * nz > 17) continue;
        const T d[3] = {dx, dy, X[2] - T(nz)};
        const T r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        if (!(r2 < R2)) continue;
        fn(d, r2, nx == 0 && ny == 0 && nz == 0);
    }
}

/* sin and cos of 2 pi x.  FP32: exact reduction to r = x - rint(x) in
 * [-1/2, 1/2], then the hardware sin/cos of 2 pi r (|2 pi r| <= pi, absolute
 * error ~4e-7, below the rounding of h.X itself); FP64: sincospi. */
__device__ __forceinline__ void t_sincos2pi(float x, float *s, float *c) {
    const float r = x - rintf(x);
    __sincosf(6.2831853071795865f * r, s, c);
}
__device__ __forceinline__ void t_sincos2pi(double x, double *s, double *c) { sincospi(2.0 * x, s, c); }

/* The reciprocal-space sum of green_ewald (tigergrav/green.hpp:237-264) over
 * the 61 vectors h with first non-zero component > 0: the terms of h and -h
 * are equal (H(h) is even/odd in h like cos/sin), so the table holds 2 H(h)
 * and each pair costs one term; h = 0 has H = 0. */
/* one coefficient row (HS values) with 16-byte loads */
__device__ __forceinline__ void load_row(const float *p, float *H) {
#pragma unroll
    for (int k = 0; k < HS / 4; k++) {
        const float4 v = __ldg(reinterpret_cast<const float4 *>(p) + k);
        H[4 * k] = v.x, H[4 * k + 1] = v.y, H[4 * k + 2] = v.z, H[4 * k + 3] = v.w;
    }
}
__device__ __forceinline__ void load_row(const double *p, double *H) {
#pragma unroll
    for (int k = 0; k < HS / 2; k++) {
        const double2 v = __ldg(reinterpret_cast<const double2 *>(p) + k);
        H[2 * k] = v.x, H[2 * k + 1] = v.y;
    }
}

template <class T>
__device__ __forceinline__ void ewald_four_term(T *D, const T *X, float4 h, const T *Hrow) {
    T H[HS];
    load_row(Hrow, H);
    const T hdotdx = X[0] * T(h.x) + X[1] * T(h.y) + X[2] * T(h.z);
    T si, co;
    t_sincos2pi(hdotdx, &si, &co);
    D[E0()] = fma(H[E0()], co, D[E0()]);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        D[E1(a)] = fma(H[E1(a)], si, D[E1(a)]);
#pragma unroll
        for (int b = 0; b <= a; b++) {
            D[E2(a, b)] = fma(H[E2(a, b)], co, D[E2(a, b)]);
#pragma unroll
            for (int c = 0; c <= b; c++) {
                D[E3(a, b, c)] = fma(H[E3(a, b, c)], si, D[E3(a, b, c)]);
#pragma unroll
                for (int d = 0; d <= c; d++) D[E4(a, b, c, d)] = fma(H[E4(a, b, c, d)], co, D[E4(a, b, c, d)]);
            }
        }
    }
}

/* Final assembly of green_ewald (tigergrav/green.hpp:265-285) applied to a
 * partial sum: adds pi/4 + 1/r and subtracts the direct derivatives.  Linear
 * in D, so it may be applied to one lane's partial sum of a split evaluation. */
template <class T, class A>
__device__ __forceinline__ void ewald_finish(A *D, const T *X) {
    T D1[LP];
    green_direct<T>(X, D1);
    D[E0()] += T(0.78539816339744831) - D1[E0()];
#pragma unroll
    for (int i = 1; i < LP; i++) D[i] -= D1[i];
}

/* ---- contractions (src/gravity.cpp:26-169) ---- */

/* M2L: multipole M at dX -> expansion L (src/gravity.cpp:26-90) */
template <class T, class A>
__device__ __forceinline__ void contract_M2L(A *L, const T *M, const T *D) {
    A L0 = M[0] * D[E0()];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = a; b < 3; b++) {
            L0 += M[M2(a, b)] * D[E2(a, b)] * factor<T>(E2(a, b));
#pragma unroll
            for (int c = b; c < 3; c++) L0 -= M[M3(a, b, c)] * D[E3(a, b, c)] * factor<T>(E3(a, b, c));
        }
    L[E0()] += L0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        A La = M[0] * D[E1(a)];
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int c = b; c < 3; c++) {
                La += M[M2(c, b)] * D[E3(a, b, c)] * factor<T>(E2(c, b));
#pragma unroll
                for (int d = c; d < 3; d++) La -= M[M3(b, c, d)] * D[E4(a, b, c, d)] * factor<T>(E3(b, c, d));
            }
        L[E1(a)] += La;
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = a; b < 3; b++) {
            A Lab = M[0] * D[E2(a, b)];
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int d = c; d < 3; d++) Lab += M[M2(c, d)] * D[E4(a, b, c, d)] * factor<T>(E2(c, d));
            L[E2(a, b)] += Lab;
        }
#pragma unroll
    for (int i = 10; i < LP; i++) L[i] += M[0] * D[i];
}

/* P2L: point mass m at dX -> expansion L (src/gravity.cpp:92-121) */
template <class T, class A>
__device__ __forceinline__ void contract_P2L(A *L, T m, const T *D) {
#pragma unroll
    for (int i = 0; i < LP; i++) L[i] += m * D[i];
}

/* M2P: multipole M at dX -> potential and acceleration at a particle
 * (src/gravity.cpp:123-169).  As in the reference, the potential's octupole
 * sum runs a over all three axes (lines 141-147). */
template <class T>
__device__ __forceinline__ void contract_M2P(T &phi, T *g, const T *M, const T *D) {
    T ffirst = M[0] * D[E0()];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = a; b < 3; b++) ffirst += M[M2(a, b)] * D[E2(a, b)] * factor<T>(E2(a, b));
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int c = b; c < 3; c++) ffirst -= M[M3(a, b, c)] * D[E3(a, b, c)] * factor<T>(E3(a, b, c));
    phi = ffirst;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        T ga = -(M[0] * D[E1(a)]);
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int c = b; c < 3; c++) {
                ga -= M[M2(c, b)] * D[E3(a, b, c)] * factor<T>(E2(c, b));
#pragma unroll
                for (int d = c; d < 3; d++) ga += M[M3(c, b, d)] * D[E4(a, b, c, d)] * factor<T>(E3(b, c, d));
            }
        g[a] = ga;
    }
}

/* L2L: expansion<double>::operator<<= (tigergrav/expansion.hpp:184-233) */
__device__ __forceinline__ void L2L(double *me, const double *dX) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
        me[E0()] += me[E1(a)] * dX[a];
#pragma unroll
        for (int b = 0; b <= a; b++) {
            me[E0()] += me[E2(a, b)] * dX[a] * dX[b] * c_factor_d[E2(a, b)];
#pragma unroll
            for (int c = 0; c <= b; c++) {
                me[E0()] += me[E3(a, b, c)] * dX[a] * dX[b] * dX[c] * c_factor_d[E3(a, b, c)];
#pragma unroll
                for (int d = 0; d <= c; d++)
                    me[E0()] += me[E4(a, b, c, d)] * dX[a] * dX[b] * dX[c] * dX[d] * c_factor_d[E4(a, b, c, d)];
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            me[E1(a)] += me[E2(a, b)] * dX[b];
#pragma unroll
            for (int c = 0; c <= b; c++) {
                me[E1(a)] += me[E3(a, b, c)] * dX[b] * dX[c] * c_factor_d[E2(b, c)];
#pragma unroll
                for (int d = 0; d <= c; d++) me[E1(a)] += me[E4(a, b, c, d)] * dX[b] * dX[c] * dX[d] * c_factor_d[E3(b, c, d)];
            }
        }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b <= a; b++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                me[E2(a, b)] += me[E3(a, b, c)] * dX[c];
#pragma unroll
                for (int d = 0; d <= c; d++) me[E2(a, b)] += me[E4(a, b, c, d)] * dX[c] * dX[d] * c_factor_d[E2(c, d)];
            }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b <= a; b++)
#pragma unroll
            for (int c = 0; c <= b; c++)
#pragma unroll
                for (int d = 0; d < 3; d++) me[E3(a, b, c)] += me[E4(a, b, c, d)] * dX[d];
}

/* L2P: expansion<T>::translate_L2 (tigergrav/expansion.hpp:235-269) */
template <class T>
__device__ __forceinline__ void L2P(const T *me, const T *dX, T &phi, T *g) {
    T p = me[E0()];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        p += me[E1(a)] * dX[a];
#pragma unroll
        for (int b = a; b < 3; b++) {
            p += me[E2(a, b)] * dX[a] * dX[b] * factor<T>(E2(a, b));
#pragma unroll
            for (int c = b; c < 3; c++) {
                p += me[E3(a, b, c)] * dX[a] * dX[b] * dX[c] * factor<T>(E3(a, b, c));
#pragma unroll
                for (int d = c; d < 3; d++) p += me[E4(a, b, c, d)] * dX[a] * dX[b] * dX[c] * dX[d] * factor<T>(E4(a, b, c, d));
            }
        }
    }
    phi = p;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        T ga = -me[E1(a)];
#pragma unroll
        for (int b = 0; b < 3; b++) {
            ga -= me[E2(a, b)] * dX[b];
#pragma unroll
            for (int c = b; c < 3; c++) {
                ga -= me[E3(a, b, c)] * dX[b] * dX[c] * factor<T>(E2(b, c));
#pragma unroll
                for (int d = c; d < 3; d++) ga -= me[E4(a, b, c, d)] * dX[b] * dX[c] * dX[d] * factor<T>(E3(b, c, d));
            }
        }
        g[a] = ga;
    }
}

/* M2M: multipole<float>::operator>>= (tigergrav/multipole.hpp:116-135) */
__device__ __forceinline__ void M2M(float *me, const float *Y) {
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
        for (int q = p; q < 3; q++)
#pragma unroll
            for (int l = q; l < 3; l++) {
                float m3 = me[M3(p, q, l)];
                m3 = __fadd_rn(m3, __fmul_rn(__fmul_rn(__fmul_rn(me[0], Y[p]), Y[q]), Y[l]));
                m3 = __fadd_rn(m3, __fmul_rn(me[M2(p, q)], Y[l]));
                m3 = __fadd_rn(m3, __fmul_rn(me[M2(q, l)], Y[p]));
                m3 = __fadd_rn(m3, __fmul_rn(me[M2(l, p)], Y[q]));
                me[M3(p, q, l)] = m3;
            }
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
        for (int q = p; q < 3; q++)
            me[M2(p, q)] = __fadd_rn(me[M2(p, q)], __fmul_rn(__fmul_rn(me[0], Y[p]), Y[q]));
}

/* Kahan-compensated accumulator (FP32 path) */
struct KahanF {
    float s, c;
    __device__ __forceinline__ void init() { s = 0.0f; c = 0.0f; }
    __device__ __forceinline__ void add(float x) {
        const float y = __fsub_rn(x, c);
        const float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
    __device__ __forceinline__ float value() const { return s - c; }
};

/* status flags written by kernels (never trap) */
enum : uint32_t {
    DEV_ERR_OVERFLOW_NEXT = 1u,
    DEV_ERR_OVERFLOW_LIST = 2u,
    DEV_ERR_OVERFLOW_SCRATCH = 4u,
    DEV_ERR_DEPTH = 8u,
    DEV_ERR_BADINDEX = 16u,
    DEV_ERR_SPIN = 32u,
    DEV_ERR_NONFINITE = 64u, /* a non-finite input value (velocity) */
};

} // namespace tg
