/*
 * tg_ewald_sep.cuh -- the reciprocal-space part of the leaf-sink Ewald
 * interactions (PP_E and PC_E, src/gravity.cpp:491-678) summed per sink leaf
 * instead of per interaction.  Included by tg_gravity.cu; FP32 path only.
 *
 * green_ewald's reciprocal sum (tigergrav/green.hpp:237-264) over the 61
 * half-space vectors h is, component by component,
 *     D_g(x) = sum_h H_h,g trig_|g|(2 pi h.x),  H_h,g = c_h s_|g| h^g,
 * with trig = cos for even and sin for odd order, s_n = -1/pi, 2, 4 pi,
 * -8 pi^2, -16 pi^3, and c_h = 2 exp(-pi^2 h^2 / 4) / h^2 (the table of
 * k_periodic_parts).  For an interaction x = x_i - X_j, trig(th_i - th_j)
 * expands into cos/sin of th_i = 2 pi h.x_i and th_j = 2 pi h.X_j, and the
 * M2P contraction of a source's multipole with D collapses per h to four
 * scalars of the source, m_0 = M0, m_2 = sum f M2 h h, m_3 = sum f M3 h h h
 * and the potential's m_3' (the reference's octupole loop, a over all axes).
 * So each sink leaf needs, per h, only the sums over its PP_E and PC_E
 * sources of m_k cos th_j and m_k sin th_j (8 numbers); every sink particle
 * then evaluates 61 terms once.  The per-interaction work keeps the
 * real-space images and the nearest-image term; the interactions, the
 * vectors h and the coefficients are the reference's, only the order of the
 * additions changes.  Exception: an interaction with r <= 1e-6 is phi0 alone
 * in the reference (green.hpp:270-273), so its reciprocal terms, which the
 * leaf sums include, are subtracted by that interaction.
 *
 * Phases are exact: h.x mod 1 is an integer sum of the fixed-point
 * coordinates modulo 2^32 (plus 1/2 per odd h component for the 0.5 offset),
 * then the hardware sin/cos of 2 pi r with r in [-1/2, 1/2).
 */
#pragma once

constexpr int EW_SEP_K = 8; /* per h: (cos, sin) sums of m_0, m_2, m_3', m_3 */

/* (cos, sin) of 2 pi h.x for fixed-point x */
__device__ __forceinline__ float2 sep_cs(int32_t x0, int32_t x1, int32_t x2, float4 h) {
    const int hx = (int)h.x, hy = (int)h.y, hz = (int)h.z;
    const long long P = (long long)hx * x0 + (long long)hy * x1 + (long long)hz * x2;
    uint32_t u = (uint32_t)(unsigned long long)P;
    if ((hx + hy + hz) & 1) u += 0x80000000u;
    const float r = (float)(int32_t)u * 2.3283064365386963e-10f; /* 2^-32: r in [-1/2, 1/2) */
    float s, c;
    __sincosf(6.2831853071795865f * r, &s, &c);
    return make_float2(c, s);
}

/* per node: (cos, sin) at its centre of mass; per leaf also the sums over its particles */
__global__ void k_ewald_sf(int64_t nn, const int32_t *__restrict__ pb, const int32_t *__restrict__ pe,
                           const int32_t *__restrict__ child0, const MSrc *__restrict__ ms,
                           const int4 *__restrict__ pos, EwaldTables E, float2 *__restrict__ nt,
                           float2 *__restrict__ sf) {
    const int lane = threadIdx.x & 31;
    const int64_t node = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (node >= nn) return;
    const int32_t b = pb[node], e = pe[node];
    const bool leaf = child0[node] < 0;
    const MSrc &s = ms[node];
    for (int t = lane; t < NFOUR_HALF; t += 32) {
        const float4 h = __ldg(&E.four[t]);
        float2 cs = make_float2(0.0f, 0.0f), acc = make_float2(0.0f, 0.0f);
        if (e > b) cs = sep_cs(s.x[0], s.x[1], s.x[2], h);
        if (leaf)
            for (int32_t j = b; j < e; j++) {
                const int4 p = pos[j];
                const float2 q = sep_cs(p.x, p.y, p.z, h);
                acc.x += q.x;
                acc.y += q.y;
            }
        nt[node * NFOUR_HALF + t] = cs;
        sf[node * NFOUR_HALF + t] = acc;
    }
}

/* monomial weights of h for m_2, m_3 and m_3' (the M2P contraction's loops, tg_common.cuh) */
struct SepQ {
    float q2[6], q3[10], q3p[10];
};
__device__ __forceinline__ void sep_q(float4 hv, SepQ &Q) {
    const float h[3] = {hv.x, hv.y, hv.z};
#pragma unroll
    for (int i = 0; i < 10; i++) Q.q3[i] = Q.q3p[i] = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = a; b < 3; b++) {
            Q.q2[I2(a, b)] = factor<float>(E2(a, b)) * h[a] * h[b];
#pragma unroll
            for (int c = b; c < 3; c++) Q.q3[I3(a, b, c)] = factor<float>(E3(a, b, c)) * h[a] * h[b] * h[c];
        }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int c = b; c < 3; c++) Q.q3p[I3(a, b, c)] += factor<float>(E3(a, b, c)) * h[a] * h[b] * h[c];
}

/* the reciprocal-only sums of one PP_E pair: (sum H0 cos, -sum H sin) */
__device__ __forceinline__ void pp_ewald_recip(const EwaldTables &E, const float *dX, float &ph, float *g) {
    ph = 0.0f;
    g[0] = g[1] = g[2] = 0.0f;
    for (int t = 0; t < NFOUR_HALF; t++) {
        const float4 h = __ldg(&E.four[t]);
        float s, c;
        t_sincos2pi(dX[0] * h.x + dX[1] * h.y + dX[2] * h.z, &s, &c);
        const float4 q = __ldg(&E.Pf[t]);
        ph += q.x * c;
        g[0] -= q.y * s;
        g[1] -= q.z * s;
        g[2] -= q.w * s;
    }
}

/*
 * Real-space images in lockstep.  The sinks of one leaf and the particles of
 * one source leaf (or one source node's centre) lie within a few leaf widths
 * of each other, so the lattice vectors that any of their pairs needs are
 * those within R + rho of the separation of the two boxes' centres (rho: the
 * largest deviation of a pair's separation from it).  A block lists that set
 * once per source in lexicographic order (ew_image_set), and every thread
 * then runs the same counted loop over it, testing its own pair's cut
 * |X - n|^2 < R^2 per image: the lanes of a warp stay together, where the
 * per-thread walk of ewald_images ran a different number of images per lane
 * and spent square roots and conversions on its ranges.  The images visited,
 * their order and their arithmetic (d = X - n in FP32) are those of
 * ewald_images.  A pair whose nearest image wraps differently from the
 * centres' (the centres' separation near +-1/2) shifts the list by its wrap k:
 * n = m - k.  The |n|^2 <= 17 limit of the reference's lattice never binds in
 * FP32: |n| <= |X| + R < sqrt(3)/2 + 2.1, so |n|^2 <= 8.
 */
constexpr int EW_IMG_CAP = 512; /* >= the lattice points within 3.84 + sqrt(3)/2 of any centre (436) */

/* all 64 threads of the block: the lattice vectors m with |c - m| < rr in
 * lexicographic order into img, and their count.  rr < 3.84 (two boxes of at
 * most unit width: rho <= sqrt(3)), so at most 9 x 9 columns (nx, ny). */
__device__ __forceinline__ int ew_image_set(const float *c, float rr, float4 *img, int *s_tmp, int &s0) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int x0 = (int)floorf(c[0] - rr), y0 = (int)floorf(c[1] - rr);
    const int nyr = (int)floorf(c[1] + rr) - y0 + 1;
    const int ncol = ((int)floorf(c[0] + rr) - x0 + 1) * nyr;
    int total = 0;
    for (int c0 = 0; c0 < ncol; c0 += 64) { /* block-uniform; column order = lexicographic (nx, ny) */
        const int col = c0 + tid;
        int ix = 0, iy = 0, z0 = 0, cnt = 0;
        if (col < ncol) {
            ix = x0 + col / nyr;
            iy = y0 + col % nyr;
            const float dx = c[0] - (float)ix, dy = c[1] - (float)iy;
            const float rz2 = rr * rr - dx * dx - dy * dy;
            if (rz2 > 0.0f) {
                const float rz = sqrtf(rz2);
                z0 = (int)ceilf(c[2] - rz);
                cnt = max(0, (int)floorf(c[2] + rz) - z0 + 1);
            }
        }
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) s_tmp[w] = incl;
        __syncthreads();
        const int base = total + (w ? s_tmp[0] : 0) + incl - cnt;
        for (int q = 0; q < cnt; q++)
            if (base + q < EW_IMG_CAP) img[base + q] = make_float4((float)ix, (float)iy, (float)(z0 + q), 0.0f);
        if (ix == 0 && iy == 0 && z0 <= 0 && 0 < z0 + cnt) s_tmp[2] = base - z0; /* m = 0: always listed */
        total += s_tmp[0] + s_tmp[1];
        __syncthreads();
    }
    s0 = s_tmp[2];
    return min(total, EW_IMG_CAP);
}

/* the geometry of one (sink box, source) pairing for ew_image_set: centre
 * separation c (box units), the radius rr of the set for a cut R, and whether
 * any pair can wrap differently from the centres.  Boxes: fixed-point
 * min / max per axis (a source point has min = max). */
struct EwPairing {
    int32_t a[3], b[3]; /* the sink box's and the source's centres, fixed point */
    int32_t C[3];       /* a - b wrapped */
    float c[3];
    float rr;
    bool wrap;
};
__device__ __forceinline__ void ew_pairing(const int32_t *sink_lo, const int32_t *sink_hi, const int32_t *src_lo,
                                           const int32_t *src_hi, float R, EwPairing &Q) {
    float e2 = 0.0f;
    Q.wrap = false;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        Q.a[d] = (int32_t)(((long long)sink_lo[d] + sink_hi[d]) >> 1);
        Q.b[d] = (int32_t)(((long long)src_lo[d] + src_hi[d]) >> 1);
        Q.C[d] = (int32_t)((uint32_t)Q.a[d] - (uint32_t)Q.b[d]);
        Q.c[d] = (float)Q.C[d] * 2.3283064365386963e-10f;
        /* |x - a| + |y - b| <= ext over the two boxes, fixed point */
        const long long ext = (((long long)sink_hi[d] - sink_lo[d]) >> 1) + (((long long)src_hi[d] - src_lo[d]) >> 1) + 2;
        const float ef = (float)ext * 2.3283064365386963e-10f;
        e2 += ef * ef;
        const long long Cabs = Q.C[d] < 0 ? -(long long)Q.C[d] : (long long)Q.C[d];
        if (Cabs + ext >= (1LL << 31)) Q.wrap = true;
    }
    Q.rr = R + sqrtf(e2) * 1.001f + 1.0e-3f;
}
/* a pair's wrap k (n = m - k) on one axis: x - y as the centres see it minus
 * its minimum image, in units of the box */
__device__ __forceinline__ float ew_wrap_k(int32_t C, int32_t x, int32_t ca, int32_t y, int32_t cb) {
    const long long D = (long long)C + ((long long)x - ca) - ((long long)y - cb);
    const long long dxi = (long long)(int32_t)((uint32_t)x - (uint32_t)y);
    return (float)((D - dxi) >> 32);
}

/* image visitors for the Ewald sums below: the per-thread walk, or a shared list */
struct ImgWalk {
    template <class F> __device__ __forceinline__ void operator()(const float *X, F &&fn, float R2) const {
        ewald_images<float>(X, fn, R2);
    }
};
struct ImgList {
    const float4 *img;
    int n, s0;  /* s0: the index of m = 0 */
    bool wrap;  /* block-uniform: some pair of the pairing wraps differently from the centres */
    float k0, k1, k2;
    template <class F> __device__ __forceinline__ void operator()(const float *X, F &&fn, float R2) const {
        if (!wrap) { /* k = 0 for every pair: n = m, the origin at s0 for all lanes */
            for (int s = 0; s < n; s++) {
                const float4 m = img[s];
                const float d[3] = {X[0] - m.x, X[1] - m.y, X[2] - m.z};
                const float r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                if (s == s0) fn(d, r2, true); /* |X| < R: the origin is always inside the cut */
                else if (r2 < R2) fn(d, r2, false);
            }
            return;
        }
        for (int s = 0; s < n; s++) {
            const float4 m = img[s];
            const float n0 = m.x - k0, n1 = m.y - k1, n2 = m.z - k2;
            const float d[3] = {X[0] - n0, X[1] - n1, X[2] - n2};
            const float r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (!(r2 < R2)) continue;
            fn(d, r2, n0 == 0.0f && n1 == 0.0f && n2 == 0.0f);
        }
    }
};

/* PP_E pair without its reciprocal terms (those come from the leaf sums) */
template <class V = ImgWalk>
__device__ __forceinline__ void pp_ewald_pair_sep(const EwaldTables &E, const float *dX0, float &phi, float *g,
                                                  const V &images = V()) {
    const float r2 = dX0[0] * dX0[0] + dX0[1] * dX0[1] + dX0[2] * dX0[2];
    if (!(r2 > 1.0e-12f)) { /* phi0 alone: take back what the leaf sums add for this pair */
        float ph, gr[3];
        pp_ewald_recip(E, dX0, ph, gr);
        phi = EWALD_PHI0 - ph;
        for (int d = 0; d < 3; d++) g[d] = -gr[d];
        return;
    }
    float ph = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
    images(dX0, [&](const float *d, float rr2, bool origin) {
        if (origin) return;
        const float rinv = t_rsqrt(rr2);
        const float r = rr2 * rinv;
        float expfac;
        const float erfc = t_erfcexp(2.0f * r, &expfac);
        const float d0 = -erfc * rinv;
        const float expfactor = 2.2567583341910252f * r * expfac;
        const float d1 = (expfactor + erfc) * rinv * rinv * rinv;
        ph += d0;
        gx -= d[0] * d1;
        gy -= d[1] * d1;
        gz -= d[2] * d1;
    }, ewald_rcut2_pp<float>());
    const float rinv = t_rsqrt(r2);
    float p0, f0;
    ewald_nearest<float>(r2 * rinv, rinv, p0, f0);
    phi = ph + (0.78539816339744831f + p0);
    g[0] = gx + dX0[0] * f0;
    g[1] = gy + dX0[1] * f0;
    g[2] = gz + dX0[2] * f0;
}

/* green_ewald without its reciprocal terms (FP32) */
template <class V = ImgWalk>
__device__ __forceinline__ void green_ewald_sep(const EwaldTables &E, const float *X, float *D, const V &images = V()) {
#pragma unroll
    for (int k = 0; k < LP; k++) D[k] = 0.0f;
    const float r2 = X[0] * X[0] + X[1] * X[1] + X[2] * X[2];
    if (!(r2 > 1.0e-12f)) { /* phi0 alone, minus the reciprocal terms the leaf sums add */
        for (int t = 0; t < NFOUR_HALF; t++) ewald_four_term<float>(D, X, __ldg(&E.four[t]), E.Hf + HS * t);
#pragma unroll
        for (int k = 0; k < LP; k++) D[k] = -D[k];
        D[E0()] += EWALD_PHI0;
        return;
    }
    EwaldMom<float> mom;
    mom.init();
    images(X, [&](const float *d, float rr2, bool origin) {
        if (origin) ewald_origin_add(D, mom, d, rr2);
        else ewald_real_image<float>(D, mom, d, rr2);
    }, ewald_rcut2<float>());
    ewald_mom_finish<float>(D, mom);
    D[E0()] += 0.78539816339744831f; /* pi/4 (tigergrav/green.hpp:270) */
}

/*
 * The reciprocal part at one sink particle from its leaf's sums T[h][8]
 * (double): with E_n(A, B) = cos th_i A + sin th_i B (n even) or
 * sin th_i A - cos th_i B (n odd),
 *   phi += sum_h c_h (s0 E0(m0) + s2 E2(m2) - s3 E3(m3'))
 *   g_a += sum_h c_h h_a (-s1 E1(m0) - s3 E3(m2) + s4 E4(m3))
 * (contract_M2P with D's reciprocal terms; a particle source has m0 = m).
 */
/* c_h as the coefficient table has it: float c0, doubled for -h */
__device__ __forceinline__ double sep_ct(float4 hv) {
    const double pi = 3.141592653589793;
    const double h2 = (double)hv.x * hv.x + (double)hv.y * hv.y + (double)hv.z * hv.z;
    const double c0 = 1.0 / h2 * exp(-pi * pi * h2 / 4.0);
    return 2.0 * (double)(float)c0;
}

__device__ __forceinline__ void sep_eval(const EwaldTables &E, const double *T, const double *ctab, int32_t x0,
                                         int32_t x1, int32_t x2, double &phi, double *g) {
    const double pi = 3.141592653589793;
    const double s0 = -1.0 / pi, s1 = 2.0, s2 = 4.0 * pi, s3 = -8.0 * pi * pi, s4 = -16.0 * pi * pi * pi;
    double ph = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    for (int t = 0; t < NFOUR_HALF; t++) {
        const float4 hv = __ldg(&E.four[t]);
        const double ct = ctab[t];
        const float2 cs = sep_cs(x0, x1, x2, hv);
        const double C = cs.x, S = cs.y;
        const double *A = T + EW_SEP_K * t;
        const double ev0 = C * A[0] + S * A[1], od0 = S * A[0] - C * A[1];
        const double ev2 = C * A[2] + S * A[3], od2 = S * A[2] - C * A[3];
        const double od3p = S * A[4] - C * A[5];
        const double ev3 = C * A[6] + S * A[7];
        ph += ct * (s0 * ev0 + s2 * ev2 - s3 * od3p);
        const double w = ct * (-s1 * od0 - s3 * od2 + s4 * ev3);
        gx += w * hv.x;
        gy += w * hv.y;
        gz += w * hv.z;
    }
    phi += ph;
    g[0] += gx;
    g[1] += gy;
    g[2] += gz;
}
