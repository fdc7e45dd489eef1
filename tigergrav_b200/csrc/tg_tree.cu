/*
 * tg_tree.cu -- tree construction and multipoles.
 *
 * The reference builds its tree by repeated passes of tree::refine
 * (src/tree.cpp:122-201): every leaf holding more than parts_per_node
 * particles is split at the midpoint of its box along the longest axis,
 * ties going to the lowest axis, so the split axis cycles x, y, z with the
 * level and a node at level L is exactly the set of particles whose 3L-bit
 * Morton prefix (x bit first) equals the node's box id (src/range.cpp:134-168).
 *
 * Here: 63-bit Morton keys from the top 21 bits of each coordinate, one radix
 * sort, then one pass per level: a node at level L with more than leaf_max
 * particles gets two children whose boundary is found by binary search for
 * key bit (62 - L) in the node's sorted range.  Nodes are numbered level by
 * level in increasing box id, so ids match the oracle's breadth-first order.
 *
 * compute_multipoles (src/tree.cpp:203-296) runs bottom-up, one launch per
 * level: leaves do COM + P2M (src/part_vect.cpp:542-635) with one warp per
 * leaf; internal nodes combine their children (COM, M2M, radius bound).
 * Centres of mass, radii and the opening radii use IEEE double operations
 * without contraction (__dadd_rn/__dmul_rn/__ddiv_rn/__dsqrt_rn), so node
 * positions and radii are bit-identical to the reference's arithmetic.
 */
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cstring>

#include "tg_solver.cuh"

namespace tg {

__device__ __forceinline__ unsigned long long spread3(unsigned int v) {
    unsigned long long x = v & 0x1fffffu; /* 21 bits */
    x = (x | (x << 32)) & 0x1f00000000ffffull;
    x = (x | (x << 16)) & 0x1f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

__global__ void k_keys(const int4 *__restrict__ pos, int64_t n, unsigned long long *__restrict__ keys,
                       int32_t *__restrict__ idx) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 p = pos[i];
    const unsigned ux = ((unsigned)p.x ^ 0x80000000u) >> 11;
    const unsigned uy = ((unsigned)p.y ^ 0x80000000u) >> 11;
    const unsigned uz = ((unsigned)p.z ^ 0x80000000u) >> 11;
    keys[i] = (spread3(ux) << 2) | (spread3(uy) << 1) | spread3(uz);
    idx[i] = (int32_t)i;
}

__global__ void k_gather(const int4 *__restrict__ pos, const float4 *__restrict__ vel, const int32_t *__restrict__ idx,
                         int64_t n, int4 *__restrict__ pos_out, float4 *__restrict__ vel_out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t j = idx[i];
    pos_out[i] = pos[j];
    vel_out[i] = vel[j];
}

__global__ void k_root(int64_t n, int32_t *pb, int32_t *pe, int32_t *child0, int32_t *parent,
                       unsigned long long *key, unsigned char *level) {
    pb[0] = 0;
    pe[0] = (int32_t)n;
    child0[0] = -1;
    parent[0] = -1;
    key[0] = 0ull;
    level[0] = 0;
}

__global__ void k_flag(int64_t first, int64_t count, const int32_t *__restrict__ pb, const int32_t *__restrict__ pe,
                       int leaf_max, int32_t *__restrict__ flag) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int64_t i = first + k;
    flag[k] = (pe[i] - pb[i] > leaf_max) ? 1 : 0;
}

__global__ void k_split(int64_t first, int64_t count, int64_t next_first, int L, const int32_t *__restrict__ flag,
                        const int32_t *__restrict__ scan, const unsigned long long *__restrict__ keys,
                        int32_t *pb, int32_t *pe, int32_t *child0, int32_t *parent, unsigned long long *nkey,
                        unsigned char *level) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int64_t i = first + k;
    if (!flag[k]) {
        child0[i] = -1;
        return;
    }
    const unsigned long long bit = 1ull << (62 - L);
    const unsigned long long target = nkey[i] | bit;
    int32_t lo = pb[i], hi = pe[i];
    const int32_t b = lo, e = hi;
    while (lo < hi) { /* first key >= target */
        const int32_t mid = lo + ((hi - lo) >> 1);
        if (keys[mid] < target) lo = mid + 1;
        else hi = mid;
    }
    const int64_t c = next_first + 2 * (int64_t)scan[k];
    child0[i] = (int32_t)c;
    pb[c] = b;
    pe[c] = lo;
    pb[c + 1] = lo;
    pe[c + 1] = e;
    parent[c] = parent[c + 1] = (int32_t)i;
    child0[c] = child0[c + 1] = -1;
    nkey[c] = nkey[i];
    nkey[c + 1] = nkey[i] | bit;
    level[c] = level[c + 1] = (unsigned char)(L + 1);
}

template <class T>
static int grow_keep(DevBuf<T> &b, size_t used, size_t need, cudaStream_t st) {
    if (b.n >= need && b.p) return TG_OK;
    DevBuf<T> nb;
    TG_TRY(ensure(nb, need * 2));
    if (used && b.p) TG_CUDA(cudaMemcpyAsync(nb.p, b.p, used * sizeof(T), cudaMemcpyDeviceToDevice, st));
    TG_CUDA(cudaStreamSynchronize(st));
    release(b);
    b = nb;
    return TG_OK;
}

static int grow_nodes(Solver &S, size_t used, size_t need, cudaStream_t st) {
    TG_TRY(grow_keep(S.nd_pb, used, need, st));
    TG_TRY(grow_keep(S.nd_pe, used, need, st));
    TG_TRY(grow_keep(S.nd_child0, used, need, st));
    TG_TRY(grow_keep(S.nd_parent, used, need, st));
    TG_TRY(grow_keep(S.nd_key, used, need, st));
    TG_TRY(grow_keep(S.nd_level, used, need, st));
    return TG_OK;
}

int tree_build(Solver &S, cudaStream_t st) {
    const int64_t n = S.n;
    if (n <= 0) return TG_ERR_STATE;
    const int TPB = 256;
    const int nb = (int)((n + TPB - 1) / TPB);
    TG_TRY(ensure(S.keys, n));
    TG_TRY(ensure(S.keys_alt, n));
    TG_TRY(ensure(S.idx, n));
    TG_TRY(ensure(S.idx_alt, n));
    TG_TRY(ensure(S.pos_alt, n));
    TG_TRY(ensure(S.vel_alt, n));
    k_keys<<<nb, TPB, 0, st>>>(S.pos.p, n, S.keys.p, S.idx.p);
    TG_TRY(launched(S));
    size_t tmp = 0;
    TG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, S.keys.p, S.keys_alt.p, S.idx.p, S.idx_alt.p, (int)n, 0, 63, st));
    TG_TRY(ensure(S.cub_tmp, tmp));
    TG_CUDA(cub::DeviceRadixSort::SortPairs(S.cub_tmp.p, tmp, S.keys.p, S.keys_alt.p, S.idx.p, S.idx_alt.p, (int)n, 0, 63,
                                            st));
    k_gather<<<nb, TPB, 0, st>>>(S.pos.p, S.vel.p, S.idx_alt.p, n, S.pos_alt.p, S.vel_alt.p);
    TG_TRY(launched(S));
    std::swap(S.pos, S.pos_alt);
    std::swap(S.vel, S.vel_alt);
    std::swap(S.keys, S.keys_alt); /* S.keys now sorted */

    /* level-by-level split */
    size_t cap_guess = (size_t)(4 * n / (S.prm.leaf_max > 0 ? S.prm.leaf_max : 1) + 1024);
    TG_TRY(grow_nodes(S, 0, cap_guess, st));
    k_root<<<1, 1, 0, st>>>(n, S.nd_pb.p, S.nd_pe.p, S.nd_child0.p, S.nd_parent.p, S.nd_key.p, S.nd_level.p);
    TG_TRY(launched(S));
    S.level_off.assign(1, 0);
    S.level_off.push_back(1);
    S.level_leaves.clear();
    int L = 0;
    for (;;) {
        const int64_t first = S.level_off[L], count = S.level_off[L + 1] - S.level_off[L];
        TG_TRY(ensure(S.nd_flag, count + 1));
        TG_TRY(ensure(S.nd_scan, count + 1));
        const int g = (int)((count + TPB - 1) / TPB);
        k_flag<<<g, TPB, 0, st>>>(first, count, S.nd_pb.p, S.nd_pe.p, S.prm.leaf_max, S.nd_flag.p);
        TG_TRY(launched(S));
        size_t stmp = 0;
        TG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, stmp, S.nd_flag.p, S.nd_scan.p, (int)count, st));
        TG_TRY(ensure(S.cub_tmp, stmp));
        TG_CUDA(cub::DeviceScan::ExclusiveSum(S.cub_tmp.p, stmp, S.nd_flag.p, S.nd_scan.p, (int)count, st));
        int32_t h2[2];
        TG_CUDA(cudaMemcpyAsync(S.h_small + 2048, S.nd_scan.p + count - 1, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                st));
        TG_CUDA(cudaMemcpyAsync(S.h_small + 2052, S.nd_flag.p + count - 1, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                st));
        TG_CUDA(cudaStreamSynchronize(st));
        std::memcpy(h2, S.h_small + 2048, sizeof(h2));
        const int64_t nsplit = (int64_t)h2[0] + h2[1];
        S.level_leaves.push_back(count - nsplit); /* nodes of this level that stay leaves (empty ones too) */
        if (nsplit == 0) break;
        if (L >= 63) return TG_ERR_DEPTH; /* children would need key bit -1 */
        const int64_t next_first = S.level_off[L + 1];
        const int64_t need = next_first + 2 * nsplit;
        TG_TRY(grow_nodes(S, (size_t)next_first, (size_t)need, st));
        k_split<<<g, TPB, 0, st>>>(first, count, next_first, L, S.nd_flag.p, S.nd_scan.p, S.keys.p, S.nd_pb.p,
                                   S.nd_pe.p, S.nd_child0.p, S.nd_parent.p, S.nd_key.p, S.nd_level.p);
        TG_TRY(launched(S));
        S.level_off.push_back(need);
        L++;
    }
    S.depth = L;
    S.nnodes = S.level_off.back();
    S.have_tree = true;
    S.fof_link = 0.0;
    S.have_multipoles = S.have_lists = S.have_forces = false;
    return TG_OK;
}

/* box_id_to_range (src/range.cpp:134-168) for the node with Morton prefix
 * `key` (prefix bits at the top of 63) at level L. */
__device__ void box_range(unsigned long long key, int L, double *mn, double *mx) {
    unsigned long long id = (L == 0) ? 1ull : ((1ull << L) | (key >> (63 - L)));
    double x[3] = {0.0, 0.0, 0.0}, dx[3] = {1.0, 1.0, 1.0};
    while (id != 1ull) {
        const double t1 = x[0], t2 = dx[0];
        x[0] = x[2];
        x[2] = x[1];
        x[1] = t1;
        dx[0] = dx[2];
        dx[2] = dx[1];
        dx[1] = t2;
        x[0] = (id & 1ull) ? __dadd_rn(__dmul_rn(0.5, x[0]), 0.5) : __dmul_rn(0.5, x[0]);
        dx[0] = __dmul_rn(dx[0], 0.5);
        id >>= 1;
    }
    for (int d = 0; d < 3; d++) {
        mn[d] = x[d];
        mx[d] = __dadd_rn(x[d], dx[d]);
    }
}

__device__ __forceinline__ double dnorm(const double *v) {
    double r = __dmul_rn(v[0], v[0]);
    r = __dadd_rn(r, __dmul_rn(v[1], v[1]));
    r = __dadd_rn(r, __dmul_rn(v[2], v[2]));
    return __dsqrt_rn(r);
}

/* range_max_span (src/range.cpp:18-24) of a fixed-point AABB */
__device__ __forceinline__ float aabb_span(const int32_t *a) {
    double s = 0.0;
    for (int d = 0; d < 3; d++) {
        const double w = __dadd_rn(pos2d(a[3 + d]), -pos2d(a[d]));
        s = __dadd_rn(s, __dmul_rn(w, w));
    }
    return __double2float_rn(__dsqrt_rn(s));
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_min_i(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_max_i(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

/* One warp per node of one level. */
__global__ void k_multipoles(int64_t first, int64_t count, float mass, const int4 *__restrict__ pos,
                             const int32_t *__restrict__ pb, const int32_t *__restrict__ pe,
                             const int32_t *__restrict__ child0, const unsigned long long *__restrict__ nkey,
                             const unsigned char *__restrict__ nlevel, MSrc *__restrict__ ms, float *__restrict__ nr,
                             float *__restrict__ nrmax, int32_t *__restrict__ aabb, double *__restrict__ prange) {
    const int lane = threadIdx.x & 31;
    const int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (k >= count) return;
    const int64_t i = first + k;
    const int32_t b = pb[i], e = pe[i];
    const int32_t cnt = e - b;
    if (cnt == 0) {
        if (lane == 0) {
            double mn[3], mx[3];
            box_range(nkey[i], nlevel[i], mn, mx);
            MSrc s;
            for (int q = 0; q < MP; q++) s.m[q] = 0.0f;
            for (int d = 0; d < 3; d++) s.x[d] = d2pos(__dmul_rn(0.5, __dadd_rn(mx[d], -mn[d])));
            ms[i] = s;
            nr[i] = 0.0f;
            nrmax[i] = 0.0f;
            for (int d = 0; d < 3; d++) {
                prange[6 * i + d] = mn[d];
                prange[6 * i + 3 + d] = mx[d];
                aabb[6 * i + d] = 0x7fffffff;
                aabb[6 * i + 3 + d] = (int32_t)0x80000000;
            }
        }
        return;
    }
    const int32_t c0 = child0[i];
    if (c0 < 0) {
        /* leaf: COM (exact double sums), P2M in float, radius, AABB */
        double s[3] = {0.0, 0.0, 0.0};
        int mn[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, mxv[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
        for (int32_t j = b + lane; j < e; j += 32) {
            const int4 p = pos[j];
            const int pp[3] = {p.x, p.y, p.z};
            for (int d = 0; d < 3; d++) {
                s[d] += pos2d(pp[d]);
                mn[d] = min(mn[d], pp[d]);
                mxv[d] = max(mxv[d], pp[d]);
            }
        }
        int32_t X[3];
        double Xd[3];
        for (int d = 0; d < 3; d++) {
            const double tot = warp_sum_d(s[d]);
            X[d] = d2pos(__ddiv_rn(tot, (double)cnt));
            Xd[d] = pos2d(X[d]);
            mn[d] = warp_min_i(mn[d]);
            mxv[d] = warp_max_i(mxv[d]);
        }
        float M[MP];
        for (int q = 0; q < MP; q++) M[q] = 0.0f;
        float r = 0.0f;
        for (int32_t j = b + lane; j < e; j += 32) {
            const int4 p = pos[j];
            const int pp[3] = {p.x, p.y, p.z};
            double dd[3];
            float dx[3];
            for (int d = 0; d < 3; d++) {
                dd[d] = __dadd_rn(pos2d(pp[d]), -Xd[d]);
                dx[d] = __double2float_rn(dd[d]);
            }
            r = fmaxf(r, __double2float_rn(dnorm(dd)));
            M[0] += mass;
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int q = 0; q <= a; q++) {
                    const float Xjk = __fmul_rn(dx[a], dx[q]);
                    M[M2(a, q)] = __fadd_rn(M[M2(a, q)], __fmul_rn(mass, Xjk));
#pragma unroll
                    for (int l = 0; l <= q; l++)
                        M[M3(a, q, l)] = __fadd_rn(M[M3(a, q, l)], __fmul_rn(__fmul_rn(mass, Xjk), dx[l]));
                }
        }
        for (int q = 0; q < MP; q++) M[q] = warp_sum_f(M[q]);
        r = warp_max_f(r);
        if (lane == 0) {
            MSrc o;
            for (int q = 0; q < MP; q++) o.m[q] = M[q];
            for (int d = 0; d < 3; d++) o.x[d] = X[d];
            ms[i] = o;
            nr[i] = r;
            int32_t a6[6] = {mn[0], mn[1], mn[2], mxv[0], mxv[1], mxv[2]};
            for (int d = 0; d < 6; d++) aabb[6 * i + d] = a6[d];
            nrmax[i] = aabb_span(a6);
            for (int d = 0; d < 3; d++) {
                prange[6 * i + d] = pos2d(mn[d]);
                prange[6 * i + 3 + d] = pos2d(mxv[d]);
            }
        }
        return;
    }
    if (lane != 0) return;
    /* internal node: combine children (src/tree.cpp:236-287) */
    const int32_t cl = c0, cr = c0 + 1;
    const int32_t Nl = pe[cl] - pb[cl], Nr = pe[cr] - pb[cr];
    const MSrc ml = ms[cl], mr = ms[cr];
    int32_t X[3];
    double Xd[3], XL[3], XR[3];
    for (int d = 0; d < 3; d++) {
        XL[d] = pos2d(ml.x[d]);
        XR[d] = pos2d(mr.x[d]);
        const double num = __dadd_rn(__dmul_rn(XL[d], (double)Nl), __dmul_rn(XR[d], (double)Nr));
        X[d] = d2pos(__ddiv_rn(num, (double)cnt));
        Xd[d] = pos2d(X[d]);
    }
    float ML[MP], MR[MP];
    for (int q = 0; q < MP; q++) {
        ML[q] = ml.m[q];
        MR[q] = mr.m[q];
    }
    double dld[3], drd[3];
    float dl[3], dr[3];
    for (int d = 0; d < 3; d++) {
        dld[d] = __dadd_rn(XL[d], -Xd[d]);
        drd[d] = __dadd_rn(XR[d], -Xd[d]);
        dl[d] = __double2float_rn(dld[d]);
        dr[d] = __double2float_rn(drd[d]);
    }
    M2M(ML, dl);
    M2M(MR, dr);
    MSrc o;
    for (int q = 0; q < MP; q++) o.m[q] = __fadd_rn(ML[q], MR[q]);
    for (int d = 0; d < 3; d++) o.x[d] = X[d];
    float r;
    const float rl = nr[cl], rr = nr[cr];
    if (Nl == 0) r = rr;
    else if (Nr == 0) r = rl;
    else r = __double2float_rn(fmax(__dadd_rn(dnorm(dld), (double)rl), __dadd_rn(dnorm(drd), (double)rr)));
    double pmn[3], pmx[3];
    for (int d = 0; d < 3; d++) {
        pmn[d] = fmin(prange[6 * cl + d], prange[6 * cr + d]);
        pmx[d] = fmax(prange[6 * cl + 3 + d], prange[6 * cr + 3 + d]);
    }
    double rmax8 = 0.0;
    for (int c = 0; c < 8; c++) {
        double dd[3];
        for (int d = 0; d < 3; d++) dd[d] = __dadd_rn(Xd[d], -(((c >> d) & 1) ? pmx[d] : pmn[d]));
        rmax8 = fmax(rmax8, dnorm(dd));
    }
    r = fminf(r, __double2float_rn(rmax8));
    ms[i] = o;
    nr[i] = r;
    int32_t a6[6];
    for (int d = 0; d < 3; d++) {
        a6[d] = min(aabb[6 * cl + d], aabb[6 * cr + d]);
        a6[3 + d] = max(aabb[6 * cl + 3 + d], aabb[6 * cr + 3 + d]);
    }
    for (int d = 0; d < 6; d++) aabb[6 * i + d] = a6[d];
    nrmax[i] = aabb_span(a6);
    for (int d = 0; d < 3; d++) {
        prange[6 * i + d] = pmn[d];
        prange[6 * i + 3 + d] = pmx[d];
    }
}

int tree_multipoles(Solver &S, cudaStream_t st) {
    if (!S.have_tree) return TG_ERR_STATE;
    const int64_t nn = S.nnodes;
    TG_TRY(ensure(S.nd_ms, nn));
    TG_TRY(ensure(S.nd_r, nn));
    TG_TRY(ensure(S.nd_rmax, nn));
    TG_TRY(ensure(S.nd_aabb, 6 * nn));
    TG_TRY(ensure(S.nd_prange, 6 * nn));
    const float mass = (float)S.prm.m;
    for (int L = S.depth; L >= 0; L--) {
        const int64_t first = S.level_off[L], count = S.level_off[L + 1] - S.level_off[L];
        if (count <= 0) continue;
        const int TPB = 128;
        const int64_t threads = count * 32;
        const int g = (int)((threads + TPB - 1) / TPB);
        k_multipoles<<<g, TPB, 0, st>>>(first, count, mass, S.pos.p, S.nd_pb.p, S.nd_pe.p, S.nd_child0.p, S.nd_key.p,
                                        S.nd_level.p, S.nd_ms.p, S.nd_r.p, S.nd_rmax.p, S.nd_aabb.p, S.nd_prange.p);
        TG_TRY(launched(S));
    }
    S.have_multipoles = true;
    S.have_lists = S.have_forces = false;
    return TG_OK;
}

} // namespace tg
