/*
 * tg_fof.cu -- friends-of-friends groups on the tree and their catalogue
 * (tree::find_groups, src/tree.cpp:637-759; part_vect_find_groups,
 * src/part_vect.cpp:85-124; groups_add_particle1/2 and groups_finish1/2,
 * src/groups.cpp:124-226).
 *
 * Friends: two particles whose squared fixed-point separation, taken as the
 * int32 difference of their coordinates (the nearest periodic image), is below
 * L2 = Lint^2 and non-zero, with Lint = (uint64)(l N^(-1/3) (2^32 - 1)) and l
 * the linking length in mean spacings -- the reference's test
 * (src/part_vect.cpp:87-104).  A group is a connected component of the
 * friend graph (the fixed point of the reference's min-label propagation);
 * a particle without friends belongs to none (DEFAULT_GROUP).  Without the
 * periodic box the separation is the plain int64 difference.
 *
 * GPU form:
 *   k_fof_pairs   one thread per leaf walks the tree with a private stack
 *                 and keeps each leaf pair (a <= b) whose particle AABBs are
 *                 closer than Lint (per-axis gap, periodic when the box is;
 *                 exact in fixed point, so no friend pair is lost);
 *   k_fof_link    one warp per leaf pair tests its particle pairs and joins
 *                 friends in a lock-free union-find: parents only ever point
 *                 to smaller sorted indices, roots are hooked with atomicCAS;
 *   k_fof_roots   the root of every particle (a read-only walk up the
 *                 parents), and at each root the smallest caller index of its
 *                 group -- the group id reported (the reference labels by its
 *                 own storage order).
 * Catalogue: members sorted by root (CUB radix sort), one block per group sums
 * the offsets from the root particle (nearest image) and the velocities in a
 * fixed order, then radii a |x - centre|, velocity dispersion and the median
 * radius (a radix select inside the block).
 */
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cub/cub.cuh>

namespace tg {

constexpr int FOF_STACK = 128;
constexpr int FOF_TPB = 64; /* threads per group in the catalogue (most groups have 2-3 members) */

__global__ void k_fof_init(int64_t n, int32_t *P, int64_t *__restrict__ gmin, uint8_t *__restrict__ has_friend) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    P[i] = (int32_t)i;
    gmin[i] = 0x7fffffffffffffffll;
    has_friend[i] = 0;
}

__global__ void k_fof_leaves(int64_t nn, const int32_t *__restrict__ pb, const int32_t *__restrict__ pe,
                             const int32_t *__restrict__ child0, int32_t *__restrict__ leaves,
                             unsigned long long *__restrict__ cnt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    if (child0[i] < 0 && pe[i] > pb[i]) leaves[atomicAdd(cnt, 1ull)] = (int32_t)i;
}

/* squared AABB gap of two nodes in fixed point, or ~0 when some axis gap alone is >= Lint */
__device__ __forceinline__ unsigned long long fof_gap2(const int32_t *A, const int32_t *B, long long Lint,
                                                       int periodic) {
    unsigned long long s = 0ull;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const long long la = A[d], ha = A[3 + d], lb = B[d], hb = B[3 + d];
        long long g = max(0ll, max(lb - ha, la - hb));
        if (periodic && g > 0) {
            const long long wrap = 4294967296ll - (max(ha, hb) - min(la, lb));
            g = min(g, max(wrap, 0ll));
        }
        if (g >= Lint) return ~0ull;
        s += (unsigned long long)(g * g);
    }
    return s;
}

/* candidate leaf pairs (a <= b by node id) that may hold a pair of friends */
__global__ void k_fof_pairs(int32_t nleaves, const int32_t *__restrict__ leaves, const int32_t *__restrict__ pb,
                            const int32_t *__restrict__ pe, const int32_t *__restrict__ child0,
                            const int32_t *__restrict__ aabb, long long Lint, unsigned long long L2, int periodic,
                            int2 *__restrict__ pairs, unsigned long long cap, unsigned long long *__restrict__ cnt,
                            uint32_t *__restrict__ err) {
    const int32_t li = blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= nleaves) return;
    const int32_t a = leaves[li];
    int32_t A[6];
    for (int d = 0; d < 6; d++) A[d] = aabb[6 * a + d];
    int32_t stack[FOF_STACK];
    int top = 0;
    stack[top++] = 0;
    while (top > 0) {
        const int32_t b = stack[--top];
        if (pe[b] == pb[b]) continue;
        int32_t B[6];
        for (int d = 0; d < 6; d++) B[d] = aabb[6 * b + d];
        if (fof_gap2(A, B, Lint, periodic) >= L2) continue;
        const int32_t c = child0[b];
        if (c < 0) {
            if (b >= a) {
                const unsigned long long k = atomicAdd(cnt, 1ull);
                if (k < cap) pairs[k] = make_int2(a, b);
            }
            continue;
        }
        if (top + 2 > FOF_STACK) {
            atomicOr(err, 2u);
            continue;
        }
        stack[top++] = c;
        stack[top++] = c + 1;
    }
}

/* root of x; parents are read through volatile loads because other warps hook roots concurrently */
__device__ __forceinline__ int32_t fof_find(int32_t *P, int32_t x) {
    volatile int32_t *V = P;
    int32_t p = V[x];
    while (p != x) { /* path halving: every write points further towards the root */
        const int32_t g = V[p];
        if (g != p) V[x] = g;
        x = p;
        p = V[x];
    }
    return x;
}

__device__ void fof_union(int32_t *P, int32_t a, int32_t b, int32_t max_tries, uint32_t *err) {
    for (int it = 0; it < max_tries; it++) {
        a = fof_find(P, a);
        b = fof_find(P, b);
        if (a == b) return;
        if (a > b) {
            const int32_t t = a;
            a = b;
            b = t;
        }
        /* hook the larger root under the smaller one, if it is still a root */
        if (atomicCAS(&P[b], b, a) == b) return;
    }
    atomicOr(err, 4u);
}

__device__ __forceinline__ unsigned long long fof_d2(int4 p, int4 q, int periodic) {
    long long dx, dy, dz;
    if (periodic) { /* the reference's int32 difference: nearest image */
        dx = (int32_t)((uint32_t)p.x - (uint32_t)q.x);
        dy = (int32_t)((uint32_t)p.y - (uint32_t)q.y);
        dz = (int32_t)((uint32_t)p.z - (uint32_t)q.z);
    } else { /* |d| >= 2^31 already means d2 >= 2^62 > L2: clamp so the sum cannot wrap */
        dx = min(llabs((long long)p.x - q.x), 2147483648ll);
        dy = min(llabs((long long)p.y - q.y), 2147483648ll);
        dz = min(llabs((long long)p.z - q.z), 2147483648ll);
    }
    return (unsigned long long)(dx * dx) + (unsigned long long)(dy * dy) + (unsigned long long)(dz * dz);
}

/* one warp per candidate leaf pair: join every pair of friends */
__global__ void k_fof_link(int64_t npairs, const int2 *__restrict__ pairs, const int32_t *__restrict__ pb,
                           const int32_t *__restrict__ pe, const int4 *__restrict__ pos, unsigned long long L2,
                           int periodic, int32_t *P, uint8_t *__restrict__ has_friend, int32_t max_tries,
                           uint32_t *__restrict__ err) {
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= npairs) return;
    const int2 pr = pairs[w];
    const int32_t a0 = pb[pr.x], a1 = pe[pr.x], b0 = pb[pr.y], b1 = pe[pr.y];
    const bool self = pr.x == pr.y;
    for (int32_t i = a0 + lane; i < a1; i += 32) {
        const int4 xi = pos[i];
        bool fi = false;
        for (int32_t j = self ? i + 1 : b0; j < b1; j++) {
            const unsigned long long d2 = fof_d2(xi, pos[j], periodic);
            if (d2 < L2 && d2 != 0ull) {
                fi = true;
                has_friend[j] = 1;
                fof_union(P, i, j, max_tries, err);
            }
        }
        if (fi) has_friend[i] = 1;
    }
}

/* root of every particle (into R), and at each root the smallest caller index of its group.
 * P is only read here: path compression while other threads take R from the
 * same paths could leave a particle pointing at an inner node. */
__global__ void k_fof_roots(int64_t n, const int32_t *__restrict__ P, const int4 *__restrict__ pos,
                            int32_t *__restrict__ R, int64_t *__restrict__ gmin) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t x = (int32_t)i, p = P[x];
    while (p != x) { /* parents strictly decrease: ends within n steps */
        x = p;
        p = P[x];
    }
    R[i] = x;
    atomicMin((unsigned long long *)&gmin[x], (unsigned long long)pos[i].w);
}

/* group id per caller index (-1: no friend); sort keys for the catalogue; group count */
__global__ void k_fof_out(int64_t n, const int32_t *__restrict__ R, const int4 *__restrict__ pos,
                          const int64_t *__restrict__ gmin, const uint8_t *__restrict__ has_friend,
                          int64_t *__restrict__ group, int32_t *__restrict__ key, int32_t *__restrict__ member,
                          unsigned long long *__restrict__ cnt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool f = has_friend[i] != 0;
    const int32_t r = R[i];
    group[pos[i].w] = f ? gmin[r] : -1;
    key[i] = f ? r : 0x7fffffff;
    member[i] = (int32_t)i;
    if (f && r == (int32_t)i) atomicAdd(cnt, 1ull);
}

/*
 * One block per group: centre = root position + mean nearest-image offset
 * (wrapped into [0,1)), mean velocity / a, then per member the radius
 * a |nearest image (x - centre)| (src/groups.cpp:184-190, as float), its
 * maximum, the velocity dispersion sqrt(mean (v/a - <v/a>)^2) per axis, and
 * the median radius, element N/2 of the sorted radii (src/groups.cpp:217-221),
 * by a radix select over the float bit patterns (radii are >= 0, so their
 * bits order like their values): four 8-bit histogram passes in shared
 * memory.  All sums run in a fixed order: deterministic.
 * stats per group (13 doubles): x[3], v[3], dv[3], rmax, N, id, rc
 */
__global__ void __launch_bounds__(FOF_TPB) k_group_stats(int64_t n, const int32_t *__restrict__ roots,
                                                         const int32_t *__restrict__ off,
                                                         const int32_t *__restrict__ cnt, const int32_t *__restrict__ member,
                                                         const int4 *__restrict__ pos, const float4 *__restrict__ vel,
                                                         const int64_t *__restrict__ gmin, double a, int periodic,
                                                         float *radii, double *__restrict__ stats,
                                                         uint32_t *__restrict__ err) {
    const int g = blockIdx.x;
    const int32_t b = off[g], N = cnt[g];
    const int32_t root = roots[g];
    if (b < 0 || N <= 0 || (int64_t)b + N > n || root < 0 || root >= n) { /* cannot happen: checked, not trusted */
        if (threadIdx.x == 0) atomicOr(err, 16u);
        return;
    }
    const int4 anchor = pos[root];
    __shared__ double red[6][FOF_TPB];
    __shared__ double cen[6];
    __shared__ unsigned int hist[256];
    __shared__ unsigned int sel_prefix, sel_k;
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int32_t j = threadIdx.x; j < N; j += FOF_TPB) {
        const int32_t i = member[b + j];
        const int4 p = pos[i];
        const float4 v = vel[i];
        const int32_t q[3] = {(int32_t)((uint32_t)p.x - (uint32_t)anchor.x), (int32_t)((uint32_t)p.y - (uint32_t)anchor.y),
                              (int32_t)((uint32_t)p.z - (uint32_t)anchor.z)};
        const long long qd[3] = {(long long)p.x - anchor.x, (long long)p.y - anchor.y, (long long)p.z - anchor.z};
        for (int d = 0; d < 3; d++) s[d] += periodic ? (double)q[d] : (double)qd[d];
        s[3] += v.x;
        s[4] += v.y;
        s[5] += v.z;
    }
    for (int k = 0; k < 6; k++) red[k][threadIdx.x] = s[k];
    __syncthreads();
    for (int h = FOF_TPB / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            for (int k = 0; k < 6; k++) red[k][threadIdx.x] += red[k][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int32_t ax[3] = {anchor.x, anchor.y, anchor.z};
        for (int d = 0; d < 3; d++) {
            double c = pos2d(ax[d]) + red[d][0] / (4294967296.0 * N);
            if (periodic) c -= floor(c);
            cen[d] = c;
            cen[3 + d] = red[3 + d][0] / N / a;
        }
        sel_prefix = 0u;
        sel_k = (unsigned int)(N / 2);
    }
    __syncthreads();
    for (int k = 0; k < 4; k++) s[k] = 0.0;
    for (int32_t j = threadIdx.x; j < N; j += FOF_TPB) {
        const int32_t i = member[b + j];
        const int4 p = pos[i];
        const float4 v = vel[i];
        const int32_t px[3] = {p.x, p.y, p.z};
        const float pv[3] = {v.x, v.y, v.z};
        double r2 = 0.0;
        for (int d = 0; d < 3; d++) {
            double dx = fabs(pos2d(px[d]) - cen[d]);
            if (periodic) dx = fmin(dx, 1.0 - dx);
            r2 += dx * dx;
            const double dv = pv[d] / a - cen[3 + d];
            s[d] += dv * dv;
        }
        const float r = (float)(a * sqrt(r2));
        radii[b + j] = r;
        s[3] = fmax(s[3], (double)r);
    }
    __syncthreads(); /* radii[] complete and red[] free */
    for (int k = 0; k < 4; k++) red[k][threadIdx.x] = s[k];
    __syncthreads();
    for (int h = FOF_TPB / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            for (int k = 0; k < 3; k++) red[k][threadIdx.x] += red[k][threadIdx.x + h];
            red[3][threadIdx.x] = fmax(red[3][threadIdx.x], red[3][threadIdx.x + h]);
        }
        __syncthreads();
    }
    /* element N/2 of the sorted radii: radix select, 8 bits a pass from the top */
    unsigned int mask = 0u;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int q = threadIdx.x; q < 256; q += FOF_TPB) hist[q] = 0u;
        __syncthreads();
        const unsigned int pre = sel_prefix;
        for (int32_t j = threadIdx.x; j < N; j += FOF_TPB) {
            const unsigned int u = __float_as_uint(radii[b + j]);
            if ((u & mask) == pre) atomicAdd(&hist[(u >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned int k = sel_k, c = 0u;
            int bin = 0;
            for (; bin < 255; bin++) {
                if (c + hist[bin] > k) break;
                c += hist[bin];
            }
            sel_k = k - c;
            sel_prefix = pre | ((unsigned int)bin << shift);
        }
        mask |= 255u << shift;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double *o = stats + 13 * (int64_t)g;
        for (int d = 0; d < 3; d++) {
            o[d] = cen[d];
            o[3 + d] = cen[3 + d];
            o[6 + d] = sqrt(red[d][0] / N);
        }
        o[9] = red[3][0];
        o[10] = N;
        o[11] = (double)gmin[root];
        o[12] = (double)__uint_as_float(sel_prefix);
    }
}

/*
 * Friends-of-friends on the current tree.  group_dev (device, n int64, caller
 * order) receives the group ids; *ngroups the number of groups.  Leaves the
 * sorted members and per-group runs in the FoF buffers for fof_catalog.
 */
static int fof_run(Solver &S, double link_len, int64_t *group_dev, int64_t *ngroups, cudaStream_t st) {
    const int64_t n = S.n, nn = S.nnodes;
    const double frac = link_len * std::pow((double)n, -1.0 / 3.0);
    if (!(frac > 0.0) || !(frac < 0.5)) return TG_ERR_ARG;
    const long long Lint = (long long)(unsigned long long)(frac * 4294967295.0); /* src/part_vect.cpp:87 */
    const unsigned long long L2 = (unsigned long long)Lint * (unsigned long long)Lint;
    const int periodic = S.prm.ewald ? 1 : 0;
    TG_TRY(ensure(S.fof_P, n));
    TG_TRY(ensure(S.fof_gmin, n));
    TG_TRY(ensure(S.fof_has, n));
    TG_TRY(ensure(S.fof_leaves, nn));
    const int gn = (int)((n + 255) / 256);
    k_fof_init<<<gn, 256, 0, st>>>(n, S.fof_P.p, S.fof_gmin.p, S.fof_has.p);
    TG_TRY(launched(S));
    TG_CUDA(cudaMemsetAsync(S.dev_cnt.p, 0, 16 * sizeof(unsigned long long), st));
    TG_CUDA(cudaMemsetAsync(S.dev_err.p, 0, sizeof(uint32_t), st));
    k_fof_leaves<<<(int)((nn + 255) / 256), 256, 0, st>>>(nn, S.nd_pb.p, S.nd_pe.p, S.nd_child0.p, S.fof_leaves.p,
                                                         S.dev_cnt.p);
    TG_TRY(launched(S));
    TG_CUDA(cudaMemcpyAsync(S.h_cnt, S.dev_cnt.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    const int32_t nleaves = (int32_t)S.h_cnt[0];
    /* candidate pairs; grow and repeat when the first guess was short */
    unsigned long long cap = S.fof_pairs.n ? S.fof_pairs.n : (unsigned long long)nleaves * 16 + 1024;
    unsigned long long npairs = 0;
    for (int attempt = 0; attempt < 2; attempt++) {
        TG_TRY(ensure(S.fof_pairs, cap));
        cap = S.fof_pairs.n;
        TG_CUDA(cudaMemsetAsync(S.dev_cnt.p + 1, 0, sizeof(unsigned long long), st));
        k_fof_pairs<<<(nleaves + 127) / 128, 128, 0, st>>>(nleaves, S.fof_leaves.p, S.nd_pb.p, S.nd_pe.p,
                                                            S.nd_child0.p, S.nd_aabb.p, Lint, L2, periodic,
                                                            S.fof_pairs.p, cap, S.dev_cnt.p + 1, S.dev_err.p);
        TG_TRY(launched(S));
        TG_CUDA(cudaMemcpyAsync(S.h_cnt, S.dev_cnt.p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        TG_CUDA(cudaStreamSynchronize(st));
        npairs = S.h_cnt[1];
        if (npairs <= cap) break;
        cap = npairs;
    }
    if (npairs > cap) return TG_ERR_NOMEM;
    if (npairs > 0) {
        const int64_t threads = (int64_t)npairs * 32;
        k_fof_link<<<(int)((threads + 255) / 256), 256, 0, st>>>((int64_t)npairs, S.fof_pairs.p, S.nd_pb.p, S.nd_pe.p,
                                                                 S.pos.p, L2, periodic, S.fof_P.p, S.fof_has.p,
                                                                 S.fof_tries, S.dev_err.p);
        TG_TRY(launched(S));
    }
    TG_TRY(ensure(S.fof_key, 2 * n));
    TG_TRY(ensure(S.fof_mem, 2 * n));
    int32_t *R = S.fof_key.p + n; /* roots; this half of the key buffer is free until the catalogue sorts */
    k_fof_roots<<<gn, 256, 0, st>>>(n, S.fof_P.p, S.pos.p, R, S.fof_gmin.p);
    TG_TRY(launched(S));
    TG_CUDA(cudaMemsetAsync(S.dev_cnt.p + 2, 0, sizeof(unsigned long long), st));
    k_fof_out<<<gn, 256, 0, st>>>(n, R, S.pos.p, S.fof_gmin.p, S.fof_has.p, group_dev, S.fof_key.p,
                                  S.fof_mem.p, S.dev_cnt.p + 2);
    TG_TRY(launched(S));
    uint32_t err = 0;
    TG_TRY(read_err(S, st, &err));
    if (err & 4u) return TG_ERR_TIMEOUT; /* a union ran out of hook attempts */
    if (err) return TG_ERR_CAPACITY;
    TG_CUDA(cudaMemcpyAsync(S.h_cnt, S.dev_cnt.p, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    S.fof_ngroups = (int64_t)S.h_cnt[2];
    S.fof_npairs = (int64_t)npairs;
    if (ngroups) *ngroups = S.fof_ngroups;
    return TG_OK;
}

/*
 * Catalogue of the groups found by fof_run (ids ascending by the host).
 * out: 14 doubles per group: id, N, x[3], v[3], dv[3], rmax, rc, 0.
 */
static int fof_catalog(Solver &S, double a, std::vector<double> &out, cudaStream_t st) {
    const int64_t n = S.n, ng = S.fof_ngroups;
    out.assign(14 * ng, 0.0);
    if (ng == 0) return TG_OK;
    const int periodic = S.prm.ewald ? 1 : 0;
    int32_t *key_in = S.fof_key.p, *key_out = S.fof_key.p + n;
    int32_t *mem_in = S.fof_mem.p, *mem_out = S.fof_mem.p + n;
    size_t tmp = 0;
    TG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key_in, key_out, mem_in, mem_out, (int)n, 0, 32, st));
    TG_TRY(ensure(S.cub_tmp, tmp));
    TG_CUDA(cub::DeviceRadixSort::SortPairs(S.cub_tmp.p, tmp, key_in, key_out, mem_in, mem_out, (int)n, 0, 32, st));
    /* runs of equal roots: the groups first (keys < INT_MAX), then at most one run of loners */
    /* sized for n runs, the most there can be, so the encode never writes past them */
    TG_TRY(ensure(S.fof_runs, 3 * (n + 1)));
    int32_t *roots = S.fof_runs.p, *cnt = roots + (n + 1), *off = cnt + (n + 1);
    size_t tmp2 = 0;
    TG_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, tmp2, key_out, roots, cnt, S.dev_cnt.p + 3, (int)n, st));
    TG_TRY(ensure(S.cub_tmp, tmp2));
    TG_CUDA(cub::DeviceRunLengthEncode::Encode(S.cub_tmp.p, tmp2, key_out, roots, cnt, S.dev_cnt.p + 3, (int)n, st));
    TG_CUDA(cudaMemcpyAsync(S.h_cnt + 3, S.dev_cnt.p + 3, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    const int64_t runs = (int64_t)S.h_cnt[3];
    if (runs != ng && runs != ng + 1) return TG_ERR_STATE; /* one run per group, plus the loners */
    size_t tmp3 = 0;
    TG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp3, cnt, off, (int)ng, st));
    TG_TRY(ensure(S.cub_tmp, tmp3));
    TG_CUDA(cub::DeviceScan::ExclusiveSum(S.cub_tmp.p, tmp3, cnt, off, (int)ng, st));
    TG_TRY(ensure(S.fof_radii, n));
    TG_TRY(ensure(S.fof_stats, 13 * ng));
    TG_CUDA(cudaMemsetAsync(S.dev_err.p, 0, sizeof(uint32_t), st));
    k_group_stats<<<(int)ng, FOF_TPB, 0, st>>>(n, roots, off, cnt, mem_out, S.pos.p, S.vel.p, S.fof_gmin.p, a,
                                              periodic, S.fof_radii.p, S.fof_stats.p, S.dev_err.p);
    TG_TRY(launched(S));
    uint32_t err = 0;
    TG_TRY(read_err(S, st, &err));
    if (err) return TG_ERR_STATE;
    std::vector<double> h(13 * ng);
    TG_CUDA(cudaMemcpyAsync(h.data(), S.fof_stats.p, sizeof(double) * 13 * ng, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    std::vector<int64_t> order(ng);
    for (int64_t g = 0; g < ng; g++) order[g] = g;
    std::sort(order.begin(), order.end(), [&](int64_t p, int64_t q) { return h[13 * p + 11] < h[13 * q + 11]; });
    for (int64_t k = 0; k < ng; k++) {
        const double *s = &h[13 * order[k]];
        double *o = &out[14 * k];
        o[0] = s[11];
        o[1] = s[10];
        for (int d = 0; d < 9; d++) o[2 + d] = s[d];
        o[11] = s[9];
        o[12] = s[12];
    }
    return TG_OK;
}

} // namespace tg

extern "C" int tg_find_groups(tg_solver *s, double link_len, int64_t *group, int64_t *ngroups, int where,
                              void *stream) {
    if (!s || (where != TG_HOST && where != TG_DEVICE)) return TG_ERR_ARG;
    tg::Solver &S = s->S;
    if (S.n <= 0) return TG_ERR_STATE;
    if (!(link_len > 0.0) || !std::isfinite(link_len)) return TG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    TG_CUDA(cudaSetDevice(S.dev));
    if (!S.have_tree) TG_TRY(tg::tree_build(S, st));
    if (!S.have_multipoles) TG_TRY(tg::tree_multipoles(S, st));
    TG_TRY(tg::ensure(S.fof_group, S.n));
    int64_t *gdev = where == TG_DEVICE && group ? group : S.fof_group.p;
    TG_TRY(tg::fof_run(S, link_len, gdev, ngroups, st));
    if (group && where == TG_HOST) {
        TG_CUDA(cudaMemcpyAsync(group, gdev, sizeof(int64_t) * S.n, cudaMemcpyDeviceToHost, st));
        TG_CUDA(cudaStreamSynchronize(st));
    }
    S.fof_link = link_len;
    return TG_OK;
}

extern "C" int tg_group_catalog(tg_solver *s, double a, double *out, int64_t capacity, int64_t *ngroups,
                                void *stream) {
    if (!s || !ngroups || !(a > 0.0)) return TG_ERR_ARG;
    tg::Solver &S = s->S;
    if (S.fof_link <= 0.0 || !S.have_tree) return TG_ERR_STATE;
    *ngroups = S.fof_ngroups;
    if (!out) return TG_OK;
    if (capacity < S.fof_ngroups) return TG_ERR_SIZE;
    TG_CUDA(cudaSetDevice(S.dev));
    std::vector<double> h;
    TG_TRY(tg::fof_catalog(S, a, h, (cudaStream_t)stream));
    if (!h.empty()) std::memcpy(out, h.data(), sizeof(double) * h.size());
    return TG_OK;
}

extern "C" int tg_set_fof_retry_limit(tg_solver *s, int32_t tries) {
    if (!s || tries < 0) return TG_ERR_ARG;
    s->S.fof_tries = tries;
    return TG_OK;
}
