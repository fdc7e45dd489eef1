/*
 * tg_walk.cu -- interaction-list generation (tree::kick_fmm, src/tree.cpp:378-635).
 *
 * The reference walks the tree top-down carrying two check lists (direct and
 * Ewald) of check_items {node, opened}.  At every node with particles
 * (src/tree.cpp:424-504):
 *     far & opened      -> CP  (particles of an opened leaf into the expansion)
 *     far & !opened     -> CC  (multipole into the expansion)
 *     near & leaf       -> kept, marked opened
 *     near & internal   -> replaced by its two children
 * and both children inherit the resulting list.  At a leaf the list is then
 * drained until empty (src/tree.cpp:530-602):
 *     opened            -> PP  (regardless of distance)
 *     !opened & far     -> PC
 *     !opened & near    -> opened leaf / children, as above.
 * far(direct) = d > (r_a + r_b)/theta && d > r_a + r_b + h with d the
 * minimum-image centre distance; far(Ewald) uses d = max(0.25, d) and, for
 * the node itself (d = 0), rmax < r_ewald.  The float/double mix of the
 * reference (float radii sum, double theta_inv and h) is kept so decisions,
 * and therefore the lists, are identical to the reference's.
 *
 * GPU form: the node stage runs level-synchronously, one warp per node,
 * reading the parent's list (ids with bit 31 = opened) and writing the CC/CP
 * lists and the node's own next list.  Each warp classifies its input twice
 * (count, then write) so every output list is contiguous and in the
 * reference's order: opened leaves first, then child pairs.  The leaf drain
 * is one persistent launch: each warp takes leaves from an atomic counter
 * and iterates in a private global scratch area.  Capacity overflows never
 * write out of bounds: they set a flag and the host regrows and repeats.
 */
#include <algorithm>
#include <cstring>

#include "tg_solver.cuh"

namespace tg {

struct WalkParams {
    double theta_inv;
    double h;
    float r_ewald;
    int ewald;
    const int32_t *nact; /* active particles per node (rung steps); nullptr: every particle is a sink */
};

constexpr uint32_t OPENED = 0x80000000u;
constexpr uint32_t ID_MASK = 0x7fffffffu;

struct NodeView {
    const int32_t *pb, *pe, *child0;
    const MSrc *ms;
    const float *r, *rmax;
    /* what the opening test reads of a check item, packed: (COM x, y, z, r
     * bits) and child0, or NODE_EMPTY for a node without particles -- two
     * loads per item instead of six scattered ones */
    const int4 *wx;
    const int32_t *kind;
};

constexpr int32_t NODE_EMPTY = -2;

/* the packed records of NodeView::wx / kind, one thread per node */
__global__ void k_walk_records(int64_t nn, const int32_t *__restrict__ pb, const int32_t *__restrict__ pe,
                               const int32_t *__restrict__ child0, const MSrc *__restrict__ ms,
                               const float *__restrict__ r, int4 *__restrict__ wx, int32_t *__restrict__ kind) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    wx[i] = make_int4(ms[i].x[0], ms[i].x[1], ms[i].x[2], __float_as_int(r[i]));
    kind[i] = pe[i] == pb[i] ? NODE_EMPTY : child0[i];
}

__device__ __forceinline__ double near_sep(const double *x) {
    double d = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double a = fabs(x[k]);
        const double t = fmin(a, __dadd_rn(1.0, -a));
        d = __dadd_rn(d, __dmul_rn(t, t));
    }
    return __dsqrt_rn(d);
}

__device__ __forceinline__ double vnorm(const double *x) {
    double d = __dmul_rn(x[0], x[0]);
    d = __dadd_rn(d, __dmul_rn(x[1], x[1]));
    d = __dadd_rn(d, __dmul_rn(x[2], x[2]));
    return __dsqrt_rn(d);
}

/* src/tree.cpp:428-429 (node stage) and 536-537 (leaf drain) */
__device__ __forceinline__ bool far_direct(const WalkParams &W, const double *X, float r, const int32_t *cx, float cr) {
    double dX[3];
#pragma unroll
    for (int k = 0; k < 3; k++) dX[k] = __dadd_rn(X[k], -pos2d(cx[k]));
    const double dx = W.ewald ? near_sep(dX) : vnorm(dX);
    const float rs = __fadd_rn(r, cr);
    return dx > __dmul_rn((double)rs, W.theta_inv) && dx > __dadd_rn((double)rs, W.h);
}

/* src/tree.cpp:452-459 and 570-577, with ewald_far_separation (src/gravity.cpp:20-23) */
__device__ __forceinline__ bool far_ewald(const WalkParams &W, const double *X, float r, float rmax, const int32_t *cx,
                                          float cr) {
    double dX[3];
#pragma unroll
    for (int k = 0; k < 3; k++) dX[k] = __dadd_rn(X[k], -pos2d(cx[k]));
    const double dx = fmax(0.25, near_sep(dX));
    double dot = __dmul_rn(dX[0], dX[0]);
    dot = __dadd_rn(dot, __dmul_rn(dX[1], dX[1]));
    dot = __dadd_rn(dot, __dmul_rn(dX[2], dX[2]));
    if (dot > 0.0) {
        const float rs = __fadd_rn(r, cr);
        return dx > __dmul_rn((double)rs, W.theta_inv) && dx > __dadd_rn((double)rs, W.h);
    }
    return rmax < W.r_ewald;
}

/* classification codes */
enum { C_SKIP = 0, C_FAR_OPEN = 1, C_FAR = 2, C_NEAR_LEAF = 3, C_NEAR_INT = 4 };

__device__ __forceinline__ int classify(const WalkParams &W, const NodeView &V, bool ewald_list, const double *X,
                                        float r, float rmax, uint32_t item, int32_t nnodes, uint32_t *err) {
    const int32_t c = (int32_t)(item & ID_MASK);
    if (c >= nnodes) {
        atomicOr(err, DEV_ERR_BADINDEX);
        return C_SKIP;
    }
    const int32_t k = V.kind[c];
    if (k == NODE_EMPTY) return C_SKIP;
    const int4 q = V.wx[c];
    const int32_t cx[3] = {q.x, q.y, q.z};
    const float cr = __int_as_float(q.w);
    const bool far = ewald_list ? far_ewald(W, X, r, rmax, cx, cr) : far_direct(W, X, r, cx, cr);
    if (far) return (item & OPENED) ? C_FAR_OPEN : C_FAR;
    return k < 0 ? C_NEAR_LEAF : C_NEAR_INT;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

/* Node stage for one list of one node (src/tree.cpp:424-476). */
__device__ void node_stage_list(const WalkParams &W, const NodeView &V, bool ewald_list, const double *X, float r,
                                float rmax, const int32_t *in, int32_t nin, int32_t nnodes, int32_t *pool_cc,
                                int64_t cap_cc, unsigned long long *top_cc, int64_t *off_cc, int32_t *len_cc,
                                int32_t *pool_cp, int64_t cap_cp, unsigned long long *top_cp, int64_t *off_cp,
                                int32_t *len_cp, int32_t *pool_nx, int64_t cap_nx, unsigned long long *top_nx,
                                int64_t *off_nx, int32_t *len_nx, uint32_t *err) {
    const int lane = threadIdx.x & 31;
    /* pass 1: counts */
    int n_cc = 0, n_cp = 0, n_lf = 0, n_int = 0;
    for (int32_t base = 0; base < nin; base += 32) {
        const int32_t j = base + lane;
        int code = C_SKIP;
        if (j < nin) code = classify(W, V, ewald_list, X, r, rmax, (uint32_t)in[j], nnodes, err);
        n_cp += __popc(__ballot_sync(0xffffffffu, code == C_FAR_OPEN));
        n_cc += __popc(__ballot_sync(0xffffffffu, code == C_FAR));
        n_lf += __popc(__ballot_sync(0xffffffffu, code == C_NEAR_LEAF));
        n_int += __popc(__ballot_sync(0xffffffffu, code == C_NEAR_INT));
    }
    const int n_nx = n_lf + 2 * n_int;
    unsigned long long b_cc = 0, b_cp = 0, b_nx = 0;
    int ok = 1;
    if (lane == 0) {
        if (n_cc) b_cc = atomicAdd(top_cc, (unsigned long long)n_cc);
        if (n_cp) b_cp = atomicAdd(top_cp, (unsigned long long)n_cp);
        if (n_nx) b_nx = atomicAdd(top_nx, (unsigned long long)n_nx);
        if (b_cc + n_cc > (unsigned long long)cap_cc || b_cp + n_cp > (unsigned long long)cap_cp) {
            atomicOr(err, DEV_ERR_OVERFLOW_LIST);
            ok = 0;
        }
        if (b_nx + n_nx > (unsigned long long)cap_nx) {
            atomicOr(err, DEV_ERR_OVERFLOW_NEXT);
            ok = 0;
        }
        *off_cc = (int64_t)b_cc;
        *len_cc = ok ? n_cc : 0;
        *off_cp = (int64_t)b_cp;
        *len_cp = ok ? n_cp : 0;
        *off_nx = (int64_t)b_nx;
        *len_nx = ok ? n_nx : 0;
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (!ok) return;
    b_cc = __shfl_sync(0xffffffffu, b_cc, 0);
    b_cp = __shfl_sync(0xffffffffu, b_cp, 0);
    b_nx = __shfl_sync(0xffffffffu, b_nx, 0);
    /* pass 2: write */
    int r_cc = 0, r_cp = 0, r_lf = 0, r_int = 0;
    const uint32_t lt = lanemask_lt();
    for (int32_t base = 0; base < nin; base += 32) {
        const int32_t j = base + lane;
        int code = C_SKIP;
        uint32_t item = 0;
        if (j < nin) {
            item = (uint32_t)in[j];
            code = classify(W, V, ewald_list, X, r, rmax, item, nnodes, err);
        }
        const uint32_t m_cp = __ballot_sync(0xffffffffu, code == C_FAR_OPEN);
        const uint32_t m_cc = __ballot_sync(0xffffffffu, code == C_FAR);
        const uint32_t m_lf = __ballot_sync(0xffffffffu, code == C_NEAR_LEAF);
        const uint32_t m_in = __ballot_sync(0xffffffffu, code == C_NEAR_INT);
        const int32_t id = (int32_t)(item & ID_MASK);
        if (code == C_FAR_OPEN) pool_cp[b_cp + r_cp + __popc(m_cp & lt)] = id;
        if (code == C_FAR) pool_cc[b_cc + r_cc + __popc(m_cc & lt)] = id;
        if (code == C_NEAR_LEAF) pool_nx[b_nx + r_lf + __popc(m_lf & lt)] = (int32_t)(item | OPENED);
        if (code == C_NEAR_INT) {
            const int32_t c0 = V.kind[id]; /* an internal node: its child0 */
            const int64_t q = b_nx + n_lf + 2 * (r_int + __popc(m_in & lt));
            pool_nx[q] = c0;
            pool_nx[q + 1] = c0 + 1;
        }
        r_cp += __popc(m_cp);
        r_cc += __popc(m_cc);
        r_lf += __popc(m_lf);
        r_int += __popc(m_in);
    }
}

__global__ void k_node_stage(WalkParams W, NodeView V, int64_t first, int64_t count, int32_t nnodes,
                             const int32_t *__restrict__ parent, int32_t **pools, const int64_t *caps,
                             unsigned long long *tops, int64_t **loff, int32_t **llen, const int32_t *nx_in_d,
                             const int32_t *nx_in_e, int32_t *nx_out_d, int32_t *nx_out_e, int64_t cap_nx_d,
                             int64_t cap_nx_e, unsigned long long *nx_top, int64_t *nx_off_d, int32_t *nx_len_d,
                             int64_t *nx_off_e, int32_t *nx_len_e, uint32_t *err) {
    const int lane = threadIdx.x & 31;
    const int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (k >= count) return;
    const int32_t i = (int32_t)(first + k);
    /* a node without active particles gets no lists (src/tree.cpp:396): it stays a source only */
    if (V.pe[i] == V.pb[i] || (W.nact && W.nact[i] == 0)) {
        if (lane == 0) {
            nx_len_d[i] = 0;
            nx_len_e[i] = 0;
            for (int q = 0; q < 4; q++) llen[q][i] = 0;
        }
        return;
    }
    const MSrc &s = V.ms[i];
    const double X[3] = {pos2d(s.x[0]), pos2d(s.x[1]), pos2d(s.x[2])};
    const float r = V.r[i], rmax = V.rmax[i];
    const int32_t root_item = 0;
    const int32_t *in_d, *in_e;
    int32_t nin_d, nin_e;
    const int32_t p = parent[i];
    if (p < 0) {
        in_d = in_e = &root_item;
        nin_d = 1;
        nin_e = W.ewald ? 1 : 0;
    } else {
        in_d = nx_in_d + nx_off_d[p];
        nin_d = nx_len_d[p];
        in_e = nx_in_e + nx_off_e[p];
        nin_e = W.ewald ? nx_len_e[p] : 0;
    }
    node_stage_list(W, V, false, X, r, rmax, in_d, nin_d, nnodes, pools[TG_CC_D], caps[TG_CC_D], &tops[TG_CC_D],
                    &loff[TG_CC_D][i], &llen[TG_CC_D][i], pools[TG_CP_D], caps[TG_CP_D], &tops[TG_CP_D],
                    &loff[TG_CP_D][i], &llen[TG_CP_D][i], nx_out_d, cap_nx_d, &nx_top[0], &nx_off_d[i],
                    &nx_len_d[i], err);
    node_stage_list(W, V, true, X, r, rmax, in_e, nin_e, nnodes, pools[TG_CC_E], caps[TG_CC_E], &tops[TG_CC_E],
                    &loff[TG_CC_E][i], &llen[TG_CC_E][i], pools[TG_CP_E], caps[TG_CP_E], &tops[TG_CP_E],
                    &loff[TG_CP_E][i], &llen[TG_CP_E][i], nx_out_e, cap_nx_e, &nx_top[1], &nx_off_e[i],
                    &nx_len_e[i], err);
}

/* Leaf drain for one list (src/tree.cpp:530-602); scratch layout per warp:
 * [bufA | bufB | outPP | outPC], each `cap` entries. */
__device__ void drain_list(const WalkParams &W, const NodeView &V, bool ewald_list, const double *X, float r,
                           float rmax, const int32_t *in, int32_t nin, int32_t nnodes, int32_t *scr, int64_t cap,
                           int32_t *pool_pp, int64_t cap_pp, unsigned long long *top_pp, int64_t *off_pp,
                           int32_t *len_pp, int32_t *pool_pc, int64_t cap_pc, unsigned long long *top_pc,
                           int64_t *off_pc, int32_t *len_pc, uint32_t *err) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    int32_t *bufA = scr, *bufB = scr + cap, *outPP = scr + 2 * cap, *outPC = scr + 3 * cap;
    int n_pp = 0, n_pc = 0;
    const int32_t *cur = in;
    int32_t ncur = nin;
    bool ok = true;
    int iter = 0;
    while (ncur > 0 && ok) {
        if (++iter > 200) { /* the tree depth bounds the iterations; guard anyway */
            if (lane == 0) atomicOr(err, DEV_ERR_SPIN);
            ok = false;
            break;
        }
        int32_t *nxt = (cur == bufA) ? bufB : bufA;
        /* pass 1: count opened-leaf entries of the next list (to order children after them) */
        int n_lf = 0, n_int = 0, c_pp = 0, c_pc = 0;
        for (int32_t base = 0; base < ncur; base += 32) {
            const int32_t j = base + lane;
            int code = C_SKIP;
            uint32_t item = 0;
            if (j < ncur) {
                item = (uint32_t)cur[j];
                code = classify(W, V, ewald_list, X, r, rmax, item, nnodes, err);
            }
            const bool opened = (item & OPENED) && code != C_SKIP;
            c_pp += __popc(__ballot_sync(0xffffffffu, opened));
            c_pc += __popc(__ballot_sync(0xffffffffu, !opened && (code == C_FAR || code == C_FAR_OPEN)));
            n_lf += __popc(__ballot_sync(0xffffffffu, !opened && code == C_NEAR_LEAF));
            n_int += __popc(__ballot_sync(0xffffffffu, !opened && code == C_NEAR_INT));
        }
        if (n_pp + c_pp > cap || n_pc + c_pc > cap || n_lf + 2 * n_int > cap) {
            if (lane == 0) atomicOr(err, DEV_ERR_OVERFLOW_SCRATCH);
            ok = false;
            break;
        }
        int r_lf = 0, r_int = 0;
        for (int32_t base = 0; base < ncur; base += 32) {
            const int32_t j = base + lane;
            int code = C_SKIP;
            uint32_t item = 0;
            if (j < ncur) {
                item = (uint32_t)cur[j];
                code = classify(W, V, ewald_list, X, r, rmax, item, nnodes, err);
            }
            const bool opened = (item & OPENED) && code != C_SKIP;
            const bool pc = !opened && (code == C_FAR || code == C_FAR_OPEN);
            const bool lf = !opened && code == C_NEAR_LEAF;
            const bool in_ = !opened && code == C_NEAR_INT;
            const uint32_t m_pp = __ballot_sync(0xffffffffu, opened);
            const uint32_t m_pc = __ballot_sync(0xffffffffu, pc);
            const uint32_t m_lf = __ballot_sync(0xffffffffu, lf);
            const uint32_t m_in = __ballot_sync(0xffffffffu, in_);
            const int32_t id = (int32_t)(item & ID_MASK);
            if (opened) outPP[n_pp + __popc(m_pp & lt)] = id;
            if (pc) outPC[n_pc + __popc(m_pc & lt)] = id;
            if (lf) nxt[r_lf + __popc(m_lf & lt)] = (int32_t)(item | OPENED);
            if (in_) {
                const int32_t c0 = V.kind[id]; /* an internal node: its child0 */
                const int32_t q = n_lf + 2 * (r_int + __popc(m_in & lt));
                nxt[q] = c0;
                nxt[q + 1] = c0 + 1;
            }
            n_pp += __popc(m_pp);
            n_pc += __popc(m_pc);
            r_lf += __popc(m_lf);
            r_int += __popc(m_in);
        }
        __syncwarp();
        cur = nxt;
        ncur = n_lf + 2 * n_int;
    }
    /* publish */
    unsigned long long b_pp = 0, b_pc = 0;
    int okw = ok ? 1 : 0;
    if (lane == 0) {
        if (okw) {
            if (n_pp) b_pp = atomicAdd(top_pp, (unsigned long long)n_pp);
            if (n_pc) b_pc = atomicAdd(top_pc, (unsigned long long)n_pc);
            if (b_pp + n_pp > (unsigned long long)cap_pp || b_pc + n_pc > (unsigned long long)cap_pc) {
                atomicOr(err, DEV_ERR_OVERFLOW_LIST);
                okw = 0;
            }
        }
        *off_pp = (int64_t)b_pp;
        *len_pp = okw ? n_pp : 0;
        *off_pc = (int64_t)b_pc;
        *len_pc = okw ? n_pc : 0;
    }
    okw = __shfl_sync(0xffffffffu, okw, 0);
    if (!okw) return;
    b_pp = __shfl_sync(0xffffffffu, b_pp, 0);
    b_pc = __shfl_sync(0xffffffffu, b_pc, 0);
    __syncwarp();
    for (int j = lane; j < n_pp; j += 32) pool_pp[b_pp + j] = outPP[j];
    for (int j = lane; j < n_pc; j += 32) pool_pc[b_pc + j] = outPC[j];
}

__global__ void k_leaf_drain(WalkParams W, NodeView V, int64_t first, int64_t count, int32_t nnodes,
                             int32_t **pools, const int64_t *caps, unsigned long long *tops, int64_t **loff,
                             int32_t **llen, const int32_t *nx_pool_d, const int32_t *nx_pool_e,
                             const int64_t *nx_off_d, const int32_t *nx_len_d, const int64_t *nx_off_e,
                             const int32_t *nx_len_e, int32_t *scratch, int64_t scr_cap,
                             unsigned long long *work_counter, uint32_t *err) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int32_t *scr = scratch + warp * 4 * scr_cap;
    for (;;) {
        int64_t k = 0;
        if (lane == 0) k = (int64_t)atomicAdd(work_counter, 1ull);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= count) break;
        const int32_t i = (int32_t)(first + k);
        /* the leaves of this level with (active) particles */
        if (V.child0[i] >= 0 || V.pe[i] == V.pb[i] || (W.nact && W.nact[i] == 0)) continue;
        const MSrc &s = V.ms[i];
        const double X[3] = {pos2d(s.x[0]), pos2d(s.x[1]), pos2d(s.x[2])};
        const float r = V.r[i], rmax = V.rmax[i];
        drain_list(W, V, false, X, r, rmax, nx_pool_d + nx_off_d[i], nx_len_d[i], nnodes, scr, scr_cap,
                   pools[TG_PP_D], caps[TG_PP_D], &tops[TG_PP_D], &loff[TG_PP_D][i], &llen[TG_PP_D][i],
                   pools[TG_PC_D], caps[TG_PC_D], &tops[TG_PC_D], &loff[TG_PC_D][i], &llen[TG_PC_D][i], err);
        if (W.ewald) {
            drain_list(W, V, true, X, r, rmax, nx_pool_e + nx_off_e[i], nx_len_e[i], nnodes, scr, scr_cap,
                       pools[TG_PP_E], caps[TG_PP_E], &tops[TG_PP_E], &loff[TG_PP_E][i], &llen[TG_PP_E][i],
                       pools[TG_PC_E], caps[TG_PC_E], &tops[TG_PC_E], &loff[TG_PC_E][i], &llen[TG_PC_E][i], err);
        } else if (lane == 0) {
            llen[TG_PP_E][i] = 0;
            llen[TG_PC_E][i] = 0;
        }
    }
}

__global__ void k_collect_leaves(int64_t nn, const int32_t *pb, const int32_t *pe, const int32_t *child0,
                                 const int32_t *nact, int32_t *leaves, unsigned long long *count) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    if (child0[i] < 0 && pe[i] > pb[i] && (!nact || nact[i] > 0)) {
        const unsigned long long k = atomicAdd(count, 1ull);
        leaves[k] = (int32_t)i;
    }
}

__global__ void k_zero_leaf_lens(int64_t nn, int32_t *l4, int32_t *l5, int32_t *l6, int32_t *l7) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    l4[i] = l5[i] = l6[i] = l7[i] = 0;
}

/* per-list interaction counts: counts[k] = sum over nodes of len (and pair
 * weighting by sink / source particle counts, done on the host side) */

int tree_walk(Solver &S, cudaStream_t st) {
    if (!S.have_multipoles) return TG_ERR_STATE;
    const int64_t nn = S.nnodes;
    WalkParams W;
    W.theta_inv = 1.0 / S.prm.theta;
    W.h = S.prm.soft_len;
    W.r_ewald = (float)(2.0 * S.prm.theta * std::pow(1.0e-3 / 8.0, 1.0 / 3.0));
    W.ewald = S.prm.ewald ? 1 : 0;
    W.nact = S.walk_nact;
    TG_TRY(ensure(S.wk_wx, nn));
    TG_TRY(ensure(S.wk_kind, nn));
    k_walk_records<<<(int)((nn + 255) / 256), 256, 0, st>>>(nn, S.nd_pb.p, S.nd_pe.p, S.nd_child0.p, S.nd_ms.p,
                                                            S.nd_r.p, S.wk_wx.p, S.wk_kind.p);
    TG_TRY(launched(S));
    NodeView V{S.nd_pb.p, S.nd_pe.p, S.nd_child0.p, S.nd_ms.p, S.nd_r.p, S.nd_rmax.p, S.wk_wx.p, S.wk_kind.p};

    for (int k = 0; k < NLIST; k++) {
        TG_TRY(ensure(S.loff[k], nn));
        TG_TRY(ensure(S.llen[k], nn));
    }
    for (int q = 0; q < 2; q++) {
        TG_TRY(ensure(S.nxt_off[q], nn));
        TG_TRY(ensure(S.nxt_len[q], nn));
    }
    TG_TRY(ensure(S.pool_top, NLIST + 2 + 2));
    TG_TRY(ensure(S.idx, nn)); /* leaf id list (idx is free after the build) */
    /* device-side pointer tables, kept with the solver: a cudaFree per walk
     * would wait for the whole device, so concurrent solvers (batches) would
     * serialise on it */
    static_assert(NLIST == 8, "");
    DevBuf<int32_t *> &d_pools = S.wk_pools, &d_llen = S.wk_llen;
    DevBuf<int64_t *> &d_loff = S.wk_loff;
    DevBuf<int64_t> &d_caps = S.wk_caps;
    TG_TRY(ensure(d_pools, NLIST));
    TG_TRY(ensure(d_llen, NLIST));
    TG_TRY(ensure(d_loff, NLIST));
    TG_TRY(ensure(d_caps, NLIST));

    /* collect leaves */
    TG_CUDA(cudaMemsetAsync(S.pool_top.p, 0, sizeof(unsigned long long) * (NLIST + 4), st));
    {
        const int g = (int)((nn + 255) / 256);
        k_collect_leaves<<<g, 256, 0, st>>>(nn, S.nd_pb.p, S.nd_pe.p, S.nd_child0.p, S.walk_nact, S.idx.p, S.pool_top.p + NLIST + 2);
        TG_TRY(launched(S));
    }
    unsigned long long nleaves_h = 0;
    TG_TRY(read_small(S, st, &nleaves_h, S.pool_top.p + NLIST + 2, sizeof(unsigned long long)));
    const int32_t nleaves = (int32_t)nleaves_h;

    /* capacities: those that served the last walk, else sized from the tree;
     * on an overflow the pools grow to the totals the walk asked for */
    int64_t cap[NLIST];
    int64_t cap_nx[2] = {0, 0};
    {
        const int64_t base_nodes = nn + 64;
        const int64_t base_leaves = nleaves + 64;
        const int64_t dflt[NLIST] = {160 * base_nodes,
                                     16 * base_nodes,
                                     (S.prm.ewald ? 32 : 1) * base_nodes,
                                     (S.prm.ewald ? 8 : 1) * base_nodes,
                                     16 * base_leaves,
                                     96 * base_leaves,
                                     (S.prm.ewald ? 16 : 1) * base_leaves,
                                     (S.prm.ewald ? 32 : 1) * base_leaves};
        for (int k = 0; k < NLIST; k++)
            cap[k] = S.cap_start > 0 ? S.cap_start : (S.list_cap[k] > 0 ? S.list_cap[k] : dflt[k]);
        /* the next lists of one level: a few hundred entries per node of the widest level */
        int64_t widest = 1;
        for (int L = 0; L <= S.depth; L++) widest = std::max(widest, S.level_off[L + 1] - S.level_off[L]);
        const int64_t dflt_nx[2] = {256 * widest + 4096, (S.prm.ewald ? 64 : 1) * widest + 4096};
        for (int q = 0; q < 2; q++)
            cap_nx[q] = S.cap_start > 0 ? S.cap_start : (S.nx_cap[q] > 0 ? S.nx_cap[q] : dflt_nx[q]);
        if (S.scratch_per_warp == 0) S.scratch_per_warp = 4096;
        if (S.cap_start > 0) S.scratch_per_warp = std::min<int64_t>(S.scratch_per_warp, S.cap_start);
    }
    int tries = 0;
    const int nlev = S.depth + 1;
    for (;;) {
        for (int k = 0; k < NLIST; k++) TG_TRY(ensure(S.pool[k], cap[k]));
        /* next lists: two halves per kind, the levels alternate between them */
        TG_TRY(ensure(S.nxt_pool[0], 2 * (size_t)cap_nx[0]));
        TG_TRY(ensure(S.nxt_pool[1], 2 * (size_t)cap_nx[1]));
        TG_TRY(ensure(S.nx_top, 2 * (size_t)nlev + 2 * (size_t)nlev));
        S.drain_warps = S.num_sms * 16;
        TG_TRY(ensure(S.scratch, (size_t)S.drain_warps * 4 * S.scratch_per_warp));
        int32_t *h_pools[NLIST], *h_llen[NLIST];
        int64_t *h_loff[NLIST];
        for (int k = 0; k < NLIST; k++) {
            h_pools[k] = S.pool[k].p;
            h_llen[k] = S.llen[k].p;
            h_loff[k] = S.loff[k].p;
        }
        /* the tables go up from pinned memory; the stream is waited for below
         * (read_err) before this area is written again */
        unsigned char *up = S.h_small;
        std::memcpy(up, h_pools, sizeof(h_pools));
        std::memcpy(up + 64, h_llen, sizeof(h_llen));
        std::memcpy(up + 128, h_loff, sizeof(h_loff));
        std::memcpy(up + 192, cap, sizeof(cap));
        TG_CUDA(cudaMemcpyAsync(d_pools.p, up, sizeof(h_pools), cudaMemcpyHostToDevice, st));
        TG_CUDA(cudaMemcpyAsync(d_llen.p, up + 64, sizeof(h_llen), cudaMemcpyHostToDevice, st));
        TG_CUDA(cudaMemcpyAsync(d_loff.p, up + 128, sizeof(h_loff), cudaMemcpyHostToDevice, st));
        TG_CUDA(cudaMemcpyAsync(d_caps.p, up + 192, sizeof(cap), cudaMemcpyHostToDevice, st));
        TG_CUDA(cudaMemsetAsync(S.pool_top.p, 0, sizeof(unsigned long long) * NLIST, st));
        /* per level: next-list tops (direct, ewald) and the drain's work counter */
        TG_CUDA(cudaMemsetAsync(S.nx_top.p, 0, sizeof(unsigned long long) * 4 * nlev, st));
        TG_CUDA(cudaMemsetAsync(S.dev_err.p, 0, sizeof(uint32_t), st));
        {
            const int g = (int)((nn + 255) / 256);
            k_zero_leaf_lens<<<g, 256, 0, st>>>(nn, S.llen[4].p, S.llen[5].p, S.llen[6].p, S.llen[7].p);
            TG_TRY(launched(S));
        }
        for (int L = 0; L <= S.depth; L++) {
            const int64_t first = S.level_off[L], count = S.level_off[L + 1] - S.level_off[L];
            if (count <= 0) continue;
            const size_t in_h = (size_t)((L + 1) & 1), out_h = (size_t)(L & 1);
            int32_t *const nd_in = S.nxt_pool[0].p + in_h * cap_nx[0], *const ne_in = S.nxt_pool[1].p + in_h * cap_nx[1];
            int32_t *const nd_out = S.nxt_pool[0].p + out_h * cap_nx[0];
            int32_t *const ne_out = S.nxt_pool[1].p + out_h * cap_nx[1];
            unsigned long long *const lt = S.nx_top.p + 4 * (size_t)L; /* direct, ewald, drain counter */
            {
                const int TPB = 128;
                const int g = (int)((count * 32 + TPB - 1) / TPB);
                k_node_stage<<<g, TPB, 0, st>>>(W, V, first, count, (int32_t)nn, S.nd_parent.p, d_pools.p, d_caps.p,
                                                S.pool_top.p, d_loff.p, d_llen.p, nd_in, ne_in, nd_out, ne_out,
                                                cap_nx[0], cap_nx[1], lt, S.nxt_off[0].p, S.nxt_len[0].p,
                                                S.nxt_off[1].p, S.nxt_len[1].p, S.dev_err.p);
                TG_TRY(launched(S));
            }
            if (S.level_leaves[L] > 0) { /* drain this level's leaves while their next lists are live */
                const int TPB = 128;
                const int64_t want = std::min<int64_t>(S.drain_warps, S.level_leaves[L]);
                const int g = (int)((want * 32 + TPB - 1) / TPB);
                k_leaf_drain<<<g, TPB, 0, st>>>(W, V, first, count, (int32_t)nn, d_pools.p, d_caps.p, S.pool_top.p,
                                                d_loff.p, d_llen.p, nd_out, ne_out, S.nxt_off[0].p, S.nxt_len[0].p,
                                                S.nxt_off[1].p, S.nxt_len[1].p, S.scratch.p, S.scratch_per_warp,
                                                lt + 2, S.dev_err.p);
                TG_TRY(launched(S));
            }
        }
        uint32_t err = 0;
        TG_TRY(read_err(S, st, &err));
        if (err & (DEV_ERR_BADINDEX | DEV_ERR_SPIN)) {
            return TG_ERR_STATE;
        }
        if (!err) break;
        if (++tries > 24) {
            return TG_ERR_CAPACITY;
        }
        /* the pool tops kept counting past a full pool: they are what this
         * walk asked for, unless a next-list or scratch overflow starved the
         * levels below (then the lists keep their size until a walk that is
         * not starved has counted them, and the next lists at least double) */
        std::vector<unsigned long long> tops(NLIST), ltops(4 * (size_t)nlev);
        TG_CUDA(cudaMemcpyAsync(tops.data(), S.pool_top.p, sizeof(unsigned long long) * NLIST, cudaMemcpyDeviceToHost,
                                st));
        TG_CUDA(cudaMemcpyAsync(ltops.data(), S.nx_top.p, sizeof(unsigned long long) * 4 * nlev,
                                cudaMemcpyDeviceToHost, st));
        TG_CUDA(cudaStreamSynchronize(st));
        const bool starved = (err & (DEV_ERR_OVERFLOW_NEXT | DEV_ERR_OVERFLOW_SCRATCH)) != 0;
        if (!starved)
            for (int k = 0; k < NLIST; k++)
                if ((int64_t)tops[k] > cap[k]) cap[k] = (int64_t)tops[k] + (int64_t)(tops[k] / 8) + 1024;
        for (int q = 0; q < 2; q++) {
            int64_t t = 0;
            for (int L = 0; L < nlev; L++) t = std::max<int64_t>(t, (int64_t)ltops[4 * (size_t)L + q]);
            if (t > cap_nx[q]) cap_nx[q] = std::max(2 * cap_nx[q], t + t / 8 + 1024);
        }
        if (err & DEV_ERR_OVERFLOW_SCRATCH) S.scratch_per_warp *= 2;
    }
    for (int k = 0; k < NLIST; k++) S.list_cap[k] = cap[k];
    S.nx_cap[0] = cap_nx[0];
    S.nx_cap[1] = cap_nx[1];
    S.st.walk_retries = tries;
    S.st.leaves = nleaves;
    S.have_lists = true;
    S.have_forces = false;
    return TG_OK;
}

} // namespace tg
