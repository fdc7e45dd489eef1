/*
 * tg_solver.cuh -- host-side solver state and the internal entry points the
 * C ABI (tg_capi.cu) drives.  Device data layout (all in particle/node order
 * after the Morton sort; "sorted order"):
 *
 *   particles  pos[n]   int4   (x, y, z fixed point, w = caller index)
 *              vel[n]   float4 (vx, vy, vz, 0)
 *              acc[n]   float4 (phi, gx, gy, gz)      FP32 path
 *              accd[n]  double4-like 4 doubles        FP64 path
 *   nodes      level order, increasing box id within a level
 *              nd_pb/pe  int32 particle range
 *              nd_child0 int32 (-1 leaf), nd_parent int32, nd_key u64 (Morton prefix << (63-level))
 *              nd_ms[n]  tg_msrc: 17 multipole floats + com int32[3] (80 B, the reference's multi_src)
 *              nd_r, nd_rmax float, nd_cnt int32, nd_level uint8
 *              nd_aabb  6 int32 (particle AABB, fixed point), nd_prange 6 double
 *              nd_L     35 doubles (local expansion after L2L)
 *   lists      per kind k: nd_loff[k][node] (int64), nd_llen[k][node] (int32) into pool[k]
 */
#pragma once

#include <atomic>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tigergrav_b200.h"
#include "tg_common.cuh"

#define TG_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t _e = (call);                                                               \
        if (_e != cudaSuccess) {                                                               \
            tg::set_last_cuda_error(_e, #call, __FILE__, __LINE__);                            \
            return TG_ERR_CUDA;                                                                \
        }                                                                                      \
    } while (0)

#define TG_TRY(call)                                                                           \
    do {                                                                                       \
        int _s = (call);                                                                       \
        if (_s != TG_OK) return _s;                                                            \
    } while (0)

namespace tg {

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line);

struct __align__(16) MSrc {
    float m[MP];
    int32_t x[3];
};
static_assert(sizeof(MSrc) == 80, "multi_src layout");

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0; /* capacity in elements */
};

constexpr int NLIST = 8;

struct Solver {
    tg_params prm{};
    int dev = 0;
    int64_t n = 0;
    bool have_tree = false, have_multipoles = false, have_lists = false, have_forces = false;

    /* particles */
    DevBuf<int4> pos, pos_alt;
    DevBuf<float4> vel, vel_alt;
    DevBuf<float4> acc;
    DevBuf<double> accd; /* FP64 path: 4 per particle */
    DevBuf<unsigned long long> keys, keys_alt;
    DevBuf<int32_t> idx, idx_alt;
    DevBuf<unsigned char> cub_tmp;

    /* nodes */
    int64_t nnodes = 0;
    std::vector<int64_t> level_off;    /* host: first node of each level, size depth+2 */
    std::vector<int64_t> level_leaves; /* host: leaves (childless nodes) of each level, size depth+1 */
    int depth = 0;
    DevBuf<int32_t> nd_pb, nd_pe, nd_child0, nd_parent, nd_flag, nd_scan;
    DevBuf<unsigned long long> nd_key;
    DevBuf<unsigned char> nd_level;
    DevBuf<MSrc> nd_ms;
    DevBuf<float> nd_r, nd_rmax;
    DevBuf<int32_t> nd_aabb;   /* 6 per node: min xyz, max xyz (fixed point) */
    DevBuf<double> nd_prange;  /* 6 per node: min xyz, max xyz */
    DevBuf<double> nd_L;       /* 35 per node */
    DevBuf<double> nd_Lloc;    /* 35 per node: CC/CP contributions */

    /* walk */
    DevBuf<int64_t> loff[NLIST];
    DevBuf<int32_t> llen[NLIST];
    DevBuf<int32_t> pool[NLIST];
    DevBuf<unsigned long long> pool_top; /* NLIST + 2 counters */
    DevBuf<int64_t> nxt_off[2];          /* per node: offset of next list (direct, ewald) */
    DevBuf<int32_t> nxt_len[2];
    DevBuf<int32_t> nxt_pool[2];         /* two halves each: even and odd levels */
    DevBuf<unsigned long long> nx_top;   /* per level: next-list tops (direct, ewald), drain counter, spare */
    DevBuf<int32_t *> wk_pools, wk_llen; /* device copies of the list pointer tables */
    DevBuf<int64_t *> wk_loff;
    DevBuf<int64_t> wk_caps;
    DevBuf<int4> wk_wx;                  /* per node: COM and r packed for the opening tests */
    DevBuf<int32_t> wk_kind;             /* per node: child0, or empty */
    DevBuf<int32_t> scratch;             /* leaf drain per-warp scratch */
    int64_t scratch_per_warp = 0;
    int drain_warps = 0;
    int64_t list_cap[NLIST] = {0, 0, 0, 0, 0, 0, 0, 0}; /* pool capacities that served the last walk */
    int64_t nx_cap[2] = {0, 0};
    int64_t cap_start = 0; /* tg_set_walk_capacity: first capacity of every pool (0: sized from the tree) */

    /* status / stats */
    DevBuf<uint32_t> dev_err;
    DevBuf<unsigned long long> dev_cnt; /* 16 counters */
    uint32_t *h_err = nullptr;          /* pinned */
    unsigned long long *h_cnt = nullptr;
    void *h_stage = nullptr;            /* pinned staging for host transfers */
    /* pinned, 4 KB: [0, 2048) uploads of small tables, [2048, 4096) small
     * readbacks (pageable copies would go through the driver's staging,
     * which host threads driving other solvers contend for) */
    unsigned char *h_small = nullptr;
    size_t h_stage_bytes = 0;

    /* Ewald tables */
    /* leapfrog checkpoints (caller order) and adjoint state */
    DevBuf<int32_t> ck_x;
    DevBuf<float> ck_v;
    int ck_steps = -1;
    double ck_dt = 0.0;
    DevBuf<double> adj_x, adj_v, tid_u, tid_o, tid_U, tid_V;
    DevBuf<int32_t> ew_cnt, ew_off; /* leaf Ewald chunks per leaf, and their exclusive scan */
    DevBuf<double> ew_part;          /* 64 x 4 partial sums per chunk */
    DevBuf<float4> ew_real, ew_four;
    DevBuf<float> ew_Hf;
    DevBuf<double> ew_Hd;
    DevBuf<float4> ew_Pf;
    DevBuf<double2> ew_Pd;
    DevBuf<float2> ew_nt, ew_sf; /* per node and h: (cos, sin) at the centre of mass; per leaf: sums over particles */
    DevBuf<float> ew_tpart;      /* per leaf Ewald chunk and h: 8 reciprocal-space source sums */
    bool have_tables = false;

    /* rung (individual) time steps: the rung lives in vel[i].w */
    DevBuf<int32_t> rung_flag, rung_scan, rung_nact; /* active flag per particle, its scan, active per node */
    DevBuf<int8_t> rung_out;                         /* caller-order rungs for tg_get_rungs */
    const int32_t *walk_nact = nullptr;              /* set during a rung step's walk only */

    /* friends-of-friends (sorted order unless noted) */
    DevBuf<int32_t> fof_P, fof_leaves, fof_key, fof_mem, fof_runs;
    DevBuf<int64_t> fof_gmin, fof_group; /* fof_group: caller order */
    DevBuf<uint8_t> fof_has;
    DevBuf<int2> fof_pairs;
    DevBuf<float> fof_radii;
    DevBuf<double> fof_stats;
    int64_t fof_ngroups = 0, fof_npairs = 0;
    double fof_link = 0.0; /* linking length of the groups held, 0: none for this tree */
    int32_t fof_tries = 65536; /* hook attempts per union before the union-find gives up */

    /* events for phase timing */
    cudaEvent_t ev[8];
    bool have_events = false;
    bool pp_timed = false; /* ev[6] marks the start of the FP32 PP kernel in the last solve */
    bool kd_timed = false; /* ev[7] marks a fused kick-drift that the last solve's build followed */
    bool kd_pending = false;
    tg_stats st{};
    int num_sms = 148;
    int64_t launches = 0; /* kernels of this library launched on this handle */
};

/* count a kernel launch of this library and check it */
inline int launched(Solver &S) {
    S.launches++;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_cuda_error(e, "kernel launch", __FILE__, __LINE__);
        return TG_ERR_CUDA;
    }
    return TG_OK;
}

/* device bytes held by every DevBuf of the process (all handles) */
inline std::atomic<long long> g_dev_bytes{0};

template <class T>
int ensure(DevBuf<T> &b, size_t count) {
    if (b.n >= count && b.p) return TG_OK;
    if (b.p) {
        cudaFree(b.p);
        g_dev_bytes -= (long long)(b.n * sizeof(T));
    }
    b.p = nullptr;
    b.n = 0;
    size_t c = count < 16 ? 16 : count;
    c = c + c / 4;
    if (cudaMalloc(&b.p, c * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return TG_ERR_NOMEM;
    }
    b.n = c;
    g_dev_bytes += (long long)(c * sizeof(T));
    return TG_OK;
}
template <class T>
void release(DevBuf<T> &b) {
    if (b.p) {
        cudaFree(b.p);
        g_dev_bytes -= (long long)(b.n * sizeof(T));
    }
    b.p = nullptr;
    b.n = 0;
}

int init_constants();
int ewald_tables(Solver &S, cudaStream_t st);
int tree_build(Solver &S, cudaStream_t st);
int tree_multipoles(Solver &S, cudaStream_t st);
int tree_walk(Solver &S, cudaStream_t st);
int gravity_forces(Solver &S, cudaStream_t st);
int kick(Solver &S, double dt, cudaStream_t st);
int drift(Solver &S, double dt, cudaStream_t st);
int kick_drift(Solver &S, double dt_close, double dt_open, double dt_drift, cudaStream_t st);
int energy(Solver &S, double out[5], cudaStream_t st);
int truth(Solver &S, const int64_t *samples, int64_t ns, double alpha, double *phi, double *g, cudaStream_t st);
int read_err(Solver &S, cudaStream_t st, uint32_t *err);
/* bytes (<= 2048) from device memory to dst through the pinned h_small; waits for st */
int read_small(Solver &S, cudaStream_t st, void *dst, const void *src, size_t bytes);
int fp32_peak(int device, double *tflops, cudaStream_t st);

} // namespace tg
