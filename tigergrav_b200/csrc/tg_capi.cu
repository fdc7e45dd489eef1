/*
 * tg_capi.cu -- the C ABI (include/tigergrav_b200.h) over the solver.
 */
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include <string>

#include "tg_solver.cuh"

struct tg_solver {
    tg::Solver S;
};

namespace tg {

static thread_local char g_cuda_msg[256] = {0};

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line) {
    snprintf(g_cuda_msg, sizeof(g_cuda_msg), "%s: %s (%s:%d)", cudaGetErrorString(e), what, file, line);
    cudaGetLastError();
}

int read_err(Solver &S, cudaStream_t st, uint32_t *err) {
    TG_CUDA(cudaMemcpyAsync(S.h_err, S.dev_err.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    *err = *S.h_err;
    return TG_OK;
}

int read_small(Solver &S, cudaStream_t st, void *dst, const void *src, size_t bytes) {
    if (bytes > 2048 || !S.h_small) return TG_ERR_ARG;
    TG_CUDA(cudaMemcpyAsync(S.h_small + 2048, src, bytes, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    std::memcpy(dst, S.h_small + 2048, bytes);
    return TG_OK;
}

EwaldTables solver_tables(Solver &S);
int seam_pp(Solver *, const tg_params &, int, int, int64_t, const int64_t *, const int32_t *, const int64_t *,
            const int32_t *, double *, const EwaldTables &, cudaStream_t);
int seam_pc(const tg_params &, int, int64_t, const int64_t *, const int32_t *, const int64_t *, const float *,
            const int32_t *, double *, const EwaldTables &, cudaStream_t);
int seam_node(const tg_params &, int, int, int64_t, const int32_t *, const int64_t *, const float *, const int32_t *,
              double *, const EwaldTables &, cudaStream_t);

static std::mutex g_const_mtx;
static bool g_const_done[64] = {false};

static int ensure_constants(int dev) {
    std::lock_guard<std::mutex> lk(g_const_mtx);
    if (dev < 0 || dev >= 64) return TG_ERR_ARG;
    if (!g_const_done[dev]) {
        TG_TRY(init_constants());
        g_const_done[dev] = true;
    }
    return TG_OK;
}

static int validate(const tg_params *p) {
    if (!p) return TG_ERR_ARG;
    if (!(p->theta > 0.0) || !(p->soft_len > 0.0) || !(p->m > 0.0)) return TG_ERR_ARG;
    if (!std::isfinite(p->theta) || !std::isfinite(p->soft_len) || !std::isfinite(p->m) || !std::isfinite(p->G))
        return TG_ERR_ARG;
    if (p->leaf_max < 1 || p->leaf_max > 128) return TG_ERR_ARG;
    if (p->precision != TG_PREC_F32 && p->precision != TG_PREC_F64) return TG_ERR_ARG;
    int nd = 0;
    if (cudaGetDeviceCount(&nd) != cudaSuccess) {
        cudaGetLastError();
        return TG_ERR_CUDA;
    }
    if (p->device < 0 || p->device >= nd) return TG_ERR_ARG;
    return TG_OK;
}

__global__ void k_pack(int64_t n, const int32_t *x, const float *v, int4 *pos, float4 *vel, uint32_t *err) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pos[i] = make_int4(x[3 * i], x[3 * i + 1], x[3 * i + 2], (int)i);
    float4 q = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (v) {
        q = make_float4(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.0f);
        /* a NaN / inf velocity would drift into an undefined fixed-point position */
        if (!isfinite(q.x) || !isfinite(q.y) || !isfinite(q.z)) atomicOr(err, DEV_ERR_NONFINITE);
    }
    vel[i] = q;
}

__global__ void k_unpack(int64_t n, const int4 *pos, const float4 *vel, int32_t *x, float *v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 p = pos[i];
    const int64_t c = p.w;
    if (x) {
        x[3 * c] = p.x;
        x[3 * c + 1] = p.y;
        x[3 * c + 2] = p.z;
    }
    if (v) {
        const float4 q = vel[i];
        v[3 * c] = q.x;
        v[3 * c + 1] = q.y;
        v[3 * c + 2] = q.z;
    }
}

__global__ void k_unpack_forces(int64_t n, const int4 *pos, const float4 *acc, const double *accd, float *phi_f,
                                float *g_f, double *phi_d, double *g_d) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t c = pos[i].w;
    double a[4];
    if (accd) {
        for (int k = 0; k < 4; k++) a[k] = accd[4 * i + k];
    } else {
        const float4 q = acc[i];
        a[0] = q.x;
        a[1] = q.y;
        a[2] = q.z;
        a[3] = q.w;
    }
    if (phi_f) phi_f[c] = (float)a[0];
    if (phi_d) phi_d[c] = a[0];
    for (int d = 0; d < 3; d++) {
        if (g_f) g_f[3 * c + d] = (float)a[1 + d];
        if (g_d) g_d[3 * c + d] = a[1 + d];
    }
}

/* interaction counts and reference flops, one warp per node */
__global__ void k_count(int64_t nn, const int32_t *pb, const int32_t *pe, const int32_t *child0,
                        const int32_t *const *pools, const int64_t *const *loff, const int32_t *const *llen,
                        unsigned long long *cnt, double *flops) {
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= nn) return;
    const int64_t nsink = pe[i] - pb[i];
    if (nsink == 0) return;
    unsigned long long c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    /* node stage: CC (nodes), CP (particles) */
    for (int k = 0; k < 4; k++) {
        const int32_t len = llen[k][i];
        const int32_t *l = pools[k] + loff[k][i];
        for (int32_t j = lane; j < len; j += 32) {
            if (k == TG_CC_D || k == TG_CC_E) c[k] += 1;
            else c[k] += (unsigned long long)(pe[l[j]] - pb[l[j]]);
        }
    }
    if (child0[i] < 0) {
        for (int k = 4; k < 8; k++) {
            const int32_t len = llen[k][i];
            const int32_t *l = pools[k] + loff[k][i];
            for (int32_t j = lane; j < len; j += 32) {
                if (k == TG_PC_D || k == TG_PC_E) c[k] += 1;
                else c[k] += (unsigned long long)(pe[l[j]] - pb[l[j]]);
            }
        }
    }
    for (int k = 0; k < 8; k++)
        for (int o = 16; o > 0; o >>= 1) c[k] += __shfl_xor_sync(0xffffffffu, c[k], o);
    if (lane == 0) {
        /* kinds -> counters: 0 PP_D pairs, 1 PP_E, 2 PC_D, 3 PC_E, 4 CC_D, 5 CC_E, 6 CP_D, 7 CP_E */
        const unsigned long long pp_d = c[TG_PP_D] * nsink, pp_e = c[TG_PP_E] * nsink;
        const unsigned long long pc_d = c[TG_PC_D] * nsink, pc_e = c[TG_PC_E] * nsink;
        atomicAdd(&cnt[0], pp_d);
        atomicAdd(&cnt[1], pp_e);
        atomicAdd(&cnt[2], pc_d);
        atomicAdd(&cnt[3], pc_e);
        atomicAdd(&cnt[4], c[TG_CC_D]);
        atomicAdd(&cnt[5], c[TG_CC_E]);
        atomicAdd(&cnt[6], c[TG_CP_D]);
        atomicAdd(&cnt[7], c[TG_CP_E]);
        double f = 1025.0 * c[TG_CC_D] + 455.0 * c[TG_CP_D] + 251975.0 * c[TG_CC_E] + 251233.0 * c[TG_CP_E];
        if (child0[i] < 0) {
            f += (double)((74 + 15) * c[TG_PP_D] + 16 * 4 + 5) * nsink; /* PP_direct is called for every leaf */
            f += 581.0 * pc_d + 56245.0 * pp_e + 251531.0 * pc_e;
            f += 64.0 * nsink; /* P2M, src/tree.cpp:234 */
        }
        atomicAdd(flops, f);
    }
}

static int stage_host(Solver &S, size_t bytes) {
    if (S.h_stage_bytes >= bytes) return TG_OK;
    if (S.h_stage) cudaFreeHost(S.h_stage);
    S.h_stage = nullptr;
    S.h_stage_bytes = 0;
    if (cudaMallocHost(&S.h_stage, bytes) != cudaSuccess) {
        cudaGetLastError();
        return TG_ERR_NOMEM;
    }
    S.h_stage_bytes = bytes;
    return TG_OK;
}

/* true when the caller's host buffer is page-locked (cudaHostAlloc /
 * cudaHostRegister): it is then copied directly, without staging */
static bool is_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

/* copy a host buffer into a device buffer (pageable buffers through pinned staging) */
static int h2d(Solver &S, void *dst, const void *src, size_t bytes, cudaStream_t st) {
    if (is_pinned(src)) {
        TG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
        TG_CUDA(cudaStreamSynchronize(st));
        return TG_OK;
    }
    TG_TRY(stage_host(S, bytes));
    std::memcpy(S.h_stage, src, bytes);
    TG_CUDA(cudaMemcpyAsync(dst, S.h_stage, bytes, cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaStreamSynchronize(st));
    return TG_OK;
}
static int d2h(Solver &S, void *dst, const void *src, size_t bytes, cudaStream_t st) {
    if (is_pinned(dst)) {
        TG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
        TG_CUDA(cudaStreamSynchronize(st));
        return TG_OK;
    }
    TG_TRY(stage_host(S, bytes));
    TG_CUDA(cudaMemcpyAsync(S.h_stage, src, bytes, cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    std::memcpy(dst, S.h_stage, bytes);
    return TG_OK;
}

static int phase_ms(Solver &S, int a, int b, double *out) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, S.ev[a], S.ev[b]) != cudaSuccess) {
        cudaGetLastError();
        ms = 0.0f;
    }
    *out = ms;
    return TG_OK;
}

} // namespace tg

using namespace tg;

static inline cudaStream_t STREAM(void *s) { return (cudaStream_t)s; }

#define CHECK_HANDLE(s)                                                                        \
    do {                                                                                       \
        if (!(s)) return TG_ERR_ARG;                                                           \
        if (cudaSetDevice((s)->S.dev) != cudaSuccess) {                                        \
            cudaGetLastError();                                                                \
            return TG_ERR_CUDA;                                                                \
        }                                                                                      \
    } while (0)

extern "C" {

const char *tg_error_string(int status) {
    switch (status) {
    case TG_OK: return "ok";
    case TG_ERR_ARG: return "bad argument";
    case TG_ERR_CUDA: return g_cuda_msg[0] ? g_cuda_msg : "CUDA error";
    case TG_ERR_CAPACITY: return "interaction-list capacity exceeded";
    case TG_ERR_DEPTH: return "more than leaf_max particles in a 63-level box";
    case TG_ERR_TIMEOUT: return "bounded device wait timed out";
    case TG_ERR_STATE: return "call out of order";
    case TG_ERR_NOMEM: return "device allocation failed";
    case TG_ERR_SIZE: return "n exceeds TG_NOALLOC_MAX_N (67108864), the capacity of tg_energy_noalloc's fixed scratch";
    default: return "unknown status";
    }
}

const char *tg_version(void) { return "tigergrav_b200 0.1 (sm_100a)"; }

int tg_create(const tg_params *params, tg_solver **out) {
    if (!out) return TG_ERR_ARG;
    *out = nullptr;
    TG_TRY(validate(params));
    TG_CUDA(cudaSetDevice(params->device));
    TG_TRY(ensure_constants(params->device));
    tg_solver *h = new tg_solver();
    Solver &S = h->S;
    S.prm = *params;
    S.dev = params->device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, S.dev) == cudaSuccess) S.num_sms = prop.multiProcessorCount;
    int rc = ensure(S.dev_err, 4);
    if (rc == TG_OK) rc = ensure(S.dev_cnt, 16);
    if (rc == TG_OK && cudaMallocHost(&S.h_err, sizeof(uint32_t) * 4) != cudaSuccess) rc = TG_ERR_NOMEM;
    if (rc == TG_OK && cudaMallocHost(&S.h_cnt, sizeof(unsigned long long) * 16) != cudaSuccess) rc = TG_ERR_NOMEM;
    if (rc == TG_OK && cudaMallocHost((void **)&S.h_small, 4096) != cudaSuccess) rc = TG_ERR_NOMEM;
    if (rc == TG_OK) {
        bool ok = true;
        for (int k = 0; k < 8; k++) ok = ok && cudaEventCreate(&S.ev[k]) == cudaSuccess;
        S.have_events = ok;
        if (!ok) rc = TG_ERR_CUDA;
    }
    if (rc != TG_OK) {
        cudaGetLastError();
        tg_destroy(h);
        return rc;
    }
    *out = h;
    return TG_OK;
}

int tg_destroy(tg_solver *s) {
    if (!s) return TG_ERR_ARG;
    Solver &S = s->S;
    cudaSetDevice(S.dev);
    cudaDeviceSynchronize();
    release(S.pos); release(S.pos_alt); release(S.vel); release(S.vel_alt); release(S.acc); release(S.accd);
    release(S.keys); release(S.keys_alt); release(S.idx); release(S.idx_alt); release(S.cub_tmp);
    release(S.nd_pb); release(S.nd_pe); release(S.nd_child0); release(S.nd_parent); release(S.nd_flag);
    release(S.nd_scan); release(S.nd_key); release(S.nd_level); release(S.nd_ms); release(S.nd_r);
    release(S.nd_rmax); release(S.nd_aabb); release(S.nd_prange); release(S.nd_L); release(S.nd_Lloc);
    for (int k = 0; k < NLIST; k++) {
        release(S.loff[k]);
        release(S.llen[k]);
        release(S.pool[k]);
    }
    release(S.pool_top);
    for (int q = 0; q < 2; q++) {
        release(S.nxt_off[q]);
        release(S.nxt_len[q]);
        release(S.nxt_pool[q]);
    }
    release(S.nx_top);
    release(S.wk_pools);
    release(S.wk_llen);
    release(S.wk_loff);
    release(S.wk_caps);
    release(S.wk_wx);
    release(S.wk_kind);
    release(S.scratch); release(S.dev_err); release(S.dev_cnt);
    release(S.ew_real); release(S.ew_four); release(S.ew_Hf); release(S.ew_Hd); release(S.ew_Pf); release(S.ew_Pd);
    release(S.ew_cnt); release(S.ew_off); release(S.ew_part); release(S.ew_nt); release(S.ew_sf); release(S.ew_tpart);
    release(S.ck_x); release(S.ck_v); release(S.adj_x); release(S.adj_v); release(S.tid_u); release(S.tid_o);
    release(S.tid_U); release(S.tid_V);
    release(S.fof_P); release(S.fof_leaves); release(S.fof_key); release(S.fof_mem); release(S.fof_runs);
    release(S.fof_gmin); release(S.fof_group); release(S.fof_has); release(S.fof_pairs); release(S.fof_radii);
    release(S.fof_stats);
    release(S.rung_flag); release(S.rung_scan); release(S.rung_nact); release(S.rung_out);
    if (S.h_err) cudaFreeHost(S.h_err);
    if (S.h_cnt) cudaFreeHost(S.h_cnt);
    if (S.h_small) cudaFreeHost(S.h_small);
    if (S.h_stage) cudaFreeHost(S.h_stage);
    if (S.have_events)
        for (int k = 0; k < 8; k++) cudaEventDestroy(S.ev[k]);
    cudaGetLastError();
    delete s;
    return TG_OK;
}

int tg_set_particles(tg_solver *s, const int32_t *x, const float *v, int64_t n, int where, void *stream) {
    CHECK_HANDLE(s);
    Solver &S = s->S;
    if (!x || n < 1 || n > 0x7ffffff0ll || (where != TG_HOST && where != TG_DEVICE)) return TG_ERR_ARG;
    cudaStream_t st = STREAM(stream);
    TG_TRY(ensure(S.pos, n));
    TG_TRY(ensure(S.vel, n));
    TG_TRY(ensure(S.pos_alt, n));
    TG_TRY(ensure(S.vel_alt, n));
    const int32_t *dx = x;
    const float *dv = v;
    if (where == TG_HOST) {
        TG_TRY(h2d(S, S.pos_alt.p, x, sizeof(int32_t) * 3 * n, st));
        dx = (const int32_t *)S.pos_alt.p;
        if (v) {
            TG_TRY(h2d(S, S.vel_alt.p, v, sizeof(float) * 3 * n, st));
            dv = (const float *)S.vel_alt.p;
        }
    }
    if (dv) TG_CUDA(cudaMemsetAsync(S.dev_err.p, 0, sizeof(uint32_t), st));
    k_pack<<<(int)((n + 255) / 256), 256, 0, st>>>(n, dx, dv, S.pos.p, S.vel.p, S.dev_err.p);
    TG_TRY(launched(S));
    S.have_tree = S.have_multipoles = S.have_lists = S.have_forces = false;
    if (dv) {
        uint32_t err = 0;
        TG_TRY(read_err(S, st, &err));
        if (err & DEV_ERR_NONFINITE) {
            S.n = 0; /* nothing loaded: later calls answer TG_ERR_STATE */
            return TG_ERR_ARG;
        }
    }
    S.n = n;
    S.st.n = n;
    return TG_OK;
}

int tg_get_particles(tg_solver *s, int32_t *x, float *v, int where, void *stream) {
    CHECK_HANDLE(s);
    Solver &S = s->S;
    if (S.n <= 0) return TG_ERR_STATE;
    cudaStream_t st = STREAM(stream);
    const int64_t n = S.n;
    if (where == TG_DEVICE) {
        k_unpack<<<(int)((n + 255) / 256), 256, 0, st>>>(n, S.pos.p, S.vel.p, x, v);
        TG_TRY(launched(S));
        return TG_OK;
    }
    TG_TRY(ensure(S.pos_alt, n));
    TG_TRY(ensure(S.vel_alt, n));
    int32_t *tx = (int32_t *)S.pos_alt.p;
    float *tv = (float *)S.vel_alt.p;
    k_unpack<<<(int)((n + 255) / 256), 256, 0, st>>>(n, S.pos.p, S.vel.p, x ? tx : nullptr, v ? tv : nullptr);
    TG_TRY(launched(S));
    if (x) TG_TRY(d2h(S, x, tx, sizeof(int32_t) * 3 * n, st));
    if (v) TG_TRY(d2h(S, v, tv, sizeof(float) * 3 * n, st));
    return TG_OK;
}

int tg_build(tg_solver *s, void *stream) {
    CHECK_HANDLE(s);
    Solver &S = s->S;
    if (S.n <= 0) return TG_ERR_STATE;
    cudaStream_t st = STREAM(stream);
    if (S.have_events) TG_CUDA(cudaEventRecord(S.ev[0], st));
    S.kd_timed = S.kd_pending; /* ev[7] .. ev[0]: the fused kick-drift before this build */
    S.kd_pending = false;
    TG_TRY(tree_build(S, st));
    if (S.have_events) TG_CUDA(cudaEventRecord(S.ev[1], st));
    return TG_OK;
}

int tg_multipoles(tg_solver *s, void *stream) {
    CHECK_HANDLE(s);
    Solver &S = s->S;
    cudaStream_t st = STREAM(stream);
    TG_TRY(tree_multipoles(S, st));
    if (S.have_events) TG_CUDA(cudaEventRecord(S.ev[2], st));
    return TG_OK;
}

int tg_walk(tg_solver *s, void *stream) {
    CHECK_HANDLE(s);
    return tree_walk(s->S, STREAM(stream));
}

int tg_set_walk_capacity(tg_solver *s, int64_t entries) {
    CHECK_HANDLE(s);
    if (entries < 0) return TG_ERR_ARG;
    tg::Solver &S = s->S;
    S.cap_start = entries;
    for (int k = 0; k < tg::NLIST; k++) S.list_cap[k] = 0;
    S.nx_cap[0] = S.nx_cap[1] = 0;
    if (entries > 0) S.scratch_per_warp = 0;
    return TG_OK;
}

int tg_forces(tg_solver *s, void *stream) {
    CHECK_HANDLE(s);
    return gravity_forces(s->S, STREAM(stream));
}

int tg_solve_gravity(tg_solver *s, void *stream) {
    CHECK_HANDLE(s);
    TG_TRY(tg_build(s, stream));
    TG_TRY(tg_multipoles(s, stream));
    TG_TRY(tg_walk(s, stream));
    TG_TRY(tg_forces(s, stream));
    return TG_OK;
}

static int get_forces_impl(tg_solver *s, float *phi_f, float *g_f, double *phi_d, double *g_d, int where,
                           void *stream) {
    CHECK_HANDLE(s);
    Solver &S = s->S;
    if (!S.have_forces) return TG_ERR_STATE;
    cudaStream_t st = STREAM(stream);
    const int64_t n = S.n;
    const bool f64 = S.prm.precision == TG_PREC_F64;
    if (where == TG_DEVICE) {
        k_unpack_forces<<<(int)((n + 255) / 256), 256, 0, st>>>(n, S.pos.p, f64 ? nullptr : S.acc.p,
                                                                f64 ? S.accd.p : nullptr, phi_f, g_f, phi_d, g_d);
        TG_TRY(launched(S));
        return TG_OK;
    }
    /* host: unpack into device scratch (keys/keys_alt hold >= 8n bytes each) then copy */
    const size_t es = phi_d || g_d ? sizeof(double) : sizeof(float);
    TG_TRY(ensure(S.keys_alt, (size_t)4 * n * es / 8 + 8));
    char *tmp = (char *)S.keys_alt.p;
    void *tphi = tmp, *tg = tmp + es * n;
    k_unpack_forces<<<(int)((n + 255) / 256), 256, 0, st>>>(
        n, S.pos.p, f64 ? nullptr : S.acc.p, f64 ? S.accd.p : nullptr, phi_f ? (float *)tphi : nullptr,
        g_f ? (float *)tg : nullptr, phi_d ? (double *)tphi : nullptr, g_d ? (double *)tg : nullptr);
    TG_TRY(launched(S));
    if (phi_f) TG_TRY(d2h(S, phi_f, tphi, sizeof(float) * n, st));
    if (g_f) TG_TRY(d2h(S, g_f, tg, sizeof(float) * 3 * n, st));
    if (phi_d) TG_TRY(d2h(S, phi_d, tphi, sizeof(double) * n, st));
    if (g_d) TG_TRY(d2h(S, g_d, tg, sizeof(double) * 3 * n, st));
    return TG_OK;
}

int tg_get_forces(tg_solver *s, float *phi, float *g, int where, void *stream) {
    return get_forces_impl(s, phi, g, nullptr, nullptr, where, stream);
}
int tg_get_forces_f64(tg_solver *s, double *phi, double *g, int where, void *stream) {
    return get_forces_impl(s, nullptr, nullptr, phi, g, where, stream);
}

int tg_kick(tg_solver *s, double dt, void *stream) {
    CHECK_HANDLE(s);
    if (!std::isfinite(dt)) return TG_ERR_ARG;
    return kick(s->S, dt, STREAM(stream));
}

int tg_drift(tg_solver *s, double dt, void *stream) {
    CHECK_HANDLE(s);
    if (!std::isfinite(dt)) return TG_ERR_ARG;
    return drift(s->S, dt, STREAM(stream));
}

int tg_energy(tg_solver *s, double out[5], void *stream) {
    CHECK_HANDLE(s);
    if (!out) return TG_ERR_ARG;
    return energy(s->S, out, STREAM(stream));
}

int tg_kick_drift(tg_solver *s, double dt_close, double dt_open, double dt_drift, void *stream) {
    CHECK_HANDLE(s);
    if (!std::isfinite(dt_close) || !std::isfinite(dt_open) || !std::isfinite(dt_drift)) return TG_ERR_ARG;
    if (s->S.n <= 0) return TG_ERR_STATE;
    cudaStream_t st = STREAM(stream);
    if (s->S.have_events) TG_CUDA(cudaEventRecord(s->S.ev[7], st));
    TG_TRY(kick_drift(s->S, dt_close, dt_open, dt_drift, st));
    s->S.kd_pending = true;
    return TG_OK;
}

int tg_leapfrog(tg_solver *s, double dt, int n_steps, void *stream) {
    CHECK_HANDLE(s);
    if (n_steps < 0 || !std::isfinite(dt)) return TG_ERR_ARG;
    if (!s->S.have_forces) TG_TRY(tg_solve_gravity(s, stream));
    if (n_steps == 0) return TG_OK;
    /* K D [solve] K per step, with each step's closing kick fused with the
     * next step's opening kick and drift: the same arithmetic as kick, drift,
     * solve, kick */
    TG_TRY(tg_kick_drift(s, 0.0, 0.5 * dt, dt, stream));
    for (int k = 0; k < n_steps; k++) {
        TG_TRY(tg_solve_gravity(s, stream));
        if (k + 1 < n_steps) TG_TRY(tg_kick_drift(s, 0.5 * dt, 0.5 * dt, dt, stream));
        else TG_TRY(tg_kick(s, 0.5 * dt, stream));
    }
    return TG_OK;
}

/* ---- differentiation ---- */

int tg_forward(tg_solver *s, double dt, int n_steps, void *stream) {
    CHECK_HANDLE(s);
    Solver &S = s->S;
    if (n_steps < 0 || !std::isfinite(dt) || S.n <= 0) return TG_ERR_ARG;
    cudaStream_t st = STREAM(stream);
    const int64_t n = S.n;
    TG_TRY(ensure(S.ck_x, (size_t)3 * n * (n_steps + 1)));
    TG_TRY(ensure(S.ck_v, (size_t)3 * n * (n_steps + 1)));
    S.ck_steps = -1;
    if (!S.have_forces) TG_TRY(tg_solve_gravity(s, stream));
    const int gn = (int)((n + 255) / 256);
    k_unpack<<<gn, 256, 0, st>>>(n, S.pos.p, S.vel.p, S.ck_x.p, S.ck_v.p);
    TG_TRY(launched(S));
    for (int k = 0; k < n_steps; k++) {
        TG_TRY(tg_kick(s, 0.5 * dt, stream));
        TG_TRY(tg_drift(s, dt, stream));
        TG_TRY(tg_solve_gravity(s, stream));
        TG_TRY(tg_kick(s, 0.5 * dt, stream));
        k_unpack<<<gn, 256, 0, st>>>(n, S.pos.p, S.vel.p, S.ck_x.p + (size_t)3 * n * (k + 1),
                                     S.ck_v.p + (size_t)3 * n * (k + 1));
        TG_TRY(launched(S));
    }
    S.ck_steps = n_steps;
    S.ck_dt = dt;
    return TG_OK;
}

/* tree, multipoles and lists at checkpoint k */
static int at_checkpoint(tg_solver *s, int k, cudaStream_t st) {
    Solver &S = s->S;
    const int64_t n = S.n;
    k_pack<<<(int)((n + 255) / 256), 256, 0, st>>>(n, S.ck_x.p + (size_t)3 * n * k, S.ck_v.p + (size_t)3 * n * k,
                                                   S.pos.p, S.vel.p, S.dev_err.p); /* checkpoints are finite */
    TG_TRY(launched(S));
    S.have_tree = S.have_multipoles = S.have_lists = S.have_forces = false;
    TG_TRY(tg_build(s, st));
    TG_TRY(tg_multipoles(s, st));
    TG_TRY(tg_walk(s, st));
    return TG_OK;
}

int tg_backward(tg_solver *s, const double *gx, const double *gv, double *gx0, double *gv0, int where, void *stream) {
    CHECK_HANDLE(s);
    Solver &S = s->S;
    if (S.ck_steps < 0) return TG_ERR_STATE;
    if (!gx || !gx0 || (where != TG_HOST && where != TG_DEVICE)) return TG_ERR_ARG;
    cudaStream_t st = STREAM(stream);
    const int64_t n = S.n;
    const size_t bytes = sizeof(double) * 3 * n;
    const int K = S.ck_steps;
    const double dt = S.ck_dt, G = S.prm.G;
    TG_TRY(ensure(S.adj_x, 3 * n));
    TG_TRY(ensure(S.adj_v, 3 * n));
    const cudaMemcpyKind in = where == TG_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const cudaMemcpyKind out = where == TG_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    TG_CUDA(cudaMemcpyAsync(S.adj_x.p, gx, bytes, in, st));
    if (gv) TG_CUDA(cudaMemcpyAsync(S.adj_v.p, gv, bytes, in, st));
    else TG_CUDA(cudaMemsetAsync(S.adj_v.p, 0, bytes, st));
    const int gn3 = (int)((3 * n + 255) / 256);
    if (gv) {
        TG_TRY(at_checkpoint(s, K, st));
        TG_TRY(tidal_apply(S, S.adj_v.p, S.adj_x.p, 0.5 * dt * G, st));
    }
    for (int k = K - 1; k >= 0; k--) {
        k_axpy3<<<gn3, 256, 0, st>>>(n, dt, S.adj_x.p, S.adj_v.p);
        TG_TRY(launched(S));
        TG_TRY(at_checkpoint(s, k, st));
        TG_TRY(tidal_apply(S, S.adj_v.p, S.adj_x.p, (k > 0 ? dt : 0.5 * dt) * G, st));
    }
    TG_CUDA(cudaMemcpyAsync(gx0, S.adj_x.p, bytes, out, st));
    if (gv0) TG_CUDA(cudaMemcpyAsync(gv0, S.adj_v.p, bytes, out, st));
    TG_CUDA(cudaStreamSynchronize(st));
    return TG_OK;
}

int tg_tidal(tg_solver *s, const double *u, double *out, int where, void *stream) {
    CHECK_HANDLE(s);
    Solver &S = s->S;
    if (!u || !out || (where != TG_HOST && where != TG_DEVICE)) return TG_ERR_ARG;
    if (!S.have_lists) return TG_ERR_STATE;
    cudaStream_t st = STREAM(stream);
    const int64_t n = S.n;
    const size_t bytes = sizeof(double) * 3 * n;
    TG_TRY(ensure(S.adj_x, 3 * n));
    TG_TRY(ensure(S.adj_v, 3 * n));
    TG_CUDA(cudaMemcpyAsync(S.adj_v.p, u, bytes, where == TG_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                            st));
    TG_CUDA(cudaMemsetAsync(S.adj_x.p, 0, bytes, st));
    TG_TRY(tidal_apply(S, S.adj_v.p, S.adj_x.p, 1.0, st));
    TG_CUDA(cudaMemcpyAsync(out, S.adj_x.p, bytes, where == TG_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                            st));
    TG_CUDA(cudaStreamSynchronize(st));
    return TG_OK;
}

int tg_get_stats(tg_solver *s, tg_stats *out) {
    CHECK_HANDLE(s);
    if (!out) return TG_ERR_ARG;
    Solver &S = s->S;
    S.st.n = S.n;
    S.st.nodes = S.nnodes;
    S.st.depth = S.depth;
    if (S.have_lists) {
        cudaStream_t st = 0;
        TG_CUDA(cudaDeviceSynchronize());
        DevBuf<const int32_t *> d_pools;
        DevBuf<const int64_t *> d_loff;
        DevBuf<const int32_t *> d_llen;
        DevBuf<double> d_fl;
        TG_TRY(ensure(d_pools, NLIST));
        TG_TRY(ensure(d_loff, NLIST));
        TG_TRY(ensure(d_llen, NLIST));
        TG_TRY(ensure(d_fl, 1));
        const int32_t *hp[NLIST], *hl[NLIST];
        const int64_t *ho[NLIST];
        for (int k = 0; k < NLIST; k++) {
            hp[k] = S.pool[k].p;
            hl[k] = S.llen[k].p;
            ho[k] = S.loff[k].p;
        }
        TG_CUDA(cudaMemcpy(d_pools.p, hp, sizeof(hp), cudaMemcpyHostToDevice));
        TG_CUDA(cudaMemcpy(d_loff.p, ho, sizeof(ho), cudaMemcpyHostToDevice));
        TG_CUDA(cudaMemcpy(d_llen.p, hl, sizeof(hl), cudaMemcpyHostToDevice));
        TG_CUDA(cudaMemset(S.dev_cnt.p, 0, sizeof(unsigned long long) * 16));
        TG_CUDA(cudaMemset(d_fl.p, 0, sizeof(double)));
        const int64_t nn = S.nnodes;
        k_count<<<(int)((nn * 32 + 127) / 128), 128, 0, st>>>(nn, S.nd_pb.p, S.nd_pe.p, S.nd_child0.p, d_pools.p,
                                                              d_loff.p, d_llen.p, S.dev_cnt.p, d_fl.p);
        TG_CUDA(cudaGetLastError());
        unsigned long long c[8];
        double fl = 0;
        TG_CUDA(cudaMemcpy(c, S.dev_cnt.p, sizeof(c), cudaMemcpyDeviceToHost));
        TG_CUDA(cudaMemcpy(&fl, d_fl.p, sizeof(double), cudaMemcpyDeviceToHost));
        release(d_pools);
        release(d_loff);
        release(d_llen);
        release(d_fl);
        for (int k = 0; k < 8; k++) S.st.counts[k] = c[k];
        S.st.flops = fl;
        /* reference filing: PC counted under CP (src/tree.cpp:618,627) */
        S.st.ref_stats[0] = c[0];
        S.st.ref_stats[1] = c[1];
        S.st.ref_stats[2] = c[4];
        S.st.ref_stats[3] = c[5];
        S.st.ref_stats[4] = c[6] + c[2];
        S.st.ref_stats[5] = c[7] + c[3];
    }
    if (S.have_events && S.have_forces) {
        phase_ms(S, 0, 1, &S.st.ms_build);
        phase_ms(S, 1, 2, &S.st.ms_multipoles);
        phase_ms(S, 2, 3, &S.st.ms_walk);
        phase_ms(S, 3, 4, &S.st.ms_nodes);
        phase_ms(S, 4, 5, &S.st.ms_leaves);
        S.st.ms_pp = 0.0;
        if (S.pp_timed) phase_ms(S, 6, 5, &S.st.ms_pp);
        S.st.ms_kick_drift = 0.0;
        if (S.kd_timed) phase_ms(S, 7, 0, &S.st.ms_kick_drift);
    }
    S.st.launches = S.launches;
    S.st.device_bytes = (int64_t)g_dev_bytes.load();
    *out = S.st;
    return TG_OK;
}

int tg_memory_report(tg_solver *s, char *buf, int64_t cap) {
    if (!s || !buf || cap < 1) return TG_ERR_ARG;
    Solver &S = s->S;
    std::string out;
    int64_t total = 0;
    auto add = [&](const char *name, size_t bytes) {
        if (!bytes) return;
        total += (int64_t)bytes;
        out += name;
        out += " " + std::to_string(bytes) + "\n";
    };
#define TG_MEM(b) add(#b, S.b.n * sizeof(*S.b.p))
    TG_MEM(pos); TG_MEM(pos_alt); TG_MEM(vel); TG_MEM(vel_alt); TG_MEM(acc); TG_MEM(accd); TG_MEM(keys);
    TG_MEM(keys_alt); TG_MEM(idx); TG_MEM(idx_alt); TG_MEM(cub_tmp); TG_MEM(nd_pb); TG_MEM(nd_pe); TG_MEM(nd_child0);
    TG_MEM(nd_parent); TG_MEM(nd_flag); TG_MEM(nd_scan); TG_MEM(nd_key); TG_MEM(nd_level); TG_MEM(nd_ms);
    TG_MEM(nd_r); TG_MEM(nd_rmax); TG_MEM(nd_aabb); TG_MEM(nd_prange); TG_MEM(nd_L); TG_MEM(nd_Lloc);
    TG_MEM(loff[0]); TG_MEM(llen[0]); TG_MEM(pool[0]); TG_MEM(pool[1]); TG_MEM(pool[2]); TG_MEM(pool[3]);
    TG_MEM(pool[4]); TG_MEM(pool[5]); TG_MEM(pool[6]); TG_MEM(pool[7]); TG_MEM(nxt_pool[0]); TG_MEM(nxt_pool[1]);
    TG_MEM(nxt_off[0]); TG_MEM(nxt_len[0]); TG_MEM(scratch); TG_MEM(ew_cnt); TG_MEM(ew_off); TG_MEM(ew_part);
    TG_MEM(ew_nt); TG_MEM(ew_sf); TG_MEM(ew_tpart); TG_MEM(ck_x); TG_MEM(ck_v); TG_MEM(adj_x); TG_MEM(adj_v);
    TG_MEM(tid_u); TG_MEM(tid_o); TG_MEM(tid_U); TG_MEM(tid_V); TG_MEM(fof_P); TG_MEM(fof_key); TG_MEM(fof_mem);
    TG_MEM(fof_pairs); TG_MEM(rung_flag); TG_MEM(rung_scan); TG_MEM(rung_nact);
#undef TG_MEM
    out += "total " + std::to_string(total) + "\n";
    if ((int64_t)out.size() + 1 > cap) return TG_ERR_SIZE;
    std::memcpy(buf, out.c_str(), out.size() + 1);
    return TG_OK;
}

int64_t tg_num_nodes(tg_solver *s) {
    if (!s) return -1;
    return s->S.have_tree ? s->S.nnodes : 0;
}

int tg_get_nodes(tg_solver *s, uint64_t *boxid, int32_t *level, int64_t *pbegin, int64_t *pend, int32_t *child0,
                 int32_t *parent, int32_t *x, float *r, float *rmax, float *m) {
    CHECK_HANDLE(s);
    Solver &S = s->S;
    if (!S.have_tree) return TG_ERR_STATE;
    TG_CUDA(cudaDeviceSynchronize());
    const int64_t nn = S.nnodes;
    std::vector<int32_t> pb(nn), pe(nn), c0(nn), par(nn);
    std::vector<unsigned long long> key(nn);
    std::vector<unsigned char> lv(nn);
    TG_CUDA(cudaMemcpy(pb.data(), S.nd_pb.p, 4 * nn, cudaMemcpyDeviceToHost));
    TG_CUDA(cudaMemcpy(pe.data(), S.nd_pe.p, 4 * nn, cudaMemcpyDeviceToHost));
    TG_CUDA(cudaMemcpy(c0.data(), S.nd_child0.p, 4 * nn, cudaMemcpyDeviceToHost));
    TG_CUDA(cudaMemcpy(par.data(), S.nd_parent.p, 4 * nn, cudaMemcpyDeviceToHost));
    TG_CUDA(cudaMemcpy(key.data(), S.nd_key.p, 8 * nn, cudaMemcpyDeviceToHost));
    TG_CUDA(cudaMemcpy(lv.data(), S.nd_level.p, nn, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < nn; i++) {
        const int L = lv[i];
        if (boxid) boxid[i] = L == 0 ? 1ull : ((1ull << L) | (key[i] >> (63 - L)));
        if (level) level[i] = L;
        if (pbegin) pbegin[i] = pb[i];
        if (pend) pend[i] = pe[i];
        if (child0) child0[i] = c0[i];
        if (parent) parent[i] = par[i];
    }
    if (S.have_multipoles) {
        std::vector<MSrc> ms(nn);
        TG_CUDA(cudaMemcpy(ms.data(), S.nd_ms.p, sizeof(MSrc) * nn, cudaMemcpyDeviceToHost));
        if (r) TG_CUDA(cudaMemcpy(r, S.nd_r.p, 4 * nn, cudaMemcpyDeviceToHost));
        if (rmax) TG_CUDA(cudaMemcpy(rmax, S.nd_rmax.p, 4 * nn, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < nn; i++) {
            if (x)
                for (int d = 0; d < 3; d++) x[3 * i + d] = ms[i].x[d];
            if (m)
                for (int q = 0; q < MP; q++) m[MP * i + q] = ms[i].m[q];
        }
    }
    return TG_OK;
}

int tg_get_perm(tg_solver *s, int64_t *perm) {
    CHECK_HANDLE(s);
    Solver &S = s->S;
    if (!perm || S.n <= 0) return TG_ERR_ARG;
    TG_CUDA(cudaDeviceSynchronize());
    std::vector<int4> p(S.n);
    TG_CUDA(cudaMemcpy(p.data(), S.pos.p, sizeof(int4) * S.n, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < S.n; i++) perm[i] = p[i].w;
    return TG_OK;
}

int64_t tg_list_size(tg_solver *s, int kind) {
    if (!s || kind < 0 || kind >= NLIST || !s->S.have_lists) return -1;
    Solver &S = s->S;
    if (cudaSetDevice(S.dev) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    std::vector<int32_t> len(S.nnodes);
    if (cudaMemcpy(len.data(), S.llen[kind].p, 4 * S.nnodes, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    int64_t tot = 0;
    for (auto l : len) tot += l;
    return tot;
}

int tg_get_list(tg_solver *s, int kind, int64_t *offsets, int32_t *ids) {
    CHECK_HANDLE(s);
    Solver &S = s->S;
    if (kind < 0 || kind >= NLIST || !offsets) return TG_ERR_ARG;
    if (!S.have_lists) return TG_ERR_STATE;
    TG_CUDA(cudaDeviceSynchronize());
    const int64_t nn = S.nnodes;
    std::vector<int32_t> len(nn);
    std::vector<int64_t> off(nn);
    TG_CUDA(cudaMemcpy(len.data(), S.llen[kind].p, 4 * nn, cudaMemcpyDeviceToHost));
    TG_CUDA(cudaMemcpy(off.data(), S.loff[kind].p, 8 * nn, cudaMemcpyDeviceToHost));
    int64_t o = 0;
    for (int64_t i = 0; i < nn; i++) {
        offsets[i] = o;
        if (ids && len[i] > 0) TG_CUDA(cudaMemcpy(ids + o, S.pool[kind].p + off[i], 4 * len[i], cudaMemcpyDeviceToHost));
        o += len[i];
    }
    offsets[nn] = o;
    return TG_OK;
}

/* ---- kernel-level seams ---- */
struct SeamTables {
    Solver S;
    bool ready = false;
};
static std::mutex g_seam_mtx;
static SeamTables *g_seam[64] = {nullptr};

static int seam_tables(int dev, EwaldTables *E, cudaStream_t st) {
    std::lock_guard<std::mutex> lk(g_seam_mtx);
    if (dev < 0 || dev >= 64) return TG_ERR_ARG;
    if (!g_seam[dev]) g_seam[dev] = new SeamTables();
    if (!g_seam[dev]->ready) {
        TG_TRY(ewald_tables(g_seam[dev]->S, st));
        g_seam[dev]->ready = true;
    }
    *E = solver_tables(g_seam[dev]->S);
    return TG_OK;
}

#define SEAM_PROLOGUE()                                                                        \
    TG_TRY(validate(params));                                                                  \
    TG_CUDA(cudaSetDevice(params->device));                                                    \
    TG_TRY(ensure_constants(params->device));                                                  \
    if (ngroups < 0) return TG_ERR_ARG;                                                        \
    if (ngroups == 0) return TG_OK;                                                            \
    EwaldTables E;                                                                             \
    TG_TRY(seam_tables(params->device, &E, STREAM(stream)));

static void seam_flops(uint64_t *flops, const int64_t *sink_off, const int64_t *src_off, int64_t ngroups, int kind,
                       int do_phi) {
    if (!flops) return;
    std::vector<int64_t> so(ngroups + 1), yo(ngroups + 1);
    if (sink_off) cudaMemcpy(so.data(), sink_off, 8 * (ngroups + 1), cudaMemcpyDeviceToHost);
    cudaMemcpy(yo.data(), src_off, 8 * (ngroups + 1), cudaMemcpyDeviceToHost);
    uint64_t f = 0;
    for (int64_t g = 0; g < ngroups; g++) {
        const uint64_t nx = sink_off ? (uint64_t)(so[g + 1] - so[g]) : 1, ny = (uint64_t)(yo[g + 1] - yo[g]);
        switch (kind) {
        case 0: f += nx ? ((74 + (do_phi ? 15 : 0)) * ny + 16 * 4 + 5) * nx : 0; break; /* PP_direct */
        case 1: f += 56245ull * ny * nx; break;
        case 2: f += 581ull * ny * nx; break;
        case 3: f += 251531ull * ny * nx; break;
        case 4: f += 1025ull * ny; break;
        case 5: f += 251975ull * ny; break;
        case 6: f += 455ull * ny; break;
        case 7: f += 251233ull * ny; break;
        }
    }
    *flops = f;
}

int tg_gravity_PP_direct(const tg_params *params, int64_t ngroups, const int64_t *sink_off, const int32_t *sink_x,
                         const int64_t *src_off, const int32_t *src_x, double *f, int do_phi, uint64_t *flops,
                         void *stream) {
    SEAM_PROLOGUE();
    TG_TRY(seam_pp(nullptr, *params, 0, do_phi, ngroups, sink_off, sink_x, src_off, src_x, f, E, STREAM(stream)));
    seam_flops(flops, sink_off, src_off, ngroups, 0, do_phi);
    return TG_OK;
}
int tg_gravity_PP_ewald(const tg_params *params, int64_t ngroups, const int64_t *sink_off, const int32_t *sink_x,
                        const int64_t *src_off, const int32_t *src_x, double *f, uint64_t *flops, void *stream) {
    SEAM_PROLOGUE();
    TG_TRY(seam_pp(nullptr, *params, 1, 1, ngroups, sink_off, sink_x, src_off, src_x, f, E, STREAM(stream)));
    seam_flops(flops, sink_off, src_off, ngroups, 1, 1);
    return TG_OK;
}
int tg_gravity_PC_direct(const tg_params *params, int64_t ngroups, const int64_t *sink_off, const int32_t *sink_x,
                         const int64_t *src_off, const float *src_m, const int32_t *src_x, double *f, uint64_t *flops,
                         void *stream) {
    SEAM_PROLOGUE();
    TG_TRY(seam_pc(*params, 0, ngroups, sink_off, sink_x, src_off, src_m, src_x, f, E, STREAM(stream)));
    seam_flops(flops, sink_off, src_off, ngroups, 2, 1);
    return TG_OK;
}
int tg_gravity_PC_ewald(const tg_params *params, int64_t ngroups, const int64_t *sink_off, const int32_t *sink_x,
                        const int64_t *src_off, const float *src_m, const int32_t *src_x, double *f, uint64_t *flops,
                        void *stream) {
    SEAM_PROLOGUE();
    TG_TRY(seam_pc(*params, 1, ngroups, sink_off, sink_x, src_off, src_m, src_x, f, E, STREAM(stream)));
    seam_flops(flops, sink_off, src_off, ngroups, 3, 1);
    return TG_OK;
}
int tg_gravity_CC_direct(const tg_params *params, int64_t ngroups, const int32_t *sink_x, const int64_t *src_off,
                         const float *src_m, const int32_t *src_x, double *L, uint64_t *flops, void *stream) {
    SEAM_PROLOGUE();
    TG_TRY(seam_node(*params, 0, 1, ngroups, sink_x, src_off, src_m, src_x, L, E, STREAM(stream)));
    seam_flops(flops, nullptr, src_off, ngroups, 4, 1);
    return TG_OK;
}
int tg_gravity_CC_ewald(const tg_params *params, int64_t ngroups, const int32_t *sink_x, const int64_t *src_off,
                        const float *src_m, const int32_t *src_x, double *L, uint64_t *flops, void *stream) {
    SEAM_PROLOGUE();
    TG_TRY(seam_node(*params, 1, 1, ngroups, sink_x, src_off, src_m, src_x, L, E, STREAM(stream)));
    seam_flops(flops, nullptr, src_off, ngroups, 5, 1);
    return TG_OK;
}
int tg_gravity_CP_direct(const tg_params *params, int64_t ngroups, const int32_t *sink_x, const int64_t *src_off,
                         const int32_t *src_x, double *L, uint64_t *flops, void *stream) {
    SEAM_PROLOGUE();
    TG_TRY(seam_node(*params, 0, 0, ngroups, sink_x, src_off, nullptr, src_x, L, E, STREAM(stream)));
    seam_flops(flops, nullptr, src_off, ngroups, 6, 1);
    return TG_OK;
}
int tg_gravity_CP_ewald(const tg_params *params, int64_t ngroups, const int32_t *sink_x, const int64_t *src_off,
                        const int32_t *src_x, double *L, uint64_t *flops, void *stream) {
    SEAM_PROLOGUE();
    TG_TRY(seam_node(*params, 1, 0, ngroups, sink_x, src_off, nullptr, src_x, L, E, STREAM(stream)));
    seam_flops(flops, nullptr, src_off, ngroups, 7, 1);
    return TG_OK;
}

int tg_device_fp32_peak(int device, double *tflops, void *stream) {
    if (!tflops) return TG_ERR_ARG;
    TG_CUDA(cudaSetDevice(device));
    return fp32_peak(device, tflops, STREAM(stream));
}

int tg_truth(tg_solver *s, const int64_t *samples, int64_t ns, double alpha, double *phi, double *g, void *stream) {
    CHECK_HANDLE(s);
    if (!samples || ns <= 0) return TG_ERR_ARG;
    return truth(s->S, samples, ns, alpha, phi, g, STREAM(stream));
}

} // extern "C"
