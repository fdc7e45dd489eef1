/*
 * tg_noalloc.cu -- energy and momentum reductions that allocate nothing.
 *
 * tg_energy reduces over a solver's particles with a scratch buffer it
 * allocates with cudaMalloc.  Some callers cannot allocate device memory at
 * the point they need the reduction: a host code that hands this library
 * a fixed memory arena up front (and forbids allocation in its time loop),
 * a caller whose device memory is already committed to its own particle
 * arrays, or code running where an allocation would synchronise the device.
 * tg_energy_noalloc serves them: the caller passes its own velocity and
 * potential arrays and an output slot, and the per-block partial sums live
 * in a fixed array compiled into the library (g_noalloc_scratch below,
 * 2.5 MiB, held by every GPU that loads the library until the process
 * exits).  Its size caps n at TG_NOALLOC_MAX_N particles.
 *
 * Host code cannot use g_noalloc_scratch as a device address (in host code
 * the name is a host-side stand-in): the first call on each device looks up
 * the array's device address with cudaGetSymbolAddress, with that device
 * current, and caches it.  Make that first call before any stream capture.
 *
 * Every call writes every partial it later reads, so nothing has to start
 * at zero; the array keeps the last call's partial sums.  All calls share
 * the one array, so calls that overlap on the GPU (different streams or
 * host threads without ordering between them) race and must be avoided.
 */
#include <mutex>

#include "tg_solver.cuh"

namespace tg {

constexpr int NOALLOC_CHUNK = 1024; /* particles reduced per partial (256 threads x 4) */
constexpr int64_t NOALLOC_MAX_PARTS = TG_NOALLOC_MAX_N / NOALLOC_CHUNK;

static __device__ __align__(256) double g_noalloc_scratch[5 * NOALLOC_MAX_PARTS];

static std::mutex g_noalloc_mtx;
static double *g_noalloc_ptr[64] = {nullptr};

/* device address of g_noalloc_scratch on the current device (set up once) */
static int noalloc_scratch(int dev, double **out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mtx);
    if (dev < 0 || dev >= 64) return TG_ERR_ARG;
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            set_last_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
            return TG_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = (double *)p;
    }
    *out = g_noalloc_ptr[dev];
    return TG_OK;
}

/* one block per NOALLOC_CHUNK particles: E_kin, E_pot, sum v (x, y, z) */
__global__ void k_energy_noalloc_partial(int64_t n, const float *__restrict__ v, const float *__restrict__ phi,
                                         double m, double G, double *__restrict__ part) {
    __shared__ double sh[5][256];
    double e[5] = {0, 0, 0, 0, 0};
    const int64_t base = (int64_t)blockIdx.x * NOALLOC_CHUNK;
    for (int k = threadIdx.x; k < NOALLOC_CHUNK; k += blockDim.x) {
        const int64_t i = base + k;
        if (i >= n) break;
        const double vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2];
        e[0] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
        if (phi) e[1] += 0.5 * m * (double)phi[i] * G;
        e[2] += vx;
        e[3] += vy;
        e[4] += vz;
    }
    for (int k = 0; k < 5; k++) sh[k][threadIdx.x] = e[k];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int k = 0; k < 5; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 5; k++) part[5 * (int64_t)blockIdx.x + k] = sh[k][0];
}

__global__ void k_energy_noalloc_final(int64_t nparts, const double *__restrict__ part, int64_t n,
                                       double *__restrict__ out) {
    __shared__ double sh[5][256];
    double e[5] = {0, 0, 0, 0, 0};
    for (int64_t b = threadIdx.x; b < nparts; b += blockDim.x)
        for (int k = 0; k < 5; k++) e[k] += part[5 * b + k];
    for (int k = 0; k < 5; k++) sh[k][threadIdx.x] = e[k];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int k = 0; k < 5; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sh[0][0];
        out[1] = sh[1][0];
        for (int k = 2; k < 5; k++) out[k] = sh[k][0] / (double)n;
    }
}

/* the launches of one call, with `device` current */
static int energy_noalloc_on(const float *v, const float *phi, int64_t n, double m, double G, double *out,
                             int device, cudaStream_t st) {
    double *part = nullptr;
    TG_TRY(noalloc_scratch(device, &part));
    const int64_t nparts = (n + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK;
    k_energy_noalloc_partial<<<(unsigned)nparts, 256, 0, st>>>(n, v, phi, m, G, part);
    TG_CUDA(cudaGetLastError());
    k_energy_noalloc_final<<<1, 256, 0, st>>>(nparts, part, n, out);
    TG_CUDA(cudaGetLastError());
    return TG_OK;
}

} // namespace tg

extern "C" int tg_energy_noalloc(const float *v, const float *phi, int64_t n, double m, double G, double *out,
                                 int device, void *stream) {
    using namespace tg;
    if (!v || !out || n < 1 || !std::isfinite(m) || !std::isfinite(G)) return TG_ERR_ARG;
    if (n > TG_NOALLOC_MAX_N) return TG_ERR_SIZE;
    /* the caller's thread keeps its current device: switch only for the call */
    int prev = -1;
    TG_CUDA(cudaGetDevice(&prev));
    if (prev != device) TG_CUDA(cudaSetDevice(device));
    const int rc = energy_noalloc_on(v, phi, n, m, G, out, device, (cudaStream_t)stream);
    if (prev != device) {
        const cudaError_t e = cudaSetDevice(prev);
        if (e != cudaSuccess && rc == TG_OK) {
            set_last_cuda_error(e, "cudaSetDevice (restoring the caller's device)", __FILE__, __LINE__);
            return TG_ERR_CUDA;
        }
    }
    return rc;
}
