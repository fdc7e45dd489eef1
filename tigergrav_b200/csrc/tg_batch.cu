/*
 * tg_batch.cu -- many independent periodic unit boxes of uneven sizes in one
 * call (the batching workload; no counterpart in the reference, which runs
 * one box per process).
 *
 * Each box is an ordinary solver handle with its own m = 1/N_b and
 * soft_len = 0.02 N_b^(-1/3) (the reference's defaults for m_tot = 1,
 * src/options.cpp:86-88).  A batch call runs the boxes on nstreams CUDA
 * streams, each driven by its own host thread, so the host round trips that
 * a single solve makes between kernels (tree levels, list capacities, Ewald
 * chunk totals) overlap with other boxes' kernels instead of idling the GPU.
 * Boxes are handed out largest first from a shared counter.
 *
 * tg_batch_autotune times one evaluation of each box for each candidate
 * leaf size (after a warm-up solve) and keeps the fastest per box.
 */
#include <algorithm>
#include <atomic>
#include <thread>

struct tg_batch {
    std::vector<tg_solver *> box;
    std::vector<int64_t> count, off;
    std::vector<int32_t> order; /* boxes by decreasing size */
    std::vector<cudaStream_t> streams;
    int32_t nstreams = 1;
    int dev = 0;
};

namespace {

/* run fn(box, stream) for every box on the batch's streams; first error wins */
template <class F>
int batch_run(tg_batch *b, F &&fn) {
    std::atomic<int> next{0}, err{TG_OK};
    auto worker = [&](int t) {
        if (cudaSetDevice(b->dev) != cudaSuccess) {
            err.store(TG_ERR_CUDA);
            return;
        }
        for (;;) {
            const int k = next.fetch_add(1);
            if (k >= (int)b->order.size() || err.load() != TG_OK) break;
            const int bx = b->order[k];
            const int rc = fn(bx, b->streams[t]);
            if (rc != TG_OK) {
                int expect = TG_OK;
                err.compare_exchange_strong(expect, rc);
            }
        }
        if (cudaStreamSynchronize(b->streams[t]) != cudaSuccess) err.store(TG_ERR_CUDA);
    };
    std::vector<std::thread> th;
    for (int t = 0; t < b->nstreams; t++) th.emplace_back(worker, t);
    for (auto &t : th) t.join();
    return err.load();
}

} // namespace

extern "C" {

int tg_batch_create(const tg_params *params, int32_t nboxes, const int64_t *counts, int32_t nstreams,
                    tg_batch **out) {
    if (!out || !params || !counts || nboxes < 1 || nstreams < 1 || nstreams > 64) return TG_ERR_ARG;
    *out = nullptr;
    tg_batch *b = new tg_batch();
    b->dev = params->device;
    b->nstreams = nstreams;
    int64_t o = 0;
    for (int32_t i = 0; i < nboxes; i++) {
        if (counts[i] < 1) {
            tg_batch_destroy(b);
            return TG_ERR_ARG;
        }
        tg_params p = *params;
        p.m = 1.0 / (double)counts[i];
        p.soft_len = 0.02 * std::pow((double)counts[i], -1.0 / 3.0);
        tg_solver *s = nullptr;
        const int rc = tg_create(&p, &s);
        if (rc != TG_OK) {
            tg_batch_destroy(b);
            return rc;
        }
        b->box.push_back(s);
        b->count.push_back(counts[i]);
        b->off.push_back(o);
        o += counts[i];
        b->order.push_back(i);
    }
    b->off.push_back(o);
    std::stable_sort(b->order.begin(), b->order.end(),
                     [&](int32_t a, int32_t c) { return b->count[a] > b->count[c]; });
    if (cudaSetDevice(b->dev) != cudaSuccess) {
        tg_batch_destroy(b);
        return TG_ERR_CUDA;
    }
    for (int t = 0; t < nstreams; t++) {
        cudaStream_t st;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            tg_batch_destroy(b);
            return TG_ERR_CUDA;
        }
        b->streams.push_back(st);
    }
    *out = b;
    return TG_OK;
}

int tg_batch_destroy(tg_batch *b) {
    if (!b) return TG_ERR_ARG;
    cudaSetDevice(b->dev);
    for (auto st : b->streams) cudaStreamDestroy(st);
    for (auto s : b->box) tg_destroy(s);
    delete b;
    return TG_OK;
}

int64_t tg_batch_size(tg_batch *b) { return b ? b->off.back() : -1; }

int tg_batch_set_particles(tg_batch *b, const int32_t *x, const float *v, int where) {
    if (!b || !x) return TG_ERR_ARG;
    return batch_run(b, [&](int i, cudaStream_t st) -> int {
        return tg_set_particles(b->box[i], x + 3 * b->off[i], v ? v + 3 * b->off[i] : nullptr, b->count[i], where, st);
    });
}

int tg_batch_solve(tg_batch *b) {
    if (!b) return TG_ERR_ARG;
    return batch_run(b, [&](int i, cudaStream_t st) -> int { return tg_solve_gravity(b->box[i], st); });
}

int tg_batch_leapfrog(tg_batch *b, double dt, int n_steps) {
    if (!b) return TG_ERR_ARG;
    return batch_run(b, [&](int i, cudaStream_t st) -> int { return tg_leapfrog(b->box[i], dt, n_steps, st); });
}

int tg_batch_get_forces(tg_batch *b, float *phi, float *g, int where) {
    if (!b) return TG_ERR_ARG;
    return batch_run(b, [&](int i, cudaStream_t st) -> int {
        return tg_get_forces(b->box[i], phi ? phi + b->off[i] : nullptr, g ? g + 3 * b->off[i] : nullptr, where, st);
    });
}

int tg_batch_autotune(tg_batch *b, const int32_t *leaf_sizes, int32_t nsizes, int32_t *chosen) {
    if (!b || !leaf_sizes || nsizes < 1) return TG_ERR_ARG;
    for (int32_t k = 0; k < nsizes; k++)
        if (leaf_sizes[k] < 1 || leaf_sizes[k] > 128) return TG_ERR_ARG;
    const int nb = (int)b->box.size();
    std::vector<float> best(nb, 3.0e38f);
    std::vector<int32_t> pick(nb, b->box[0]->S.prm.leaf_max);
    for (int32_t k = 0; k < nsizes; k++) {
        const int rc = batch_run(b, [&](int i, cudaStream_t st) -> int {
            tg::Solver &S = b->box[i]->S;
            S.prm.leaf_max = leaf_sizes[k];
            TG_TRY(tg_solve_gravity(b->box[i], st)); /* warm-up: buffers sized for this leaf size */
            struct Events { /* destroyed on every return path */
                cudaEvent_t e[2] = {nullptr, nullptr};
                ~Events() {
                    for (cudaEvent_t x : e)
                        if (x) cudaEventDestroy(x);
                }
            } ev;
            TG_CUDA(cudaEventCreate(&ev.e[0]));
            TG_CUDA(cudaEventCreate(&ev.e[1]));
            TG_CUDA(cudaEventRecord(ev.e[0], st));
            TG_TRY(tg_solve_gravity(b->box[i], st));
            TG_CUDA(cudaEventRecord(ev.e[1], st));
            TG_CUDA(cudaEventSynchronize(ev.e[1]));
            float ms = 0.0f;
            TG_CUDA(cudaEventElapsedTime(&ms, ev.e[0], ev.e[1])); /* a failed timing is an error, not 0 ms */
            if (ms < best[i]) {
                best[i] = ms;
                pick[i] = leaf_sizes[k];
            }
            return TG_OK;
        });
        if (rc != TG_OK) return rc;
    }
    for (int i = 0; i < nb; i++) {
        b->box[i]->S.prm.leaf_max = pick[i];
        b->box[i]->S.have_tree = b->box[i]->S.have_multipoles = b->box[i]->S.have_lists = false;
        b->box[i]->S.have_forces = false;
        if (chosen) chosen[i] = pick[i];
    }
    return TG_OK;
}

} // extern "C"
