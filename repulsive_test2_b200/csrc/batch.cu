// Multi-curve batch: one sobolevStepSet per curve for many independent curves
// (own topology, vertices, constraint set and options each), run concurrently.
//
// The reference steps one curve per call (src/core/optimizer.ts:231-440); a
// batch of curves is that call repeated. Here every curve has its own context
// (its own streams and device buffers) and a pool of host threads drives the
// contexts, so the launches of different curves overlap on the GPU: a curve
// of a few hundred vertices fills a handful of SMs, and many of them fill the
// device. Curves are taken largest first. Results per curve are those of
// tpe_sobolev_step on the same inputs (the same kernels on the same data).
#include <algorithm>
#include <atomic>
#include <numeric>
#include <system_error>
#include <thread>
#include <vector>

#include "tpe_internal.h"

struct tpe_batch {
    int32_t device = 0;
    std::vector<tpe_ctx*> ctxs;
    std::vector<int32_t> V;
};

extern "C" {

tpe_batch* tpe_batch_create(int32_t device, int32_t ncurves, int32_t* status) {
    if (ncurves <= 0) {
        if (status) *status = TPE_ERR_BAD_ARG;
        return nullptr;
    }
    tpe_batch* b = new (std::nothrow) tpe_batch();
    if (!b) {
        if (status) *status = TPE_ERR_OUT_OF_MEMORY;
        return nullptr;
    }
    b->device = device;
    try {
        b->ctxs.reserve((size_t)ncurves);
        b->V.assign((size_t)ncurves, 0);
    } catch (...) {
        delete b;
        if (status) *status = TPE_ERR_OUT_OF_MEMORY;
        return nullptr;
    }
    for (int32_t i = 0; i < ncurves; i++) {
        int32_t st = TPE_OK;
        tpe_ctx* c = tpe_create(device, &st);
        if (!c || st != TPE_OK) {
            for (tpe_ctx* x : b->ctxs) tpe_destroy(x);
            delete b;
            if (status) *status = st != TPE_OK ? st : TPE_ERR_CUDA;
            return nullptr;
        }
        b->ctxs.push_back(c);  // within the reserved capacity
    }
    if (status) *status = TPE_OK;
    return b;
}

void tpe_batch_destroy(tpe_batch* b) {
    if (!b) return;
    for (tpe_ctx* c : b->ctxs) tpe_destroy(c);
    delete b;
}

tpe_ctx* tpe_batch_context(tpe_batch* b, int32_t i) {
    if (!b || i < 0 || i >= (int32_t)b->ctxs.size()) return nullptr;
    return b->ctxs[i];
}

int32_t tpe_batch_set_topology(tpe_batch* b, int32_t i, const int32_t* edges, int32_t E,
                               int32_t V) {
    return tpe::guarded(nullptr, [&]() -> int32_t {
        if (!b || i < 0 || i >= (int32_t)b->ctxs.size()) return TPE_ERR_BAD_ARG;
        const int32_t st = tpe_set_topology(b->ctxs[i], edges, E, V);
        if (st == TPE_OK) b->V[i] = V;
        return st;
    });
}

int32_t tpe_step_batch(tpe_batch* b, const double* const* xyz, const tpe_constraint* const* sets,
                       const int32_t* nblocks, const tpe_step_opts* opts, double* const* xyz_out,
                       tpe_step_stats* stats, int32_t* status, int32_t max_threads) {
    return tpe::guarded(nullptr, [&]() -> int32_t {
        if (!b || !xyz || !nblocks || !opts || !xyz_out || !stats || !status) return TPE_ERR_BAD_ARG;
        const int32_t n = (int32_t)b->ctxs.size();
        std::vector<int32_t> order((size_t)n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(),
                         [&](int32_t x, int32_t y) { return b->V[x] > b->V[y]; });
        int32_t nt = max_threads > 0 ? max_threads : (int32_t)std::thread::hardware_concurrency();
        nt = std::max(1, std::min(nt, n));
        std::atomic<int32_t> next{0};
        auto work = [&]() {
            for (;;) {
                const int32_t q = next.fetch_add(1);
                if (q >= n) break;
                const int32_t i = order[(size_t)q];
                status[i] = tpe_sobolev_step(b->ctxs[i], xyz[i], sets ? sets[i] : nullptr, nblocks[i],
                                             &opts[i], xyz_out[i], &stats[i], nullptr, nullptr);
            }
        };
        // a thread that cannot start leaves its share to the others (an exception
        // here with threads running would end the process)
        std::vector<std::thread> pool;
        pool.reserve((size_t)nt);
        for (int32_t t = 1; t < nt; t++) {
            try {
                pool.emplace_back(work);
            } catch (const std::system_error&) {
                break;
            }
        }
        work();
        for (auto& th : pool) th.join();
        for (int32_t i = 0; i < n; i++)
            if (status[i] != TPE_OK) return status[i];
        return TPE_OK;
    });
}

}  // extern "C"
