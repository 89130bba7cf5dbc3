// gp_batch.cu -- batched mode: many independent graphs in one call.
//
// No counterpart in the reference (it partitions one graph per process run).
// Worker threads, each owning a CUDA stream, a pinned status buffer and its
// own device arenas, take graphs from a shared queue ordered largest first
// (n + m, longest-processing-time order).  A call runs in three stages over
// chunks of graphs whose hierarchies fit in a share of the free device
// memory:
//   A  workers coarsen each graph and partition its coarsest level (the
//      host-driven phase of the V-cycle; many graphs in flight at once);
//   B  one persistent kernel refines the small levels of every graph of the
//      chunk (k_refine_chains: a device work queue of per-graph level chains,
//      one block per chain, no host round trip between levels or iterations);
//   C  workers refine the remaining large levels of each graph with the
//      multi-kernel loop and write its result.
// Every graph's result is exactly what gp_partition_device returns for it:
// the one-block loop and the multi-kernel loop take the same integer
// decisions.  Results are independent of the worker count and of the order
// in which graphs complete.
#define GP_TU_ID 7   // site ids of the bounds-checked build
#include "gp_internal.cuh"

#include <atomic>
#include <mutex>
#include <thread>
#include <memory>
#include <numeric>
#include <cstring>
#include <functional>

namespace gp {

struct BatchWorker {
    Arena keep, tmp;
    cudaStream_t s = nullptr;
    cudaEvent_t done = nullptr;
    int64_t* pinned = nullptr;
    ~BatchWorker() {
        if (s) cudaStreamDestroy(s);
        if (done) cudaEventDestroy(done);
        if (pinned) cudaFreeHost(pinned);
    }
};

struct BatchPool {
    std::mutex mu;                                  // one batch call per device at a time
    std::vector<std::unique_ptr<BatchWorker>> workers;
};

static BatchPool* batch_pool(int dev) {
    static std::mutex gmu;
    static std::unique_ptr<BatchPool> pools[64];
    if (dev < 0 || dev >= 64) throw GpError(GP_EINVAL, "device index out of range");
    std::lock_guard<std::mutex> lk(gmu);
    if (!pools[dev]) pools[dev].reset(new BatchPool());
    return pools[dev].get();
}

void release_batch_workers(int dev) {
    BatchPool* P = batch_pool(dev);
    std::lock_guard<std::mutex> lk(P->mu);
    P->workers.clear();
}

}  // namespace gp

using namespace gp;

extern "C" int gp_partition_batch_device(int32_t ngraphs, const int64_t* ns, const int64_t* ms,
                                         const int64_t* const* d_rowptrs, const int32_t* const* d_colidxs,
                                         const int32_t* const* d_vwgts, const int32_t* const* d_ewgts,
                                         const int32_t* ks, const float* imbalances, const uint64_t* seeds,
                                         int32_t* const* d_parts_out, void* stream, int32_t workers,
                                         const gp_options* opt, gp_stats* stats) {
    t_err.clear();
    try {
        if (ngraphs < 0) throw GpError(GP_EINVAL, "ngraphs must be >= 0");
        if (ngraphs == 0) return GP_OK;
        if (!ns || !ms || !d_rowptrs || !d_colidxs || !ks || !imbalances || !seeds || !d_parts_out)
            throw GpError(GP_EINVAL, "null array");
        for (int32_t i = 0; i < ngraphs; ++i) {
            check_args(ns[i], ks[i], imbalances[i]);
            if (ns[i] > 0 && (!d_rowptrs[i] || !d_colidxs[i] || !d_parts_out[i]))
                throw GpError(GP_EINVAL, "null array of graph " + std::to_string(i));
            if (ms[i] < 0) throw GpError(GP_EINVAL, "negative entry count of graph " + std::to_string(i));
        }
        if (workers <= 0) workers = 16;
        // concurrent V-cycles share the GPU: small grids per launch overlap
        // better than the single-graph default (unless the caller chose)
        gp_options bopt;
        if (opt) bopt = *opt;
        else { memset(&bopt, 0, sizeof bopt); bopt.version = GP_OPTIONS_VERSION; }
        if (bopt.ctas_per_sm <= 0) bopt.ctas_per_sm = 8;
        opt = &bopt;
        workers = std::min<int32_t>(workers, ngraphs);
        int dev = 0;
        GP_CUDA(cudaGetDevice(&dev));
        int sms = 148;
        GP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        ensure_kernel_caps(dev);
        BatchPool* P = batch_pool(dev);
        std::lock_guard<std::mutex> lk(P->mu);
        while ((int32_t)P->workers.size() < workers) {
            std::unique_ptr<BatchWorker> w(new BatchWorker());
            GP_CUDA(cudaStreamCreateWithFlags(&w->s, cudaStreamNonBlocking));
            GP_CUDA(cudaEventCreateWithFlags(&w->done, cudaEventDisableTiming));
            GP_CUDA(cudaMallocHost(&w->pinned, 64 * sizeof(int64_t)));
            P->workers.push_back(std::move(w));
        }
        // largest graphs first
        std::vector<int32_t> order((size_t)ngraphs);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
            return ns[a] + ms[a] > ns[b] + ms[b]; });
        // fork: workers start after prior work on the caller's stream
        cudaStream_t parent = (cudaStream_t)stream;
        cudaEvent_t fork;
        GP_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
        struct EvGuard { cudaEvent_t e; ~EvGuard() { cudaEventDestroy(e); } } fg{fork};
        GP_CUDA(cudaEventRecord(fork, parent));
        for (int32_t w = 0; w < workers; ++w) GP_CUDA(cudaStreamWaitEvent(P->workers[w]->s, fork, 0));
        std::atomic<bool> failed(false);
        std::mutex emu;
        int err_code = GP_OK;
        std::string err_msg;
        auto fail = [&](int code, const std::string& msg) {
            std::lock_guard<std::mutex> g2(emu);
            if (!failed.exchange(true)) { err_code = code; err_msg = msg; }
        };
        // run body(worker, item) over items [0, count) on all workers; the
        // calling thread is worker 0
        auto parallel = [&](int32_t count, const std::function<void(int32_t, int32_t)>& body) {
            std::atomic<int32_t> next(0);
            auto work = [&](int32_t wi) {
                try {
                    GP_CUDA(cudaSetDevice(dev));
                    for (;;) {
                        if (failed.load()) break;
                        const int32_t j = next.fetch_add(1);
                        if (j >= count) break;
                        body(wi, j);
                    }
                } catch (const GpError& e) {
                    fail(e.code, e.what());
                } catch (const std::exception& e) {
                    fail(GP_EINTERNAL, e.what());
                }
            };
            std::vector<std::thread> threads;
            for (int32_t w = 1; w < workers; ++w) threads.emplace_back(work, w);
            work(0);
            for (auto& t : threads) t.join();
        };
        auto make_ctx = [&](BatchWorker& W) {
            Ctx c;
            c.s = W.s; c.keep = &W.keep; c.tmp = &W.tmp; c.sm_count = sms; c.h_pinned = W.pinned;
            return c;
        };
        // every worker stream waits for all of them (stage boundaries)
        auto barrier_streams = [&]() {
            std::vector<cudaEvent_t> evs((size_t)workers);
            for (int32_t w = 0; w < workers; ++w) {
                GP_CUDA(cudaEventCreateWithFlags(&evs[w], cudaEventDisableTiming));
                GP_CUDA(cudaEventRecord(evs[w], P->workers[w]->s));
            }
            for (int32_t w = 0; w < workers; ++w)
                for (int32_t v = 0; v < workers; ++v)
                    if (v != w) GP_CUDA(cudaStreamWaitEvent(P->workers[w]->s, evs[v], 0));
            for (auto e : evs) cudaEventDestroy(e);
        };
        // chunks of the LPT order whose estimated hierarchies (coarse levels,
        // buckets, refinement buffers) fit in half the free device memory
        size_t free_b = 0, total_b = 0;
        GP_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const double budget = 0.5 * (double)free_b;
        int32_t c0 = 0;
        while (c0 < ngraphs && !failed.load()) {
            int32_t c1 = c0;
            double est = 0;
            while (c1 < ngraphs) {
                const int32_t i = order[c1];
                const double e = 96.0 * (double)ns[i] + 24.0 * (double)ms[i];
                if (c1 > c0 && est + e > budget) break;
                est += e;
                ++c1;
            }
            const int32_t cnt = c1 - c0;
            for (int32_t w = 0; w < workers; ++w) { P->workers[w]->keep.reset(); P->workers[w]->tmp.reset(); }
            std::vector<std::unique_ptr<VState>> states((size_t)cnt);
            std::unique_ptr<ChainBatch, void (*)(ChainBatch*)> cb(chain_batch_new(), chain_batch_delete);
            Tracer tr;
            // ---- stage A: coarsening and initial partition
            parallel(cnt, [&](int32_t wi, int32_t j) {
                BatchWorker& W = *P->workers[wi];
                const int32_t i = order[c0 + j];
                if (ns[i] == 0) { if (stats) memset(&stats[i], 0, sizeof(gp_stats)); return; }
                Ctx c = make_ctx(W);
                W.tmp.reset();
                DGraph g;
                g.n = ns[i]; g.m = ms[i]; g.rp = d_rowptrs[i]; g.ci = d_colidxs[i];
                g.vw = d_vwgts ? d_vwgts[i] : nullptr;
                g.ew = d_ewgts ? d_ewgts[i] : nullptr;
                GP_CUDA(cudaMemcpyAsync(W.pinned, d_rowptrs[i], sizeof(int64_t), cudaMemcpyDeviceToHost, W.s));
                GP_CUDA(cudaMemcpyAsync(W.pinned + 1, d_rowptrs[i] + ns[i], sizeof(int64_t),
                                        cudaMemcpyDeviceToHost, W.s));
                c.sync();
                if (W.pinned[0] != 0 || W.pinned[1] != ms[i])
                    throw GpError(GP_EINVAL, "graph " + std::to_string(i) + ": rowptr[0] must be 0 and rowptr[n] = m");
                states[j].reset(new VState());
                vc_begin(c, g, ks[i], imbalances[i], seeds[i], opt, *states[j], tr);
                chain_add(c, cb.get(), *states[j]);
            });
            if (failed.load()) break;
            // ---- stage B: the small levels of every graph in one persistent launch
            barrier_streams();
            {
                BatchWorker& W = *P->workers[0];
                Ctx c = make_ctx(W);
                W.tmp.reset();
                chain_run(c, cb.get());
            }
            barrier_streams();
            // ---- stage C: the large levels and the results
            parallel(cnt, [&](int32_t wi, int32_t j) {
                if (!states[j]) return;
                BatchWorker& W = *P->workers[wi];
                const int32_t i = order[c0 + j];
                VState& S = *states[j];
                Ctx c = make_ctx(W);
                W.tmp.reset();
                if (S.P.k > 1)
                    for (int l = S.refined_to - 1; l >= 0; --l) vc_level(c, S, l, tr);
                vc_end(c, S, d_parts_out[i], stats ? &stats[i] : nullptr);
            });
            if (failed.load()) break;
            barrier_streams();
            c0 = c1;
        }
        for (int32_t w = 0; w < workers; ++w) GP_CUDA(cudaEventRecord(P->workers[w]->done, P->workers[w]->s));
        // join: the caller's stream is ordered after every worker
        for (int32_t w = 0; w < workers; ++w) GP_CUDA(cudaStreamWaitEvent(parent, P->workers[w]->done, 0));
        for (int32_t w = 0; w < workers; ++w) {
            P->workers[w]->keep.consolidate();
            P->workers[w]->tmp.consolidate();
        }
        if (failed.load()) throw GpError(err_code, err_msg);
        GP_CUDA(cudaStreamSynchronize(parent));
        return GP_OK;
    } catch (const GpError& e) {
        t_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        t_err = e.what();
        return GP_EINTERNAL;
    }
}
