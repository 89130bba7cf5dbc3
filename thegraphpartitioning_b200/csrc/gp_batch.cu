// gp_batch.cu -- batched mode: many independent graphs in one call.
//
// No counterpart in the reference (it partitions one graph per process run).
// Worker threads, each owning a CUDA stream, a pinned status buffer and its
// own device arenas, take graphs from a shared queue ordered largest first
// (n + m, longest-processing-time order) and run the same deterministic
// V-cycle as gp_partition_device on their stream.  Many small graphs thus
// keep the GPU busy concurrently while each V-cycle's host-side control waits
// only on its own stream.  Results are independent of the worker count and
// of the order in which graphs complete.
#include "gp_internal.cuh"

#include <atomic>
#include <mutex>
#include <thread>
#include <memory>
#include <numeric>
#include <cstring>

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
        std::atomic<int32_t> next(0);
        std::atomic<bool> failed(false);
        std::mutex emu;
        int err_code = GP_OK;
        std::string err_msg;
        auto work = [&](int32_t wi) {
            BatchWorker& W = *P->workers[wi];
            try {
                GP_CUDA(cudaSetDevice(dev));
                for (;;) {
                    if (failed.load()) break;
                    const int32_t j = next.fetch_add(1);
                    if (j >= ngraphs) break;
                    const int32_t i = order[j];
                    if (ns[i] == 0) { if (stats) memset(&stats[i], 0, sizeof(gp_stats)); continue; }
                    Ctx c;
                    c.s = W.s; c.keep = &W.keep; c.tmp = &W.tmp; c.sm_count = sms; c.h_pinned = W.pinned;
                    W.keep.reset();
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
                    Tracer tr;
                    run_vcycle(c, g, ks[i], imbalances[i], seeds[i], opt, d_parts_out[i], stats ? &stats[i] : nullptr, tr);
                }
                GP_CUDA(cudaEventRecord(W.done, W.s));
            } catch (const GpError& e) {
                std::lock_guard<std::mutex> g2(emu);
                if (!failed.exchange(true)) { err_code = e.code; err_msg = e.what(); }
                cudaEventRecord(W.done, W.s);
            } catch (const std::exception& e) {
                std::lock_guard<std::mutex> g2(emu);
                if (!failed.exchange(true)) { err_code = GP_EINTERNAL; err_msg = e.what(); }
                cudaEventRecord(W.done, W.s);
            }
        };
        std::vector<std::thread> threads;
        for (int32_t w = 1; w < workers; ++w) threads.emplace_back(work, w);
        work(0);
        for (auto& t : threads) t.join();
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
