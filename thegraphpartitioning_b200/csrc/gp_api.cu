// gp_api.cu -- C ABI entry points and the V-cycle driver.
//
// Replaces main() of the reference (src/gpu_part.cu:878-1390): argument
// checks (src/gpu_part.cu:880-894), coarsening stop rule
// (src/gpu_part.cu:897, 1003, 1069), the coarsen -> initial partition ->
// refine/uncoarsen sequence and the final cut (src/gpu_part.cu:1285-1289).
// Differences by design: every step runs on the device (no gpmetis process,
// no per-element host partCount rebuild), errors are returned instead of
// exit(), and all integer results are deterministic for a given seed.
#define GP_TU_ID 5   // site ids of the bounds-checked build
#include "gp_internal.cuh"

#include <mutex>
#include <memory>
#include <cstring>

namespace gp {

thread_local std::string t_err;

#ifdef GP_CHECKED
// the per-translation-unit violation counters of the bounds-checked build
static std::vector<chk_fetch_fn>& chk_fetchers() {
    static std::vector<chk_fetch_fn> v;
    return v;
}
void chk_register(chk_fetch_fn f) { chk_fetchers().push_back(f); }
#endif

// ---------------------------------------------------------------- device state
struct DevState {
    std::mutex mu;
    Arena keep, tmp;
    int64_t* pinned = nullptr;
    int sm_count = 148;
    bool init = false;
};

static DevState* dev_state(int dev) {
    static std::mutex gmu;
    static std::unique_ptr<DevState> states[64];
    if (dev < 0 || dev >= 64) throw GpError(GP_EINVAL, "device index out of range");
    std::lock_guard<std::mutex> lk(gmu);
    if (!states[dev]) states[dev].reset(new DevState());
    return states[dev].get();
}

void ensure_kernel_caps(int dev) {
    static std::mutex mu;
    static bool done[64] = {};
    if (dev < 0 || dev >= 64) throw GpError(GP_EINVAL, "device index out of range");
    std::lock_guard<std::mutex> lk(mu);
    if (done[dev]) return;
    coarsen_smem_caps();
    refine_smem_caps();
    initpart_smem_caps();
    done[dev] = true;
}

static void ensure_init(DevState& S, int dev) {
    ensure_kernel_caps(dev);
    if (S.init) return;
    GP_CUDA(cudaDeviceGetAttribute(&S.sm_count, cudaDevAttrMultiProcessorCount, dev));
    GP_CUDA(cudaMallocHost(&S.pinned, 64 * sizeof(int64_t)));
    S.init = true;
}

// ---------------------------------------------------------------- validation
enum { V_ROWPTR = 1, V_VWGT = 2, V_COLIDX = 3, V_SELF = 4, V_EWGT = 5, V_PART = 6 };

__device__ __forceinline__ void report(unsigned long long* err, int code, int64_t idx) {
    atomicMin(err, ((unsigned long long)code << 48) | (unsigned long long)(idx & ((1ll << 48) - 1)));
}

__global__ void k_check_rowptr(int64_t n, int64_t m, const int64_t* __restrict__ rp, const int32_t* __restrict__ vw,
                               unsigned long long* err, int64_t* sums) {
    int64_t local = 0;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = rp[v], b = rp[v + 1];
        if (a < 0 || b < a || b > m) report(err, V_ROWPTR, v);
        const int32_t w = vw ? vw[v] : 1;
        if (w < 1) report(err, V_VWGT, v);
        local += w;
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) atomicAdd((unsigned long long*)&sums[0], (unsigned long long)local);
}

// one entry: weight >= 1, column id in range, no self loop (the smallest
// (code, index) reported wins, whatever the order of the checks)
__device__ __forceinline__ void check_entry(int64_t n, int64_t e, int64_t v, int32_t u, int32_t w, int check,
                                            unsigned long long* err, int64_t& local) {
    if (w < 1) report(err, V_EWGT, e);
    local += w;
    if (check >= 1) {
        if (u < 0 || u >= n) report(err, V_COLIDX, e);
        else if (u == v) report(err, V_SELF, v);
    }
}
// entries of a row-pointer-checked CSR, entry-sliced (csr_row_of /
// csr_window_lane), eight groups of 32 entries loaded together
__global__ void k_check_rows(int64_t n, int64_t m, int64_t slice, const int64_t* __restrict__ rp,
                             const int32_t* __restrict__ ci,
                             const int32_t* __restrict__ ew, int check, unsigned long long* err, int64_t* sums) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t nslice = (m + slice - 1) / slice;
    int64_t local = 0;
    for (int64_t sl = wid; sl < nslice; sl += nw) {
        const int64_t o0 = sl * slice, o1 = o0 + slice < m ? o0 + slice : m;
        int64_t cb = csr_row_of(rp, n, o0), s = 0, wend = 0;
        auto window = [&]() {
            s = cb + lane < n ? rp[cb + lane] : m;
            wend = rp[cb + 32 < n ? cb + 32 : n];
        };
        window();
        int64_t o = o0;
        while (o < o1) {
            const int64_t lim = o1 < wend ? o1 : wend;
            if (o + 256 <= lim) {
                int32_t u[8], w[8];
                int64_t v[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int64_t oi = o + 32 * q + lane;
                    v[q] = cb + csr_window_lane(s, oi);
                    u[q] = check >= 1 ? __ldcs(&ci[oi]) : 0;
                    w[q] = ew ? __ldcs(&ew[oi]) : 1;
                }
#pragma unroll
                for (int q = 0; q < 8; ++q) check_entry(n, o + 32 * q + lane, v[q], u[q], w[q], check, err, local);
                o += 256;
            } else if (o < lim) {
                const int64_t oi = o + lane;
                const int64_t v = cb + csr_window_lane(s, oi);
                if (oi < lim) check_entry(n, oi, v, check >= 1 ? ci[oi] : 0, ew ? ew[oi] : 1, check, err, local);
                o = o + 32 < lim ? o + 32 : lim;
            } else {
                cb += 32;   // o >= wend: o lies in a later row
                window();
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if (lane == 0) atomicAdd((unsigned long long*)&sums[1], (unsigned long long)local);
}

// symmetry: every entry (v,u,w) has a partner (u,v,w).  Both directions are
// packed as (min,max,w) keys, sorted, and must pair up exactly.
__global__ void k_sym_keys(int64_t n, const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                           const int32_t* __restrict__ ew, int nb, uint64_t* __restrict__ keys, int32_t* __restrict__ vals) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = wid; v < n; v += nw)
        for (int64_t e = rp[v] + lane; e < rp[v + 1]; e += 32) {
            const uint64_t u = (uint32_t)ci[e];
            const uint64_t a = (uint64_t)v < u ? (uint64_t)v : u, b = (uint64_t)v < u ? u : (uint64_t)v;
            keys[e] = (a << nb) | b;
            // direction bit in the payload; weight kept for the pair comparison
            vals[e] = (int32_t)(((uint32_t)(ew ? ew[e] : 1) << 1) | ((uint64_t)v < u ? 0u : 1u));
        }
}
__global__ void k_sym_check(int64_t m, const uint64_t* __restrict__ keys, const int32_t* __restrict__ vals,
                            unsigned long long* err) {
    // sorted by key; within a key, payload order is arbitrary: check that the
    // run has even length and equal counts of both directions per weight by
    // pairing sorted payloads of the run (runs are short: duplicates only)
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        if (i > 0 && keys[i - 1] == keys[i]) continue;
        int64_t j = i;
        int64_t up = 0, down = 0, wsum_up = 0, wsum_down = 0;
        while (j < m && keys[j] == keys[i]) {
            const uint32_t pv = (uint32_t)vals[j];
            if (pv & 1u) { ++down; wsum_down += pv >> 1; } else { ++up; wsum_up += pv >> 1; }
            ++j;
        }
        if (up != down || wsum_up != wsum_down) report(err, 7, i);
    }
}

static std::string verr(int code, int64_t idx) {
    switch (code) {
    case V_ROWPTR: return "rowptr is not non-decreasing within [0, m] at vertex " + std::to_string(idx);
    case V_VWGT: return "vertex weight < 1 at vertex " + std::to_string(idx);
    case V_COLIDX: return "column index out of range at entry " + std::to_string(idx);
    case V_SELF: return "self-loop at vertex " + std::to_string(idx);
    case V_EWGT: return "edge weight < 1 at entry " + std::to_string(idx);
    case V_PART: return "part id out of range at vertex " + std::to_string(idx);
    case 7: return "graph is not symmetric";
    default: return "invalid input";
    }
}

static int bits_for(int64_t x) {
    int b = 1;
    while ((1ll << b) < x) ++b;
    return b;
}

// returns total vertex weight
static int64_t validate(Ctx& c, const DGraph& g, int check) {
    auto mk = c.tmp->save();
    unsigned long long* err = (unsigned long long*)c.tmp_alloc<int64_t>(4);
    int64_t* sums = c.tmp_alloc<int64_t>(2);
    GP_CUDA(cudaMemsetAsync(err, 0xff, 8, c.s));
    memset_async(c, sums, 0, 16);
    k_check_rowptr<<<grid_for(g.n, 256), 256, 0, c.s>>>(g.n, g.m, g.rp, g.vw, err, sums);
    GP_LAUNCHED(c);
    GP_CUDA(cudaMemcpyAsync(c.h_pinned, err, 8, cudaMemcpyDeviceToHost, c.s));
    c.sync();
    uint64_t e0 = (uint64_t)c.h_pinned[0];
    if (e0 != ~0ull) throw GpError(GP_EINVAL, verr((int)(e0 >> 48), (int64_t)(e0 & ((1ull << 48) - 1))));
    const int64_t slice = csr_slice(g.m, c.sm_count);
    k_check_rows<<<grid_for((g.m + slice - 1) / slice * 32, 256, c.sm_count * 8), 256, 0, c.s>>>(
        g.n, g.m, slice, g.rp, g.ci, g.ew, check, err, sums);
    GP_LAUNCHED(c);
    c.bytes += 8 * (g.n + 1) + (g.vw ? 4 * g.n : 0) + (check >= 1 ? 4 * g.m : 0) + (g.ew ? 4 * g.m : 0);
    GP_CUDA(cudaMemcpyAsync(c.h_pinned, err, 8, cudaMemcpyDeviceToHost, c.s));
    GP_CUDA(cudaMemcpyAsync(c.h_pinned + 1, sums, 16, cudaMemcpyDeviceToHost, c.s));
    c.sync();
    e0 = (uint64_t)c.h_pinned[0];
    if (e0 != ~0ull) throw GpError(GP_EINVAL, verr((int)(e0 >> 48), (int64_t)(e0 & ((1ull << 48) - 1))));
    const int64_t W = c.h_pinned[1], EW = c.h_pinned[2];
    if (W > INT32_MAX) throw GpError(GP_EINVAL, "sum of vertex weights exceeds int32");
    if (EW > INT32_MAX) throw GpError(GP_EINVAL, "sum of edge weights exceeds int32");
    if (check >= 2 && g.m > 0) {
        const int nb = bits_for(g.n);
        uint64_t* keys = c.tmp_alloc<uint64_t>(g.m);
        uint64_t* keys2 = c.tmp_alloc<uint64_t>(g.m);
        int32_t* vals = c.tmp_alloc<int32_t>(g.m);
        int32_t* vals2 = c.tmp_alloc<int32_t>(g.m);
        k_sym_keys<<<grid_for(g.n * 32, 256, c.sm_count * 8), 256, 0, c.s>>>(g.n, g.rp, g.ci, g.ew, nb, keys, vals);
        GP_LAUNCHED(c);
        radix_sort_pairs(c, keys, vals, keys2, vals2, g.m, 2 * nb);
        k_sym_check<<<grid_for(g.m, 256), 256, 0, c.s>>>(g.m, keys, vals, err);
        GP_LAUNCHED(c);
        GP_CUDA(cudaMemcpyAsync(c.h_pinned, err, 8, cudaMemcpyDeviceToHost, c.s));
        c.sync();
        e0 = (uint64_t)c.h_pinned[0];
        if (e0 != ~0ull) throw GpError(GP_EINVAL, verr((int)(e0 >> 48), 0));
    }
    c.tmp->restore(mk);
    return W;
}

__global__ void k_check_part(int64_t n, const int32_t* __restrict__ part, int32_t k, unsigned long long* err) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = part[v];
        if (p < 0 || p >= k) report(err, V_PART, v);
    }
}

// ---------------------------------------------------------------- tracing helpers
template <class T>
static std::vector<T> to_host(Ctx& c, const T* d, int64_t count) {
    std::vector<T> h((size_t)std::max<int64_t>(count, 1));
    if (count > 0) GP_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(T) * count, cudaMemcpyDeviceToHost, c.s));
    c.sync();
    return h;
}

// ---------------------------------------------------------------- V-cycle

// Phase 1: validation, coarsening, refinement buffers and the initial
// partition.  Everything the later phases need stays in S (hierarchy and
// buffers in c.keep, which must outlive the V-cycle).
void vc_begin(Ctx& c, const DGraph& g0, int32_t k, float imbalance, uint64_t seed, const gp_options* opt,
              VState& S, const Tracer& tr, const gp_gnn* gnn) {
    Params& P = S.P;
    P.gnn = gnn;
    resolve_options(opt, k, &P.o);
    P.k = k; P.seed = seed; P.imbalance = imbalance;
    c.ctas_per_sm = P.o.ctas_per_sm;
    Timer& tm = S.tm;
    c.profile = P.o.profile > 0;
    if (c.profile) { c.ev_a = tm.e[6]; c.ev_b = tm.e[7]; }
    GP_CUDA(cudaEventRecord(tm.e[0], c.s));
    P.W = validate(c, g0, P.o.check_input);
    P.Lmax = compute_lmax(P.W, k, imbalance);
    P.maxvw = std::max<int64_t>(1, (3 * P.W) / (2 * (int64_t)P.o.coarsen_to));
    S.g0 = g0;
    const int64_t n0 = g0.n;
    std::vector<Level>& lv = S.lv;
    lv.assign(1, Level());
    lv[0].g = g0;
    S.best_trial = -1; S.iters = 0;
    if (k == 1) {
        S.L = 0;
        S.refined_to = 0;
        GP_CUDA(cudaEventRecord(tm.e[1], c.s));
        GP_CUDA(cudaEventRecord(tm.e[2], c.s));
        S.take(c);
        return;
    }
    lv[0].heavy_deg = P.o.heavy_deg;
    lv[0].item_len = P.o.item_len;
    build_heavy(c, lv[0]);
    // ---- coarsening
    while (lv.back().g.n > P.o.coarsen_to && (int)lv.size() < 64) {
        const int level = (int)lv.size() - 1;
        auto mk = c.tmp->save();
        int32_t* match = c.tmp_alloc<int32_t>(lv.back().g.n);
        int32_t* prio = nullptr;
        const bool scored = P.gnn && gnn_scores_level(P.gnn, level);
        if (scored) {
            prio = c.tmp_alloc<int32_t>(lv.back().g.m);
            GP_CUDA(cudaEventRecord(tm.e[4], c.s));
            gnn_level_priorities(c, P.gnn, lv.back(), level, prio);
            GP_CUDA(cudaEventRecord(tm.e[5], c.s));
            if (tr.on()) {
                auto hp = to_host(c, prio, lv.back().g.m);
                gp_trace_event ev; memset(&ev, 0, sizeof ev);
                ev.kind = GP_TR_PRIO; ev.level = level; ev.n = lv.back().g.n; ev.m = lv.back().g.m;
                ev.a0 = hp.data();
                tr.emit(ev);
            }
        }
        int rounds = 0;
        const int64_t pairs = match_level(c, lv.back(), level, P, match, &rounds, prio);
        if (scored) c.ms_gnn += tm.ms(4, 5);   // match_level has synchronized the stream
        const int64_t n = lv.back().g.n;
        if (tr.on()) {
            auto h = to_host(c, match, n);
            gp_trace_event ev; memset(&ev, 0, sizeof ev);
            ev.kind = GP_TR_MATCH; ev.level = level; ev.iter = rounds; ev.n = n; ev.m = lv.back().g.m;
            ev.count = pairs; ev.a0 = h.data();
            tr.emit(ev);
        }
        if (20 * (n - pairs) > 19 * n) { c.tmp->restore(mk); break; }
        Level cl;
        contract_level(c, lv.back(), cl, match);
        c.tmp->restore(mk);
        if (tr.on()) {
            auto cm = to_host(c, lv.back().cmap, n);
            auto rp = to_host(c, cl.g.rp, cl.g.n + 1);
            auto ci = to_host(c, cl.g.ci, cl.g.m);
            auto ew = to_host(c, cl.g.ew, cl.g.m);
            auto vw = to_host(c, cl.g.vw, cl.g.n);
            gp_trace_event ev; memset(&ev, 0, sizeof ev);
            ev.kind = GP_TR_CONTRACT; ev.level = level; ev.n = cl.g.n; ev.m = cl.g.m;
            ev.a0 = cm.data(); ev.rowptr = rp.data(); ev.colidx = ci.data(); ev.ewgt = ew.data(); ev.vwgt = vw.data();
            tr.emit(ev);
        }
        cl.heavy_deg = P.o.heavy_deg;
        cl.item_len = P.o.item_len;
        build_heavy(c, cl);
        lv.push_back(cl);
    }
    GP_CUDA(cudaEventRecord(tm.e[1], c.s));
    // ---- refinement buffers (finest size)
    RefineBufs& B = S.B;
    B.part = c.keep_alloc<int32_t>(n0);
    B.part_next = c.keep_alloc<int32_t>(n0);
    B.best = c.keep_alloc<int32_t>(n0);
    B.pc = c.keep_alloc<uint16_t>(n0);
    B.pc_next = c.keep_alloc<uint16_t>(n0);
    B.dest = c.keep_alloc<int32_t>(n0);
    B.pdg = k <= 1024 ? c.keep_alloc<uint64_t>(n0) : nullptr;
    B.gain = c.keep_alloc<int32_t>(n0);
    B.mp = P.gnn && gnn_has_move_head(P.gnn) ? c.keep_alloc<int32_t>(n0) : nullptr;
    B.lock = c.keep_alloc<uint8_t>(n0);
    B.lock_next = c.keep_alloc<uint8_t>(n0);
    B.pw = c.keep_alloc<int64_t>(k);
    B.best_pw = c.keep_alloc<int64_t>(k);
    B.status = c.keep_alloc<int64_t>(S_NSLOTS);
    for (int b = 0; b < 3; ++b) B.clist[b] = c.keep_alloc<int32_t>(n0);
    B.wfirst_cap = conn_max_warps(c) + 1;
    B.wfirst = c.keep_alloc<int64_t>(B.wfirst_cap);
    int64_t hmax = 1;
    for (const Level& l : lv) hmax = std::max(hmax, l.nheavy);
    B.hhist = c.keep_alloc<int32_t>(hmax * k);
    B.hsum = c.keep_alloc<int64_t>(2 * hmax);
    B.hdone = c.keep_alloc<int32_t>(hmax);
    memset_async(c, B.hhist, 0, sizeof(int32_t) * hmax * k);
    memset_async(c, B.hsum, 0, sizeof(int64_t) * 2 * hmax);
    memset_async(c, B.hdone, 0, sizeof(int32_t) * hmax);
    B.ckeys = c.keep_alloc<uint64_t>(n0);
    B.cvals = c.keep_alloc<int32_t>(n0);
    B.ckeys2 = c.keep_alloc<uint64_t>(n0);
    B.cvals2 = c.keep_alloc<int32_t>(n0);
    // ---- initial partition
    const int L = (int)lv.size() - 1;
    S.L = L;
    S.refined_to = L + 1;
    S.best_trial = initial_partition(c, lv[L], P, B.part);
    part_weights(c, lv[L].g, B.part, k, B.pw);
    if (tr.on()) {
        int64_t* d_c = c.tmp_alloc<int64_t>(1);
        cut_and_weights(c, lv[L].g, B.part, k, d_c, nullptr);
        auto cut2 = to_host(c, d_c, 1);
        auto pw = to_host(c, B.pw, k);
        auto hp = to_host(c, B.part, lv[L].g.n);
        gp_trace_event ev; memset(&ev, 0, sizeof ev);
        ev.kind = GP_TR_INITPART; ev.level = L; ev.iter = S.best_trial; ev.n = lv[L].g.n; ev.m = lv[L].g.m;
        ev.cut = cut2[0] / 2; ev.maxpw = *std::max_element(pw.begin(), pw.begin() + k); ev.a0 = hp.data();
        tr.emit(ev);
    }
    GP_CUDA(cudaEventRecord(tm.e[2], c.s));
    S.take(c);
}

// Phase 2, one level at a time from the coarsest (l = S.L) to the input
// (l = 0): projection of the coarser level's partition, then refinement.
void vc_level(Ctx& c, VState& S, int l, const Tracer& tr) {
    if (l != S.refined_to - 1) throw GpError(GP_EINTERNAL, "levels must be refined coarsest first");
    const Params& P = S.P;
    RefineBufs& B = S.B;
    std::vector<Level>& lv = S.lv;
    c.ctas_per_sm = P.o.ctas_per_sm;
    c.profile = P.o.profile > 0;
    if (c.profile) { c.ev_a = S.tm.e[6]; c.ev_b = S.tm.e[7]; }
    if (l < S.L) {
        project(c, lv[l], B.part, B.part_next);
        std::swap(B.part, B.part_next);
    }
    S.iters += refine_level(c, lv[l], P, B, l, tr);
    if (tr.on()) {
        int64_t* d_c = c.tmp_alloc<int64_t>(1);
        cut_and_weights(c, lv[l].g, B.part, P.k, d_c, nullptr);
        auto cut2 = to_host(c, d_c, 1);
        auto pw = to_host(c, B.pw, P.k);
        auto hp = to_host(c, B.part, lv[l].g.n);
        gp_trace_event ev; memset(&ev, 0, sizeof ev);
        ev.kind = GP_TR_LEVEL_DONE; ev.level = l; ev.n = lv[l].g.n; ev.m = lv[l].g.m;
        ev.cut = cut2[0] / 2; ev.maxpw = *std::max_element(pw.begin(), pw.begin() + P.k); ev.a0 = hp.data();
        tr.emit(ev);
    }
    S.refined_to = l;
    S.take(c);
}

// Phase 3: the result into d_out and the exact result record.
void vc_end(Ctx& c, VState& S, int32_t* d_out, gp_stats* st) {
    const Params& P = S.P;
    const int32_t k = P.k;
    const int64_t n0 = S.g0.n;
    if (k == 1) memset_async(c, d_out, 0, sizeof(int32_t) * n0);
    else GP_CUDA(cudaMemcpyAsync(d_out, S.B.part, sizeof(int32_t) * n0, cudaMemcpyDeviceToDevice, c.s));
    GP_CUDA(cudaEventRecord(S.tm.e[3], c.s));
    int64_t* d_c = c.tmp_alloc<int64_t>(1);
    int64_t* d_pw = c.tmp_alloc<int64_t>(k);
    cut_and_weights(c, S.g0, d_out, k, d_c, d_pw);
    auto cut2 = to_host(c, d_c, 1);
    auto pw = to_host(c, d_pw, k);
    S.take(c);
    if (st) {
        memset(st, 0, sizeof *st);
        st->cut = cut2[0] / 2;
        st->max_part_weight = *std::max_element(pw.begin(), pw.begin() + k);
        st->total_weight = P.W;
        st->max_allowed = P.Lmax;
        st->imbalance = (double)st->max_part_weight * k / (double)P.W - 1.0;
        st->levels = (int32_t)S.lv.size();
        st->coarsest_n = (int32_t)S.lv.back().g.n;
        st->best_trial = S.best_trial;
        st->refine_iters = S.iters;
        st->algo_bytes = S.bytes;
        st->kernel_launches = S.launches;
        st->ms_coarsen = S.tm.ms(0, 1);
        st->ms_initial = S.tm.ms(1, 2);
        st->ms_refine = S.tm.ms(2, 3);
        st->ms_total = S.tm.ms(0, 3);
        st->ms_conn = S.ms_conn;
        st->conn_launches = S.conn_launches;
        st->conn_bytes = S.conn_bytes;
    }
}

void run_vcycle(Ctx& c, const DGraph& g0, int32_t k, float imbalance, uint64_t seed, const gp_options* opt,
                int32_t* d_out, gp_stats* st, const Tracer& tr, const gp_gnn* gnn) {
    VState S;
    vc_begin(c, g0, k, imbalance, seed, opt, S, tr, gnn);
    if (k > 1)
        for (int l = S.L; l >= 0; --l) vc_level(c, S, l, tr);
    vc_end(c, S, d_out, st);
    c.ms_gnn = S.ms_gnn;
}

struct CallGuard {
    DevState* S;
    std::unique_lock<std::mutex> lk;
    Ctx c;
    explicit CallGuard(cudaStream_t s) {
        int dev = 0;
        GP_CUDA(cudaGetDevice(&dev));
        S = dev_state(dev);
        lk = std::unique_lock<std::mutex>(S->mu);
        ensure_init(*S, dev);
        c.s = s;
        c.keep = &S->keep;
        c.tmp = &S->tmp;
        c.sm_count = S->sm_count;
        c.h_pinned = S->pinned;
    }
    ~CallGuard() {
        S->keep.consolidate();
        S->tmp.consolidate();
    }
};

int check_args(int64_t n, int32_t k, float imbalance) {
    if (n < 0) throw GpError(GP_EINVAL, "n must be >= 0");
    if (k < 1 || k > GP_MAX_K) throw GpError(GP_EINVAL, "k must be in [1, " + std::to_string(GP_MAX_K) + "]");
    if (!(imbalance >= 0.0f) || !std::isfinite(imbalance)) throw GpError(GP_EINVAL, "imbalance must be finite and >= 0");
    if (n > 0 && k > n) throw GpError(GP_EINVAL, "k must not exceed the number of vertices");
    if (n > (int64_t)INT32_MAX - 1) throw GpError(GP_EINVAL, "n must fit in int32");
    return 0;
}

template <class F>
static int guarded(F&& f) {
    t_err.clear();
    try {
        f();
        return GP_OK;
    } catch (const GpError& e) {
        t_err = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        t_err = "host allocation failed";
        return GP_ENOMEM;
    } catch (const std::exception& e) {
        t_err = e.what();
        return GP_EINTERNAL;
    }
}

}  // namespace gp

using namespace gp;

extern "C" {

const char* gp_last_error(void) { return t_err.c_str(); }

const char* gp_version(void) {
#ifdef GP_CHECKED
    return "thegraphpartitioning_b200 0.2 (sm_100a, bounds-checked)";
#else
    return "thegraphpartitioning_b200 0.2 (sm_100a)";
#endif
}

int gp_checked_violations(int64_t* count, int32_t* first_site, int32_t clear) {
    return guarded([&] {
        if (!count || !first_site) throw GpError(GP_EINVAL, "null output");
#ifdef GP_CHECKED
        GP_CUDA(cudaDeviceSynchronize());
        unsigned long long c = 0, f = 0;
        for (chk_fetch_fn fn : chk_fetchers()) fn(&c, &f, clear != 0);
        GP_CUDA(cudaGetLastError());
        *count = (int64_t)c;
        *first_site = f ? (int32_t)(f - 1) : -1;
#else
        (void)clear;
        *count = -1;
        *first_site = -1;
        throw GpError(GP_EINVAL, "not the bounds-checked build (libgp_b200_checked.so)");
#endif
    });
}

int gp_default_options(gp_options* opt) {
    return guarded([&] {
        if (!opt) throw GpError(GP_EINVAL, "null options");
        resolve_options(nullptr, 2, opt);
        opt->coarsen_to = 0;  // auto: max(1024, 32*k)
    });
}

int gp_partition_device(int64_t n, const int64_t* d_rowptr, const int32_t* d_colidx, const int32_t* d_vwgt,
                        const int32_t* d_ewgt, int32_t k, float imbalance, uint64_t seed, int32_t* d_part_out,
                        void* stream, const gp_options* opt, gp_stats* stats, gp_trace_fn trace, void* trace_user) {
    return guarded([&] {
        check_args(n, k, imbalance);
        if (n == 0) { if (stats) memset(stats, 0, sizeof *stats); return; }
        if (!d_rowptr || !d_colidx || !d_part_out) throw GpError(GP_EINVAL, "null array");
        CallGuard G((cudaStream_t)stream);
        Ctx& c = G.c;
        DGraph g;
        g.n = n;
        g.rp = d_rowptr;
        GP_CUDA(cudaMemcpyAsync(c.h_pinned, d_rowptr, sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
        GP_CUDA(cudaMemcpyAsync(c.h_pinned + 1, d_rowptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
        c.sync();
        if (c.h_pinned[0] != 0) throw GpError(GP_EINVAL, "rowptr[0] must be 0");
        g.m = c.h_pinned[1];
        if (g.m < 0) throw GpError(GP_EINVAL, "rowptr[n] must be >= 0");
        g.ci = d_colidx; g.ew = d_ewgt; g.vw = d_vwgt;
        Tracer tr; tr.fn = trace; tr.user = trace_user;
        run_vcycle(c, g, k, imbalance, seed, opt, d_part_out, stats, tr);
        c.sync();
    });
}

int gp_partition_learned_device(int64_t n, const int64_t* d_rowptr, const int32_t* d_colidx, const int32_t* d_vwgt,
                                const int32_t* d_ewgt, int32_t k, float imbalance, uint64_t seed, int32_t* d_part_out,
                                void* stream, const gp_options* opt, gp_stats* stats, const gp_gnn* model,
                                int32_t fallback, gp_learned_report* report, gp_trace_fn trace, void* trace_user) {
    return guarded([&] {
        check_args(n, k, imbalance);
        if (!model) throw GpError(GP_EINVAL, "null model");
        if (report) memset(report, 0, sizeof *report);
        if (n == 0) { if (stats) memset(stats, 0, sizeof *stats); return; }
        if (!d_rowptr || !d_colidx || !d_part_out) throw GpError(GP_EINVAL, "null array");
        CallGuard G((cudaStream_t)stream);
        Ctx& c = G.c;
        DGraph g;
        g.n = n;
        g.rp = d_rowptr;
        GP_CUDA(cudaMemcpyAsync(c.h_pinned, d_rowptr, sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
        GP_CUDA(cudaMemcpyAsync(c.h_pinned + 1, d_rowptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
        c.sync();
        if (c.h_pinned[0] != 0) throw GpError(GP_EINVAL, "rowptr[0] must be 0");
        g.m = c.h_pinned[1];
        if (g.m < 0) throw GpError(GP_EINVAL, "rowptr[n] must be >= 0");
        g.ci = d_colidx; g.ew = d_ewgt; g.vw = d_vwgt;
        Tracer tr; tr.fn = trace; tr.user = trace_user;
        // the scorer's float sums follow the row layout, so the learned
        // V-cycle uses one fixed heavy-row threshold and piece length
        gp_options lopt;
        if (opt) lopt = *opt;
        else { memset(&lopt, 0, sizeof lopt); lopt.version = GP_OPTIONS_VERSION; }
        lopt.heavy_deg = kLearnedHeavyDeg;
        lopt.item_len = kLearnedItemLen;
        // the move-order head runs in the multi-kernel refinement loop only
        if (gnn_has_move_head(model)) lopt.small_level_n = 0;
        opt = &lopt;
        gp_stats sl;
        c.ms_gnn = 0;
        run_vcycle(c, g, k, imbalance, seed, opt, d_part_out, &sl, tr, model);
        c.sync();
        gp_stats kept = sl;
        gp_learned_report rep;
        memset(&rep, 0, sizeof rep);
        rep.cut_learned = sl.cut; rep.max_part_weight_learned = sl.max_part_weight; rep.ms_learned = sl.ms_total;
        rep.ms_gnn = c.ms_gnn;
        rep.kept_learned = 1;
        if (fallback) {
            // the plain V-cycle into scratch; its result replaces the learned one
            // unless the learned partition is at least as balanced (within the
            // bound) and cuts no more
            int32_t* plain = c.keep_alloc<int32_t>(n);   // the call's arena, like every other buffer
            gp_stats sp;
            Tracer none;
            run_vcycle(c, g, k, imbalance, seed, opt, plain, &sp, none);
            rep.cut_plain = sp.cut; rep.max_part_weight_plain = sp.max_part_weight; rep.ms_plain = sp.ms_total;
            const bool bl = sl.max_part_weight <= sl.max_allowed, bp = sp.max_part_weight <= sp.max_allowed;
            const bool keep_learned = (bl && !bp) || (bl == bp && sl.cut <= sp.cut);
            rep.kept_learned = keep_learned ? 1 : 0;
            if (!keep_learned) {
                GP_CUDA(cudaMemcpyAsync(d_part_out, plain, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, c.s));
                kept = sp;
            }
            c.sync();
        }
        if (stats) *stats = kept;
        if (report) *report = rep;
    });
}

int gp_partition_ex(int64_t n, const int64_t* rowptr, const int32_t* colidx, const int32_t* vwgt, const int32_t* ewgt,
                    int32_t k, float imbalance, uint64_t seed, int32_t* part_out, const gp_options* opt,
                    gp_stats* stats, gp_trace_fn trace, void* trace_user) {
    return guarded([&] {
        check_args(n, k, imbalance);
        if (n == 0) { if (stats) memset(stats, 0, sizeof *stats); return; }
        if (!rowptr || !colidx || !part_out) throw GpError(GP_EINVAL, "null array");
        if (rowptr[0] != 0) throw GpError(GP_EINVAL, "rowptr[0] must be 0");
        const int64_t m = rowptr[n];
        if (m < 0) throw GpError(GP_EINVAL, "rowptr[n] must be >= 0");
        cudaStream_t s = nullptr;
        GP_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        struct SD { cudaStream_t s; ~SD() { cudaStreamDestroy(s); } } sd{s};
        CallGuard G(s);
        Ctx& c = G.c;
        Timer tm;
        GP_CUDA(cudaEventRecord(tm.e[4], s));
        int64_t* drp = c.keep_alloc<int64_t>(n + 1);
        int32_t* dci = c.keep_alloc<int32_t>(m);
        int32_t* dvw = vwgt ? c.keep_alloc<int32_t>(n) : nullptr;
        int32_t* dew = ewgt ? c.keep_alloc<int32_t>(m) : nullptr;
        int32_t* dout = c.keep_alloc<int32_t>(n);
        GP_CUDA(cudaMemcpyAsync(drp, rowptr, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, s));
        if (m) GP_CUDA(cudaMemcpyAsync(dci, colidx, sizeof(int32_t) * m, cudaMemcpyHostToDevice, s));
        if (vwgt) GP_CUDA(cudaMemcpyAsync(dvw, vwgt, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
        if (ewgt && m) GP_CUDA(cudaMemcpyAsync(dew, ewgt, sizeof(int32_t) * m, cudaMemcpyHostToDevice, s));
        GP_CUDA(cudaEventRecord(tm.e[5], s));
        DGraph g;
        g.n = n; g.m = m; g.rp = drp; g.ci = dci; g.ew = dew; g.vw = dvw;
        Tracer tr; tr.fn = trace; tr.user = trace_user;
        run_vcycle(c, g, k, imbalance, seed, opt, dout, stats, tr);
        GP_CUDA(cudaEventRecord(tm.e[6], s));
        GP_CUDA(cudaMemcpyAsync(part_out, dout, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
        GP_CUDA(cudaEventRecord(tm.e[7], s));
        c.sync();
        if (stats) {
            stats->ms_h2d = tm.ms(4, 5);
            stats->ms_d2h = tm.ms(6, 7);
        }
    });
}

int gp_partition(int64_t n, const int64_t* rowptr, const int32_t* colidx, const int32_t* vwgt, const int32_t* ewgt,
                 int32_t k, float imbalance, uint64_t seed, int32_t* part_out) {
    return gp_partition_ex(n, rowptr, colidx, vwgt, ewgt, k, imbalance, seed, part_out, nullptr, nullptr, nullptr, nullptr);
}

int gp_edge_cut_device(int64_t n, const int64_t* d_rowptr, const int32_t* d_colidx, const int32_t* d_ewgt,
                       const int32_t* d_vwgt, const int32_t* d_part, int32_t k, void* stream, int64_t* cut_out,
                       int64_t* part_weights_out) {
    return guarded([&] {
        if (n < 0) throw GpError(GP_EINVAL, "n must be >= 0");
        if (k < 1 || k > GP_MAX_K) throw GpError(GP_EINVAL, "k must be in [1, " + std::to_string(GP_MAX_K) + "]");
        if (!cut_out) throw GpError(GP_EINVAL, "null cut_out");
        if (n == 0) {
            *cut_out = 0;
            if (part_weights_out) for (int q = 0; q < k; ++q) part_weights_out[q] = 0;
            return;
        }
        if (!d_rowptr || !d_colidx || !d_part) throw GpError(GP_EINVAL, "null array");
        CallGuard G((cudaStream_t)stream);
        Ctx& c = G.c;
        unsigned long long* err = (unsigned long long*)c.tmp_alloc<int64_t>(1);
        GP_CUDA(cudaMemsetAsync(err, 0xff, 8, c.s));
        k_check_part<<<grid_for(n, 256), 256, 0, c.s>>>(n, d_part, k, err);
        GP_LAUNCHED(c);
        GP_CUDA(cudaMemcpyAsync(c.h_pinned, err, 8, cudaMemcpyDeviceToHost, c.s));
        GP_CUDA(cudaMemcpyAsync(c.h_pinned + 1, d_rowptr + n, 8, cudaMemcpyDeviceToHost, c.s));
        c.sync();
        const uint64_t e0 = (uint64_t)c.h_pinned[0];
        if (e0 != ~0ull) throw GpError(GP_EINVAL, verr((int)(e0 >> 48), (int64_t)(e0 & ((1ull << 48) - 1))));
        DGraph g;
        g.n = n; g.m = c.h_pinned[1]; g.rp = d_rowptr; g.ci = d_colidx; g.ew = d_ewgt; g.vw = d_vwgt;
        int64_t* d_c = c.tmp_alloc<int64_t>(1);
        int64_t* d_pw = c.tmp_alloc<int64_t>(k);
        cut_and_weights(c, g, d_part, k, d_c, d_pw);
        GP_CUDA(cudaMemcpyAsync(c.h_pinned, d_c, 8, cudaMemcpyDeviceToHost, c.s));
        if (part_weights_out)
            GP_CUDA(cudaMemcpyAsync(part_weights_out, d_pw, sizeof(int64_t) * k, cudaMemcpyDeviceToHost, c.s));
        c.sync();
        *cut_out = c.h_pinned[0] / 2;
    });
}

int gp_release_workspace(void) {
    return guarded([&] {
        int dev = 0;
        GP_CUDA(cudaGetDevice(&dev));
        DevState* S = dev_state(dev);
        std::lock_guard<std::mutex> lk(S->mu);
        S->keep.release();
        S->tmp.release();
        release_batch_workers(dev);
    });
}

}  // extern "C"
