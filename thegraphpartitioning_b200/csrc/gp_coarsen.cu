// gp_coarsen.cu -- matching and contraction kernels of one coarsening level.
//
// Replaces matchVertices / rematchVertices / resetMatch / mapVertices /
// relabel_coarse_vertices_kernel / countUniqueEdges / prefix_sum /
// fillEdgeArrays / updateRowPtr (src/gpu_part.cu:55-250) and the host loop
// around them (src/gpu_part.cu:1003-1152).
//
// Layout: CSR with int64 row pointers, int32 column ids and int32 weights;
// a NULL weight array means unit weights (the input level only).  Rows longer
// than kHeavyDeg are handled by one CTA each (blocks [0, nheavy) of a launch);
// all other rows by one warp each (grid-stride over the remaining blocks).
#define GP_TU_ID 2   // site ids of the bounds-checked build
#include "gp_internal.cuh"

namespace gp {

// ---------------------------------------------------------------- degree buckets
// Lists in any order (each row is processed on its own).  Appends are
// aggregated per warp: one atomic per warp and bucket.
__device__ __forceinline__ void warp_append(bool take, int32_t v, int32_t* list, int64_t* count, int64_t cap) {
    const uint32_t m = __ballot_sync(0xffffffffu, take);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == __ffs(m) - 1) base = atomicAdd((unsigned long long*)count, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
    const int64_t idx = (int64_t)base + __popc(m & ((1u << lane) - 1u));
    if (take && GP_IN(idx, cap)) list[idx] = v;
}

__global__ void k_buckets(const int64_t* __restrict__ rp, int64_t n, int32_t heavy_deg, int64_t heavy_cap,
                          int32_t* __restrict__ heavy,
                          int32_t* __restrict__ b0, int32_t* __restrict__ b1, int32_t* __restrict__ b2,
                          int64_t* __restrict__ count) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const int64_t v = base + threadIdx.x;
        const int64_t d = v < n ? rp[v + 1] - rp[v] : -1;
        warp_append(v < n && d <= kTile8, (int32_t)v, b0, &count[0], n);
        warp_append(d > kTile8 && d <= kTile32, (int32_t)v, b1, &count[1], n);
        warp_append(d > kTile32 && d <= heavy_deg, (int32_t)v, b2, &count[2], n);
        warp_append(d > heavy_deg, (int32_t)v, heavy, &count[3], heavy_cap);
    }
}

__global__ void k_heavy_bounds(const int64_t* __restrict__ rp, const int32_t* __restrict__ heavy, int64_t nh,
                               int64_t* __restrict__ out) {
    for (int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; h < nh; h += (int64_t)gridDim.x * blockDim.x) {
        out[2 * h] = rp[heavy[h]];
        out[2 * h + 1] = rp[heavy[h] + 1];
    }
}

// cost of light unit u (order: bucket 2, bucket 1, groups of 4 of bucket 0)
__global__ void k_unit_cost(const int64_t* __restrict__ rp, const int32_t* __restrict__ b0, int64_t n0,
                            const int32_t* __restrict__ b1, int64_t n1, const int32_t* __restrict__ b2, int64_t n2,
                            int64_t* __restrict__ cost) {
    const int64_t U0 = (n0 + 3) / 4, U = n2 + n1 + U0;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < U; u += (int64_t)gridDim.x * blockDim.x) {
        int64_t cst = 32;
        if (u < n2) cst += rp[b2[u] + 1] - rp[b2[u]];
        else if (u < n2 + n1) cst += rp[b1[u - n2] + 1] - rp[b1[u - n2]];
        else {
            const int64_t g = u - n2 - n1;
            for (int i = 0; i < 4 && 4 * g + i < n0; ++i) cst += rp[b0[4 * g + i] + 1] - rp[b0[4 * g + i]];
        }
        cost[u] = cst;
    }
}

void build_heavy(Ctx& c, Level& L) {
    auto mk = c.tmp->save();
    int64_t* d_cnt = c.tmp_alloc<int64_t>(4);
    memset_async(c, d_cnt, 0, 4 * sizeof(int64_t));
    const int64_t heavy_cap = std::max<int64_t>(1, L.g.m / L.heavy_deg + 1);
    L.heavy = c.keep_alloc<int32_t>(heavy_cap);
    for (int b = 0; b < 3; ++b) L.bucket[b] = c.keep_alloc<int32_t>(L.g.n);
    k_buckets<<<grid_for(L.g.n, 256), 256, 0, c.s>>>(L.g.rp, L.g.n, L.heavy_deg, heavy_cap, L.heavy, L.bucket[0], L.bucket[1], L.bucket[2],
                                                     d_cnt);
    GP_LAUNCHED(c);
    c.bytes += 8 * (L.g.n + 1) + 4 * L.g.n;
    GP_CUDA(cudaMemcpyAsync(c.h_pinned, d_cnt, 4 * sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
    c.sync();
    for (int b = 0; b < 3; ++b) L.nbucket[b] = c.h_pinned[b];
    L.nheavy = c.h_pinned[3];
    c.tmp->restore(mk);
    // items: heavy row h covers [rp[v], rp[v+1]) in pieces of at most item_len
    std::vector<int64_t> rb((size_t)std::max<int64_t>(L.nheavy, 1)), re((size_t)std::max<int64_t>(L.nheavy, 1));
    if (L.nheavy > 0) {
        // row bounds of the heavy rows
        int64_t* d_rb = c.tmp_alloc<int64_t>(2 * L.nheavy);
        k_heavy_bounds<<<grid_for(L.nheavy, 256), 256, 0, c.s>>>(L.g.rp, L.heavy, L.nheavy, d_rb);
        GP_LAUNCHED(c);
        std::vector<int64_t> hb((size_t)(2 * L.nheavy));
        GP_CUDA(cudaMemcpyAsync(hb.data(), d_rb, sizeof(int64_t) * 2 * L.nheavy, cudaMemcpyDeviceToHost, c.s));
        c.sync();
        c.tmp->restore(mk);
        for (int64_t h = 0; h < L.nheavy; ++h) { rb[h] = hb[2 * h]; re[h] = hb[2 * h + 1]; }
    }
    std::vector<int32_t> irow, rows_items((size_t)std::max<int64_t>(L.nheavy, 1)), rows_first((size_t)std::max<int64_t>(L.nheavy, 1));
    std::vector<int64_t> ib, ie;
    for (int64_t h = 0; h < L.nheavy; ++h) {
        rows_first[h] = (int32_t)irow.size();
        int32_t cnt = 0;
        for (int64_t b = rb[h]; b < re[h]; b += L.item_len) {
            irow.push_back((int32_t)h);
            ib.push_back(b);
            ie.push_back(std::min<int64_t>(b + L.item_len, re[h]));
            ++cnt;
        }
        rows_items[h] = cnt;
    }
    L.nitems = (int64_t)irow.size();
    {
        L.nunits = L.nbucket[2] + L.nbucket[1] + (L.nbucket[0] + 3) / 4;
        int64_t* cost = c.tmp_alloc<int64_t>(L.nunits + 1);
        L.unit_cost = c.keep_alloc<int64_t>(L.nunits + 1);
        k_unit_cost<<<grid_for(L.nunits, 256), 256, 0, c.s>>>(L.g.rp, L.bucket[0], L.nbucket[0], L.bucket[1],
                                                              L.nbucket[1], L.bucket[2], L.nbucket[2], cost);
        GP_LAUNCHED(c);
        scan_excl_i64(c, cost, L.unit_cost, L.nunits, L.unit_cost + L.nunits);
        c.tmp->restore(mk);
    }
    L.item_row = c.keep_alloc<int32_t>(L.nitems);
    L.item_beg = c.keep_alloc<int64_t>(L.nitems);
    L.item_end = c.keep_alloc<int64_t>(L.nitems);
    L.row_items = c.keep_alloc<int32_t>(L.nheavy);
    L.row_first = c.keep_alloc<int32_t>(L.nheavy);
    if (L.nitems > 0) {
        GP_CUDA(cudaMemcpyAsync(L.item_row, irow.data(), sizeof(int32_t) * L.nitems, cudaMemcpyHostToDevice, c.s));
        GP_CUDA(cudaMemcpyAsync(L.item_beg, ib.data(), sizeof(int64_t) * L.nitems, cudaMemcpyHostToDevice, c.s));
        GP_CUDA(cudaMemcpyAsync(L.item_end, ie.data(), sizeof(int64_t) * L.nitems, cudaMemcpyHostToDevice, c.s));
        GP_CUDA(cudaMemcpyAsync(L.row_items, rows_items.data(), sizeof(int32_t) * L.nheavy, cudaMemcpyHostToDevice, c.s));
        GP_CUDA(cudaMemcpyAsync(L.row_first, rows_first.data(), sizeof(int32_t) * L.nheavy, cudaMemcpyHostToDevice, c.s));
        c.sync();  // host vectors go out of scope
    }
}

// ---------------------------------------------------------------- argmax helpers
// Larger key wins; equal keys: smaller id wins (ids compared unsigned so that
// -1, meaning "none", loses every tie).
__device__ __forceinline__ void argmax_merge(uint64_t& k, int32_t& id, uint64_t k2, int32_t i2) {
    if (k2 > k || (k2 == k && (uint32_t)i2 < (uint32_t)id)) { k = k2; id = i2; }
}
__device__ __forceinline__ void warp_argmax(uint64_t& k, int32_t& id) { group_argmax64(0xffffffffu, k, id); }
// the two best distinct neighbours (by argmax_merge's order; a neighbour
// listed twice counts with its larger key) among those offered so far
__device__ __forceinline__ bool key_before(uint64_t k2, int32_t i2, uint64_t k, int32_t i) {
    return k2 > k || (k2 == k && (uint32_t)i2 < (uint32_t)i);
}
__device__ __forceinline__ void top2_insert(uint64_t& k1, int32_t& i1, uint64_t& k2, int32_t& i2, uint64_t k,
                                            int32_t i) {
    if (i == i1) { if (k > k1) k1 = k; return; }
    if (i == i2) {
        if (k > k2) k2 = k;
        if (key_before(k2, i2, k1, i1)) { const uint64_t tk = k1; const int32_t ti = i1; k1 = k2; i1 = i2; k2 = tk; i2 = ti; }
        return;
    }
    if (key_before(k, i, k1, i1)) { k2 = k1; i2 = i1; k1 = k; i1 = i; }
    else if (key_before(k, i, k2, i2)) { k2 = k; i2 = i; }
}
// block-wide; result valid in thread 0
__device__ __forceinline__ void block_argmax(uint64_t& k, int32_t& id, uint64_t* sk, int32_t* sid) {
    warp_argmax(k, id);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) { sk[w] = k; sid[w] = id; }
    __syncthreads();
    if (w == 0) {
        k = lane < nw ? sk[lane] : 0;
        id = lane < nw ? sid[lane] : -1;
        warp_argmax(k, id);
    }
    __syncthreads();
}

// ---------------------------------------------------------------- matching
// MODE 0: proposal to the best eligible unmatched neighbour (handshake round).
// MODE 1: anchor = best neighbour over all neighbours (two-hop pairing).
// Work units as in the connectivity pass: rows of the three degree buckets
// (4 rows per warp for bucket 0, one per warp otherwise), heavy rows one per
// CTA in blocks [0, nheavy).
struct MatchArgs {
    DGraph g;
    const int32_t* heavy;
    int64_t nheavy;
    const int32_t* item_row;   // heavy rows split into items (one CTA each)
    const int64_t* item_beg;
    const int64_t* item_end;
    const int32_t* row_items;
    const int32_t* row_first;
    int64_t nitems;
    uint64_t* ikey;            // per-item partial best
    int32_t* iid;
    int32_t* hdone;            // per heavy row: items finished (reset by the last)
    const int32_t* list[3];   // rows to process, by degree bucket
    int64_t nlist[3];
    const int32_t* match;
    int32_t* out;             // MODE 0: proposals
    uint32_t salt;
    int64_t maxvw;
    uint64_t* keys;           // MODE 1: (anchor << nbits | v)
    int64_t* nkeys;
    int nbits;
    const int32_t* prio;      // learned priorities per entry (nullptr: edge weights)
    int2* cand;               // MODE 0, rows of 33+ entries (one piece): the best eligible
    uint8_t* cmore;           // neighbours of the row's last scan (warp rows: the best; CTA rows:
                              // the two best) and whether it had more (nullptr: no cache)
    int32_t* anchor0;         // the same rows' best neighbour in round 0; with no weight check
                              // that is the two-hop anchor (MODE 1 reads it instead of scanning)
    const uint8_t* hdead;     // MODE 0: heavy rows left without an eligible neighbour (nullptr: none)
    int any_matched;          // MODE 0: 0 in the first round (no neighbour to look up in match[])
    int check_vw;             // MODE 0: 0 when no two vertices of the level can exceed maxvw
};

// high word of an entry's matching priority: learned score or edge weight
__device__ __forceinline__ int32_t key_word(const MatchArgs& A, int64_t e) {
    return A.prio ? A.prio[e] : (A.g.ew ? __ldcs(&A.g.ew[e]) : 1);
}

template <int MODE>
__device__ __forceinline__ bool match_ok(const MatchArgs& A, int64_t v, int32_t u, int64_t vwv) {
    if (u == (int32_t)v || !GP_IN(u, A.g.n)) return false;
    if (MODE == 0) {
        if (A.any_matched && A.match[u] != -1) return false;
        if (A.check_vw && vwv + (A.g.vw ? A.g.vw[u] : 1) > A.maxvw) return false;
    }
    return true;
}

template <int MODE>
__device__ __forceinline__ void match_emit(const MatchArgs& A, bool valid, int64_t v, int32_t best) {
    if (MODE == 0) {
        if (valid) A.out[v] = best;
        return;
    }
    const bool take = valid && best >= 0;
    const uint32_t m = __ballot_sync(0xffffffffu, take);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == __ffs(m) - 1) base = atomicAdd((unsigned long long*)A.nkeys, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
    const int64_t idx = (int64_t)base + __popc(m & ((1u << lane) - 1u));
    if (take && GP_IN(idx, A.g.n)) A.keys[idx] = ((uint64_t)(uint32_t)best << A.nbits) | (uint64_t)v;
}

template <int MODE, int TILE>
__device__ __forceinline__ void match_tile(const MatchArgs& A, int64_t v) {
    const int lane = threadIdx.x & 31, tl = lane & (TILE - 1);
    bool valid = v >= 0;
    if (valid && A.match[v] != -1) valid = false;  // matched already (round 0 / anchors)
    uint64_t bk = 0;
    int32_t bid = -1;
    if (valid) {
        const int64_t e = A.g.rp[v] + tl;
        if (e < A.g.rp[v + 1]) {
            const int32_t u = __ldcs(&A.g.ci[e]);
            const int64_t vwv = A.g.vw ? A.g.vw[v] : 1;
            if (match_ok<MODE>(A, v, u, vwv)) {
                bk = edge_key(key_word(A, e), edge_hash(A.salt, (int32_t)v, u));
                bid = u;
            }
        }
    }
    tile_argmax64<TILE>(bk, bid);
    const bool lead = tl == 0;
    if (MODE == 0) {
        if (lead && v >= 0) A.out[v] = valid ? bid : -1;
    } else {
        match_emit<MODE>(A, lead && valid, v, bid);
    }
}

template <int MODE>
__global__ void __launch_bounds__(256, 6) k_match_scan(MatchArgs A) {
    __shared__ uint64_t sk[32];
    __shared__ int32_t sid[32];
    const int lane = threadIdx.x & 31;
    if ((int64_t)blockIdx.x < A.nitems) {
        // one piece of a long row per CTA; the last piece of a row reduces
        // the partial bests of all its pieces in item order
        const int32_t h = A.item_row[blockIdx.x];
        const int64_t v = A.heavy[h];
        if (A.match[v] != -1 || (A.hdead && A.hdead[h])) { if (MODE == 0 && threadIdx.x == 0) A.out[v] = -1; return; }
        const int nit = A.row_items[h];
        if (MODE == 1 && A.anchor0 && nit == 1) {
            if (threadIdx.x < 32) match_emit<MODE>(A, threadIdx.x == 0, v, A.anchor0[v]);
            return;
        }
        // a row in one piece keeps its two best eligible neighbours (as the warp rows do)
        const bool cached = MODE == 0 && A.cand && nit == 1;
        if (cached && A.any_matched) {
            const int2 cc = A.cand[v];
            const int32_t m1 = cc.x >= 0 ? A.match[cc.x] : 0, m2 = cc.y >= 0 ? A.match[cc.y] : 0;
            int32_t r = -2;
            if (cc.x >= 0 && m1 == -1) r = cc.x;
            else if (cc.y >= 0 && m2 == -1) r = cc.y;
            else if (!A.cmore[v]) r = -1;
            if (r != -2) { if (threadIdx.x == 0) A.out[v] = r; return; }
        }
        const int64_t vwv = A.g.vw ? A.g.vw[v] : 1;
        uint64_t bk = 0; int32_t bid = -1;
        uint64_t k2 = 0; int32_t i2 = -1, cnt = 0;
        const int64_t beg = A.item_beg[blockIdx.x], end = A.item_end[blockIdx.x];
        const int32_t* kw = A.prio ? A.prio : A.g.ew;
        const bool v4 = aligned16(A.g.ci) && aligned16(kw);
        for (int64_t base = beg & ~(int64_t)3; base < end; base += 4 * (int64_t)blockDim.x) {
            int32_t uu[4], ww[4];
            const int64_t e4 = base + 4 * threadIdx.x;
            ld4_row(A.g.ci, e4, beg, end, v4, -1, uu);
            if (kw) ld4_row(kw, e4, beg, end, v4, 0, ww);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if (uu[c] < 0 || !match_ok<MODE>(A, v, uu[c], vwv)) continue;
                const uint64_t key = edge_key(kw ? ww[c] : 1, edge_hash(A.salt, (int32_t)v, uu[c]));
                if (cached) { top2_insert(bk, bid, k2, i2, key, uu[c]); ++cnt; }
                else argmax_merge(bk, bid, key, uu[c]);
            }
        }
        if (cached) {
            __shared__ int32_t s_best, s_cnt;
            const uint64_t k1 = bk;
            const int32_t i1 = bid;
            block_argmax(bk, bid, sk, sid);
            if (threadIdx.x == 0) { s_best = bid; s_cnt = 0; }
            __syncthreads();
            uint64_t ks = i1 == s_best ? k2 : k1;
            int32_t is = i1 == s_best ? i2 : i1;
            block_argmax(ks, is, sk, sid);
            const int32_t wc = (int32_t)__reduce_add_sync(0xffffffffu, (uint32_t)cnt);
            if (lane == 0 && wc) atomicAdd(&s_cnt, wc);
            __syncthreads();
            if (threadIdx.x == 0) {
                A.cand[v] = make_int2(s_best, ks ? is : -1);
                A.cmore[v] = s_cnt > 2 ? 1 : 0;
                if (!A.any_matched && A.anchor0) A.anchor0[v] = s_best;
                A.out[v] = s_best;
            }
            return;
        }
        block_argmax(bk, bid, sk, sid);
        __shared__ int s_last;
        if (threadIdx.x == 0) {
            s_last = 1;
            if (nit > 1) {
                A.ikey[blockIdx.x] = bk;
                A.iid[blockIdx.x] = bid;
                __threadfence();
                s_last = atomicAdd(&A.hdone[h], 1) == nit - 1;
                if (s_last) {
                    __threadfence();
                    bk = 0; bid = -1;
                    const int32_t f = A.row_first[h];
                    for (int i = 0; i < nit; ++i)
                        argmax_merge(bk, bid, __ldcg((const unsigned long long*)&A.ikey[f + i]), __ldcg(&A.iid[f + i]));
                    A.hdone[h] = 0;
                }
            }
        }
        __syncthreads();
        if (s_last && threadIdx.x < 32) match_emit<MODE>(A, threadIdx.x == 0, v, bid);
        return;
    }
    const int64_t wid = ((int64_t)(blockIdx.x - A.nitems) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)(gridDim.x - A.nitems) * blockDim.x) >> 5;
    const int64_t U0 = (A.nlist[0] + 3) / 4, U1 = A.nlist[1], U2 = A.nlist[2];
    for (int64_t u = wid; u < U0 + U1 + U2; u += nw) {
        if (u < U0) {
            const int64_t i = u * 4 + (lane >> 3);
            match_tile<MODE, kTile8>(A, i < A.nlist[0] ? A.list[0][i] : -1);
        } else if (u < U0 + U1) {
            match_tile<MODE, kTile32>(A, A.list[1][u - U0]);
        } else {
            const int64_t v = A.list[2][u - U0 - U1];
            const bool valid = A.match[v] == -1;
            uint64_t bk = 0; int32_t bid = -1;
            bool scan = valid;
            if (MODE == 1 && valid && A.anchor0) { bid = A.anchor0[v]; scan = false; }
            if (MODE == 0 && valid && A.cand && A.any_matched) {
                // neighbours only ever become matched, so the row's cached best
                // eligible neighbour, if still unmatched, is its best eligible
                // neighbour; with it matched and no other eligible entry, none
                const int2 cc = A.cand[v];
                const int32_t m1 = cc.x >= 0 ? A.match[cc.x] : 0, m2 = cc.y >= 0 ? A.match[cc.y] : 0;
                if (cc.x >= 0 && m1 == -1) { bid = cc.x; scan = false; }
                else if (cc.y >= 0 && m2 == -1) { bid = cc.y; scan = false; }
                else if (!A.cmore[v]) { bid = -1; scan = false; }
            }
            int32_t cnt = 0;   // eligible entries
            if (scan) {
                const int64_t vwv = A.g.vw ? A.g.vw[v] : 1;
                const int64_t beg = A.g.rp[v], end = A.g.rp[v + 1];
                // 128 entries per sweep, four consecutive ones per lane (16-byte loads)
                const int32_t* kw = A.prio ? A.prio : A.g.ew;
                const bool v4 = aligned16(A.g.ci) && aligned16(kw);
                for (int64_t base = beg & ~(int64_t)3; base < end; base += 128) {
                    int32_t uu[4], ww[4], mm[4], vv[4];
                    const int64_t e4 = base + 4 * lane;
                    ld4_row(A.g.ci, e4, beg, end, v4, -1, uu);
                    if (kw) ld4_row(kw, e4, beg, end, v4, 0, ww);
                    else {
#pragma unroll
                        for (int c = 0; c < 4; ++c) ww[c] = 1;
                    }
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const bool ok = uu[c] >= 0 && GP_IN(uu[c], A.g.n);
                        if (!ok) uu[c] = -1;
                        mm[c] = (MODE == 0 && A.any_matched && ok) ? A.match[uu[c]] : -1;
                        vv[c] = (MODE == 0 && A.check_vw && ok && A.g.vw) ? A.g.vw[uu[c]] : 1;
                    }
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const int32_t x = uu[c];
                        if (x < 0 || x == (int32_t)v) continue;
                        if (MODE == 0 && (mm[c] != -1 || (A.check_vw && vwv + vv[c] > A.maxvw))) continue;
                        const uint64_t key = edge_key(ww[c], edge_hash(A.salt, (int32_t)v, x));
                        argmax_merge(bk, bid, key, x);
                        if (MODE == 0 && A.cand) ++cnt;
                    }
                }
                warp_argmax(bk, bid);
                if (MODE == 0 && A.cand) {
                    // warp rows keep the best only (a second candidate costs more in
                    // round 0 than the rescans it saves)
                    const int32_t tot = (int32_t)__reduce_add_sync(0xffffffffu, (uint32_t)cnt);
                    if (lane == 0) {
                        A.cand[v] = make_int2(bid, -1);
                        A.cmore[v] = tot > 1 ? 1 : 0;
                        if (!A.any_matched && A.anchor0) A.anchor0[v] = bid;
                    }
                }
            }
            if (MODE == 0) { if (lane == 0) A.out[v] = valid ? bid : -1; }
            else match_emit<MODE>(A, lane == 0 && valid, v, bid);
        }
    }
}

// Mutual proposals become pairs; vertices left unmatched go to the next
// round's worklists, bucketed by degree (any order: each vertex's proposal is
// its own).  A vertex that proposed nobody has no unmatched neighbour within
// the weight cap, and never will (vertices only become matched), so it leaves
// the worklists; a heavy one is flagged in hdead instead (heavy vertices are
// not listed: their CTAs check match[] and hdead[] directly).  next_n[3]
// counts the heavy vertices still live.
__global__ void k_handshake(const int64_t* __restrict__ rp, int64_t n, int32_t heavy_deg, const int32_t* l0,
                            const int32_t* l1,
                            const int32_t* l2, int64_t n0, int64_t n1, int64_t n2, const int32_t* __restrict__ heavy,
                            int64_t nheavy,
                            const int32_t* __restrict__ prop, int32_t* __restrict__ match, int64_t* __restrict__ pairs,
                            int32_t* nl0, int32_t* nl1, int32_t* nl2, int64_t* next_n, uint8_t* __restrict__ hdead) {
    int64_t local = 0;
    const int64_t total = n0 + n1 + n2 + nheavy;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < total; base += stride) {
        const int64_t i = base + threadIdx.x;
        int64_t v = -1;
        if (i < n0) v = l0[i];
        else if (i < n0 + n1) v = l1[i - n0];
        else if (i < n0 + n1 + n2) v = l2[i - n0 - n1];
        else if (i < total) v = heavy[i - n0 - n1 - n2];
        const bool is_heavy = i >= n0 + n1 + n2;
        bool left = false;
        int64_t d = 0;
        if (v >= 0 && match[v] == -1 && !(is_heavy && hdead[i - n0 - n1 - n2])) {
            const int32_t u = prop[v];
            if (u >= 0 && GP_IN(u, n) && prop[u] == (int32_t)v) {
                match[v] = u;
                if (v < u) ++local;
            } else if (u < 0) {
                if (is_heavy) hdead[i - n0 - n1 - n2] = 1;
            } else if (is_heavy) {
                atomicAdd((unsigned long long*)&next_n[3], 1ull);
            } else {
                left = true;
                d = rp[v + 1] - rp[v];
            }
        }
        warp_append(left && d <= kTile8, (int32_t)v, nl0, &next_n[0], n);
        warp_append(left && d > kTile8 && d <= kTile32, (int32_t)v, nl1, &next_n[1], n);
        warp_append(left && d > kTile32 && d <= heavy_deg, (int32_t)v, nl2, &next_n[2], n);
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd((unsigned long long*)pairs, (unsigned long long)local);
}

// sorted (anchor << nbits | v) keys: pair ranks (0,1), (2,3), ... of each anchor group
__global__ void k_twohop_pair(const uint64_t* __restrict__ keys, int64_t cnt, int64_t n, int nbits,
                              const int32_t* __restrict__ vw,
                              int64_t maxvw, int32_t* __restrict__ match, int64_t* __restrict__ pairs) {
    int64_t local = 0;
    const uint64_t lowmask = (1ull << nbits) - 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t a = keys[i] >> nbits;
        // first index of this anchor group (lower bound)
        int64_t lo = 0, hi = i;
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if ((keys[mid] >> nbits) < a) lo = mid + 1; else hi = mid;
        }
        if (((i - lo) & 1) || i + 1 >= cnt || (keys[i + 1] >> nbits) != a) continue;
        const int32_t x = (int32_t)(keys[i] & lowmask), y = (int32_t)(keys[i + 1] & lowmask);
        if (!GP_IN(x, n) || !GP_IN(y, n)) continue;
        const int64_t wx = vw ? vw[x] : 1, wy = vw ? vw[y] : 1;
        if (wx + wy <= maxvw) { match[x] = y; match[y] = x; ++local; }
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd((unsigned long long*)pairs, (unsigned long long)local);
}

static int bits_for(int64_t x) {  // bits to represent values in [0, x)
    int b = 1;
    while ((1ll << b) < x) ++b;
    return b;
}

__global__ void k_max_vw(int64_t n, const int32_t* __restrict__ vw, int64_t* __restrict__ out) {
    int32_t mx = 0;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        mx = vw[v] > mx ? vw[v] : mx;
    for (int o = 16; o > 0; o >>= 1) { const int32_t y = __shfl_xor_sync(0xffffffffu, mx, o); mx = y > mx ? y : mx; }
    if ((threadIdx.x & 31) == 0 && mx) atomicMax((unsigned long long*)out, (unsigned long long)mx);
}

int64_t match_level(Ctx& c, const Level& L, int level, const Params& P, int32_t* match, int* rounds_out,
                    const int32_t* prio) {
    const DGraph& g = L.g;
    const uint32_t salt = edge_salt(P.seed, level);
    auto mk = c.tmp->save();
    int32_t* prop = c.tmp_alloc<int32_t>(g.n);
    int32_t* wl[2][3];
    for (int s2 = 0; s2 < 2; ++s2)
        for (int b = 0; b < 3; ++b) wl[s2][b] = c.tmp_alloc<int32_t>(std::max<int64_t>(L.nbucket[b], 1));
    int64_t* d_cnt = c.tmp_alloc<int64_t>(8);
    GP_CUDA(cudaMemsetAsync(match, 0xff, sizeof(int32_t) * g.n, c.s));
    MatchArgs A;
    A.g = g; A.heavy = L.heavy; A.nheavy = L.nheavy; A.match = match; A.out = prop; A.salt = salt;
    A.item_row = L.item_row; A.item_beg = L.item_beg; A.item_end = L.item_end; A.row_items = L.row_items;
    A.row_first = L.row_first; A.nitems = L.nitems;
    A.ikey = c.tmp_alloc<uint64_t>(std::max<int64_t>(L.nitems, 1));
    A.iid = c.tmp_alloc<int32_t>(std::max<int64_t>(L.nitems, 1));
    A.hdone = c.tmp_alloc<int32_t>(std::max<int64_t>(L.nheavy, 1));
    memset_async(c, A.hdone, 0, sizeof(int32_t) * std::max<int64_t>(L.nheavy, 1));
    A.maxvw = P.maxvw; A.keys = nullptr; A.nkeys = nullptr; A.nbits = 0; A.prio = prio;
    // rows of 33+ entries keep their two best eligible neighbours between rounds (written by round 0)
    A.cand = c.tmp_alloc<int2>(g.n);
    A.cmore = c.tmp_alloc<uint8_t>(g.n);
    A.anchor0 = c.tmp_alloc<int32_t>(g.n);
    // weight cap: skip the per-neighbour weight check when the two heaviest
    // vertices of the level together stay within maxvw
    A.check_vw = 0;
    if (g.vw) {
        int64_t* d_mx = c.tmp_alloc<int64_t>(1);
        memset_async(c, d_mx, 0, sizeof(int64_t));
        k_max_vw<<<grid_for(g.n, 256, c.sm_count * 4), 256, 0, c.s>>>(g.n, g.vw, d_mx);
        GP_LAUNCHED(c);
        A.check_vw = 2 * read_i64(c, d_mx) > P.maxvw ? 1 : 0;
    } else {
        A.check_vw = 2 > P.maxvw ? 1 : 0;
    }
    uint8_t* hdead = c.tmp_alloc<uint8_t>(std::max<int64_t>(L.nheavy, 1));
    memset_async(c, hdead, 0, std::max<int64_t>(L.nheavy, 1));
    A.hdead = hdead;
    for (int b = 0; b < 3; ++b) { A.list[b] = L.bucket[b]; A.nlist[b] = L.nbucket[b]; }
    int64_t pairs = 0, heavy_live = L.nheavy;
    int rounds = 0;
    bool anchors_ready = false;   // round 0 ran and wrote anchor0
    for (int r = 0; r < P.o.match_rounds; ++r) {
        const int64_t units = (A.nlist[0] + 3) / 4 + A.nlist[1] + A.nlist[2];
        // nobody left who can propose: this round would add no pair
        if (units == 0 && heavy_live == 0) { rounds = r + 1; break; }
        A.any_matched = r > 0 ? 1 : 0;
        const int grid = (int)L.nitems + grid_for(units * 32, 256, c.sm_count * c.ctas_per_sm);
        memset_async(c, d_cnt, 0, 5 * sizeof(int64_t));
        k_match_scan<0><<<grid, 256, 0, c.s>>>(A);
        GP_LAUNCHED(c);
        if (r == 0) anchors_ready = true;
        int32_t** nxt = wl[r & 1];
        const int64_t tot = A.nlist[0] + A.nlist[1] + A.nlist[2] + L.nheavy;
        k_handshake<<<grid_for(tot, 256), 256, 0, c.s>>>(g.rp, g.n, L.heavy_deg, A.list[0], A.list[1], A.list[2], A.nlist[0], A.nlist[1],
                                                         A.nlist[2], L.heavy, L.nheavy, prop, match, d_cnt, nxt[0],
                                                         nxt[1], nxt[2], d_cnt + 1, hdead);
        GP_LAUNCHED(c);
        const int64_t share = g.n ? (tot * 1000) / g.n : 0;
        c.bytes += (L.scan_bytes() + 4 * g.m) * share / 1000 + 16 * tot;
        GP_CUDA(cudaMemcpyAsync(c.h_pinned, d_cnt, 5 * sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
        c.sync();
        const int64_t newp = c.h_pinned[0];
        heavy_live = c.h_pinned[4];
        rounds = r + 1;
        pairs += newp;
        for (int b = 0; b < 3; ++b) { A.list[b] = nxt[b]; A.nlist[b] = c.h_pinned[1 + b]; }
        if (newp == 0) break;
    }
    if (P.o.two_hop > 0 && 4 * (g.n - pairs) > 3 * g.n) {
        const int nb = bits_for(g.n);
        uint64_t* keys = c.tmp_alloc<uint64_t>(g.n);
        uint64_t* keys2 = c.tmp_alloc<uint64_t>(g.n);
        int32_t* vals = c.tmp_alloc<int32_t>(g.n);
        int32_t* vals2 = c.tmp_alloc<int32_t>(g.n);
        memset_async(c, d_cnt, 0, 2 * sizeof(int64_t));
        MatchArgs B2 = A;
        B2.hdead = nullptr;   // anchors: the top neighbour over all neighbours
        B2.cand = nullptr; B2.cmore = nullptr;
        // round 0 saw every neighbour but v itself when no pair can exceed the weight cap
        if (A.check_vw || !anchors_ready) B2.anchor0 = nullptr;
        B2.any_matched = 1;
        for (int b = 0; b < 3; ++b) { B2.list[b] = L.bucket[b]; B2.nlist[b] = L.nbucket[b]; }
        B2.out = nullptr; B2.keys = keys; B2.nkeys = d_cnt + 1; B2.nbits = nb;
        const int64_t units = (B2.nlist[0] + 3) / 4 + B2.nlist[1] + B2.nlist[2];
        const int grid = (int)L.nitems + grid_for(units * 32, 256, c.sm_count * c.ctas_per_sm);
        k_match_scan<1><<<grid, 256, 0, c.s>>>(B2);
        GP_LAUNCHED(c);
        c.bytes += L.scan_bytes() + 4 * g.n;
        int64_t cnt = read_i64(c, d_cnt + 1);
        if (cnt > 1) {
            GP_CUDA(cudaMemsetAsync(vals, 0, sizeof(int32_t) * cnt, c.s));
            radix_sort_pairs(c, keys, vals, keys2, vals2, cnt, 2 * nb);
            k_twohop_pair<<<grid_for(cnt, 256), 256, 0, c.s>>>(keys, cnt, g.n, nb, g.vw, P.maxvw, match, d_cnt);
            GP_LAUNCHED(c);
            c.bytes += 24 * cnt;
            pairs += read_i64(c, d_cnt);
        }
    }
    c.tmp->restore(mk);
    if (rounds_out) *rounds_out = rounds;
    return pairs;
}

// ---------------------------------------------------------------- contraction
__global__ void k_rep_flags(int64_t n, const int32_t* __restrict__ match, int32_t* __restrict__ flag) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = match[v];
        flag[v] = (u < 0 || v < u) ? 1 : 0;
    }
}

// cmap for every fine vertex; members, weight and row-length bound per coarse vertex
__global__ void k_cmap(DGraph g, const int32_t* __restrict__ match, const int64_t* __restrict__ cid,
                       int32_t* __restrict__ cmap, int32_t* __restrict__ mem, int32_t* __restrict__ cvw,
                       int64_t* __restrict__ cdeg) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < g.n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = match[v];
        const bool rep = (u < 0 || v < u);
        const int64_t r = rep ? v : u;
        if (!GP_IN(r, g.n)) continue;
        const int32_t cc = (int32_t)cid[r];
        cmap[v] = cc;
        if (rep) {
            mem[2 * (int64_t)cc] = (int32_t)v;
            mem[2 * (int64_t)cc + 1] = u;
            int64_t w = g.vw ? g.vw[v] : 1;
            int64_t d = g.rp[v + 1] - g.rp[v];
            if (u >= 0) { w += g.vw ? g.vw[u] : 1; d += g.rp[u + 1] - g.rp[u]; }
            cvw[cc] = (int32_t)w;
            cdeg[cc] = d;
        }
    }
}

// ---- row dedup in first-occurrence order
// Coarse row c walks N(a) then N(b) (a = representative, b = partner) in CSR
// order; position j in that walk.  Every coarse neighbour is kept once, at
// the rank of its first position, with the weights of all its positions
// summed; c itself is dropped.
//
// Tiers A, B, C and C2 read the walk straight from the fine CSR, mapping each
// column id through cmap as they go, and read it once.  Tier D reads its rows
// three times, so k_fill_walk_d first writes those rows, mapped, into a walk
// layout (row c at off[c]).  Every tier writes its unique entries at off[c]
// (a bound on the row) and k_contract_copy packs them.  Tiers by row length d:
//   A  d <= 128        one warp, 256-slot table in shared memory
//   A2 d <= 256        one warp, 512-slot table
//   B  d <= 512        one warp, 1024-slot table (11 KB per warp: 20 warps per SM)
//   C1 d <= 2048       one CTA of 256 threads, two-phase (first position kept by
//                      atomicMax of deg - j), 4096-slot table on chip (54 KB: four
//                      CTAs per SM)
//   C  d <= 4096       the same with 512 threads and an 8192-slot table (108 KB: two
//                      CTAs per SM)
//   C2 d <= 12288      the same with 1024 threads and a 16384-slot table (196 KB:
//                      one CTA per SM; load factor at most 3/4)
//   C3 d <= 65536      one 1024-thread CTA, the C2 table in P = 2..8 passes: pass p
//                      dedups the keys whose pass hash is p, first positions are
//                      marked in a shared-memory bitmap of the whole walk
//   D  longer          pieces of 16K entries, one CTA each, table in global memory
// A and B insert 32 entries at a time in walk order (match_any leaders), so
// new neighbours get consecutive ranks; C and D rank first positions with one
// block scan over per-thread contiguous segments.  The on-chip tables are
// cleared once per CTA and afterwards only in the slots a row used.
constexpr int TA_ROW = 128, TA_SLOTS = 256;
constexpr int TA2_ROW = 256, TA2_SLOTS = 512;
constexpr int TB_ROW = 512, TB_SLOTS = 1024, TB_WARPS = 4;
constexpr int TC1_ROW = 2048, TC1_SLOTS = 4096, TC1_T = 256;
constexpr int TC_ROW = 4096, TC_SLOTS = 8192, TC_T = 512;
constexpr int TC2_ROW = 12288, TC2_SLOTS = 16384, TC2_T = 1024;
constexpr int TC3_ROW = 65536, TC3_KEYS = 12288;   // at most TC3_KEYS walk entries per pass on average
constexpr int TD_T = 1024;
constexpr int32_t EMPTY_KEY = -1;

__device__ __forceinline__ uint32_t slot_hash(int32_t key, int lg) {
    return ((uint32_t)key * 0x9E3779B1u) >> (32 - lg);
}

// The walk of coarse row c in the fine CSR: positions [0, da) are a's row,
// [da, deg) b's row (a = representative, b = partner or none).
struct Walk {
    int64_t ea, da, eb;
    __device__ __forceinline__ int64_t entry(int64_t j) const { return j < da ? ea + j : eb + (j - da); }
};
__device__ __forceinline__ Walk walk_of(const DGraph& g, const int32_t* __restrict__ mem, int64_t c) {
    const int32_t a = mem[2 * c], b = mem[2 * c + 1];
    Walk W;
    W.ea = g.rp[a];
    W.da = g.rp[a + 1] - W.ea;
    W.eb = b >= 0 ? g.rp[b] : 0;
    return W;
}
// mapped id and weight of walk position j
__device__ __forceinline__ void walk_load(const DGraph& g, const int32_t* __restrict__ cmap, const Walk& W, int64_t j,
                                          int32_t& cu, int32_t& w) {
    const int64_t e = W.entry(j);
    const int32_t u = __ldcs(&g.ci[e]);
    cu = GP_IN(u, g.n) ? cmap[u] : 0;
    w = g.ew ? __ldcs(&g.ew[e]) : 1;
}

// tier-D rows in walk layout, by the pieces the tier-D kernels use
struct TierD;
__global__ void k_fill_walk_d(TierD D, DGraph g, const int32_t* __restrict__ cmap, const int32_t* __restrict__ mem,
                              const int64_t* __restrict__ off, int32_t* __restrict__ mapped, int32_t* __restrict__ mw);

// Ordered insertion of one walk by one warp into a shared-memory table.
// okey/wacc: output ids and weights by rank (shared), oslot: the slot of each
// rank (the row's used slots, cleared afterwards); returns the row length.
template <int SLOTS, class IdxT>
__device__ __forceinline__ int32_t warp_dedup(const DGraph& g, const int32_t* __restrict__ cmap, const Walk& W,
                                              int64_t deg, int32_t self, int32_t* key, IdxT* tidx, IdxT* oslot,
                                              int32_t* okey, int32_t* wacc, int lg) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    int32_t count = 0;
    int32_t cu_next = -1, w_next = 0;
    if (lane < deg) walk_load(g, cmap, W, lane, cu_next, w_next);
    for (int64_t base = 0; base < deg; base += 32) {
        const int64_t j = base + lane;
        const int32_t cu = cu_next, wt = w_next;
        // prefetch the next chunk
        if (j + 32 < deg) walk_load(g, cmap, W, j + 32, cu_next, w_next);
        const bool act = (j < deg) && cu != self;
        const uint32_t peers = __match_any_sync(0xffffffffu, act ? (uint32_t)cu : (0x80000000u | (uint32_t)lane));
        const int leader = __ffs(peers) - 1;
        bool isnew = false;
        int32_t h = -1;
        if (act && lane == leader) {
            h = (int32_t)slot_hash(cu, lg);
            for (int probe = 0; probe < SLOTS; ++probe) {
                const int32_t old = atomicCAS(&key[h], EMPTY_KEY, cu);
                if (old == EMPTY_KEY) { isnew = true; break; }
                if (old == cu) break;
                h = (h + 1) & (SLOTS - 1);
            }
        }
        const uint32_t newmask = __ballot_sync(0xffffffffu, isnew);
        int32_t idx = -1;
        if (isnew) {
            idx = count + __popc(newmask & lt);
            tidx[h] = (IdxT)idx;
            oslot[idx] = (IdxT)h;
            okey[idx] = cu;
        }
        __syncwarp();
        if (act && lane == leader && !isnew) idx = tidx[h];
        idx = __shfl_sync(0xffffffffu, idx, leader);
        if (act) atomicAdd(&wacc[idx], wt);
        count += __popc(newmask);
        __syncwarp();
    }
    return count;
}

template <int MAXROW, int SLOTS, class IdxT>
__host__ __device__ constexpr size_t warp_dedup_smem() {
    return ((sizeof(int32_t) * (SLOTS + 2 * MAXROW) + sizeof(IdxT) * (SLOTS + MAXROW)) + 15) & ~(size_t)15;
}

// tiers A (MAXROW 128) and B (MAXROW 1024): one warp per row
template <int MAXROW, int SLOTS, int WARPS, class IdxT>
__global__ void __launch_bounds__(WARPS * 32) k_dedup_warp(DGraph g, const int32_t* __restrict__ cmap,
                                                           const int32_t* __restrict__ mem, int64_t nc, int64_t minrow,
                                                           const int64_t* __restrict__ off,
                                                           const int64_t* __restrict__ cdeg, int32_t* __restrict__ tci,
                                                           int32_t* __restrict__ tew, int32_t* __restrict__ cnt) {
    // dynamic shared memory per warp: key[SLOTS] okey[MAXROW] wacc[MAXROW] idx[SLOTS] oslot[MAXROW]
    extern __shared__ int32_t dsm[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const size_t per_warp = warp_dedup_smem<MAXROW, SLOTS, IdxT>() / sizeof(int32_t);
    int32_t* key = dsm + w * per_warp;
    int32_t* okey = key + SLOTS;
    int32_t* wacc = okey + MAXROW;
    IdxT* tidx = (IdxT*)(wacc + MAXROW);
    IdxT* oslot = tidx + SLOTS;
    for (int i = lane; i < SLOTS; i += 32) key[i] = EMPTY_KEY;
    for (int i = lane; i < MAXROW; i += 32) wacc[i] = 0;
    __syncwarp();
    int lg = 0;
    while ((1 << lg) < SLOTS) ++lg;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = wid; c < nc; c += nw) {
        const int64_t deg = cdeg[c];
        if (deg > MAXROW || deg < minrow) continue;
        const int64_t o = off[c];
        const int32_t count = warp_dedup<SLOTS, IdxT>(g, cmap, walk_of(g, mem, c), deg, (int32_t)c, key, tidx, oslot,
                                                      okey, wacc, lg);
        for (int i = lane; i < count; i += 32) {
            tci[o + i] = okey[i];
            tew[o + i] = wacc[i];
            wacc[i] = 0;
            key[oslot[i]] = EMPTY_KEY;
        }
        if (lane == 0) cnt[c] = count;
        __syncwarp();
    }
}

__device__ __forceinline__ int32_t block_scan_excl(int32_t x, int32_t* sh, int32_t& total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) { int32_t y = __shfl_up_sync(0xffffffffu, inc, o); if (lane >= o) inc += y; }
    if (lane == 31) sh[w] = inc;
    __syncthreads();
    if (w == 0) {
        int32_t s2 = lane < nw ? sh[lane] : 0, i2 = s2;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) { int32_t y = __shfl_up_sync(0xffffffffu, i2, o); if (lane >= o) i2 += y; }
        if (lane < nw) sh[lane] = i2 - s2;
        if (lane == nw - 1) sh[32] = i2;
    }
    __syncthreads();
    const int32_t r = inc - x + sh[w];
    total = sh[32];
    __syncthreads();
    return r;
}

// rows longer than TB_ROW: lists of the on-chip tiers C1 (<= TC1_ROW), C
// (<= TC_ROW), C2 (<= TC2_ROW), C3 (<= TC3_ROW) and of tier D.  count[0] =
// rows of tier C, count[1] = rows of tier D, count[2] = longest tier-D row,
// count[3] = rows of tier C2, count[4] = rows of tier C3, count[5] = rows of
// tier C1
__global__ void k_long_rows(int64_t nc, const int64_t* __restrict__ cdeg, int32_t* __restrict__ listC1,
                            int32_t* __restrict__ listC, int32_t* __restrict__ listC2, int32_t* __restrict__ listC3,
                            int32_t* __restrict__ listD, int64_t* __restrict__ count) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = cdeg[c];
        if (d <= TB_ROW) continue;
        if (d <= TC1_ROW) {
            unsigned long long slot = atomicAdd((unsigned long long*)&count[5], 1ull);
            listC1[slot] = (int32_t)c;
        } else if (d <= TC_ROW) {
            unsigned long long slot = atomicAdd((unsigned long long*)&count[0], 1ull);
            listC[slot] = (int32_t)c;
        } else if (d <= TC2_ROW) {
            unsigned long long slot = atomicAdd((unsigned long long*)&count[3], 1ull);
            listC2[slot] = (int32_t)c;
        } else if (d <= TC3_ROW) {
            unsigned long long slot = atomicAdd((unsigned long long*)&count[4], 1ull);
            listC3[slot] = (int32_t)c;
        } else {
            unsigned long long slot = atomicAdd((unsigned long long*)&count[1], 1ull);
            listD[slot] = (int32_t)c;
            atomicMax((unsigned long long*)&count[2], (unsigned long long)d);
        }
    }
}

// tiers C and C2: one CTA per row, table in shared memory, two phases.
// Phase 1 reads the walk once (straight from the fine CSR) and inserts every
// entry into a 64-bit slot (key + 1) << 32 | (deg - j), zero meaning empty:
// the claiming compare-and-swap stores the first position seen, later copies
// raise it by atomicMax (the largest deg - j is the first occurrence);
// weights add up in wsum, and position j keeps its slot in hj[j].  Phase 2:
// warps ballot the first-occurrence flags (slot value == deg - j) of 32
// consecutive positions into one word each, one block scan over the word
// popcounts gives each word's base rank, and a second sweep writes the first
// occurrences at base + rank within the word, then empties their slots (each
// used slot has exactly one first occurrence), so the table is clear for the
// CTA's next row.  words: 2 * ceil(deg/32) ints (bits, then prefix).
constexpr uint16_t NO_SLOT = 0xFFFF;
template <int T>
__device__ void cta_dedup(const DGraph& g, const int32_t* __restrict__ cmap, const Walk& W, int64_t o, int64_t deg,
                          int32_t self, unsigned long long* slot, int32_t* wsum, uint16_t* hj, int lg,
                          int32_t* words, int32_t* __restrict__ tci, int32_t* __restrict__ tew, int32_t* cnt_out,
                          int32_t* sh, int32_t* err) {
    const uint32_t S = 1u << lg, mask = S - 1u;
    for (int64_t base = 0; base < deg; base += 4 * T) {
        int32_t cu[4], wt[4];
        unsigned long long val[4], old[4];
        uint32_t h[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int64_t j = base + c * T + threadIdx.x;
            cu[c] = self; wt[c] = 0;
            if (j < deg) walk_load(g, cmap, W, j, cu[c], wt[c]);
            val[c] = ((unsigned long long)((uint32_t)cu[c] + 1u) << 32) | (uint32_t)(deg - j);
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            h[c] = slot_hash(cu[c], lg);
            old[c] = cu[c] != self ? atomicCAS(&slot[h[c]], 0ull, val[c]) : 0ull;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int64_t j = base + c * T + threadIdx.x;
            if (j >= deg) continue;
            if (cu[c] == self) { hj[j] = NO_SLOT; continue; }
            const uint32_t tag = (uint32_t)cu[c] + 1u;
            uint32_t probe = 1;
            while (old[c] != 0ull && (uint32_t)(old[c] >> 32) != tag && probe < S) {
                h[c] = (h[c] + 1) & mask;
                old[c] = atomicCAS(&slot[h[c]], 0ull, val[c]);
                ++probe;
            }
            if (old[c] != 0ull && (uint32_t)(old[c] >> 32) != tag) { atomicExch(err, 1); hj[j] = NO_SLOT; continue; }
            if (old[c] != 0ull && old[c] < val[c]) atomicMax(&slot[h[c]], val[c]);
            atomicAdd(&wsum[h[c]], wt[c]);
            hj[j] = (uint16_t)h[c];
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = T / 32;
    const int64_t nwords = (deg + 31) / 32;
    int32_t* bits = words;
    int32_t* wpre = words + nwords;
    for (int64_t wi = wid; wi < nwords; wi += nwarp) {
        const int64_t j = wi * 32 + lane;
        bool first = false;
        if (j < deg) {
            const uint16_t hh = hj[j];
            first = hh != NO_SLOT && (uint32_t)slot[hh] == (uint32_t)(deg - j);
        }
        const uint32_t word = __ballot_sync(0xffffffffu, first);
        if (lane == 0) bits[wi] = (int32_t)word;
    }
    __syncthreads();
    // exclusive scan of word popcounts: contiguous word ranges per thread
    const int64_t per = (nwords + T - 1) / T;
    const int64_t w0 = (int64_t)threadIdx.x * per, w1 = w0 + per < nwords ? w0 + per : nwords;
    int32_t mine = 0;
    for (int64_t wi = w0; wi < w1; ++wi) mine += __popc((uint32_t)bits[wi]);
    int32_t tot;
    int32_t run = block_scan_excl(mine, sh, tot);
    for (int64_t wi = w0; wi < w1; ++wi) { wpre[wi] = run; run += __popc((uint32_t)bits[wi]); }
    __syncthreads();
    const uint32_t lt = (1u << lane) - 1u;
    for (int64_t wi = wid; wi < nwords; wi += nwarp) {
        const uint32_t word = (uint32_t)bits[wi];
        if (!((word >> lane) & 1u)) continue;
        const uint16_t hh = hj[wi * 32 + lane];
        const int32_t r = wpre[wi] + __popc(word & lt);
        if (!GP_IN(r, deg) || !GP_IN(hh, S)) continue;
        tci[o + r] = (int32_t)((uint32_t)(slot[hh] >> 32) - 1u);
        tew[o + r] = wsum[hh];
    }
    __syncthreads();
    for (int64_t wi = wid; wi < nwords; wi += nwarp) {
        const uint32_t word = (uint32_t)bits[wi];
        if (!((word >> lane) & 1u)) continue;
        const uint16_t hh = hj[wi * 32 + lane];
        slot[hh] = 0ull;
        wsum[hh] = 0;
    }
    if (threadIdx.x == 0) *cnt_out = tot;
    __syncthreads();
}

// shared memory of an on-chip tier: SLOTS 64-bit slots and int32 weight sums,
// a slot id per walk position, two words per 32 entries of the longest row
template <int SLOTS, int MAXROW>
constexpr size_t cta_dedup_smem() {
    return (sizeof(unsigned long long) + sizeof(int32_t)) * SLOTS + sizeof(uint16_t) * MAXROW +
           sizeof(int32_t) * 2 * ((MAXROW + 31) / 32);
}

// tiers C and C2: table of at least twice the row length, at most SLOTS
template <int T, int SLOTS, int MAXROW>
__global__ void __launch_bounds__(T) k_dedup_cta_smem(DGraph g, const int32_t* __restrict__ cmap,
                                                      const int32_t* __restrict__ mem, const int32_t* __restrict__ list,
                                                      int64_t nlist, const int64_t* __restrict__ off,
                                                      const int64_t* __restrict__ cdeg, int32_t* __restrict__ tci,
                                                      int32_t* __restrict__ tew, int32_t* __restrict__ cnt,
                                                      int32_t* __restrict__ err) {
    static_assert(SLOTS <= 65535, "slot ids are 16-bit");
    extern __shared__ __align__(16) unsigned char stab_raw[];
    unsigned long long* slot = (unsigned long long*)stab_raw;          // SLOTS
    int32_t* wsum = (int32_t*)(slot + SLOTS);                          // SLOTS
    uint16_t* hj = (uint16_t*)(wsum + SLOTS);                          // MAXROW
    int32_t* words = (int32_t*)(hj + ((MAXROW + 1) & ~1));             // 2 * MAXROW / 32
    __shared__ int32_t sh[33];
    for (int i = threadIdx.x; i < SLOTS; i += T) { slot[i] = 0ull; wsum[i] = 0; }
    __syncthreads();
    for (int64_t li = blockIdx.x; li < nlist; li += gridDim.x) {
        const int64_t c = list[li];
        const int64_t deg = cdeg[c];
        int64_t S = 1;
        int lg = 0;
        while (S < 2 * deg && S < SLOTS) { S <<= 1; ++lg; }
        cta_dedup<T>(g, cmap, walk_of(g, mem, c), off[c], deg, (int32_t)c, slot, wsum, hj, lg, words, tci, tew,
                     &cnt[c], sh, err);
    }
}

// rows of a one-CTA-per-row tier, longest walk first: the block scheduler
// starts CTAs in list order, so the long rows no longer trail the launch
__global__ void k_len_keys(const int32_t* __restrict__ list, int64_t nlist, const int64_t* __restrict__ cdeg,
                           int64_t maxrow, uint64_t* __restrict__ keys, int32_t* __restrict__ vals) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nlist; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = list[i];
        const int64_t d = cdeg[c];
        keys[i] = (uint64_t)(d < maxrow ? maxrow - d : 0);
        vals[i] = c;
    }
}
static int32_t* longest_first(Ctx& c, const int32_t* list, int64_t nlist, const int64_t* cdeg, int64_t maxrow) {
    uint64_t* keys = c.tmp_alloc<uint64_t>(nlist);
    uint64_t* keys2 = c.tmp_alloc<uint64_t>(nlist);
    int32_t* vals = c.tmp_alloc<int32_t>(nlist);
    int32_t* vals2 = c.tmp_alloc<int32_t>(nlist);
    k_len_keys<<<grid_for(nlist, 256), 256, 0, c.s>>>(list, nlist, cdeg, maxrow, keys, vals);
    GP_LAUNCHED(c);
    radix_sort_pairs(c, keys, vals, keys2, vals2, nlist, bits_for(maxrow + 1));
    return vals;
}

// tier C3: one 1024-thread CTA per row of TC2_ROW < d <= TC3_ROW walk entries.
// Pass 0 gathers the walk through cmap once and leaves the mapped ids and
// weights in the row's range of the scratch arrays (key_at, w_at); passes
// 1..P-1 read them from there (P = the power of two with d / P <= TC3_KEYS).
// Pass p inserts only the keys whose pass hash is p into the 16384-slot table
// (the same 64-bit slots as tier C: (key + 1) << 32 | (d - j), first position
// kept by atomicMax, weights summed), then every used slot marks its first
// position in a bitmap of the walk, leaves its weight sum at that position of
// w_at (later passes never read the weights of another pass's keys), and is
// cleared.  After the passes one block scan ranks
// the marked positions and the keys are written in first-occurrence order, as
// every other tier writes them.
constexpr size_t tc3_smem() {
    return (sizeof(unsigned long long) + sizeof(int32_t)) * TC2_SLOTS + sizeof(uint32_t) * 2 * (TC3_ROW / 32);
}
__device__ __forceinline__ uint32_t pass_of(int32_t key, int lgp) {
    return lgp ? ((uint32_t)key * 0x85EBCA77u) >> (32 - lgp) : 0u;
}
__global__ void __launch_bounds__(TC2_T) k_dedup_multipass(DGraph g, const int32_t* __restrict__ cmap,
                                                           const int32_t* __restrict__ mem,
                                                           const int32_t* __restrict__ list, int64_t nlist,
                                                           const int64_t* __restrict__ off,
                                                           const int64_t* __restrict__ cdeg,
                                                           int32_t* __restrict__ key_at, int32_t* __restrict__ w_at,
                                                           int32_t* __restrict__ tci, int32_t* __restrict__ tew,
                                                           int32_t* __restrict__ cnt, int32_t* __restrict__ err) {
    constexpr int T = TC2_T, S = TC2_SLOTS, LG = 14;
    static_assert((1 << LG) == S, "table size");
    extern __shared__ __align__(16) unsigned char mp_raw[];
    unsigned long long* slot = (unsigned long long*)mp_raw;            // S
    int32_t* wsum = (int32_t*)(slot + S);                              // S
    uint32_t* bits = (uint32_t*)(wsum + S);                            // TC3_ROW / 32
    int32_t* wpre = (int32_t*)(bits + TC3_ROW / 32);                   // TC3_ROW / 32
    __shared__ int32_t sh[33];
    for (int i = threadIdx.x; i < S; i += T) { slot[i] = 0ull; wsum[i] = 0; }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = T / 32;
    for (int64_t li = blockIdx.x; li < nlist; li += gridDim.x) {
        const int64_t c = list[li];
        const int64_t deg = cdeg[c], o = off[c];
        const int32_t self = (int32_t)c;
        const Walk W = walk_of(g, mem, c);
        const int64_t nwords = (deg + 31) / 32;
        int lgp = 0;
        while ((deg >> lgp) > TC3_KEYS) ++lgp;
        for (int64_t i = threadIdx.x; i < nwords; i += T) bits[i] = 0u;
        __syncthreads();
        for (uint32_t pass = 0; pass < (1u << lgp); ++pass) {
            for (int64_t base = 0; base < deg; base += 4 * T) {
                int32_t cu[4], wt[4];
                if (pass == 0) {
                    // all four gathers in flight before the stores
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int64_t j = base + q * T + threadIdx.x;
                        cu[q] = self; wt[q] = 0;
                        if (j < deg) walk_load(g, cmap, W, j, cu[q], wt[q]);
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int64_t j = base + q * T + threadIdx.x;
                        if (j < deg) { key_at[o + j] = cu[q]; w_at[o + j] = wt[q]; }
                        if (cu[q] != self && pass_of(cu[q], lgp) != pass) cu[q] = self;
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int64_t j = base + q * T + threadIdx.x;
                        cu[q] = j < deg ? __ldcg(&key_at[o + j]) : self;
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int64_t j = base + q * T + threadIdx.x;
                        if (cu[q] != self && pass_of(cu[q], lgp) != pass) cu[q] = self;
                        wt[q] = cu[q] != self ? __ldcg(&w_at[o + j]) : 0;
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (cu[q] == self) continue;
                    const int64_t j = base + q * T + threadIdx.x;
                    const unsigned long long val = ((unsigned long long)((uint32_t)cu[q] + 1u) << 32) | (uint32_t)(deg - j);
                    const uint32_t tag = (uint32_t)cu[q] + 1u;
                    uint32_t h = slot_hash(cu[q], LG);
                    unsigned long long old = atomicCAS(&slot[h], 0ull, val);
                    uint32_t probe = 1;
                    while (old != 0ull && (uint32_t)(old >> 32) != tag && probe < (uint32_t)S) {
                        h = (h + 1) & (S - 1);
                        old = atomicCAS(&slot[h], 0ull, val);
                        ++probe;
                    }
                    if (old != 0ull && (uint32_t)(old >> 32) != tag) { atomicExch(err, 1); continue; }
                    if (old != 0ull && old < val) atomicMax(&slot[h], val);
                    atomicAdd(&wsum[h], wt[q]);
                }
            }
            __syncthreads();
            // the pass's keys: mark first positions, park key and weight there, clear
            for (int i = threadIdx.x; i < S; i += T) {
                const unsigned long long v = slot[i];
                if (!v) continue;
                const int64_t j = deg - (int64_t)(uint32_t)v;
                if (GP_IN(j, deg)) {
                    atomicOr(&bits[j >> 5], 1u << (j & 31));
                    w_at[o + j] = wsum[i];
                }
                slot[i] = 0ull;
                wsum[i] = 0;
            }
            __syncthreads();
        }
        // ranks of the marked positions: contiguous word ranges per thread
        const int64_t per = (nwords + T - 1) / T;
        const int64_t w0 = (int64_t)threadIdx.x * per, w1 = w0 + per < nwords ? w0 + per : nwords;
        int32_t mine = 0;
        for (int64_t wi = w0; wi < w1; ++wi) mine += __popc(bits[wi]);
        int32_t tot;
        int32_t run = block_scan_excl(mine, sh, tot);
        for (int64_t wi = w0; wi < w1; ++wi) { wpre[wi] = run; run += __popc(bits[wi]); }
        __syncthreads();
        const uint32_t lt = (1u << lane) - 1u;
        for (int64_t wi = wid; wi < nwords; wi += nwarp) {
            const uint32_t word = bits[wi];
            if (!((word >> lane) & 1u)) continue;
            const int64_t j = wi * 32 + lane;
            const int32_t r = wpre[wi] + __popc(word & lt);
            if (!GP_IN(r, deg)) continue;
            tci[o + r] = key_at[o + j];
            tew[o + r] = w_at[o + j];
        }
        if (threadIdx.x == 0) cnt[c] = tot;
        __syncthreads();
    }
}

// tier D split over CTAs: rows longer than TC_ROW are cut into pieces of
// TD_PIECE entries, one CTA each, all pieces of a row sharing that row's
// global table.  D1 inserts: a 64-bit slot holds (key + 1) << 32 | (deg - j),
// zero meaning empty; the claiming compare-and-swap stores the first
// position seen, later copies of the key raise it by atomicMax (the largest
// deg - j is the first occurrence), weights add up in a 32-bit array.  D2 ballots the
// first-occurrence flags of each 32-entry word, a device-wide scan of the word
// popcounts ranks the words of every row, D3 writes the first occurrences at
// their ranks.  Same output as one CTA per row: unique neighbours in order of
// first occurrence with summed weights.
constexpr int64_t TD_PIECE = 16384;   // multiple of 32
struct TierD {
    const int32_t* rc;      // coarse row of each tier-D row
    const int32_t* rlg;     // log2 of its table size
    const int64_t* rtab;    // table offset
    const int64_t* rword;   // first word of the row in the word arrays
    const int32_t* prow;    // row of each piece
    const int64_t* pbeg;    // entry range of the piece within the row
    const int64_t* pend;
    unsigned long long* slot;   // tables: (key + 1) << 32 | (deg - first position), 0 = empty
    int32_t* wsum;              // weight sums
    uint32_t* bits;         // first-occurrence flags, one word per 32 entries
    int32_t* wcnt;          // their popcounts
    const int64_t* wpre;    // exclusive prefix of wcnt (+ total)
};

// mapped ids and weights of the tier-D rows in walk layout, one CTA per piece
__global__ void __launch_bounds__(TD_T) k_fill_walk_d(TierD D, DGraph g, const int32_t* __restrict__ cmap,
                                                      const int32_t* __restrict__ mem, const int64_t* __restrict__ off,
                                                      int32_t* __restrict__ mapped, int32_t* __restrict__ mw) {
    const int32_t c = D.rc[D.prow[blockIdx.x]];
    const Walk W = walk_of(g, mem, c);
    const int64_t o = off[c];
    for (int64_t j = D.pbeg[blockIdx.x] + threadIdx.x; j < D.pend[blockIdx.x]; j += TD_T)
        walk_load(g, cmap, W, j, mapped[o + j], mw[o + j]);
}

__device__ __forceinline__ uint32_t td_lookup(const unsigned long long* slot, int32_t cu, int lg) {
    const uint32_t mask = (1u << lg) - 1u;
    const uint32_t tag = (uint32_t)cu + 1u;
    uint32_t h = slot_hash(cu, lg);
    for (uint32_t probe = 0; probe <= mask && (uint32_t)(slot[h] >> 32) != tag; ++probe) h = (h + 1) & mask;
    return h;
}

__global__ void __launch_bounds__(TD_T) k_td_insert(TierD D, const int64_t* __restrict__ off,
                                                    const int64_t* __restrict__ cdeg,
                                                    const int32_t* __restrict__ mapped, const int32_t* __restrict__ mw,
                                                    int32_t* __restrict__ err) {
    const int32_t r = D.prow[blockIdx.x];
    const int32_t self = D.rc[r];
    const int lg = D.rlg[r];
    const uint32_t mask = (1u << lg) - 1u;
    unsigned long long* slot = D.slot + D.rtab[r];
    int32_t* wsum = D.wsum + D.rtab[r];
    const int64_t o = off[self], deg = cdeg[self], end = D.pend[blockIdx.x];
    for (int64_t base = D.pbeg[blockIdx.x]; base < end; base += 4 * TD_T) {
        int32_t cu[4], wt[4];
        unsigned long long val[4], old[4];
        uint32_t h[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int64_t j = base + c * TD_T + threadIdx.x;
            cu[c] = j < end ? __ldcs(&mapped[o + j]) : self;
            wt[c] = j < end ? __ldcs(&mw[o + j]) : 0;
            val[c] = ((unsigned long long)((uint32_t)cu[c] + 1u) << 32) | (uint32_t)(deg - j);
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            h[c] = slot_hash(cu[c], lg);
            old[c] = cu[c] != self ? atomicCAS(&slot[h[c]], 0ull, val[c]) : 0ull;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            if (cu[c] == self) continue;
            const uint32_t tag = (uint32_t)cu[c] + 1u;
            uint32_t probe = 1;
            while (old[c] != 0ull && (uint32_t)(old[c] >> 32) != tag && probe <= mask) {
                h[c] = (h[c] + 1) & mask;
                old[c] = atomicCAS(&slot[h[c]], 0ull, val[c]);
                ++probe;
            }
            if (old[c] != 0ull && (uint32_t)(old[c] >> 32) != tag) { atomicExch(err, 1); continue; }
            // claimed with this position, or the key was there: keep the earliest position
            if (old[c] != 0ull && old[c] < val[c]) atomicMax(&slot[h[c]], val[c]);
            atomicAdd(&wsum[h[c]], wt[c]);
        }
    }
}

__global__ void __launch_bounds__(TD_T) k_td_flags(TierD D, const int64_t* __restrict__ off,
                                                   const int64_t* __restrict__ cdeg,
                                                   const int32_t* __restrict__ mapped) {
    const int32_t r = D.prow[blockIdx.x];
    const int32_t self = D.rc[r];
    const int lg = D.rlg[r];
    const unsigned long long* slot = D.slot + D.rtab[r];
    const int64_t o = off[self], deg = cdeg[self];
    const int lane = threadIdx.x & 31;
    const int64_t w0 = D.pbeg[blockIdx.x] / 32, w1 = (D.pend[blockIdx.x] + 31) / 32;
    for (int64_t wi = w0 + (threadIdx.x >> 5); wi < w1; wi += TD_T / 32) {
        const int64_t j = wi * 32 + lane;
        bool first = false;
        if (j < deg) {
            const int32_t cu = mapped[o + j];
            if (cu != self) first = (uint32_t)slot[td_lookup(slot, cu, lg)] == (uint32_t)(deg - j);
        }
        const uint32_t word = __ballot_sync(0xffffffffu, first);
        if (lane == 0) {
            D.bits[D.rword[r] + wi] = word;
            D.wcnt[D.rword[r] + wi] = __popc(word);
        }
    }
}

__global__ void __launch_bounds__(TD_T) k_td_write(TierD D, const int64_t* __restrict__ off,
                                                   const int64_t* __restrict__ cdeg,
                                                   const int32_t* __restrict__ mapped, int32_t* __restrict__ tci,
                                                   int32_t* __restrict__ tew, int32_t* __restrict__ rowcnt) {
    const int32_t r = D.prow[blockIdx.x];
    const int32_t self = D.rc[r];
    const int lg = D.rlg[r];
    const unsigned long long* slot = D.slot + D.rtab[r];
    const int32_t* wsum = D.wsum + D.rtab[r];
    const int64_t o = off[self], deg = cdeg[self];
    const int64_t rw = D.rword[r], nwords = (deg + 31) / 32;
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const int64_t w0 = D.pbeg[blockIdx.x] / 32, w1 = (D.pend[blockIdx.x] + 31) / 32;
    for (int64_t wi = w0 + (threadIdx.x >> 5); wi < w1; wi += TD_T / 32) {
        const uint32_t word = D.bits[rw + wi];
        if (!((word >> lane) & 1u)) continue;
        const int32_t cu = mapped[o + wi * 32 + lane];
        const int64_t rank = D.wpre[rw + wi] - D.wpre[rw] + __popc(word & lt);
        if (!GP_IN(rank, deg)) continue;
        tci[o + rank] = cu;
        tew[o + rank] = wsum[td_lookup(slot, cu, lg)];
    }
    if (D.pbeg[blockIdx.x] == 0 && threadIdx.x == 0) rowcnt[self] = (int32_t)(D.wpre[rw + nwords] - D.wpre[rw]);
}

__global__ void k_td_rows(const int32_t* __restrict__ list, int64_t n, const int64_t* __restrict__ cdeg,
                          int64_t* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = cdeg[list[i]];
}

// warp per coarse row: temporary (walk-bound offsets) -> final CSR
// Packs every row's deduplicated entries (crp[c + 1] - crp[c] of them at
// walk offset off[c] of tci / tew) into the coarse CSR.  The output is cut
// into slices of `slice` entries (csr_slice), one warp each: the warp finds the row
// holding its first entry by binary search over crp, then keeps a window of
// 32 consecutive rows (start and source offset, one row per lane); the row of
// an output position is the last window row starting at or before it (five
// shuffle steps).  Eight groups of 32 entries are loaded before any is stored.
__device__ __forceinline__ int64_t cp_source(int64_t oi, int64_t s, int64_t src) {
    const int l = csr_window_lane(s, oi);
    return __shfl_sync(0xffffffffu, src, l) + (oi - __shfl_sync(0xffffffffu, s, l));
}
__global__ void __launch_bounds__(256) k_contract_copy(int64_t nc, int64_t cm, int64_t slice,
                                                       const int64_t* __restrict__ off,
                                                       const int64_t* __restrict__ crp, const int32_t* __restrict__ tci,
                                                       const int32_t* __restrict__ tew, int32_t* __restrict__ ci,
                                                       int32_t* __restrict__ ew) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t nslice = (cm + slice - 1) / slice;
    for (int64_t sl = wid; sl < nslice; sl += nw) {
        const int64_t o0 = sl * slice, o1 = o0 + slice < cm ? o0 + slice : cm;
        int64_t cb = csr_row_of(crp, nc, o0), s = 0, src = 0, wend = 0;
        auto window = [&]() {   // rows cb .. cb + 31; wend = first output entry past them
            const int64_t r = cb + lane;
            s = r < nc ? crp[r] : cm;
            src = r < nc ? off[r] : 0;
            wend = crp[cb + 32 < nc ? cb + 32 : nc];
        };
        window();
        int64_t o = o0;
        while (o < o1) {
            const int64_t lim = o1 < wend ? o1 : wend;
            if (o + 256 <= lim) {
                int32_t a[8], b[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int64_t p = cp_source(o + 32 * q + lane, s, src);
                    a[q] = __ldcs(&tci[p]);
                    b[q] = __ldcs(&tew[p]);
                }
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    ci[o + 32 * q + lane] = a[q];
                    ew[o + 32 * q + lane] = b[q];
                }
                o += 256;
            } else if (o < lim) {
                const int64_t oi = o + lane;
                const int64_t p = cp_source(oi, s, src);
                if (oi < lim) { ci[oi] = tci[p]; ew[oi] = tew[p]; }
                o = o + 32 < lim ? o + 32 : lim;
            } else {
                cb += 32;   // o >= wend: o lies in a later row
                window();
            }
        }
    }
}

void contract_level(Ctx& c, Level& fine, Level& coarse, const int32_t* match) {
    const DGraph& g = fine.g;
    auto mk = c.tmp->save();
    int32_t* flag = c.tmp_alloc<int32_t>(g.n);
    int64_t* cid = c.tmp_alloc<int64_t>(g.n);
    int64_t* d_tot = c.tmp_alloc<int64_t>(4);
    k_rep_flags<<<grid_for(g.n, 256), 256, 0, c.s>>>(g.n, match, flag);
    GP_LAUNCHED(c);
    scan_excl_i32_to_i64(c, flag, cid, g.n, d_tot);
    const int64_t nc = read_i64(c, d_tot);
    fine.cmap = c.keep_alloc<int32_t>(g.n);
    int32_t* mem = c.tmp_alloc<int32_t>(2 * nc);
    int32_t* cvw = c.keep_alloc<int32_t>(nc);
    int64_t* cdeg = c.tmp_alloc<int64_t>(nc);
    k_cmap<<<grid_for(g.n, 256), 256, 0, c.s>>>(g, match, cid, fine.cmap, mem, cvw, cdeg);
    GP_LAUNCHED(c);
    int64_t* off = c.tmp_alloc<int64_t>(nc + 1);
    scan_excl_i64(c, cdeg, off, nc, off + nc);
    const int64_t T = g.m;
    int32_t* mapped = c.tmp_alloc<int32_t>(T);
    int32_t* mw = c.tmp_alloc<int32_t>(T);
    int32_t* tci = c.tmp_alloc<int32_t>(T);
    int32_t* tew = c.tmp_alloc<int32_t>(T);
    int32_t* rowcnt = c.tmp_alloc<int32_t>(nc);
    int32_t* listC1 = c.tmp_alloc<int32_t>(nc);
    int32_t* listC = c.tmp_alloc<int32_t>(nc);
    int32_t* listC2 = c.tmp_alloc<int32_t>(nc);
    int32_t* listC3 = c.tmp_alloc<int32_t>(nc);
    int32_t* listD = c.tmp_alloc<int32_t>(nc);
    int64_t* lcount = c.tmp_alloc<int64_t>(6);
    int32_t* err = c.tmp_alloc<int32_t>(1);
    memset_async(c, lcount, 0, 6 * sizeof(int64_t));
    memset_async(c, err, 0, sizeof(int32_t));
    {
        constexpr size_t smA = 8 * warp_dedup_smem<TA_ROW, TA_SLOTS, int32_t>();
        constexpr size_t smA2 = 8 * warp_dedup_smem<TA2_ROW, TA2_SLOTS, int16_t>();
        constexpr size_t smB = TB_WARPS * warp_dedup_smem<TB_ROW, TB_SLOTS, int16_t>();
        auto kA = k_dedup_warp<TA_ROW, TA_SLOTS, 8, int32_t>;
        auto kA2 = k_dedup_warp<TA2_ROW, TA2_SLOTS, 8, int16_t>;
        auto kB = k_dedup_warp<TB_ROW, TB_SLOTS, TB_WARPS, int16_t>;
        kA<<<grid_for(nc * 32, 256, c.sm_count * c.ctas_per_sm), 256, smA, c.s>>>(g, fine.cmap, mem, nc, 0, off, cdeg,
                                                                                  tci, tew, rowcnt);
        GP_LAUNCHED(c);
        kA2<<<grid_for(nc * 32, 256, c.sm_count * c.ctas_per_sm), 256, smA2, c.s>>>(g, fine.cmap, mem, nc, TA_ROW + 1,
                                                                                    off, cdeg, tci, tew, rowcnt);
        GP_LAUNCHED(c);
        kB<<<grid_for(nc * 32, TB_WARPS * 32, c.sm_count * c.ctas_per_sm), TB_WARPS * 32, smB, c.s>>>(
            g, fine.cmap, mem, nc, TA2_ROW + 1, off, cdeg, tci, tew, rowcnt);
        GP_LAUNCHED(c);
    }
    k_long_rows<<<grid_for(nc, 256), 256, 0, c.s>>>(nc, cdeg, listC1, listC, listC2, listC3, listD, lcount);
    GP_LAUNCHED(c);
    GP_CUDA(cudaMemcpyAsync(c.h_pinned, lcount, 6 * sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
    c.sync();
    const int64_t nC = c.h_pinned[0], nD = c.h_pinned[1], maxD = c.h_pinned[2], nC2 = c.h_pinned[3];
    const int64_t nC3 = c.h_pinned[4], nC1 = c.h_pinned[5];
    if (nC1 > 0) {
        k_dedup_cta_smem<TC1_T, TC1_SLOTS, TC1_ROW>
            <<<(unsigned)std::min<int64_t>(nC1, (int64_t)c.sm_count * c.ctas_per_sm), TC1_T,
               cta_dedup_smem<TC1_SLOTS, TC1_ROW>(), c.s>>>(g, fine.cmap, mem, listC1, nC1, off, cdeg, tci, tew, rowcnt,
                                                            err);
        GP_LAUNCHED(c);
    }
    if (nC > 0) {
        // one CTA per row: the block scheduler balances rows of unequal length
        k_dedup_cta_smem<TC_T, TC_SLOTS, TC_ROW>
            <<<(unsigned)std::min<int64_t>(nC, (int64_t)c.sm_count * c.ctas_per_sm), TC_T,
               cta_dedup_smem<TC_SLOTS, TC_ROW>(), c.s>>>(g, fine.cmap, mem, listC, nC, off, cdeg, tci, tew, rowcnt,
                                                          err);
        GP_LAUNCHED(c);
    }
    if (nC2 > c.sm_count) listC2 = longest_first(c, listC2, nC2, cdeg, TC2_ROW);
    if (nC3 > c.sm_count) listC3 = longest_first(c, listC3, nC3, cdeg, TC3_ROW);
    if (nC2 > 0) {
        k_dedup_cta_smem<TC2_T, TC2_SLOTS, TC2_ROW>
            <<<(unsigned)std::min<int64_t>(nC2, (int64_t)c.sm_count * c.ctas_per_sm), TC2_T,
               cta_dedup_smem<TC2_SLOTS, TC2_ROW>(), c.s>>>(g, fine.cmap, mem, listC2, nC2, off, cdeg, tci, tew, rowcnt,
                                                            err);
        GP_LAUNCHED(c);
    }
    if (nC3 > 0) {
        // key and weight of each first occurrence are parked at its walk position
        // in mapped / mw (free at these rows: only tier-D rows use them otherwise)
        k_dedup_multipass<<<(unsigned)std::min<int64_t>(nC3, (int64_t)c.sm_count * c.ctas_per_sm), TC2_T, tc3_smem(),
                            c.s>>>(g, fine.cmap, mem, listC3, nC3, off, cdeg, mapped, mw, tci, tew, rowcnt, err);
        GP_LAUNCHED(c);
    }
    if (nD > 0) {
        (void)maxD;
        // row lengths to the host: tables, word ranges and pieces
        int64_t* d_deg = c.tmp_alloc<int64_t>(nD);
        k_td_rows<<<grid_for(nD, 256), 256, 0, c.s>>>(listD, nD, cdeg, d_deg);
        GP_LAUNCHED(c);
        std::vector<int64_t> hdeg((size_t)nD);
        std::vector<int32_t> hlist((size_t)nD);
        GP_CUDA(cudaMemcpyAsync(hdeg.data(), d_deg, sizeof(int64_t) * nD, cudaMemcpyDeviceToHost, c.s));
        GP_CUDA(cudaMemcpyAsync(hlist.data(), listD, sizeof(int32_t) * nD, cudaMemcpyDeviceToHost, c.s));
        c.sync();
        std::vector<int32_t> rlg((size_t)nD), prow;
        std::vector<int64_t> rtab((size_t)nD), rword((size_t)nD), pbeg, pend;
        int64_t tab = 0, words = 0;
        for (int64_t r = 0; r < nD; ++r) {
            int64_t S = 2;
            int lg = 1;
            while (S < 2 * hdeg[r]) { S <<= 1; ++lg; }
            rlg[r] = lg; rtab[r] = tab; rword[r] = words;
            tab += S;
            words += (hdeg[r] + 31) / 32;
            for (int64_t b = 0; b < hdeg[r]; b += TD_PIECE) {
                prow.push_back((int32_t)r);
                pbeg.push_back(b);
                pend.push_back(std::min<int64_t>(b + TD_PIECE, hdeg[r]));
            }
        }
        const int64_t np = (int64_t)prow.size();
        TierD D;
        int32_t* d_rc = c.tmp_alloc<int32_t>(nD);
        int32_t* d_rlg = c.tmp_alloc<int32_t>(nD);
        int64_t* d_rtab = c.tmp_alloc<int64_t>(nD);
        int64_t* d_rword = c.tmp_alloc<int64_t>(nD);
        int32_t* d_prow = c.tmp_alloc<int32_t>(np);
        int64_t* d_pbeg = c.tmp_alloc<int64_t>(np);
        int64_t* d_pend = c.tmp_alloc<int64_t>(np);
        GP_CUDA(cudaMemcpyAsync(d_rc, hlist.data(), sizeof(int32_t) * nD, cudaMemcpyHostToDevice, c.s));
        GP_CUDA(cudaMemcpyAsync(d_rlg, rlg.data(), sizeof(int32_t) * nD, cudaMemcpyHostToDevice, c.s));
        GP_CUDA(cudaMemcpyAsync(d_rtab, rtab.data(), sizeof(int64_t) * nD, cudaMemcpyHostToDevice, c.s));
        GP_CUDA(cudaMemcpyAsync(d_rword, rword.data(), sizeof(int64_t) * nD, cudaMemcpyHostToDevice, c.s));
        GP_CUDA(cudaMemcpyAsync(d_prow, prow.data(), sizeof(int32_t) * np, cudaMemcpyHostToDevice, c.s));
        GP_CUDA(cudaMemcpyAsync(d_pbeg, pbeg.data(), sizeof(int64_t) * np, cudaMemcpyHostToDevice, c.s));
        GP_CUDA(cudaMemcpyAsync(d_pend, pend.data(), sizeof(int64_t) * np, cudaMemcpyHostToDevice, c.s));
        D.rc = d_rc; D.rlg = d_rlg; D.rtab = d_rtab; D.rword = d_rword;
        D.prow = d_prow; D.pbeg = d_pbeg; D.pend = d_pend;
        D.slot = c.tmp_alloc<unsigned long long>(tab);
        D.wsum = c.tmp_alloc<int32_t>(tab);
        D.bits = (uint32_t*)c.tmp_alloc<int32_t>(words);
        D.wcnt = c.tmp_alloc<int32_t>(words);
        int64_t* wpre = c.tmp_alloc<int64_t>(words + 1);
        D.wpre = wpre;
        GP_CUDA(cudaMemsetAsync(D.slot, 0, sizeof(unsigned long long) * tab, c.s));
        GP_CUDA(cudaMemsetAsync(D.wsum, 0, sizeof(int32_t) * tab, c.s));
        k_fill_walk_d<<<(unsigned)np, TD_T, 0, c.s>>>(D, g, fine.cmap, mem, off, mapped, mw);
        GP_LAUNCHED(c);
        k_td_insert<<<(unsigned)np, TD_T, 0, c.s>>>(D, off, cdeg, mapped, mw, err);
        GP_LAUNCHED(c);
        k_td_flags<<<(unsigned)np, TD_T, 0, c.s>>>(D, off, cdeg, mapped);
        GP_LAUNCHED(c);
        scan_excl_i32_to_i64(c, D.wcnt, wpre, words, wpre + words);
        k_td_write<<<(unsigned)np, TD_T, 0, c.s>>>(D, off, cdeg, mapped, tci, tew, rowcnt);
        GP_LAUNCHED(c);
    }
    int64_t* crp = c.keep_alloc<int64_t>(nc + 1);
    scan_excl_i32_to_i64(c, rowcnt, crp, nc, crp + nc);
    GP_CUDA(cudaMemcpyAsync(c.h_pinned, crp + nc, sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
    GP_CUDA(cudaMemcpyAsync(c.h_pinned + 1, err, sizeof(int32_t), cudaMemcpyDeviceToHost, c.s));
    c.sync();
    const int64_t mc = c.h_pinned[0];
    if ((int32_t)c.h_pinned[1] != 0) throw GpError(GP_EINTERNAL, "contraction hash table overflow");
    int32_t* cci = c.keep_alloc<int32_t>(mc);
    int32_t* cew = c.keep_alloc<int32_t>(mc);
    const int64_t cslice = csr_slice(mc, c.sm_count);
    k_contract_copy<<<grid_for((mc + cslice - 1) / cslice * 32, 256, c.sm_count * c.ctas_per_sm), 256, 0, c.s>>>(
        nc, mc, cslice, off, crp, tci, tew, cci, cew);
    GP_LAUNCHED(c);
    // rows read twice (count and rank for long rows), cmap gathered per entry,
    // unique entries written to the temporary and copied once
    c.bytes += 2 * (8 * (g.n + 1) + 8 * g.m) + 4 * g.m + 8 * (nc + 1) + 4 * nc + 24 * mc + 24 * nc;
    coarse.g.n = nc;
    coarse.g.m = mc;
    coarse.g.rp = crp;
    coarse.g.ci = cci;
    coarse.g.ew = cew;
    coarse.g.vw = cvw;
    c.tmp->restore(mk);
}

// shared-memory caps of the contraction kernels above 48 KB; set once per
// device (the cap is per kernel and shared by every thread of the process)
void coarsen_smem_caps() {
    constexpr size_t smA = 8 * warp_dedup_smem<TA_ROW, TA_SLOTS, int32_t>();
    constexpr size_t smA2 = 8 * warp_dedup_smem<TA2_ROW, TA2_SLOTS, int16_t>();
    constexpr size_t smB = TB_WARPS * warp_dedup_smem<TB_ROW, TB_SLOTS, int16_t>();
    GP_CUDA(cudaFuncSetAttribute(k_dedup_warp<TA_ROW, TA_SLOTS, 8, int32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smA));
    GP_CUDA(cudaFuncSetAttribute(k_dedup_warp<TA2_ROW, TA2_SLOTS, 8, int16_t>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smA2));
    GP_CUDA(cudaFuncSetAttribute(k_dedup_warp<TB_ROW, TB_SLOTS, TB_WARPS, int16_t>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smB));
    GP_CUDA(cudaFuncSetAttribute(k_dedup_cta_smem<TC1_T, TC1_SLOTS, TC1_ROW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cta_dedup_smem<TC1_SLOTS, TC1_ROW>()));
    GP_CUDA(cudaFuncSetAttribute(k_dedup_cta_smem<TC_T, TC_SLOTS, TC_ROW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cta_dedup_smem<TC_SLOTS, TC_ROW>()));
    GP_CUDA(cudaFuncSetAttribute(k_dedup_cta_smem<TC2_T, TC2_SLOTS, TC2_ROW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cta_dedup_smem<TC2_SLOTS, TC2_ROW>()));
    GP_CUDA(cudaFuncSetAttribute(k_dedup_multipass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc3_smem()));
}

}  // namespace gp
