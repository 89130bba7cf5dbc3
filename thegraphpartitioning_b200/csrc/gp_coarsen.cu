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
#include "gp_internal.cuh"

namespace gp {

// ---------------------------------------------------------------- heavy list
__global__ void k_heavy_list(const int64_t* __restrict__ rp, int64_t n, int32_t* __restrict__ list,
                             int64_t* __restrict__ count) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        if (rp[v + 1] - rp[v] > kHeavyDeg) {
            unsigned long long slot = atomicAdd((unsigned long long*)count, 1ull);
            list[slot] = (int32_t)v;
        }
    }
}

void build_heavy(Ctx& c, Level& L) {
    int64_t* d_cnt = c.tmp_alloc<int64_t>(1);
    memset_async(c, d_cnt, 0, sizeof(int64_t));
    L.heavy = c.keep_alloc<int32_t>(std::max<int64_t>(1, L.g.m / kHeavyDeg + 1));
    k_heavy_list<<<grid_for(L.g.n, 256), 256, 0, c.s>>>(L.g.rp, L.g.n, L.heavy, d_cnt);
    GP_LAUNCHED(c);
    c.bytes += 8 * (L.g.n + 1);
    L.nheavy = read_i64(c, d_cnt);
}

// ---------------------------------------------------------------- argmax helpers
// Larger key wins; equal keys: smaller id wins (ids compared unsigned so that
// -1, meaning "none", loses every tie).
__device__ __forceinline__ void argmax_merge(uint64_t& k, int32_t& id, uint64_t k2, int32_t i2) {
    if (k2 > k || (k2 == k && (uint32_t)i2 < (uint32_t)id)) { k = k2; id = i2; }
}
__device__ __forceinline__ void warp_argmax(uint64_t& k, int32_t& id) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        uint64_t k2 = __shfl_xor_sync(0xffffffffu, k, o);
        int32_t i2 = __shfl_xor_sync(0xffffffffu, id, o);
        argmax_merge(k, id, k2, i2);
    }
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
template <int MODE>
__device__ __forceinline__ void scan_best(const DGraph& g, int64_t v, int64_t beg, int64_t end, int64_t stride,
                                          int64_t start, const int32_t* __restrict__ match,
                                          uint64_t salt, int64_t maxvw, uint64_t& bk, int32_t& bid) {
    const int64_t vwv = g.vw ? g.vw[v] : 1;
    for (int64_t e = beg + start; e < end; e += stride) {
        const int32_t u = g.ci[e];
        if (u == v) continue;
        if (MODE == 0) {
            if (match[u] != -1) continue;
            if (vwv + (g.vw ? g.vw[u] : 1) > maxvw) continue;
        }
        const int32_t w = g.ew ? g.ew[e] : 1;
        argmax_merge(bk, bid, edge_key(w, edge_hash(salt, (int32_t)v, u)), u);
    }
}

// Light rows: one warp per entry of the worklist `wl` (nullptr: every vertex,
// wl_n = n); rows longer than kHeavyDeg are skipped there and handled by the
// first nheavy CTAs, one row each.
template <int MODE>
__global__ void __launch_bounds__(256) k_match_scan(DGraph g, const int32_t* __restrict__ heavy, int64_t nheavy,
                                                    const int32_t* __restrict__ wl, int64_t wl_n,
                                                    const int32_t* __restrict__ match, int32_t* __restrict__ out,
                                                    uint64_t salt, int64_t maxvw,
                                                    uint64_t* __restrict__ list_keys, int64_t* __restrict__ list_cnt,
                                                    int nbits) {
    __shared__ uint64_t sk[32];
    __shared__ int32_t sid[32];
    auto emit = [&](int64_t v, int32_t best) {
        if (MODE == 0) {
            out[v] = best;
        } else if (best >= 0) {
            unsigned long long slot = atomicAdd((unsigned long long*)list_cnt, 1ull);
            list_keys[slot] = ((uint64_t)(uint32_t)best << nbits) | (uint64_t)v;
        }
    };
    if ((int64_t)blockIdx.x < nheavy) {
        const int64_t v = heavy[blockIdx.x];
        if (match[v] != -1) { if (MODE == 0 && threadIdx.x == 0) out[v] = -1; return; }
        uint64_t bk = 0; int32_t bid = -1;
        scan_best<MODE>(g, v, g.rp[v], g.rp[v + 1], blockDim.x, threadIdx.x, match, salt, maxvw, bk, bid);
        block_argmax(bk, bid, sk, sid);
        if (threadIdx.x == 0) emit(v, bid);
        return;
    }
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)(blockIdx.x - nheavy) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)(gridDim.x - nheavy) * blockDim.x) >> 5;
    for (int64_t i = wid; i < wl_n; i += nw) {
        const int64_t v = wl ? wl[i] : i;
        const int64_t beg = g.rp[v], end = g.rp[v + 1];
        if (end - beg > kHeavyDeg) continue;
        if (match[v] != -1) { if (MODE == 0 && lane == 0) out[v] = -1; continue; }
        if (MODE == 1 && end == beg) continue;
        uint64_t bk = 0; int32_t bid = -1;
        scan_best<MODE>(g, v, beg, end, 32, lane, match, salt, maxvw, bk, bid);
        warp_argmax(bk, bid);
        if (lane == 0) emit(v, bid);
    }
}

// Mutual proposals become pairs; vertices left unmatched are appended to the
// next round's worklist (any order: each vertex's proposal is its own).
__global__ void k_handshake(const int32_t* __restrict__ wl, int64_t wl_n, const int32_t* __restrict__ prop,
                            int32_t* __restrict__ match, int64_t* __restrict__ pairs,
                            int32_t* __restrict__ next_wl, int64_t* __restrict__ next_n) {
    int64_t local = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < wl_n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = wl ? wl[i] : i;
        if (match[v] != -1) continue;
        const int32_t u = prop[v];
        if (u >= 0 && prop[u] == (int32_t)v) {
            match[v] = u;
            if (v < u) ++local;
        } else {
            unsigned long long slot = atomicAdd((unsigned long long*)next_n, 1ull);
            next_wl[slot] = (int32_t)v;
        }
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd((unsigned long long*)pairs, (unsigned long long)local);
}

// sorted (anchor << nbits | v) keys: pair ranks (0,1), (2,3), ... of each anchor group
__global__ void k_twohop_pair(const uint64_t* __restrict__ keys, int64_t cnt, int nbits, const int32_t* __restrict__ vw,
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

int64_t match_level(Ctx& c, const Level& L, int level, const Params& P, int32_t* match, int* rounds_out) {
    const DGraph& g = L.g;
    const uint64_t salt = level_salt(P.seed, level);
    auto mk = c.tmp->save();
    int32_t* prop = c.tmp_alloc<int32_t>(g.n);
    int32_t* wl[2] = {c.tmp_alloc<int32_t>(g.n), c.tmp_alloc<int32_t>(g.n)};
    int64_t* d_pairs = c.tmp_alloc<int64_t>(4);
    GP_CUDA(cudaMemsetAsync(match, 0xff, sizeof(int32_t) * g.n, c.s));
    const int light_blocks = grid_for(g.n * 32, 256, c.sm_count * 8);
    const int grid = (int)L.nheavy + light_blocks;
    int64_t pairs = 0;
    int rounds = 0;
    const int32_t* cur = nullptr;   // round 0: every vertex
    int64_t cur_n = g.n;
    for (int r = 0; r < P.o.match_rounds && cur_n > 0; ++r) {
        int32_t* next = wl[r & 1];
        memset_async(c, d_pairs, 0, 2 * sizeof(int64_t));
        k_match_scan<0><<<grid, 256, 0, c.s>>>(g, L.heavy, L.nheavy, cur, cur_n, match, prop, salt, P.maxvw,
                                               nullptr, nullptr, 0);
        GP_LAUNCHED(c);
        k_handshake<<<grid_for(cur_n, 256), 256, 0, c.s>>>(cur, cur_n, prop, match, d_pairs, next, d_pairs + 1);
        GP_LAUNCHED(c);
        c.bytes += (L.scan_bytes() + 4 * g.m) * cur_n / std::max<int64_t>(g.n, 1) + 16 * cur_n;
        GP_CUDA(cudaMemcpyAsync(c.h_pinned, d_pairs, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
        c.sync();
        const int64_t newp = c.h_pinned[0];
        rounds = r + 1;
        pairs += newp;
        cur = next;
        cur_n = c.h_pinned[1];
        if (newp == 0) break;
    }
    if (P.o.two_hop > 0 && 4 * (g.n - pairs) > 3 * g.n) {
        const int nb = bits_for(g.n);
        uint64_t* keys = c.tmp_alloc<uint64_t>(g.n);
        uint64_t* keys2 = c.tmp_alloc<uint64_t>(g.n);
        int32_t* vals = c.tmp_alloc<int32_t>(g.n);
        int32_t* vals2 = c.tmp_alloc<int32_t>(g.n);
        memset_async(c, d_pairs, 0, 2 * sizeof(int64_t));
        k_match_scan<1><<<grid, 256, 0, c.s>>>(g, L.heavy, L.nheavy, nullptr, g.n, match, nullptr, salt, P.maxvw,
                                               keys, d_pairs + 1, nb);
        GP_LAUNCHED(c);
        c.bytes += L.scan_bytes() + 4 * g.n;
        int64_t cnt = read_i64(c, d_pairs + 1);
        if (cnt > 1) {
            GP_CUDA(cudaMemsetAsync(vals, 0, sizeof(int32_t) * cnt, c.s));
            radix_sort_pairs(c, keys, vals, keys2, vals2, cnt, 2 * nb);
            k_twohop_pair<<<grid_for(cnt, 256), 256, 0, c.s>>>(keys, cnt, nb, g.vw, P.maxvw, match, d_pairs);
            GP_LAUNCHED(c);
            c.bytes += 24 * cnt;
            pairs += read_i64(c, d_pairs);
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
constexpr int SMALL_ROW = 128;          // rows up to this length: one warp, 256-slot table on chip
constexpr int SMALL_SLOTS = 256;
constexpr int MID_ROW = 8192;           // rows up to this length: one warp, private table in global memory
constexpr int MID_SLOTS = 2 * MID_ROW;
constexpr int BIG_T = 1024;             // longer rows: one CTA each, two-phase
constexpr int32_t EMPTY_KEY = -1;

__device__ __forceinline__ uint32_t slot_hash(int32_t key, int lg) {
    return ((uint32_t)key * 0x9E3779B1u) >> (32 - lg);
}

__device__ __forceinline__ void row_entry(const DGraph& g, int32_t a, int32_t b, int64_t da, int64_t j,
                                          const int32_t* __restrict__ cmap, int32_t& cu, int32_t& w) {
    const int64_t e = j < da ? g.rp[a] + j : g.rp[b] + (j - da);
    cu = cmap[g.ci[e]];
    w = g.ew ? g.ew[e] : 1;
}

// one warp per coarse row with at most SMALL_ROW entries; table in shared memory
__global__ void __launch_bounds__(256) k_contract_small(DGraph g, int64_t nc, const int32_t* __restrict__ mem,
                                                        const int32_t* __restrict__ cmap, const int64_t* __restrict__ off,
                                                        const int64_t* __restrict__ cdeg, int32_t* __restrict__ tci,
                                                        int32_t* __restrict__ tew, int32_t* __restrict__ cnt) {
    __shared__ int32_t s_key[8][SMALL_SLOTS];
    __shared__ int32_t s_idx[8][SMALL_SLOTS];
    __shared__ int32_t s_okey[8][SMALL_ROW];
    __shared__ int32_t s_w[8][SMALL_ROW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t* key = s_key[w];
    int32_t* tidx = s_idx[w];
    int32_t* okey = s_okey[w];
    int32_t* wacc = s_w[w];
    for (int i = lane; i < SMALL_SLOTS; i += 32) key[i] = EMPTY_KEY;
    for (int i = lane; i < SMALL_ROW; i += 32) wacc[i] = 0;
    __syncwarp();
    const uint32_t lt = (1u << lane) - 1u;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = wid; c < nc; c += nw) {
        const int64_t deg = cdeg[c];
        if (deg > SMALL_ROW) continue;
        const int32_t a = mem[2 * c], b = mem[2 * c + 1];
        const int64_t da = g.rp[a + 1] - g.rp[a];
        int32_t count = 0;
        for (int64_t base = 0; base < deg; base += 32) {
            const int64_t j = base + lane;
            int32_t cu = -1, wt = 0;
            if (j < deg) row_entry(g, a, b, da, j, cmap, cu, wt);
            const bool act = (j < deg) && cu != (int32_t)c;
            const uint32_t peers = __match_any_sync(0xffffffffu, act ? (uint32_t)cu : (0x80000000u | (uint32_t)lane));
            const int leader = __ffs(peers) - 1;
            bool isnew = false;
            int32_t h = -1;
            if (act && lane == leader) {
                h = (int32_t)slot_hash(cu, 8);
                for (int probe = 0; probe < SMALL_SLOTS; ++probe) {
                    const int32_t old = atomicCAS(&key[h], EMPTY_KEY, cu);
                    if (old == EMPTY_KEY) { isnew = true; break; }
                    if (old == cu) break;
                    h = (h + 1) & (SMALL_SLOTS - 1);
                }
            }
            const uint32_t newmask = __ballot_sync(0xffffffffu, isnew);
            int32_t idx = -1;
            if (isnew) {
                idx = count + __popc(newmask & lt);
                tidx[h] = idx;
                okey[idx] = cu;
            }
            __syncwarp();
            if (act && lane == leader && !isnew) idx = tidx[h];
            idx = __shfl_sync(0xffffffffu, idx, leader);
            if (act) atomicAdd(&wacc[idx], wt);
            count += __popc(newmask);
            __syncwarp();
        }
        const int64_t o = off[c];
        for (int i = lane; i < count; i += 32) {
            tci[o + i] = okey[i];
            tew[o + i] = wacc[i];
            wacc[i] = 0;
        }
        for (int i = lane; i < SMALL_SLOTS; i += 32) key[i] = EMPTY_KEY;
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

// rows of SMALL_ROW < d <= MID_ROW go to list1, longer ones to list2 (with
// the size of their global table); list order is irrelevant (rows are independent)
__global__ void k_big_rows(int64_t nc, const int64_t* __restrict__ cdeg, int32_t* __restrict__ list1,
                           int32_t* __restrict__ list2, int64_t* __restrict__ tsize, int64_t* __restrict__ count) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = cdeg[c];
        if (d <= SMALL_ROW) continue;
        if (d <= MID_ROW) {
            unsigned long long slot = atomicAdd((unsigned long long*)&count[0], 1ull);
            list1[slot] = (int32_t)c;
        } else {
            unsigned long long slot = atomicAdd((unsigned long long*)&count[1], 1ull);
            list2[slot] = (int32_t)c;
            int64_t S = 1;
            while (S < 2 * d) S <<= 1;
            tsize[slot] = S;
        }
    }
}

// one warp per row of list1, chunks of 32 entries in row order; the table
// (key, output rank) lives in the warp's private global region (L2 resident),
// output entries and weights go straight to the temporary row.
__global__ void __launch_bounds__(256) k_contract_mid(DGraph g, const int32_t* __restrict__ list, int64_t nlist,
                                                      const int32_t* __restrict__ mem, const int32_t* __restrict__ cmap,
                                                      const int64_t* __restrict__ off, const int64_t* __restrict__ cdeg,
                                                      int32_t* __restrict__ wtab, int32_t* __restrict__ tci,
                                                      int32_t* __restrict__ tew, int32_t* __restrict__ cnt,
                                                      int32_t* __restrict__ err) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    int32_t* key = wtab + wid * (2 * (int64_t)MID_SLOTS);
    int32_t* tidx = key + MID_SLOTS;
    const uint32_t lt = (1u << lane) - 1u;
    for (int64_t li = wid; li < nlist; li += nw) {
        const int64_t c = list[li];
        const int64_t deg = cdeg[c];
        int S = 1, lg = 0;
        while (S < 2 * deg) { S <<= 1; ++lg; }
        for (int i = lane; i < S; i += 32) key[i] = EMPTY_KEY;
        __syncwarp();
        const int32_t a = mem[2 * c], b = mem[2 * c + 1];
        const int64_t da = g.rp[a + 1] - g.rp[a];
        const int64_t o = off[c];
        int32_t count = 0;
        for (int64_t base = 0; base < deg; base += 32) {
            const int64_t j = base + lane;
            int32_t cu = -1, wt = 0;
            if (j < deg) row_entry(g, a, b, da, j, cmap, cu, wt);
            const bool act = (j < deg) && cu != (int32_t)c;
            const uint32_t peers = __match_any_sync(0xffffffffu, act ? (uint32_t)cu : (0x80000000u | (uint32_t)lane));
            const int leader = __ffs(peers) - 1;
            bool isnew = false;
            int32_t h = -1;
            if (act && lane == leader) {
                h = (int32_t)slot_hash(cu, lg);
                bool placed = false;
                for (int probe = 0; probe < S; ++probe) {
                    const int32_t old = atomicCAS(&key[h], EMPTY_KEY, cu);
                    if (old == EMPTY_KEY) { isnew = true; placed = true; break; }
                    if (old == cu) { placed = true; break; }
                    h = (h + 1) & (S - 1);
                }
                if (!placed) atomicExch(err, 1);
            }
            const uint32_t newmask = __ballot_sync(0xffffffffu, isnew);
            int32_t idx = -1;
            if (isnew) {
                idx = count + __popc(newmask & lt);
                tidx[h] = idx;
                tci[o + idx] = cu;
                tew[o + idx] = 0;
            }
            __syncwarp();
            if (act && lane == leader && !isnew && h >= 0) idx = tidx[h];
            idx = __shfl_sync(0xffffffffu, idx, leader);
            if (act && idx >= 0) atomicAdd(&tew[o + idx], wt);
            count += __popc(newmask);
            __syncwarp();
        }
        if (lane == 0) cnt[c] = count;
        __syncwarp();
    }
}

// one CTA per row of list2 (hubs): table in the global region toff; phase 1
// inserts (first position by atomicMin, weights by atomicAdd), phase 2 ranks
// first positions with a block scan in row order.
__global__ void __launch_bounds__(BIG_T) k_contract_big(DGraph g, const int32_t* __restrict__ list, int64_t nbig,
                                                        const int32_t* __restrict__ mem, const int32_t* __restrict__ cmap,
                                                        const int64_t* __restrict__ off, const int64_t* __restrict__ cdeg,
                                                        const int64_t* __restrict__ toff, int32_t* __restrict__ gtab,
                                                        int32_t* __restrict__ tci, int32_t* __restrict__ tew,
                                                        int32_t* __restrict__ cnt, int32_t* __restrict__ err) {
    __shared__ int32_t sh[33];
    for (int64_t li = blockIdx.x; li < nbig; li += gridDim.x) {
        const int64_t c = list[li];
        const int64_t deg = cdeg[c];
        int64_t S = 1;
        int lg = 0;
        while (S < 2 * deg) { S <<= 1; ++lg; }
        int32_t* keys = gtab + 3 * toff[li];
        int32_t* minpos = keys + S;
        int32_t* wsum = minpos + S;
        for (int64_t i = threadIdx.x; i < S; i += BIG_T) { keys[i] = EMPTY_KEY; minpos[i] = INT32_MAX; wsum[i] = 0; }
        __syncthreads();
        const int32_t a = mem[2 * c], b = mem[2 * c + 1];
        const int64_t da = g.rp[a + 1] - g.rp[a];
        for (int64_t j = threadIdx.x; j < deg; j += BIG_T) {
            int32_t cu, wt;
            row_entry(g, a, b, da, j, cmap, cu, wt);
            if (cu == (int32_t)c) continue;
            uint32_t h = slot_hash(cu, lg);
            bool placed = false;
            for (int64_t probe = 0; probe < S; ++probe) {
                const int32_t old = atomicCAS(&keys[h], EMPTY_KEY, cu);
                if (old == EMPTY_KEY || old == cu) { placed = true; break; }
                h = (h + 1) & (uint32_t)(S - 1);
            }
            if (!placed) { atomicExch(err, 1); continue; }
            atomicMin(&minpos[h], (int32_t)j);
            atomicAdd(&wsum[h], wt);
        }
        __syncthreads();
        int32_t carry = 0;
        const int64_t o = off[c];
        for (int64_t base = 0; base < deg; base += BIG_T) {
            const int64_t j = base + threadIdx.x;
            int32_t first = 0, cu = -1;
            uint32_t h = 0;
            if (j < deg) {
                int32_t wt;
                row_entry(g, a, b, da, j, cmap, cu, wt);
                if (cu != (int32_t)c) {
                    h = slot_hash(cu, lg);
                    for (int64_t probe = 0; probe < S && keys[h] != cu; ++probe) h = (h + 1) & (uint32_t)(S - 1);
                    first = (keys[h] == cu && minpos[h] == (int32_t)j) ? 1 : 0;
                }
            }
            int32_t tot;
            const int32_t r = block_scan_excl(first, sh, tot);
            if (first) { tci[o + carry + r] = cu; tew[o + carry + r] = wsum[h]; }
            carry += tot;
        }
        if (threadIdx.x == 0) cnt[c] = carry;
        __syncthreads();
    }
}

// warp per coarse row: temporary (row bound offsets) -> final CSR
__global__ void __launch_bounds__(256) k_contract_copy(int64_t nc, const int64_t* __restrict__ off,
                                                       const int64_t* __restrict__ crp, const int32_t* __restrict__ tci,
                                                       const int32_t* __restrict__ tew, int32_t* __restrict__ ci,
                                                       int32_t* __restrict__ ew) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = wid; c < nc; c += nw) {
        const int64_t src = off[c], dst = crp[c], len = crp[c + 1] - crp[c];
        for (int64_t i = lane; i < len; i += 32) { ci[dst + i] = tci[src + i]; ew[dst + i] = tew[src + i]; }
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
    int32_t* tci = c.tmp_alloc<int32_t>(T);
    int32_t* tew = c.tmp_alloc<int32_t>(T);
    int32_t* rowcnt = c.tmp_alloc<int32_t>(nc);
    int32_t* list1 = c.tmp_alloc<int32_t>(nc);
    int32_t* list2 = c.tmp_alloc<int32_t>(nc);
    int64_t* tsize = c.tmp_alloc<int64_t>(nc + 1);
    int32_t* err = c.tmp_alloc<int32_t>(1);
    memset_async(c, d_tot + 1, 0, 2 * sizeof(int64_t));
    memset_async(c, err, 0, sizeof(int32_t));
    k_contract_small<<<grid_for(nc * 32, 256, c.sm_count * 8), 256, 0, c.s>>>(g, nc, mem, fine.cmap, off, cdeg, tci,
                                                                             tew, rowcnt);
    GP_LAUNCHED(c);
    k_big_rows<<<grid_for(nc, 256), 256, 0, c.s>>>(nc, cdeg, list1, list2, tsize, d_tot + 1);
    GP_LAUNCHED(c);
    GP_CUDA(cudaMemcpyAsync(c.h_pinned, d_tot + 1, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
    c.sync();
    const int64_t nmid = c.h_pinned[0], nbig = c.h_pinned[1];
    if (nmid > 0) {
        const int blocks = grid_for(nmid * 32, 256, c.sm_count * 8);
        const int64_t warps = (int64_t)blocks * 8;
        int32_t* wtab = c.tmp_alloc<int32_t>(warps * 2 * MID_SLOTS);
        k_contract_mid<<<blocks, 256, 0, c.s>>>(g, list1, nmid, mem, fine.cmap, off, cdeg, wtab, tci, tew, rowcnt, err);
        GP_LAUNCHED(c);
    }
    if (nbig > 0) {
        int64_t* toff = c.tmp_alloc<int64_t>(nbig + 1);
        scan_excl_i64(c, tsize, toff, nbig, toff + nbig);
        const int64_t tslots = read_i64(c, toff + nbig);
        int32_t* gtab = c.tmp_alloc<int32_t>(3 * std::max<int64_t>(tslots, 1));
        k_contract_big<<<(unsigned)std::min<int64_t>(nbig, (int64_t)c.sm_count * 2), BIG_T, 0, c.s>>>(
            g, list2, nbig, mem, fine.cmap, off, cdeg, toff, gtab, tci, tew, rowcnt, err);
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
    k_contract_copy<<<grid_for(nc * 32, 256, c.sm_count * 8), 256, 0, c.s>>>(nc, off, crp, tci, tew, cci, cew);
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

}  // namespace gp
