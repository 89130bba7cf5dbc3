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

template <int MODE>
__global__ void __launch_bounds__(256) k_match_scan(DGraph g, const int32_t* __restrict__ heavy, int64_t nheavy,
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
    for (int64_t v = wid; v < g.n; v += nw) {
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

__global__ void k_handshake(int64_t n, const int32_t* __restrict__ prop, int32_t* __restrict__ match,
                            int64_t* __restrict__ pairs) {
    int64_t local = 0;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        if (match[v] != -1) continue;
        const int32_t u = prop[v];
        if (u >= 0 && prop[u] == (int32_t)v) {
            match[v] = u;
            if (v < u) ++local;
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
    int64_t* d_pairs = c.tmp_alloc<int64_t>(2);
    GP_CUDA(cudaMemsetAsync(match, 0xff, sizeof(int32_t) * g.n, c.s));
    const int light_blocks = grid_for(g.n * 32, 256, c.sm_count * 8);
    const int grid = (int)L.nheavy + light_blocks;
    int64_t pairs = 0;
    int rounds = 0;
    for (int r = 0; r < P.o.match_rounds; ++r) {
        memset_async(c, d_pairs, 0, sizeof(int64_t));
        k_match_scan<0><<<grid, 256, 0, c.s>>>(g, L.heavy, L.nheavy, match, prop, salt, P.maxvw, nullptr, nullptr, 0);
        GP_LAUNCHED(c);
        k_handshake<<<grid_for(g.n, 256), 256, 0, c.s>>>(g.n, prop, match, d_pairs);
        GP_LAUNCHED(c);
        c.bytes += L.scan_bytes() + 4 * g.m /*match[u]*/ + 12 * g.n;
        int64_t newp = read_i64(c, d_pairs);
        rounds = r + 1;
        pairs += newp;
        if (newp == 0) break;
    }
    if (P.o.two_hop > 0 && 4 * (g.n - pairs) > 3 * g.n) {
        const int nb = bits_for(g.n);
        uint64_t* keys = c.tmp_alloc<uint64_t>(g.n);
        uint64_t* keys2 = c.tmp_alloc<uint64_t>(g.n);
        int32_t* vals = c.tmp_alloc<int32_t>(g.n);
        int32_t* vals2 = c.tmp_alloc<int32_t>(g.n);
        memset_async(c, d_pairs, 0, 2 * sizeof(int64_t));
        k_match_scan<1><<<grid, 256, 0, c.s>>>(g, L.heavy, L.nheavy, match, nullptr, salt, P.maxvw, keys, d_pairs + 1, nb);
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

// warp per coarse vertex: write (c << nb | cmap[u], w) for every entry of its members' rows
__global__ void __launch_bounds__(256) k_fill(DGraph g, int64_t nc, const int32_t* __restrict__ mem,
                                              const int32_t* __restrict__ cmap, const int64_t* __restrict__ off,
                                              int nb, uint64_t* __restrict__ keys, int32_t* __restrict__ vals) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t cc = wid; cc < nc; cc += nw) {
        int64_t pos = off[cc];
        const uint64_t hi = (uint64_t)cc << nb;
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const int32_t x = mem[2 * cc + t];
            if (x < 0) continue;
            const int64_t beg = g.rp[x], end = g.rp[x + 1];
            for (int64_t e = beg + lane; e < end; e += 32) {
                keys[pos + (e - beg)] = hi | (uint32_t)cmap[g.ci[e]];
                vals[pos + (e - beg)] = g.ew ? g.ew[e] : 1;
            }
            pos += end - beg;
        }
    }
}

// unique flags over sorted keys: first of a run and not a self-loop
__global__ void k_uniq_flags(const uint64_t* __restrict__ keys, int64_t T, int nb, int32_t* __restrict__ flag,
                             int32_t* __restrict__ rowcnt) {
    const uint64_t lowmask = (1ull << nb) - 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < T; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        const bool head = (i == 0) || (keys[i - 1] != k);
        const bool self = (k >> nb) == (k & lowmask);
        const int f = (head && !self) ? 1 : 0;
        flag[i] = f;
        if (f) atomicAdd(&rowcnt[k >> nb], 1);
    }
}

__global__ void k_uniq_write(const uint64_t* __restrict__ keys, const int32_t* __restrict__ vals, int64_t T, int nb,
                             const int32_t* __restrict__ flag, const int64_t* __restrict__ pos,
                             int32_t* __restrict__ ci, int32_t* __restrict__ ew) {
    const uint64_t lowmask = (1ull << nb) - 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < T; i += (int64_t)gridDim.x * blockDim.x) {
        if (!flag[i]) continue;
        const uint64_t k = keys[i];
        int64_t s = vals[i];
        for (int64_t j = i + 1; j < T && keys[j] == k; ++j) s += vals[j];
        ci[pos[i]] = (int32_t)(k & lowmask);
        ew[pos[i]] = (int32_t)s;
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
    int64_t* off = c.tmp_alloc<int64_t>(nc);
    scan_excl_i64(c, cdeg, off, nc, d_tot + 1);
    const int64_t T = g.m;
    const int nb = bits_for(nc);
    uint64_t* keys = c.tmp_alloc<uint64_t>(T);
    int32_t* vals = c.tmp_alloc<int32_t>(T);
    uint64_t* keys2 = c.tmp_alloc<uint64_t>(T);
    int32_t* vals2 = c.tmp_alloc<int32_t>(T);
    k_fill<<<grid_for(nc * 32, 256, c.sm_count * 8), 256, 0, c.s>>>(g, nc, mem, fine.cmap, off, nb, keys, vals);
    GP_LAUNCHED(c);
    radix_sort_pairs(c, keys, vals, keys2, vals2, T, 2 * nb);
    int32_t* uflag = c.tmp_alloc<int32_t>(T);
    int32_t* rowcnt = c.tmp_alloc<int32_t>(nc);
    int64_t* upos = c.tmp_alloc<int64_t>(T);
    memset_async(c, rowcnt, 0, sizeof(int32_t) * nc);
    k_uniq_flags<<<grid_for(T, 256), 256, 0, c.s>>>(keys, T, nb, uflag, rowcnt);
    GP_LAUNCHED(c);
    scan_excl_i32_to_i64(c, uflag, upos, T, d_tot + 2);
    const int64_t mc = read_i64(c, d_tot + 2);
    int64_t* crp = c.keep_alloc<int64_t>(nc + 1);
    scan_excl_i32_to_i64(c, rowcnt, crp, nc, crp + nc);
    int32_t* cci = c.keep_alloc<int32_t>(mc);
    int32_t* cew = c.keep_alloc<int32_t>(mc);
    k_uniq_write<<<grid_for(T, 256), 256, 0, c.s>>>(keys, vals, T, nb, uflag, upos, cci, cew);
    GP_LAUNCHED(c);
    c.bytes += 2 * (8 * (g.n + 1) + 8 * g.m) + 8 * (nc + 1) + 8 * mc + 4 * nc + 12 * T;
    coarse.g.n = nc;
    coarse.g.m = mc;
    coarse.g.rp = crp;
    coarse.g.ci = cci;
    coarse.g.ew = cew;
    coarse.g.vw = cvw;
    c.tmp->restore(mk);
}

}  // namespace gp
