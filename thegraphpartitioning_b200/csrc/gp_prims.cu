// gp_prims.cu -- arena, prefix scans and the LSD radix sort.
//
// Scans are three-phase (tile reduce -> scan of tile sums -> tile scan), each
// tile 256 threads x 8 items.  The radix sort is a stable LSD sort of 64-bit
// keys with 32-bit payloads, 8-bit digits: per pass a tile histogram kernel, a
// scan of the digit-major (digit, tile) count table, and a scatter kernel that
// ranks items stably inside the tile with warp match/ballot and per-warp digit
// counters in shared memory.
#define GP_TU_ID 1   // site ids of the bounds-checked build
#include "gp_common.cuh"

#include <algorithm>
#include <cstring>

namespace gp {

// ================================================================ arena
void* Arena::alloc(size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    if (!chunks_.empty()) {
        for (size_t i = cur_; i < chunks_.size(); ++i) {
            Chunk& ch = chunks_[i];
            if (i > cur_) ch.off = 0;
            if (ch.off + bytes <= ch.size) {
                cur_ = i;
                void* p = ch.p + ch.off;
                ch.off += bytes;
                used_total_ += bytes;
                peak_total_ = std::max(peak_total_, used_total_);
                return p;
            }
        }
    }
    size_t last = chunks_.empty() ? 0 : chunks_.back().size;
    size_t sz = std::max<size_t>(bytes, std::max<size_t>(last * 2, (size_t)64 << 20));
    char* p = nullptr;
    cudaError_t e = cudaMalloc(&p, sz);
    if (e != cudaSuccess) {
        cudaGetLastError();
        sz = bytes;
        e = cudaMalloc(&p, sz);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw GpError(GP_ENOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
        }
    }
    chunks_.push_back(Chunk{p, sz, bytes});
    cur_ = chunks_.size() - 1;
    used_total_ += bytes;
    peak_total_ = std::max(peak_total_, used_total_);
    return p;
}

void Arena::restore(const Mark& m) {
    if (chunks_.empty()) return;
    for (size_t i = m.chunk + 1; i < chunks_.size(); ++i) chunks_[i].off = 0;
    cur_ = m.chunk;
    chunks_[cur_].off = m.off;
    used_total_ = m.total;
}

void Arena::reset() {
    for (auto& ch : chunks_) ch.off = 0;
    cur_ = 0;
    used_total_ = 0;
}

void Arena::consolidate() {
    if (chunks_.size() <= 1) { reset(); peak_total_ = 0; return; }
    size_t want = 0;
    for (auto& ch : chunks_) want += ch.size;
    want = std::max(want, peak_total_);
    release();
    char* p = nullptr;
    if (cudaMalloc(&p, want) == cudaSuccess) chunks_.push_back(Chunk{p, want, 0});
    else cudaGetLastError();
    cur_ = 0; used_total_ = 0; peak_total_ = 0;
}

void Arena::release() {
    for (auto& ch : chunks_) cudaFree(ch.p);
    chunks_.clear();
    cur_ = 0; used_total_ = 0;
}

size_t Arena::capacity() const {
    size_t s = 0;
    for (auto& ch : chunks_) s += ch.size;
    return s;
}

// ================================================================ helpers
int64_t read_i64(Ctx& c, const int64_t* d) {
    GP_CUDA(cudaMemcpyAsync(c.h_pinned, d, sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
    c.sync();
    return c.h_pinned[0];
}

void memset_async(Ctx& c, void* p, int value, size_t bytes) {
    if (bytes) GP_CUDA(cudaMemsetAsync(p, value, bytes, c.s));
}

// ================================================================ scan
constexpr int SCAN_T = 256;
constexpr int SCAN_I = 8;
constexpr int SCAN_TILE = SCAN_T * SCAN_I;

template <class TI, class TO>
__global__ void k_tile_reduce(const TI* __restrict__ in, int64_t n, TO* __restrict__ tile_sums) {
    __shared__ TO sh[33];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    TO s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_I; ++i) {
        int64_t idx = base + (int64_t)i * SCAN_T + threadIdx.x;
        if (idx < n) s += (TO)in[idx];
    }
    TO tot;
    block_excl_scan<TO>(s, sh, tot);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// single block: exclusive scan of the tile sums, in place; writes the grand total
template <class T>
__global__ void k_scan_small(T* __restrict__ a, int64_t n, T* __restrict__ total) {
    __shared__ T sh[33];
    T carry = 0;
    for (int64_t base = 0; base < n; base += blockDim.x) {
        int64_t idx = base + threadIdx.x;
        T x = idx < n ? a[idx] : T(0);
        T tot;
        T e = block_excl_scan<T>(x, sh, tot);
        if (idx < n) a[idx] = carry + e;
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <class TI, class TO>
__global__ void k_tile_scan(const TI* __restrict__ in, TO* __restrict__ out, int64_t n,
                            const TO* __restrict__ tile_offs) {
    __shared__ TO sh[33];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_I;
    TO v[SCAN_I];
    TO s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_I; ++i) {
        int64_t idx = base + i;
        v[i] = idx < n ? (TO)in[idx] : TO(0);
        s += v[i];
    }
    TO tot;
    TO e = block_excl_scan<TO>(s, sh, tot) + tile_offs[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_I; ++i) {
        int64_t idx = base + i;
        if (idx < n) out[idx] = e;
        e += v[i];
    }
}

template <class TI, class TO>
static void scan_excl(Ctx& c, const TI* in, TO* out, int64_t n, TO* d_total) {
    if (n <= 0) {
        if (d_total) GP_CUDA(cudaMemsetAsync(d_total, 0, sizeof(TO), c.s));
        return;
    }
    auto m = c.tmp->save();
    int64_t nt = (n + SCAN_TILE - 1) / SCAN_TILE;
    TO* sums = c.tmp_alloc<TO>(nt);
    k_tile_reduce<TI, TO><<<(unsigned)nt, SCAN_T, 0, c.s>>>(in, n, sums);
    GP_LAUNCHED(c);
    k_scan_small<TO><<<1, 1024, 0, c.s>>>(sums, nt, d_total);
    GP_LAUNCHED(c);
    k_tile_scan<TI, TO><<<(unsigned)nt, SCAN_T, 0, c.s>>>(in, out, n, sums);
    GP_LAUNCHED(c);
    c.bytes += (int64_t)(2 * sizeof(TI) + sizeof(TO)) * n;
    c.tmp->restore(m);
}

void scan_excl_i32_to_i64(Ctx& c, const int32_t* in, int64_t* out, int64_t n, int64_t* d_total) {
    scan_excl<int32_t, int64_t>(c, in, out, n, d_total);
}
void scan_excl_i64(Ctx& c, const int64_t* in, int64_t* out, int64_t n, int64_t* d_total) {
    scan_excl<int64_t, int64_t>(c, in, out, n, d_total);
}

// ================================================================ radix sort
constexpr int RS_T = 256;                 // threads per tile
constexpr int RS_I = 8;                   // items per thread
constexpr int RS_TILE = RS_T * RS_I;      // 2048 items
constexpr int RS_W = RS_T / 32;           // warps per tile
constexpr int RS_WITEMS = 32 * RS_I;      // items per warp (contiguous)

// digit-major counts: counts[d * ntiles + tile]
__global__ void k_rs_hist(const uint64_t* __restrict__ keys, int64_t n, int shift,
                          int32_t* __restrict__ counts, int64_t ntiles) {
    __shared__ int32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RS_TILE;
#pragma unroll
    for (int i = 0; i < RS_I; ++i) {
        int64_t idx = base + (int64_t)i * RS_T + threadIdx.x;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 0xFF], 1);
    }
    __syncthreads();
    counts[(int64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(RS_T) k_rs_scatter(const uint64_t* __restrict__ kin, const int32_t* __restrict__ vin,
                             uint64_t* __restrict__ kout, int32_t* __restrict__ vout,
                             int64_t n, int shift, const int64_t* __restrict__ offs, int64_t ntiles) {
    __shared__ int32_t wcnt[RS_W][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < RS_W * 256; i += RS_T) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const int64_t wbase = (int64_t)blockIdx.x * RS_TILE + (int64_t)w * RS_WITEMS;
    uint64_t k[RS_I];
    int32_t v[RS_I];
    uint32_t dg[RS_I];
    const uint32_t lt = (1u << lane) - 1u;
    // pass A: per-warp digit counts
#pragma unroll
    for (int i = 0; i < RS_I; ++i) {
        int64_t idx = wbase + i * 32 + lane;
        bool ok = idx < n;
        k[i] = ok ? kin[idx] : 0;
        v[i] = ok ? vin[idx] : 0;
        dg[i] = ok ? (uint32_t)((k[i] >> shift) & 0xFF) : 256u;
        uint32_t peers = __match_any_sync(0xffffffffu, dg[i]);
        int leader = __ffs(peers) - 1;
        if (ok && lane == leader) wcnt[w][dg[i]] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // exclusive prefix over warps per digit, plus the global tile offset
    {
        int d = threadIdx.x;  // RS_T == 256 digits
        int64_t off = offs[(int64_t)d * ntiles + blockIdx.x];
        int32_t run = 0;
#pragma unroll
        for (int ww = 0; ww < RS_W; ++ww) {
            int32_t cnt = wcnt[ww][d];
            wcnt[ww][d] = run;
            run += cnt;
        }
        // store the 64-bit base split: tile offsets fit int64; keep it in a
        // second table indexed by digit
        __shared__ int64_t dbase[256];
        dbase[d] = off;
        __syncthreads();
        // pass B: positions
#pragma unroll
        for (int i = 0; i < RS_I; ++i) {
            int64_t idx = wbase + i * 32 + lane;
            bool ok = idx < n;
            uint32_t peers = __match_any_sync(0xffffffffu, dg[i]);
            int leader = __ffs(peers) - 1;
            int32_t basecnt = ok ? wcnt[w][dg[i]] : 0;
            __syncwarp();
            if (ok) {
                int64_t pos = dbase[dg[i]] + basecnt + __popc(peers & lt);
                if (GP_IN(pos, n)) {
                    kout[pos] = k[i];
                    vout[pos] = v[i];
                }
                if (lane == leader) wcnt[w][dg[i]] = basecnt + __popc(peers);
            }
            __syncwarp();
        }
    }
}

void radix_sort_pairs(Ctx& c, uint64_t* keys, int32_t* vals, uint64_t* keys_tmp, int32_t* vals_tmp,
                      int64_t n, int bits) {
    if (n <= 1 || bits <= 0) return;
    auto m = c.tmp->save();
    const int64_t ntiles = (n + RS_TILE - 1) / RS_TILE;
    int32_t* counts = c.tmp_alloc<int32_t>(256 * ntiles);
    int64_t* offs = c.tmp_alloc<int64_t>(256 * ntiles);
    int passes = (bits + 7) / 8;
    uint64_t* ka = keys; int32_t* va = vals;
    uint64_t* kb = keys_tmp; int32_t* vb = vals_tmp;
    for (int p = 0; p < passes; ++p) {
        int shift = 8 * p;
        k_rs_hist<<<(unsigned)ntiles, RS_T, 0, c.s>>>(ka, n, shift, counts, ntiles);
        GP_LAUNCHED(c);
        scan_excl_i32_to_i64(c, counts, offs, 256 * ntiles, nullptr);
        k_rs_scatter<<<(unsigned)ntiles, RS_T, 0, c.s>>>(ka, va, kb, vb, n, shift, offs, ntiles);
        GP_LAUNCHED(c);
        c.bytes += n * (8 + 2 * 12);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    if (ka != keys) {
        GP_CUDA(cudaMemcpyAsync(keys, ka, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, c.s));
        GP_CUDA(cudaMemcpyAsync(vals, va, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, c.s));
    }
    c.tmp->restore(m);
}

}  // namespace gp
