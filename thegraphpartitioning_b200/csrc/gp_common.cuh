// gp_common.cuh -- shared definitions of the B200 partitioner library.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>
#include <stdexcept>

#include "../../include/gp_partition.h"

namespace gp {

// ---------------------------------------------------------------- errors
// Library code throws GpError internally; the C-ABI entry points catch it and
// turn it into a return code plus gp_last_error() text.  Nothing exits.
struct GpError : std::runtime_error {
    int code;
    GpError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define GP_CUDA(call)                                                              \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess)                                                     \
            throw ::gp::GpError(e_ == cudaErrorMemoryAllocation ? GP_ENOMEM : GP_ECUDA, \
                                std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define GP_LAUNCHED(ctx)                                                           \
    do {                                                                           \
        cudaError_t e_ = cudaGetLastError();                                       \
        if (e_ != cudaSuccess)                                                     \
            throw ::gp::GpError(GP_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
        (ctx).launches++;                                                          \
    } while (0)

// ---------------------------------------------------------------- bounds-checked build
// Compiled with -DGP_CHECKED (libgp_b200_checked.so), GP_IN(i, n) tests a
// data-dependent index before the access it guards: a failing check counts a
// violation, records the first failing site (translation unit and line) and
// the access is skipped.  In the regular build GP_IN is the constant true.
// Each translation unit has its own counters; gp_checked_violations() sums
// them.  This is the device-side stand-in for a memory checker: the checks
// run at full speed on the GPU inside the normal kernels.
#ifndef GP_TU_ID
#define GP_TU_ID 0
#endif
#ifdef GP_CHECKED
static __device__ unsigned long long g_chk_count;
static __device__ unsigned long long g_chk_first;   // site + 1 of the first violation (0: none)
__device__ __forceinline__ bool chk_in(int64_t i, int64_t n, int site) {
    if (i >= 0 && i < n) return true;
    atomicAdd(&g_chk_count, 1ull);
    atomicCAS(&g_chk_first, 0ull, (unsigned long long)site + 1ull);
    return false;
}
#define GP_IN(i, n) (::gp::chk_in((int64_t)(i), (int64_t)(n), GP_TU_ID * 100000 + __LINE__))
typedef void (*chk_fetch_fn)(unsigned long long* count, unsigned long long* first, bool clear);
void chk_register(chk_fetch_fn f);
namespace {
void chk_fetch_tu(unsigned long long* count, unsigned long long* first, bool clear) {
    unsigned long long c = 0, f = 0;
    cudaMemcpyFromSymbol(&c, g_chk_count, sizeof c);
    cudaMemcpyFromSymbol(&f, g_chk_first, sizeof f);
    if (clear) {
        const unsigned long long z = 0;
        cudaMemcpyToSymbol(g_chk_count, &z, sizeof z);
        cudaMemcpyToSymbol(g_chk_first, &z, sizeof z);
    }
    *count += c;
    if (!*first) *first = f;
}
struct ChkRegister { ChkRegister() { chk_register(&chk_fetch_tu); } };
ChkRegister chk_register_tu;
}  // namespace
#else
#define GP_IN(i, n) true
#endif

// ---------------------------------------------------------------- rules
// The deterministic rule set shared with the CPU oracle (oracle/oracle.cpp
// restates the same functions independently).
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
    // splitmix64 finalizer (published constants of Stafford's Mix13)
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27; x *= 0x94d049bb133111ebULL;
    x ^= x >> 31; return x;
}
__host__ __device__ __forceinline__ uint64_t level_salt(uint64_t seed, int level) {
    return mix64(seed ^ mix64(0x9E3779B97F4A7C15ULL * (uint64_t)(level + 1)));
}
__host__ __device__ __forceinline__ uint64_t trial_salt(uint64_t seed, int t) {
    return mix64(seed ^ mix64(0xD1B54A32D192ED03ULL * (uint64_t)(t + 1)));
}
__host__ __device__ __forceinline__ uint64_t depth_salt(uint64_t tsalt, int d) {
    return mix64(tsalt ^ mix64(0x8CB92BA72F3D8DD7ULL * (uint64_t)(d + 1)));
}
// MurmurHash3's 32-bit finalizer (Appleby, published constants)
__host__ __device__ __forceinline__ uint32_t fmix32(uint32_t h) {
    h ^= h >> 16; h *= 0x85EBCA6Bu;
    h ^= h >> 13; h *= 0xC2B2AE35u;
    h ^= h >> 16; return h;
}
// 32-bit salt of a level's matching tie-break (high half of the level salt)
__host__ __device__ __forceinline__ uint32_t edge_salt(uint64_t seed, int level) {
    return (uint32_t)(level_salt(seed, level) >> 32);
}
// Symmetric per-edge tie-break: the two ids, ordered, times two odd constants
// (golden ratio, xxHash's second prime) plus the salt, then fmix32.  All
// 32-bit: two IMADs and the finalizer per entry of every matching round.
__host__ __device__ __forceinline__ uint32_t edge_hash(uint32_t salt, int32_t a, int32_t b) {
    const uint32_t lo = (uint32_t)(a < b ? a : b), hi = (uint32_t)(a < b ? b : a);
    return fmix32(lo * 0x9E3779B1u + hi * 0x85EBCA77u + salt);
}
__host__ __device__ __forceinline__ uint64_t edge_key(int32_t w, uint32_t h) {
    return ((uint64_t)(uint32_t)w << 32) | h;
}
__host__ __device__ __forceinline__ uint32_t mag_bucket(uint32_t x) {
    if (x < 64) return x;
#ifdef __CUDA_ARCH__
    int e = 31 - __clz(x);
#else
    int e = 31 - __builtin_clz(x);
#endif
    uint32_t mant = (x >> (e - 4)) & 15u;
    return 64u + (uint32_t)(e - 6) * 16u + mant;
}
#ifdef __CUDACC__
// Argmax over the lanes of `mask` (every lane of the group calls it with the
// group's mask) of (64-bit key, id): the largest key, ties to the smaller id
// compared unsigned (so -1, "none", loses every tie).  Three redux.sync steps:
// the key's high half, its low half among the lanes holding the top high
// half, then the id among the lanes holding the top key.
__device__ __forceinline__ void group_argmax64(uint32_t mask, uint64_t& k, int32_t& id) {
    const uint32_t hi = (uint32_t)(k >> 32), lo = (uint32_t)k;
    const uint32_t mh = __reduce_max_sync(mask, hi);
    const uint32_t ml = __reduce_max_sync(mask, hi == mh ? lo : 0u);
    const uint32_t mi = __reduce_min_sync(mask, (hi == mh && lo == ml) ? (uint32_t)id : 0xffffffffu);
    k = ((uint64_t)mh << 32) | ml;
    id = (int32_t)mi;
}
// Entry slices of a CSR (rp: n + 1 row starts, nondecreasing): the row holding
// entry o is the last row starting at or before it (empty rows share starts).
// A warp walking a slice of entries keeps a window of 32 consecutive rows, one
// start per lane (rows past n start at m); csr_window_lane gives the lane of
// the window row holding entry oi, which must lie inside the window.
__device__ __forceinline__ int64_t csr_row_of(const int64_t* __restrict__ rp, int64_t n, int64_t o) {
    int64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (rp[mid] <= o) lo = mid; else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ int csr_window_lane(int64_t s, int64_t oi) {
    int l = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
        const int64_t sv = __shfl_sync(0xffffffffu, s, l + step);
        if (sv <= oi) l += step;
    }
    return l;
}
// entries per warp of an entry-sliced pass over m entries: about 32 warps
// per SM, at least 256 and at most 16384 entries each (a multiple of 256)
inline int64_t csr_slice(int64_t m, int sm_count) {
    int64_t s = (m + (int64_t)sm_count * 32 - 1) / ((int64_t)sm_count * 32);
    s = (s + 255) & ~(int64_t)255;
    return s < 256 ? 256 : (s > 16384 ? 16384 : s);
}
// The same argmax and a sum over aligned groups of TILE lanes (TILE a power of
// two <= 32; every lane of the warp calls them).  A group smaller than the
// warp reduces with butterfly shuffles inside the group: a redux.sync whose
// member mask differs between the lanes of one warp runs once per group.
template <int TILE>
__device__ __forceinline__ void tile_argmax64(uint64_t& k, int32_t& id) {
    if constexpr (TILE == 32) {
        group_argmax64(0xffffffffu, k, id);
    } else {
#pragma unroll
        for (int o = TILE / 2; o > 0; o >>= 1) {
            const uint64_t k2 = __shfl_xor_sync(0xffffffffu, k, o);
            const int32_t i2 = __shfl_xor_sync(0xffffffffu, id, o);
            if (k2 > k || (k2 == k && (uint32_t)i2 < (uint32_t)id)) { k = k2; id = i2; }
        }
    }
}
template <int TILE>
__device__ __forceinline__ uint32_t tile_sum_u32(uint32_t x) {
    if constexpr (TILE == 32) {
        return __reduce_add_sync(0xffffffffu, x);
    } else {
#pragma unroll
        for (int o = TILE / 2; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        return x;
    }
}
#endif
// Four consecutive entries [e, e + 4) of a row [beg, end) of a CSR array
// (column ids, weights or per-entry priorities), e a multiple of 4: one
// 16-byte streaming load when the array is 16-byte aligned (v4) and all four
// lie inside the row, else element loads; positions outside the row read as
// `fill`.  Nothing outside the row is read.
__device__ __forceinline__ void ld4_row(const int32_t* __restrict__ a, int64_t e, int64_t beg, int64_t end, bool v4,
                                        int32_t fill, int32_t (&x)[4]) {
    if (v4 && e >= beg && e + 3 < end) {
        const int4 t = __ldcs(reinterpret_cast<const int4*>(a + e));
        x[0] = t.x; x[1] = t.y; x[2] = t.z; x[3] = t.w;
    } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) x[c] = (e + c >= beg && e + c < end) ? __ldcs(a + e + c) : fill;
    }
}
__host__ __device__ __forceinline__ bool aligned16(const void* p) {
    return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

template <class T>
__device__ __forceinline__ T warp_incl_scan(T x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// block-wide exclusive scan of one value per thread; sh_warp holds 33 values;
// returns the block total in `total`
template <class T>
__device__ __forceinline__ T block_excl_scan(T x, T* sh_warp, T& total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T inc = warp_incl_scan(x);
    if (lane == 31) sh_warp[w] = inc;
    __syncthreads();
    if (w == 0) {
        T s = lane < nw ? sh_warp[lane] : T(0);
        T si = warp_incl_scan(s);
        if (lane < nw) sh_warp[lane] = si - s;
        if (lane == nw - 1) sh_warp[32] = si;
    }
    __syncthreads();
    T r = inc - x + sh_warp[w];
    total = sh_warp[32];
    __syncthreads();
    return r;
}

__host__ __device__ __forceinline__ uint32_t loss_bucket(int32_t loss) {
    if (loss >= 0) return 480u + mag_bucket((uint32_t)loss);
    return 480u - mag_bucket((uint32_t)(-(int64_t)loss));
}

// ---------------------------------------------------------------- arena
// Grow-only device memory cache.  A call bump-allocates from chunks; when a
// call needed more than one chunk, the chunks are merged into one at the end
// so that the next call of the same size allocates nothing.
class Arena {
public:
    ~Arena() { release(); }
    void* alloc(size_t bytes);
    void reset();            // forget all allocations of the call
    size_t mark() const { return used_total_; }
    void release();          // free device memory
    void consolidate();      // merge chunks after a call
    size_t capacity() const;
    // stack-like scratch: restore to an earlier mark (only within the last chunk)
    struct Mark { size_t chunk, off, total; };
    Mark save() const { return Mark{cur_, chunks_.empty() ? 0 : chunks_[cur_].off, used_total_}; }
    void restore(const Mark& m);
private:
    struct Chunk { char* p; size_t size; size_t off; };
    std::vector<Chunk> chunks_;
    size_t cur_ = 0;
    size_t used_total_ = 0;
    size_t peak_total_ = 0;
};

// ---------------------------------------------------------------- context
struct Ctx {
    cudaStream_t s = nullptr;
    Arena* keep = nullptr;     // lives for the whole call (hierarchy)
    Arena* tmp = nullptr;      // scratch, restored after each step
    int64_t launches = 0;
    int64_t bytes = 0;         // algorithmic bytes of executed passes
    int sm_count = 148;
    int ctas_per_sm = 64;         // grid cap of row-scanning kernels, CTAs per SM (gp_options.ctas_per_sm)
    int64_t* h_pinned = nullptr;  // small pinned staging buffer (64 int64)
    // opt-in timing of the connectivity pass
    bool profile = false;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;
    double ms_conn = 0;
    double ms_gnn = 0;            // learned mode: device time of the scorer's inference
    int64_t conn_launches = 0, conn_bytes = 0;
    template <class T> T* keep_alloc(int64_t count) { return (T*)keep->alloc(sizeof(T) * (size_t)(count > 0 ? count : 1)); }
    template <class T> T* tmp_alloc(int64_t count) { return (T*)tmp->alloc(sizeof(T) * (size_t)(count > 0 ? count : 1)); }
    void sync() { GP_CUDA(cudaStreamSynchronize(s)); }
};

// Device-side view of one level of the hierarchy.
struct DGraph {
    int64_t n = 0, m = 0;
    const int64_t* rp = nullptr;
    const int32_t* ci = nullptr;
    const int32_t* ew = nullptr;   // nullptr = unit
    const int32_t* vw = nullptr;   // nullptr = unit
};

// ---------------------------------------------------------------- launch helpers
inline int grid_for(int64_t items, int per_block, int cap = 148 * 16) {
    int64_t g = (items + per_block - 1) / per_block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}
constexpr int kHeavyDeg = 4096;   // default: rows longer than this take whole CTAs (gp_options.heavy_deg)
constexpr int kItemLen = 32768;   // default: entries of one CTA item of a long row (gp_options.item_len)
// the learned V-cycle's fixed row layout (its scorer's float sums follow it)
constexpr int kLearnedHeavyDeg = 2048;
constexpr int kLearnedItemLen = 16384;

// ---------------------------------------------------------------- primitives (gp_prims.cu)
// exclusive scan; out may alias in; returns total on the host if total_out != nullptr
void scan_excl_i32_to_i64(Ctx& c, const int32_t* in, int64_t* out, int64_t n, int64_t* d_total);
void scan_excl_i64(Ctx& c, const int64_t* in, int64_t* out, int64_t n, int64_t* d_total);
// LSD radix sort of (key, val) pairs by the low `bits` bits of key.  Result in
// keys/vals (ping-pong through the provided temporaries).
void radix_sort_pairs(Ctx& c, uint64_t* keys, int32_t* vals, uint64_t* keys_tmp, int32_t* vals_tmp,
                      int64_t n, int bits);
int64_t read_i64(Ctx& c, const int64_t* d);   // synchronous small read
void memset_async(Ctx& c, void* p, int value, size_t bytes);

}  // namespace gp
