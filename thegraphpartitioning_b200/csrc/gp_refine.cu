// gp_refine.cu -- gain refinement, rebalancing and projection.
//
// Replaces deterministicRefinement (src/gpu_part.cu:509-759) with its kernels
// computeGainsAndDestinations, markCandidates, tokenPassing,
// bufferCandidateMoves, computeAvailableCapacity, bitonicSortStep/customSortMoves,
// selectMoves, commitMoves (src/gpu_part.cu:258-397, 472-506), the edge-cut
// kernel (src/gpu_part.cu:400-423) and kwayMapCoarseToFine (src/gpu_part.cu:763-772).
//
// One refinement iteration:
//   k_conn      one pass over every row: exact int32 part-connectivity histogram
//               in shared memory (warp-private for rows <= kHeavyDeg, CTA-wide
//               for longer rows), cut contribution of every vertex (so the cut
//               of the current state costs no extra pass), and the move proposal
//               of the mode the device derives from the part weights
//               (label propagation when no part exceeds Lmax, else rebalancing).
//   LP:         k_lp_apply (the connectivity pass already copied part/lock into
//               the next buffers): each candidate re-evaluates its gain
//               against the proposals of higher-priority neighbours
//               ((gain desc, id asc)) and moves when that gain is >= 0;
//               double-buffered part/lock arrays, part-weight deltas aggregated
//               per CTA in shared memory.
//   rebalance:  candidates (keys = source | loss bucket | id) are radix sorted,
//               exclusive prefix sums of vertex weight select the moves that
//               cover each source's excess and fit each destination's capacity
//               (weak) or the concatenated free capacities (strong).
#define GP_TU_ID 4   // site ids of the bounds-checked build
#include "gp_internal.cuh"

#include <cstring>
#include <mutex>

namespace gp {

constexpr int RT = 256;              // threads per CTA
constexpr int RW = RT / 32;          // warps per CTA
enum { MODE_LP = 0, MODE_RB = 1, MODE_EVAL = 2 };

__device__ __forceinline__ void argmax_q(uint64_t& bk, int32_t& bq, uint64_t k2, int32_t q2) {
    if (k2 > bk || (k2 == bk && (uint32_t)q2 < (uint32_t)bq)) { bk = k2; bq = q2; }
}
__device__ __forceinline__ void warp_argmax_q(uint64_t& bk, int32_t& bq) { group_argmax64(0xffffffffu, bk, bq); }
template <class T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Argmax over a lane group of (connectivity h > 0, part q): largest h, ties
// to the smaller q; h = 0 means "no candidate" and yields (0, -1).  Two
// redux.sync steps replace the shuffle tree (connectivities fit in 32 bits).
__device__ __forceinline__ void group_argmax_u32(uint32_t mask, uint64_t& bk, int32_t& bq, uint32_t h, int32_t q) {
    const uint32_t mh = __reduce_max_sync(mask, h);
    const uint32_t mq = __reduce_min_sync(mask, (h != 0u && h == mh) ? (uint32_t)q : 0xffffffffu);
    bk = mh;
    bq = mh ? (int32_t)mq : -1;
}
// group_argmax_u32 over aligned groups of TILE lanes (see tile_argmax64)
template <int TILE>
__device__ __forceinline__ void tile_argmax_u32(uint64_t& bk, int32_t& bq, uint32_t h, int32_t q) {
    if constexpr (TILE == 32) {
        group_argmax_u32(0xffffffffu, bk, bq, h, q);
    } else {
        uint32_t kq = h ? (uint32_t)q : 0xffffffffu;
#pragma unroll
        for (int o = TILE / 2; o > 0; o >>= 1) {
            const uint32_t h2 = __shfl_xor_sync(0xffffffffu, h, o), q2 = __shfl_xor_sync(0xffffffffu, kq, o);
            if (h2 > h || (h2 == h && q2 < kq)) { h = h2; kq = q2; }
        }
        bk = h;
        bq = h ? (int32_t)kq : -1;
    }
}
__device__ __forceinline__ void argmax_u32(uint32_t& bh, int32_t& bq, uint32_t h, int32_t q) {
    if (h > bh || (h == bh && (uint32_t)q < (uint32_t)bq)) { bh = h; bq = q; }
}

// LP candidate rule: gain >= 0, or -gain < own/den
__device__ __forceinline__ bool lp_candidate(int64_t g, int64_t own, int32_t den) {
    return g >= 0 || -g < own / den;
}

// ------------------------------------------------------------------ k_conn
// One unit of work per warp: 4 rows of bucket 0 (8 lanes each), or 1 row of
// bucket 1, or 1 row of bucket 2; rows longer than kHeavyDeg take CTAs
// [0, nheavy).  Buckets 0/1 keep their entries in registers: a bucket-0 lane
// sums the weights of its 8-lane tile's entries of the same part with seven
// shuffles, a bucket-1 row adds its entries into the warp's shared-memory
// histogram and reads its own part's bin back; bucket 2 and heavy rows build
// the whole shared-memory histogram.
// status: [S_CROSS] += directed cross weight; [S_MAXPW], [S_MODE], [S_LIGHT]
// written by CTA 0; LP candidates are appended to clist[bucket] (any order:
// each is evaluated on its own), with [S_NL0..S_NL2] their counts and
// [S_CDEG] the sum of their degrees.  Rebalance candidates are the vertices
// with dest >= 0; they are compacted in vertex order afterwards.
struct ConnArgs {
    DGraph g;
    int32_t k;
    int64_t Lmax;
    int32_t den;
    int force_eval;
    const int32_t* part;
    const uint8_t* lock;
    const int64_t* pw;
    const int32_t* heavy;
    const int32_t* item_row;
    const int64_t* item_beg;
    const int64_t* item_end;
    const int32_t* row_items;
    int64_t nitems;
    const int32_t* bucket[3];
    int64_t nbucket[3];
    const int64_t* wfirst;      // first light unit of each light warp, and the end (nw + 1)
    int32_t* dest;
    int32_t* gain;
    int32_t* part_next;         // label propagation: part and cleared lock copied here for the
    uint8_t* lock_next;         // move step (nullptr: not needed)
    const void* pc;             // the part array as gathered per neighbour: PT[n], a uint8 or uint16
                                // copy of part (k <= 256 / k <= 1024), or part itself (int32)
    void* pc_next;              // copy of part_next in the same type (nullptr: none kept)
    int64_t* status;
    int32_t* clist[3];
    int32_t* hhist;
    int64_t* hsum;
    int32_t* hdone;
    uint64_t* pdg;              // label propagation: pdg_pack(part, dest, gain) per row (nullptr: none)
};

// one word per vertex for the move step: part (bits 44-53), dest + 1 (bits
// 32-43; 0: no proposal) and gain (bits 0-31); k <= 1024
__device__ __forceinline__ uint64_t pdg_pack(int32_t p, int32_t d, int32_t g) {
    return ((uint64_t)(uint32_t)p << 44) | ((uint64_t)(uint32_t)(d + 1) << 32) | (uint64_t)(uint32_t)g;
}
__device__ __forceinline__ int32_t pdg_part(uint64_t x) { return (int32_t)((x >> 44) & 0x3FFu); }
__device__ __forceinline__ int32_t pdg_dest(uint64_t x) { return (int32_t)((x >> 32) & 0xFFFu) - 1; }
__device__ __forceinline__ int32_t pdg_gain(uint64_t x) { return (int32_t)(uint32_t)x; }

// part id of neighbour u from the gather copy (read-only in the kernel)
template <class PT>
__device__ __forceinline__ int32_t gpart(const void* pc, int32_t u, int64_t n) {
    return GP_IN(u, n) ? (int32_t)__ldg((const PT*)pc + u) : 0;
}

// rebalance moves keep the gather copy of part current (pcb bytes per id)
__device__ __forceinline__ void store_pc(void* pc, int pcb, int64_t v, int32_t d) {
    if (!pc) return;
    if (pcb == 1) ((uint8_t*)pc)[v] = (uint8_t)d;
    else ((uint16_t*)pc)[v] = (uint16_t)d;
}

__device__ __forceinline__ void hist_add(int32_t* hist, int32_t q, int32_t w, bool valid, int32_t k) {
    if (valid && GP_IN(q, k)) atomicAdd(&hist[q], w);
}

// warp-aggregated append of the lanes with take set
__device__ __forceinline__ void warp_push(bool take, int32_t v, int32_t* list, int64_t* count, int64_t cap) {
    const uint32_t m = __ballot_sync(0xffffffffu, take);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == __ffs(m) - 1) base = atomicAdd((unsigned long long*)count, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
    const int64_t idx = (int64_t)base + __popc(m & ((1u << lane) - 1u));
    if (take && GP_IN(idx, cap)) list[idx] = v;
}

// decision of one row from its best other part (bq, bk), own connectivity
// and total weighted degree; returns true when an LP candidate is recorded
template <class PT>
__device__ __forceinline__ bool conn_decide(const ConnArgs& A, int mode, bool active, int64_t v, int32_t p,
                                            int64_t tot, int64_t cross, uint64_t bk, int32_t bq, int32_t light) {
    if (mode == MODE_LP && A.part_next) {
        A.part_next[v] = p; A.lock_next[v] = 0;
        if (A.pc_next) ((PT*)A.pc_next)[v] = (PT)p;
    }
    const int64_t own = tot - cross;
    int32_t d = -1, gn = 0;
    bool cand = false;
    if (mode == MODE_LP) {
        if (active && bq >= 0) {
            const int64_t gg = (int64_t)bk - own;
            if (lp_candidate(gg, own, A.den)) { d = bq; gn = (int32_t)gg; cand = true; }
        }
    } else if (mode == MODE_RB && active) {
        const int64_t cd = bq >= 0 ? (int64_t)bk : 0;
        d = bq >= 0 ? bq : light;
        gn = -(int32_t)(own - cd);
    }
    A.dest[v] = d;
    A.gain[v] = gn;
    if (mode == MODE_LP && A.pdg) A.pdg[v] = pdg_pack(p, d, gn);
    return cand;
}

// one row of the connectivity pass: id (-1: none), entry range, part, and
// whether it looks for a move in this mode
struct ConnRow {
    int64_t beg, end;
    int32_t v, p;
    bool active;
};
__device__ __forceinline__ ConnRow conn_row(const ConnArgs& A, int64_t v, int mode, const uint8_t* over) {
    ConnRow r;
    r.v = (int32_t)v; r.beg = 0; r.end = 0; r.p = -1; r.active = false;
    if (v >= 0) {
        r.beg = A.g.rp[v]; r.end = A.g.rp[v + 1];
        r.p = A.part[v];
        r.active = (mode == MODE_LP && !A.lock[v]) || (mode == MODE_RB && over[r.p]);
    }
    return r;
}
// shared-memory copy of a ConnRow (pa: part, bit 31 = active)
struct ConnRowS {
    int64_t beg, end;
    int32_t v, pa;
};
__device__ __forceinline__ ConnRowS conn_stage(const ConnRow& r) {
    ConnRowS s;
    s.beg = r.beg; s.end = r.end; s.v = r.v;
    s.pa = (int32_t)((uint32_t)r.p | (r.active ? 0x80000000u : 0u));
    return s;
}
__device__ __forceinline__ ConnRow conn_unstage(const ConnRowS& s) {
    ConnRow r;
    r.beg = s.beg; r.end = s.end; r.v = s.v;
    r.p = s.v >= 0 ? (int32_t)((uint32_t)s.pa & 0x7fffffffu) : -1;
    r.active = s.v >= 0 && s.pa < 0;
    return r;
}
// the LP candidate list and its count slot of bucket b
__device__ __forceinline__ int64_t* conn_list_count(const ConnArgs& A, int b) {
    return &A.status[b == 0 ? S_NL0 : (b == 1 ? S_NL1 : S_NL2)];
}

// rows of at most TILE entries, TILE lanes per row, 32/TILE rows per warp.
// Every lane ends with the connectivity of the row to its entry's part; lanes
// of the same part hold the same value, which the argmax (ties to the smaller
// part) does not mind.  hist: the warp's k zeroed bins (TILE == 32 only; left
// zeroed).  Returns true on the row's first lane when the row is an LP
// candidate (the caller appends it).
template <int TILE, class PT>
__device__ __forceinline__ bool conn_tile(const ConnArgs& A, const ConnRow& R, int mode, const uint8_t* over,
                                          int32_t light, int32_t* hist, int64_t& acc) {
    const int lane = threadIdx.x & 31, tl = lane & (TILE - 1);
    const int64_t v = R.v, beg = R.beg, end = R.end;
    const int32_t p = R.p;
    const bool active = R.active;
    const int64_t e = beg + tl;
    const bool has = v >= 0 && e < end;
    int32_t q = -1, w = 0;
    if (has) { q = gpart<PT>(A.pc, __ldcs(&A.g.ci[e]), A.g.n); w = A.g.ew ? __ldcs(&A.g.ew[e]) : 1; }
    const int32_t cross = (int32_t)tile_sum_u32<TILE>((has && q != p) ? (uint32_t)w : 0u);
    const int32_t tot = (int32_t)tile_sum_u32<TILE>((uint32_t)w);
    uint32_t connq = 0;
    if constexpr (TILE == 32) {
        if (active) {  // one row per warp: uniform
            const bool in = has && q != p && GP_IN(q, A.k);   // the own part's bin is not needed
            if (in) atomicAdd(&hist[q], w);
            __syncwarp();
            if (in) connq = (uint32_t)hist[q];
            __syncwarp();
            if (in) hist[q] = 0;
            __syncwarp();
        }
    } else {
        const int32_t qk = has ? q : -1;
        connq = has ? (uint32_t)w : 0u;
#pragma unroll
        for (int d = 1; d < TILE; ++d) {
            const int src = (lane & ~(TILE - 1)) | ((tl + d) & (TILE - 1));
            const int32_t q2 = __shfl_sync(0xffffffffu, qk, src);
            const int32_t w2 = __shfl_sync(0xffffffffu, w, src);
            if (has && q2 == q) connq += (uint32_t)w2;
        }
    }
    uint64_t bk;
    int32_t bq;
    tile_argmax_u32<TILE>(bk, bq, (active && has && q != p && (mode != MODE_RB || !over[q])) ? connq : 0u, q);
    bool take = false;
    if (tl == 0 && v >= 0) {
        acc += cross;
        take = conn_decide<PT>(A, mode, active, v, p, tot, cross, bk, bq, light);
    }
    return take;
}

// bucket 2: one row per warp, shared-memory histogram.  The row is swept
// 128 entries at a time (4 independent loads per lane in flight).  The own
// part is never added (its connectivity is tot - cross), which keeps the
// most contended bin out of the shared-memory atomics.  For rows at least as
// long as k, or k <= kBinsK, the best part is taken over the k histogram bins,
// otherwise over the row's entries again (same candidates: parts with a
// non-zero connection).
constexpr int kBinsK = 256;
template <class PT>
__device__ __forceinline__ bool conn_warp(const ConnArgs& A, const ConnRow& R, int mode, const uint8_t* over,
                                          int32_t light, int32_t* hist, int64_t& acc) {
    const int lane = threadIdx.x & 31;
    const int64_t v = R.v, beg = R.beg, end = R.end;
    const int32_t p = R.p;
    const bool active = R.active;
    int32_t cross = 0, tot = 0;
    // 128 entries per sweep, four consecutive ones per lane (16-byte loads)
    const bool v4 = aligned16(A.g.ci) && aligned16(A.g.ew);
    for (int64_t base = beg & ~(int64_t)3; base < end; base += 128) {
        int32_t u[4], w[4], q[4];
        const int64_t e4 = base + 4 * lane;
        ld4_row(A.g.ci, e4, beg, end, v4, -1, u);
        if (A.g.ew) ld4_row(A.g.ew, e4, beg, end, v4, 0, w);
        else {
#pragma unroll
            for (int c = 0; c < 4; ++c) w[c] = u[c] >= 0 ? 1 : 0;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) q[c] = u[c] >= 0 ? gpart<PT>(A.pc, u[c], A.g.n) : -1;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            tot += w[c];
            if (q[c] >= 0 && q[c] != p) cross += w[c];
            if (active) hist_add(hist, q[c], w[c], q[c] >= 0 && q[c] != p, A.k);
        }
    }
    cross = (int32_t)__reduce_add_sync(0xffffffffu, (uint32_t)cross);
    tot = (int32_t)__reduce_add_sync(0xffffffffu, (uint32_t)tot);
    uint64_t bk = 0;
    int32_t bq = -1;
    if (active) {
        __syncwarp();
        uint32_t lh = 0;
        int32_t lq = -1;
        if (end - beg >= A.k || A.k <= kBinsK) {
            for (int q = lane; q < A.k; q += 32) {
                const int32_t h = hist[q];
                if (h > 0 && q != p && (mode != MODE_RB || !over[q])) argmax_u32(lh, lq, (uint32_t)h, q);
            }
            group_argmax_u32(0xffffffffu, bk, bq, lh, lq);
            __syncwarp();
            for (int q = lane; q < A.k; q += 32) hist[q] = 0;
        } else {
            for (int64_t e = beg + lane; e < end; e += 32) {
                const int32_t q = gpart<PT>(A.pc, __ldcs(&A.g.ci[e]), A.g.n);
                if (!GP_IN(q, A.k)) continue;
                if (q != p && (mode != MODE_RB || !over[q])) argmax_u32(lh, lq, (uint32_t)hist[q], q);
            }
            group_argmax_u32(0xffffffffu, bk, bq, lh, lq);
            __syncwarp();
            for (int64_t e = beg + lane; e < end; e += 32) {
                const int32_t q = gpart<PT>(A.pc, __ldcs(&A.g.ci[e]), A.g.n);
                if (GP_IN(q, A.k)) hist[q] = 0;
            }
        }
        __syncwarp();
    }
    bool take = false;
    if (lane == 0) {
        acc += cross;
        take = conn_decide<PT>(A, mode, active, v, p, tot, cross, bk, bq, light);
    }
    return take;
}

// append a row decided by conn_tile / conn_warp to list b at once
__device__ __forceinline__ void conn_push_now(const ConnArgs& A, bool take, const ConnRow& R, int b) {
    if (take) atomicAdd((unsigned long long*)&A.status[S_CDEG], (unsigned long long)(R.end - R.beg));
    warp_push(take, R.v, A.clist[b], conn_list_count(A, b), A.g.n);
}

template <class PT>
__global__ void __launch_bounds__(RT, 5) k_conn(ConnArgs A) {
    extern __shared__ int32_t csm[];
    const int32_t k = A.k;
    const int64_t Lmax = A.Lmax;
    const int kpad = (k + 15) & ~15;
    uint8_t* over = (uint8_t*)csm;
    int32_t* hist_all = csm + kpad / 4;
    __shared__ int64_t s_red[RW];
    __shared__ uint64_t s_k[RW];
    __shared__ int32_t s_q[RW];
    __shared__ int64_t s_maxpw;
    __shared__ int32_t s_light;
    __shared__ ConnRowS s_rows[RT];   // light warps: 32 staged rows each
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;

    // over flags, heaviest part, lightest non-overweight part (ties: lower id)
    int64_t mx = 0;
    uint64_t lk = 0; int32_t lq = -1;  // argmax of (~pw) == argmin pw
    for (int q = threadIdx.x; q < k; q += RT) {
        const int64_t x = A.pw[q];
        over[q] = x > Lmax;
        mx = x > mx ? x : mx;
        if (x <= Lmax) argmax_q(lk, lq, ~(uint64_t)x, q);
    }
    for (int i = threadIdx.x; i < RW * k; i += RT) hist_all[i] = 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) { int64_t y = __shfl_xor_sync(0xffffffffu, mx, o); mx = y > mx ? y : mx; }
    warp_argmax_q(lk, lq);
    if (lane == 0) { s_red[w] = mx; s_k[w] = lk; s_q[w] = lq; }
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t m2 = 0; uint64_t k2 = 0; int32_t q2 = -1;
        for (int i = 0; i < RW; ++i) { m2 = s_red[i] > m2 ? s_red[i] : m2; argmax_q(k2, q2, s_k[i], s_q[i]); }
        s_maxpw = m2; s_light = q2;
    }
    __syncthreads();
    const int64_t maxpw = s_maxpw;
    const int32_t light = s_light;
    const int mode = A.force_eval ? MODE_EVAL : (maxpw > Lmax ? MODE_RB : MODE_LP);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        A.status[S_MAXPW] = maxpw; A.status[S_MODE] = mode; A.status[S_LIGHT] = light;
    }
    int64_t acc = 0;  // directed cross weight (this thread)

    if ((int64_t)blockIdx.x < A.nitems) {
        // ---- one piece of a long row per CTA; pieces of the same row are
        // combined in global accumulators and the last CTA decides
        int32_t* hist = hist_all;
        const int32_t h = A.item_row[blockIdx.x];
        const int64_t v = A.heavy[h];
        const int nit = A.row_items[h];
        const int32_t p = A.part[v];
        const bool active = (mode == MODE_LP && !A.lock[v]) || (mode == MODE_RB && over[p]);
        const int64_t beg = A.item_beg[blockIdx.x], end = A.item_end[blockIdx.x];
        int64_t cross = 0, tot = 0;
        const bool v4 = aligned16(A.g.ci) && aligned16(A.g.ew);
        for (int64_t base = beg & ~(int64_t)3; base < end; base += 4 * RT) {
            int32_t uu[4], ww[4], qq[4];
            const int64_t e4 = base + 4 * threadIdx.x;
            ld4_row(A.g.ci, e4, beg, end, v4, -1, uu);
            if (A.g.ew) ld4_row(A.g.ew, e4, beg, end, v4, 0, ww);
            else {
#pragma unroll
                for (int c = 0; c < 4; ++c) ww[c] = uu[c] >= 0 ? 1 : 0;
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) qq[c] = uu[c] >= 0 ? gpart<PT>(A.pc, uu[c], A.g.n) : -1;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                tot += ww[c];
                if (qq[c] >= 0 && qq[c] != p) cross += ww[c];
                if (active) hist_add(hist, qq[c], ww[c], qq[c] >= 0 && qq[c] != p, k);
            }
        }
        cross = warp_sum(cross); tot = warp_sum(tot);
        acc += (lane == 0) ? cross : 0;  // the cut adds every piece
        __syncthreads();
        if (lane == 0) { s_red[w] = cross; s_k[w] = (uint64_t)tot; }
        __syncthreads();
        __shared__ int s_last;
        if (threadIdx.x == 0) {
            int64_t c2 = 0, t2 = 0;
            for (int i = 0; i < RW; ++i) { c2 += s_red[i]; t2 += (int64_t)s_k[i]; }
            s_red[0] = c2; s_k[0] = (uint64_t)t2;
            s_last = 1;
        }
        __syncthreads();
        if (nit > 1) {
            if (active)
                for (int q = threadIdx.x; q < k; q += RT)
                    if (hist[q]) atomicAdd(&A.hhist[(int64_t)h * k + q], hist[q]);
            if (threadIdx.x == 0) {
                atomicAdd((unsigned long long*)&A.hsum[2 * h], (unsigned long long)s_red[0]);
                atomicAdd((unsigned long long*)&A.hsum[2 * h + 1], (unsigned long long)s_k[0]);
            }
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) s_last = (atomicAdd(&A.hdone[h], 1) == nit - 1) ? 1 : 0;
            __syncthreads();
            if (s_last) {
                __threadfence();
                for (int q = threadIdx.x; q < k; q += RT) {
                    hist[q] = active ? __ldcg(&A.hhist[(int64_t)h * k + q]) : 0;
                    A.hhist[(int64_t)h * k + q] = 0;
                }
                if (threadIdx.x == 0) {
                    s_red[0] = (int64_t)__ldcg((const unsigned long long*)&A.hsum[2 * h]);
                    s_k[0] = (uint64_t)__ldcg((const unsigned long long*)&A.hsum[2 * h + 1]);
                    A.hsum[2 * h] = 0; A.hsum[2 * h + 1] = 0; A.hdone[h] = 0;
                }
                __syncthreads();
            }
        }
        if (s_last) {
            cross = s_red[0]; tot = (int64_t)s_k[0];
            __syncthreads();
            uint64_t bk = 0; int32_t bq = -1;
            if (active)
                for (int q = threadIdx.x; q < k; q += RT)
                    if (q != p && hist[q] > 0 && (mode != MODE_RB || !over[q])) argmax_q(bk, bq, (uint64_t)hist[q], q);
            warp_argmax_q(bk, bq);
            if (lane == 0) { s_k[w] = bk; s_q[w] = bq; }
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int i = 1; i < RW; ++i) argmax_q(bk, bq, s_k[i], s_q[i]);
                const int64_t rdeg = A.g.rp[v + 1] - A.g.rp[v];
                if (conn_decide<PT>(A, mode, active, v, p, tot, cross, bk, bq, light))
                    atomicAdd((unsigned long long*)&A.status[S_CDEG], (unsigned long long)rdeg);
            }
        }
    } else {
        int32_t* hist = hist_all + w * k;
        ConnRowS* rows = s_rows + w * 32;
        const int64_t wid = ((int64_t)(blockIdx.x - A.nitems) * RT + threadIdx.x) >> 5;
        const int64_t U2 = A.nbucket[2], U1 = A.nbucket[1];
        // contiguous units of equal total cost (k_warp_bounds), taken 8 at a
        // time: lane l first fetches row slot l (unit l / 4; its row, or the
        // (l % 4)-th row of a group of 4), so the list and row-header loads of
        // 8 units are in flight together; the candidates of the 8 units are
        // appended together afterwards (one atomic per list present)
        const int64_t u0 = A.wfirst[wid], u1 = A.wfirst[wid + 1];
        int64_t cdeg = 0;   // degree sum of this lane's candidates
        for (int64_t ub = u0; ub < u1; ub += 8) {
            const int nu = (int)(u1 - ub < 8 ? u1 - ub : 8);
            {
                const int64_t u = ub + (lane >> 2);
                const int sub = lane & 3;
                int64_t v = -1;
                if (u < ub + nu) {
                    if (u < U2) { if (sub == 0) v = A.bucket[2][u]; }
                    else if (u < U2 + U1) { if (sub == 0) v = A.bucket[1][u - U2]; }
                    else {
                        const int64_t i = (u - U2 - U1) * 4 + sub;
                        if (i < A.nbucket[0]) v = A.bucket[0][i];
                    }
                }
                rows[lane] = conn_stage(conn_row(A, v, mode, over));
            }
            __syncwarp();
            uint32_t takes = 0;   // bit s: row slot s is a candidate
            for (int j = 0; j < nu; ++j) {
                const int64_t u = ub + j;
                if (u < U2) {
                    const bool t = conn_warp<PT>(A, conn_unstage(rows[4 * j]), mode, over, light, hist, acc);
                    takes |= (__ballot_sync(0xffffffffu, t) & 1u) << (4 * j);
                } else if (u < U2 + U1) {
                    const bool t = conn_tile<kTile32, PT>(A, conn_unstage(rows[4 * j]), mode, over, light, hist, acc);
                    takes |= (__ballot_sync(0xffffffffu, t) & 1u) << (4 * j);
                } else {
                    const bool t = conn_tile<kTile8, PT>(A, conn_unstage(rows[4 * j + (lane >> 3)]), mode, over, light,
                                                         hist, acc);
                    const uint32_t b = __ballot_sync(0xffffffffu, t);   // lanes 0, 8, 16, 24
                    takes |= ((b & 1u) | ((b >> 7) & 2u) | ((b >> 14) & 4u) | ((b >> 21) & 8u)) << (4 * j);
                }
            }
            {
                const bool t = (takes >> lane) & 1u;
                const ConnRowS rs = rows[lane];
                const int64_t u = ub + (lane >> 2);
                const int lb = u < U2 ? 2 : (u < U2 + U1 ? 1 : 0);
                if (t) cdeg += rs.end - rs.beg;
#pragma unroll
                for (int b = 0; b < 3; ++b) warp_push(t && lb == b, rs.v, A.clist[b], conn_list_count(A, b), A.g.n);
            }
            __syncwarp();
        }
        cdeg = warp_sum(cdeg);
        if (lane == 0 && cdeg) atomicAdd((unsigned long long*)&A.status[S_CDEG], (unsigned long long)cdeg);
    }
    acc = warp_sum(acc);
    __syncthreads();
    if (lane == 0) s_red[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t s = 0;
        for (int i = 0; i < RW; ++i) s += s_red[i];
        if (s) atomicAdd((unsigned long long*)&A.status[S_CROSS], (unsigned long long)s);
    }
}

// ------------------------------------------------------------------ LP apply
template <class PT>
__device__ __forceinline__ int32_t ab_term(const DGraph& g, int64_t e, int64_t v, int32_t p, int32_t d, int32_t gv,
                                           const void* pc, const int32_t* __restrict__ dest,
                                           const int32_t* __restrict__ gain, const uint64_t* __restrict__ pdg) {
    const int32_t u = __ldcs(&g.ci[e]);
    if (!GP_IN(u, g.n)) return 0;
    int32_t pu, du, gu = 0;
    if (pdg) {
        const uint64_t x = pdg[u];
        pu = pdg_part(x); du = pdg_dest(x); gu = pdg_gain(x);
    } else {
        pu = gpart<PT>(pc, u, g.n);
        du = dest[u];
        if (du >= 0) gu = gain[u];
    }
    if (du >= 0 && (gu > gv || (gu == gv && u < (int32_t)v))) pu = du;
    const int32_t wt = g.ew ? __ldcs(&g.ew[e]) : 1;
    return pu == d ? wt : (pu == p ? -wt : 0);
}

struct ApplyArgs {
    DGraph g;
    int32_t k;
    const int32_t* part;
    const int32_t* dest;
    const int32_t* gain;
    const int32_t* heavy;
    const int32_t* item_row;
    const int64_t* item_beg;
    const int64_t* item_end;
    const int32_t* row_items;
    int64_t nitems;
    const int32_t* clist[3];
    const int64_t* status;
    int32_t* part_next;
    uint8_t* lock_next;
    const void* pc;             // gather copy of part (as in ConnArgs)
    void* pc_next;              // its copy of part_next (nullptr: none kept)
    int64_t* pw;
    int64_t* moves_out;
    int64_t* hsum;
    int32_t* hdone;
    const uint64_t* pdg;        // packed part / dest / gain of every vertex (nullptr: gather them apart)
};

template <class PT>
__device__ __forceinline__ void ab_commit(const ApplyArgs& A, int64_t v, int32_t p, int32_t d, int64_t* delta,
                                          int64_t& moves) {
    if (!GP_IN(d, A.k) || !GP_IN(p, A.k)) return;
    A.part_next[v] = d;
    if (A.pc_next) ((PT*)A.pc_next)[v] = (PT)d;
    A.lock_next[v] = 1;
    const int64_t wv = A.g.vw ? A.g.vw[v] : 1;
    atomicAdd((unsigned long long*)&delta[d], (unsigned long long)wv);
    atomicAdd((unsigned long long*)&delta[p], (unsigned long long)(-wv));
    ++moves;
}

// candidate rows of at most TILE entries, TILE lanes each
template <int TILE, class PT>
__device__ __forceinline__ void ab_tile(const ApplyArgs& A, int64_t v, int64_t* delta, int64_t& moves) {
    const int lane = threadIdx.x & 31, tl = lane & (TILE - 1);
    int32_t t = 0, p = -1, d = -1;
    if (v >= 0) {
        d = A.dest[v]; p = A.part[v];
        const int32_t gv = A.gain[v];
        const int64_t e = A.g.rp[v] + tl;
        if (e < A.g.rp[v + 1]) t = ab_term<PT>(A.g, e, v, p, d, gv, A.pc, A.dest, A.gain, A.pdg);
    }
#pragma unroll
    for (int o = TILE / 2; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (tl == 0 && v >= 0 && t >= 0) ab_commit<PT>(A, v, p, d, delta, moves);
}

// this thread's part (thread t of nt) of the ab_term sum over entries
// [beg, end) of row v: four consecutive entries at a time (16-byte loads),
// the four neighbours' part and destination gathers in flight together
template <class PT>
__device__ __forceinline__ int32_t ab_sum(const ApplyArgs& A, int64_t beg, int64_t end, int t, int nt, int64_t v,
                                          int32_t p, int32_t d, int32_t gv) {
    int32_t g2 = 0;
    const bool v4 = aligned16(A.g.ci) && aligned16(A.g.ew);
    for (int64_t base = beg & ~(int64_t)3; base < end; base += 4 * (int64_t)nt) {
        int32_t uu[4], ww[4], pu[4], du[4];
        const int64_t e4 = base + 4 * t;
        ld4_row(A.g.ci, e4, beg, end, v4, -1, uu);
        if (A.g.ew) ld4_row(A.g.ew, e4, beg, end, v4, 0, ww);
        else {
#pragma unroll
            for (int c = 0; c < 4; ++c) ww[c] = uu[c] >= 0 ? 1 : 0;
        }
        int32_t gu[4];
        if (A.pdg) {   // one gather per entry: part, dest and gain in one word
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const bool ok = uu[c] >= 0 && GP_IN(uu[c], A.g.n);
                const uint64_t x = ok ? A.pdg[uu[c]] : 0ull;
                pu[c] = ok ? pdg_part(x) : -1; du[c] = pdg_dest(x); gu[c] = pdg_gain(x);
            }
        } else {
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const bool ok = uu[c] >= 0 && GP_IN(uu[c], A.g.n);
                pu[c] = ok ? gpart<PT>(A.pc, uu[c], A.g.n) : -1;
                du[c] = ok ? A.dest[uu[c]] : -1;
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) gu[c] = du[c] >= 0 ? A.gain[uu[c]] : 0;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            if (uu[c] < 0 || pu[c] < 0) continue;
            int32_t q = pu[c];
            if (du[c] >= 0 && (gu[c] > gv || (gu[c] == gv && uu[c] < (int32_t)v))) q = du[c];
            g2 += q == d ? ww[c] : (q == p ? -ww[c] : 0);
        }
    }
    return g2;
}

// one candidate row of 33..heavy_deg entries per warp, 128 entries per sweep
template <class PT>
__device__ __forceinline__ void ab_warp(const ApplyArgs& A, int64_t v, int64_t* delta, int64_t& moves) {
    const int lane = threadIdx.x & 31;
    const int32_t d = A.dest[v], p = A.part[v], gv = A.gain[v];
    const int32_t g2 = warp_sum(ab_sum<PT>(A, A.g.rp[v], A.g.rp[v + 1], lane, 32, v, p, d, gv));
    if (lane == 0 && g2 >= 0) ab_commit<PT>(A, v, p, d, delta, moves);
}

template <class PT>
__global__ void __launch_bounds__(RT) k_lp_apply(ApplyArgs A) {
    extern __shared__ int64_t delta[];
    __shared__ int64_t s_red[RW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q = threadIdx.x; q < A.k; q += RT) delta[q] = 0;
    __syncthreads();
    int64_t moves = 0;
    if ((int64_t)blockIdx.x < A.nitems) {
        const int32_t h = A.item_row[blockIdx.x];
        const int64_t v = A.heavy[h];
        const int32_t d = A.dest[v];
        if (d >= 0) {
            const int nit = A.row_items[h];
            const int32_t p = A.part[v], gv = A.gain[v];
            int32_t g2 = ab_sum<PT>(A, A.item_beg[blockIdx.x], A.item_end[blockIdx.x], threadIdx.x, RT, v, p, d, gv);
            g2 = warp_sum(g2);
            if (lane == 0) s_red[w] = g2;
            __syncthreads();
            if (threadIdx.x == 0) {
                int64_t sum = 0;
                for (int i = 0; i < RW; ++i) sum += s_red[i];
                bool last = true;
                if (nit > 1) {
                    atomicAdd((unsigned long long*)&A.hsum[2 * h], (unsigned long long)sum);
                    __threadfence();
                    last = atomicAdd(&A.hdone[h], 1) == nit - 1;
                    if (last) {
                        __threadfence();
                        sum = (int64_t)__ldcg((const unsigned long long*)&A.hsum[2 * h]);
                        A.hsum[2 * h] = 0;
                        A.hdone[h] = 0;
                    }
                }
                if (last && sum >= 0) ab_commit<PT>(A, v, p, d, delta, moves);
            }
        }
    } else {
        const int64_t n0 = A.status[S_NL0], n1 = A.status[S_NL1], n2 = A.status[S_NL2];
        const int64_t U0 = (n0 + 3) / 4;
        const int64_t wid = ((int64_t)(blockIdx.x - A.nitems) * RT + threadIdx.x) >> 5;
        const int64_t nw = ((int64_t)(gridDim.x - A.nitems) * RT) >> 5;
        for (int64_t u = wid; u < U0 + n1 + n2; u += nw) {
            if (u < U0) {
                const int64_t i = u * 4 + (lane >> 3);
                ab_tile<kTile8, PT>(A, i < n0 ? A.clist[0][i] : -1, delta, moves);
            } else if (u < U0 + n1) {
                ab_tile<kTile32, PT>(A, A.clist[1][u - U0], delta, moves);
            } else {
                ab_warp<PT>(A, A.clist[2][u - U0 - n1], delta, moves);
            }
        }
    }
    moves = warp_sum(moves);
    __syncthreads();
    if (lane == 0 && moves) atomicAdd((unsigned long long*)A.moves_out, (unsigned long long)moves);
    for (int q = threadIdx.x; q < A.k; q += RT)
        if (delta[q]) atomicAdd((unsigned long long*)&A.pw[q], (unsigned long long)delta[q]);
}

// ------------------------------------------------------------------ rebalance
__global__ void k_gather_vw(int64_t cnt, const int32_t* __restrict__ vidx, const int32_t* __restrict__ vw,
                            int32_t* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = vw ? vw[vidx[i]] : 1;
}

constexpr int RB_SHIFT = 10;   // key = segment << 10 | loss bucket

__global__ void k_rb_flags(int64_t n, const int32_t* __restrict__ dest, int32_t* __restrict__ flag) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        flag[v] = dest[v] >= 0 ? 1 : 0;
}

// candidates in vertex order with key (source << 10 | bucket(loss))
__global__ void k_rb_compact(int64_t n, const int32_t* __restrict__ flag, const int64_t* __restrict__ pos,
                             const int32_t* __restrict__ part, const int32_t* __restrict__ gain,
                             uint64_t* __restrict__ keys, int32_t* __restrict__ vals) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        if (!flag[v]) continue;
        const int64_t i = pos[v];
        keys[i] = ((uint64_t)(uint32_t)part[v] << RB_SHIFT) | loss_bucket(-gain[v]);
        vals[i] = (int32_t)v;
    }
}

__device__ __forceinline__ int64_t seg_start(const uint64_t* keys, int64_t i, uint64_t seg) {
    int64_t lo = 0, hi = i;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if ((keys[mid] >> RB_SHIFT) < seg) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// first index of every key segment (key >> RB_SHIFT = d, d = 0..k) of a
// sorted candidate list: k + 1 searches instead of one per candidate
__global__ void k_seg_first(int64_t cnt, const uint64_t* __restrict__ keys, int32_t k, int64_t* __restrict__ first) {
    for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d <= k; d += (int64_t)gridDim.x * blockDim.x)
        first[d] = seg_start(keys, cnt, (uint64_t)d);
}

// flag[i] = 1 when the move keeps its source within the excess prefix
__global__ void k_rb_source(int64_t cnt, const uint64_t* __restrict__ keys, const int64_t* __restrict__ segf,
                            const int64_t* __restrict__ pre, const int64_t* __restrict__ pw, int64_t Lmax,
                            int32_t* __restrict__ flag) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t src = keys[i] >> RB_SHIFT;
        const int64_t s = segf[src];
        flag[i] = (pre[i] - pre[s]) < (pw[src] - Lmax) ? 1 : 0;
    }
}

// weak: accepted moves, in list order, re-keyed by (dest << 10 | bucket)
__global__ void k_rb_rekey(int64_t cnt, const uint64_t* __restrict__ keys, const int32_t* __restrict__ vals,
                           const int32_t* __restrict__ flag, const int64_t* __restrict__ pos,
                           const int32_t* __restrict__ dest, uint64_t* __restrict__ keys2, int32_t* __restrict__ vals2) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        if (!flag[i]) continue;
        const int32_t v = vals[i];
        const int64_t j = pos[i];
        keys2[j] = ((uint64_t)(uint32_t)dest[v] << RB_SHIFT) | (keys[i] & ((1ull << RB_SHIFT) - 1));
        vals2[j] = v;
    }
}

// part-weight changes and moves of a block, added to the global totals once
// per part (dynamic shared memory: k int64)
__device__ __forceinline__ void rb_delta_begin(int64_t* delta, int32_t k) {
    for (int q = threadIdx.x; q < k; q += blockDim.x) delta[q] = 0;
    __syncthreads();
}
__device__ __forceinline__ void rb_delta_end(int64_t* delta, int32_t k, int64_t nmoves, int64_t* __restrict__ pw,
                                             int64_t* __restrict__ moves) {
    for (int o = 16; o > 0; o >>= 1) nmoves += __shfl_xor_sync(0xffffffffu, nmoves, o);
    if ((threadIdx.x & 31) == 0 && nmoves) atomicAdd((unsigned long long*)moves, (unsigned long long)nmoves);
    __syncthreads();
    for (int q = threadIdx.x; q < k; q += blockDim.x)
        if (delta[q]) atomicAdd((unsigned long long*)&pw[q], (unsigned long long)delta[q]);
}

// weak: keep moves whose destination prefix fits the capacity; apply
__global__ void k_rb_weak_apply(int64_t cnt, const uint64_t* __restrict__ keys, const int64_t* __restrict__ segf,
                                const int32_t* __restrict__ vals, const int64_t* __restrict__ pre,
                                const int32_t* __restrict__ vw, const int64_t* __restrict__ pw_snap, int64_t Lmax,
                                int32_t k, int32_t* __restrict__ part, void* pc, int pcb, uint8_t* __restrict__ lock,
                                int64_t* __restrict__ pw, int64_t* __restrict__ moves) {
    extern __shared__ int64_t rb_delta[];
    rb_delta_begin(rb_delta, k);
    int64_t nm = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t d = keys[i] >> RB_SHIFT;
        const int64_t s = segf[d];
        const int32_t v = vals[i];
        const int64_t wv = vw ? vw[v] : 1;
        if ((pre[i] - pre[s]) + wv <= Lmax - pw_snap[d]) {
            const int32_t p = part[v];
            part[v] = (int32_t)d; lock[v] = 1;
            store_pc(pc, pcb, v, (int32_t)d);
            if (GP_IN(d, k) && GP_IN(p, k)) {
                atomicAdd((unsigned long long*)&rb_delta[d], (unsigned long long)wv);
                atomicAdd((unsigned long long*)&rb_delta[p], (unsigned long long)(-wv));
            }
            ++nm;
        }
    }
    rb_delta_end(rb_delta, k, nm, pw, moves);
}

// strong: cumulative free capacity of non-overweight parts
__global__ void k_cumfree(int32_t k, const int64_t* __restrict__ pw, int64_t Lmax, int64_t* __restrict__ cum) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int64_t s = 0;
    cum[0] = 0;
    for (int q = 0; q < k; ++q) {
        const int64_t x = pw[q];
        s += (x > Lmax) ? 0 : (Lmax - x);
        cum[q + 1] = s;
    }
}

__global__ void k_mask_vw(int64_t cnt, const int32_t* __restrict__ flag, const int32_t* __restrict__ wvals,
                          int32_t* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = flag[i] ? wvals[i] : 0;
}

__global__ void k_rb_strong_apply(int64_t cnt, const int32_t* __restrict__ vals, const int32_t* __restrict__ flag,
                                  const int64_t* __restrict__ P, const int32_t* __restrict__ vw,
                                  const int64_t* __restrict__ cum, int32_t k, int32_t* __restrict__ part,
                                  void* pc, int pcb, uint8_t* __restrict__ lock, int64_t* __restrict__ pw,
                                  int64_t* __restrict__ moves) {
    extern __shared__ int64_t rb_delta[];
    rb_delta_begin(rb_delta, k);
    int64_t nm = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        if (!flag[i]) continue;
        const int64_t pre = P[i];
        if (pre >= cum[k]) continue;
        // q with cum[q] <= pre < cum[q+1]: last index with cum <= pre
        int lo = 0, hi = k;  // search in cum[0..k]
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (cum[mid] <= pre) lo = mid; else hi = mid - 1;
        }
        const int q = lo;
        const int32_t v = vals[i];
        const int64_t wv = vw ? vw[v] : 1;
        if (q < k && pre + wv <= cum[q + 1]) {
            const int32_t p = part[v];
            part[v] = q; lock[v] = 1;
            store_pc(pc, pcb, v, q);
            if (GP_IN(p, k)) {
                atomicAdd((unsigned long long*)&rb_delta[q], (unsigned long long)wv);
                atomicAdd((unsigned long long*)&rb_delta[p], (unsigned long long)(-wv));
            }
            ++nm;
        }
    }
    rb_delta_end(rb_delta, k, nm, pw, moves);
}

// ------------------------------------------------------------------ projection, weights, cut
__global__ void k_project(int64_t n, const int32_t* __restrict__ cmap, const int32_t* __restrict__ pc,
                          int32_t* __restrict__ pf) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        pf[v] = pc[cmap[v]];
}

__global__ void k_part_weights(int64_t n, const int32_t* __restrict__ part, const int32_t* __restrict__ vw, int32_t k,
                               int64_t* __restrict__ pw) {
    extern __shared__ int64_t spw[];
    for (int q = threadIdx.x; q < k; q += blockDim.x) spw[q] = 0;
    __syncthreads();
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        atomicAdd((unsigned long long*)&spw[part[v]], (unsigned long long)(vw ? vw[v] : 1));
    __syncthreads();
    for (int q = threadIdx.x; q < k; q += blockDim.x)
        if (spw[q]) atomicAdd((unsigned long long*)&pw[q], (unsigned long long)spw[q]);
}

// warp per row: directed cross weight (d_cross2 accumulates 2*cut)
// directed cross weight, entry-sliced (csr_row_of / csr_window_lane): each
// lane of a window also holds its row's part; eight groups of 32 entries have
// their column ids loaded, then their neighbours' parts gathered, together
__global__ void __launch_bounds__(RT) k_cut(DGraph g, int64_t slice, const int32_t* __restrict__ part,
                                            int64_t* __restrict__ cross2) {
    __shared__ int64_t s_red[RW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t wid = ((int64_t)blockIdx.x * RT + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * RT) >> 5;
    const int64_t n = g.n, m = g.m, nslice = (m + slice - 1) / slice;
    int64_t acc = 0;
    for (int64_t sl = wid; sl < nslice; sl += nw) {
        const int64_t o0 = sl * slice, o1 = o0 + slice < m ? o0 + slice : m;
        int64_t cb = csr_row_of(g.rp, n, o0), s = 0, wend = 0;
        int32_t pv = 0;
        auto window = [&]() {
            const int64_t r = cb + lane;
            s = r < n ? g.rp[r] : m;
            pv = r < n ? part[r] : 0;
            wend = g.rp[cb + 32 < n ? cb + 32 : n];
        };
        window();
        int64_t o = o0;
        while (o < o1) {
            const int64_t lim = o1 < wend ? o1 : wend;
            if (o + 256 <= lim) {
                int32_t u[8], pr[8], wt[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int64_t oi = o + 32 * q + lane;
                    pr[q] = __shfl_sync(0xffffffffu, pv, csr_window_lane(s, oi));
                    u[q] = __ldcs(&g.ci[oi]);
                    wt[q] = g.ew ? __ldcs(&g.ew[oi]) : 1;
                }
#pragma unroll
                for (int q = 0; q < 8; ++q) u[q] = GP_IN(u[q], n) ? part[u[q]] : pr[q];
#pragma unroll
                for (int q = 0; q < 8; ++q) acc += u[q] != pr[q] ? wt[q] : 0;
                o += 256;
            } else if (o < lim) {
                const int64_t oi = o + lane;
                const int32_t p = __shfl_sync(0xffffffffu, pv, csr_window_lane(s, oi));
                if (oi < lim) {
                    const int32_t u = __ldcs(&g.ci[oi]);
                    if (GP_IN(u, n) && part[u] != p) acc += g.ew ? __ldcs(&g.ew[oi]) : 1;
                }
                o = o + 32 < lim ? o + 32 : lim;
            } else {
                cb += 32;   // o >= wend: o lies in a later row
                window();
            }
        }
    }
    acc = warp_sum(acc);
    if (lane == 0) s_red[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t s = 0;
        for (int i = 0; i < RW; ++i) s += s_red[i];
        if (s) atomicAdd((unsigned long long*)cross2, (unsigned long long)s);
    }
}

void project(Ctx& c, const Level& fine, const int32_t* part_coarse, int32_t* part_fine) {
    k_project<<<grid_for(fine.g.n, 256), 256, 0, c.s>>>(fine.g.n, fine.cmap, part_coarse, part_fine);
    GP_LAUNCHED(c);
    c.bytes += 12 * fine.g.n;
}

void part_weights(Ctx& c, const DGraph& g, const int32_t* part, int32_t k, int64_t* pw) {
    memset_async(c, pw, 0, sizeof(int64_t) * k);
    k_part_weights<<<grid_for(g.n, 256, c.sm_count * 4), 256, sizeof(int64_t) * k, c.s>>>(g.n, part, g.vw, k, pw);
    GP_LAUNCHED(c);
    c.bytes += 4 * g.n + (g.vw ? 4 * g.n : 0);
}

void cut_and_weights(Ctx& c, const DGraph& g, const int32_t* part, int32_t k, int64_t* d_cross2, int64_t* d_pw) {
    memset_async(c, d_cross2, 0, sizeof(int64_t));
    const int64_t slice = csr_slice(g.m, c.sm_count);
    k_cut<<<grid_for((g.m + slice - 1) / slice * 32, RT, c.sm_count * c.ctas_per_sm), RT, 0, c.s>>>(g, slice, part,
                                                                                                   d_cross2);
    GP_LAUNCHED(c);
    c.bytes += 8 * (g.n + 1) + 8 * g.m + (g.ew ? 4 * g.m : 0) + 4 * g.n;
    if (d_pw) part_weights(c, g, part, k, d_pw);
}

// ------------------------------------------------------------------ one-CTA refinement
// A level with at most small_level_n (<= kCtaMaxN) vertices and no row longer
// than kHeavyDeg is refined by one thread block in one launch: the whole
// iteration loop of refine_level (connectivity pass, label propagation with
// afterburner, weak/strong rebalancing, best-state tracking and the stop
// rules) runs on the device, with the same per-row helpers as the
// multi-kernel path and the same integer results.  Rebalance candidates are
// sorted by a bitonic network in shared memory on unique 64-bit keys
// (source, loss bucket, id), then (destination, loss bucket, source, id).
constexpr int CT = 1024, CW = CT / 32;
constexpr int64_t kCtaMaxN = 16384;                 // candidates sorted in shared memory (8 B each)

struct CtaRefineArgs {
    DGraph g;
    int32_t k;
    int64_t Lmax;
    int32_t den, max_iters, patience, strong_after;
    const int32_t* bucket[3];
    int64_t nbucket[3];
    int32_t* part;
    int32_t* part_next;
    uint8_t* lock;
    uint8_t* lock_next;
    int32_t* best;
    int64_t* pw;          // in: part weights of part; out: those of the kept state
    int32_t* dest;
    int32_t* gain;
    int64_t* status;      // counters of the per-row helpers
    int32_t* clist[3];
    int64_t* pre;         // n scratch
    int32_t* flag;        // n scratch
    uint64_t* gkeys;      // n scratch
    int32_t* tr_arrays;   // optional: per step dest[n], gain[n], part[n]
    int64_t* tr_scalars;  // optional: per step mode, cut before, max part weight before, moves
    int64_t* out;         // [0] steps
};

__device__ __forceinline__ int64_t cta_sum(int64_t x, int64_t* sh) {
    int64_t tot;
    block_excl_scan<int64_t>(x, sh, tot);
    return tot;
}

// exclusive prefix sums of val(i), i < cnt, in index order into out; returns the total
template <class F>
__device__ int64_t cta_scan(int64_t cnt, F val, int64_t* out, int64_t* sh) {
    const int64_t per = (cnt + CT - 1) / CT;
    const int64_t b = (int64_t)threadIdx.x * per, e = b + per < cnt ? b + per : cnt;
    int64_t s = 0;
    for (int64_t i = b; i < e; ++i) s += val(i);
    int64_t tot;
    int64_t base = block_excl_scan<int64_t>(s, sh, tot);
    for (int64_t i = b; i < e; ++i) { const int64_t x = val(i); out[i] = base; base += x; }
    __syncthreads();
    return tot;
}

// ascending bitonic sort of N (a power of two) unique keys in shared memory.
// Compare-exchange steps whose partner is within 16 positions run on
// registers with warp shuffles (element i sits in lane i % 32 of its warp,
// partner i ^ stride in the same warp); wider steps go through shared memory,
// one block barrier each.
__device__ void cta_bitonic(uint64_t* a, int N) {
    const int tid = threadIdx.x;
    const int E = N > CT ? N / CT : 1;
    // strides top, top/2, ..., 1 of merge size `size` (size 0: every size 2..top*2)
    auto warp_steps = [&](int size, int top) {
        for (int e = 0; e < E; ++e) {
            const int i = e * CT + tid;
            const bool valid = i < N;
            uint64_t x = valid ? a[i] : ~0ull;
            const int s0 = size ? size : 2, s1 = size ? size : 2 * top;
            for (int sz = s0; sz <= s1; sz <<= 1) {
                for (int stride = size ? top : (sz >> 1); stride > 0; stride >>= 1) {
                    const uint64_t y = __shfl_xor_sync(0xffffffffu, x, stride);
                    const bool up = (i & sz) == 0, lower = (i & stride) == 0;
                    x = (lower == up) ? (x < y ? x : y) : (x < y ? y : x);
                }
            }
            if (valid) a[i] = x;
        }
        __syncthreads();
    };
    // merge sizes up to 32: within warps
    warp_steps(0, (N < 32 ? N : 32) >> 1);
    for (int size = 64; size <= N; size <<= 1) {
        for (int stride = size >> 1; stride >= 32; stride >>= 1) {
            for (int i = tid; i < N; i += CT) {
                const int j = i ^ stride;
                if (j > i) {
                    const uint64_t x = a[i], y = a[j];
                    const bool up = (i & size) == 0;
                    if ((x > y) == up) { a[i] = y; a[j] = x; }
                }
            }
            __syncthreads();
        }
        warp_steps(size, 16);
    }
}

// first index in [0, i] whose key has the same segment (key >> shift) as key i
__device__ __forceinline__ int cta_seg_start(const uint64_t* a, int i, int shift) {
    const uint64_t seg = a[i] >> shift;
    int lo = 0, hi = i;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((a[mid] >> shift) < seg) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// One rebalance step by one thread block (the rules of the multi-kernel path
// below: candidates ordered (source, loss bucket, id); a source keeps the
// prefix before the vertex below its excess; weak: per destination, ordered
// (destination, loss bucket, source, id), moves that fit the remaining
// capacity; strong: kept moves laid over the concatenated free capacities).
// cand: the candidates in vertex order (ncand of them), or nullptr to take
// every v < n with dest[v] >= 0.  s_pw (shared) is updated; returns this
// thread's move count.  Needs ncand <= kCtaMaxN.
struct RbCta {
    const int32_t* vw;
    int32_t* part;
    void* pc;                   // gather copy of part to keep current (nullptr: none)
    int pcb;                    // its bytes per id
    uint8_t* lock;
    const int32_t* dest;
    const int32_t* gain;
    int64_t* pre;
    int32_t* flag;
    uint64_t* gkeys;
    int32_t k;
    int64_t Lmax;
};

__device__ int64_t cta_rebalance(const RbCta& R, int mode, int64_t n, const int32_t* cand, int64_t ncand_in,
                                 int64_t* s_pw, int64_t* s_snap, int64_t* s_cum, uint64_t* s_keys, int64_t* sh) {
    const int32_t k = R.k;
    const int64_t Lmax = R.Lmax;
    int32_t* part = R.part;
    uint8_t* lock = R.lock;
    int64_t moves = 0;
    for (int q = threadIdx.x; q < k; q += CT) s_snap[q] = s_pw[q];
    __syncthreads();
    int64_t ncand = ncand_in;
    auto key1 = [&](uint32_t v) -> uint64_t {
        const uint64_t key = ((uint64_t)(uint32_t)part[v] << RB_SHIFT) | loss_bucket(-R.gain[v]);
        return (key << 32) | v;
    };
    if (cand == nullptr) {
        // candidates in vertex order, then sorted by (source, loss bucket, id)
        ncand = cta_scan(n, [&](int64_t v) -> int64_t { return R.dest[v] >= 0 ? 1 : 0; }, R.pre, sh);
        for (int64_t v = threadIdx.x; v < n; v += CT)
            if (R.dest[v] >= 0) s_keys[R.pre[v]] = key1((uint32_t)v);
    } else {
        for (int64_t i = threadIdx.x; i < ncand; i += CT) s_keys[i] = key1((uint32_t)cand[i]);
    }
    int N = 1;
    while (N < ncand) N <<= 1;
    for (int64_t i = ncand + threadIdx.x; i < N; i += CT) s_keys[i] = ~0ull;
    __syncthreads();
    cta_bitonic(s_keys, N);
    auto vwt = [&](uint32_t v) -> int64_t { return R.vw ? R.vw[v] : 1; };
    cta_scan(ncand, [&](int64_t i) -> int64_t { return vwt((uint32_t)s_keys[i]); }, R.pre, sh);
    // kept: the source's prefix before the vertex is below its excess
    for (int64_t i = threadIdx.x; i < ncand; i += CT) {
        const uint32_t src = (uint32_t)(s_keys[i] >> (32 + RB_SHIFT));
        const int s0 = cta_seg_start(s_keys, (int)i, 32 + RB_SHIFT);
        R.flag[i] = (R.pre[i] - R.pre[s0]) < (s_snap[src] - Lmax) ? 1 : 0;
    }
    __syncthreads();
    if (mode == 1) {
        // kept moves re-keyed (dest, loss bucket, source, id): 10 + 10 + 10 + 32 bits
        const int64_t n2 = cta_scan(ncand, [&](int64_t i) -> int64_t { return R.flag[i]; }, R.pre, sh);
        for (int64_t i = threadIdx.x; i < ncand; i += CT)
            if (R.flag[i]) {
                const uint64_t key = s_keys[i];
                const uint32_t v = (uint32_t)key, b = (uint32_t)(key >> 32) & ((1u << RB_SHIFT) - 1);
                const uint32_t src = (uint32_t)(key >> (32 + RB_SHIFT));
                R.gkeys[R.pre[i]] = ((((uint64_t)(uint32_t)R.dest[v] << RB_SHIFT | b) << RB_SHIFT | src) << 32) | v;
            }
        __syncthreads();
        int N2 = 1;
        while (N2 < n2) N2 <<= 1;
        for (int64_t i = threadIdx.x; i < N2; i += CT) s_keys[i] = i < n2 ? R.gkeys[i] : ~0ull;
        __syncthreads();
        cta_bitonic(s_keys, N2);
        cta_scan(n2, [&](int64_t i) -> int64_t { return vwt((uint32_t)s_keys[i]); }, R.pre, sh);
        for (int64_t i = threadIdx.x; i < n2; i += CT) {
            const uint32_t v = (uint32_t)s_keys[i];
            const int32_t d = (int32_t)(s_keys[i] >> (32 + 2 * RB_SHIFT));
            const int s0 = cta_seg_start(s_keys, (int)i, 32 + 2 * RB_SHIFT);
            const int64_t wv = vwt(v);
            if ((R.pre[i] - R.pre[s0]) + wv <= Lmax - s_snap[d]) {
                const int32_t p = part[v];
                part[v] = d; lock[v] = 1;
                store_pc(R.pc, R.pcb, v, d);
                atomicAdd((unsigned long long*)&s_pw[d], (unsigned long long)wv);
                atomicAdd((unsigned long long*)&s_pw[p], (unsigned long long)(-wv));
                ++moves;
            }
        }
    } else {
        // free capacities of the parts within Lmax, concatenated (k <= CT)
        {
            const int64_t f = (threadIdx.x < k && s_snap[threadIdx.x] <= Lmax) ? Lmax - s_snap[threadIdx.x] : 0;
            int64_t tot;
            const int64_t ex = block_excl_scan<int64_t>(f, sh, tot);
            if (threadIdx.x < k) s_cum[threadIdx.x] = ex;
            if (threadIdx.x == 0) s_cum[k] = tot;
            __syncthreads();
        }
        cta_scan(ncand, [&](int64_t i) -> int64_t { return R.flag[i] ? vwt((uint32_t)s_keys[i]) : 0; }, R.pre, sh);
        for (int64_t i = threadIdx.x; i < ncand; i += CT) {
            if (!R.flag[i]) continue;
            const int64_t pre = R.pre[i];
            if (pre >= s_cum[k]) continue;
            int lo = 0, hi = k;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (s_cum[mid] <= pre) lo = mid; else hi = mid - 1;
            }
            const uint32_t v = (uint32_t)s_keys[i];
            const int64_t wv = vwt(v);
            if (lo < k && pre + wv <= s_cum[lo + 1]) {
                const int32_t p = part[v];
                part[v] = lo; lock[v] = 1;
                store_pc(R.pc, R.pcb, v, lo);
                atomicAdd((unsigned long long*)&s_pw[lo], (unsigned long long)wv);
                atomicAdd((unsigned long long*)&s_pw[p], (unsigned long long)(-wv));
                ++moves;
            }
        }
    }
    __syncthreads();
    return moves;
}

// one rebalance step of the multi-kernel loop in one launch: candidates from
// dest (n <= kCtaMaxN, locks cleared here) or from a compacted list; part
// weights in and out of global memory; the step's moves added to *moves_out
__global__ void __launch_bounds__(CT, 1) k_rb_step_cta(RbCta R, int mode, int64_t n, const int32_t* cand,
                                                        int64_t ncand, int64_t* pw, int64_t* moves_out) {
    extern __shared__ __align__(16) unsigned char rsm[];
    const int32_t k = R.k;
    int64_t* s_pw = (int64_t*)rsm;
    int64_t* s_snap = s_pw + k;
    int64_t* s_cum = s_snap + 2 * k;
    uint64_t* s_keys = (uint64_t*)(rsm + (((size_t)(4 * k + 1) * 8 + k + 15) & ~(size_t)15));
    __shared__ int64_t sh[33];
    for (int q = threadIdx.x; q < k; q += CT) s_pw[q] = pw[q];
    if (cand == nullptr)
        for (int64_t v = threadIdx.x; v < n; v += CT) R.lock[v] = 0;
    __syncthreads();
    const int64_t moves = cta_sum(cta_rebalance(R, mode, n, cand, ncand, s_pw, s_snap, s_cum, s_keys, sh), sh);
    for (int q = threadIdx.x; q < k; q += CT) pw[q] = s_pw[q];
    if (threadIdx.x == 0) *moves_out += moves;
}

// the whole refinement loop of one level by one block of CT threads; rsm:
// cta_refine_smem(k) bytes of dynamic shared memory
__device__ void cta_refine_level(const CtaRefineArgs& R, unsigned char* rsm) {
    const int32_t k = R.k;
    const int64_t Lmax = R.Lmax, n = R.g.n;
    int64_t* s_pw = (int64_t*)rsm;               // k: current part weights
    int64_t* s_snap = s_pw + k;                  // k: weights at the start of a rebalance step
    int64_t* s_best = s_snap + k;                // k: weights of the kept state
    int64_t* s_cum = s_best + k;                 // k + 1: free capacity prefix (strong)
    uint8_t* s_over = (uint8_t*)(s_cum + k + 1); // k
    unsigned char* big = rsm + (((size_t)(4 * k + 1) * 8 + k + 15) & ~(size_t)15);
    int32_t* s_hist = (int32_t*)big;             // CW * k connectivity histograms, or
    uint64_t* s_keys = (uint64_t*)big;           // up to kCtaMaxN sort keys
    __shared__ int64_t sh[33];
    __shared__ uint64_t s_lk[CW];
    __shared__ int32_t s_lq[CW];
    __shared__ int64_t s_mx[CW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t* part = R.part;
    int32_t* part_next = R.part_next;
    uint8_t* lock = R.lock;
    uint8_t* lock_next = R.lock_next;
    for (int q = threadIdx.x; q < k; q += CT) s_pw[q] = R.pw[q];
    for (int64_t v = threadIdx.x; v < n; v += CT) lock[v] = 0;
    __syncthreads();
    int64_t best_cut = 0, best_mp = 0, prev_moves = -1, nmoves = 0;
    int stall = 0, rb_streak = 0, steps = 0, last_mode = 0;
    const int64_t U2 = R.nbucket[2], U1 = R.nbucket[1], U0 = (R.nbucket[0] + 3) / 4;
    for (int it = 0;; ++it) {
        const bool final_eval = it == R.max_iters;
        // ---- part-weight summary (as k_conn's prologue)
        int64_t mx = 0;
        uint64_t lk = 0; int32_t lq = -1;
        for (int q = threadIdx.x; q < k; q += CT) {
            const int64_t x = s_pw[q];
            s_over[q] = x > Lmax;
            mx = x > mx ? x : mx;
            if (x <= Lmax) argmax_q(lk, lq, ~(uint64_t)x, q);
        }
        for (int i = threadIdx.x; i < CW * k; i += CT) s_hist[i] = 0;
        if (threadIdx.x < S_NRESET) R.status[threadIdx.x] = 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) { const int64_t y = __shfl_xor_sync(0xffffffffu, mx, o); mx = y > mx ? y : mx; }
        warp_argmax_q(lk, lq);
        if (lane == 0) { s_mx[w] = mx; s_lk[w] = lk; s_lq[w] = lq; }
        __syncthreads();
        int64_t maxpw = 0; uint64_t lk2 = 0; int32_t light = -1;
        for (int i = 0; i < CW; ++i) { maxpw = s_mx[i] > maxpw ? s_mx[i] : maxpw; argmax_q(lk2, light, s_lk[i], s_lq[i]); }
        const int dmode = final_eval ? MODE_EVAL : (maxpw > Lmax ? MODE_RB : MODE_LP);
        // ---- connectivity pass
        ConnArgs CA;
        CA.g = R.g; CA.k = k; CA.Lmax = Lmax; CA.den = R.den; CA.force_eval = final_eval ? 1 : 0;
        CA.part = part; CA.lock = lock; CA.pw = s_pw; CA.heavy = nullptr; CA.item_row = nullptr;
        CA.item_beg = nullptr; CA.item_end = nullptr; CA.row_items = nullptr; CA.nitems = 0;
        for (int b = 0; b < 3; ++b) { CA.bucket[b] = R.bucket[b]; CA.nbucket[b] = R.nbucket[b]; CA.clist[b] = R.clist[b]; }
        CA.wfirst = nullptr;
        CA.dest = R.dest; CA.gain = R.gain; CA.status = R.status;
        CA.part_next = nullptr; CA.lock_next = nullptr;
        CA.pc = part; CA.pc_next = nullptr; CA.pdg = nullptr;
        CA.hhist = nullptr; CA.hsum = nullptr; CA.hdone = nullptr;
        int64_t acc = 0;
        int32_t* hist = s_hist + w * k;
        for (int64_t u = w; u < U2 + U1 + U0; u += CW) {
            if (u < U2) {
                const ConnRow r = conn_row(CA, R.bucket[2][u], dmode, s_over);
                conn_push_now(CA, conn_warp<int32_t>(CA, r, dmode, s_over, light, hist, acc), r, 2);
            } else if (u < U2 + U1) {
                const ConnRow r = conn_row(CA, R.bucket[1][u - U2], dmode, s_over);
                conn_push_now(CA, conn_tile<kTile32, int32_t>(CA, r, dmode, s_over, light, hist, acc), r, 1);
            } else {
                const int64_t i = (u - U2 - U1) * 4 + (lane >> 3);
                const ConnRow r = conn_row(CA, i < R.nbucket[0] ? R.bucket[0][i] : -1, dmode, s_over);
                conn_push_now(CA, conn_tile<kTile8, int32_t>(CA, r, dmode, s_over, light, hist, acc), r, 0);
            }
        }
        acc = warp_sum(acc);
        const int64_t cur_cut = cta_sum(lane == 0 ? acc : 0, sh) / 2;   // also orders the pass
        const int64_t cur_mp = maxpw;
        // ---- best state and stop rules (every thread holds the same values)
        if (it == 0) {
            best_cut = cur_cut; best_mp = cur_mp;
            for (int64_t v = threadIdx.x; v < n; v += CT) R.best[v] = part[v];
            for (int q = threadIdx.x; q < k; q += CT) s_best[q] = s_pw[q];
        } else {
            const bool cb = cur_mp <= Lmax, bb = best_mp <= Lmax;
            bool better = false, signif = false;
            if (cb && !bb) { better = true; signif = true; }
            else if (cb && bb) { better = cur_cut < best_cut; signif = 1000 * cur_cut < 999 * best_cut; }
            else if (!cb && !bb) { better = cur_mp < best_mp || (cur_mp == best_mp && cur_cut < best_cut); signif = cur_mp < best_mp; }
            if (better) {
                best_cut = cur_cut; best_mp = cur_mp;
                for (int64_t v = threadIdx.x; v < n; v += CT) R.best[v] = part[v];
                for (int q = threadIdx.x; q < k; q += CT) s_best[q] = s_pw[q];
            }
            stall = signif ? 0 : stall + 1;
            const bool lp_idle = (last_mode == 0 && nmoves == 0 && prev_moves == 0);
            prev_moves = nmoves;
            bool rb_stuck = false;
            if (last_mode != 0 && nmoves == 0) {
                if (last_mode == 1) rb_streak = R.strong_after; else rb_stuck = true;
            }
            if (stall >= R.patience || lp_idle || rb_stuck) break;
        }
        if (final_eval) break;
        int mode;
        if (dmode == MODE_RB) { mode = (rb_streak >= R.strong_after) ? 2 : 1; ++rb_streak; }
        else { mode = 0; rb_streak = 0; }
        last_mode = mode;
        int64_t moves = 0;
        __syncthreads();
        if (mode == 0) {
            for (int64_t v = threadIdx.x; v < n; v += CT) { part_next[v] = part[v]; lock_next[v] = 0; }
            __syncthreads();
            ApplyArgs AA;
            AA.g = R.g; AA.k = k; AA.part = part; AA.dest = R.dest; AA.gain = R.gain; AA.heavy = nullptr;
            AA.item_row = nullptr; AA.item_beg = nullptr; AA.item_end = nullptr; AA.row_items = nullptr; AA.nitems = 0;
            for (int b = 0; b < 3; ++b) AA.clist[b] = R.clist[b];
            AA.status = R.status; AA.part_next = part_next; AA.lock_next = lock_next; AA.pw = nullptr;
            AA.pc = part; AA.pc_next = nullptr;
            AA.moves_out = nullptr; AA.hsum = nullptr; AA.hdone = nullptr; AA.pdg = nullptr;
            for (int64_t u = w; u < U2 + U1 + U0; u += CW) {
                if (u < U2) {
                    const int64_t v = R.bucket[2][u];
                    if (R.dest[v] >= 0) ab_warp<int32_t>(AA, v, s_pw, moves);
                } else if (u < U2 + U1) {
                    const int64_t v = R.bucket[1][u - U2];
                    ab_tile<kTile32, int32_t>(AA, R.dest[v] >= 0 ? v : -1, s_pw, moves);
                } else {
                    const int64_t i = (u - U2 - U1) * 4 + (lane >> 3);
                    const int64_t v = i < R.nbucket[0] ? R.bucket[0][i] : -1;
                    ab_tile<kTile8, int32_t>(AA, (v >= 0 && R.dest[v] >= 0) ? v : -1, s_pw, moves);
                }
            }
            nmoves = cta_sum(moves, sh);
            int32_t* tp = part; part = part_next; part_next = tp;
            uint8_t* tl = lock; lock = lock_next; lock_next = tl;
        } else {
            for (int64_t v = threadIdx.x; v < n; v += CT) lock[v] = 0;
            __syncthreads();
            RbCta RA;
            RA.vw = R.g.vw; RA.part = part; RA.pc = nullptr; RA.pcb = 0; RA.lock = lock; RA.dest = R.dest;
            RA.gain = R.gain; RA.pre = R.pre;
            RA.flag = R.flag; RA.gkeys = R.gkeys; RA.k = k; RA.Lmax = Lmax;
            moves = cta_rebalance(RA, mode, n, nullptr, 0, s_pw, s_snap, s_cum, s_keys, sh);
            nmoves = cta_sum(moves, sh);
        }
        if (R.tr_arrays) {
            int32_t* t = R.tr_arrays + (int64_t)steps * 3 * n;
            for (int64_t v = threadIdx.x; v < n; v += CT) { t[v] = R.dest[v]; t[n + v] = R.gain[v]; t[2 * n + v] = part[v]; }
            if (threadIdx.x == 0) {
                int64_t* sc = R.tr_scalars + 4 * steps;
                sc[0] = mode; sc[1] = cur_cut; sc[2] = cur_mp; sc[3] = nmoves;
            }
        }
        ++steps;
        __syncthreads();
    }
    __syncthreads();
    // the kept state
    for (int64_t v = threadIdx.x; v < n; v += CT) R.part[v] = R.best[v];
    for (int q = threadIdx.x; q < k; q += CT) R.pw[q] = s_best[q];
    if (threadIdx.x == 0) R.out[0] = steps;
}

__global__ void __launch_bounds__(CT, 1) k_refine_cta(CtaRefineArgs R) {
    extern __shared__ __align__(16) unsigned char rsm[];
    cta_refine_level(R, rsm);
}

// ------------------------------------------------------------------ batched one-block levels
// A chain is the run of one graph's levels, coarsest first, that one block
// refines (at most kCtaMaxN vertices, no row longer than kHeavyDeg).  The
// persistent kernel k_refine_chains takes chains from a device work queue (an
// atomic ticket over the chains, ordered by cost, largest first) and, for
// each level of the chain, projects the coarser level's partition and runs
// the level's whole refinement loop, with no host round trip between
// levels or iterations.  Chains are independent, so no block ever waits for
// another.
struct ChainItem {
    CtaRefineArgs R;          // R.part receives the projected partition
    const int32_t* cmap;      // fine -> coarse map of this level (nullptr: coarsest level, no projection)
    const int32_t* pcoarse;   // refined partition of the next coarser level
};

__global__ void __launch_bounds__(CT, 1) k_refine_chains(const int32_t* __restrict__ chain_first,
                                                         const int32_t* __restrict__ chain_len, int32_t nchains,
                                                         const ChainItem* __restrict__ items, int32_t* ticket) {
    extern __shared__ __align__(16) unsigned char rsm[];
    __shared__ int32_t s_chain;
    for (;;) {
        if (threadIdx.x == 0) s_chain = atomicAdd(ticket, 1);
        __syncthreads();
        const int32_t ch = s_chain;
        __syncthreads();
        if (ch >= nchains) return;
        for (int32_t t = 0; t < chain_len[ch]; ++t) {
            const ChainItem& it = items[chain_first[ch] + t];
            if (it.cmap)
                for (int64_t v = threadIdx.x; v < it.R.g.n; v += CT) it.R.part[v] = it.pcoarse[it.cmap[v]];
            __syncthreads();
            cta_refine_level(it.R, rsm);
            __syncthreads();
        }
    }
}

static size_t cta_refine_smem(int32_t k) {
    const size_t head = (((size_t)(4 * k + 1) * 8 + k + 15) & ~(size_t)15);
    const size_t hist = sizeof(int32_t) * CW * (size_t)k, keys = sizeof(uint64_t) * kCtaMaxN;
    return head + (hist > keys ? hist : keys);
}

void refine_smem_caps() {
    GP_CUDA(cudaFuncSetAttribute(k_refine_cta, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cta_refine_smem(GP_MAX_K)));
    GP_CUDA(cudaFuncSetAttribute(k_rb_step_cta, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cta_refine_smem(GP_MAX_K)));
    GP_CUDA(cudaFuncSetAttribute(k_refine_chains, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cta_refine_smem(GP_MAX_K)));
}

static bool cta_refine_ok(const Level& L, const Params& P) {
    const int64_t lim = std::min<int64_t>(P.o.small_level_n, kCtaMaxN);
    return P.o.small_level_n > 0 && L.nheavy == 0 && L.g.n <= lim && P.k <= GP_MAX_K;
}

static int refine_level_cta(Ctx& c, const Level& L, const Params& P, RefineBufs& B, int level, const Tracer& tr) {
    const DGraph& g = L.g;
    const int64_t n = g.n;
    auto mk = c.tmp->save();
    CtaRefineArgs R;
    R.g = g; R.k = P.k; R.Lmax = P.Lmax; R.den = P.o.lp_filter_den; R.max_iters = P.o.refine_max_iters;
    R.patience = P.o.refine_patience; R.strong_after = P.o.strong_after;
    for (int b = 0; b < 3; ++b) { R.bucket[b] = L.bucket[b]; R.nbucket[b] = L.nbucket[b]; R.clist[b] = B.clist[b]; }
    R.part = B.part; R.part_next = B.part_next; R.lock = B.lock; R.lock_next = B.lock_next; R.best = B.best;
    R.pw = B.pw; R.dest = B.dest; R.gain = B.gain; R.status = B.status;
    R.pre = c.tmp_alloc<int64_t>(n);
    R.flag = c.tmp_alloc<int32_t>(n);
    R.gkeys = c.tmp_alloc<uint64_t>(n);
    R.tr_arrays = nullptr; R.tr_scalars = nullptr;
    if (tr.on()) {
        R.tr_arrays = c.tmp_alloc<int32_t>((int64_t)P.o.refine_max_iters * 3 * n);
        R.tr_scalars = c.tmp_alloc<int64_t>((int64_t)P.o.refine_max_iters * 4);
    }
    R.out = c.tmp_alloc<int64_t>(1);
    k_refine_cta<<<1, CT, cta_refine_smem(P.k), c.s>>>(R);
    GP_LAUNCHED(c);
    const int steps = (int)read_i64(c, R.out);
    // each step: one connectivity pass plus its move step; one closing pass
    c.bytes += (int64_t)(steps + 1) * (L.scan_bytes() + 13 * n) + (int64_t)steps * (9 * n + 16 * n);
    if (tr.on() && steps > 0) {
        std::vector<int32_t> arr((size_t)steps * 3 * n);
        std::vector<int64_t> sc((size_t)steps * 4);
        GP_CUDA(cudaMemcpyAsync(arr.data(), R.tr_arrays, sizeof(int32_t) * arr.size(), cudaMemcpyDeviceToHost, c.s));
        GP_CUDA(cudaMemcpyAsync(sc.data(), R.tr_scalars, sizeof(int64_t) * sc.size(), cudaMemcpyDeviceToHost, c.s));
        c.sync();
        for (int it = 0; it < steps; ++it) {
            gp_trace_event ev;
            memset(&ev, 0, sizeof ev);
            ev.kind = GP_TR_REFINE_ITER; ev.level = level; ev.iter = it; ev.mode = (int32_t)sc[4 * it];
            ev.n = n; ev.m = g.m; ev.cut = sc[4 * it + 1]; ev.maxpw = sc[4 * it + 2]; ev.count = sc[4 * it + 3];
            int32_t* base = arr.data() + (size_t)it * 3 * n;
            ev.a0 = base; ev.a1 = base + n; ev.a2 = base + 2 * n;
            tr.emit(ev);
        }
    }
    c.tmp->restore(mk);
    return steps;
}

static bool chain_level_ok(const Level& L, const Params& P) {
    return L.nheavy == 0 && L.g.n <= kCtaMaxN && P.k <= GP_MAX_K;
}

struct ChainBatch {
    std::mutex mu;
    std::vector<ChainItem> items;
    struct Rec { VState* S; int32_t first, len; int64_t cost; };
    std::vector<Rec> chains;
    int32_t kmax = 2;
};

ChainBatch* chain_batch_new() { return new ChainBatch(); }
void chain_batch_delete(ChainBatch* cb) { delete cb; }

int chain_add(Ctx& c, ChainBatch* cb, VState& S) {
    const Params& P = S.P;
    if (P.k <= 1 || S.refined_to != S.L + 1) return 0;
    int s = S.L + 1;
    while (s > 0 && chain_level_ok(S.lv[s - 1], P)) --s;
    const int len = S.L + 1 - s;
    if (len == 0) return 0;
    int64_t nmax = 1, cost = 0;
    for (int l = s; l <= S.L; ++l) { nmax = std::max(nmax, S.lv[l].g.n); cost += S.lv[l].g.n + S.lv[l].g.m; }
    RefineBufs& B = S.B;
    int64_t* pre = c.keep_alloc<int64_t>(nmax);
    int32_t* flag = c.keep_alloc<int32_t>(nmax);
    uint64_t* gkeys = c.keep_alloc<uint64_t>(nmax);
    std::vector<ChainItem> mine((size_t)len);
    for (int t = 0; t < len; ++t) {
        const int l = S.L - t;
        const Level& L = S.lv[l];
        ChainItem& it = mine[t];
        CtaRefineArgs& R = it.R;
        R.g = L.g; R.k = P.k; R.Lmax = P.Lmax; R.den = P.o.lp_filter_den; R.max_iters = P.o.refine_max_iters;
        R.patience = P.o.refine_patience; R.strong_after = P.o.strong_after;
        for (int b = 0; b < 3; ++b) { R.bucket[b] = L.bucket[b]; R.nbucket[b] = L.nbucket[b]; R.clist[b] = B.clist[b]; }
        // the partition alternates between the two part buffers level by level
        int32_t* cur = (t & 1) ? B.part_next : B.part;
        int32_t* other = (t & 1) ? B.part : B.part_next;
        R.part = cur; R.part_next = other; R.lock = B.lock; R.lock_next = B.lock_next; R.best = B.best;
        R.pw = B.pw; R.dest = B.dest; R.gain = B.gain; R.status = B.status;
        R.pre = pre; R.flag = flag; R.gkeys = gkeys;
        R.tr_arrays = nullptr; R.tr_scalars = nullptr;
        R.out = nullptr;   // set by chain_run
        it.cmap = t == 0 ? nullptr : L.cmap;
        it.pcoarse = other;
    }
    std::lock_guard<std::mutex> lk(cb->mu);
    cb->chains.push_back({&S, (int32_t)cb->items.size(), (int32_t)len, cost});
    cb->items.insert(cb->items.end(), mine.begin(), mine.end());
    cb->kmax = std::max(cb->kmax, P.k);
    return len;
}

void chain_run(Ctx& c, ChainBatch* cb) {
    const int32_t nch = (int32_t)cb->chains.size();
    if (nch == 0) return;
    // largest chains first
    std::vector<int32_t> order((size_t)nch);
    for (int32_t i = 0; i < nch; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return cb->chains[a].cost > cb->chains[b].cost; });
    std::vector<int32_t> hfirst((size_t)nch), hlen((size_t)nch);
    for (int32_t i = 0; i < nch; ++i) { hfirst[i] = cb->chains[order[i]].first; hlen[i] = cb->chains[order[i]].len; }
    auto mk = c.tmp->save();
    const int64_t ni = (int64_t)cb->items.size();
    ChainItem* d_items = (ChainItem*)c.tmp->alloc(sizeof(ChainItem) * (size_t)ni);
    int32_t* d_first = c.tmp_alloc<int32_t>(nch);
    int32_t* d_len = c.tmp_alloc<int32_t>(nch);
    int32_t* d_ticket = c.tmp_alloc<int32_t>(1);
    int64_t* d_steps = c.tmp_alloc<int64_t>(ni);
    for (int64_t i = 0; i < ni; ++i) cb->items[i].R.out = d_steps + i;
    GP_CUDA(cudaMemcpyAsync(d_items, cb->items.data(), sizeof(ChainItem) * (size_t)ni, cudaMemcpyHostToDevice, c.s));
    GP_CUDA(cudaMemcpyAsync(d_first, hfirst.data(), sizeof(int32_t) * nch, cudaMemcpyHostToDevice, c.s));
    GP_CUDA(cudaMemcpyAsync(d_len, hlen.data(), sizeof(int32_t) * nch, cudaMemcpyHostToDevice, c.s));
    memset_async(c, d_ticket, 0, sizeof(int32_t));
    const size_t smem = cta_refine_smem(cb->kmax);
    int per_sm = 1;
    GP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_refine_chains, CT, smem));
    const int grid = (int)std::min<int64_t>(nch, (int64_t)std::max(per_sm, 1) * c.sm_count);
    k_refine_chains<<<grid, CT, smem, c.s>>>(d_first, d_len, nch, d_items, d_ticket);
    GP_LAUNCHED(c);
    // steps of every level; the partition ends in the buffer of the last level
    std::vector<int64_t> steps((size_t)ni);
    GP_CUDA(cudaMemcpyAsync(steps.data(), d_steps, sizeof(int64_t) * (size_t)ni, cudaMemcpyDeviceToHost, c.s));
    c.sync();
    c.tmp->restore(mk);
    for (auto& rec : cb->chains) {
        VState& S = *rec.S;
        for (int t = 0; t < rec.len; ++t) {
            const Level& L = S.lv[S.L - t];
            const int64_t n = L.g.n;
            const int64_t st = steps[rec.first + t];
            S.iters += (int)st;
            S.bytes += (st + 1) * (L.scan_bytes() + 13 * n) + st * (9 * n + 16 * n) + (t ? 12 * n : 0);
        }
        if ((rec.len - 1) & 1) std::swap(S.B.part, S.B.part_next);
        S.refined_to = S.L + 1 - rec.len;
    }
}

// ------------------------------------------------------------------ level controller
static int bits_for(int64_t x) {
    int b = 1;
    while ((1ll << b) < x) ++b;
    return b;
}

static void trace_iter(Ctx& c, const RefineBufs& B, int64_t n, int64_t m, int level, int it, int mode,
                       int64_t cut_before, int64_t mp_before, const Tracer& tr) {
    std::vector<int32_t> d(n), gn(n), p(n);
    GP_CUDA(cudaMemcpyAsync(d.data(), B.dest, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c.s));
    GP_CUDA(cudaMemcpyAsync(gn.data(), B.gain, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c.s));
    GP_CUDA(cudaMemcpyAsync(p.data(), B.part, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c.s));
    GP_CUDA(cudaMemcpyAsync(c.h_pinned, B.status + S_STEP_MOVES, sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
    c.sync();
    gp_trace_event ev;
    memset(&ev, 0, sizeof ev);
    ev.kind = GP_TR_REFINE_ITER; ev.level = level; ev.iter = it; ev.mode = mode;
    ev.n = n; ev.m = m; ev.cut = cut_before; ev.maxpw = mp_before; ev.count = c.h_pinned[0];
    ev.a0 = d.data(); ev.a1 = gn.data(); ev.a2 = p.data();
    tr.emit(ev);
}

// the part array as the neighbour gathers read it: 1 or 2 bytes per vertex
__global__ void k_compact_part(int64_t n, const int32_t* __restrict__ part, void* pc, int pcb) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        store_pc(pc, pcb, v, part[v]);
}

int64_t conn_max_warps(const Ctx& c) { return (int64_t)c.sm_count * c.ctas_per_sm * RW; }

// light warp t of a connectivity pass over nw warps takes the units
// [first unit with cost prefix >= T * t / nw, the same for t + 1), T the total
// cost: contiguous ranges of equal cost, the same for every pass of a level
__global__ void k_warp_bounds(const int64_t* __restrict__ cost, int64_t nunits, int64_t nw,
                              int64_t* __restrict__ out) {
    const int64_t T = cost[nunits];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= nw; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t target = (T * t) / nw;
        int64_t lo = 0, hi = nunits;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (cost[mid] < target) lo = mid + 1; else hi = mid;
        }
        out[t] = lo;
    }
}

int refine_level(Ctx& c, const Level& L, const Params& P, RefineBufs& B, int level, const Tracer& tr) {
    if (cta_refine_ok(L, P)) return refine_level_cta(c, L, P, B, level, tr);
    const DGraph& g = L.g;
    const int64_t n = g.n;
    const int32_t k = P.k;
    const int64_t Lmax = P.Lmax;
    memset_async(c, B.lock, 0, n);
    // neighbour gathers read a uint8 (k <= 256) or uint16 copy of part, kept
    // current by every step that moves vertices: a quarter or half of the
    // bytes per gather, and of the array that has to stay in L2
    B.pcb = k <= 256 ? 1 : 2;
    k_compact_part<<<grid_for(n, 256), 256, 0, c.s>>>(n, B.part, B.pc, B.pcb);
    GP_LAUNCHED(c);
    c.bytes += 4 * n + B.pcb * n;
    const int kpad = (k + 15) & ~15;
    const size_t conn_smem = kpad + sizeof(int32_t) * RW * k;
    // at most 1024 + 32 * GP_MAX_K bytes: below the 48 KB default, no attribute needed
    const int light_blocks = (int)std::min<int64_t>(grid_for(n * 32, RT, c.sm_count * c.ctas_per_sm),
                                                    (B.wfirst_cap - 1) / RW);
    const int grid = (int)L.nitems + light_blocks;
    {
        const int64_t nw = (int64_t)light_blocks * RW;
        k_warp_bounds<<<grid_for(nw + 1, 256), 256, 0, c.s>>>(L.unit_cost, L.nunits, nw, B.wfirst);
        GP_LAUNCHED(c);
    }
    int64_t best_cut = 0, best_mp = 0;
    int stall = 0, rb_streak = 0, steps = 0, last_mode = 0;
    int64_t prev_moves = -1;
    const int nb_k = bits_for(k);
    for (int it = 0;; ++it) {
        const bool final_eval = (it == P.o.refine_max_iters);
        GP_CUDA(cudaMemsetAsync(B.status, 0, sizeof(int64_t) * S_NRESET, c.s));
        if (c.profile) GP_CUDA(cudaEventRecord(c.ev_a, c.s));
        ConnArgs CA;
        CA.g = g; CA.k = k; CA.Lmax = Lmax; CA.den = P.o.lp_filter_den; CA.force_eval = final_eval ? 1 : 0;
        CA.part = B.part; CA.lock = B.lock; CA.pw = B.pw; CA.heavy = L.heavy;
        CA.item_row = L.item_row; CA.item_beg = L.item_beg; CA.item_end = L.item_end; CA.row_items = L.row_items;
        CA.nitems = L.nitems; CA.hhist = B.hhist; CA.hsum = B.hsum; CA.hdone = B.hdone;
        for (int b = 0; b < 3; ++b) { CA.bucket[b] = L.bucket[b]; CA.nbucket[b] = L.nbucket[b]; CA.clist[b] = B.clist[b]; }
        CA.wfirst = B.wfirst;
        CA.dest = B.dest; CA.gain = B.gain; CA.status = B.status;
        CA.part_next = B.part_next; CA.lock_next = B.lock_next;   // the LP step's starting copy
        CA.pc = B.pc; CA.pc_next = B.pc_next; CA.pdg = B.pdg;
        if (B.pcb == 1) k_conn<uint8_t><<<grid, RT, conn_smem, c.s>>>(CA);
        else k_conn<uint16_t><<<grid, RT, conn_smem, c.s>>>(CA);
        GP_LAUNCHED(c);
        if (c.profile) GP_CUDA(cudaEventRecord(c.ev_b, c.s));
        // rowptr, colidx, weights, gathered part[u] (pcb bytes); part[v], lock[v] read; dest, gain written
        const int64_t conn_bytes = L.scan_bytes() - (4 - B.pcb) * g.m + 4 * n + n + 8 * n;
        c.bytes += conn_bytes;
        GP_CUDA(cudaMemcpyAsync(c.h_pinned, B.status, sizeof(int64_t) * S_NSLOTS, cudaMemcpyDeviceToHost, c.s));
        c.sync();
        if (c.profile) {
            float t = 0;
            GP_CUDA(cudaEventElapsedTime(&t, c.ev_a, c.ev_b));
            c.ms_conn += t;
            c.conn_launches += 1;
            c.conn_bytes += conn_bytes;
        }
        const int64_t cur_cut = c.h_pinned[S_CROSS] / 2;
        const int64_t cur_mp = c.h_pinned[S_MAXPW];
        const int dev_mode = (int)c.h_pinned[S_MODE];
        const int64_t nlist = c.h_pinned[S_NL0] + c.h_pinned[S_NL1] + c.h_pinned[S_NL2];
        const int64_t cdeg = c.h_pinned[S_CDEG];
        if (it == 0) {
            best_cut = cur_cut; best_mp = cur_mp;
            GP_CUDA(cudaMemcpyAsync(B.best, B.part, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, c.s));
            GP_CUDA(cudaMemcpyAsync(B.best_pw, B.pw, sizeof(int64_t) * k, cudaMemcpyDeviceToDevice, c.s));
        } else {
            const int64_t nmoves = c.h_pinned[S_STEP_MOVES];
            const bool cb = cur_mp <= Lmax, bb = best_mp <= Lmax;
            bool better = false, signif = false;
            if (cb && !bb) { better = true; signif = true; }
            else if (cb && bb) { better = cur_cut < best_cut; signif = 1000 * cur_cut < 999 * best_cut; }
            else if (!cb && !bb) { better = cur_mp < best_mp || (cur_mp == best_mp && cur_cut < best_cut); signif = cur_mp < best_mp; }
            if (better) {
                best_cut = cur_cut; best_mp = cur_mp;
                GP_CUDA(cudaMemcpyAsync(B.best, B.part, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, c.s));
                GP_CUDA(cudaMemcpyAsync(B.best_pw, B.pw, sizeof(int64_t) * k, cudaMemcpyDeviceToDevice, c.s));
            }
            stall = signif ? 0 : stall + 1;
            const bool lp_idle = (last_mode == 0 && nmoves == 0 && prev_moves == 0);
            prev_moves = nmoves;
            // a rebalance step that moved nothing: weak escalates to strong, strong ends the level
            bool rb_stuck = false;
            if (last_mode != 0 && nmoves == 0) {
                if (last_mode == 1) rb_streak = P.o.strong_after; else rb_stuck = true;
            }
            if (stall >= P.o.refine_patience || lp_idle || rb_stuck) break;
        }
        if (final_eval) break;
        int mode;
        if (dev_mode == MODE_RB) { mode = (rb_streak >= P.o.strong_after) ? 2 : 1; ++rb_streak; }
        else { mode = 0; rb_streak = 0; }
        last_mode = mode;
        int64_t* moves_d = B.status + S_STEP_MOVES;  // moves of this step, read at the next sync
        memset_async(c, moves_d, 0, sizeof(int64_t));
        if (mode == 0) {
            // part_next / lock_next were filled by the connectivity pass
            ApplyArgs AA;
            AA.g = g; AA.k = k; AA.part = B.part; AA.dest = B.dest; AA.gain = B.gain; AA.heavy = L.heavy;
            AA.item_row = L.item_row; AA.item_beg = L.item_beg; AA.item_end = L.item_end; AA.row_items = L.row_items;
            AA.nitems = L.nitems; AA.hsum = B.hsum; AA.hdone = B.hdone;
            for (int b = 0; b < 3; ++b) AA.clist[b] = B.clist[b];
            AA.status = B.status; AA.part_next = B.part_next; AA.lock_next = B.lock_next; AA.pw = B.pw;
            AA.moves_out = moves_d;
            AA.pc = B.pc; AA.pc_next = B.pc_next; AA.pdg = B.pdg;
            if (B.mp && P.gnn && gnn_has_move_head(P.gnn)) {
                // learned order of the afterburner: (move priority, id) instead of (gain, id)
                gnn_move_priorities(c, P.gnn, g, level, B.dest, B.gain, B.mp);
                AA.gain = B.mp;
                AA.pdg = nullptr;   // the packed words hold the gains
                if (tr.on()) {
                    std::vector<int32_t> hm((size_t)n);
                    GP_CUDA(cudaMemcpyAsync(hm.data(), B.mp, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c.s));
                    c.sync();
                    gp_trace_event ev;
                    memset(&ev, 0, sizeof ev);
                    ev.kind = GP_TR_MOVE_PRIO; ev.level = level; ev.iter = it; ev.n = n; ev.m = g.m;
                    ev.a0 = hm.data();
                    tr.emit(ev);
                }
            }
            if (B.pcb == 1) k_lp_apply<uint8_t><<<grid, RT, sizeof(int64_t) * k, c.s>>>(AA);
            else k_lp_apply<uint16_t><<<grid, RT, sizeof(int64_t) * k, c.s>>>(AA);
            GP_LAUNCHED(c);
            // copy pass + afterburner: candidate rows with gathered part (pcb bytes), dest and gain per entry
            c.bytes += (9 + B.pcb) * n + 16 * nlist + cdeg * (4 + (g.ew ? 4 : 0) + 8 + B.pcb);
            std::swap(B.part, B.part_next);
            std::swap(B.lock, B.lock_next);
            std::swap(B.pc, B.pc_next);
        } else if (n <= kCtaMaxN) {
            // the whole step in one thread block
            auto mk = c.tmp->save();
            RbCta RA;
            RA.vw = g.vw; RA.part = B.part; RA.pc = B.pc; RA.pcb = B.pcb; RA.lock = B.lock; RA.dest = B.dest;
            RA.gain = B.gain;
            RA.pre = c.tmp_alloc<int64_t>(n); RA.flag = c.tmp_alloc<int32_t>(n); RA.gkeys = c.tmp_alloc<uint64_t>(n);
            RA.k = k; RA.Lmax = Lmax;
            k_rb_step_cta<<<1, CT, cta_refine_smem(k), c.s>>>(RA, mode, n, nullptr, 0, B.pw, moves_d);
            GP_LAUNCHED(c);
            c.bytes += 4 * n + 12 * n + 80 * n;
            c.tmp->restore(mk);
        } else {
            memset_async(c, B.lock, 0, n);
            auto mk = c.tmp->save();
            // candidates (dest >= 0) in vertex order, keyed (source, bucket); stable sort -> (source, bucket, id)
            int32_t* flag = c.tmp_alloc<int32_t>(n);
            int64_t* vpos = c.tmp_alloc<int64_t>(n + 1);
            k_rb_flags<<<grid_for(n, 256), 256, 0, c.s>>>(n, B.dest, flag);
            GP_LAUNCHED(c);
            scan_excl_i32_to_i64(c, flag, vpos, n, vpos + n);
            const int64_t ncand = read_i64(c, vpos + n);
            c.bytes += 4 * n + 12 * n;
            if (ncand > 0 && ncand <= kCtaMaxN) {
                // few candidates: sort, select and apply in one thread block
                k_rb_compact<<<grid_for(n, 256), 256, 0, c.s>>>(n, flag, vpos, B.part, B.gain, B.ckeys, B.cvals);
                GP_LAUNCHED(c);
                RbCta RA;
                RA.vw = g.vw; RA.part = B.part; RA.pc = B.pc; RA.pcb = B.pcb; RA.lock = B.lock; RA.dest = B.dest;
                RA.gain = B.gain;
                RA.pre = c.tmp_alloc<int64_t>(ncand); RA.flag = c.tmp_alloc<int32_t>(ncand);
                RA.gkeys = c.tmp_alloc<uint64_t>(ncand); RA.k = k; RA.Lmax = Lmax;
                k_rb_step_cta<<<1, CT, cta_refine_smem(k), c.s>>>(RA, mode, n, B.cvals, ncand, B.pw, moves_d);
                GP_LAUNCHED(c);
                c.bytes += 80 * ncand;
            } else if (ncand > 0) {
                k_rb_compact<<<grid_for(n, 256), 256, 0, c.s>>>(n, flag, vpos, B.part, B.gain, B.ckeys, B.cvals);
                GP_LAUNCHED(c);
                const int bits = RB_SHIFT + nb_k;
                radix_sort_pairs(c, B.ckeys, B.cvals, B.ckeys2, B.cvals2, ncand, bits);
                int32_t* wv = c.tmp_alloc<int32_t>(ncand);
                int64_t* pre = c.tmp_alloc<int64_t>(ncand + 1);
                int32_t* acc = c.tmp_alloc<int32_t>(ncand);
                int64_t* pw_snap = c.tmp_alloc<int64_t>(k);
                GP_CUDA(cudaMemcpyAsync(pw_snap, B.pw, sizeof(int64_t) * k, cudaMemcpyDeviceToDevice, c.s));
                k_gather_vw<<<grid_for(ncand, 256), 256, 0, c.s>>>(ncand, B.cvals, g.vw, wv);
                GP_LAUNCHED(c);
                scan_excl_i32_to_i64(c, wv, pre, ncand, nullptr);
                int64_t* segf = c.tmp_alloc<int64_t>(k + 1);
                k_seg_first<<<grid_for(k + 1, 256), 256, 0, c.s>>>(ncand, B.ckeys, k, segf);
                GP_LAUNCHED(c);
                k_rb_source<<<grid_for(ncand, 256), 256, 0, c.s>>>(ncand, B.ckeys, segf, pre, B.pw, Lmax, acc);
                GP_LAUNCHED(c);
                if (mode == 1) {
                    int64_t* apos = c.tmp_alloc<int64_t>(ncand + 1);
                    scan_excl_i32_to_i64(c, acc, apos, ncand, apos + ncand);
                    const int64_t n2 = read_i64(c, apos + ncand);
                    if (n2 > 0) {
                        k_rb_rekey<<<grid_for(ncand, 256), 256, 0, c.s>>>(ncand, B.ckeys, B.cvals, acc, apos, B.dest,
                                                                        B.ckeys2, B.cvals2);
                        GP_LAUNCHED(c);
                        radix_sort_pairs(c, B.ckeys2, B.cvals2, B.ckeys, B.cvals, n2, bits);
                        k_gather_vw<<<grid_for(n2, 256), 256, 0, c.s>>>(n2, B.cvals2, g.vw, wv);
                        GP_LAUNCHED(c);
                        scan_excl_i32_to_i64(c, wv, pre, n2, nullptr);
                        k_seg_first<<<grid_for(k + 1, 256), 256, 0, c.s>>>(n2, B.ckeys2, k, segf);
                        GP_LAUNCHED(c);
                        k_rb_weak_apply<<<grid_for(n2, 256), 256, sizeof(int64_t) * k, c.s>>>(
                            n2, B.ckeys2, segf, B.cvals2, pre, g.vw, pw_snap, Lmax, k, B.part, B.pc, B.pcb, B.lock, B.pw,
                            moves_d);
                        GP_LAUNCHED(c);
                    }
                } else {
                    int64_t* cum = c.tmp_alloc<int64_t>(k + 1);
                    int32_t* wm = c.tmp_alloc<int32_t>(ncand);
                    k_cumfree<<<1, 32, 0, c.s>>>(k, B.pw, Lmax, cum);
                    GP_LAUNCHED(c);
                    k_mask_vw<<<grid_for(ncand, 256), 256, 0, c.s>>>(ncand, acc, wv, wm);
                    GP_LAUNCHED(c);
                    scan_excl_i32_to_i64(c, wm, pre, ncand, nullptr);
                    k_rb_strong_apply<<<grid_for(ncand, 256), 256, sizeof(int64_t) * k, c.s>>>(
                        ncand, B.cvals, acc, pre, g.vw, cum, k, B.part, B.pc, B.pcb, B.lock, B.pw, moves_d);
                    GP_LAUNCHED(c);
                }
                c.bytes += 80 * ncand;
            }
            c.tmp->restore(mk);
        }
        ++steps;
        if (tr.on()) trace_iter(c, B, n, g.m, level, it, mode, cur_cut, cur_mp, tr);
    }
    GP_CUDA(cudaMemcpyAsync(B.part, B.best, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, c.s));
    GP_CUDA(cudaMemcpyAsync(B.pw, B.best_pw, sizeof(int64_t) * k, cudaMemcpyDeviceToDevice, c.s));
    return steps;
}

}  // namespace gp
