// gp_gnn.cu -- learned edge scores for the matching priority.
//
// No counterpart in the reference: its run log names a GNNcoarsening.cu
// (script/run.txt:5-6) that is not in the repository.  This is a small
// message-passing network whose only output is an integer priority per
// directed entry; matching uses it in place of the edge weight, so every
// partition decision stays integer and deterministic given the priorities.
//
// Per level graph (CSR, weights NULL = 1):
//   x_v  = [log2(1+deg)/8, log2(1+wdeg)/16, log2(1+vw)/16, level/16]      (4)
//   a_v  = mean_{u in N(v)} x_u                                            (4)
//   h1_v = ReLU(W1 [x_v; a_v] + b1)                                        (64)
//   m_v  = P h1_v                    (message sent to the neighbours)      (8)
//   c_v  = mean_{u in N(v)} m_u                                            (8)
//   h2_v = ReLU(W2 [h1_v; c_v] + b2)                                       (64)
//   z_v  = Z h2_v                                                          (4)
//   t_vu = sum_j A_j z_v[j] z_u[j] + beta log2(1+w)/8 + gamma (w/wdeg_v + w/wdeg_u) + delta
//          + eta log2(1 + cn_vu)/7
// cn_vu counts common neighbours through 128-bit neighbour signatures: bit
// b(x) = fmix32(x * 0x9E3779B1) >> 25 is set in sig_v for every neighbour x
// of v, and cn_vu = popcount(sig_v & sig_u) without the bits b(v) and b(u)
// (an exact integer on both sides; at most 128).
// t is symmetric bit-for-bit (the same products in the same order), so both
// endpoints of an edge see the same priority clamp(round(t * 2^16) + 2^30).
// Weights are stored in BF16 and every product is accumulated in FP32.
// Training (binary cross-entropy on "edge ends up inside a part" labels) uses
// the backward kernels below; no gradient needs a scatter because the graph
// is symmetric (each row owner gathers what its neighbours would send).
//
// Move-order head: label-propagation candidates (vertex v proposing part
// dest_v with integer gain g_v) are scored by a second small network,
//   f_v = [sign(g) log2(1+|g|)/16, log2(1+deg_v)/8, log2(1+vw_v)/16, level/16]
//   s_v = w2 . ReLU(W1 f_v + b1) + b2                (hidden 16)
//   mprio_v = clamp(rint(s_v * 2^12), -2^30, 2^30)
// and the afterburner treats the neighbours of higher (mprio, lower id) as
// moved first, in place of the (gain, id) order.  It is trained on which
// candidates of the plain partitioner end the level in their proposed part.
#define GP_TU_ID 8   // site ids of the bounds-checked build
#include "gp_internal.cuh"

#include <cuda_bf16.h>
#include <mutex>

namespace gp {

// parameter layout (floats)
constexpr int H = 64, F0 = 4, MSG = 8, ZD = 4;
constexpr int O_W1 = 0, O_B1 = O_W1 + H * 2 * F0, O_P = O_B1 + H, O_W2 = O_P + MSG * H, O_B2 = O_W2 + H * (H + MSG),
              O_Z = O_B2 + H, O_A = O_Z + ZD * H, O_BETA = O_A + ZD, O_GAMMA = O_BETA + 1, O_DELTA = O_GAMMA + 1,
              O_ETA = O_DELTA + 1, NPARAM = O_ETA + 1;
constexpr int NEDGE = ZD + 4;   // A, beta, gamma, delta, eta
// move-order head: W1[MH, MF] b1[MH] w2[MH] b2
constexpr int MH = 16, MF = 4;
constexpr int MO_W1 = 0, MO_B1 = MO_W1 + MH * MF, MO_W2 = MO_B1 + MH, MO_B2 = MO_W2 + MH, MNPARAM = MO_B2 + 1;

}  // namespace gp

struct gp_gnn {
    float* master = nullptr;          // FP32 master weights (device)
    __nv_bfloat16* w16 = nullptr;     // BF16 weights used by every kernel (device)
    float* grad = nullptr;            // gradients (device)
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    int64_t step = 0;
    float hedge[gp::NEDGE] = {};      // host copy of the BF16-rounded A, beta, gamma, delta, eta
    int32_t prio_bits = 16;           // priority = rint(logit * 2^prio_bits) + 2^30
    int32_t max_level = -1;           // learned priorities at levels <= max_level (-1: every level)
    // move-order head (no allocation until its parameters are set)
    float* mh_master = nullptr;
    __nv_bfloat16* mh_w16 = nullptr;
    float* mh_grad = nullptr;
    float* mh_m = nullptr;
    float* mh_v = nullptr;
    int64_t mh_step = 0;
    int32_t move_head = 0;            // 1: the learned V-cycle orders moves by the head
    gp::Arena arena;                  // per-vertex activations
    gp::Arena keep;                   // row buckets of graphs scored outside a V-cycle
};

namespace gp {

__device__ __forceinline__ float wload(const __nv_bfloat16* w, int i) { return __bfloat162float(w[i]); }

template <int F>
__device__ __forceinline__ void warp_reduce_vec(float (&x)[F]) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int j = 0; j < F; ++j) x[j] += __shfl_xor_sync(0xffffffffu, x[j], o);
}

// ---------------------------------------------------------------- row visits
// The level graph's rows in the degree buckets the matching uses: rows of at
// most 8 entries four to a warp (8 lanes each), rows of 9..32 entries one
// warp, rows of 33..2048 entries one warp looping, longer rows split into CTA
// items of at most 16384 entries.  Every sum below adds in a fixed order (the
// lane layout, then a shuffle tree, then item order), so results are
// reproducible run to run.
struct GnnRows {
    DGraph g;
    const int32_t* b[3];
    int64_t nb[3];
    const int32_t* heavy;
    int64_t nheavy;
    const int32_t* item_row;
    const int64_t* item_beg;
    const int64_t* item_end;
    int64_t nitems;
    const int32_t* row_items;
    const int32_t* row_first;
};

static GnnRows gnn_rows(const Level& L) {
    GnnRows R;
    R.g = L.g;
    for (int i = 0; i < 3; ++i) { R.b[i] = L.bucket[i]; R.nb[i] = L.nbucket[i]; }
    R.heavy = L.heavy; R.nheavy = L.nheavy;
    R.item_row = L.item_row; R.item_beg = L.item_beg; R.item_end = L.item_end; R.nitems = L.nitems;
    R.row_items = L.row_items; R.row_first = L.row_first;
    return R;
}

template <int F>
__device__ __forceinline__ void tile_reduce(float (&x)[F], int width) {
    for (int o = width / 2; o > 0; o >>= 1)
#pragma unroll
        for (int j = 0; j < F; ++j) x[j] += __shfl_xor_sync(0xffffffffu, x[j], o);
}

// out_v = fin(v, sum over entries e of row v of val(e)) for every vertex v.
// CTAs [0, nitems) each sum one item of a long row into ipart[item]; the
// long rows are finished by k_gnn_rowsum_heavy.
template <int F, class Val, class Fin>
__global__ void __launch_bounds__(256) k_gnn_rowsum(GnnRows R, Val val, Fin fin, float* __restrict__ ipart) {
    const int lane = threadIdx.x & 31;
    if ((int64_t)blockIdx.x < R.nitems) {
        __shared__ float sp[8][F];
        float acc[F];
#pragma unroll
        for (int j = 0; j < F; ++j) acc[j] = 0.f;
        const int64_t end = R.item_end[blockIdx.x];
        for (int64_t e = R.item_beg[blockIdx.x] + threadIdx.x; e < end; e += blockDim.x) val(e, acc);
        tile_reduce<F>(acc, 32);
        if (lane == 0)
#pragma unroll
            for (int j = 0; j < F; ++j) sp[threadIdx.x >> 5][j] = acc[j];
        __syncthreads();
        if (threadIdx.x < F) {
            float t = 0.f;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sp[w][threadIdx.x];
            ipart[blockIdx.x * F + threadIdx.x] = t;
        }
        return;
    }
    const int64_t wid = ((int64_t)(blockIdx.x - R.nitems) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)(gridDim.x - R.nitems) * blockDim.x) >> 5;
    const int64_t U0 = (R.nb[0] + 3) / 4, U1 = R.nb[1], U2 = R.nb[2];
    for (int64_t u = wid; u < U0 + U1 + U2; u += nw) {
        float acc[F];
#pragma unroll
        for (int j = 0; j < F; ++j) acc[j] = 0.f;
        int64_t v;
        int width;
        if (u < U0) {
            const int64_t i = u * 4 + (lane >> 3);
            v = i < R.nb[0] ? R.b[0][i] : -1;
            width = 8;
            if (v >= 0) {
                const int64_t e = R.g.rp[v] + (lane & 7);
                if (e < R.g.rp[v + 1]) val(e, acc);
            }
        } else {
            v = u < U0 + U1 ? R.b[1][u - U0] : R.b[2][u - U0 - U1];
            width = 32;
            const int64_t end = R.g.rp[v + 1];
            for (int64_t e = R.g.rp[v] + lane; e < end; e += 32) val(e, acc);
        }
        tile_reduce<F>(acc, width);
        if (v >= 0 && (lane & (width - 1)) == 0) fin(v, acc);
    }
}

// finish the long rows: item partial sums added in item order
template <int F, class Fin>
__global__ void k_gnn_rowsum_heavy(GnnRows R, Fin fin, const float* __restrict__ ipart) {
    for (int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; h < R.nheavy; h += (int64_t)gridDim.x * blockDim.x) {
        float acc[F];
#pragma unroll
        for (int j = 0; j < F; ++j) acc[j] = 0.f;
        const int32_t f = R.row_first[h], cnt = R.row_items[h];
        for (int i = 0; i < cnt; ++i)
#pragma unroll
            for (int j = 0; j < F; ++j) acc[j] += ipart[(int64_t)(f + i) * F + j];
        fin(R.heavy[h], acc);
    }
}

// op(v, e) for every entry e of every row v, in the same row layout
template <class Op>
__global__ void __launch_bounds__(256) k_gnn_entries(GnnRows R, Op op) {
    const int lane = threadIdx.x & 31;
    if ((int64_t)blockIdx.x < R.nitems) {
        const int64_t v = R.heavy[R.item_row[blockIdx.x]];
        const int64_t end = R.item_end[blockIdx.x];
        for (int64_t e = R.item_beg[blockIdx.x] + threadIdx.x; e < end; e += blockDim.x) op(v, e);
        return;
    }
    const int64_t wid = ((int64_t)(blockIdx.x - R.nitems) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)(gridDim.x - R.nitems) * blockDim.x) >> 5;
    const int64_t U0 = (R.nb[0] + 3) / 4, U1 = R.nb[1], U2 = R.nb[2];
    for (int64_t u = wid; u < U0 + U1 + U2; u += nw) {
        if (u < U0) {
            const int64_t i = u * 4 + (lane >> 3);
            if (i < R.nb[0]) {
                const int64_t v = R.b[0][i];
                const int64_t e = R.g.rp[v] + (lane & 7);
                if (e < R.g.rp[v + 1]) op(v, e);
            }
        } else {
            const int64_t v = u < U0 + U1 ? R.b[1][u - U0] : R.b[2][u - U0 - U1];
            const int64_t end = R.g.rp[v + 1];
            for (int64_t e = R.g.rp[v] + lane; e < end; e += 32) op(v, e);
        }
    }
}

// entry values and row finishers
struct ValWeight {          // edge weight
    const int32_t* ew;
    __device__ void operator()(int64_t e, float (&a)[1]) const { a[0] += (float)__ldcs(&ew[e]); }
};
struct ValRow4 {            // the neighbour's 4-float row
    const int32_t* ci; const float4* in;
    __device__ void operator()(int64_t e, float (&a)[4]) const {
        const float4 x = in[__ldcs(&ci[e])];
        a[0] += x.x; a[1] += x.y; a[2] += x.z; a[3] += x.w;
    }
};
struct ValRow8 {            // the neighbour's 8-float row
    const int32_t* ci; const float4* in;
    __device__ void operator()(int64_t e, float (&a)[8]) const {
        const int64_t u = __ldcs(&ci[e]);
        const float4 x = in[2 * u], y = in[2 * u + 1];
        a[0] += x.x; a[1] += x.y; a[2] += x.z; a[3] += x.w;
        a[4] += y.x; a[5] += y.y; a[6] += y.z; a[7] += y.w;
    }
};
struct FinStore1 {
    float* out;
    __device__ void operator()(int64_t v, float (&a)[1]) const { out[v] = a[0]; }
};
template <int F>
struct FinMean {            // out_v = sum / deg_v (0 for an isolated vertex)
    const int64_t* rp; float* out;
    __device__ void operator()(int64_t v, float (&a)[F]) const {
        const int64_t d = rp[v + 1] - rp[v];
        const float inv = d > 0 ? 1.f / (float)d : 0.f;
#pragma unroll
        for (int j = 0; j < F; ++j) out[F * v + j] = a[j] * inv;
    }
};

// x_v; wdeg_v = deg_v when the graph has unit weights, else the weighted
// degree computed by a row sum beforehand
__global__ void k_gnn_vfeat(int64_t n, const int64_t* __restrict__ rp, const int32_t* __restrict__ vw, float level,
                            int unit_w, float4* __restrict__ x, float* __restrict__ wdeg) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const float deg = (float)(rp[v + 1] - rp[v]);
        float s;
        if (unit_w) { s = deg; wdeg[v] = s; }
        else s = wdeg[v];
        const float w = vw ? (float)vw[v] : 1.f;
        x[v] = make_float4(log2f(1.f + deg) * 0.125f, log2f(1.f + s) * 0.0625f, log2f(1.f + w) * 0.0625f,
                           level * 0.0625f);
    }
}

// h1 = ReLU(W1 [x; a] + b1), m = P h1; thread per vertex, weights in shared memory
__global__ void __launch_bounds__(128) k_gnn_l1(int64_t n, const __nv_bfloat16* __restrict__ w,
                                                const float* __restrict__ x, const float* __restrict__ a,
                                                float* __restrict__ m, float* __restrict__ h1_out) {
    __shared__ float sW1[H * 2 * F0], sB1[H], sP[MSG * H];
    for (int i = threadIdx.x; i < H * 2 * F0; i += blockDim.x) sW1[i] = wload(w, O_W1 + i);
    for (int i = threadIdx.x; i < H; i += blockDim.x) sB1[i] = wload(w, O_B1 + i);
    for (int i = threadIdx.x; i < MSG * H; i += blockDim.x) sP[i] = wload(w, O_P + i);
    __syncthreads();
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        float in[2 * F0];
#pragma unroll
        for (int j = 0; j < F0; ++j) { in[j] = x[F0 * v + j]; in[F0 + j] = a[F0 * v + j]; }
        float mm[MSG];
#pragma unroll
        for (int j = 0; j < MSG; ++j) mm[j] = 0.f;
        for (int i = 0; i < H; ++i) {
            float s = sB1[i];
#pragma unroll
            for (int j = 0; j < 2 * F0; ++j) s += sW1[i * 2 * F0 + j] * in[j];
            s = s > 0.f ? s : 0.f;
            if (h1_out) h1_out[H * v + i] = s;
#pragma unroll
            for (int j = 0; j < MSG; ++j) mm[j] += sP[j * H + i] * s;
        }
#pragma unroll
        for (int j = 0; j < MSG; ++j) m[MSG * v + j] = mm[j];
    }
}

// h2 = ReLU(W2 [h1; c] + b2), z = Z h2 (h1 recomputed from x, a); thread per vertex.
// W2 is staged transposed so that one h1 (or c) component updates all 64
// accumulators from one contiguous shared-memory row; each h2 sum still adds
// its terms in input order.
__global__ void __launch_bounds__(128) k_gnn_l2(int64_t n, const __nv_bfloat16* __restrict__ w,
                                                const float* __restrict__ x, const float* __restrict__ a,
                                                const float* __restrict__ c, float* __restrict__ z,
                                                float* __restrict__ h2_out) {
    __shared__ float sW1[H * 2 * F0], sB1[H], sW2T[(H + MSG) * H], sB2[H], sZ[ZD * H];
    for (int i = threadIdx.x; i < H * 2 * F0; i += blockDim.x) sW1[i] = wload(w, O_W1 + i);
    for (int i = threadIdx.x; i < H; i += blockDim.x) { sB1[i] = wload(w, O_B1 + i); sB2[i] = wload(w, O_B2 + i); }
    for (int i = threadIdx.x; i < H * (H + MSG); i += blockDim.x) {
        const int r = i / (H + MSG), q = i % (H + MSG);
        sW2T[q * H + r] = wload(w, O_W2 + i);
    }
    for (int i = threadIdx.x; i < ZD * H; i += blockDim.x) sZ[i] = wload(w, O_Z + i);
    __syncthreads();
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        float in[2 * F0];
#pragma unroll
        for (int j = 0; j < F0; ++j) { in[j] = x[F0 * v + j]; in[F0 + j] = a[F0 * v + j]; }
        // keep the staged weights in shared memory: without this barrier the
        // compiler hoists every constant-indexed weight read out of the vertex
        // loop and spills them
        asm volatile("" ::: "memory");
        float acc[H];
#pragma unroll
        for (int i = 0; i < H; ++i) acc[i] = sB2[i];
#pragma unroll 1
        for (int q = 0; q < H; ++q) {
            float s = sB1[q];
#pragma unroll
            for (int j = 0; j < 2 * F0; ++j) s += sW1[q * 2 * F0 + j] * in[j];
            s = s > 0.f ? s : 0.f;
            const float* col = sW2T + q * H;
#pragma unroll
            for (int i = 0; i < H; ++i) acc[i] += col[i] * s;
        }
#pragma unroll 1
        for (int q = 0; q < MSG; ++q) {
            const float s = c[MSG * v + q];
            const float* col = sW2T + (H + q) * H;
#pragma unroll
            for (int i = 0; i < H; ++i) acc[i] += col[i] * s;
        }
        float zz[ZD];
#pragma unroll
        for (int j = 0; j < ZD; ++j) zz[j] = 0.f;
#pragma unroll
        for (int i = 0; i < H; ++i) {
            const float s = acc[i] > 0.f ? acc[i] : 0.f;
            if (h2_out) h2_out[H * v + i] = s;
#pragma unroll
            for (int j = 0; j < ZD; ++j) zz[j] += sZ[j * H + i] * s;
        }
#pragma unroll
        for (int j = 0; j < ZD; ++j) z[ZD * v + j] = zz[j];
    }
}

// signature bit of vertex x (0..127)
__host__ __device__ __forceinline__ uint32_t nb_bit(int32_t x) { return fmix32((uint32_t)x * 0x9E3779B1u) >> 25; }

// 128-bit neighbour signature of every vertex, one warp per row
__global__ void k_gnn_sig(DGraph g, uint4* __restrict__ sig) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = wid; v < g.n; v += nw) {
        uint32_t w0 = 0, w1 = 0, w2 = 0, w3 = 0;
        for (int64_t e = g.rp[v] + lane; e < g.rp[v + 1]; e += 32) {
            const uint32_t b = nb_bit(__ldcs(&g.ci[e])), m = 1u << (b & 31), q = b >> 5;
            w0 |= q == 0 ? m : 0u; w1 |= q == 1 ? m : 0u; w2 |= q == 2 ? m : 0u; w3 |= q == 3 ? m : 0u;
        }
        w0 = __reduce_or_sync(0xffffffffu, w0); w1 = __reduce_or_sync(0xffffffffu, w1);
        w2 = __reduce_or_sync(0xffffffffu, w2); w3 = __reduce_or_sync(0xffffffffu, w3);
        if (lane == 0) sig[v] = make_uint4(w0, w1, w2, w3);
    }
}

// log2(1 + common-neighbour count) / 7 of the entry (v, u)
__device__ __forceinline__ float cn_feat(const uint4* __restrict__ sig, int64_t v, int64_t u) {
    const uint4 a = sig[v], b = sig[u];
    uint32_t m0 = a.x & b.x, m1 = a.y & b.y, m2 = a.z & b.z, m3 = a.w & b.w;
    const uint32_t bv = nb_bit((int32_t)v), bu = nb_bit((int32_t)u);
    const uint32_t cv = ~(1u << (bv & 31)), cu = ~(1u << (bu & 31));
    m0 &= (bv >> 5) == 0 ? cv : ~0u; m1 &= (bv >> 5) == 1 ? cv : ~0u;
    m2 &= (bv >> 5) == 2 ? cv : ~0u; m3 &= (bv >> 5) == 3 ? cv : ~0u;
    m0 &= (bu >> 5) == 0 ? cu : ~0u; m1 &= (bu >> 5) == 1 ? cu : ~0u;
    m2 &= (bu >> 5) == 2 ? cu : ~0u; m3 &= (bu >> 5) == 3 ? cu : ~0u;
    const int cnt = __popc(m0) + __popc(m1) + __popc(m2) + __popc(m3);
    return log2f(1.f + (float)cnt) * (1.f / 7.f);
}

__device__ __forceinline__ float edge_logit(const float* __restrict__ sA, float beta, float gamma, float delta,
                                            float eta, float fcn, const float* zv, const float* __restrict__ z,
                                            int64_t u, float w, float wdv, float wdu) {
    const float4 q = reinterpret_cast<const float4*>(z)[u];
    const float zu[ZD] = {q.x, q.y, q.z, q.w};
    float t = 0.f;
#pragma unroll
    for (int j = 0; j < ZD; ++j) t += sA[j] * (zv[j] * zu[j]);
    t += beta * (log2f(1.f + w) * 0.125f);
    t += gamma * (w / wdv + w / wdu);
    t += delta;
    return t + eta * fcn;
}

// clamp(rint(t * 2^bits) + 2^30, 0, 2^31 - 128) with pscale = 2^bits; the
// offset is added in integer arithmetic (a float32 sum near 2^30 would round
// to multiples of 128).  Fewer bits leave more ties to the hash tie-break.
__device__ __forceinline__ int32_t logit_prio(float t, float pscale) {
    float q = rintf(t * pscale);
    q = fminf(fmaxf(q, -1073741824.f), 1073741696.f);
    return (int32_t)q + 1073741824;
}

// per entry: priority (matching) and/or logit (checks)
struct EdgeOp {
    DGraph g;
    const float* z; const float* wdeg; const uint4* sig;
    float A[ZD]; float beta, gamma, delta, eta, pscale;
    int32_t* prio; float* logit;
    __device__ void operator()(int64_t v, int64_t e) const {
        const int64_t u = __ldcs(&g.ci[e]);
        float zv[ZD];
        const float4 q = reinterpret_cast<const float4*>(z)[v];
        zv[0] = q.x; zv[1] = q.y; zv[2] = q.z; zv[3] = q.w;
        const float t = edge_logit(A, beta, gamma, delta, eta, cn_feat(sig, v, u), zv, z, u,
                                   g.ew ? (float)__ldcs(&g.ew[e]) : 1.f, wdeg[v], wdeg[u]);
        if (prio) prio[e] = logit_prio(t, pscale);
        if (logit) logit[e] = t;
    }
};

// ------------------------------------------------------------------ training
// loss and dt per entry; dz_v = 2 sum_u dt_vu A (.) z_u; gradients of A, beta, gamma, delta
__global__ void k_gnn_edge_bwd(DGraph g, const __nv_bfloat16* __restrict__ w, const float* __restrict__ z,
                               const float* __restrict__ wdeg, const uint4* __restrict__ sig,
                               const uint8_t* __restrict__ label, float inv_e, float* __restrict__ dz,
                               float* __restrict__ grad, float* __restrict__ loss) {
    __shared__ float sA[ZD];
    __shared__ float sc[4];
    __shared__ float sg[ZD + 5];
    if (threadIdx.x < ZD) sA[threadIdx.x] = wload(w, O_A + threadIdx.x);
    if (threadIdx.x < 4) sc[threadIdx.x] = wload(w, O_BETA + threadIdx.x);
    if (threadIdx.x < ZD + 5) sg[threadIdx.x] = 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    float gA[ZD] = {0.f, 0.f, 0.f, 0.f}, gb = 0.f, gg = 0.f, gd = 0.f, ge = 0.f, ls = 0.f;
    for (int64_t v = wid; v < g.n; v += nw) {
        float zv[ZD], dzv[ZD];
#pragma unroll
        for (int j = 0; j < ZD; ++j) { zv[j] = z[ZD * v + j]; dzv[j] = 0.f; }
        const float wdv = wdeg[v];
        for (int64_t e = g.rp[v] + lane; e < g.rp[v + 1]; e += 32) {
            const int64_t u = g.ci[e];
            const float we = g.ew ? (float)g.ew[e] : 1.f;
            const float fcn = cn_feat(sig, v, u);
            const float t = edge_logit(sA, sc[0], sc[1], sc[2], sc[3], fcn, zv, z, u, we, wdv, wdeg[u]);
            const float y = label[e] ? 1.f : 0.f;
            const float s = 1.f / (1.f + expf(-t));
            // BCE with logits, stable form
            ls += (fmaxf(t, 0.f) - t * y + log1pf(expf(-fabsf(t)))) * inv_e;
            const float dt = (s - y) * inv_e;
#pragma unroll
            for (int j = 0; j < ZD; ++j) {
                const float zu = z[ZD * u + j];
                gA[j] += dt * zv[j] * zu;
                dzv[j] += 2.f * dt * sA[j] * zu;
            }
            gb += dt * (log2f(1.f + we) * 0.125f);
            gg += dt * (we / wdv + we / wdeg[u]);
            gd += dt;
            ge += dt * fcn;
        }
        warp_reduce_vec<ZD>(dzv);
        if (lane < ZD) {
            float r = 0.f;
#pragma unroll
            for (int j = 0; j < ZD; ++j) if (j == lane) r = dzv[j];
            dz[ZD * v + lane] = r;
        }
    }
    float part[ZD + 5] = {gA[0], gA[1], gA[2], gA[3], gb, gg, gd, ls, ge};
    warp_reduce_vec<ZD + 5>(part);
    if (lane == 0)
        for (int j = 0; j < ZD + 5; ++j) atomicAdd(&sg[j], part[j]);
    __syncthreads();
    if (threadIdx.x < ZD) atomicAdd(&grad[O_A + threadIdx.x], sg[threadIdx.x]);
    if (threadIdx.x == ZD) atomicAdd(&grad[O_BETA], sg[ZD]);
    if (threadIdx.x == ZD + 1) atomicAdd(&grad[O_GAMMA], sg[ZD + 1]);
    if (threadIdx.x == ZD + 2) atomicAdd(&grad[O_DELTA], sg[ZD + 2]);
    if (threadIdx.x == ZD + 3) atomicAdd(loss, sg[ZD + 3]);
    if (threadIdx.x == ZD + 4) atomicAdd(&grad[O_ETA], sg[ZD + 4]);
}

// dpre2 = (Z^T dz) * [h2 > 0]; dh1 (direct part) and dc from W2^T dpre2; thread per vertex
__global__ void __launch_bounds__(128) k_gnn_l2_bwd(int64_t n, const __nv_bfloat16* __restrict__ w,
                                                    const float* __restrict__ dz, const float* __restrict__ h2,
                                                    float* __restrict__ dpre2, float* __restrict__ dh1,
                                                    float* __restrict__ dc) {
    __shared__ float sW2[H * (H + MSG)], sZ[ZD * H];
    for (int i = threadIdx.x; i < H * (H + MSG); i += blockDim.x) sW2[i] = wload(w, O_W2 + i);
    for (int i = threadIdx.x; i < ZD * H; i += blockDim.x) sZ[i] = wload(w, O_Z + i);
    __syncthreads();
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        float d[ZD];
#pragma unroll
        for (int j = 0; j < ZD; ++j) d[j] = dz[ZD * v + j];
        float acc[H + MSG];
#pragma unroll
        for (int j = 0; j < H + MSG; ++j) acc[j] = 0.f;
#pragma unroll 1
        for (int i = 0; i < H; ++i) {
            float s = 0.f;
#pragma unroll
            for (int j = 0; j < ZD; ++j) s += sZ[j * H + i] * d[j];
            s = h2[H * v + i] > 0.f ? s : 0.f;
            dpre2[H * v + i] = s;
            const float* row = sW2 + i * (H + MSG);
#pragma unroll
            for (int j = 0; j < H + MSG; ++j) acc[j] += row[j] * s;
        }
#pragma unroll
        for (int j = 0; j < H; ++j) dh1[H * v + j] = acc[j];
#pragma unroll
        for (int j = 0; j < MSG; ++j) dc[MSG * v + j] = acc[H + j];
    }
}

// dm_u = sum_{v in N(u)} dc_v / deg_v (symmetric graph: the row owner gathers)
__global__ void k_gnn_msg_bwd(DGraph g, const float* __restrict__ dc, float* __restrict__ dm) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = wid; u < g.n; u += nw) {
        float acc[MSG];
#pragma unroll
        for (int j = 0; j < MSG; ++j) acc[j] = 0.f;
        for (int64_t e = g.rp[u] + lane; e < g.rp[u + 1]; e += 32) {
            const int64_t v = g.ci[e];
            const float inv = 1.f / (float)(g.rp[v + 1] - g.rp[v]);
#pragma unroll
            for (int j = 0; j < MSG; ++j) acc[j] += dc[MSG * v + j] * inv;
        }
        warp_reduce_vec<MSG>(acc);
        if (lane < MSG) {
            float r = 0.f;
#pragma unroll
            for (int j = 0; j < MSG; ++j) if (j == lane) r = acc[j];
            dm[MSG * u + lane] = r;
        }
    }
}

// dpre1 = (dh1 + P^T dm) * [h1 > 0]; thread per vertex
__global__ void __launch_bounds__(128) k_gnn_l1_bwd(int64_t n, const __nv_bfloat16* __restrict__ w,
                                                    const float* __restrict__ dh1, const float* __restrict__ dm,
                                                    const float* __restrict__ h1, float* __restrict__ dpre1) {
    __shared__ float sP[MSG * H];
    for (int i = threadIdx.x; i < MSG * H; i += blockDim.x) sP[i] = wload(w, O_P + i);
    __syncthreads();
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        float d[MSG];
#pragma unroll
        for (int j = 0; j < MSG; ++j) d[j] = dm[MSG * v + j];
        for (int i = 0; i < H; ++i) {
            float s = dh1[H * v + i];
#pragma unroll
            for (int j = 0; j < MSG; ++j) s += sP[j * H + i] * d[j];
            dpre1[H * v + i] = h1[H * v + i] > 0.f ? s : 0.f;
        }
    }
}

// grad[o + i*C + j] += sum_v A[v*ra + i] * B[v*rb + j]  (i < R, j < C; B == nullptr: ones)
// CTA per chunk of 64 vertices, rows staged in shared memory; each thread
// keeps its (up to OP_PER_THREAD) output sums in registers across all of its
// CTA's chunks and adds them to grad once at the end.
constexpr int OP_CHUNK = 64, OP_THREADS = 256, OP_PER_THREAD = 18;   // R*C <= 256*18 (W2: 64*72)
__global__ void __launch_bounds__(OP_THREADS) k_gnn_outer(int64_t n, const float* __restrict__ A, int ra, int R,
                                                          const float* __restrict__ B, int rb, int C,
                                                          float* __restrict__ grad, int o) {
    extern __shared__ float sm[];
    float* sa = sm;                       // OP_CHUNK * R
    float* sb = sm + OP_CHUNK * R;        // OP_CHUNK * C
    float acc[OP_PER_THREAD];
#pragma unroll
    for (int q = 0; q < OP_PER_THREAD; ++q) acc[q] = 0.f;
    for (int64_t base = (int64_t)blockIdx.x * OP_CHUNK; base < n; base += (int64_t)gridDim.x * OP_CHUNK) {
        const int cnt = (int)((n - base) < OP_CHUNK ? (n - base) : OP_CHUNK);
        for (int i = threadIdx.x; i < OP_CHUNK * R; i += blockDim.x) {
            const int v = i / R, r = i % R;
            sa[i] = v < cnt ? A[(base + v) * ra + r] : 0.f;
        }
        for (int i = threadIdx.x; i < OP_CHUNK * C; i += blockDim.x) {
            const int v = i / C, cc = i % C;
            sb[i] = v < cnt ? (B ? B[(base + v) * rb + cc] : 1.f) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < OP_PER_THREAD; ++q) {
            const int idx = threadIdx.x + q * OP_THREADS;
            if (idx < R * C) {
                const int i = idx / C, j = idx % C;
                float s = 0.f;
                for (int v = 0; v < cnt; ++v) s += sa[v * R + i] * sb[v * C + j];
                acc[q] += s;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < OP_PER_THREAD; ++q) {
        const int idx = threadIdx.x + q * OP_THREADS;
        if (idx < R * C && acc[q] != 0.f) atomicAdd(&grad[o + idx], acc[q]);
    }
}

// [x; a] and [h1; c] rows for the weight gradients
__global__ void k_gnn_concat(int64_t n, const float* __restrict__ p, int fp, const float* __restrict__ q, int fq,
                             float* __restrict__ out) {
    const int f = fp + fq;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * f; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = i / f;
        const int j = (int)(i % f);
        out[i] = j < fp ? p[v * fp + j] : q[v * fq + (j - fp)];
    }
}

__global__ void k_gnn_adam(int np, float* __restrict__ master, __nv_bfloat16* __restrict__ w16,
                           const float* __restrict__ grad, float* __restrict__ m, float* __restrict__ v, float lr,
                           float b1, float b2, float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        const float gr = grad[i];
        m[i] = b1 * m[i] + (1.f - b1) * gr;
        v[i] = b2 * v[i] + (1.f - b2) * gr * gr;
        master[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
        w16[i] = __float2bfloat16(master[i]);
    }
}

__global__ void k_gnn_to_bf16(int np, const float* __restrict__ master, __nv_bfloat16* __restrict__ w16) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x)
        w16[i] = __float2bfloat16(master[i]);
}

// ------------------------------------------------------------------ host
struct GnnActs {
    float *x, *wdeg, *a, *m, *c, *z, *h1, *h2;
    uint4* sig;               // neighbour signatures (common-neighbour feature)
};

static void gnn_forward(Ctx& c, const gp_gnn* G, const Level& L, int level, bool keep, GnnActs& A) {
    const DGraph& g = L.g;
    const int64_t n = g.n;
    const GnnRows R = gnn_rows(L);
    A.x = c.tmp_alloc<float>(F0 * n);
    A.wdeg = c.tmp_alloc<float>(n);
    A.a = c.tmp_alloc<float>(F0 * n);
    A.m = c.tmp_alloc<float>(MSG * n);
    A.c = c.tmp_alloc<float>(MSG * n);
    A.z = c.tmp_alloc<float>(ZD * n);
    A.h1 = keep ? c.tmp_alloc<float>(H * n) : nullptr;
    A.h2 = keep ? c.tmp_alloc<float>(H * n) : nullptr;
    float* ipart = c.tmp_alloc<float>(MSG * std::max<int64_t>(L.nitems, 1));
    const int64_t U = (L.nbucket[0] + 3) / 4 + L.nbucket[1] + L.nbucket[2];
    const int rg = (int)(L.nitems + grid_for(U * 32, 256, c.sm_count * 16));
    const int vg = grid_for(n, 256, c.sm_count * 8), tg = grid_for(n, 128, c.sm_count * 8);
    const int hg = grid_for(std::max<int64_t>(L.nheavy, 1), 128);
    if (g.ew) {
        k_gnn_rowsum<1><<<rg, 256, 0, c.s>>>(R, ValWeight{g.ew}, FinStore1{A.wdeg}, ipart);
        GP_LAUNCHED(c);
        if (L.nheavy) { k_gnn_rowsum_heavy<1><<<hg, 128, 0, c.s>>>(R, FinStore1{A.wdeg}, ipart); GP_LAUNCHED(c); }
    }
    k_gnn_vfeat<<<vg, 256, 0, c.s>>>(n, g.rp, g.vw, (float)level, g.ew ? 0 : 1, (float4*)A.x, A.wdeg);
    GP_LAUNCHED(c);
    A.sig = (uint4*)c.tmp->alloc(sizeof(uint4) * (size_t)std::max<int64_t>(n, 1));
    k_gnn_sig<<<grid_for(n * 32, 256, c.sm_count * 16), 256, 0, c.s>>>(g, A.sig);
    GP_LAUNCHED(c);
    k_gnn_rowsum<F0><<<rg, 256, 0, c.s>>>(R, ValRow4{g.ci, (const float4*)A.x}, FinMean<F0>{g.rp, A.a}, ipart);
    GP_LAUNCHED(c);
    if (L.nheavy) { k_gnn_rowsum_heavy<F0><<<hg, 128, 0, c.s>>>(R, FinMean<F0>{g.rp, A.a}, ipart); GP_LAUNCHED(c); }
    k_gnn_l1<<<tg, 128, 0, c.s>>>(n, G->w16, A.x, A.a, A.m, A.h1);
    GP_LAUNCHED(c);
    k_gnn_rowsum<MSG><<<rg, 256, 0, c.s>>>(R, ValRow8{g.ci, (const float4*)A.m}, FinMean<MSG>{g.rp, A.c}, ipart);
    GP_LAUNCHED(c);
    if (L.nheavy) { k_gnn_rowsum_heavy<MSG><<<hg, 128, 0, c.s>>>(R, FinMean<MSG>{g.rp, A.c}, ipart); GP_LAUNCHED(c); }
    k_gnn_l2<<<tg, 128, 0, c.s>>>(n, G->w16, A.x, A.a, A.c, A.z, A.h2);
    GP_LAUNCHED(c);
    // row sums: rowptr, column ids (+ weights), gathered neighbour rows; per-vertex arrays
    c.bytes += 3 * (8 * (n + 1) + 4 * g.m) + (g.ew ? 8 * g.m : 0) + 4 * g.m * (F0 + MSG) +
               4 * n * (F0 * 3 + MSG * 2 + ZD + 2);
}

static EdgeOp edge_op(const gp_gnn* G, const DGraph& g, const GnnActs& A, int32_t* prio, float* logit) {
    EdgeOp op;
    op.g = g; op.z = A.z; op.wdeg = A.wdeg;
    for (int j = 0; j < ZD; ++j) op.A[j] = G->hedge[j];
    op.beta = G->hedge[ZD]; op.gamma = G->hedge[ZD + 1]; op.delta = G->hedge[ZD + 2]; op.eta = G->hedge[ZD + 3];
    op.sig = A.sig;
    op.pscale = ldexpf(1.f, G->prio_bits);
    op.prio = prio; op.logit = logit;
    return op;
}

static void gnn_edges(Ctx& c, const gp_gnn* G, const Level& L, const GnnActs& A, int32_t* prio, float* logit) {
    const int64_t U = (L.nbucket[0] + 3) / 4 + L.nbucket[1] + L.nbucket[2];
    const int rg = (int)(L.nitems + grid_for(U * 32, 256, c.sm_count * 16));
    k_gnn_entries<<<rg, 256, 0, c.s>>>(gnn_rows(L), edge_op(G, L.g, A, prio, logit));
    GP_LAUNCHED(c);
    c.bytes += 8 * (L.g.n + 1) + 4 * L.g.m * (2 + ZD + 1) + (L.g.ew ? 4 * L.g.m : 0) + 4 * L.g.n * (ZD + 1);
}

bool gnn_scores_level(const gp_gnn* G, int level) { return G->max_level < 0 || level <= G->max_level; }

// ------------------------------------------------------------------ move-order head
__device__ __forceinline__ void move_features(int32_t gain, int64_t deg, int32_t vw, int level, float (&f)[MF]) {
    const float mag = log2f(1.f + fabsf((float)gain)) * (1.f / 16.f);
    f[0] = gain < 0 ? -mag : mag;
    f[1] = log2f(1.f + (float)deg) * 0.125f;
    f[2] = log2f(1.f + (float)vw) * (1.f / 16.f);
    f[3] = (float)level * (1.f / 16.f);
}

// score of one feature row from parameters staged in shared memory (FP32 accumulate)
__device__ __forceinline__ float move_score(const float* __restrict__ sp, const float (&f)[MF], float (&h)[MH]) {
    float s = sp[MO_B2];
#pragma unroll
    for (int i = 0; i < MH; ++i) {
        float a = sp[MO_B1 + i];
#pragma unroll
        for (int j = 0; j < MF; ++j) a += sp[MO_W1 + i * MF + j] * f[j];
        h[i] = a;
        s += sp[MO_W2 + i] * (a > 0.f ? a : 0.f);
    }
    return s;
}

__device__ __forceinline__ int32_t move_prio(float s) {
    const float q = fminf(fmaxf(rintf(s * 4096.f), -1073741824.f), 1073741824.f);
    return (int32_t)q;
}

__device__ __forceinline__ void stage_head(const __nv_bfloat16* __restrict__ w, float* sp) {
    for (int i = threadIdx.x; i < MNPARAM; i += blockDim.x) sp[i] = wload(w, i);
    __syncthreads();
}

// features of every candidate (dest >= 0; others get zeros)
__global__ void k_move_feat(int64_t n, const int64_t* __restrict__ rp, const int32_t* __restrict__ vw,
                            const int32_t* __restrict__ dest, const int32_t* __restrict__ gain, int level,
                            float* __restrict__ feat) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        float f[MF] = {0.f, 0.f, 0.f, 0.f};
        if (dest[v] >= 0) move_features(gain[v], rp[v + 1] - rp[v], vw ? vw[v] : 1, level, f);
#pragma unroll
        for (int j = 0; j < MF; ++j) feat[MF * v + j] = f[j];
    }
}

// move priorities of the candidates of one label-propagation step
__global__ void k_move_prio(int64_t n, const int64_t* __restrict__ rp, const int32_t* __restrict__ vw,
                            const int32_t* __restrict__ dest, const int32_t* __restrict__ gain, int level,
                            const __nv_bfloat16* __restrict__ w, int32_t* __restrict__ mp) {
    __shared__ float sp[MNPARAM];
    stage_head(w, sp);
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        int32_t r = 0;
        if (dest[v] >= 0) {
            float f[MF], h[MH];
            move_features(gain[v], rp[v + 1] - rp[v], vw ? vw[v] : 1, level, f);
            r = move_prio(move_score(sp, f, h));
        }
        mp[v] = r;
    }
}

// scores (and priorities) of feature rows
__global__ void k_move_score(int64_t ns, const float* __restrict__ feat, const __nv_bfloat16* __restrict__ w,
                             float* __restrict__ score, int32_t* __restrict__ prio) {
    __shared__ float sp[MNPARAM];
    stage_head(w, sp);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += (int64_t)gridDim.x * blockDim.x) {
        float f[MF], h[MH];
#pragma unroll
        for (int j = 0; j < MF; ++j) f[j] = feat[MF * i + j];
        const float s = move_score(sp, f, h);
        if (score) score[i] = s;
        if (prio) prio[i] = move_prio(s);
    }
}

// mean binary cross-entropy of the scores against the labels and its
// gradient: per-thread register accumulation over a strided run of
// samples, then warp and block reductions (no atomic per sample)
__global__ void __launch_bounds__(256) k_move_grad(int64_t ns, const float* __restrict__ feat,
                                                   const uint8_t* __restrict__ label,
                                                   const __nv_bfloat16* __restrict__ w, float inv_n,
                                                   float* __restrict__ grad, float* __restrict__ loss) {
    __shared__ float sp[MNPARAM];
    __shared__ float sg[MNPARAM + 1];
    for (int i = threadIdx.x; i <= MNPARAM; i += blockDim.x) sg[i] = 0.f;
    stage_head(w, sp);
    float g[MNPARAM + 1];
#pragma unroll
    for (int j = 0; j <= MNPARAM; ++j) g[j] = 0.f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += (int64_t)gridDim.x * blockDim.x) {
        float f[MF], h[MH];
#pragma unroll
        for (int j = 0; j < MF; ++j) f[j] = feat[MF * i + j];
        const float s = move_score(sp, f, h);
        const float y = label[i] ? 1.f : 0.f;
        g[MNPARAM] += (fmaxf(s, 0.f) - s * y + log1pf(expf(-fabsf(s)))) * inv_n;
        const float ds = (1.f / (1.f + expf(-s)) - y) * inv_n;
        g[MO_B2] += ds;
#pragma unroll
        for (int k2 = 0; k2 < MH; ++k2) {
            const float a = h[k2];
            g[MO_W2 + k2] += ds * (a > 0.f ? a : 0.f);
            const float dh = a > 0.f ? ds * sp[MO_W2 + k2] : 0.f;
            g[MO_B1 + k2] += dh;
#pragma unroll
            for (int j = 0; j < MF; ++j) g[MO_W1 + k2 * MF + j] += dh * f[j];
        }
    }
#pragma unroll
    for (int j = 0; j <= MNPARAM; ++j) {
        float x = g[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&sg[j], x);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < MNPARAM; j += blockDim.x) atomicAdd(&grad[j], sg[j]);
    if (threadIdx.x == 0) atomicAdd(loss, sg[MNPARAM]);
}

bool gnn_has_move_head(const gp_gnn* G) { return G && G->move_head; }

// move priorities of one label-propagation step of the learned V-cycle
void gnn_move_priorities(Ctx& c, const gp_gnn* G, const DGraph& g, int level, const int32_t* dest,
                         const int32_t* gain, int32_t* mp) {
    k_move_prio<<<grid_for(g.n, 256, c.sm_count * 8), 256, 0, c.s>>>(g.n, g.rp, g.vw, dest, gain, level, G->mh_w16,
                                                                   mp);
    GP_LAUNCHED(c);
    c.bytes += 8 * (g.n + 1) + 16 * g.n;
}

// learned matching priorities of one level (called by the V-cycle driver)
void gnn_level_priorities(Ctx& c, const gp_gnn* G, const Level& L, int level, int32_t* prio) {
    auto mk = c.tmp->save();
    GnnActs A;
    gnn_forward(c, G, L, level, false, A);
    gnn_edges(c, G, L, A, prio, nullptr);
    c.tmp->restore(mk);
}

// BF16-rounded edge coefficients mirrored on the host (they travel as kernel arguments)
static void refresh_host_edge(gp_gnn* G, cudaStream_t s) {
    __nv_bfloat16 h[NEDGE];
    GP_CUDA(cudaMemcpyAsync(h, G->w16 + O_A, sizeof h, cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaStreamSynchronize(s));
    for (int j = 0; j < NEDGE; ++j) G->hedge[j] = __bfloat162float(h[j]);
}

// loss and gradients of one graph (gradients accumulated into G->grad)
static float gnn_grad(Ctx& c, gp_gnn* G, const Level& L, int level, const uint8_t* label) {
    const DGraph& g = L.g;
    const int64_t n = g.n;
    auto mk = c.tmp->save();
    GnnActs A;
    gnn_forward(c, G, L, level, true, A);
    float* dz = c.tmp_alloc<float>(ZD * n);
    float* dpre2 = c.tmp_alloc<float>(H * n);
    float* dh1 = c.tmp_alloc<float>(H * n);
    float* dc = c.tmp_alloc<float>(MSG * n);
    float* dm = c.tmp_alloc<float>(MSG * n);
    float* dpre1 = c.tmp_alloc<float>(H * n);
    float* xa = c.tmp_alloc<float>(2 * F0 * n);
    float* hc = c.tmp_alloc<float>((H + MSG) * n);
    float* loss = c.tmp_alloc<float>(1);
    memset_async(c, loss, 0, sizeof(float));
    const int wg = grid_for(n * 32, 256, c.sm_count * 8), tg = grid_for(n, 128, c.sm_count * 8);
    const float inv_e = g.m > 0 ? 1.f / (float)g.m : 0.f;
    k_gnn_edge_bwd<<<wg, 256, 0, c.s>>>(g, G->w16, A.z, A.wdeg, A.sig, label, inv_e, dz, G->grad, loss);
    GP_LAUNCHED(c);
    k_gnn_l2_bwd<<<tg, 128, 0, c.s>>>(n, G->w16, dz, A.h2, dpre2, dh1, dc);
    GP_LAUNCHED(c);
    k_gnn_msg_bwd<<<wg, 256, 0, c.s>>>(g, dc, dm);
    GP_LAUNCHED(c);
    k_gnn_l1_bwd<<<tg, 128, 0, c.s>>>(n, G->w16, dh1, dm, A.h1, dpre1);
    GP_LAUNCHED(c);
    const int cg = grid_for(n, OP_CHUNK, c.sm_count * 4);
    k_gnn_concat<<<grid_for(n * 2 * F0, 256), 256, 0, c.s>>>(n, A.x, F0, A.a, F0, xa);
    GP_LAUNCHED(c);
    k_gnn_concat<<<grid_for(n * (H + MSG), 256), 256, 0, c.s>>>(n, A.h1, H, A.c, MSG, hc);
    GP_LAUNCHED(c);
    auto outer = [&](const float* a, int ra, int R, const float* b, int rb, int C, int o) {
        const size_t smem = sizeof(float) * OP_CHUNK * (R + C);
        if (R * C > OP_THREADS * OP_PER_THREAD) throw GpError(GP_EINTERNAL, "outer product too large");
        k_gnn_outer<<<cg, OP_THREADS, smem, c.s>>>(n, a, ra, R, b, rb, C, G->grad, o);
        GP_LAUNCHED(c);
    };
    outer(dz, ZD, ZD, A.h2, H, H, O_Z);            // dZ = dz h2^T
    outer(dpre2, H, H, hc, H + MSG, H + MSG, O_W2); // dW2 = dpre2 [h1; c]^T
    outer(dpre2, H, H, nullptr, 0, 1, O_B2);        // db2
    outer(dm, MSG, MSG, A.h1, H, H, O_P);           // dP = dm h1^T
    outer(dpre1, H, H, xa, 2 * F0, 2 * F0, O_W1);   // dW1 = dpre1 [x; a]^T
    outer(dpre1, H, H, nullptr, 0, 1, O_B1);        // db1
    float h = 0.f;
    GP_CUDA(cudaMemcpyAsync(&h, loss, sizeof(float), cudaMemcpyDeviceToHost, c.s));
    c.sync();
    c.tmp->restore(mk);
    return h;
}

// per-call context on the current device (own stream and arenas)
// per-call context on the current device: the model's own arenas, the caller's stream
struct GnnCall {
    Ctx c;
    int64_t pinned[64];
    explicit GnnCall(gp_gnn* G, cudaStream_t s) {
        int dev = 0;
        GP_CUDA(cudaGetDevice(&dev));
        c.s = s;
        c.keep = &G->keep;
        c.tmp = &G->arena;
        GP_CUDA(cudaDeviceGetAttribute(&c.sm_count, cudaDevAttrMultiProcessorCount, dev));
        c.h_pinned = pinned;
    }
    ~GnnCall() { c.tmp->reset(); c.keep->reset(); }
};

// the row buckets of a graph scored outside a V-cycle
static Level level_of(Ctx& c, const DGraph& g) {
    Level L;
    L.g = g;
    build_heavy(c, L);
    return L;
}

static DGraph mkgraph(int64_t n, int64_t m, const int64_t* rp, const int32_t* ci, const int32_t* vw, const int32_t* ew) {
    DGraph g;
    g.n = n; g.m = m; g.rp = rp; g.ci = ci; g.vw = vw; g.ew = ew;
    return g;
}

template <class F>
static int gnn_guard(F&& f) {
    t_err.clear();
    try {
        f();
        return GP_OK;
    } catch (const GpError& e) {
        t_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        t_err = e.what();
        return GP_EINTERNAL;
    }
}

}  // namespace gp

using namespace gp;

extern "C" {

int gp_gnn_num_params(void) { return NPARAM; }

int gp_gnn_create(gp_gnn** out) {
    return gnn_guard([&] {
        if (!out) throw GpError(GP_EINVAL, "null handle pointer");
        gp_gnn* G = new gp_gnn();
        GP_CUDA(cudaMalloc(&G->master, sizeof(float) * NPARAM));
        GP_CUDA(cudaMalloc(&G->w16, sizeof(__nv_bfloat16) * NPARAM));
        GP_CUDA(cudaMalloc(&G->grad, sizeof(float) * NPARAM));
        GP_CUDA(cudaMalloc(&G->adam_m, sizeof(float) * NPARAM));
        GP_CUDA(cudaMalloc(&G->adam_v, sizeof(float) * NPARAM));
        GP_CUDA(cudaMemset(G->master, 0, sizeof(float) * NPARAM));
        GP_CUDA(cudaMemset(G->w16, 0, sizeof(__nv_bfloat16) * NPARAM));
        GP_CUDA(cudaMemset(G->grad, 0, sizeof(float) * NPARAM));
        GP_CUDA(cudaMemset(G->adam_m, 0, sizeof(float) * NPARAM));
        GP_CUDA(cudaMemset(G->adam_v, 0, sizeof(float) * NPARAM));
        *out = G;
    });
}

int gp_gnn_destroy(gp_gnn* G) {
    return gnn_guard([&] {
        if (!G) return;
        cudaFree(G->master); cudaFree(G->w16); cudaFree(G->grad); cudaFree(G->adam_m); cudaFree(G->adam_v);
        cudaFree(G->mh_master); cudaFree(G->mh_w16); cudaFree(G->mh_grad); cudaFree(G->mh_m); cudaFree(G->mh_v);
        delete G;
    });
}

// host FP32 parameters in (master copy; the kernels use their BF16 rounding)
int gp_gnn_set_params(gp_gnn* G, const float* params, int32_t np) {
    return gnn_guard([&] {
        if (!G || !params || np != NPARAM) throw GpError(GP_EINVAL, "bad parameter array");
        GP_CUDA(cudaMemcpy(G->master, params, sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
        k_gnn_to_bf16<<<grid_for(NPARAM, 256), 256>>>(NPARAM, G->master, G->w16);
        GP_CUDA(cudaGetLastError());
        GP_CUDA(cudaDeviceSynchronize());
        G->step = 0;
        GP_CUDA(cudaMemset(G->adam_m, 0, sizeof(float) * NPARAM));
        GP_CUDA(cudaMemset(G->adam_v, 0, sizeof(float) * NPARAM));
        refresh_host_edge(G, nullptr);
    });
}

int gp_gnn_set_prio_bits(gp_gnn* G, int32_t bits) {
    return gnn_guard([&] {
        if (!G || bits < 0 || bits > 16) throw GpError(GP_EINVAL, "prio bits must be in [0, 16]");
        G->prio_bits = bits;
    });
}

int gp_gnn_get_prio_bits(const gp_gnn* G) { return G ? G->prio_bits : -1; }

int gp_gnn_set_max_level(gp_gnn* G, int32_t level) {
    return gnn_guard([&] {
        if (!G || level < -1) throw GpError(GP_EINVAL, "max level must be >= -1");
        G->max_level = level;
    });
}

int gp_gnn_get_max_level(const gp_gnn* G) { return G ? G->max_level : -2; }

int gp_gnn_get_params(const gp_gnn* G, float* params, int32_t np) {
    return gnn_guard([&] {
        if (!G || !params || np != NPARAM) throw GpError(GP_EINVAL, "bad parameter array");
        GP_CUDA(cudaMemcpy(params, G->master, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
    });
}

// per-entry learned priorities (and logits) of one graph at `level`
int gp_gnn_forward_device(gp_gnn* G, int64_t n, const int64_t* d_rowptr, const int32_t* d_colidx,
                          const int32_t* d_vwgt, const int32_t* d_ewgt, int32_t level, void* stream,
                          int32_t* d_prio_out, float* d_logit_out) {
    return gnn_guard([&] {
        if (!G || n < 0) throw GpError(GP_EINVAL, "bad arguments");
        if (n == 0) return;
        if (!d_rowptr || !d_colidx) throw GpError(GP_EINVAL, "null array");
        GnnCall call(G, (cudaStream_t)stream);
        GP_CUDA(cudaMemcpyAsync(call.pinned, d_rowptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, call.c.s));
        call.c.sync();
        const DGraph g = mkgraph(n, call.pinned[0], d_rowptr, d_colidx, d_vwgt, d_ewgt);
        const Level L = level_of(call.c, g);
        GnnActs A;
        gnn_forward(call.c, G, L, level, false, A);
        gnn_edges(call.c, G, L, A, d_prio_out, d_logit_out);
        call.c.sync();
    });
}

// loss and gradient (host arrays) of one labelled graph; gradients are not accumulated across calls
int gp_gnn_grad_device(gp_gnn* G, int64_t n, const int64_t* d_rowptr, const int32_t* d_colidx, const int32_t* d_vwgt,
                       const int32_t* d_ewgt, int32_t level, const uint8_t* d_label, void* stream, float* loss_out,
                       float* grad_out) {
    return gnn_guard([&] {
        if (!G || n <= 0 || !d_label || !d_rowptr || !d_colidx) throw GpError(GP_EINVAL, "bad arguments");
        GnnCall call(G, (cudaStream_t)stream);
        GP_CUDA(cudaMemcpyAsync(call.pinned, d_rowptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, call.c.s));
        call.c.sync();
        const DGraph g = mkgraph(n, call.pinned[0], d_rowptr, d_colidx, d_vwgt, d_ewgt);
        GP_CUDA(cudaMemsetAsync(G->grad, 0, sizeof(float) * NPARAM, call.c.s));
        const float l = gnn_grad(call.c, G, level_of(call.c, g), level, d_label);
        if (loss_out) *loss_out = l;
        if (grad_out) GP_CUDA(cudaMemcpy(grad_out, G->grad, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
    });
}

// one Adam step on the summed gradients of `ngraphs` labelled graphs
int gp_gnn_train_step_device(gp_gnn* G, int32_t ngraphs, const int64_t* ns, const int64_t* const* d_rowptrs,
                             const int32_t* const* d_colidxs, const int32_t* const* d_vwgts,
                             const int32_t* const* d_ewgts, const int32_t* levels,
                             const uint8_t* const* d_labels, float lr, void* stream, float* loss_out) {
    return gnn_guard([&] {
        if (!G || ngraphs <= 0 || !ns || !d_rowptrs || !d_colidxs || !d_labels)
            throw GpError(GP_EINVAL, "bad arguments");
        GnnCall call(G, (cudaStream_t)stream);
        GP_CUDA(cudaMemsetAsync(G->grad, 0, sizeof(float) * NPARAM, call.c.s));
        float tot = 0.f;
        for (int32_t i = 0; i < ngraphs; ++i) {
            if (ns[i] <= 0) continue;
            GP_CUDA(cudaMemcpyAsync(call.pinned, d_rowptrs[i] + ns[i], sizeof(int64_t), cudaMemcpyDeviceToHost, call.c.s));
            call.c.sync();
            const DGraph g = mkgraph(ns[i], call.pinned[0], d_rowptrs[i], d_colidxs[i], d_vwgts ? d_vwgts[i] : nullptr,
                                     d_ewgts ? d_ewgts[i] : nullptr);
            auto km = call.c.keep->save();
            tot += gnn_grad(call.c, G, level_of(call.c, g), levels ? levels[i] : 0, d_labels[i]);
            call.c.keep->restore(km);
        }
        G->step += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - powf(b1, (float)G->step), c2 = 1.f - powf(b2, (float)G->step);
        k_gnn_adam<<<grid_for(NPARAM, 256), 256, 0, call.c.s>>>(NPARAM, G->master, G->w16, G->grad, G->adam_m,
                                                                G->adam_v, lr, b1, b2, 1e-8f, c1, c2);
        GP_LAUNCHED(call.c);
        refresh_host_edge(G, call.c.s);
        if (loss_out) *loss_out = tot / (float)ngraphs;
    });
}

// ---- move-order head
int gp_gnn_move_num_params(void) { return MNPARAM; }

int gp_gnn_set_move_params(gp_gnn* G, const float* params, int32_t np) {
    return gnn_guard([&] {
        if (!G) throw GpError(GP_EINVAL, "null model");
        if (np == 0) { G->move_head = 0; return; }
        if (!params || np != MNPARAM) throw GpError(GP_EINVAL, "bad move-head parameter array");
        if (!G->mh_master) {
            GP_CUDA(cudaMalloc(&G->mh_master, sizeof(float) * MNPARAM));
            GP_CUDA(cudaMalloc(&G->mh_w16, sizeof(__nv_bfloat16) * MNPARAM));
            GP_CUDA(cudaMalloc(&G->mh_grad, sizeof(float) * (MNPARAM + 1)));   // + the loss
            GP_CUDA(cudaMalloc(&G->mh_m, sizeof(float) * MNPARAM));
            GP_CUDA(cudaMalloc(&G->mh_v, sizeof(float) * MNPARAM));
        }
        GP_CUDA(cudaMemcpy(G->mh_master, params, sizeof(float) * MNPARAM, cudaMemcpyHostToDevice));
        k_gnn_to_bf16<<<1, 128>>>(MNPARAM, G->mh_master, G->mh_w16);
        GP_CUDA(cudaGetLastError());
        GP_CUDA(cudaMemset(G->mh_m, 0, sizeof(float) * MNPARAM));
        GP_CUDA(cudaMemset(G->mh_v, 0, sizeof(float) * MNPARAM));
        GP_CUDA(cudaDeviceSynchronize());
        G->mh_step = 0;
        G->move_head = 1;
    });
}

int gp_gnn_get_move_params(const gp_gnn* G, float* params, int32_t np) {
    return gnn_guard([&] {
        if (!G || !params || np != MNPARAM) throw GpError(GP_EINVAL, "bad move-head parameter array");
        if (!G->move_head) throw GpError(GP_EINVAL, "the model has no move-order head");
        GP_CUDA(cudaMemcpy(params, G->mh_master, sizeof(float) * MNPARAM, cudaMemcpyDeviceToHost));
    });
}

int gp_gnn_move_features_device(int64_t n, const int64_t* d_rowptr, const int32_t* d_vwgt, const int32_t* d_dest,
                                const int32_t* d_gain, int32_t level, void* stream, float* d_feat_out) {
    return gnn_guard([&] {
        if (n < 0 || (n > 0 && (!d_rowptr || !d_dest || !d_gain || !d_feat_out))) throw GpError(GP_EINVAL, "bad arguments");
        if (n == 0) return;
        k_move_feat<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, d_rowptr, d_vwgt, d_dest, d_gain, level,
                                                                       d_feat_out);
        GP_CUDA(cudaGetLastError());
        GP_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    });
}

int gp_gnn_move_scores_device(gp_gnn* G, int64_t ns, const float* d_feat, void* stream, float* d_score_out,
                              int32_t* d_prio_out) {
    return gnn_guard([&] {
        if (!G || !G->move_head) throw GpError(GP_EINVAL, "the model has no move-order head");
        if (ns < 0 || (ns > 0 && !d_feat)) throw GpError(GP_EINVAL, "bad arguments");
        if (ns == 0) return;
        k_move_score<<<grid_for(ns, 256), 256, 0, (cudaStream_t)stream>>>(ns, d_feat, G->mh_w16, d_score_out,
                                                                         d_prio_out);
        GP_CUDA(cudaGetLastError());
        GP_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    });
}

static float move_grad(gp_gnn* G, int64_t ns, const float* d_feat, const uint8_t* d_label, cudaStream_t s) {
    GP_CUDA(cudaMemsetAsync(G->mh_grad, 0, sizeof(float) * (MNPARAM + 1), s));
    float* d_loss = G->mh_grad + MNPARAM;
    if (ns > 0) {
        k_move_grad<<<grid_for(ns, 256, 148 * 4), 256, 0, s>>>(ns, d_feat, d_label, G->mh_w16, 1.f / (float)ns,
                                                               G->mh_grad, d_loss);
        GP_CUDA(cudaGetLastError());
    }
    float h = 0.f;
    GP_CUDA(cudaMemcpyAsync(&h, d_loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    GP_CUDA(cudaStreamSynchronize(s));
    return h;
}

int gp_gnn_move_grad_device(gp_gnn* G, int64_t ns, const float* d_feat, const uint8_t* d_label, void* stream,
                            float* loss_out, float* grad_out) {
    return gnn_guard([&] {
        if (!G || !G->move_head) throw GpError(GP_EINVAL, "the model has no move-order head");
        if (ns < 0 || (ns > 0 && (!d_feat || !d_label))) throw GpError(GP_EINVAL, "bad arguments");
        const float l = move_grad(G, ns, d_feat, d_label, (cudaStream_t)stream);
        if (loss_out) *loss_out = l;
        if (grad_out) GP_CUDA(cudaMemcpy(grad_out, G->mh_grad, sizeof(float) * MNPARAM, cudaMemcpyDeviceToHost));
    });
}

int gp_gnn_move_train_step_device(gp_gnn* G, int64_t ns, const float* d_feat, const uint8_t* d_label, float lr,
                                  void* stream, float* loss_out) {
    return gnn_guard([&] {
        if (!G || !G->move_head) throw GpError(GP_EINVAL, "the model has no move-order head");
        if (ns <= 0 || !d_feat || !d_label) throw GpError(GP_EINVAL, "bad arguments");
        cudaStream_t s = (cudaStream_t)stream;
        const float l = move_grad(G, ns, d_feat, d_label, s);
        G->mh_step += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - powf(b1, (float)G->mh_step), c2 = 1.f - powf(b2, (float)G->mh_step);
        k_gnn_adam<<<1, 128, 0, s>>>(MNPARAM, G->mh_master, G->mh_w16, G->mh_grad, G->mh_m, G->mh_v, lr, b1, b2,
                                     1e-8f, c1, c2);
        GP_CUDA(cudaGetLastError());
        GP_CUDA(cudaStreamSynchronize(s));
        if (loss_out) *loss_out = l;
    });
}

}  // extern "C"
