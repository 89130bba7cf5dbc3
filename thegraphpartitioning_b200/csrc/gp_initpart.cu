// gp_initpart.cu -- GPU initial partition of the coarsest graph.
//
// Replaces convertCSRtoMETISandRun + the `gpmetis -ptype=rb` subprocess and the
// partition-file read-back (src/gpu_part.cu:803-864, 1157-1185).  One CTA runs
// one seeded trial of recursive bisection entirely on chip-resident control
// state: at each depth every label with more than one part is split by
//   1. seed = vertex of the label with the smallest (top-32 hash bits, id),
//   2. BFS inside the label from the seed; the farthest vertex (smallest id on
//      ties) becomes the pseudo-peripheral start,
//   3. BFS from the start; vertices are ordered by (distance, id), unreached
//      ones last,
//   4. the left side is the longest prefix of that order whose weight is at
//      most target = W_label * left_parts / parts, plus the next vertex when
//      that lands strictly closer to the target.
// The prefix is found without sorting: a per-label binary search over the key
// domain (distance * n + id) with shared-memory weight sums.  Labels are part
// ranges identified by their first part.  Trials run in parallel, one per CTA;
// the kept trial is the balanced one with the lowest cut (lowest trial id on
// ties), else the one with the smallest heaviest part.
#define GP_TU_ID 3   // site ids of the bounds-checked build
#include "gp_internal.cuh"

namespace gp {

constexpr int IP_T = 1024;
constexpr int32_t IP_INF = 0x7fffffff;

struct IpShared {
    int32_t* cnt;     // parts per label (label = first part)
    int32_t* cnt_d;   // snapshot at the start of a depth
    int32_t* incl;
    int64_t* WL;
    int64_t* target;
    uint64_t* s0;
    uint64_t* pk;
    int64_t* lo;
    int64_t* hi;
    int64_t* flo;
    int64_t* fsum;
    int64_t* xw;
};

// Adds w to sum[L] for every lane of the warp, one shared-memory atomic per
// distinct label in the warp (lanes of one label are combined by match_any +
// reduce).  L < 0: the lane adds nothing.  Exact: a label's weights total at
// most the graph's vertex weight, which fits in 32 bits.
__device__ __forceinline__ void ip_label_add(int64_t* sum, int32_t L, uint32_t w) {
    const uint32_t peers = __match_any_sync(0xffffffffu, (uint32_t)L);
    const uint32_t tot = __reduce_add_sync(peers, L >= 0 ? w : 0u);
    const int lane = threadIdx.x & 31;
    if (L >= 0 && lane == __ffs(peers) - 1 && tot) atomicAdd((unsigned long long*)&sum[L], (unsigned long long)tot);
}

// atomicMin (MAX = false) or atomicMax (MAX = true) of 64-bit keys into
// slot[L], one shared-memory atomic per distinct label in the warp.  L < 0:
// the lane takes no part.
template <bool MAX>
__device__ __forceinline__ void ip_label_ext(uint64_t* slot, int32_t L, uint64_t key) {
    const uint32_t peers = __match_any_sync(0xffffffffu, (uint32_t)L);
    const uint32_t hi = (uint32_t)(key >> 32), lo = (uint32_t)key;
    const uint32_t ident = MAX ? 0u : 0xffffffffu;
    const uint32_t bh = MAX ? __reduce_max_sync(peers, L >= 0 ? hi : ident) : __reduce_min_sync(peers, L >= 0 ? hi : ident);
    const uint32_t cand = (L >= 0 && hi == bh) ? lo : ident;
    const uint32_t bl = MAX ? __reduce_max_sync(peers, cand) : __reduce_min_sync(peers, cand);
    const int lane = threadIdx.x & 31;
    if (L >= 0 && lane == __ffs(peers) - 1) {
        const unsigned long long best = ((unsigned long long)bh << 32) | bl;
        if (MAX) atomicMax((unsigned long long*)&slot[L], best);
        else atomicMin((unsigned long long*)&slot[L], best);
    }
}

__device__ __forceinline__ int64_t ip_key(int32_t d, int64_t v, int64_t n) {
    return (int64_t)(d == IP_INF ? n : d) * n + v;
}

// BFS inside each splitting label from src (stored as vertex id in srcs[label]);
// dist[] must be IP_INF for all vertices of splitting labels except sources.
__device__ void ip_bfs(const DGraph& g, const int32_t* lab, int32_t* dist, const IpShared& S, int* flags) {
    const int64_t n = g.n;
    if (threadIdx.x == 0) { flags[0] = 0; flags[1] = 0; flags[2] = 0; }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int32_t r = 0;; ++r) {
        // one warp per frontier vertex: rows of the coarsest graph can be long
        for (int64_t v = wid; v < n; v += nw) {
            const int32_t L = lab[v];
            if (S.cnt_d[L] <= 1 || dist[v] != r) continue;
            for (int64_t e = g.rp[v] + lane; e < g.rp[v + 1]; e += 32) {
                const int32_t u = g.ci[e];
                if (lab[u] == L && dist[u] == IP_INF) { dist[u] = r + 1; flags[r % 3] = 1; }
            }
        }
        if (threadIdx.x == 0) flags[(r + 1) % 3] = 0;
        __syncthreads();
        if (!flags[r % 3]) break;
    }
    __syncthreads();
}

// labels and distances live in shared memory when they fit (on_chip), else in
// the trial's slices of the global arrays; the kept labels are written out
__global__ void __launch_bounds__(IP_T) k_initpart(DGraph g, int32_t k, uint64_t seed, int32_t* __restrict__ labels,
                                                    int32_t* __restrict__ dists, int64_t* __restrict__ tcut,
                                                    int64_t* __restrict__ tmaxpw, int key_iters, int on_chip) {
    extern __shared__ int64_t ipsm[];
    __shared__ int flags[3];
    __shared__ int any;
    __shared__ int64_t red[IP_T / 32];
    const int64_t n = g.n;
    const int t = blockIdx.x;
    IpShared S;
    {
        int64_t* p = ipsm;
        S.WL = p; p += k; S.target = p; p += k; S.lo = p; p += k; S.hi = p; p += k;
        S.flo = p; p += k; S.fsum = p; p += k; S.xw = p; p += k;
        S.s0 = (uint64_t*)p; p += k; S.pk = (uint64_t*)p; p += k;
        int32_t* q = (int32_t*)p;
        S.cnt = q; q += k; S.cnt_d = q; q += k; S.incl = q; q += k;
    }
    int32_t* glab = labels + (int64_t)t * n;
    int32_t* lab = glab;
    int32_t* dist = dists + (int64_t)t * n;
    if (on_chip) {
        int32_t* q = (int32_t*)(ipsm + 9 * (int64_t)k) + 3 * (int64_t)k;
        lab = q;
        dist = q + n;
    }
    const uint64_t ts = trial_salt(seed, t);
    for (int64_t v = threadIdx.x; v < n; v += blockDim.x) lab[v] = 0;
    for (int q = threadIdx.x; q < k; q += blockDim.x) S.cnt[q] = (q == 0) ? k : 0;
    __syncthreads();
    for (int d = 0;; ++d) {
        if (threadIdx.x == 0) any = 0;
        __syncthreads();
        for (int q = threadIdx.x; q < k; q += blockDim.x) {
            S.cnt_d[q] = S.cnt[q];
            if (S.cnt[q] > 1) any = 1;
            S.WL[q] = 0; S.s0[q] = ~0ull; S.pk[q] = 0;
        }
        __syncthreads();
        if (!any) break;
        const uint64_t ds = depth_salt(ts, d);
        // label weights and seeds (warp-uniform trip count for the label sums)
        for (int64_t v0 = threadIdx.x & ~31; v0 < n; v0 += blockDim.x) {
            const int64_t v = v0 + (threadIdx.x & 31);
            int32_t L = v < n ? lab[v] : -1;
            if (L >= 0 && S.cnt_d[L] <= 1) L = -1;
            ip_label_add(S.WL, L, L >= 0 ? (uint32_t)(g.vw ? g.vw[v] : 1) : 0u);
            const uint64_t h = L >= 0 ? (((mix64(ds ^ (uint64_t)(uint32_t)v) >> 32) << 32) | (uint32_t)v) : ~0ull;
            ip_label_ext<false>(S.s0, L, h);
        }
        __syncthreads();
        // BFS 1 from the seed
        for (int64_t v = threadIdx.x; v < n; v += blockDim.x) {
            const int32_t L = lab[v];
            if (S.cnt_d[L] <= 1) continue;
            dist[v] = ((S.s0[L] & 0xffffffffull) == (uint64_t)v) ? 0 : IP_INF;
        }
        __syncthreads();
        ip_bfs(g, lab, dist, S, flags);
        // pseudo-peripheral vertex: max distance, smallest id
        for (int64_t v0 = threadIdx.x & ~31; v0 < n; v0 += blockDim.x) {
            const int64_t v = v0 + (threadIdx.x & 31);
            int32_t L = v < n ? lab[v] : -1;
            if (L >= 0 && (S.cnt_d[L] <= 1 || dist[v] == IP_INF)) L = -1;
            const uint64_t key = L >= 0 ? (((uint64_t)(uint32_t)dist[v] << 32) | (uint64_t)(0xffffffffu - (uint32_t)v)) : 0ull;
            ip_label_ext<true>(S.pk, L, key);
        }
        __syncthreads();
        for (int64_t v = threadIdx.x; v < n; v += blockDim.x) {
            const int32_t L = lab[v];
            if (S.cnt_d[L] <= 1) continue;
            const uint32_t src = 0xffffffffu - (uint32_t)(S.pk[L] & 0xffffffffull);
            dist[v] = ((uint32_t)v == src) ? 0 : IP_INF;
        }
        __syncthreads();
        ip_bfs(g, lab, dist, S, flags);
        // binary search of the split key per label
        for (int q = threadIdx.x; q < k; q += blockDim.x) {
            const int32_t c = S.cnt_d[q];
            if (c > 1) {
                S.target[q] = S.WL[q] * (c / 2) / c;
                S.lo[q] = 0; S.hi[q] = n * (n + 1); S.flo[q] = 0; S.xw[q] = 0;
            }
        }
        __syncthreads();
        for (int it = 0; it < key_iters; ++it) {
            for (int q = threadIdx.x; q < k; q += blockDim.x) S.fsum[q] = 0;
            __syncthreads();
            for (int64_t v0 = threadIdx.x & ~31; v0 < n; v0 += blockDim.x) {
                const int64_t v = v0 + (threadIdx.x & 31);
                int32_t L = v < n ? lab[v] : -1;
                if (L >= 0 && S.cnt_d[L] <= 1) L = -1;
                bool below = false;
                if (L >= 0) below = ip_key(dist[v], v, n) < ((S.lo[L] + S.hi[L]) >> 1);
                ip_label_add(S.fsum, below ? L : -1, below ? (uint32_t)(g.vw ? g.vw[v] : 1) : 0u);
            }
            __syncthreads();
            for (int q = threadIdx.x; q < k; q += blockDim.x) {
                if (S.cnt_d[q] <= 1 || S.hi[q] - S.lo[q] <= 1) continue;
                const int64_t mid = (S.lo[q] + S.hi[q]) >> 1;
                if (S.fsum[q] <= S.target[q]) { S.lo[q] = mid; S.flo[q] = S.fsum[q]; }
                else S.hi[q] = mid;
            }
            __syncthreads();
        }
        for (int64_t v = threadIdx.x; v < n; v += blockDim.x) {
            const int32_t L = lab[v];
            if (S.cnt_d[L] <= 1) continue;
            if (ip_key(dist[v], v, n) == S.lo[L]) S.xw[L] = g.vw ? g.vw[v] : 1;
        }
        __syncthreads();
        for (int q = threadIdx.x; q < k; q += blockDim.x) {
            const int32_t c = S.cnt_d[q];
            if (c > 1) {
                S.incl[q] = (S.xw[q] > 0 && 2 * S.target[q] > 2 * S.flo[q] + S.xw[q]) ? 1 : 0;
                S.cnt[q] = c / 2;
                S.cnt[q + c / 2] = c - c / 2;
            }
        }
        __syncthreads();
        for (int64_t v = threadIdx.x; v < n; v += blockDim.x) {
            const int32_t L = lab[v];
            const int32_t c = S.cnt_d[L];
            if (c <= 1) continue;
            const int64_t key = ip_key(dist[v], v, n);
            const bool left = key < S.lo[L] || (key == S.lo[L] && S.incl[L]);
            if (!left) lab[v] = L + c / 2;
        }
        __syncthreads();
    }
    // evaluate the trial: cut and heaviest part
    for (int q = threadIdx.x; q < k; q += blockDim.x) S.WL[q] = 0;
    __syncthreads();
    int64_t cross = 0;
    {
        const int lane = threadIdx.x & 31;
        for (int64_t v = threadIdx.x >> 5; v < n; v += blockDim.x >> 5) {
            const int32_t p = lab[v];
            if (lane == 0) atomicAdd((unsigned long long*)&S.WL[p], (unsigned long long)(g.vw ? g.vw[v] : 1));
            for (int64_t e = g.rp[v] + lane; e < g.rp[v + 1]; e += 32)
                if (lab[g.ci[e]] != p) cross += g.ew ? g.ew[e] : 1;
        }
    }
    for (int o = 16; o > 0; o >>= 1) cross += __shfl_xor_sync(0xffffffffu, cross, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cross;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t s = 0;
        for (int i = 0; i < IP_T / 32; ++i) s += red[i];
        int64_t mp = 0;
        for (int q = 0; q < k; ++q) mp = S.WL[q] > mp ? S.WL[q] : mp;
        tcut[t] = s / 2;
        tmaxpw[t] = mp;
    }
    if (on_chip)
        for (int64_t v = threadIdx.x; v < n; v += blockDim.x) glab[v] = lab[v];
}

__global__ void k_pick_trial(int T, const int64_t* __restrict__ tcut, const int64_t* __restrict__ tmaxpw, int64_t Lmax,
                             int64_t* __restrict__ best) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int bt = 0;
    for (int t = 1; t < T; ++t) {
        const bool bal = tmaxpw[t] <= Lmax, bbal = tmaxpw[bt] <= Lmax;
        bool better;
        if (bal != bbal) better = bal;
        else if (!bal && tmaxpw[t] != tmaxpw[bt]) better = tmaxpw[t] < tmaxpw[bt];
        else better = tcut[t] < tcut[bt];
        if (better) bt = t;
    }
    best[0] = bt;
}

static int bits_for64(int64_t x) {
    int b = 1;
    while (b < 63 && (1ll << b) < x) ++b;
    return b;
}

size_t initpart_smem_max();

int initial_partition(Ctx& c, const Level& L, const Params& P, int32_t* part_out) {
    const int64_t n = L.g.n;
    const int T = P.o.init_trials;
    auto mk = c.tmp->save();
    int32_t* labels = c.tmp_alloc<int32_t>((int64_t)T * n);
    int32_t* dists = c.tmp_alloc<int32_t>((int64_t)T * n);
    int64_t* tcut = c.tmp_alloc<int64_t>(T);
    int64_t* tmaxpw = c.tmp_alloc<int64_t>(T);
    int64_t* best = c.tmp_alloc<int64_t>(1);
    const size_t base = (size_t)P.k * (9 * sizeof(int64_t) + 3 * sizeof(int32_t));
    const size_t onchip = base + 2 * sizeof(int32_t) * (size_t)n;
    const bool on_chip = onchip <= initpart_smem_max();
    const size_t smem = on_chip ? onchip : base;
    const int key_iters = bits_for64(n * (n + 1)) + 1;
    k_initpart<<<T, IP_T, smem, c.s>>>(L.g, P.k, P.seed, labels, dists, tcut, tmaxpw, key_iters, on_chip ? 1 : 0);
    GP_LAUNCHED(c);
    k_pick_trial<<<1, 32, 0, c.s>>>(T, tcut, tmaxpw, P.Lmax, best);
    GP_LAUNCHED(c);
    const int bt = (int)read_i64(c, best);
    GP_CUDA(cudaMemcpyAsync(part_out, labels + (int64_t)bt * n, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, c.s));
    c.bytes += (int64_t)T * (L.scan_bytes() * 4 + 8 * n);
    c.tmp->restore(mk);
    return bt;
}

// k_initpart may use the whole opt-in shared memory of a block (per-label
// arrays, plus labels and distances when they fit); set once per device (the
// cap is per kernel, shared by every thread of the process)
static size_t g_ip_smem_max = 0;

size_t initpart_smem_max() { return g_ip_smem_max; }

void initpart_smem_caps() {
    int dev = 0, optin = 0;
    GP_CUDA(cudaGetDevice(&dev));
    GP_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t need = (size_t)GP_MAX_K * (9 * sizeof(int64_t) + 3 * sizeof(int32_t));
    // static shared memory of the kernel (flags, reductions) stays outside the cap
    const size_t cap = std::max(need, (size_t)optin > 4096 ? (size_t)optin - 4096 : need);
    GP_CUDA(cudaFuncSetAttribute(k_initpart, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap));
    g_ip_smem_max = cap;
}

}  // namespace gp
