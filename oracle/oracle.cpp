// oracle.cpp -- CPU oracle of the deterministic multilevel k-way V-cycle.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
// calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg do, and only as the checker (or as the timed CPU baseline).
//
// It is a plain sequential restatement of the rules that the CUDA kernels in
// thegraphpartitioning_b200/csrc implement in parallel.  The reference
// (iamrupamroyy/TheGraphPartitioning, src/gpu_part.cu) is non-deterministic
// (atomic claim order in matchVertices, atomic slot order in
// bufferCandidateMoves/selectMoves) and its contraction is structurally wrong
// (countUniqueEdges runs over coarse ids with fine rows), so it cannot serve as
// a bit-exact oracle.  Each function below cites the reference step whose
// intent it restates and states the deterministic rule used instead.  Partition
// results are therefore not pinned by reference outputs; they are pinned by
// known-answer tests (grids, paths, disjoint cliques) and by exact invariants.
//
// Everything is integer: weights are int32 with int32-bounded totals, gains
// are exact, cuts are int64.  The only floating-point step is the balance
// bound Lmax = floor((1+eps)*W/k), computed in double once per call by the
// same expression on both sides.

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <string>
#include <vector>
#include <cmath>
#include <climits>

#include "../include/gp_partition.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) { g_err = msg; return code; }

struct Graph {
    int64_t n = 0;
    std::vector<int64_t> rp;
    std::vector<int32_t> ci, ew, vw;
    int64_t m() const { return rp[n]; }
};

// ---------------------------------------------------------------- hashing
// splitmix64 finalizer (Steele, Lea, Flood 2014; constants of Stafford's
// "Mix13" variant as published with splitmix64).
inline uint64_t mix64(uint64_t x) {
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27; x *= 0x94d049bb133111ebULL;
    x ^= x >> 31; return x;
}
inline uint64_t level_salt(uint64_t seed, int level) {
    return mix64(seed ^ mix64(0x9E3779B97F4A7C15ULL * (uint64_t)(level + 1)));
}
// MurmurHash3's 32-bit finalizer (Appleby; its published constants).
inline uint32_t fmix32(uint32_t h) {
    h ^= h >> 16; h *= 0x85EBCA6Bu;
    h ^= h >> 13; h *= 0xC2B2AE35u;
    h ^= h >> 16; return h;
}
// The matching tie-break of a level is salted with the level salt's high half.
inline uint32_t edge_salt(uint64_t seed, int level) { return (uint32_t)(level_salt(seed, level) >> 32); }
// Symmetric per-edge tie-break hash: both endpoints see the same value.  The
// ordered ids are spread by two odd constants (the 32-bit golden ratio and
// xxHash's PRIME32_2), summed with the salt modulo 2^32 and finalized.
inline uint32_t edge_hash(uint32_t salt, int32_t a, int32_t b) {
    uint32_t lo = (uint32_t)std::min(a, b), hi = (uint32_t)std::max(a, b);
    return fmix32(lo * 0x9E3779B1u + hi * 0x85EBCA77u + salt);
}
// Matching priority of an edge: heavier first, then the hash.
inline uint64_t edge_key(int32_t w, uint32_t h) { return ((uint64_t)(uint32_t)w << 32) | h; }

inline uint64_t trial_salt(uint64_t seed, int t) {
    return mix64(seed ^ mix64(0xD1B54A32D192ED03ULL * (uint64_t)(t + 1)));
}
inline uint64_t depth_salt(uint64_t tsalt, int d) {
    return mix64(tsalt ^ mix64(0x8CB92BA72F3D8DD7ULL * (uint64_t)(d + 1)));
}

// Monotone log-scale bucket of a rebalancing loss (10 bits, [1, 959]).
inline uint32_t mag_bucket(uint32_t x) {
    if (x < 64) return x;
    int e = 31 - __builtin_clz(x);
    uint32_t mant = (x >> (e - 4)) & 15u;
    return 64u + (uint32_t)(e - 6) * 16u + mant;
}
inline uint32_t loss_bucket(int32_t loss) {
    if (loss >= 0) return 480u + mag_bucket((uint32_t)loss);
    return 480u - mag_bucket((uint32_t)(-(int64_t)loss));
}

// ------------------------------------------------------------ parameters
// Per-level matching priorities (learned mode): prio(user, level, m) returns
// one int32 per directed entry of that level's graph, or NULL for the edge
// weights.  The priorities are an input here: the oracle checks that the
// integer decisions taken from them are the same on both sides.
typedef const int32_t* (*prio_fn_t)(void* user, int32_t level, int64_t m);
// Per-step move priorities (learned move order): mprio(user, level, iter, n)
// returns one int32 per vertex for the label-propagation step `iter` of
// `level`, or NULL for the (gain, id) order.  An input, like prio.
typedef const int32_t* (*mprio_fn_t)(void* user, int32_t level, int32_t iter, int64_t n);

struct Params {
    int32_t k;
    int64_t W;       // total vertex weight
    int64_t Lmax;    // max allowed part weight
    uint64_t seed;
    gp_options o;
    int64_t maxvw;   // coarse vertex weight cap
    prio_fn_t prio = nullptr;
    void* prio_user = nullptr;
    mprio_fn_t mprio = nullptr;
    void* mprio_user = nullptr;
};

void resolve_options(const gp_options* in, int64_t n, int32_t k, gp_options* o) {
    gp_options d;
    memset(&d, 0, sizeof d);
    if (in) d = *in;
    d.version = GP_OPTIONS_VERSION;
    if (d.coarsen_to <= 0) d.coarsen_to = (int32_t)std::max<int64_t>(1024, 32LL * k);
    if (d.match_rounds <= 0) d.match_rounds = 4;
    if (d.two_hop == 0) d.two_hop = 1;          // <0: off
    if (d.init_trials <= 0) d.init_trials = 64;
    if (d.refine_max_iters <= 0) d.refine_max_iters = 64;
    if (d.refine_patience <= 0) d.refine_patience = 4;
    if (d.lp_filter_den <= 0) d.lp_filter_den = 4;
    if (d.strong_after <= 0) d.strong_after = 2;
    if (d.check_input == 0) d.check_input = 1;  // <0: no structural checks
    (void)n;
    *o = d;
}

int64_t compute_lmax(int64_t W, int32_t k, float imbalance) {
    double lim = (1.0 + (double)imbalance) * (double)W / (double)k;
    int64_t l = (int64_t)std::floor(lim);
    int64_t avg = (W + k - 1) / k;
    return std::max(l, avg);
}

// ------------------------------------------------------------ tracing
struct Tracer {
    gp_trace_fn fn = nullptr;
    void* user = nullptr;
    void emit(const gp_trace_event& e) const { if (fn) fn(user, &e); }
};

// ------------------------------------------------------------ metrics
// Exact cut: sum of directed cross entries / 2.  Follows compute_edgecut
// (src/gpu_part.cu:400-423, 468) with an int64 accumulator.
int64_t edge_cut(const Graph& g, const std::vector<int32_t>& part) {
    int64_t s = 0;
    for (int64_t v = 0; v < g.n; ++v)
        for (int64_t e = g.rp[v]; e < g.rp[v + 1]; ++e)
            if (part[g.ci[e]] != part[v]) s += g.ew[e];
    return s / 2;
}
void part_weights(const Graph& g, const std::vector<int32_t>& part, int32_t k, std::vector<int64_t>& pw) {
    pw.assign(k, 0);
    for (int64_t v = 0; v < g.n; ++v) pw[part[v]] += g.vw[v];
}
int64_t max_of(const std::vector<int64_t>& a) {
    int64_t m = 0;
    for (int64_t x : a) m = std::max(m, x);
    return m;
}

// ------------------------------------------------------------ matching
// Restates the intent of matchVertices/rematchVertices (src/gpu_part.cu:55-106)
// and the host convergence loop (src/gpu_part.cu:1014-1046): heavy-edge
// matching.  Deterministic rule instead of the atomicCAS claim: in each round
// every unmatched vertex proposes to its eligible unmatched neighbour of
// highest priority edge_key(w, edge_hash) (ties: lower id); a pair is matched
// when the proposals are mutual.  Rounds stop when one adds no pair or after
// match_rounds.  Eligible: combined vertex weight <= maxvw.
// Then, when the level would shrink by less than a quarter, leftover vertices
// that share the same anchor (their top-priority neighbour, matched or not)
// are paired in id order within each anchor group (two-hop pairing).
std::vector<int32_t> match_level(const Graph& g, int level, const Params& P, int* rounds_out, int64_t* pairs_out) {
    const int64_t n = g.n;
    const uint32_t salt = edge_salt(P.seed, level);
    const int32_t* pr = P.prio ? P.prio(P.prio_user, level, g.m()) : nullptr;
    const int32_t* key_w = pr ? pr : g.ew.data();   // high word of the matching priority
    std::vector<int32_t> match(n, -1), prop(n, -1);
    int64_t pairs = 0;
    int rounds = 0;
    for (int r = 0; r < P.o.match_rounds; ++r) {
        for (int64_t v = 0; v < n; ++v) {
            prop[v] = -1;
            if (match[v] != -1) continue;
            int32_t best = -1;
            uint64_t bk = 0;
            for (int64_t e = g.rp[v]; e < g.rp[v + 1]; ++e) {
                int32_t u = g.ci[e];
                if (u == v || match[u] != -1) continue;
                if ((int64_t)g.vw[v] + g.vw[u] > P.maxvw) continue;
                uint64_t key = edge_key(key_w[e], edge_hash(salt, (int32_t)v, u));
                if (best < 0 || key > bk || (key == bk && u < best)) { bk = key; best = u; }
            }
            prop[v] = best;
        }
        int64_t newp = 0;
        for (int64_t v = 0; v < n; ++v) {
            if (match[v] != -1) continue;
            int32_t u = prop[v];
            if (u >= 0 && prop[u] == v) { match[v] = u; if (v < u) ++newp; }
        }
        rounds = r + 1;
        pairs += newp;
        if (newp == 0) break;
    }
    if (P.o.two_hop > 0 && 4 * (n - pairs) > 3 * n) {
        // anchor = top-priority neighbour over all neighbours
        std::vector<std::pair<int32_t, int32_t>> lst;  // (anchor, v)
        for (int64_t v = 0; v < n; ++v) {
            if (match[v] != -1 || g.rp[v] == g.rp[v + 1]) continue;
            int32_t best = -1;
            uint64_t bk = 0;
            for (int64_t e = g.rp[v]; e < g.rp[v + 1]; ++e) {
                int32_t u = g.ci[e];
                if (u == v) continue;
                uint64_t key = edge_key(key_w[e], edge_hash(salt, (int32_t)v, u));
                if (best < 0 || key > bk || (key == bk && u < best)) { bk = key; best = u; }
            }
            if (best >= 0) lst.push_back({best, (int32_t)v});
        }
        std::sort(lst.begin(), lst.end());
        size_t i = 0;
        while (i < lst.size()) {
            size_t j = i;
            while (j < lst.size() && lst[j].first == lst[i].first) ++j;
            for (size_t a = i; a + 1 < j; a += 2) {
                int32_t x = lst[a].second, y = lst[a + 1].second;
                if ((int64_t)g.vw[x] + g.vw[y] <= P.maxvw) { match[x] = y; match[y] = x; ++pairs; }
            }
            i = j;
        }
    }
    if (rounds_out) *rounds_out = rounds;
    if (pairs_out) *pairs_out = pairs;
    return match;
}

// ------------------------------------------------------------ contraction
// Restates mapVertices + relabel_coarse_vertices_kernel + countUniqueEdges +
// prefix_sum + fillEdgeArrays (src/gpu_part.cu:109-242): the coarse vertex of
// a pair {a<b} is represented by a; coarse ids are an exclusive scan of the
// representative flags in vertex order (not an atomic counter); the coarse
// row of c lists the coarse neighbours met while walking N(a) then N(b) in
// CSR order, mapped through cmap, without c itself, each at the position of
// its first occurrence, with the weights of all its occurrences summed (not
// a 64-bit mod mask that drops colliding neighbours); coarse vertex weight =
// sum of the fine weights (the reference keeps none).
void contract(const Graph& g, const std::vector<int32_t>& match, std::vector<int32_t>& cmap, Graph& cg) {
    const int64_t n = g.n;
    cmap.assign(n, -1);
    std::vector<int32_t> first, second;
    int64_t nc = 0;
    for (int64_t v = 0; v < n; ++v) {
        int32_t u = match[v];
        if (u < 0 || v < u) { cmap[v] = (int32_t)nc++; first.push_back((int32_t)v); second.push_back(u); }
    }
    for (int64_t v = 0; v < n; ++v) {
        int32_t u = match[v];
        if (u >= 0 && u < v) cmap[v] = cmap[u];
    }
    cg.n = nc;
    cg.rp.assign(nc + 1, 0);
    cg.vw.assign(nc, 0);
    cg.ci.clear(); cg.ew.clear();
    std::vector<int64_t> stamp(nc, -1), slot(nc, 0);
    for (int64_t c = 0; c < nc; ++c) {
        int32_t mem[2] = {first[c], second[c]};
        int64_t vwsum = 0;
        for (int t = 0; t < 2; ++t) {
            int32_t x = mem[t];
            if (x < 0) continue;
            vwsum += g.vw[x];
            for (int64_t e = g.rp[x]; e < g.rp[x + 1]; ++e) {
                const int32_t cu = cmap[g.ci[e]];
                if (cu == c) continue;
                if (stamp[cu] != c) {
                    stamp[cu] = c;
                    slot[cu] = (int64_t)cg.ci.size();
                    cg.ci.push_back(cu);
                    cg.ew.push_back(g.ew[e]);
                } else {
                    cg.ew[slot[cu]] += g.ew[e];
                }
            }
        }
        cg.vw[c] = (int32_t)vwsum;
        cg.rp[c + 1] = (int64_t)cg.ci.size();
    }
}

// ------------------------------------------------------------ initial partition
// Replaces convertCSRtoMETISandRun + the gpmetis subprocess
// (src/gpu_part.cu:803-864, 1157-1185).  init_trials independent trials of
// recursive bisection; each bisection of a label orders its vertices by BFS
// distance from a pseudo-peripheral vertex (ties by id) and cuts the order at
// the prefix whose weight is closest to the label's share.  Best trial:
// balanced first, then lowest cut, then lowest trial id.
const int32_t INF = INT32_MAX;

void bfs_label(const Graph& g, const std::vector<int32_t>& label, int32_t L, int32_t src, std::vector<int32_t>& dist, std::vector<int32_t>& frontier, std::vector<int32_t>& next) {
    frontier.clear();
    dist[src] = 0;
    frontier.push_back(src);
    int32_t r = 0;
    while (!frontier.empty()) {
        next.clear();
        for (int32_t v : frontier)
            for (int64_t e = g.rp[v]; e < g.rp[v + 1]; ++e) {
                int32_t u = g.ci[e];
                if (label[u] == L && dist[u] == INF) { dist[u] = r + 1; next.push_back(u); }
            }
        frontier.swap(next);
        ++r;
    }
}

std::vector<int32_t> initial_partition(const Graph& g, const Params& P, int* best_trial_out) {
    const int64_t n = g.n;
    const int32_t k = P.k;
    std::vector<int32_t> best_part;
    int best_t = -1;
    int64_t best_cut = 0, best_mp = 0;
    bool best_bal = false;
    std::vector<int32_t> label(n), dist1(n), dist2(n), cnt(k), frontier, next, members;
    std::vector<int64_t> pw;
    for (int t = 0; t < P.o.init_trials; ++t) {
        const uint64_t ts = trial_salt(P.seed, t);
        std::fill(label.begin(), label.end(), 0);
        std::fill(cnt.begin(), cnt.end(), 0);
        cnt[0] = k;
        for (int d = 0;; ++d) {
            bool any = false;
            for (int32_t L = 0; L < k; ++L) if (cnt[L] > 1) any = true;
            if (!any) break;
            const uint64_t ds = depth_salt(ts, d);
            std::vector<int32_t> newlabel = label;
            const std::vector<int32_t> cnt_d = cnt;  // labels split at this depth
            for (int32_t L = 0; L < k; ++L) {
                if (cnt_d[L] <= 1) continue;
                const int32_t c = cnt_d[L], cl = c / 2;
                members.clear();
                int64_t WL = 0;
                for (int64_t v = 0; v < n; ++v) if (label[v] == L) { members.push_back((int32_t)v); WL += g.vw[v]; }
                cnt[L] = cl;
                cnt[L + cl] = c - cl;
                if (members.empty()) continue;
                const int64_t target = WL * cl / c;
                // seed: smallest (top 32 hash bits, id)
                int32_t s0 = -1; uint64_t hb = 0;
                for (int32_t v : members) {
                    uint64_t h = ((mix64(ds ^ (uint64_t)(uint32_t)v) >> 32) << 32) | (uint32_t)v;
                    if (s0 < 0 || h < hb) { hb = h; s0 = v; }
                }
                for (int32_t v : members) { dist1[v] = INF; dist2[v] = INF; }
                bfs_label(g, label, L, s0, dist1, frontier, next);
                int32_t s = -1, db = -1;
                for (int32_t v : members)
                    if (dist1[v] != INF && (dist1[v] > db || (dist1[v] == db && v < s))) { db = dist1[v]; s = v; }
                bfs_label(g, label, L, s, dist2, frontier, next);
                std::vector<std::pair<int32_t, int32_t>> ord;
                ord.reserve(members.size());
                for (int32_t v : members) ord.push_back({dist2[v], v});
                std::sort(ord.begin(), ord.end());
                int64_t acc = 0;
                size_t j = 0;
                while (j < ord.size() && acc + g.vw[ord[j].second] <= target) { acc += g.vw[ord[j].second]; ++j; }
                if (j < ord.size() && 2 * target > 2 * acc + g.vw[ord[j].second]) ++j;
                for (size_t i = 0; i < ord.size(); ++i) newlabel[ord[i].second] = (i < j) ? L : L + cl;
            }
            label.swap(newlabel);
        }
        int64_t cut = edge_cut(g, label);
        part_weights(g, label, k, pw);
        int64_t mp = max_of(pw);
        bool bal = mp <= P.Lmax;
        bool better;
        if (best_t < 0) better = true;
        else if (bal != best_bal) better = bal;
        else if (!bal && mp != best_mp) better = mp < best_mp;
        else better = cut < best_cut;
        if (better) { best_t = t; best_cut = cut; best_mp = mp; best_bal = bal; best_part = label; }
    }
    if (best_trial_out) *best_trial_out = best_t;
    return best_part;
}

// ------------------------------------------------------------ refinement
// Replaces deterministicRefinement (src/gpu_part.cu:509-759) and its kernels
// computeGainsAndDestinations / markCandidates / tokenPassing /
// bufferCandidateMoves / computeAvailableCapacity / bitonic sort /
// selectMoves / commitMoves (src/gpu_part.cu:258-397, 472-506).
//
// One iteration is either
//  * LP (partition within Lmax): every unlocked vertex proposes its most
//    connected other part d (ties: lower part); gain = conn(d) - conn(own);
//    it is a candidate when gain >= 0 or -gain < conn(own)/lp_filter_den.
//    Each candidate re-evaluates its gain assuming every candidate neighbour
//    of higher priority (gain desc, id asc) has already moved; it moves when
//    that gain is >= 0.  (Replaces the float gains with heuristic balance
//    terms and the +10-slack token passing of the reference.)
//  * rebalance (some part above Lmax): vertices of overweight parts propose
//    the most connected part that is not overweight (fallback: the lightest
//    such part); loss = conn(own) - conn(dest).  Candidates are ordered by
//    (source part, loss bucket, id); a source keeps the prefix whose weight
//    before the vertex is below its excess.  Weak mode then orders the kept
//    moves by (dest, loss bucket, source, id) and keeps those that fit the
//    destination's remaining capacity by an exclusive prefix sum; strong mode
//    (after strong_after consecutive rebalance iterations) ignores the
//    proposed destination and lays the kept moves, in source order, over the
//    concatenated free capacities of the parts by prefix sum.  (Replaces the
//    atomic-order acceptance of selectMoves, src/gpu_part.cu:373-380.)
// Vertices moved in an iteration are locked for the next one.  The best
// state (balanced before unbalanced, then lower cut; unbalanced ones by lower
// max part weight) is kept, as the reference keeps its best partition
// (src/gpu_part.cu:627-631); the loop stops after refine_patience iterations
// without a significant improvement (cut below 0.999 x best), when label
// propagation finds no move two iterations in a row, or when a strong
// rebalance moves nothing (a weak one that moves nothing escalates to strong).
struct Conn {
    std::vector<int64_t> c;
    std::vector<int32_t> touched;
    explicit Conn(int32_t k) : c(k, 0) {}
    void clear() { for (int32_t q : touched) c[q] = 0; touched.clear(); }
    void add(int32_t q, int64_t w) { if (c[q] == 0) touched.push_back(q); c[q] += w; }
};

void refine_level(const Graph& g, std::vector<int32_t>& part, const Params& P, int level, const Tracer& tr, int* iters_out) {
    const int64_t n = g.n;
    const int32_t k = P.k;
    const int64_t Lmax = P.Lmax;
    std::vector<int64_t> pw;
    part_weights(g, part, k, pw);
    std::vector<uint8_t> lock(n, 0);
    std::vector<int32_t> dest(n), gain(n), best_part = part;
    int64_t cur_cut = edge_cut(g, part), cur_mp = max_of(pw);
    int64_t best_cut = cur_cut, best_mp = cur_mp;
    int stall = 0, rb_streak = 0, it = 0;
    int64_t prev_moves = -1;
    Conn conn(k);
    std::vector<char> over(k);
    for (it = 0; it < P.o.refine_max_iters; ++it) {
        const int64_t cut_before = cur_cut, mp_before = cur_mp;
        int mode;
        if (cur_mp > Lmax) { mode = (rb_streak >= P.o.strong_after) ? 2 : 1; ++rb_streak; }
        else { mode = 0; rb_streak = 0; }
        std::fill(dest.begin(), dest.end(), -1);
        std::fill(gain.begin(), gain.end(), 0);
        std::vector<int32_t> moved_v, moved_to;
        if (mode == 0) {
            for (int64_t v = 0; v < n; ++v) {
                if (lock[v]) continue;
                const int32_t p = part[v];
                conn.clear();
                for (int64_t e = g.rp[v]; e < g.rp[v + 1]; ++e) conn.add(part[g.ci[e]], g.ew[e]);
                const int64_t own = conn.c[p];
                int32_t d = -1; int64_t cd = 0;
                for (int32_t q : conn.touched)
                    if (q != p && conn.c[q] > 0 && (conn.c[q] > cd || (conn.c[q] == cd && q < d))) { cd = conn.c[q]; d = q; }
                if (d < 0) continue;
                const int64_t gn = cd - own;
                if (gn >= 0 || -gn < own / P.o.lp_filter_den) { dest[v] = d; gain[v] = (int32_t)gn; }
            }
            // afterburner order: (gain desc, id asc), or the learned move priorities
            const int32_t* key = gain.data();
            if (P.mprio) {
                const int32_t* mp = P.mprio(P.mprio_user, level, it, n);
                if (mp) key = mp;
            }
            for (int64_t v = 0; v < n; ++v) {
                if (dest[v] < 0) continue;
                int64_t g2 = 0;
                for (int64_t e = g.rp[v]; e < g.rp[v + 1]; ++e) {
                    const int32_t u = g.ci[e];
                    int32_t pu = part[u];
                    if (dest[u] >= 0 && (key[u] > key[v] || (key[u] == key[v] && u < v))) pu = dest[u];
                    if (pu == dest[v]) g2 += g.ew[e];
                    else if (pu == part[v]) g2 -= g.ew[e];
                }
                if (g2 >= 0) { moved_v.push_back((int32_t)v); moved_to.push_back(dest[v]); }
            }
        } else {
            for (int32_t q = 0; q < k; ++q) over[q] = pw[q] > Lmax;
            int32_t lightest = -1;
            for (int32_t q = 0; q < k; ++q)
                if (!over[q] && (lightest < 0 || pw[q] < pw[lightest])) lightest = q;
            struct Cand { uint32_t src, bucket; int32_t v, d; };
            std::vector<Cand> cands;
            for (int64_t v = 0; v < n; ++v) {
                const int32_t p = part[v];
                if (!over[p]) continue;
                conn.clear();
                for (int64_t e = g.rp[v]; e < g.rp[v + 1]; ++e) conn.add(part[g.ci[e]], g.ew[e]);
                const int64_t own = conn.c[p];
                int32_t d = -1; int64_t cd = 0;
                for (int32_t q : conn.touched)
                    if (!over[q] && conn.c[q] > 0 && (conn.c[q] > cd || (conn.c[q] == cd && q < d))) { cd = conn.c[q]; d = q; }
                if (d < 0) { d = lightest; cd = 0; }
                const int32_t loss = (int32_t)(own - cd);
                dest[v] = d; gain[v] = -loss;
                cands.push_back({(uint32_t)p, loss_bucket(loss), (int32_t)v, d});
            }
            std::sort(cands.begin(), cands.end(), [](const Cand& a, const Cand& b) {
                if (a.src != b.src) return a.src < b.src;
                if (a.bucket != b.bucket) return a.bucket < b.bucket;
                return a.v < b.v; });
            std::vector<Cand> acc;
            {
                size_t i = 0;
                while (i < cands.size()) {
                    const uint32_t s = cands[i].src;
                    const int64_t excess = pw[s] - Lmax;
                    int64_t pre = 0;
                    for (; i < cands.size() && cands[i].src == s; ++i) {
                        if (pre < excess) acc.push_back(cands[i]);
                        pre += g.vw[cands[i].v];
                    }
                }
            }
            if (mode == 1) {
                std::vector<Cand>& bd = acc;   // accepted moves, re-sorted by destination (acc is not used again)
                std::sort(bd.begin(), bd.end(), [](const Cand& a, const Cand& b) {
                    if (a.d != b.d) return a.d < b.d;
                    if (a.bucket != b.bucket) return a.bucket < b.bucket;
                    if (a.src != b.src) return a.src < b.src;
                    return a.v < b.v; });
                size_t i = 0;
                while (i < bd.size()) {
                    const int32_t d = bd[i].d;
                    const int64_t cap = Lmax - pw[d];
                    int64_t pre = 0;
                    for (; i < bd.size() && bd[i].d == d; ++i) {
                        if (pre + g.vw[bd[i].v] <= cap) { moved_v.push_back(bd[i].v); moved_to.push_back(d); }
                        pre += g.vw[bd[i].v];
                    }
                }
            } else {
                std::vector<int64_t> cum(k + 1, 0);
                for (int32_t q = 0; q < k; ++q) cum[q + 1] = cum[q] + (over[q] ? 0 : std::max<int64_t>(0, Lmax - pw[q]));
                int64_t pre = 0;
                for (const Cand& c : acc) {
                    const int64_t w = g.vw[c.v];
                    if (pre < cum[k]) {
                        // part whose free interval contains pre
                        int32_t q = (int32_t)(std::upper_bound(cum.begin(), cum.end(), pre) - cum.begin()) - 1;
                        if (pre + w <= cum[q + 1]) { moved_v.push_back(c.v); moved_to.push_back(q); }
                    }
                    pre += w;
                }
            }
        }
        std::fill(lock.begin(), lock.end(), 0);
        for (size_t i = 0; i < moved_v.size(); ++i) {
            const int32_t v = moved_v[i], d = moved_to[i];
            pw[part[v]] -= g.vw[v];
            pw[d] += g.vw[v];
            part[v] = d;
            lock[v] = 1;
        }
        const int64_t nmoves = (int64_t)moved_v.size();
        cur_cut = edge_cut(g, part);
        cur_mp = max_of(pw);
        if (tr.fn) {
            gp_trace_event ev;
            memset(&ev, 0, sizeof ev);
            ev.kind = GP_TR_REFINE_ITER; ev.level = level; ev.iter = it; ev.mode = mode;
            ev.n = n; ev.m = g.m(); ev.cut = cut_before; ev.maxpw = mp_before; ev.count = nmoves;
            ev.a0 = dest.data(); ev.a1 = gain.data(); ev.a2 = part.data();
            tr.emit(ev);
        }
        const bool cb = cur_mp <= Lmax, bb = best_mp <= Lmax;
        bool better = false, signif = false;
        if (cb && !bb) { better = true; signif = true; }
        else if (cb && bb) { better = cur_cut < best_cut; signif = 1000 * cur_cut < 999 * best_cut; }
        else if (!cb && !bb) { better = cur_mp < best_mp || (cur_mp == best_mp && cur_cut < best_cut); signif = cur_mp < best_mp; }
        if (better) { best_cut = cur_cut; best_mp = cur_mp; best_part = part; }
        stall = signif ? 0 : stall + 1;
        const bool lp_idle = (mode == 0 && nmoves == 0 && prev_moves == 0);
        prev_moves = nmoves;
        // a rebalance step that moved nothing is a fixed point of its mode:
        // weak escalates to strong at once, strong ends the level
        bool rb_stuck = false;
        if (mode != 0 && nmoves == 0) {
            if (mode == 1) rb_streak = P.o.strong_after; else rb_stuck = true;
        }
        if (stall >= P.o.refine_patience || lp_idle || rb_stuck) { ++it; break; }
    }
    part = best_part;
    if (iters_out) *iters_out += it;
}

// ------------------------------------------------------------ validation
int validate(int64_t n, const int64_t* rp, const int32_t* ci, const int32_t* vw, const int32_t* ew, int check) {
    if (rp[0] != 0) return fail(GP_EINVAL, "rowptr[0] must be 0");
    for (int64_t v = 0; v < n; ++v)
        if (rp[v + 1] < rp[v]) return fail(GP_EINVAL, "rowptr is not non-decreasing at vertex " + std::to_string(v));
    const int64_t m = rp[n];
    int64_t sv = 0, se = 0;
    for (int64_t v = 0; v < n; ++v) {
        int64_t w = vw ? vw[v] : 1;
        if (w < 1) return fail(GP_EINVAL, "vertex weight < 1 at vertex " + std::to_string(v));
        sv += w;
    }
    for (int64_t e = 0; e < m; ++e) {
        int64_t w = ew ? ew[e] : 1;
        if (w < 1) return fail(GP_EINVAL, "edge weight < 1 at entry " + std::to_string(e));
        se += w;
    }
    if (sv > INT32_MAX) return fail(GP_EINVAL, "sum of vertex weights exceeds int32");
    if (se > INT32_MAX) return fail(GP_EINVAL, "sum of edge weights exceeds int32");
    if (check >= 1) {
        for (int64_t v = 0; v < n; ++v)
            for (int64_t e = rp[v]; e < rp[v + 1]; ++e) {
                if (ci[e] < 0 || ci[e] >= n) return fail(GP_EINVAL, "column index out of range at entry " + std::to_string(e));
                if (ci[e] == v) return fail(GP_EINVAL, "self-loop at vertex " + std::to_string(v));
            }
    }
    if (check >= 2) {
        std::vector<std::pair<int64_t, int64_t>> a, b;
        a.reserve(m); b.reserve(m);
        for (int64_t v = 0; v < n; ++v)
            for (int64_t e = rp[v]; e < rp[v + 1]; ++e) {
                a.push_back({v * n + ci[e], ew ? ew[e] : 1});
                b.push_back({(int64_t)ci[e] * n + v, ew ? ew[e] : 1});
            }
        std::sort(a.begin(), a.end());
        std::sort(b.begin(), b.end());
        if (a != b) return fail(GP_EINVAL, "graph is not symmetric");
    }
    return GP_OK;
}

}  // namespace

extern "C" {

const char* gpo_last_error(void) { return g_err.c_str(); }

int gpo_default_options(gp_options* o) {
    if (!o) return fail(GP_EINVAL, "null options");
    resolve_options(nullptr, 0, 2, o);
    o->coarsen_to = 0;  // auto: max(1024, 32*k)
    return GP_OK;
}

int64_t gpo_compute_lmax(int64_t W, int32_t k, float imbalance) { return compute_lmax(W, k, imbalance); }

int gpo_partition_prio2(int64_t n, const int64_t* rowptr, const int32_t* colidx,
                        const int32_t* vwgt, const int32_t* ewgt, int32_t k,
                        float imbalance, uint64_t seed, int32_t* part_out,
                        const gp_options* opt, gp_stats* stats,
                        gp_trace_fn trace, void* trace_user, prio_fn_t prio, void* prio_user,
                        mprio_fn_t mprio, void* mprio_user);

// Full V-cycle on the CPU.  Same signature and semantics as gp_partition_ex.
int gpo_partition(int64_t n, const int64_t* rowptr, const int32_t* colidx,
                  const int32_t* vwgt, const int32_t* ewgt, int32_t k,
                  float imbalance, uint64_t seed, int32_t* part_out,
                  const gp_options* opt, gp_stats* stats,
                  gp_trace_fn trace, void* trace_user) {
    return gpo_partition_prio2(n, rowptr, colidx, vwgt, ewgt, k, imbalance, seed, part_out, opt, stats, trace,
                               trace_user, nullptr, nullptr, nullptr, nullptr);
}

// Same, with per-level matching priorities supplied by prio (learned mode).
int gpo_partition_prio(int64_t n, const int64_t* rowptr, const int32_t* colidx,
                       const int32_t* vwgt, const int32_t* ewgt, int32_t k,
                       float imbalance, uint64_t seed, int32_t* part_out,
                       const gp_options* opt, gp_stats* stats,
                       gp_trace_fn trace, void* trace_user, prio_fn_t prio, void* prio_user) {
    return gpo_partition_prio2(n, rowptr, colidx, vwgt, ewgt, k, imbalance, seed, part_out, opt, stats, trace,
                               trace_user, prio, prio_user, nullptr, nullptr);
}

// Same, plus per-step move priorities supplied by mprio (learned move order).
int gpo_partition_prio2(int64_t n, const int64_t* rowptr, const int32_t* colidx,
                        const int32_t* vwgt, const int32_t* ewgt, int32_t k,
                        float imbalance, uint64_t seed, int32_t* part_out,
                        const gp_options* opt, gp_stats* stats,
                        gp_trace_fn trace, void* trace_user, prio_fn_t prio, void* prio_user,
                        mprio_fn_t mprio, void* mprio_user) {
    g_err.clear();
    if (n < 0) return fail(GP_EINVAL, "n must be >= 0");
    if (k < 1 || k > GP_MAX_K) return fail(GP_EINVAL, "k must be in [1, " + std::to_string(GP_MAX_K) + "]");
    if (!(imbalance >= 0.0f) || !std::isfinite(imbalance)) return fail(GP_EINVAL, "imbalance must be finite and >= 0");
    if (n == 0) { if (stats) memset(stats, 0, sizeof *stats); return GP_OK; }
    if (!rowptr || !colidx || !part_out) return fail(GP_EINVAL, "null array");
    if (k > n) return fail(GP_EINVAL, "k must not exceed the number of vertices");
    if (n > INT32_MAX - 1) return fail(GP_EINVAL, "n must fit in int32");
    Params P;
    resolve_options(opt, n, k, &P.o);
    int rc = validate(n, rowptr, colidx, vwgt, ewgt, P.o.check_input);
    if (rc) return rc;
    Tracer tr; tr.fn = trace; tr.user = trace_user;
    std::vector<Graph> lv(1);
    {
        Graph& g = lv[0];
        g.n = n;
        g.rp.assign(rowptr, rowptr + n + 1);
        const int64_t m = rowptr[n];
        g.ci.assign(colidx, colidx + m);
        g.ew.assign(m, 1);
        if (ewgt) g.ew.assign(ewgt, ewgt + m);
        g.vw.assign(n, 1);
        if (vwgt) g.vw.assign(vwgt, vwgt + n);
    }
    P.k = k; P.seed = seed;
    P.prio = prio; P.prio_user = prio_user;
    P.mprio = mprio; P.mprio_user = mprio_user;
    P.W = 0;
    for (int64_t v = 0; v < n; ++v) P.W += lv[0].vw[v];
    P.Lmax = compute_lmax(P.W, k, imbalance);
    P.maxvw = std::max<int64_t>(1, (3 * P.W) / (2 * (int64_t)P.o.coarsen_to));
    std::vector<int32_t> part(n, 0);
    int best_trial = -1, iters = 0;
    std::vector<std::vector<int32_t>> cmaps;
    if (k > 1) {
        // coarsening (src/gpu_part.cu:1003-1152)
        while (lv.back().n > P.o.coarsen_to && (int)lv.size() < 64) {
            const Graph& g = lv.back();
            const int level = (int)lv.size() - 1;
            int rounds = 0; int64_t pairs = 0;
            std::vector<int32_t> match = match_level(g, level, P, &rounds, &pairs);
            if (tr.fn) {
                gp_trace_event ev; memset(&ev, 0, sizeof ev);
                ev.kind = GP_TR_MATCH; ev.level = level; ev.iter = rounds; ev.n = g.n; ev.m = g.m();
                ev.count = pairs; ev.a0 = match.data();
                tr.emit(ev);
            }
            const int64_t nc = g.n - pairs;
            if (20 * nc > 19 * g.n) break;  // coarsening stalled
            Graph cg;
            std::vector<int32_t> cmap;
            contract(g, match, cmap, cg);
            if (tr.fn) {
                gp_trace_event ev; memset(&ev, 0, sizeof ev);
                ev.kind = GP_TR_CONTRACT; ev.level = level; ev.n = cg.n; ev.m = cg.m();
                ev.a0 = cmap.data(); ev.rowptr = cg.rp.data(); ev.colidx = cg.ci.data();
                ev.ewgt = cg.ew.data(); ev.vwgt = cg.vw.data();
                tr.emit(ev);
            }
            cmaps.push_back(std::move(cmap));
            lv.push_back(std::move(cg));
        }
        const int L = (int)lv.size() - 1;
        std::vector<int32_t> cpart = initial_partition(lv[L], P, &best_trial);
        if (tr.fn) {
            gp_trace_event ev; memset(&ev, 0, sizeof ev);
            std::vector<int64_t> pw; part_weights(lv[L], cpart, k, pw);
            ev.kind = GP_TR_INITPART; ev.level = L; ev.iter = best_trial; ev.n = lv[L].n; ev.m = lv[L].m();
            ev.cut = edge_cut(lv[L], cpart); ev.maxpw = max_of(pw); ev.a0 = cpart.data();
            tr.emit(ev);
        }
        for (int l = L; l >= 0; --l) {
            if (l < L) {
                // projection (src/gpu_part.cu:763-772)
                std::vector<int32_t> fp(lv[l].n);
                for (int64_t v = 0; v < lv[l].n; ++v) fp[v] = cpart[cmaps[l][v]];
                cpart.swap(fp);
            }
            refine_level(lv[l], cpart, P, l, tr, &iters);
            if (tr.fn) {
                gp_trace_event ev; memset(&ev, 0, sizeof ev);
                std::vector<int64_t> pw; part_weights(lv[l], cpart, k, pw);
                ev.kind = GP_TR_LEVEL_DONE; ev.level = l; ev.n = lv[l].n; ev.m = lv[l].m();
                ev.cut = edge_cut(lv[l], cpart); ev.maxpw = max_of(pw); ev.a0 = cpart.data();
                tr.emit(ev);
            }
        }
        part.swap(cpart);
    }
    memcpy(part_out, part.data(), sizeof(int32_t) * n);
    if (stats) {
        memset(stats, 0, sizeof *stats);
        std::vector<int64_t> pw; part_weights(lv[0], part, k, pw);
        stats->cut = edge_cut(lv[0], part);
        stats->max_part_weight = max_of(pw);
        stats->total_weight = P.W;
        stats->max_allowed = P.Lmax;
        stats->imbalance = (double)stats->max_part_weight * k / (double)P.W - 1.0;
        stats->levels = (int32_t)lv.size();
        stats->coarsest_n = (int32_t)lv.back().n;
        stats->best_trial = best_trial;
        stats->refine_iters = iters;
    }
    return GP_OK;
}

// Exact cut and part weights of a given partition (host arrays).
int gpo_edge_cut(int64_t n, const int64_t* rowptr, const int32_t* colidx, const int32_t* ewgt,
                 const int32_t* vwgt, const int32_t* part, int32_t k, int64_t* cut_out, int64_t* pw_out) {
    g_err.clear();
    if (n < 0 || k < 1) return fail(GP_EINVAL, "bad sizes");
    int64_t s = 0;
    for (int64_t v = 0; v < n; ++v) {
        if (part[v] < 0 || part[v] >= k) return fail(GP_EINVAL, "part id out of range at vertex " + std::to_string(v));
        for (int64_t e = rowptr[v]; e < rowptr[v + 1]; ++e)
            if (part[colidx[e]] != part[v]) s += ewgt ? ewgt[e] : 1;
    }
    if (cut_out) *cut_out = s / 2;
    if (pw_out) {
        for (int32_t q = 0; q < k; ++q) pw_out[q] = 0;
        for (int64_t v = 0; v < n; ++v) pw_out[part[v]] += vwgt ? vwgt[v] : 1;
    }
    return GP_OK;
}

// Exposed pieces of the rule set, for unit tests of the hash and bucket.
uint64_t gpo_mix64(uint64_t x) { return mix64(x); }
uint32_t gpo_edge_hash(uint64_t seed, int32_t level, int32_t a, int32_t b) { return edge_hash(edge_salt(seed, level), a, b); }
uint32_t gpo_loss_bucket(int32_t loss) { return loss_bucket(loss); }

}  // extern "C"
