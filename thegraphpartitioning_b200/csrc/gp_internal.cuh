// gp_internal.cuh -- declarations shared by the library's translation units.
#pragma once

#include "gp_common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace gp {

}  // namespace gp
struct gp_gnn;   // learned edge scorer (gp_gnn.cu)
namespace gp {

struct Params {
    const gp_gnn* gnn = nullptr;   // learned matching priorities when set
    int32_t k = 2;
    int64_t W = 0;        // total vertex weight
    int64_t Lmax = 0;     // max allowed part weight
    int64_t maxvw = 0;    // coarse vertex weight cap
    uint64_t seed = 0;
    float imbalance = 0.03f;
    gp_options o{};
};

// Degree classes of the rows of one level; every kernel that works row by
// row (matching, connectivity, afterburner) schedules its units from these
// lists: bucket 0 rows go 4 to a warp (8 lanes each), bucket 1 rows one to a
// warp in registers, bucket 2 rows one to a warp with a shared-memory
// histogram, heavy rows one to a CTA.
constexpr int kTile8 = 8;         // bucket 0: degree <= 8
constexpr int kTile32 = 32;       // bucket 1: degree <= 32
struct Level {
    DGraph g;
    int32_t* cmap = nullptr;      // fine -> coarse map to the next coarser level
    int32_t heavy_deg = kHeavyDeg; // rows longer than this are heavy (whole CTAs)
    int32_t item_len = kItemLen;  // entries of one CTA item of a heavy row
    int32_t* heavy = nullptr;     // vertices with degree > heavy_deg
    int64_t nheavy = 0;
    int32_t* bucket[3] = {nullptr, nullptr, nullptr};
    int64_t nbucket[3] = {0, 0, 0};
    // heavy rows split into items of at most item_len entries, one CTA each
    int32_t* item_row = nullptr;   // index into heavy[]
    int64_t* item_beg = nullptr;   // entry range of the item
    int64_t* item_end = nullptr;
    int32_t* row_items = nullptr;  // items per heavy row
    int32_t* row_first = nullptr;  // first item of each heavy row
    int64_t nitems = 0;
    // light work units in the order bucket 2 rows, bucket 1 rows, groups of 4
    // bucket 0 rows, with the prefix sum of their costs (entries + 32): warps
    // take contiguous unit ranges of equal cost
    int64_t* unit_cost = nullptr;  // nunits + 1 prefix
    int64_t nunits = 0;
    // bytes of one neighbour scan: row pointers, column ids, weights, gathered per-neighbour int32 state
    int64_t scan_bytes() const { return 8 * (g.n + 1) + 4 * g.m + (g.ew ? 4 * g.m : 0) + 4 * g.m; }
};

// Host-side rule helpers (identical to the oracle's).
inline void resolve_options(const gp_options* in, int32_t k, gp_options* o) {
    gp_options d;
    memset(&d, 0, sizeof d);
    if (in) d = *in;
    d.version = GP_OPTIONS_VERSION;
    if (d.coarsen_to <= 0) d.coarsen_to = (int32_t)std::max<int64_t>(1024, 32LL * k);
    if (d.match_rounds <= 0) d.match_rounds = 4;
    if (d.two_hop == 0) d.two_hop = 1;
    if (d.init_trials <= 0) d.init_trials = 64;
    if (d.refine_max_iters <= 0) d.refine_max_iters = 64;
    if (d.refine_patience <= 0) d.refine_patience = 4;
    if (d.lp_filter_den <= 0) d.lp_filter_den = 4;
    if (d.strong_after <= 0) d.strong_after = 2;
    if (d.check_input == 0) d.check_input = 1;
    if (d.ctas_per_sm <= 0) d.ctas_per_sm = 64;
    if (d.heavy_deg <= 0) d.heavy_deg = kHeavyDeg;
    d.heavy_deg = std::min(std::max(d.heavy_deg, 64), 65536);
    if (d.item_len <= 0) d.item_len = kItemLen;
    d.item_len = std::min(std::max(d.item_len, d.heavy_deg), 1 << 20);
    *o = d;
}

inline int64_t compute_lmax(int64_t W, int32_t k, float imbalance) {
    double lim = (1.0 + (double)imbalance) * (double)W / (double)k;
    int64_t l = (int64_t)std::floor(lim);
    int64_t avg = (W + k - 1) / k;
    return std::max(l, avg);
}

struct Tracer {
    gp_trace_fn fn = nullptr;
    void* user = nullptr;
    bool on() const { return fn != nullptr; }
    void emit(const gp_trace_event& e) const { if (fn) fn(user, &e); }
};

// refinement buffers sized for the finest level
struct RefineBufs {
    int32_t* part = nullptr;
    int32_t* part_next = nullptr;
    int32_t* best = nullptr;
    void* pc = nullptr;           // uint8 / uint16 copy of part read by the neighbour gathers
    void* pc_next = nullptr;      // and of part_next
    int pcb = 1;                  // its bytes per vertex (1: k <= 256, 2: k <= 1024)
    int32_t* dest = nullptr;
    int32_t* gain = nullptr;
    int32_t* mp = nullptr;        // learned move priorities of a label-propagation step
    uint64_t* pdg = nullptr;      // label-propagation passes, k <= 1024: part, dest + 1 and gain of
                                  // every vertex in one word (the move step's one gather per entry)
    uint8_t* lock = nullptr;
    uint8_t* lock_next = nullptr;
    int64_t* pw = nullptr;        // k
    int64_t* best_pw = nullptr;   // k
    int64_t* status = nullptr;    // 16
    int32_t* clist[3] = {nullptr, nullptr, nullptr};   // LP candidates by degree bucket
    int64_t* wfirst = nullptr;    // first light unit of each warp of the connectivity pass (+ end)
    int64_t wfirst_cap = 0;       // its length
    // accumulators of heavy rows split over several CTAs (zero between uses)
    int32_t* hhist = nullptr;     // nheavy_max * k connectivity sums
    int64_t* hsum = nullptr;      // nheavy_max * 2: cross, total (conn) / gain (afterburner)
    int32_t* hdone = nullptr;     // nheavy_max: finished items
    uint64_t* ckeys = nullptr;    // rebalance candidate keys
    int32_t* cvals = nullptr;
    uint64_t* ckeys2 = nullptr;
    int32_t* cvals2 = nullptr;
};

// device status block of the refinement loop; slots [0, S_NRESET) are cleared
// before every connectivity pass, S_STEP_MOVES before every move step
enum StatusSlot { S_CROSS = 0, S_MAXPW = 1, S_MODE = 2, S_NL0 = 3, S_NL1 = 4, S_LIGHT = 5, S_NL2 = 6, S_CDEG = 7,
                  S_NRESET = 8, S_STEP_MOVES = 8, S_NSLOTS = 16 };

// CUDA events of the phases of one V-cycle
struct Timer {
    cudaEvent_t e[8];
    Timer() { for (auto& x : e) cudaEventCreate(&x); }
    ~Timer() { for (auto& x : e) cudaEventDestroy(x); }
    Timer(const Timer&) = delete;
    Timer& operator=(const Timer&) = delete;
    double ms(int a, int b) { float t = 0; cudaEventElapsedTime(&t, e[a], e[b]); return t; }
};

// State of one V-cycle between its phases (hierarchy and buffers live in the
// keep arena of the context that ran vc_begin).  Counters of the contexts
// that ran its phases are moved here by take().
struct VState {
    Params P;
    DGraph g0;
    std::vector<Level> lv;
    RefineBufs B;
    Timer tm;
    int L = 0, best_trial = -1, iters = 0;
    int refined_to = 1;          // finest level refined so far (L + 1: none)
    int64_t launches = 0, bytes = 0, conn_launches = 0, conn_bytes = 0;
    double ms_conn = 0, ms_gnn = 0;
    void take(Ctx& c) {
        launches += c.launches; bytes += c.bytes; ms_conn += c.ms_conn; ms_gnn += c.ms_gnn;
        conn_launches += c.conn_launches; conn_bytes += c.conn_bytes;
        c.launches = 0; c.bytes = 0; c.ms_conn = 0; c.ms_gnn = 0; c.conn_launches = 0; c.conn_bytes = 0;
    }
};

// gp_api.cu: the V-cycle as three phases (run_vcycle runs them in a row)
void vc_begin(Ctx& c, const DGraph& g0, int32_t k, float imbalance, uint64_t seed, const gp_options* opt,
              VState& S, const Tracer& tr, const gp_gnn* gnn = nullptr);
void vc_level(Ctx& c, VState& S, int l, const Tracer& tr);
void vc_end(Ctx& c, VState& S, int32_t* d_out, gp_stats* st);
void run_vcycle(Ctx& c, const DGraph& g0, int32_t k, float imbalance, uint64_t seed, const gp_options* opt,
                int32_t* d_out, gp_stats* st, const Tracer& tr, const gp_gnn* gnn = nullptr);

// gp_refine.cu: one-block levels of many V-cycles in one persistent launch.
// chain_add (thread-safe) queues the coarsest levels of S that one block
// refines (scratch from c.keep) and returns their count; chain_run launches
// the persistent kernel over every queued chain, then advances each
// VState's refined_to past its chain.
struct ChainBatch;
ChainBatch* chain_batch_new();
void chain_batch_delete(ChainBatch* cb);
int chain_add(Ctx& c, ChainBatch* cb, VState& S);
void chain_run(Ctx& c, ChainBatch* cb);
int check_args(int64_t n, int32_t k, float imbalance);
extern thread_local std::string t_err;

void ensure_kernel_caps(int dev);   // once per device, before any launch

// gp_batch.cu
void release_batch_workers(int dev);
// per-file shared-memory caps (gp_coarsen.cu, gp_initpart.cu)
void coarsen_smem_caps();
void refine_smem_caps();
void initpart_smem_caps();

// gp_gnn.cu
void gnn_level_priorities(Ctx& c, const gp_gnn* G, const Level& L, int level, int32_t* prio);
bool gnn_scores_level(const gp_gnn* G, int level);   // false: edge weights at this level
bool gnn_has_move_head(const gp_gnn* G);
void gnn_move_priorities(Ctx& c, const gp_gnn* G, const DGraph& g, int level, const int32_t* dest,
                         const int32_t* gain, int32_t* mp);

// gp_coarsen.cu
void build_heavy(Ctx& c, Level& L);
// prio: per-entry matching priority replacing the edge weight (nullptr: weights)
int64_t match_level(Ctx& c, const Level& L, int level, const Params& P, int32_t* match, int* rounds_out,
                    const int32_t* prio = nullptr);
void contract_level(Ctx& c, Level& fine, Level& coarse, const int32_t* match);

// gp_initpart.cu
int initial_partition(Ctx& c, const Level& L, const Params& P, int32_t* part_out);

// gp_refine.cu
int refine_level(Ctx& c, const Level& L, const Params& P, RefineBufs& B, int level, const Tracer& tr);
int64_t conn_max_warps(const Ctx& c);   // most light warps a connectivity pass launches
void project(Ctx& c, const Level& fine, const int32_t* part_coarse, int32_t* part_fine);
void part_weights(Ctx& c, const DGraph& g, const int32_t* part, int32_t k, int64_t* pw);
void cut_and_weights(Ctx& c, const DGraph& g, const int32_t* part, int32_t k, int64_t* d_cross2, int64_t* d_pw);

}  // namespace gp
