/*
 * gp_partition.h -- C ABI of the B200-native multilevel k-way graph partitioner.
 *
 * The reference (iamrupamroyy/TheGraphPartitioning) is a single executable whose
 * only entry point is main() in src/gpu_part.cu:878-1390; it has no library API.
 * The functions below are the library boundary that replaces that executable's
 * internals:
 *
 *   gp_partition / gp_partition_device
 *       replace the whole V-cycle driven by main(): coarsening loop
 *       (src/gpu_part.cu:1003-1152), METIS initial partition through the gpmetis
 *       subprocess (src/gpu_part.cu:803-864, 1157-1185), refinement
 *       (src/gpu_part.cu:509-759) and projection (src/gpu_part.cu:763-772,
 *       1205-1274).  The result is the per-vertex part array that the reference
 *       prints into ./finalpartition.txt (src/gpu_part.cu:1296-1322).
 *   gp_edge_cut_device
 *       replaces computeEdgeCut / compute_edgecut (src/gpu_part.cu:400-469),
 *       with an int64 accumulator instead of the reference's int32.
 *   gp_last_error
 *       replaces the reference's CUDA_CHECK -> exit(EXIT_FAILURE) convention
 *       (src/gpu_part.cu:40-47): nothing in this library exits the process.
 *
 * Graph contract (same as the files written by preprocess/conversion.py:66-93):
 * 0-based CSR, symmetric, no self-loops.  rowptr has n+1 int64 entries, colidx
 * and ewgt have rowptr[n] entries.  vwgt/ewgt may be NULL (unit weights).
 * All weights must be >= 1; the sum of vertex weights and the sum of directed
 * edge weights must each fit in int32 (so that every coarse weight, every
 * part-connectivity count and every gain is an exact int32).
 *
 * Every function returns GP_OK (0) or a negative GP_E* code and never exits.
 * gp_last_error() returns a thread-local message describing the last failure.
 */
#ifndef GP_PARTITION_H
#define GP_PARTITION_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GP_OK        0
#define GP_EINVAL   -1   /* invalid argument or malformed graph                 */
#define GP_ENOMEM   -2   /* device or host allocation failed                    */
#define GP_ECUDA    -3   /* a CUDA runtime call or kernel launch failed         */
#define GP_ETIMEOUT -4   /* a bounded device wait gave up                       */
#define GP_EINTERNAL -5  /* internal consistency check failed                   */

#define GP_MAX_K 1024    /* largest supported number of parts                   */

#define GP_OPTIONS_VERSION 1

/* Tunables of the deterministic V-cycle.  Zero in any field selects the
 * default; gp_default_options() fills the defaults explicitly.  The CPU oracle
 * reads the same structure, so a given (graph, k, imbalance, seed, options)
 * produces the same partition on both. */
typedef struct gp_options {
    int32_t version;            /* GP_OPTIONS_VERSION                                   */
    int32_t coarsen_to;         /* stop coarsening at <= this many vertices (0: auto)   */
    int32_t match_rounds;       /* max handshake rounds per level (default 4)           */
    int32_t two_hop;            /* >0 or 0: pair leftovers sharing an anchor; <0: off   */
    int32_t init_trials;        /* initial-partition trials (default 64)                */
    int32_t refine_max_iters;   /* max refinement iterations per level (default 64)     */
    int32_t refine_patience;    /* stop after this many non-improving iterations (4)    */
    int32_t lp_filter_den;      /* negative-gain filter: -gain < conn_own/den (4)      */
    int32_t strong_after;       /* consecutive rebalance iterations before strong (2)  */
    int32_t check_input;        /* 0/1: structural checks, 2: +symmetry, <0: none        */
    int32_t verbose;            /* 0: silent                                           */
    int32_t profile;            /* 1: time the connectivity pass with CUDA events       */
    int32_t small_level_n;      /* > 0: refine levels of at most this many vertices
                                   (capped at 16384) without rows above 2048 entries in
                                   one thread block, one launch per level; 0 or < 0:
                                   off.  Results are identical either way; it pays
                                   only where launches, not SMs, are scarce            */
    int32_t ctas_per_sm;        /* grid of the row-scanning kernels (matching rounds,
                                   contraction, connectivity pass, afterburner, cut): this
                                   many CTAs per SM at most (0: 64 for one graph, where
                                   many small work ranges balance better than a few
                                   large ones; 8 in gp_partition_batch_device, where
                                   concurrent V-cycles share the GPU); results are
                                   identical for every value (autotuner knob)          */
    int32_t heavy_deg;          /* rows longer than this many entries are scanned by whole
                                   CTAs (8 warps), shorter ones by one warp or a lane
                                   group (0: 4096; 64..65536); results are identical
                                   for every value (autotuner knob; the learned V-cycle
                                   always uses 2048 and an item_len of 16384)          */
    int32_t item_len;           /* entries of one CTA's piece of a long row (0: 32768;
                                   heavy_deg..1048576); results are identical (autotuner
                                   knob)                                                */
} gp_options;

/* Result record of one call. */
typedef struct gp_stats {
    int64_t cut;                /* exact edge cut of the returned partition (int64)     */
    int64_t max_part_weight;
    int64_t total_weight;       /* sum of vertex weights                               */
    int64_t max_allowed;        /* floor((1+imbalance) * total_weight / k)             */
    double  imbalance;          /* max_part_weight * k / total_weight - 1               */
    int32_t levels;             /* number of graphs in the hierarchy (>= 1)            */
    int32_t coarsest_n;
    int32_t best_trial;         /* initial-partition trial that was kept               */
    int32_t refine_iters;       /* refinement iterations over all levels               */
    int64_t algo_bytes;         /* algorithmic HBM bytes of all executed passes        */
    int64_t kernel_launches;    /* kernels this call launched                          */
    double  ms_coarsen;         /* device time per phase (CUDA events)                 */
    double  ms_initial;
    double  ms_refine;
    double  ms_project;
    double  ms_total;
    double  ms_h2d;             /* host API only: host->device copies                  */
    double  ms_d2h;
    /* opt.profile = 1: the refinement connectivity pass (the dominant kernel) */
    double  ms_conn;            /* summed CUDA-event time of its launches               */
    int64_t conn_launches;
    int64_t conn_bytes;         /* algorithmic bytes of those launches                 */
} gp_stats;

/* ---- optional tracing (tests): host copies of intermediate results ----- */
enum gp_trace_kind {
    GP_TR_MATCH = 1,       /* a0 = match[n]   (partner or -1)                        */
    GP_TR_CONTRACT = 2,    /* a0 = cmap[n]; coarse graph in rowptr/colidx/ewgt/vwgt   */
    GP_TR_INITPART = 3,    /* a0 = part[n] of the kept trial; iter = trial id        */
    GP_TR_REFINE_ITER = 4, /* a0 = dest[n] (-1: no proposal), a1 = gain[n],
                              a2 = part[n] after the iteration; cut/maxpw before it   */
    GP_TR_LEVEL_DONE = 5,  /* a0 = part[n] after refinement of this level             */
    GP_TR_PRIO = 6,        /* learned mode: a0 = matching priority per entry (m)       */
    GP_TR_MOVE_PRIO = 7    /* learned mode with a move-order head: a0 = move priority
                              per vertex (n) of a label-propagation step, before it   */
};

typedef struct gp_trace_event {
    int32_t kind;
    int32_t level;          /* 0 = input graph                                     */
    int32_t iter;
    int32_t mode;           /* refine: 0 label propagation, 1 weak, 2 strong rebalance */
    int64_t n;
    int64_t m;              /* directed entries of the graph the arrays refer to     */
    int64_t cut;
    int64_t maxpw;
    int64_t count;          /* pairs matched / moves applied                         */
    const int32_t* a0;
    const int32_t* a1;
    const int32_t* a2;
    const int64_t* rowptr;  /* GP_TR_CONTRACT: the coarse graph                     */
    const int32_t* colidx;
    const int32_t* ewgt;
    const int32_t* vwgt;
} gp_trace_event;

typedef void (*gp_trace_fn)(void* user, const gp_trace_event* ev);

/* Fill *opt with the defaults. */
int gp_default_options(gp_options* opt);

/* Partition a host-resident graph into k parts.  part_out: n int32 (host).
 * Copies the graph to the current CUDA device, runs the V-cycle there and
 * copies the part array back.  Synchronous. */
int gp_partition(int64_t n, const int64_t* rowptr, const int32_t* colidx,
                 const int32_t* vwgt, const int32_t* ewgt, int32_t k,
                 float imbalance, uint64_t seed, int32_t* part_out);

/* Same with options, statistics and tracing (any of the three may be NULL). */
int gp_partition_ex(int64_t n, const int64_t* rowptr, const int32_t* colidx,
                    const int32_t* vwgt, const int32_t* ewgt, int32_t k,
                    float imbalance, uint64_t seed, int32_t* part_out,
                    const gp_options* opt, gp_stats* stats,
                    gp_trace_fn trace, void* trace_user);

/* Device-pointer variant: every array lives in device memory of the current
 * device; work is ordered on `stream` (a cudaStream_t, NULL = legacy default
 * stream).  Returns once the partition is written (the call synchronizes the
 * stream).  One call in flight per device at a time: calls from several host
 * threads are serialized on a per-device lock. */
int gp_partition_device(int64_t n, const int64_t* d_rowptr, const int32_t* d_colidx,
                        const int32_t* d_vwgt, const int32_t* d_ewgt, int32_t k,
                        float imbalance, uint64_t seed, int32_t* d_part_out,
                        void* stream, const gp_options* opt, gp_stats* stats,
                        gp_trace_fn trace, void* trace_user);

/* Exact edge cut of a partition (device pointers).  *cut_out and
 * part_weights_out (k int64, may be NULL) are written to HOST memory.
 * Mirrors computeEdgeCut (src/gpu_part.cu:433-469) but accumulates in int64
 * and does not divide a possibly odd sum: it counts each undirected edge once
 * by summing directed cross entries and halving an even total. */
int gp_edge_cut_device(int64_t n, const int64_t* d_rowptr, const int32_t* d_colidx,
                       const int32_t* d_ewgt, const int32_t* d_vwgt,
                       const int32_t* d_part, int32_t k, void* stream,
                       int64_t* cut_out, int64_t* part_weights_out);

/* Batched mode (no counterpart in the reference): partition ngraphs
 * independent graphs held in device memory in one call.  Graph i is given by
 * ns[i] vertices, ms[i] directed entries and device pointers rowptrs[i],
 * colidxs[i], vwgts[i] (array or entries may be NULL), ewgts[i]; its result,
 * ns[i] part ids in [0, ks[i]), goes to parts_out[i].  Every graph's result is
 * exactly what gp_partition_device returns for it with the same k, imbalance,
 * seed and options.  `workers` concurrent streams (0: 16) take the graphs
 * largest first (by n + m); work starts after prior work on `stream` and
 * `stream` is ordered after all of it.  stats: ngraphs records or NULL.
 * Synchronous. */
int gp_partition_batch_device(int32_t ngraphs, const int64_t* ns, const int64_t* ms,
                              const int64_t* const* d_rowptrs, const int32_t* const* d_colidxs,
                              const int32_t* const* d_vwgts, const int32_t* const* d_ewgts,
                              const int32_t* ks, const float* imbalances, const uint64_t* seeds,
                              int32_t* const* d_parts_out, void* stream, int32_t workers,
                              const gp_options* opt, gp_stats* stats);

/* ---- learned matching priorities (no counterpart in the reference; its run
 * log names a GNNcoarsening.cu that is not in the repository) ------------- */
typedef struct gp_gnn gp_gnn;   /* a small message-passing edge scorer, device resident; its
                                   scratch memory belongs to the handle, so one call at a time
                                   per handle (use one handle per thread for concurrency) */

int gp_gnn_num_params(void);
int gp_gnn_create(gp_gnn** out);                 /* zero weights */
int gp_gnn_destroy(gp_gnn* model);
int gp_gnn_set_params(gp_gnn* model, const float* params, int32_t nparams);   /* host FP32 */
int gp_gnn_get_params(const gp_gnn* model, float* params, int32_t nparams);
/* resolution of the matching priority: rint(logit * 2^bits) + 2^30, bits in
 * [0, 16] (default 16); coarser steps leave near-equal scores to the seeded
 * hash tie-break */
int gp_gnn_set_prio_bits(gp_gnn* model, int32_t bits);
int gp_gnn_get_prio_bits(const gp_gnn* model);
/* learned priorities at levels 0..level only, edge weights above (-1: every level) */
int gp_gnn_set_max_level(gp_gnn* model, int32_t level);
int gp_gnn_get_max_level(const gp_gnn* model);
/* per-entry priorities (int32, may be NULL) and logits (float, may be NULL) of one graph */
int gp_gnn_forward_device(gp_gnn* model, int64_t n, const int64_t* d_rowptr, const int32_t* d_colidx,
                          const int32_t* d_vwgt, const int32_t* d_ewgt, int32_t level, void* stream,
                          int32_t* d_prio_out, float* d_logit_out);
/* mean binary cross-entropy of the edge logits against d_label (1: both ends in one
 * part) and its gradient (host, gp_gnn_num_params() floats) */
int gp_gnn_grad_device(gp_gnn* model, int64_t n, const int64_t* d_rowptr, const int32_t* d_colidx,
                       const int32_t* d_vwgt, const int32_t* d_ewgt, int32_t level, const uint8_t* d_label,
                       void* stream, float* loss_out, float* grad_out);
/* one Adam step on the gradients summed over ngraphs labelled graphs */
int gp_gnn_train_step_device(gp_gnn* model, int32_t ngraphs, const int64_t* ns, const int64_t* const* d_rowptrs,
                             const int32_t* const* d_colidxs, const int32_t* const* d_vwgts,
                             const int32_t* const* d_ewgts, const int32_t* levels,
                             const uint8_t* const* d_labels, float lr, void* stream, float* loss_out);
typedef struct gp_learned_report {
    int64_t cut_learned;              /* exact cut of the learned V-cycle             */
    int64_t cut_plain;                /* exact cut of the plain V-cycle (fallback != 0)   */
    int64_t max_part_weight_learned;
    int64_t max_part_weight_plain;
    double  ms_learned;               /* device time of each V-cycle                   */
    double  ms_plain;
    double  ms_gnn;                   /* part of ms_learned spent in the scorer        */
    int32_t kept_learned;             /* 1: d_part_out holds the learned partition     */
    int32_t reserved;
} gp_learned_report;

/* V-cycle whose matching priority at every level is the model's score instead
 * of the edge weight; all other rules unchanged.  fallback != 0 also runs the
 * plain V-cycle and keeps the learned partition only when it is within the
 * balance bound (or the plain one is not) and its exact cut <= the plain cut;
 * stats describe the partition returned.  The trace covers the learned run. */
int gp_partition_learned_device(int64_t n, const int64_t* d_rowptr, const int32_t* d_colidx,
                                const int32_t* d_vwgt, const int32_t* d_ewgt, int32_t k, float imbalance,
                                uint64_t seed, int32_t* d_part_out, void* stream, const gp_options* opt,
                                gp_stats* stats, const gp_gnn* model, int32_t fallback, gp_learned_report* report,
                                gp_trace_fn trace, void* trace_user);

/* Move-order head of the learned mode (no counterpart in the reference): a
 * second small network (4 features -> 16 hidden -> 1, BF16 weights, FP32
 * accumulation) scores each label-propagation candidate from its integer
 * gain, degree, vertex weight and level; the learned V-cycle's afterburner
 * then assumes the neighbours of higher (score, lower id) move first, in place
 * of the (gain, id) order.  Only the order changes: every move is still
 * re-evaluated exactly and the fallback keeps the plain partition unless the
 * learned one is at least as good.  nparams = 0 removes the head. */
int gp_gnn_move_num_params(void);
int gp_gnn_set_move_params(gp_gnn* model, const float* params, int32_t nparams);
int gp_gnn_get_move_params(const gp_gnn* model, float* params, int32_t nparams);
/* features of every candidate (d_dest[v] >= 0) of one step: 4 floats per vertex */
int gp_gnn_move_features_device(int64_t n, const int64_t* d_rowptr, const int32_t* d_vwgt, const int32_t* d_dest,
                                const int32_t* d_gain, int32_t level, void* stream, float* d_feat_out);
/* scores (float, may be NULL) and move priorities (int32, may be NULL) of ns feature rows */
int gp_gnn_move_scores_device(gp_gnn* model, int64_t ns, const float* d_feat, void* stream, float* d_score_out,
                              int32_t* d_prio_out);
/* mean binary cross-entropy of ns scored rows against d_label and its gradient (host) */
int gp_gnn_move_grad_device(gp_gnn* model, int64_t ns, const float* d_feat, const uint8_t* d_label, void* stream,
                            float* loss_out, float* grad_out);
/* one Adam step of the head on ns labelled rows */
int gp_gnn_move_train_step_device(gp_gnn* model, int64_t ns, const float* d_feat, const uint8_t* d_label, float lr,
                                  void* stream, float* loss_out);

/* Largest k accepted by gp_edge_cut_device_noalloc. */
#define GP_NOALLOC_MAX_K 1024

/* No counterpart in the reference (which has no library API).
 * Same result as gp_edge_cut_device, for callers that must not allocate:
 * code inside an allocator or memory-pool callback (an allocation there
 * re-enters the allocator), loops that forbid allocation after start-up
 * (an allocation can block or fail mid-loop), processes whose device memory
 * another framework has reserved (nothing is left to allocate).
 * gp_edge_cut_device may grow a cached workspace with cudaMalloc on first use;
 * this variant calls no cudaMalloc, cudaFree or other allocating routine.  Its
 * scratch is a fixed array in device memory (about 8 KB, held by every device
 * that loads the library until the process exits), so k must not exceed
 * GP_NOALLOC_MAX_K (GP_EINVAL otherwise).  All calls on a device share that
 * array: calls that overlap on the GPU race and must be serialized by the
 * caller.  Every call looks up the array's address in the current context.
 * Synchronizes `stream`. */
int gp_edge_cut_device_noalloc(int64_t n, const int64_t* d_rowptr, const int32_t* d_colidx,
                               const int32_t* d_ewgt, const int32_t* d_vwgt,
                               const int32_t* d_part, int32_t k, void* stream,
                               int64_t* cut_out, int64_t* part_weights_out);

/* Bounds-checked build (libgp_b200_checked.so, the same sources compiled with
 * -DGP_CHECKED; no counterpart in the reference).  Its kernels test
 * data-dependent indices (neighbour ids, part ids, hash slots, output
 * positions) before using them; a failing test is counted, the first failing
 * site is recorded as translation unit * 100000 + source line, and the access
 * is skipped.  This reports the violations counted on the current device
 * since the last clear (synchronizing it) and, with clear != 0, resets them.
 * The regular library returns GP_EINVAL. */
int gp_checked_violations(int64_t* count, int32_t* first_site, int32_t clear);

/* Release cached device workspaces of the current device. */
int gp_release_workspace(void);

/* Thread-local description of the last error ("" when none). */
const char* gp_last_error(void);

/* Library version string. */
const char* gp_version(void);

#ifdef __cplusplus
}
#endif

#endif /* GP_PARTITION_H */
