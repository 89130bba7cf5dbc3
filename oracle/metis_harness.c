/*
 * metis_harness.c -- METIS 5 baseline (test / benchmark infrastructure only).
 *
 * The reference partitions its coarsest graph by running the external
 * `gpmetis -ptype=rb` binary (src/gpu_part.cu:857).  gpmetis is not installed
 * here; this harness links the METIS library that ships with the CUDA toolkit
 * (libmetis_static.a, 64-bit idx_t) and calls its public API directly, so the
 * whole input graph can be partitioned by METIS for a quality and wall-time
 * baseline.  The prototypes below are METIS 5's documented public API; no
 * metis.h is installed.  Default options (ufactor 30 = 3% imbalance for k-way).
 */
#include <stdint.h>
#include <stdlib.h>
#include <time.h>

typedef int64_t idx_t;
typedef float real_t;

#define METIS_NOPTIONS 40
#define METIS_OPTION_SEED 8
#define METIS_OK 1

int METIS_SetDefaultOptions(idx_t *options);
int METIS_PartGraphKway(idx_t *nvtxs, idx_t *ncon, idx_t *xadj, idx_t *adjncy,
                        idx_t *vwgt, idx_t *vsize, idx_t *adjwgt, idx_t *nparts,
                        real_t *tpwgts, real_t *ubvec, idx_t *options,
                        idx_t *edgecut, idx_t *part);
int METIS_PartGraphRecursive(idx_t *nvtxs, idx_t *ncon, idx_t *xadj, idx_t *adjncy,
                             idx_t *vwgt, idx_t *vsize, idx_t *adjwgt, idx_t *nparts,
                             real_t *tpwgts, real_t *ubvec, idx_t *options,
                             idx_t *edgecut, idx_t *part);

/* Returns the METIS status (1 = OK) or -2 when host memory runs out.
 * *seconds_out receives the wall time of the METIS call alone. */
int gpm_partition(int64_t n, const int64_t *rowptr, const int32_t *colidx,
                  const int32_t *vwgt, const int32_t *ewgt, int32_t k,
                  int64_t seed, int recursive, int32_t *part_out,
                  int64_t *cut_out, double *seconds_out) {
    int64_t m = rowptr[n];
    idx_t *xadj = malloc(sizeof(idx_t) * (size_t)(n + 1));
    idx_t *adj = malloc(sizeof(idx_t) * (size_t)(m > 0 ? m : 1));
    idx_t *vw = vwgt ? malloc(sizeof(idx_t) * (size_t)n) : NULL;
    idx_t *ew = ewgt ? malloc(sizeof(idx_t) * (size_t)(m > 0 ? m : 1)) : NULL;
    idx_t *part = malloc(sizeof(idx_t) * (size_t)n);
    if (!xadj || !adj || !part || (vwgt && !vw) || (ewgt && !ew)) {
        free(xadj); free(adj); free(vw); free(ew); free(part);
        return -2;
    }
    for (int64_t i = 0; i <= n; ++i) xadj[i] = rowptr[i];
    for (int64_t e = 0; e < m; ++e) adj[e] = colidx[e];
    if (vw) for (int64_t i = 0; i < n; ++i) vw[i] = vwgt[i];
    if (ew) for (int64_t e = 0; e < m; ++e) ew[e] = ewgt[e];
    idx_t nv = n, ncon = 1, np = k, cut = 0;
    idx_t opt[METIS_NOPTIONS];
    METIS_SetDefaultOptions(opt);
    opt[METIS_OPTION_SEED] = seed;
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    int rc;
    if (k == 1) {
        for (int64_t i = 0; i < n; ++i) part[i] = 0;
        rc = METIS_OK;
    } else if (recursive) {
        rc = METIS_PartGraphRecursive(&nv, &ncon, xadj, adj, vw, NULL, ew, &np, NULL, NULL, opt, &cut, part);
    } else {
        rc = METIS_PartGraphKway(&nv, &ncon, xadj, adj, vw, NULL, ew, &np, NULL, NULL, opt, &cut, part);
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (seconds_out) *seconds_out = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
    for (int64_t i = 0; i < n; ++i) part_out[i] = (int32_t)part[i];
    if (cut_out) *cut_out = cut;
    free(xadj); free(adj); free(vw); free(ew); free(part);
    return rc;
}
