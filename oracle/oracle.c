/*
 * oracle.c -- CPU oracle for the concurrent multi-source BFS path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA path is
 * compared against; it is never the thing measured or shipped.  Only the
 * tests, the smoke check and bench.py's cpu_baseline / reference arm load
 * it (as oracle/liboracle.so).
 *
 * Parity pins (what this restatement is checked against):
 *   - oracle_groupby, oracle_teps and the depth arrays of oracle_bfs are
 *     compared in tests/test_oracle_ref.py against the reference's own host
 *     code (GroupBy.cuh, validate.h report/validate, graph.cuh deep_than_two,
 *     graph_reader.cuh) compiled from the reference sources by
 *     oracle/build_ref.sh into oracle/_ref/ref_harness;
 *   - the committed fixtures in tests/golden/ were produced by that harness
 *     and by this oracle (tests/golden/make_golden.py) and are re-checked on
 *     every CPU test run;
 *   - oracle_bfs depths are additionally cross-checked against scipy's
 *     csgraph breadth-first shortest paths (an independent implementation).
 *
 * Everything here is plain C (C11 + optional OpenMP across sources).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_OK 0
#define ORACLE_ERR_RANGE 3
#define ORACLE_ERR_OOM 4
#define ORACLE_ERR_ARG 7

/*
 * Sequential level-synchronous queue BFS from one source.
 *
 * Restates graph.cuh:39-69 (`deep_than_two`: currq/nextq, the
 * `depth[nbr]==INFTY` test, level-synchronous swap of the queues) without
 * its `level==1` early return, and writes the BFS level instead of the
 * reference's 0 marker.  INFTY follows comm.h:120 (255 for one-byte depths);
 * two-byte depths use 0xFFFF.  depth[src] = 0 (the reference's own GPU path
 * leaves sources at INFTY, expander.cuh:46 is commented out; the per-source
 * depth contract of this project uses 0, like every BFS definition).
 *
 * Returns ORACLE_ERR_RANGE when a level does not fit the depth type
 * (level > 254 for 1 byte, > 65534 for 2 bytes).
 */
static int bfs_one(const int64_t *beg, const int32_t *col, int64_t V,
                   int32_t src, int depth_bytes, void *depth_row,
                   int32_t *q_a, int32_t *q_b, int32_t *max_level)
{
    const uint32_t infty = depth_bytes == 1 ? 0xFFu : 0xFFFFu;
    const int64_t lim = depth_bytes == 1 ? 254 : 65534;
    uint8_t *d8 = (uint8_t *)depth_row;
    uint16_t *d16 = (uint16_t *)depth_row;
    if (depth_bytes == 1) memset(d8, 0xFF, (size_t)V);
    else for (int64_t i = 0; i < V; i++) d16[i] = 0xFFFF;
#define GETD(x) (depth_bytes == 1 ? (uint32_t)d8[x] : (uint32_t)d16[x])
#define SETD(x, val) do { if (depth_bytes == 1) d8[x] = (uint8_t)(val); else d16[x] = (uint16_t)(val); } while (0)
    int32_t *currq = q_a, *nextq = q_b;
    int64_t curr_sz = 1, next_sz;
    currq[0] = src;
    SETD(src, 0);
    int64_t level = 0;
    *max_level = 0;
    while (curr_sz > 0) {
        next_sz = 0;
        for (int64_t i = 0; i < curr_sz; i++) {
            int32_t f = currq[i];
            for (int64_t j = beg[f]; j < beg[f + 1]; j++) {
                int32_t nb = col[j];
                if (GETD(nb) == infty) {
                    if (level + 1 > lim) return ORACLE_ERR_RANGE;
                    SETD(nb, level + 1);
                    nextq[next_sz++] = nb;
                }
            }
        }
        if (next_sz > 0) *max_level = (int32_t)(level + 1);
        int32_t *t = currq; currq = nextq; nextq = t;
        curr_sz = next_sz;
        level++;
    }
#undef GETD
#undef SETD
    return ORACLE_OK;
}

/*
 * Per-source depths, source-major: depth_out[i*V + v] is the BFS level of v
 * from src[i] (INFTY when unreachable).  OpenMP across sources with
 * `threads` threads (<=0: all).  max_level_out receives the deepest level.
 */
int oracle_bfs(const int64_t *beg, const int32_t *col, int64_t V,
               const int32_t *src, int64_t n, int depth_bytes,
               void *depth_out, int32_t *max_level_out, int threads)
{
    if (V <= 0 || n < 0 || (depth_bytes != 1 && depth_bytes != 2)) return ORACLE_ERR_ARG;
    for (int64_t i = 0; i < n; i++)
        if (src[i] < 0 || src[i] >= V) return ORACLE_ERR_ARG;
    int rc_all = ORACLE_OK;
    int32_t ml_all = 0;
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
    {
        int32_t *qa = (int32_t *)malloc(sizeof(int32_t) * (size_t)V);
        int32_t *qb = (int32_t *)malloc(sizeof(int32_t) * (size_t)V);
        int32_t ml_local = 0;
        int rc_local = (qa && qb) ? ORACLE_OK : ORACLE_ERR_OOM;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
        for (int64_t i = 0; i < n; i++) {
            if (rc_local != ORACLE_OK) continue;
            int32_t ml = 0;
            int rc = bfs_one(beg, col, V, src[i], depth_bytes,
                             (uint8_t *)depth_out + (size_t)i * (size_t)V * (size_t)depth_bytes,
                             qa, qb, &ml);
            if (rc != ORACLE_OK) rc_local = rc;
            if (ml > ml_local) ml_local = ml;
        }
#ifdef _OPENMP
#pragma omp critical
#endif
        {
            if (rc_local != ORACLE_OK) rc_all = rc_local;
            if (ml_local > ml_all) ml_all = ml_local;
        }
        free(qa);
        free(qb);
    }
    if (max_level_out) *max_level_out = ml_all;
    return rc_all;
}

/*
 * TEPS numerator: for every source, the sum of deg(v) over the vertices it
 * reached; summed over sources.  Restates validate.h:62-76 (`report`:
 * agg_tr_edges += adj_card[i] for every depth != INFTY).
 */
int64_t oracle_teps(const int64_t *beg, int64_t V, const void *depth,
                    int64_t n, int depth_bytes)
{
    int64_t total = 0;
    for (int64_t i = 0; i < n; i++) {
        for (int64_t v = 0; v < V; v++) {
            uint32_t d = depth_bytes == 1
                ? ((const uint8_t *)depth)[i * V + v]
                : ((const uint16_t *)depth)[i * V + v];
            uint32_t inf = depth_bytes == 1 ? 0xFFu : 0xFFFFu;
            if (d != inf) total += beg[v + 1] - beg[v];
        }
    }
    return total;
}

/*
 * GroupBy source reordering.  Restates GroupBy.cuh:19-84:
 *   - a source is eligible when its degree is <= 128 and it has a neighbour
 *     of degree > 128; its hub is the FIRST such neighbour in CSR order
 *     (GroupBy.cuh:22-36);
 *   - eligible sources are bucketed by hub id with a counting sort
 *     (hubmap/huboff prefix sum, GroupBy.cuh:40-43), buckets in ascending
 *     hub id, input order inside a bucket (GroupBy.cuh:62-75);
 *   - every other source follows, in input order (GroupBy.cuh:51-58,77-82).
 * The caller then cuts the result into consecutive batches.
 */
int oracle_groupby(const int64_t *beg, const int32_t *col, int64_t V,
                   const int32_t *src, int64_t n, int32_t *out)
{
    const int64_t HUB = 128;
    int64_t *hubmap = (int64_t *)calloc((size_t)V, sizeof(int64_t));
    int64_t *huboff = (int64_t *)calloc((size_t)V, sizeof(int64_t));
    int32_t *hub_of = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    if (!hubmap || !huboff || !hub_of) { free(hubmap); free(huboff); free(hub_of); return ORACLE_ERR_OOM; }
    for (int64_t i = 0; i < n; i++) {
        int32_t s = src[i];
        hub_of[i] = -1;
        if (beg[s + 1] - beg[s] > HUB) continue;
        for (int64_t j = beg[s]; j < beg[s + 1]; j++) {
            int32_t u = col[j];
            if (beg[u + 1] - beg[u] > HUB) { hub_of[i] = u; hubmap[u]++; break; }
        }
    }
    huboff[0] = 0;
    for (int64_t i = 1; i < V; i++) huboff[i] = huboff[i - 1] + hubmap[i - 1];
    int64_t remainoff = huboff[V - 1] + hubmap[V - 1];
    for (int64_t i = 0; i < n; i++) {
        if (hub_of[i] >= 0) out[huboff[hub_of[i]]++] = src[i];
        else out[remainoff++] = src[i];
    }
    free(hubmap); free(huboff); free(hub_of);
    return ORACLE_OK;
}

/*
 * Algorithmic byte model of one batch (implementation independent; it is a
 * function of the graph and the per-source depths only).
 *
 *   w   = status word bytes (width/8), b_d = depth bytes
 *   F_l = { v : some source s has depth[s][v] == l-1 }           (the JFQ)
 *   U_l = { v : deg(v) > 0, some source s has depth[s][v] >= l } (not done)
 *   TD_l = sum_{v in F_l} (8 + w + deg(v) (4 + w))
 *   BU_l = sum_{v in U_l} (8 + 2w + k_v (4 + w)), k_v = number of neighbours
 *          scanned in CSR order until the OR of their level-(l-1) bits covers
 *          every bit v gains at level l (0 if v gains nothing)
 *   bytes = sum_l min(TD_l, BU_l) + 2 w V + V n b_d
 *
 * `depth` is source-major [n][V].  Levels run 1..max_level+1 (the last one
 * finds nothing new).  Returns the byte count (or -1 on error).
 */
int64_t oracle_bytes_alg(const int64_t *beg, const int32_t *col, int64_t V,
                         const void *depth, int64_t n, int depth_bytes,
                         int width)
{
    const int64_t w = width / 8;
    const uint32_t inf = depth_bytes == 1 ? 0xFFu : 0xFFFFu;
    int32_t maxl = 0;
#define D(s, v) (depth_bytes == 1 ? (uint32_t)((const uint8_t *)depth)[(int64_t)(s) * V + (v)] \
                                  : (uint32_t)((const uint16_t *)depth)[(int64_t)(s) * V + (v)])
    for (int64_t s = 0; s < n; s++)
        for (int64_t v = 0; v < V; v++) {
            uint32_t d = D(s, v);
            if (d != inf && (int32_t)d > maxl) maxl = (int32_t)d;
        }
    int64_t total = 2 * w * V + V * n * depth_bytes;
    const int64_t nw = (n + 63) / 64;
    uint64_t *need = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(nw > 0 ? nw : 1));
    uint64_t *acc = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(nw > 0 ? nw : 1));
    if (!need || !acc) { free(need); free(acc); return -1; }
    for (int32_t l = 1; l <= maxl + 1; l++) {
        int64_t td = 0, bu = 0;
        for (int64_t v = 0; v < V; v++) {
            int64_t deg = beg[v + 1] - beg[v];
            int in_f = 0, in_u = 0;
            for (int64_t s = 0; s < n; s++) {
                uint32_t d = D(s, v);
                if (d == (uint32_t)(l - 1)) in_f = 1;
                if (d == inf || (int32_t)d >= l) in_u = 1;
            }
            if (in_f) td += 8 + w + deg * (4 + w);
            if (in_u && deg > 0) {
                /* bits v gains at level l */
                int any = 0;
                memset(need, 0, sizeof(uint64_t) * (size_t)nw);
                for (int64_t s = 0; s < n; s++)
                    if (D(s, v) == (uint32_t)l) { need[s >> 6] |= 1ull << (s & 63); any = 1; }
                int64_t k = 0;
                if (any) {
                    memset(acc, 0, sizeof(uint64_t) * (size_t)nw);
                    for (int64_t j = beg[v]; j < beg[v + 1]; j++) {
                        int32_t u = col[j];
                        k++;
                        for (int64_t s = 0; s < n; s++) {
                            uint32_t du = D(s, u);
                            if (du != inf && (int32_t)du <= l - 1) acc[s >> 6] |= 1ull << (s & 63);
                        }
                        int covered = 1;
                        for (int64_t q = 0; q < nw; q++)
                            if (need[q] & ~acc[q]) { covered = 0; break; }
                        if (covered) break;
                    }
                }
                bu += 8 + 2 * w + k * (4 + w);
            }
        }
        total += td < bu ? td : bu;
    }
#undef D
    free(need); free(acc);
    return total;
}

/* Number of OpenMP threads the oracle uses by default. */
int oracle_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
