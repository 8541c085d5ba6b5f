/*
 * ibfs.h -- C ABI of the B200 concurrent multi-source BFS (iBFS hot path).
 *
 * Every entry point takes plain pointers and sizes, returns an ibfs_status,
 * never exits the process and never throws across the ABI.  Pointers named
 * *_host are host memory; depth outputs may be host or device memory as
 * flagged.  One handle is used by one host thread at a time; the server
 * (ibfs_server_*) is thread-safe.
 *
 * Reference interfaces each entry point replaces (file:line in iBFS):
 *   ibfs_graph_open        graph_reader::graph_reader      graph_reader.cuh:63-119
 *   ibfs_csr_read          graph_reader::graph_reader      graph_reader.cuh:63-119
 *                          (+ graph<>::alloc_array CSR upload allocator.cuh:3-80)
 *   ibfs_graph_from_csr    graph<>::graph + alloc_array    graph.cuh:246-283, allocator.cuh:18-45
 *   ibfs_graph_close       (none: the reference never frees, gpu_ibfs.cuh:100)
 *   ibfs_groupby           GroupBy                         GroupBy.cuh:6-115
 *   ibfs_groupby_csr       GroupBy                         GroupBy.cuh:6-115
 *   ibfs_run               graph<>::bfs_gpu_coalescing_mem bfs_gpu_opt.cuh:182-262
 *                          -> ibfs()                       bfs_gpu_opt.cuh:39-177
 *   ibfs_read_sources      read_src_v                      graph.cuh:99-133
 *   ibfs_teps              report                          validate.h:59-76
 *   ibfs_strerror          H_ERR / HandleError             comm.h:5-16
 *   ibfs_server_*          (none: the reference runs fixed source lists)
 */
#ifndef IBFS_H
#define IBFS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ibfs_status {
    IBFS_OK = 0,
    IBFS_ERR_IO = 1,          /* file missing / unreadable / short read      */
    IBFS_ERR_FORMAT = 2,      /* CSR files inconsistent                       */
    IBFS_ERR_RANGE = 3,       /* ids or levels do not fit the chosen types    */
    IBFS_ERR_OOM = 4,         /* host or device allocation failed             */
    IBFS_ERR_CUDA = 5,        /* a CUDA call failed                           */
    IBFS_ERR_TIMEOUT = 6,     /* a bounded device wait gave up                */
    IBFS_ERR_INVALID_ARG = 7, /* bad argument                                 */
    IBFS_ERR_UNSUPPORTED = 8, /* option combination not built                 */
    IBFS_ERR_BUSY = 9,        /* admission refused (server full)              */
    IBFS_ERR_NOT_FOUND = 10   /* unknown query id                             */
} ibfs_status;

/* Execution schedules of one run (all give identical depths). */
typedef enum ibfs_mode {
    /* host-driven level loop, one launch per phase, host sync per level:
       the reference's structure (bfs_gpu_opt.cuh:99-166) on sm_100a */
    IBFS_MODE_PLAIN = 0,
    /* one persistent level-synchronous launch for all levels of all batches */
    IBFS_MODE_PERSISTENT = 1,
    /* the PLAIN kernels (one per phase, each at its own occupancy) inside one
       CUDA graph whose conditional nodes run the batch and level loops on
       the device: no host round trip per level, no grid barrier */
    IBFS_MODE_DEVICE_LOOP = 2,
    /* the default: PERSISTENT (with use_graph) when one batch's status words
       fit in 32 MB, where per-kernel launch costs would dominate; DEVICE_LOOP
       above that */
    IBFS_MODE_AUTO = 3
} ibfs_mode;

/* Layout of the depth output of ibfs_run. */
typedef enum ibfs_layout {
    /* depth[i*V + v] = level of v from src[i], sources in the caller's order */
    IBFS_LAYOUT_SOURCE_MAJOR = 0,
    /* per batch b (after GroupBy), rows of that batch's sources:
       depth[b*V*C + v*nb + j] where C = concurrent and nb = sources in b;
       the reference's depth_merge layout (inspector.cuh:48) */
    IBFS_LAYOUT_VERTEX_MAJOR = 1
} ibfs_layout;

/* Flags of ibfs_run. */
#define IBFS_OUT_DEVICE 1u /* depth_out is a device pointer on the graph's GPU */

typedef struct ibfs_graph ibfs_graph;

typedef struct ibfs_opts {
    int32_t width;         /* status bits per vertex: 32, 64, 128 or 256          */
    int32_t concurrent;    /* sources per batch, 1..width (0: width)              */
    int32_t switch_level;  /* >= 0: fixed switch as the reference's CLI argument:
                              top-down while level <= switch_level, bottom-up after;
                              -1: alpha/beta switching                            */
    float alpha;           /* TD->BU when frontier_edges > unexplored_edges/alpha (4) */
    float beta;            /* BU->TD when frontier_vertices < V/beta (24)         */
    int32_t sml_shed;      /* degree < sml_shed: one thread per vertex (default 32) */
    int32_t lrg_shed;      /* degree > lrg_shed: CTA chunks (default 512)         */
    int32_t mode;          /* ibfs_mode (default IBFS_MODE_AUTO)                  */
    int32_t groupby;       /* 1: reorder sources with GroupBy before batching (on
                              the host); 2: the same order computed on the GPU;
                              3: a variant that groups by each source's
                              highest-degree hub, largest hubs first          */
    int32_t depth_bytes;   /* 1 (INFTY 255) or 2 (INFTY 65535); 0: 1, widened to 2
                              automatically when a level exceeds 254              */
    int32_t groups;        /* batches run concurrently (0: auto; device loop: 4)  */
    int32_t threads;       /* threads per CTA (0: 512)                            */
    int32_t ctas_per_sm;   /* persistent grid = SMs * ctas_per_sm (0: auto)       */
    int32_t use_graph;     /* persistent: 1 captures the run in a CUDA graph and
                              replays it on reuse (the device loop is always a
                              graph, rebuilt only when buffers or options move)   */
    int32_t timeout_ms;    /* budget of every bounded device wait (0: 10000)      */
    int32_t max_levels;    /* abort with IBFS_ERR_RANGE beyond this (0: 65534)    */
    int32_t debug_withhold;/* test hook: CTA 0 never arrives at its first grid
                              barrier, so every wait runs out (IBFS_ERR_TIMEOUT)  */
    int32_t occupancy;     /* persistent kernel register budget / warps per SM:
                              0: 512 threads x 2 CTAs (64 regs), 1: 256 x 6 (42),
                              2: 256 x 8 (32), 3: 512 x 1 (128)                 */
    int32_t bu_filter;     /* bottom-up reads a neighbour's status only when the
                              previous frontier bitmap has it (exact: no other
                              neighbour can add a bit): 1 on every level, 0 off,
                              -1 (default) on levels whose previous frontier
                              holds fewer than V/16 vertices                      */
    int32_t bu_thread_max; /* bottom-up: vertices of degree <= this scan alone, one
                              thread each; above it a warp scans (0: 32)          */
    int32_t td_stage;      /* 1: top-down stages each large vertex's adjacency
                              chunk in shared memory by double-buffered bulk
                              (TMA) copies (plain and device-loop schedules);
                              0 (default): reads the chunk directly              */
    int32_t sparse_push;   /* device loop: d > 0 makes a bottom-up level that
                              follows a top-down one push, top-down, the sources
                              whose previous frontier is below 1/d of the
                              batch's average, instead of letting them hold up
                              every vertex's early exit (exact either way).
                              0 (default) or < 0: off.  On R-MAT scale 24 with
                              d = 256 it measured 35.0 vs 31.1 ms per run      */
    int32_t reserved[2];
} ibfs_opts;

typedef struct ibfs_level_rec {
    int32_t batch;         /* batch index                                         */
    int32_t level;         /* level expanded                                      */
    int32_t dir;           /* 0 top-down, 1 bottom-up, -1 level 0 (seeding),
                              2 the batch's output pass (persistent, device loop) */
    int32_t pad;
    int64_t frontier;      /* vertices whose status changed at this level         */
    int64_t frontier_edges;/* sum of their degrees                                */
    int64_t expand_ns;     /* device time of the level's expand phase (persistent
                              and device loop; 0 in the plain schedule; level 0:
                              seeding; dir 2: the output pass)                    */
    int64_t inspect_ns;    /* device time of its inspect phase                    */
} ibfs_level_rec;

typedef struct ibfs_stats {
    int64_t n_sources;
    int64_t n_batches;
    int32_t max_level;      /* deepest BFS level over all sources                 */
    int32_t depth_bytes;    /* depth type actually used                           */
    int32_t width;          /* status width actually used                         */
    int32_t groups;         /* concurrent batches per launch actually used        */
    int64_t levels_total;   /* sum over batches of levels expanded                */
    int64_t td_levels;
    int64_t bu_levels;
    int64_t traversed_edges;/* sum_s sum_{v reached from s} deg(v)                */
    int64_t gpu_launches;   /* kernels launched by this run                       */
    double device_ms;       /* device time of the traversal (CUDA events)         */
    double total_ms;        /* wall time of the call incl. transfers              */
    ibfs_level_rec *levels; /* optional caller array for per-level records        */
    int32_t levels_cap;     /* its capacity                                       */
    int32_t levels_len;     /* records written                                    */
} ibfs_stats;

/* ---- status ------------------------------------------------------------ */
const char *ibfs_strerror(ibfs_status s);
/* Library version string. */
const char *ibfs_version(void);

/* ---- graph ------------------------------------------------------------- */
/* Load <beg_pos.bin> ((V+1) little-endian uint64, beg[V]=E) and <csr.bin>
   (E uint64), validate, and upload to `device`. */
ibfs_status ibfs_graph_open(const char *beg_path, const char *csr_path,
                            int device, ibfs_graph **out);
/* Same from host arrays (beg_pos int64[V+1], col int32[E]); data is copied. */
ibfs_status ibfs_graph_from_csr(const int64_t *beg_pos_host,
                                const int32_t *col_host, int64_t V,
                                int64_t E, int device, ibfs_graph **out);
/* Host-only read of the same files (graph_reader, graph_reader.cuh:63-119,
   with validation instead of asserts): beg int64[V+1], col int32[E],
   malloc'ed by the library (free with ibfs_free). */
ibfs_status ibfs_csr_read(const char *beg_path, const char *csr_path,
                          int64_t **beg, int32_t **col, int64_t *V, int64_t *E);
ibfs_status ibfs_graph_info(const ibfs_graph *g, int64_t *V, int64_t *E,
                            int64_t *max_degree);
/* Device pointers of the resident CSR (beg int64[V+1], col int32[E]), in
   the graph's internal vertex order: vertices sorted by degree, highest
   first (ties by id), every list ascending.  ibfs_graph_vertex_order gives
   the renaming; every other entry point takes and returns caller ids. */
ibfs_status ibfs_graph_device_csr(const ibfs_graph *g, const int64_t **beg,
                                  const int32_t **col);
/* Device array new_of_old[V]: the internal id of every caller vertex id. */
ibfs_status ibfs_graph_vertex_order(const ibfs_graph *g, const int32_t **new_of_old);
ibfs_status ibfs_graph_close(ibfs_graph *g);

/* ---- sources ----------------------------------------------------------- */
/* GroupBy reorder (host, exact restatement of GroupBy.cuh:19-84). */
ibfs_status ibfs_groupby(const ibfs_graph *g, const int32_t *src_host,
                         int64_t n, int32_t *out_host);
/* The batch order of ibfs_opts.groupby = 3 (no counterpart in the reference:
   its GroupBy variant keyed by each source's highest-degree hub). */
ibfs_status ibfs_groupby_maxhub(const ibfs_graph *g, const int32_t *src_host, int64_t n,
                                int32_t *out_host);
/* GroupBy of device-resident sources on the graph's GPU: the order of
   ibfs_groupby (GroupBy.cuh:19-84), from a per-vertex hub table built at
   upload and a sort of n keys.  out_dev[k] = the k-th source of the order;
   pos_dev (optional) = its index in src_dev.  Asynchronous on the graph's
   stream (ibfs_set_stream); src_dev and out_dev must not overlap. */
ibfs_status ibfs_groupby_device(ibfs_graph *g, const int32_t *src_dev, int64_t n,
                                int32_t *out_dev, int32_t *pos_dev);
/* GroupBy on host CSR arrays (no graph handle, no GPU). */
ibfs_status ibfs_groupby_csr(const int64_t *beg_host, const int32_t *col_host,
                             int64_t V, const int32_t *src_host, int64_t n,
                             int32_t *out_host);
/* The largest-hub variant (groupby = 3) on host CSR arrays; no counterpart
   in the reference. */
ibfs_status ibfs_groupby_csr_maxhub(const int64_t *beg_host, const int32_t *col_host,
                                    int64_t V, const int32_t *src_host, int64_t n,
                                    int32_t *out_host);
/* read_src_v format: one decimal vertex id per line.  With ids == NULL only
   *n is set; otherwise up to cap ids are written. */
ibfs_status ibfs_read_sources(const char *path, int32_t *ids, int64_t cap,
                              int64_t *n);
ibfs_status ibfs_write_sources(const char *path, const int32_t *ids, int64_t n);

/* ---- traversal --------------------------------------------------------- */
void ibfs_opts_default(ibfs_opts *o);
/* Concurrent BFS from n sources.  depth_out holds n*V*depth_bytes bytes in
   `layout`; flags: IBFS_OUT_DEVICE.  stats may be NULL.  Replays the cached
   CUDA graph when opts->use_graph is set and the call matches the last one. */
ibfs_status ibfs_run(ibfs_graph *g, const int32_t *src_host, int64_t n,
                     const ibfs_opts *opts, void *depth_out, int32_t layout,
                     uint32_t flags, ibfs_stats *stats);
/* Launch on a caller stream (cudaStream_t) instead of the handle's own. */
ibfs_status ibfs_set_stream(ibfs_graph *g, void *cuda_stream);

/* ---- serving (no counterpart in the reference, which runs one fixed
   source list, bfs_gpu_opt.cuh:182-262) --------------------------------- */
typedef struct ibfs_server ibfs_server;
typedef struct ibfs_server_opts {
    ibfs_opts run;           /* traversal options of every round               */
    int64_t arena_bytes;     /* device memory for per-query depth rows
                                (0: a quarter of the free device memory)       */
    int32_t max_waiting;     /* queued submissions beyond this: IBFS_ERR_BUSY  */
    int32_t round_batches;   /* batches traversed at once (the device loop's
                                concurrent groups); also the most batches'
                                worth of sources regrouped together            */
    int32_t max_wait_us;     /* a partial batch waits this long for sources
                                (only while no published batch is unclaimed)   */
    int32_t groupby;         /* regroup pending sources with GroupBy           */
    int32_t reserved[6];
} ibfs_server_opts;
typedef struct ibfs_query_info {
    int64_t n_sources;
    double latency_ms;       /* submission to depths complete on the device     */
    double queue_ms;         /* submission to the first round that included it  */
    int32_t status;          /* ibfs_status of the query                        */
    int32_t depth_bytes;
    double delivered_ms;     /* submission to depths in the caller's buffer
                                (the poll or wait that collected the query)     */
} ibfs_query_info;
typedef struct ibfs_server_stats {
    int64_t submitted, completed, refused;
    int64_t rounds;          /* batches traversed                               */
    int64_t sources, traversed_edges;
    double busy_ms;          /* device time of the serving graph's launches     */
    double wall_ms;          /* since creation                                  */
    int64_t arena_rows, arena_rows_used;
    int64_t launches;        /* serving-graph launches: batches published while
                                the graph runs join it, so launches < rounds
                                under load                                      */
} ibfs_server_stats;
void ibfs_server_opts_default(ibfs_server_opts *o);
/* Start a server (worker thread) on a resident graph. */
ibfs_status ibfs_server_create(ibfs_graph *g, const ibfs_server_opts *o,
                               ibfs_server **out);
/* Queue a query of n sources; thread safe.  IBFS_ERR_BUSY when the waiting
   queue is full, IBFS_ERR_RANGE when n rows can never fit the arena. */
ibfs_status ibfs_server_submit(ibfs_server *s, const int32_t *src_host, int64_t n,
                               uint64_t *qid);
/* Non-blocking: *done = 1 and depths [n][V] copied to depth_out (host, or
   device with IBFS_OUT_DEVICE; NULL to discard) once complete; the query is
   then forgotten. */
ibfs_status ibfs_server_poll(ibfs_server *s, uint64_t qid, void *depth_out,
                             uint32_t flags, int32_t *done, ibfs_query_info *info);
/* Blocking variant with a timeout (IBFS_ERR_TIMEOUT). */
ibfs_status ibfs_server_wait(ibfs_server *s, uint64_t qid, int32_t timeout_ms,
                             void *depth_out, uint32_t flags, ibfs_query_info *info);
ibfs_status ibfs_server_stats_get(ibfs_server *s, ibfs_server_stats *out);
/* Rows of V depths of depth_bytes each that an arena of arena_bytes holds:
   the query capacity of ibfs_server_create, capped at INT32_MAX (output
   rows are int32 indices on the device).  0 for invalid arguments. */
int64_t ibfs_server_arena_rows(int64_t arena_bytes, int64_t V, int32_t depth_bytes);
ibfs_status ibfs_server_destroy(ibfs_server *s);

/* Per-graph tuning (no counterpart in the reference, whose constants are
   fixed at comm.h:25-30 and ibfs.cu:71-72): coordinate descent over width,
   alpha/beta, queue thresholds, occupancy (persistent schedule) and
   concurrent batches, each trial a real run of `src` in the base options'
   schedule (device output, `reps` timed repeats).
   `best` receives the winner; `log` (optional) one JSON object per trial. */
ibfs_status ibfs_autotune(ibfs_graph *g, const int32_t *src_host, int64_t n,
                          const ibfs_opts *base, int32_t reps, ibfs_opts *best,
                          double *best_gteps, char *log, int32_t log_cap);

/* TEPS numerator on the host: sum over sources of deg(v) for reached v
   (validate.h:59-76) of a source-major depth array. */
ibfs_status ibfs_teps(const ibfs_graph *g, const void *depth_host, int64_t n,
                      int32_t depth_bytes, int64_t *edges);

/* Algorithmic bytes of one batch (the implementation-independent byte
   model: sum over levels of min(top-down, bottom-up) bytes plus status init
   and depth output), computed on the GPU from a device source-major depth
   array of n sources. */
ibfs_status ibfs_bytes_alg(ibfs_graph *g, const void *depth_dev, int64_t n,
                           int32_t depth_bytes, int32_t width, int64_t *bytes);

/* No counterpart in the reference.  Concurrent BFS that allocates nothing,
   for callers that cannot call cudaMalloc (a plug-in inside a process whose
   allocator owns all device memory, a latency-critical path that may not
   stall in cudaMalloc, a deployment that forbids allocation after start-up).
   All inputs and the output are the caller's device memory: the CSR
   (beg_dev int64[V+1], col_dev int32[E]), the source ids src_dev int32[n]
   and depth_dev, which receives uint8 depths (INFTY 255) in the vertex-major
   layout with batches of `width` sources: batch b at b*V*width, rows of
   min(width, n - b*width) bytes.  Scratch comes from one fixed 64 MiB device
   array inside the library (held by every GPU that loads it, until exit);
   graphs whose scratch does not fit, more than 16 batches, or a level past
   254 return IBFS_ERR_RANGE.  Runs on the calling thread's current device;
   every call looks up the array's address in the current context, and the
   first call on a device also loads the library's device code there, so
   make that first call before any stream capture.  Calls share the array: calls whose
   work overlaps on one GPU race and must be serialised by the caller.
   Synchronises `cuda_stream` (a cudaStream_t, NULL = legacy stream) before
   returning; traversed_edges (may be NULL) receives the TEPS numerator. */
ibfs_status ibfs_run_static_scratch(const int64_t *beg_dev, const int32_t *col_dev,
                                    int64_t V, int64_t E, const int32_t *src_dev,
                                    int64_t n, int32_t width, void *depth_dev,
                                    void *cuda_stream, int64_t *traversed_edges);

/* ---- synthetic inputs (seeded, deterministic, host) -------------------- */
/* Each generator symmetrises, drops self-loops, dedupes and sorts every
   adjacency list.  Arrays are malloc'ed by the library; free with ibfs_free. */
ibfs_status ibfs_gen_rmat(int32_t scale, int32_t edge_factor, double a,
                          double b, double c, uint64_t seed, int64_t **beg,
                          int32_t **col, int64_t *V, int64_t *E);
ibfs_status ibfs_gen_grid(int32_t rows, int32_t cols, double delete_frac,
                          double shortcut_frac, uint64_t seed, int64_t **beg,
                          int32_t **col, int64_t *V, int64_t *E);
ibfs_status ibfs_gen_chung_lu(int64_t n, int64_t m, double gamma,
                              double max_degree, uint64_t seed, int64_t **beg,
                              int32_t **col, int64_t *V, int64_t *E);
/* Build a CSR from an undirected edge list (same cleaning rules). */
ibfs_status ibfs_csr_from_edges(const int32_t *src, const int32_t *dst,
                                int64_t m, int64_t V, int64_t **beg,
                                int32_t **col, int64_t *E);
/* Write the reference's binary CSR pair (uint64 little-endian). */
ibfs_status ibfs_write_csr(const char *beg_path, const char *csr_path,
                           const int64_t *beg, const int32_t *col, int64_t V);

/* Edge-list text -> binary CSR files on the GPU: the reference converter
   tuple_text_to_bin.cpp:56-310 (whitespace-separated id pairs after
   `skip_lines` header lines; ids shifted by the smallest id).  clean = 0:
   the reference's CSR exactly (file order within every list, both
   directions with `reverse`, duplicates and self loops kept); clean = 1:
   symmetrised, self loops dropped, lists sorted and deduplicated.  Writes
   beg_path / csr_path in the iBFS format; V_out / E_out optional.  An odd
   number of tokens is IBFS_ERR_FORMAT. */
ibfs_status ibfs_convert_text(const char *text_path, int32_t reverse, int64_t skip_lines,
                              int32_t clean, const char *beg_path, const char *csr_path,
                              int32_t device, int64_t *V_out, int64_t *E_out);
/* Sample n distinct sources uniformly (seeded) among vertices with degree
   > 0 (component < 0) or inside the largest connected component
   (component >= 0). */
ibfs_status ibfs_sample_sources(const int64_t *beg, const int32_t *col,
                                int64_t V, int64_t n, uint64_t seed,
                                int32_t component, int32_t *out);
void ibfs_free(void *p);

#ifdef __cplusplus
}
#endif
#endif /* IBFS_H */
