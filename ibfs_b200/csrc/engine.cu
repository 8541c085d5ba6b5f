// engine.cu -- the resident-graph handle, ibfs_run and two of its schedules.
//
// Three schedules run the same phase functions (bfs_device.cuh):
//   PLAIN        host-driven level loop: one launch per phase and a host
//                synchronisation per level to read the counters -- the shape
//                of the reference's ibfs() loop (bfs_gpu_opt.cuh:99-166);
//   PERSISTENT   one cooperative launch runs every level of every batch: the
//                grid is cut into G groups of CTAs, each group owns one batch
//                at a time and synchronises with a bounded team barrier; the
//                direction decision is taken on the device.  Optionally the
//                whole run (uploads, launch, downloads) is captured once in a
//                CUDA graph and replayed;
//   DEVICE_LOOP  the plain kernels inside one CUDA graph whose conditional
//                nodes run the batch and level loops (devloop.cu).
// AUTO picks PERSISTENT for small graphs and DEVICE_LOOP otherwise.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "bfs_device.cuh"
#include "internal.h"
#include "launch_common.cuh"

namespace ibfs {

// ---------------------------------------------------------------------------
// Kernels (the persistent kernel: persistent.cuh, one translation unit per
// status width, persistent_w*.cu)
// ---------------------------------------------------------------------------
// ---- plain schedule: one kernel per phase, the whole grid is the team ----
template <int WORDS>
__global__ void __launch_bounds__(512) k_seed(Params p, int b) {
  const Team t = make_team(blockIdx.x, gridDim.x);
  const long long k0 = (long long)b * p.C;
  const int n_b = (int)min((long long)p.C, p.n_total - k0);
  seed_phase<WORDS>(p, p.groups[0], p.src + k0, n_b, t);
}

template <int WORDS>
__global__ void __launch_bounds__(512) k_inspect(Params p, GroupBufs gb, int b, int level) {
  const Team t = make_team(blockIdx.x, gridDim.x);
  const long long k0 = (long long)b * p.C;
  const int n_b = (int)min((long long)p.C, p.n_total - k0);
  inspect_phase<WORDS, false>(p, gb, &gb.ctl->par[level & 1], n_b, level,
                              level <= depth_limit(p.db), false, t);
}

__global__ void __launch_bounds__(512) k_qbuild(Params p, GroupBufs gb, int level) {
  const Team t = make_team(blockIdx.x, gridDim.x);
  qbuild_phase(p, gb, level, gb.ctl->qc[level & 1], t);
}

template <int WORDS>
__global__ void __launch_bounds__(512) k_td(Params p, GroupBufs gb, int level) {
  const Team t = make_team(blockIdx.x, gridDim.x);
  td_phase<WORDS, true>(p, gb, level, gb.ctl->qc[level & 1], t);
}

template <int WORDS>
__global__ void __launch_bounds__(512) k_bu(Params p, GroupBufs gb, int level) {
  const Team t = make_team(blockIdx.x, gridDim.x);
  bu_phase<WORDS, false, true>(p, gb, level, gb.ctl->par[(level - 1) & 1].fmask,
                               &gb.ctl->par[level & 1].hq_cnt, t, nullptr, 0, true,
                               bu_filter_level(p.bu_filter, gb.ctl->par[(level - 1) & 1].changed,
                                               p.V));
}

template <int WORDS>
__global__ void __launch_bounds__(512) k_bu_defer(Params p, GroupBufs gb, int level) {
  const Team t = make_team(blockIdx.x, gridDim.x);
  bu_defer_phase<WORDS, true>(p, gb, level, gb.ctl->par[(level - 1) & 1].fmask,
                              &gb.ctl->par[level & 1].hq_cnt, t,
                              bu_filter_level(p.bu_filter, gb.ctl->par[(level - 1) & 1].changed,
                                              p.V));
}

template <int WORDS>
__global__ void __launch_bounds__(512) k_output(Params p, GroupBufs gb, int b, int max_level) {
  __shared__ int32_t s_rows[kMaxWords * 32];
  const Team t = make_team(blockIdx.x, gridDim.x);
  const long long k0 = (long long)b * p.C;
  const int n_b = (int)min((long long)p.C, p.n_total - k0);
  load_rows(p, b, n_b, s_rows);
  output_phase<WORDS>(p, gb, batch_depth(p, b), s_rows, n_b, max_level, t);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
#define CU(call)                                       \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) {                           \
      last_cuda_error() = e_;                          \
      (void)cudaGetLastError();                        \
      return e_ == cudaErrorMemoryAllocation ? IBFS_ERR_OOM : IBFS_ERR_CUDA; \
    }                                                  \
  } while (0)

static cudaError_t& last_cuda_error() {
  static thread_local cudaError_t e = cudaSuccess;
  return e;
}

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ibfs_status ensure(size_t want) {
    if (want <= bytes && p) return IBFS_OK;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(want, 256));
    if (e != cudaSuccess) {
      p = nullptr;
      last_cuda_error() = e;
      return IBFS_ERR_OOM;
    }
    bytes = std::max<size_t>(want, 256);
    return IBFS_OK;
  }
  // Small per-run buffers grow to powers of two so that their addresses
  // (baked into cached CUDA graphs) stay put across runs of similar size.
  ibfs_status ensure_pow2(size_t want) {
    size_t r = 4096;
    while (r < want) r <<= 1;
    return want <= bytes && p ? IBFS_OK : ensure(r);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

struct PinBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ibfs_status ensure(size_t want) {
    if (want <= bytes && p) return IBFS_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    if (cudaMallocHost(&p, std::max<size_t>(want, 256)) != cudaSuccess) {
      p = nullptr;
      return IBFS_ERR_OOM;
    }
    bytes = std::max<size_t>(want, 256);
    return IBFS_OK;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

struct GroupMem {
  DevBuf last, curr, chg, qs, qm, ql, hq, ctl, planes;
  void release() {
    last.release(); curr.release(); chg.release(); qs.release();
    qm.release(); ql.release(); hq.release(); ctl.release(); planes.release();
  }
};

struct GraphCache {
  cudaGraphExec_t exec = nullptr;
  std::string key;
  void release() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    key.clear();
  }
};

}  // namespace ibfs

using namespace ibfs;

struct ibfs_graph {
  int device = 0;
  int sms = 0;
  int64_t V = 0, E = 0, max_deg = 0;
  HostCsr h;
  DevBuf beg, col;
  DevBuf gbhub;         // GroupBy's hub of every vertex (-1: not eligible), device GroupBy
  DevBuf vmap;          // caller id -> internal id (device)
  std::vector<int32_t> new_of_old;  // the same on the host
  std::vector<int64_t> dbeg_host;   // offsets of the internal (degree-ordered) CSR
  int64_t col_max = -1;             // largest neighbour id of the internal CSR
  DevBuf gbin, gbkeys;  // device GroupBy: caller-order sources, sort keys
  int64_t defer_cap = 16;  // bound on deferred bottom-up hub chunks per level
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // workspace
  std::vector<GroupMem> groups;
  DevBuf d_groups, d_src, d_outrow, d_brec, d_lrec, d_out;
  PinBuf h_src, h_outrow, h_brec, h_lrec, h_par;
  GraphCache gcache;
  // depth sink of host-buffer runs, and the device loop's per-batch done
  // flags in mapped host memory (h_done; d_done is their device address)
  DepthSink sink;
  int32_t* h_done = nullptr;
  int32_t* d_done = nullptr;
  size_t done_cap = 0;
  cudaEvent_t ev_out = nullptr;
  // device-loop graphs, keyed by the launch Params: a few entries, because a
  // server's rounds alternate between group counts (1..4 batches per round)
  static constexpr int kDlCache = 4;
  GraphCache dlcache[kDlCache];
  unsigned dl_next = 0;
  std::mutex mu;
};

namespace ibfs {

static const int kLrecCap = 1024;

static int words_for(int width) { return width / 32; }

static ibfs_status check_opts(const ibfs_opts* o) {
  if (o->width != 32 && o->width != 64 && o->width != 128 && o->width != 256)
    return IBFS_ERR_INVALID_ARG;
  if (o->concurrent < 0 || o->concurrent > o->width) return IBFS_ERR_INVALID_ARG;
  if (o->mode != IBFS_MODE_PLAIN && o->mode != IBFS_MODE_PERSISTENT &&
      o->mode != IBFS_MODE_DEVICE_LOOP && o->mode != IBFS_MODE_AUTO)
    return IBFS_ERR_INVALID_ARG;
  if (o->depth_bytes != 0 && o->depth_bytes != 1 && o->depth_bytes != 2) return IBFS_ERR_INVALID_ARG;
  if (o->threads != 0 && o->threads != 128 && o->threads != 256 && o->threads != 512)
    return IBFS_ERR_INVALID_ARG;
  if (o->alpha <= 0 || o->beta <= 0) return IBFS_ERR_INVALID_ARG;
  if (o->sml_shed < 1 || o->lrg_shed < o->sml_shed - 1) return IBFS_ERR_INVALID_ARG;
  if (o->groupby < 0 || o->groupby > 3) return IBFS_ERR_INVALID_ARG;
  if (o->groups < 0 || o->ctas_per_sm < 0 || o->timeout_ms < 0 || o->max_levels < 0)
    return IBFS_ERR_INVALID_ARG;
  if (o->bu_thread_max < 0 || o->bu_thread_max > (1 << 20)) return IBFS_ERR_INVALID_ARG;
  return IBFS_OK;
}

// Per-group workspace bytes for (V, W, C, db).
static size_t group_bytes(int64_t V, int64_t E, int words, int C, int db, int lrg, int chunk,
                          bool /*unused*/) {
  const size_t vpad = (size_t)((V + 31) & ~31LL);
  const size_t nchg = (size_t)(((V + 31) / 32 + 127) & ~127LL);
  const size_t capl = (size_t)(E / std::max(chunk, 1) + std::min<int64_t>(V, E / std::max(lrg, 1)) + 16);
  size_t b = 2 * vpad * words * 4 + nchg * 4 + 2 * (size_t)V * 4 + capl * 8 + sizeof(Ctl);
  b += (size_t)(db == 1 ? 8 : 16) * vpad * words * 4 + nchg * 4;  // planes + 2nd bitmap
  return b;
}

// Occupancy levels of the persistent kernel: threads per CTA; the CTAs per
// SM its register budget is sized for are 2, 6, 8 and 1 (the template
// arguments below).
static const int kOccThreads[4] = {512, 256, 256, 512};

static const void* persistent_for(int words, int level = 0) {
  switch (words) {
    case 1: return persistent_fn_w32(level);
    case 2: return persistent_fn_w64(level);
    case 4: return persistent_fn_w128(level);
    default: return persistent_fn_w256(level);
  }
}


template <int WORDS>
static cudaError_t launch_plain_level(const Params& p, const GroupBufs& gb, int sms, int threads,
                                      int level, int dir, cudaStream_t s) {
  if (dir == kDirTD) {
    k_qbuild<<<occ_grid((const void*)k_qbuild, threads, sms), threads, 0, s>>>(p, gb, level);
    k_td<WORDS><<<occ_grid((const void*)k_td<WORDS>, threads, sms), threads, 0, s>>>(p, gb, level);
  } else {
    k_bu<WORDS><<<occ_grid((const void*)k_bu<WORDS>, threads, sms), threads, 0, s>>>(p, gb, level);
    k_bu_defer<WORDS><<<occ_grid((const void*)k_bu_defer<WORDS>, threads, sms), threads, 0, s>>>(
        p, gb, level);
  }
  return cudaGetLastError();
}

template <int WORDS>
static cudaError_t launch_plain_inspect(const Params& p, const GroupBufs& gb, int sms, int threads,
                                        int b, int level, cudaStream_t s) {
  k_inspect<WORDS><<<occ_grid((const void*)k_inspect<WORDS>, threads, sms), threads, 0, s>>>(
      p, gb, b, level);
  return cudaGetLastError();
}

template <int WORDS>
static cudaError_t launch_plain_seed(const Params& p, int sms, int threads, int b, cudaStream_t s) {
  k_seed<WORDS><<<sms, threads, 0, s>>>(p, b);
  return cudaGetLastError();
}

template <int WORDS>
static cudaError_t launch_plain_output(const Params& p, const GroupBufs& gb, int sms, int threads,
                                       int b, int max_level, cudaStream_t s) {
  k_output<WORDS><<<occ_grid((const void*)k_output<WORDS>, threads, sms), threads, 0, s>>>(
      p, gb, b, max_level);
  return cudaGetLastError();
}

struct RunPlan {
  int words, C, nbatches, G, cpg, threads, grid, db;
  size_t smem;
  bool host_out;
};

// Allocate / reuse the workspace for G groups.
static ibfs_status ensure_workspace(ibfs_graph* g, const RunPlan& rp, const ibfs_opts& o,
                                    int layout) {
  (void)layout;
  const size_t vpad = (size_t)((g->V + 31) & ~31LL);
  const size_t nchg = (size_t)(((g->V + 31) / 32 + 127) & ~127LL);
  const int chunk = rp.threads * 4;
  const size_t capl = (size_t)(g->E / chunk + std::min<int64_t>(g->V, g->E / std::max(o.lrg_shed, 1)) + 16);
  if ((int)g->groups.size() < rp.G) g->groups.resize(rp.G);
  for (int i = 0; i < rp.G; i++) {
    GroupMem& m = g->groups[i];
    ibfs_status s;
    if ((s = m.last.ensure(vpad * rp.words * 4)) != IBFS_OK) return s;
    if ((s = m.curr.ensure(vpad * rp.words * 4)) != IBFS_OK) return s;
    if ((s = m.chg.ensure(2 * nchg * 4)) != IBFS_OK) return s;
    if ((s = m.planes.ensure((size_t)(rp.db == 1 ? 8 : 16) * vpad * rp.words * 4)) != IBFS_OK)
      return s;
    if ((s = m.qs.ensure((size_t)g->V * 4)) != IBFS_OK) return s;
    if ((s = m.qm.ensure((size_t)g->V * 4)) != IBFS_OK) return s;
    if ((s = m.ql.ensure(capl * 8)) != IBFS_OK) return s;
    if ((s = m.hq.ensure((size_t)g->defer_cap * 8)) != IBFS_OK) return s;
    if ((s = m.ctl.ensure(sizeof(Ctl))) != IBFS_OK) return s;
  }
  return IBFS_OK;
}

}  // namespace ibfs

#ifndef IBFS_BU_SKIP_EDGELESS
#define IBFS_BU_SKIP_EDGELESS 1
#endif
namespace ibfs {
// The launch parameters that depend only on the resident graph and the
// options (the run's sources, rows, output, groups and records are left
// null/zero for the caller).
void fill_graph_params(const ibfs_graph* g, const ibfs_opts& o, int words, int threads,
                       Params* pp) {
  Params& p = *pp;
  std::memset(&p, 0, sizeof(p));
  p.beg = g->beg.as<int64_t>();
  p.col = g->col.as<int32_t>();
  p.V = g->V;
  p.E = g->E;
  p.nchg = (g->V + 31) / 32;
  p.chg_stride = (p.nchg + 127) & ~127LL;  // whole 128-word blocks (vector bitmap walks)
  p.plane_stride = (long long)((g->V + 31) & ~31LL) * words;
  p.sml = o.sml_shed;
  p.lrg = o.lrg_shed;
  p.chunk = threads * 4;
  p.but = o.bu_thread_max > 0 ? o.bu_thread_max : 32;
  p.switch_level = o.switch_level;
  p.alpha = o.alpha;
  p.beta = o.beta;
  p.max_levels = o.max_levels ? o.max_levels : 65534;
  p.timeout_ns = (unsigned long long)(o.timeout_ms ? o.timeout_ms : 10000) * 1000000ull;
  p.withhold = o.debug_withhold;
  p.hub_t = kHubScan;
  p.bu_filter = o.bu_filter > 0 ? 1 : o.bu_filter == 0 ? 0 : -1;
  p.td_stage = o.td_stage > 0 ? 1 : 0;
  // sparse-source pushes on bottom-up levels: device loop only (the caller
  // clears it for the other schedules)
  p.sparse_div = o.sparse_push > 0 ? o.sparse_push : 0;
  p.col_vec = 1;
  p.vmap = g->vmap.as<int32_t>();
  // Degrees are non-increasing in the internal order: the vertices above the
  // thread-path limit form a prefix (rounded up to whole warps).  When each
  // warp owns only a few 32-vertex ranges of the bottom-up sweep (small
  // graphs), the warps that own the hub ranges would be the critical path,
  // so the prefix then gets one warp per vertex; on large graphs the ranges
  // average out and the per-lane sweep is faster (R-MAT scale 16: 1.26 ->
  // 0.45 ms per run with the prefix pass; scale 24: 34.8 vs 40.7 ms without
  // and with it).
  // Degrees are non-increasing in the internal order, so the edgeless
  // vertices form a suffix: the bottom-up sweeps stop before it (rounded up
  // to whole 32-vertex ranges).
  {
    int64_t lo = 0, hi = g->V;
    while (lo < hi) {
      const int64_t mid = (lo + hi) / 2;
      if (g->dbeg_host[(size_t)mid + 1] - g->dbeg_host[(size_t)mid] > 0) lo = mid + 1;
      else hi = mid;
    }
    p.v_nz = IBFS_BU_SKIP_EDGELESS ? std::min<int64_t>((lo + 31) & ~31LL, g->V) : g->V;
    // no edge points into the edgeless suffix (symmetric graphs): only a
    // source reaches a vertex there (a directed graph's sinks can be reached)
    p.v_reach = g->col_max < p.v_nz ? p.v_nz : g->V;
  }
  const int64_t ranges_per_warp = ((g->V + 31) / 32) / std::max<int64_t>(1, (int64_t)g->sms * 64);
  if (ranges_per_warp < 8) {
    int64_t lo = 0, hi = g->V;
    while (lo < hi) {
      const int64_t mid = (lo + hi) / 2;
      if (g->dbeg_host[(size_t)mid + 1] - g->dbeg_host[(size_t)mid] > p.but) lo = mid + 1;
      else hi = mid;
    }
    p.big_prefix = std::min<int64_t>((lo + 31) & ~31LL, (g->V + 31) & ~31LL);
  }
}

// The output pointer and the store widths its alignment allows.
void set_output_params(const ibfs_graph* g, int C, uint8_t* dout, Params* p) {
  p->out = dout;
  p->vec_out = (C % 4 == 0) && ((reinterpret_cast<uintptr_t>(dout) & 3) == 0);
  p->vec_sm = (g->V % 16 == 0 && (reinterpret_cast<uintptr_t>(dout) & 15) == 0)  ? 16
              : (g->V % 4 == 0 && (reinterpret_cast<uintptr_t>(dout) & 3) == 0) ? 4
                                                                               : 0;
}

int graph_sms(const ibfs_graph* g) { return g->sms; }
int64_t graph_defer_cap(const ibfs_graph* g) { return g->defer_cap; }
const int32_t* graph_new_of_old(const ibfs_graph* g) { return g->new_of_old.data(); }
}  // namespace ibfs

namespace ibfs {

// Key of a captured persistent run.  A captured graph holds raw addresses:
// the kernel's Params (CSR, sources, rows, output, group table, records,
// vertex map), every group's workspace (copied from the pinned group table
// at replay), the pinned staging buffers its copies read and write, and the
// device GroupBy's buffers.  Any run outside the graph path may grow (free
// and reallocate) one of them, so all of them are part of the key: a moved
// buffer means a new capture, never a replay into freed memory.
static std::string make_key(const ibfs_graph* g, const int32_t* src, int64_t n, const ibfs_opts& o,
                            void* out, int layout, uint32_t flags, const RunPlan& rp,
                            const Params& p, const GroupBufs* hgb, int G,
                            const void* const* extra, int n_extra) {
  std::string k;
  k.append(reinterpret_cast<const char*>(&o), sizeof(o));
  k.append(reinterpret_cast<const char*>(&rp), sizeof(rp));
  k.append(reinterpret_cast<const char*>(&out), sizeof(out));
  k.append(reinterpret_cast<const char*>(&layout), sizeof(layout));
  k.append(reinterpret_cast<const char*>(&flags), sizeof(flags));
  k.append(reinterpret_cast<const char*>(&n), sizeof(n));
  k.append(reinterpret_cast<const char*>(&g->stream), sizeof(g->stream));
  k.append(reinterpret_cast<const char*>(&p), sizeof(p));
  k.append(reinterpret_cast<const char*>(hgb), sizeof(GroupBufs) * (size_t)G);
  k.append(reinterpret_cast<const char*>(extra), sizeof(void*) * (size_t)n_extra);
  if (!(flags & IBFS_OUT_DEVICE)) k.append(reinterpret_cast<const char*>(src), sizeof(int32_t) * n);
  return k;
}

}  // namespace ibfs

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" const char* ibfs_strerror(ibfs_status s) {
  switch (s) {
    case IBFS_OK: return "ok";
    case IBFS_ERR_IO: return "i/o error (file missing, unreadable or short)";
    case IBFS_ERR_FORMAT: return "malformed CSR input";
    case IBFS_ERR_RANGE: return "value out of range (vertex id, edge count or BFS level)";
    case IBFS_ERR_OOM: return "out of memory";
    case IBFS_ERR_CUDA: return "CUDA error";
    case IBFS_ERR_TIMEOUT: return "a bounded device wait timed out";
    case IBFS_ERR_INVALID_ARG: return "invalid argument";
    case IBFS_ERR_UNSUPPORTED: return "unsupported option combination";
    case IBFS_ERR_BUSY: return "admission refused: server at capacity";
    case IBFS_ERR_NOT_FOUND: return "unknown query id";
  }
  return "unknown status";
}

extern "C" const char* ibfs_version(void) { return "ibfs-b200 0.1 (sm_100a)"; }

extern "C" void ibfs_opts_default(ibfs_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->width = 128;
  o->concurrent = 0;
  o->switch_level = -1;
  o->alpha = 4.0f;
  o->beta = 24.0f;
  o->sml_shed = 32;
  o->lrg_shed = 512;
  o->mode = IBFS_MODE_AUTO;
  o->groupby = 0;
  o->depth_bytes = 0;
  o->groups = 0;
  o->threads = 0;
  o->ctas_per_sm = 0;
  o->use_graph = 0;
  o->timeout_ms = 0;
  o->max_levels = 0;
  o->debug_withhold = 0;
  o->occupancy = 0;
  o->bu_filter = -1;  // default: per level, on when the previous frontier is small
  o->bu_thread_max = 32;
}

static ibfs_status upload_graph(ibfs_graph* g) {
  CU(cudaSetDevice(g->device));
  int sms = 0;
  CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
  g->sms = sms;
  ibfs_status s;
  if ((s = g->beg.ensure(sizeof(int64_t) * (size_t)(g->V + 1))) != IBFS_OK) return s;
  // + 4 entries: the bottom-up reads column ids as aligned 16-byte vectors
  if ((s = g->col.ensure(sizeof(int32_t) * (size_t)(g->E + 4))) != IBFS_OK) return s;
  CU(cudaMemset(g->col.p, 0, sizeof(int32_t) * (size_t)(g->E + 4)));
  CU(cudaStreamCreateWithFlags(&g->own_stream, cudaStreamNonBlocking));
  g->stream = g->own_stream;
  CU(cudaEventCreate(&g->ev0));
  CU(cudaEventCreate(&g->ev1));
  CU(cudaEventCreateWithFlags(&g->ev_out, cudaEventDisableTiming));
  // Internal vertex order: by degree, highest first (ties by caller id).
  // Vertices of similar degree then share warps (the bottom-up thread path
  // runs lanes of equal trip counts) and the hubs' status words, which most
  // gathers hit, are packed into a few contiguous lines of L2 -- measured on
  // R-MAT scale 24: 45.5 -> 27.6 ms per 1024-source run.  Depths do not
  // depend on the order: sources are renamed on the way in, and the output
  // pass reads statuses through the map, writing rows in the caller's order.
  // The device adjacency lists are in this order too, sorted ascending,
  // which is by neighbour degree, highest first: the bottom-up sweep stops at
  // the first neighbours that cover the missing bits, and hubs carry the
  // most bits earliest.  The host copy keeps the caller's order (GroupBy's
  // "first hub in CSR order" and the byte model use it).
  {
    const int64_t* bg = g->h.beg.data();
    const int32_t* cl = g->h.col.data();
    std::vector<int32_t> order;
    std::vector<int64_t> nbeg;
    std::vector<int32_t> dcol;
    try {
      order.resize((size_t)g->V);
      g->new_of_old.resize((size_t)g->V);
      nbeg.resize((size_t)g->V + 1);
      dcol.resize((size_t)std::max<int64_t>(g->E, 1));
    } catch (const std::bad_alloc&) {
      return IBFS_ERR_OOM;
    }
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [bg](int32_t a, int32_t b) {
      return bg[a + 1] - bg[a] > bg[b + 1] - bg[b];
    });
    for (int64_t i = 0; i < g->V; i++) g->new_of_old[(size_t)order[(size_t)i]] = (int32_t)i;
    nbeg[0] = 0;
    for (int64_t i = 0; i < g->V; i++) {
      const int32_t o = order[(size_t)i];
      nbeg[(size_t)i + 1] = nbeg[(size_t)i] + (bg[o + 1] - bg[o]);
    }
    const int32_t* nmap = g->new_of_old.data();
    int64_t col_max = -1;
#pragma omp parallel for schedule(dynamic, 4096) reduction(max : col_max)
    for (int64_t i = 0; i < g->V; i++) {
      const int32_t o = order[(size_t)i];
      int32_t* out = dcol.data() + nbeg[(size_t)i];
      const int64_t d = bg[o + 1] - bg[o];
      for (int64_t e = 0; e < d; e++) out[e] = nmap[cl[bg[o] + e]];
      std::sort(out, out + d);
      if (d > 0) col_max = std::max<int64_t>(col_max, out[d - 1]);
    }
    g->col_max = col_max;
    CU(cudaMemcpyAsync(g->beg.p, nbeg.data(), sizeof(int64_t) * (size_t)(g->V + 1),
                       cudaMemcpyHostToDevice, g->stream));
    g->dbeg_host = nbeg;  // (the copy is synchronised below)
    if (g->E)
      CU(cudaMemcpyAsync(g->col.p, dcol.data(), sizeof(int32_t) * (size_t)g->E,
                         cudaMemcpyHostToDevice, g->stream));
    if ((s = g->vmap.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(g->V, 1))) != IBFS_OK)
      return s;
    CU(cudaMemcpyAsync(g->vmap.p, nmap, sizeof(int32_t) * (size_t)g->V, cudaMemcpyHostToDevice,
                       g->stream));
    CU(cudaStreamSynchronize(g->stream));
  }
  // GroupBy's hub of every vertex (GroupBy.cuh:19-84): for degree <= 128,
  // the first neighbour in the caller's order whose degree is > 128; -1 when
  // there is none or the vertex is not eligible.  One int per vertex, so that
  // a device GroupBy is a key per source and a sort.
  {
    std::vector<int32_t> hub;
    try {
      hub.assign((size_t)g->V, -1);
    } catch (const std::bad_alloc&) {
      return IBFS_ERR_OOM;
    }
    const int64_t* bg = g->h.beg.data();
    const int32_t* cl = g->h.col.data();
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < g->V; v++) {
      if (bg[v + 1] - bg[v] > 128) continue;
      for (int64_t e = bg[v]; e < bg[v + 1]; e++) {
        const int32_t u = cl[e];
        if (bg[u + 1] - bg[u] > 128) {
          hub[(size_t)v] = u;
          break;
        }
      }
    }
    if ((s = g->gbhub.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(g->V, 1))) != IBFS_OK)
      return s;
    CU(cudaMemcpyAsync(g->gbhub.p, hub.data(), sizeof(int32_t) * (size_t)g->V,
                       cudaMemcpyHostToDevice, g->stream));
    CU(cudaStreamSynchronize(g->stream));
  }
  CU(cudaStreamSynchronize(g->stream));
  int64_t md = 0;
  for (int64_t v = 0; v < g->V; v++) md = std::max(md, g->h.beg[v + 1] - g->h.beg[v]);
  g->max_deg = md;
  // bound on the bottom-up hub chunks one level can defer
  {
    int64_t cap = 16;
    for (int64_t v = 0; v < g->V; v++) {
      const int64_t d = g->h.beg[v + 1] - g->h.beg[v];
      if (d > kHubScan) cap += (d - kHubScan + kHubChunk - 1) / kHubChunk;
    }
    g->defer_cap = cap;
  }
  return IBFS_OK;
}

static void destroy_graph(ibfs_graph* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  g->gcache.release();
  for (auto& c : g->dlcache) c.release();
  for (auto& m : g->groups) m.release();
  g->beg.release();
  g->col.release();
  g->gbhub.release();
  g->vmap.release();
  g->gbin.release();
  g->gbkeys.release();
  g->d_groups.release();
  g->d_src.release();
  g->d_outrow.release();
  g->d_brec.release();
  g->d_lrec.release();
  g->d_out.release();
  g->h_src.release();
  g->h_outrow.release();
  g->h_brec.release();
  g->h_lrec.release();
  g->h_par.release();
  g->sink.release();
  if (g->h_done) cudaFreeHost(g->h_done);
  if (g->ev_out) cudaEventDestroy(g->ev_out);
  if (g->ev0) cudaEventDestroy(g->ev0);
  if (g->ev1) cudaEventDestroy(g->ev1);
  if (g->own_stream) cudaStreamDestroy(g->own_stream);
  delete g;
}

extern "C" ibfs_status ibfs_graph_open(const char* beg_path, const char* csr_path, int device,
                                       ibfs_graph** out) {
  if (!beg_path || !csr_path || !out) return IBFS_ERR_INVALID_ARG;
  *out = nullptr;
  ibfs_graph* g = new (std::nothrow) ibfs_graph();
  if (!g) return IBFS_ERR_OOM;
  g->device = device;
  ibfs_status s = load_csr_files(beg_path, csr_path, &g->h);
  if (s == IBFS_OK) {
    g->V = g->h.V;
    g->E = g->h.E;
    s = upload_graph(g);
  }
  if (s != IBFS_OK) {
    destroy_graph(g);
    return s;
  }
  *out = g;
  return IBFS_OK;
}

extern "C" ibfs_status ibfs_graph_from_csr(const int64_t* beg_pos_host, const int32_t* col_host,
                                           int64_t V, int64_t E, int device, ibfs_graph** out) {
  if (!beg_pos_host || (!col_host && E > 0) || !out || V <= 0 || E < 0) return IBFS_ERR_INVALID_ARG;
  *out = nullptr;
  ibfs_status s = validate_csr(beg_pos_host, col_host, V, E);
  if (s != IBFS_OK) return s;
  ibfs_graph* g = new (std::nothrow) ibfs_graph();
  if (!g) return IBFS_ERR_OOM;
  g->device = device;
  try {
    g->h.V = V;
    g->h.E = E;
    g->h.beg.assign(beg_pos_host, beg_pos_host + V + 1);
    g->h.col.assign(col_host, col_host + E);
  } catch (const std::bad_alloc&) {
    delete g;
    return IBFS_ERR_OOM;
  }
  g->V = V;
  g->E = E;
  s = upload_graph(g);
  if (s != IBFS_OK) {
    destroy_graph(g);
    return s;
  }
  *out = g;
  return IBFS_OK;
}

extern "C" ibfs_status ibfs_graph_info(const ibfs_graph* g, int64_t* V, int64_t* E,
                                       int64_t* max_degree) {
  if (!g) return IBFS_ERR_INVALID_ARG;
  if (V) *V = g->V;
  if (E) *E = g->E;
  if (max_degree) *max_degree = g->max_deg;
  return IBFS_OK;
}

extern "C" ibfs_status ibfs_graph_device_csr(const ibfs_graph* g, const int64_t** beg,
                                             const int32_t** col) {
  if (!g) return IBFS_ERR_INVALID_ARG;
  if (beg) *beg = g->beg.as<int64_t>();
  if (col) *col = g->col.as<int32_t>();
  return IBFS_OK;
}

extern "C" ibfs_status ibfs_graph_vertex_order(const ibfs_graph* g, const int32_t** new_of_old) {
  if (!g || !new_of_old) return IBFS_ERR_INVALID_ARG;
  *new_of_old = g->vmap.as<int32_t>();
  return IBFS_OK;
}

extern "C" ibfs_status ibfs_graph_close(ibfs_graph* g) {
  if (!g) return IBFS_ERR_INVALID_ARG;
  destroy_graph(g);
  return IBFS_OK;
}

extern "C" ibfs_status ibfs_set_stream(ibfs_graph* g, void* cuda_stream) {
  if (!g) return IBFS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g->mu);
  g->stream = cuda_stream ? (cudaStream_t)cuda_stream : g->own_stream;
  g->gcache.release();
  return IBFS_OK;
}

// GroupBy of device-resident sources on the graph's GPU (groupby_dev.cu):
// the same order as ibfs_groupby, computed on the device.  Asynchronous on
// the graph's stream; allocates its sort keys once per size class.
extern "C" ibfs_status ibfs_groupby_device(ibfs_graph* g, const int32_t* src_dev, int64_t n,
                                           int32_t* out_dev, int32_t* pos_dev) {
  if (!g || n < 0 || (n > 0 && (!src_dev || !out_dev)) || n > INT32_MAX)
    return IBFS_ERR_INVALID_ARG;
  if (n == 0) return IBFS_OK;
  if (src_dev == out_dev) return IBFS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g->mu);
  CU(cudaSetDevice(g->device));
  ibfs_status s;
  if ((s = g->gbkeys.ensure_pow2(sizeof(unsigned long long) * groupby_dev_pad(n))) != IBFS_OK)
    return s;
  CU(groupby_dev_run(g->gbhub.as<int32_t>(), src_dev, n, g->gbkeys.as<unsigned long long>(),
                     out_dev, pos_dev, g->stream));
  return IBFS_OK;
}

extern "C" ibfs_status ibfs_groupby(const ibfs_graph* g, const int32_t* src_host, int64_t n,
                                    int32_t* out_host) {
  if (!g || (!src_host && n > 0) || (!out_host && n > 0) || n < 0) return IBFS_ERR_INVALID_ARG;
  for (int64_t i = 0; i < n; i++)
    if (src_host[i] < 0 || src_host[i] >= g->V) return IBFS_ERR_RANGE;
  groupby_host(g->h.beg.data(), g->h.col.data(), g->V, src_host, n, out_host);
  return IBFS_OK;
}

// The batch order of ibfs_opts.groupby = 3 (largest-hub variant) on the host.
extern "C" ibfs_status ibfs_groupby_maxhub(const ibfs_graph* g, const int32_t* src_host,
                                           int64_t n, int32_t* out_host) {
  if (!g || (!src_host && n > 0) || (!out_host && n > 0) || n < 0) return IBFS_ERR_INVALID_ARG;
  for (int64_t i = 0; i < n; i++)
    if (src_host[i] < 0 || src_host[i] >= g->V) return IBFS_ERR_RANGE;
  groupby_host_maxhub(g->h.beg.data(), g->h.col.data(), g->V, src_host, n, out_host);
  return IBFS_OK;
}

extern "C" ibfs_status ibfs_teps(const ibfs_graph* g, const void* depth_host, int64_t n,
                                 int32_t depth_bytes, int64_t* edges) {
  if (!g || !depth_host || !edges || n < 0 || (depth_bytes != 1 && depth_bytes != 2))
    return IBFS_ERR_INVALID_ARG;
  int64_t total = 0;
  const int64_t V = g->V;
#pragma omp parallel for reduction(+ : total) schedule(static)
  for (int64_t i = 0; i < n; i++) {
    int64_t t = 0;
    for (int64_t v = 0; v < V; v++) {
      const bool reached = depth_bytes == 1
                               ? ((const uint8_t*)depth_host)[i * V + v] != 0xFF
                               : ((const uint16_t*)depth_host)[i * V + v] != 0xFFFF;
      if (reached) t += g->h.beg[v + 1] - g->h.beg[v];
    }
    total += t;
  }
  *edges = total;
  return IBFS_OK;
}

// Order sources (GroupBy or identity) and map each ordered position to the
// caller's index.  Duplicated ids keep their order of appearance.
// rule: 0 none, 1 GroupBy (GroupBy.cuh:19-84), 3 the largest-hub variant
static void order_sources(const ibfs_graph* g, const int32_t* src, int64_t n, int rule,
                          std::vector<int32_t>* ord, std::vector<int32_t>* row) {
  ord->assign(src, src + n);
  row->resize((size_t)n);
  if (rule != 1 && rule != 3) {
    std::iota(row->begin(), row->end(), 0);
    return;
  }
  if (rule == 3) groupby_host_maxhub(g->h.beg.data(), g->h.col.data(), g->V, src, n, ord->data());
  else groupby_host(g->h.beg.data(), g->h.col.data(), g->V, src, n, ord->data());
  // map ids back to positions (stable for duplicates)
  std::vector<std::pair<int32_t, int32_t>> pos((size_t)n);
  for (int64_t i = 0; i < n; i++) pos[i] = {src[i], (int32_t)i};
  std::sort(pos.begin(), pos.end());
  std::vector<int64_t> used;
  std::vector<std::pair<int32_t, int32_t>> ordk((size_t)n);
  for (int64_t k = 0; k < n; k++) ordk[k] = {(*ord)[k], (int32_t)k};
  std::stable_sort(ordk.begin(), ordk.end(),
                   [](const std::pair<int32_t, int32_t>& a, const std::pair<int32_t, int32_t>& b) {
                     return a.first < b.first;
                   });
  // both sorted by id; equal ids pair up in order of appearance / order
  for (int64_t i = 0; i < n; i++) (*row)[ordk[i].second] = pos[i].second;
}

static ibfs_status run_once(ibfs_graph* g, const int32_t* src, int64_t n, const ibfs_opts& o,
                            int db, void* depth_out, int32_t layout, uint32_t flags,
                            ibfs_stats* st, bool* range_hit, const int32_t* rows_in = nullptr);

extern "C" ibfs_status ibfs_run(ibfs_graph* g, const int32_t* src_host, int64_t n,
                                const ibfs_opts* opts, void* depth_out, int32_t layout,
                                uint32_t flags, ibfs_stats* stats) {
  if (!g || !src_host || n <= 0 || !depth_out) return IBFS_ERR_INVALID_ARG;
  if (layout != IBFS_LAYOUT_SOURCE_MAJOR && layout != IBFS_LAYOUT_VERTEX_MAJOR)
    return IBFS_ERR_INVALID_ARG;
  ibfs_opts o;
  if (opts) o = *opts;
  else ibfs_opts_default(&o);
  ibfs_status s = check_opts(&o);
  if (s != IBFS_OK) return s;
  for (int64_t i = 0; i < n; i++)
    if (src_host[i] < 0 || src_host[i] >= g->V) return IBFS_ERR_RANGE;
  std::lock_guard<std::mutex> lk(g->mu);
  if (cudaSetDevice(g->device) != cudaSuccess) return IBFS_ERR_CUDA;
  const auto t0 = std::chrono::steady_clock::now();
  bool range_hit = false;
  int db = o.depth_bytes == 0 ? 1 : o.depth_bytes;
  s = run_once(g, src_host, n, o, db, depth_out, layout, flags, stats, &range_hit);
  if (s == IBFS_ERR_RANGE && range_hit && o.depth_bytes == 0) {
    db = 2;
    s = run_once(g, src_host, n, o, db, depth_out, layout, flags, stats, &range_hit);
  }
  if (stats) {
    stats->total_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return s;
}

// IBFS_MODE_AUTO: small graphs (one batch's status words within 32 MB, a
// few levels of short kernels) run the persistent kernel from a CUDA graph,
// where the device loop's per-kernel launch costs would dominate; larger
// ones run the device loop.
static ibfs_opts resolve_mode(const ibfs_graph* g, const ibfs_opts& in) {
  ibfs_opts o = in;
  if (o.mode == IBFS_MODE_AUTO) {
    const bool small = (double)g->V * (o.width / 8) <= 32.0 * 1024 * 1024;
    o.mode = small ? IBFS_MODE_PERSISTENT : IBFS_MODE_DEVICE_LOOP;
    if (small && !o.debug_withhold) o.use_graph = 1;
  }
  return o;
}

static ibfs_status run_once(ibfs_graph* g, const int32_t* src, int64_t n, const ibfs_opts& o_in,
                            int db, void* depth_out, int32_t layout, uint32_t flags,
                            ibfs_stats* st, bool* range_hit, const int32_t* rows_in) {
  *range_hit = false;
  const ibfs_opts o = resolve_mode(g, o_in);
  cudaStream_t s = g->stream;
  RunPlan rp;
  std::memset(&rp, 0, sizeof(rp));
  rp.words = words_for(o.width);
  rp.C = o.concurrent ? o.concurrent : o.width;
  rp.nbatches = (int)((n + rp.C - 1) / rp.C);
  const int occ_level = (o.occupancy >= 0 && o.occupancy <= 3) ? o.occupancy : 0;
  rp.threads = o.mode == IBFS_MODE_PERSISTENT ? kOccThreads[occ_level]
                                              : (o.threads ? o.threads : 512);
  rp.db = db;
  rp.host_out = !(flags & IBFS_OUT_DEVICE);
  rp.smem = 0;
  const bool persistent = o.mode == IBFS_MODE_PERSISTENT;
  const bool devloop = o.mode == IBFS_MODE_DEVICE_LOOP;
  // grid sizing
  int occ = 0;
  CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, persistent_for(rp.words, occ_level), rp.threads,
                                                   rp.smem));
  if (occ < 1) return IBFS_ERR_UNSUPPORTED;
  int per_sm = o.ctas_per_sm ? std::min(o.ctas_per_sm, occ) : occ;
  const int total_ctas = g->sms * per_sm;
  if (persistent) {
    int G = o.groups;
    if (G == 0) {
      // enough CTAs per group to sweep V with >= 8 words of 32 vertices per warp
      const int64_t want = std::max<int64_t>(1, (g->V + 32LL * 8 * (rp.threads / 32) - 1) /
                                                    (32LL * 8 * (rp.threads / 32)));
      G = (int)std::max<int64_t>(1, std::min<int64_t>(rp.nbatches, total_ctas / std::min<int64_t>(want, total_ctas)));
      // memory guard (only when the workspace has to grow to G groups)
      size_t freeb = 0, totb = 0;
      if ((int)g->groups.size() < G && cudaMemGetInfo(&freeb, &totb) == cudaSuccess) {
        const size_t per = group_bytes(g->V, g->E, rp.words, rp.C, db, o.lrg_shed, rp.threads * 4,
                                       false);
        const size_t budget = (size_t)(freeb * 0.5);
        G = (int)std::max<size_t>(1, std::min<size_t>((size_t)G, budget / std::max<size_t>(per, 1)));
      }
    }
    G = std::max(1, std::min(G, std::min(rp.nbatches, total_ctas)));
    rp.G = G;
    rp.cpg = total_ctas / G;
    rp.grid = rp.cpg * G;
  } else if (devloop) {
    // concurrent batches are parallel branches of the graph; each kernel is
    // sized by its own occupancy, so groups only overlap one batch's serial
    // stretches (decisions, small levels) with another's work
    int G = std::min(o.groups ? o.groups : 4, rp.nbatches);  // 4: best on R-MAT s22-24
    size_t freeb = 0, totb = 0;
    if (G > 1 && (int)g->groups.size() < G && cudaMemGetInfo(&freeb, &totb) == cudaSuccess) {
      const size_t per = group_bytes(g->V, g->E, rp.words, rp.C, db, o.lrg_shed, rp.threads * 4,
                                     false);
      G = (int)std::max<size_t>(1, std::min<size_t>((size_t)G, (size_t)(freeb * 0.5) /
                                                                  std::max<size_t>(per, 1)));
    }
    rp.G = std::max(1, std::min(G, rp.nbatches));
    rp.cpg = total_ctas;
    rp.grid = total_ctas;
  } else {
    rp.G = 1;
    rp.cpg = total_ctas;
    rp.grid = total_ctas;
  }
  ibfs_status es = ensure_workspace(g, rp, o, layout);
  if (es != IBFS_OK) return es;
  // ordered sources and their output rows
  std::vector<int32_t> ord, row;
  if (rows_in) {
    ord.assign(src, src + n);  // already batched by the caller (the server)
    row.assign(rows_in, rows_in + n);
  } else {
    // groupby 2: the device regroups (groupby_dev.cu) after the upload
    order_sources(g, src, n, o.groupby == 2 ? 0 : o.groupby, &ord, &row);
  }
  const bool dev_gb = o.groupby == 2 && !rows_in;
  ibfs_status bs;
  if ((bs = g->h_src.ensure(sizeof(int32_t) * n)) != IBFS_OK) return bs;
  if ((bs = g->h_outrow.ensure(sizeof(int32_t) * n)) != IBFS_OK) return bs;
  if ((bs = g->d_src.ensure_pow2(sizeof(int32_t) * n)) != IBFS_OK) return bs;
  if ((bs = g->d_outrow.ensure_pow2(sizeof(int32_t) * n)) != IBFS_OK) return bs;
  int64_t gb_launches = 0;
  if (dev_gb) {
    const int64_t npad = groupby_dev_pad(n);
    if ((bs = g->gbin.ensure_pow2(sizeof(int32_t) * n)) != IBFS_OK) return bs;
    if ((bs = g->gbkeys.ensure_pow2(sizeof(unsigned long long) * npad)) != IBFS_OK) return bs;
    int lg = 0;
    while ((1LL << lg) < npad) lg++;
    gb_launches = 2 + (npad <= 4096 ? 1 : (int64_t)lg * (lg + 1) / 2);
  }
  // sources and output rows to the device: as ordered on the host, or in the
  // caller's order and regrouped there
  auto upload_sources = [&](cudaStream_t cs) -> ibfs_status {
    if (dev_gb) {
      CU(cudaMemcpyAsync(g->gbin.p, g->h_src.p, sizeof(int32_t) * n, cudaMemcpyHostToDevice, cs));
      CU(groupby_dev_run(g->gbhub.as<int32_t>(), g->gbin.as<int32_t>(), n,
                         g->gbkeys.as<unsigned long long>(), g->d_src.as<int32_t>(),
                         g->d_outrow.as<int32_t>(), cs, g->vmap.as<int32_t>()));
    } else {
      CU(cudaMemcpyAsync(g->d_src.p, g->h_src.p, sizeof(int32_t) * n, cudaMemcpyHostToDevice, cs));
      CU(cudaMemcpyAsync(g->d_outrow.p, g->h_outrow.p, sizeof(int32_t) * n,
                         cudaMemcpyHostToDevice, cs));
    }
    return IBFS_OK;
  };
  if ((bs = g->d_brec.ensure_pow2(sizeof(BatchRec) * rp.nbatches)) != IBFS_OK) return bs;
  if ((bs = g->h_brec.ensure(sizeof(BatchRec) * rp.nbatches)) != IBFS_OK) return bs;
  if ((bs = g->d_lrec.ensure_pow2(sizeof(LevelRec) * (size_t)rp.nbatches * kLrecCap)) != IBFS_OK)
    return bs;
  if ((bs = g->h_lrec.ensure(sizeof(LevelRec) * (size_t)rp.nbatches * kLrecCap)) != IBFS_OK) return bs;
  if ((bs = g->d_groups.ensure(sizeof(GroupBufs) * rp.G)) != IBFS_OK) return bs;
  if ((bs = g->h_par.ensure(sizeof(Ctl) * rp.G + sizeof(GroupBufs) * rp.G)) != IBFS_OK) return bs;
  const size_t out_bytes = (size_t)n * (size_t)g->V * db;
  uint8_t* dout = nullptr;
  if (rp.host_out) {
    if ((bs = g->d_out.ensure(out_bytes)) != IBFS_OK) return bs;
    dout = g->d_out.as<uint8_t>();
  } else {
    dout = reinterpret_cast<uint8_t*>(depth_out);
  }
  // In the vertex-major layout batch blocks are [V][C] even for the last,
  // partial batch: the block of batch b starts at b*V*C.
  if (layout == IBFS_LAYOUT_VERTEX_MAJOR && rp.nbatches * (size_t)rp.C > (size_t)n) {
    // the last batch uses V*n_b bytes of its block; the caller buffer holds
    // exactly n*V*db bytes, which covers every block start.
  }
  {
    // sources in the graph's internal order (the device GroupBy renames its
    // output itself; it takes the caller's ids)
    int32_t* hs = g->h_src.as<int32_t>();
    if (dev_gb) std::memcpy(hs, ord.data(), sizeof(int32_t) * n);
    else
      for (int64_t k = 0; k < n; k++) hs[k] = g->new_of_old[(size_t)ord[(size_t)k]];
  }
  std::memcpy(g->h_outrow.p, row.data(), sizeof(int32_t) * n);
  GroupBufs* hgb = reinterpret_cast<GroupBufs*>(g->h_par.as<uint8_t>() + sizeof(Ctl) * rp.G);
  for (int i = 0; i < rp.G; i++) {
    GroupMem& m = g->groups[i];
    hgb[i].last = m.last.as<uint32_t>();
    hgb[i].curr = m.curr.as<uint32_t>();
    hgb[i].chg = m.chg.as<uint32_t>();
    hgb[i].qs = m.qs.as<int32_t>();
    hgb[i].qm = m.qm.as<int32_t>();
    hgb[i].ql = m.ql.as<int2>();
    hgb[i].hq = m.hq.as<int2>();
    hgb[i].ctl = m.ctl.as<Ctl>();
    hgb[i].planes = m.planes.as<uint32_t>();
  }
  Params p;
  fill_graph_params(g, o, rp.words, rp.threads, &p);
  if (!devloop) p.sparse_div = 0;
  p.src = g->d_src.as<int32_t>();
  p.out_row = g->d_outrow.as<int32_t>();
  p.n_total = n;
  p.C = rp.C;
  p.nbatches = rp.nbatches;
  p.G = rp.G;
  p.cpg = rp.cpg;
  p.db = db;
  p.layout = layout;
  p.groups = g->d_groups.as<GroupBufs>();
  p.brec = g->d_brec.as<BatchRec>();
  p.lrec = g->d_lrec.as<LevelRec>();
  p.lrec_cap = kLrecCap;
  set_output_params(g, rp.C, dout, &p);
  // Per-batch done flags of the device loop, in mapped host memory, grown in
  // powers of two so that their address (baked into cached graphs) stays put.
  if ((size_t)rp.nbatches > g->done_cap) {
    size_t cap = 64;
    while (cap < (size_t)rp.nbatches) cap <<= 1;
    if (g->h_done) cudaFreeHost(g->h_done);
    g->h_done = nullptr;
    g->d_done = nullptr;
    g->done_cap = 0;
    CU(cudaHostAlloc(reinterpret_cast<void**>(&g->h_done), cap * sizeof(int32_t),
                     cudaHostAllocMapped));
    CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&g->d_done), g->h_done, 0));
    g->done_cap = cap;
  }
  p.done_flags = g->d_done;
  // The depth sink: a finished batch's rows (or its vertex-major block) go
  // from `dout` to the caller's host buffer at the same byte offsets.
  const int32_t* rows_host = g->h_outrow.as<int32_t>();
  auto push_batch = [&](int b) -> cudaError_t {
    const int64_t n_b = std::min<int64_t>(rp.C, n - (int64_t)b * rp.C);
    const size_t rowb = (size_t)g->V * db;
    if (layout == IBFS_LAYOUT_VERTEX_MAJOR)
      return g->sink.push((size_t)b * rowb * rp.C, rowb * (size_t)n_b);
    for (int64_t j = 0; j < n_b; j++) {
      const cudaError_t e = g->sink.push((size_t)rows_host[(int64_t)b * rp.C + j] * rowb, rowb);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };

  int64_t launches = 0;
  const bool use_graph = persistent && o.use_graph && !o.debug_withhold;
  std::string key;
  bool replay = false;
  if (use_graph) {
    const void* extra[] = {g->h_src.p,  g->h_outrow.p, g->h_par.p,  g->d_src.p,
                           g->d_outrow.p, g->d_groups.p, g->d_brec.p, g->d_lrec.p,
                           g->d_out.p,  g->gbin.p,     g->gbkeys.p, g->gbhub.p};
    key = make_key(g, src, n, o, depth_out, layout, flags, rp, p, hgb, rp.G, extra,
                   (int)(sizeof(extra) / sizeof(extra[0])));
    replay = g->gcache.exec && g->gcache.key == key;
  }

  auto enqueue = [&](cudaStream_t cs, bool capturing) -> ibfs_status {
    {
      const ibfs_status us = upload_sources(cs);
      if (us != IBFS_OK) return us;
    }
    CU(cudaMemcpyAsync(g->d_groups.p, hgb, sizeof(GroupBufs) * rp.G, cudaMemcpyHostToDevice, cs));
    for (int i = 0; i < rp.G; i++) CU(cudaMemsetAsync(hgb[i].ctl, 0, sizeof(Ctl), cs));
    CU(cudaMemsetAsync(g->d_brec.p, 0, sizeof(BatchRec) * rp.nbatches, cs));
    // inside a capture a plain cudaEventRecord only orders work; an external
    // record becomes a real event-record node that replays time
    if (capturing) CU(cudaEventRecordWithFlags(g->ev0, cs, cudaEventRecordExternal));
    else CU(cudaEventRecord(g->ev0, cs));
    if (persistent) {
      cudaLaunchConfig_t cfg;
      std::memset(&cfg, 0, sizeof(cfg));
      cfg.gridDim = dim3((unsigned)rp.grid);
      cfg.blockDim = dim3((unsigned)rp.threads);
      cfg.dynamicSmemBytes = rp.smem;
      cfg.stream = cs;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeCooperative;
      attr[0].val.cooperative = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      void* args[] = {&p};
      CU(cudaLaunchKernelExC(&cfg, persistent_for(rp.words, occ_level), args));
      launches += 1;
    }
    if (capturing) CU(cudaEventRecordWithFlags(g->ev1, cs, cudaEventRecordExternal));
    else CU(cudaEventRecord(g->ev1, cs));
    if (rp.host_out) CU(cudaMemcpyAsync(depth_out, dout, out_bytes, cudaMemcpyDeviceToHost, cs));
    return IBFS_OK;
  };

  if (persistent) {
    if (use_graph) {
      if (!replay) {
        g->gcache.release();
        cudaGraph_t graph = nullptr;
        CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        ibfs_status es2 = enqueue(s, true);
        cudaGraph_t got = nullptr;
        cudaError_t ce = cudaStreamEndCapture(s, &got);
        graph = got;
        if (es2 != IBFS_OK) {
          if (graph) cudaGraphDestroy(graph);
          return es2;
        }
        if (ce != cudaSuccess) {
          last_cuda_error() = ce;
          if (graph) cudaGraphDestroy(graph);
          return IBFS_ERR_CUDA;
        }
        cudaGraphExec_t exec = nullptr;
        cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
          last_cuda_error() = ie;
          return IBFS_ERR_CUDA;
        }
        g->gcache.exec = exec;
        g->gcache.key = key;
      } else {
        launches = 1;
      }
      CU(cudaGraphLaunch(g->gcache.exec, s));
    } else {
      ibfs_status es2 = enqueue(s, false);
      if (es2 != IBFS_OK) return es2;
    }
  } else if (devloop) {
    // ---- device-driven schedule: one graph launch runs every level ------
    {
      const ibfs_status us = upload_sources(s);
      if (us != IBFS_OK) return us;
    }
    CU(cudaMemcpyAsync(g->d_groups.p, hgb, sizeof(GroupBufs) * rp.G, cudaMemcpyHostToDevice, s));
    Ctl* hctl = g->h_par.as<Ctl>();  // host staging of the G control blocks
    for (int i = 0; i < rp.G; i++) {
      std::memset(&hctl[i], 0, sizeof(Ctl));
      hctl[i].ls.n_total = n;
      hctl[i].ls.nbatches = rp.nbatches;
      CU(cudaMemcpyAsync(hgb[i].ctl, &hctl[i], sizeof(Ctl), cudaMemcpyHostToDevice, s));
    }
    CU(cudaMemsetAsync(g->d_brec.p, 0, sizeof(BatchRec) * rp.nbatches, s));
    // the graph bakes in the launch Params (device pointers, graph sizes,
    // options), the group count and the launch shapes: rebuild when any of
    // them moves.  The run's source and batch counts travel in the control
    // blocks instead, so runs of different sizes share one graph.
    Params pk = p;
    pk.n_total = 0;
    pk.nbatches = 0;
    std::string key(reinterpret_cast<const char*>(&pk), sizeof(pk));
    const int shape[4] = {rp.G, rp.threads, g->sms, rp.words};
    key.append(reinterpret_cast<const char*>(shape), sizeof(shape));
    GraphCache* slot = nullptr;
    for (auto& c : g->dlcache)
      if (c.exec && c.key == key) slot = &c;
    if (!slot) {
      slot = &g->dlcache[g->dl_next++ % ibfs_graph::kDlCache];
      slot->release();
      cudaGraph_t graph = nullptr;
      cudaError_t be = build_device_loop_graph(p, rp.words, rp.G, g->sms, rp.threads, &graph);
      if (be != cudaSuccess) {
        last_cuda_error() = be;
        (void)cudaGetLastError();
        return IBFS_ERR_CUDA;
      }
      cudaGraphExec_t exec = nullptr;
      cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) {
        last_cuda_error() = ie;
        (void)cudaGetLastError();
        return IBFS_ERR_CUDA;
      }
      slot->exec = exec;
      slot->key = key;
    }
    if (rp.host_out && dev_gb) {
      // the device GroupBy chose the rows: the sink needs them on the host
      CU(cudaMemcpyAsync(g->h_outrow.p, g->d_outrow.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost,
                         s));
      CU(cudaEventRecord(g->ev_out, s));
    }
    std::memset(g->h_done, 0, sizeof(int32_t) * (size_t)rp.nbatches);
    CU(cudaEventRecord(g->ev0, s));
    CU(cudaGraphLaunch(slot->exec, s));
    CU(cudaEventRecord(g->ev1, s));
    if (rp.host_out) {
      // Stream every batch out as soon as its done flag is up, while the
      // graph keeps traversing the others; batches whose flag never comes
      // stopped on an error, which the records report below.
      CU(g->sink.begin(g->device, depth_out, dout));
      if (dev_gb) CU(cudaEventSynchronize(g->ev_out));
      const volatile int32_t* fl = g->h_done;
      std::vector<char> taken((size_t)rp.nbatches, 0);
      int left = rp.nbatches;
      bool graph_done = false;
      while (left > 0) {
        bool any = false;
        for (int b = 0; b < rp.nbatches; b++) {
          if (taken[(size_t)b] || fl[b] == 0) continue;
          taken[(size_t)b] = 1;
          left--;
          any = true;
          CU(push_batch(b));
        }
        if (left == 0 || any) continue;
        if (graph_done) break;
        const cudaError_t q = cudaEventQuery(g->ev1);
        if (q == cudaSuccess) graph_done = true;  // one more scan, then stop
        else if (q == cudaErrorNotReady) std::this_thread::sleep_for(std::chrono::microseconds(20));
        else CU(q);
      }
      CU(g->sink.finish());
    }
  } else {
    // ---- plain schedule -------------------------------------------------
    {
      const ibfs_status us = upload_sources(s);
      if (us != IBFS_OK) return us;
    }
    CU(cudaMemcpyAsync(g->d_groups.p, hgb, sizeof(GroupBufs) * 1, cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(g->d_brec.p, 0, sizeof(BatchRec) * rp.nbatches, s));
    CU(cudaEventRecord(g->ev0, s));
    const GroupBufs gb = hgb[0];
    const int grid = g->sms, thr = rp.threads;  // launch helpers size each grid
    Par* hpar = reinterpret_cast<Par*>(g->h_par.p);
    BatchRec* hbr = g->h_brec.as<BatchRec>();
    LevelRec* hlr = g->h_lrec.as<LevelRec>();
    const size_t vpad = (size_t)((g->V + 31) & ~31LL);
    const size_t nchg = (size_t)(((g->V + 31) / 32 + 127) & ~127LL);
    if (rp.host_out) {
      CU(g->sink.begin(g->device, depth_out, dout));
      if (dev_gb) {
        CU(cudaMemcpyAsync(g->h_outrow.p, g->d_outrow.p, sizeof(int32_t) * n,
                           cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
      }
    }
    for (int b = 0; b < rp.nbatches; b++) {
      CU(cudaMemsetAsync(gb.last, 0, vpad * rp.words * 4, s));
      CU(cudaMemsetAsync(gb.curr, 0, vpad * rp.words * 4, s));
      CU(cudaMemsetAsync(gb.chg, 0, 2 * nchg * 4, s));
      CU(cudaMemsetAsync(gb.ctl, 0, sizeof(Ctl), s));
      CU(DISPATCH_WORDS(rp.words, launch_plain_seed, p, grid, thr, b, s));
      CU(DISPATCH_WORDS(rp.words, launch_plain_inspect, p, gb, grid, thr, b, 0, s));
      launches += 2;
      int level = 0, cur_dir = kDirTD, max_level = 0, td = 0, bu = 0, err = 0;
      unsigned long long m_u = (unsigned long long)g->E, teps = 0, prev_changed = 0;
      while (true) {
        CU(cudaMemcpyAsync(hpar, &gb.ctl->par[level & 1], sizeof(Par), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        const Par pr = *hpar;
        teps += pr.teps;
        m_u = m_u > pr.cdeg ? m_u - pr.cdeg : 0ull;
        int stop = 0;
        if (pr.range_err) { stop = 1; err = 3; }
        else if (pr.changed == 0) stop = 1;
        else if (level + 1 > p.max_levels) { stop = 1; err = 3; }
        if (pr.changed && !pr.range_err) max_level = level;
        const int nd = choose_dir(level + 1, cur_dir, p.switch_level, p.alpha, p.beta, pr.changed,
                                  prev_changed, pr.mf, m_u, p.V);
        prev_changed = pr.changed;
        if (level < kLrecCap) {
          LevelRec& r = hlr[(size_t)b * kLrecCap + level];
          r.batch = b; r.level = level; r.dir = level == 0 ? -1 : cur_dir; r.pad = 0;
          r.frontier = (long long)pr.changed; r.frontier_edges = (long long)pr.mf;
          r.expand_ns = r.inspect_ns = 0;
        }
        if (stop) break;
        cur_dir = nd;
        level++;
        if ((level & (level - 1)) == 0) {
          const int pb = __builtin_ctz((unsigned)level);
          CU(cudaMemsetAsync(gb.planes + (size_t)pb * p.plane_stride, 0,
                             (size_t)p.plane_stride * 4, s));
        }
        CU(cudaMemsetAsync(&gb.ctl->par[level & 1], 0, sizeof(Par), s));
        CU(cudaMemsetAsync(&gb.ctl->qc[level & 1][0], 0, sizeof(int32_t) * 4, s));
        CU(DISPATCH_WORDS(rp.words, launch_plain_level, p, gb, grid, thr, level, cur_dir, s));
        launches += 2;
        if (cur_dir == kDirTD) td++; else bu++;
        CU(DISPATCH_WORDS(rp.words, launch_plain_inspect, p, gb, grid, thr, b, level, s));
        launches += 1;
      }
      BatchRec& r = hbr[b];
      r.levels = level; r.max_level = max_level; r.td = td; r.bu = bu; r.teps = teps; r.err = err;
      if (err) {
        *range_hit = err == 3;
        if (rp.host_out) (void)g->sink.finish();  // no copy may outlive the call
        return (ibfs_status)err;
      }
      CU(DISPATCH_WORDS(rp.words, launch_plain_output, p, gb, grid, thr, b, max_level, s));
      launches += 1;
      if (rp.host_out) {
        // the batch's rows go out on the sink's stream behind its output pass
        CU(cudaEventRecord(g->ev_out, s));
        CU(g->sink.wait_for(g->ev_out));
        CU(push_batch(b));
      }
    }
    CU(cudaEventRecord(g->ev1, s));
    if (rp.host_out) CU(g->sink.finish());
  }
  CU(cudaStreamSynchronize(s));
  // collect results
  if (persistent || devloop) {
    CU(cudaMemcpyAsync(g->h_brec.p, g->d_brec.p, sizeof(BatchRec) * rp.nbatches,
                       cudaMemcpyDeviceToHost, s));
    if (st && st->levels && st->levels_cap > 0)
      CU(cudaMemcpyAsync(g->h_lrec.p, g->d_lrec.p, sizeof(LevelRec) * (size_t)rp.nbatches * kLrecCap,
                         cudaMemcpyDeviceToHost, s));
    int* herr = reinterpret_cast<int*>(g->h_par.p);  // the staged control blocks are done with
    for (int i = 0; i < rp.G; i++)
      CU(cudaMemcpyAsync(&herr[i], &hgb[i].ctl->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    int gerr = 0;
    for (int i = 0; i < rp.G; i++)
      if (herr[i] && !gerr) gerr = herr[i];
    if (gerr) {
      *range_hit = gerr == 3;
      return (ibfs_status)gerr;
    }
  }
  const BatchRec* br = g->h_brec.as<BatchRec>();
  if (st) {
    float ms = -1.0f;
    if (cudaEventElapsedTime(&ms, g->ev0, g->ev1) != cudaSuccess) {
      (void)cudaGetLastError();  // leave no stale error in the shared runtime
      ms = -1.0f;
    }
    st->n_sources = n;
    st->n_batches = rp.nbatches;
    st->depth_bytes = db;
    st->width = o.width;
    st->groups = rp.G;
    st->max_level = 0;
    st->levels_total = st->td_levels = st->bu_levels = 0;
    st->traversed_edges = 0;
    for (int b = 0; b < rp.nbatches; b++) {
      st->max_level = std::max(st->max_level, br[b].max_level);
      st->levels_total += br[b].levels;
      st->td_levels += br[b].td;
      st->bu_levels += br[b].bu;
      st->traversed_edges += (int64_t)br[b].teps;
    }
    if (devloop) {
      // kernel nodes that ran: start per group; per batch init, seed,
      // inspect(0), output, end and one decide for the final level; per
      // expanded level decide + two expand kernels + inspect, and on
      // bottom-up levels the sparse-source count, decision, push queue,
      // push chunks and bitmap clear
      launches = rp.G;
      const long long per_bu = p.sparse_div > 0 ? 9 : 4;
      for (int b = 0; b < rp.nbatches; b++)
        launches += 6 + 4LL * br[b].td + per_bu * br[b].bu;
    }
    st->gpu_launches = launches + gb_launches;
    st->device_ms = ms;
    st->levels_len = 0;
    if (st->levels && st->levels_cap > 0) {
      const LevelRec* lr = g->h_lrec.as<LevelRec>();
      int k = 0;
      for (int b = 0; b < rp.nbatches && k < st->levels_cap; b++)
        for (int l = 0; l <= std::min(br[b].levels + (persistent || devloop ? 1 : 0), kLrecCap - 1) &&
                        k < st->levels_cap; l++) {
          const LevelRec& r = lr[(size_t)b * kLrecCap + l];
          ibfs_level_rec& o2 = st->levels[k++];
          o2.batch = r.batch; o2.level = r.level; o2.dir = r.dir; o2.pad = 0;
          o2.frontier = r.frontier; o2.frontier_edges = r.frontier_edges;
          o2.expand_ns = r.expand_ns; o2.inspect_ns = r.inspect_ns;
        }
      st->levels_len = k;
    }
  }
  return IBFS_OK;
}

namespace ibfs {
// Launch the persistent kernel for an already filled Params (used by the
// static-scratch entry point in noalloc.cu; allocates nothing).
cudaError_t launch_persistent_params(const Params& p, int words, int grid, int threads,
                                     size_t smem, cudaStream_t s) {
  cudaLaunchConfig_t cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  Params q = p;
  void* args[] = {&q};
  return cudaLaunchKernelExC(&cfg, persistent_for(words), args);
}

cudaError_t persistent_occupancy(int words, int threads, size_t smem, int* per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, persistent_for(words), threads,
                                                       smem);
}
}  // namespace ibfs

namespace ibfs {
const int32_t* graph_host_col(const ibfs_graph* g) { return g->h.col.data(); }
}  // namespace ibfs

namespace ibfs {
// Run already-ordered sources whose depths go to explicit rows of a device
// array (source-major, V depths per row): the server's rounds.
ibfs_status run_rows(ibfs_graph* g, const int32_t* src, const int32_t* rows, int64_t n,
                     const ibfs_opts& o, void* dev_out, ibfs_stats* st) {
  if (!g || !src || !rows || n <= 0 || !dev_out) return IBFS_ERR_INVALID_ARG;
  ibfs_status s = check_opts(&o);
  if (s != IBFS_OK) return s;
  std::lock_guard<std::mutex> lk(g->mu);
  if (cudaSetDevice(g->device) != cudaSuccess) return IBFS_ERR_CUDA;
  bool range_hit = false;
  return run_once(g, src, n, o, o.depth_bytes ? o.depth_bytes : 1, dev_out,
                  IBFS_LAYOUT_SOURCE_MAJOR, IBFS_OUT_DEVICE, st, &range_hit, rows);
}
int graph_device(const ibfs_graph* g) { return g->device; }
const int64_t* graph_host_beg(const ibfs_graph* g) { return g->h.beg.data(); }
}  // namespace ibfs
