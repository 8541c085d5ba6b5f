// devloop.cu -- the device-loop schedule (IBFS_MODE_DEVICE_LOOP).
//
// One kernel per phase, as in the plain schedule, so that every phase runs
// with its own register budget and occupancy; the batch and level loops run
// on the device inside one CUDA graph through conditional nodes (WHILE over
// batches, WHILE over levels, SWITCH on the direction), so no level costs a
// host round trip and no phase waits at a grid barrier.
#include <cstring>

#include <cuda_runtime.h>

#include "bfs_device.cuh"
#include "internal.h"
#include "launch_common.cuh"

// CTAs per SM the compiler must fit (register budget) for the two hottest
// kernels; 0 leaves the budget to the compiler.  3 x 512 threads (at most
// 42 registers) measured best on R-MAT scale 24: 48 warps per SM keep more
// status gathers in flight than 2 x 512 at 64 registers, and 4 x 512 (32
// registers) spills more than it gains.
#ifndef IBFS_DL_BU_MINB
#define IBFS_DL_BU_MINB 3
#endif
// block size of the bottom-up kernel (the other phases run 512 threads)
#ifndef IBFS_DL_BU_THREADS
#define IBFS_DL_BU_THREADS 512
#endif
// Shared memory per bottom-up CTA for the hubs' statuses (bytes; 0: off):
// the first IBFS_BU_HUB_BYTES / (W/8) vertices of the degree order.  Off:
// with the L1 path of IBFS_BU_NC the hub words already hit L1 (R-MAT scale
// 24, one batch at a time, bottom-up per run: 19.4 ms L1 path, 20.0 ms with
// a 32 KB cache, 20.1 ms with both).
#ifndef IBFS_BU_HUB_BYTES
#define IBFS_BU_HUB_BYTES 0
#endif
#ifndef IBFS_DL_INSPECT_MINB
#define IBFS_DL_INSPECT_MINB 3
#endif
// CTAs per SM the top-down kernel must fit (0: left to the compiler)
#ifndef IBFS_DL_TD_MINB
#define IBFS_DL_TD_MINB 0
#endif
#if IBFS_DL_TD_MINB > 0
#define DL_TD_BOUNDS __launch_bounds__(512, IBFS_DL_TD_MINB)
#else
#define DL_TD_BOUNDS __launch_bounds__(512)
#endif
#if IBFS_DL_BU_MINB > 0
#define DL_BU_BOUNDS __launch_bounds__(IBFS_DL_BU_THREADS, IBFS_DL_BU_MINB)
#else
#define DL_BU_BOUNDS __launch_bounds__(IBFS_DL_BU_THREADS)
#endif
#if IBFS_DL_INSPECT_MINB > 0
#define DL_INSPECT_BOUNDS __launch_bounds__(512, IBFS_DL_INSPECT_MINB)
#else
#define DL_INSPECT_BOUNDS __launch_bounds__(512)
#endif

namespace ibfs {

// ---- device-driven schedule ------------------------------------------------
// The plain schedule's kernels inside one CUDA graph whose conditional nodes
// run the batch loop (WHILE) and the level loop (WHILE, with a SWITCH on the
// direction), so that every phase keeps the register budget and occupancy of
// its own kernel while no level needs a host round trip.  The batch and the
// level come from the group's LoopState; the decision kernel is the
// persistent kernel's top-of-level block (same rule, same records) run by one
// thread.  All kernels share one signature so that the graph builder can
// bind them uniformly: (params, group, handle 0, handle 1).
using CondH = cudaGraphConditionalHandle;

// The run's source and batch counts come from the control block, not from
// Params, so that one built graph serves runs of any size; the batch loop
// sets the size of every batch it starts (LoopState::nb).
__device__ __forceinline__ int dl_batch_size(const Params&, const LoopState& ls, int) {
  return ls.nb;
}

// Bottom-up levels run fused with their inspect work (bu_phase<.., true>):
// they write every vertex's new status into the buffer that is not `last`,
// and the decision kernel then swaps the two buffers' roles (LoopState::flip)
// instead of copying.  Every kernel sees the buffers through dl_bufs.
#ifndef IBFS_DL_FUSED_BU
#define IBFS_DL_FUSED_BU 1
#endif
__device__ __forceinline__ GroupBufs dl_bufs(const Params& p, int g) {
  GroupBufs gb = p.groups[g];
  if (gb.ctl->ls.flip) {
    uint32_t* x = gb.last;
    gb.last = gb.curr;
    gb.curr = x;
  }
  return gb;
}

// ---- serving queue ---------------------------------------------------------
__device__ __forceinline__ long long ld_acquire_sys_i64(const long long* p) {
  long long v;
  asm volatile("ld.acquire.sys.global.s64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Claim the next published batch of the serving queue (one thread).  Returns
// its slot, or -1 when no batch was published within q_wait_ns (the group
// then ends its batch loop; the host relaunches the graph for batches
// published after every group ended).  Both waits are bounded: the empty
// queue by q_wait_ns of %globaltimer, and lost compare-and-swaps (another
// group took that batch) by kClaimTries.  The short wait keeps a group that
// frees up between two publications alive instead of idle until the next
// launch.
constexpr int kClaimTries = 256;
__device__ int serve_claim(const Params& p) {
  const unsigned long long t0 = global_ns();
  int lost = 0;
  for (;;) {
    const long long t = ld_acquire_sys_i64(p.q_tail);
    const unsigned long long h = *reinterpret_cast<volatile unsigned long long*>(p.q_head);
    if ((long long)h >= t) {
      if (global_ns() - t0 >= p.q_wait_ns) return -1;
      __nanosleep(1000);
      continue;
    }
    if (atomicCAS(p.q_head, h, h + 1) == h) return (int)(h % (unsigned long long)p.q_slots);
    if (++lost >= kClaimTries) return -1;
  }
}

// Start the next batch of group g after `prev` (-1: the first).  Fixed runs
// take batches g, g + G, ...; the serving queue takes the next published
// slot and copies its sources and rows (host memory, read as volatile so
// that no stale cached copy of an earlier use of the slot is seen) into the
// device arrays that the phase kernels read.  Every thread of the block
// calls this; thread 0 decides.  Returns whether a batch was started.
__device__ bool dl_next_batch(const Params& p, Ctl* ctl, int g, int prev) {
  __shared__ int s_b, s_n;
  LoopState& ls = ctl->ls;
  if (threadIdx.x == 0) {
    int b = -1, nb = 0;
    if (p.q_slots > 0) {
      b = serve_claim(p);
      if (b >= 0) {
        nb = reinterpret_cast<const volatile int32_t*>(p.q_n)[b];
        reinterpret_cast<volatile int32_t*>(p.q_state)[b] = 1;
      }
    } else {
      b = prev < 0 ? g : prev + p.G;
      if (b < ls.nbatches) nb = (int)min((long long)p.C, ls.n_total - (long long)b * p.C);
      else b = -1;
    }
    s_b = b;
    s_n = nb;
  }
  __syncthreads();
  const int b = s_b, nb = s_n;
  if (b >= 0 && p.q_slots > 0) {
    const volatile int32_t* qs = p.q_src + (size_t)b * p.C;
    const volatile int32_t* qr = p.q_rows + (size_t)b * p.C;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
      const_cast<int32_t*>(p.src)[(size_t)b * p.C + j] = qs[j];
      const_cast<int32_t*>(p.out_row)[(size_t)b * p.C + j] = qr[j];
    }
  }
  if (threadIdx.x == 0 && b >= 0) {
    ls.batch = b;
    ls.nb = nb;
  }
  return b >= 0;
}

// Threads of the batch-loop kernels (k_dl_start, k_dl_batch_end): the
// serving queue copies a slot's sources and rows with them.
constexpr int kDlLoopThreads = 128;

// First batch of group g; the batch loop runs while it exists.
__global__ void k_dl_start(Params p, int g, CondH h_batch, CondH) {
  if (blockIdx.x != 0) return;
  Ctl* ctl = p.groups[g].ctl;
  if (threadIdx.x == 0) {
    ctl->ls.err = 0;
    ctl->ls.tail_clean = 0;  // the first batch of the launch zeroes everything
  }
  const bool go = dl_next_batch(p, ctl, g, -1);
  if (threadIdx.x == 0) cudaGraphSetConditional(h_batch, go ? 1u : 0u);
}

// Zero the group's status words and bitmaps, reset the counters and the
// loop state for the batch; arm the level loop.
template <int WORDS>
__global__ void __launch_bounds__(512) k_dl_batch_init(Params p, int g, CondH h_level, CondH) {
  const GroupBufs gb = p.groups[g];
  const Team t = make_team(blockIdx.x, gridDim.x);
  const long long vpad = (p.V + 31) & ~31LL;
  // after the group's first batch of a launch the statuses from v_reach on
  // are already zero (the previous batch cleared its sources' words there)
  const long long zv = (gb.ctl->ls.tail_clean && p.v_reach < p.V) ? p.v_reach : vpad;
  zero_words(gb.last, zv * WORDS, t);
  zero_words(gb.curr, zv * WORDS, t);
  zero_words(gb.chg, 2 * p.chg_stride, t);
  if (t.tid == 0) {
    Ctl* ctl = gb.ctl;
    memset(&ctl->par[0], 0, sizeof(Par) * 2);
    memset(&ctl->qc[0][0], 0, sizeof(ctl->qc));
    LoopState& ls = ctl->ls;
    ls.level = 0;
    ls.dir = kDirTD;
    ls.max_level = 0;
    ls.td = ls.bu = 0;
    ls.m_u = (unsigned long long)p.E;
    ls.teps = 0;
    ls.prev_changed = 0;
    ls.flip = 0;
    ls.sync = 0;
    for (int k = 0; k < kMaxWords; k++) ls.smask[k] = 0u;
    ls.sparse_try = 0;
    ls.t_lvl = ls.t_mid = global_ns();
    cudaGraphSetConditional(h_level, 1u);
  }
}

template <int WORDS>
__global__ void __launch_bounds__(512) k_dl_seed(Params p, int g, CondH, CondH) {
  const GroupBufs gb = dl_bufs(p, g);
  const int b = gb.ctl->ls.batch;
  seed_phase<WORDS>(p, gb, p.src + (long long)b * p.C, dl_batch_size(p, gb.ctl->ls, b),
                    make_team(blockIdx.x, gridDim.x));
}

template <int WORDS>
__global__ void DL_INSPECT_BOUNDS k_dl_inspect(Params p, int g, CondH, CondH) {
  const GroupBufs gb = dl_bufs(p, g);
  Ctl* ctl = gb.ctl;
  const int b = ctl->ls.batch, level = ctl->ls.level;
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->ls.t_mid = global_ns();
  inspect_phase<WORDS, false>(p, gb, &ctl->par[level & 1], dl_batch_size(p, ctl->ls, b), level,
                              level <= depth_limit(p.db), false, make_team(blockIdx.x, gridDim.x));
}

// Top of a level: read the counters of the level just inspected, stop or
// pick the next direction (choose_dir), write the level record, advance.
// h_level keeps the level loop running, h_dir selects the expand body
// (0 top-down, 1 bottom-up, 2 none: the loop ends).
__global__ void k_dl_decide(Params p, int g, CondH h_level, CondH h_dir) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Ctl* ctl = p.groups[g].ctl;
  LoopState& ls = ctl->ls;
  const int level = ls.level, b = ls.batch;
  // a fused bottom-up level left its statuses in the other buffer
  const bool was_bu = IBFS_DL_FUSED_BU && level > 0 && ls.dir == kDirBU;
  if (was_bu) ls.flip ^= 1;
  const Par& pr = ctl->par[level & 1];
  const unsigned long long changed = pr.changed, mf = pr.mf, cdeg = pr.cdeg;
  ls.teps += pr.teps;
  ls.m_u = ls.m_u > cdeg ? ls.m_u - cdeg : 0ull;
  int stop = 0, err = 0;
  if (pr.range_err) { stop = 1; err = 3; }
  else if (changed == 0) stop = 1;
  else if (level + 1 > p.max_levels) { stop = 1; err = 3; }
  if (changed && !pr.range_err) ls.max_level = level;
  const int nd = choose_dir(level + 1, ls.dir, p.switch_level, p.alpha, p.beta, changed,
                            ls.prev_changed, mf, ls.m_u, p.V);
  ls.prev_changed = changed;
  // A bottom-up level right after a top-down one looks for sparse sources
  // (k_dl_sparse_count / k_dl_sparse_decide fill smask before its pass)
#pragma unroll
  for (int k = 0; k < kMaxWords; k++) ls.smask[k] = 0u;
  ls.sparse_try = (!stop && nd == kDirBU && ls.dir == kDirTD && level > 0 && p.sparse_div > 0) ? 1 : 0;
  const unsigned long long t_now = global_ns();
  if (level < p.lrec_cap) {
    LevelRec r;
    r.batch = b; r.level = level; r.dir = level == 0 ? -1 : ls.dir; r.pad = 0;
    r.frontier = (long long)changed; r.frontier_edges = (long long)mf;
    r.expand_ns = (long long)(ls.t_mid - ls.t_lvl);
    r.inspect_ns = (long long)(t_now - ls.t_mid);
    p.lrec[(size_t)b * p.lrec_cap + level] = r;
  }
  ls.t_lvl = t_now;
  ls.err = err;
  if (!stop) {
    memset((void*)&ctl->par[(level + 1) & 1], 0, sizeof(Par));
    ctl->qc[level & 1][0] = ctl->qc[level & 1][1] = ctl->qc[level & 1][2] = 0;
    ls.sync = (was_bu && nd == kDirTD) ? 1 : 0;  // top-down needs curr == last again
    ls.dir = nd;
    ls.level = level + 1;
    if (nd == kDirTD) ls.td++; else ls.bu++;
  }
  cudaGraphSetConditional(h_level, stop ? 0u : 1u);
  cudaGraphSetConditional(h_dir, stop ? 2u : (unsigned)nd);
}

template <int WORDS>
__global__ void __launch_bounds__(512) k_dl_qbuild(Params p, int g, CondH, CondH) {
  const GroupBufs gb = dl_bufs(p, g);
  const int level = gb.ctl->ls.level;
  const Team t = make_team(blockIdx.x, gridDim.x);
  zero_plane_if_first(p, gb, level, t);
  qbuild_phase<WORDS>(p, gb, level, gb.ctl->qc[level & 1], t, gb.ctl->ls.sync != 0);
}

template <int WORDS>
__global__ void DL_TD_BOUNDS k_dl_td(Params p, int g, CondH, CondH) {
  const GroupBufs gb = dl_bufs(p, g);
  const int level = gb.ctl->ls.level;
  td_phase<WORDS, true>(p, gb, level, gb.ctl->qc[level & 1],
                                      make_team(blockIdx.x, gridDim.x));
}

template <int WORDS>
__global__ void DL_BU_BOUNDS k_dl_bu(Params p, int g, CondH, CondH) {
  const GroupBufs gb = dl_bufs(p, g);
  const LoopState& ls = gb.ctl->ls;
  const int level = ls.level;
  const Team t = make_team(blockIdx.x, gridDim.x);
  const bool filt = bu_filter_level(p.bu_filter, gb.ctl->par[(level - 1) & 1].changed, p.V);
  if (IBFS_DL_FUSED_BU) {
    bu_phase<WORDS, true, true, IBFS_BU_HUB_BYTES / (4 * WORDS)>(p, gb, level, gb.ctl->par[(level - 1) & 1].fmask,
                          &gb.ctl->par[level & 1].hq_cnt, t, &gb.ctl->par[level & 1],
                          dl_batch_size(p, ls, ls.batch), level <= depth_limit(p.db), filt,
                          ls.smask);
  } else {
    zero_plane_if_first(p, gb, level, t);
    bu_phase<WORDS, false, true>(p, gb, level, gb.ctl->par[(level - 1) & 1].fmask,
                                 &gb.ctl->par[level & 1].hq_cnt, t, nullptr, 0, true, filt);
  }
}

// The inspect step of a fused bottom-up level: deferred hubs only.
template <int WORDS>
__global__ void __launch_bounds__(512) k_dl_bu_hubs(Params p, int g, CondH, CondH) {
  const GroupBufs gb = dl_bufs(p, g);
  Ctl* ctl = gb.ctl;
  const int b = ctl->ls.batch, level = ctl->ls.level;
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->ls.t_mid = global_ns();
  const bool sparse = dl_sparse(ctl->ls, WORDS);
  bu_hub_epilogue<WORDS>(p, gb, &ctl->par[level & 1], dl_batch_size(p, ctl->ls, b), level,
                         level <= depth_limit(p.db), make_team(blockIdx.x, gridDim.x), sparse);
}

template <int WORDS>
__global__ void __launch_bounds__(512) k_dl_bu_defer(Params p, int g, CondH, CondH) {
  const GroupBufs gb = dl_bufs(p, g);
  const int level = gb.ctl->ls.level;
  if (gb.ctl->par[level & 1].hq_cnt == 0) return;  // uniform: nothing deferred
  bu_defer_phase<WORDS, true>(p, gb, level, gb.ctl->par[(level - 1) & 1].fmask,
                              &gb.ctl->par[level & 1].hq_cnt, make_team(blockIdx.x, gridDim.x),
                              bu_filter_level(p.bu_filter, gb.ctl->par[(level - 1) & 1].changed,
                                              p.V),
                              gb.ctl->ls.smask);
}

// Sparse sources of a bottom-up level that follows a top-down one: count
// every source's previous frontier, then pick the sparse ones (one thread).
template <int WORDS>
__global__ void __launch_bounds__(512) k_dl_sparse_count(Params p, int g, CondH, CondH) {
  const GroupBufs gb = dl_bufs(p, g);
  Ctl* ctl = gb.ctl;
  if (!ctl->ls.sparse_try) return;  // uniform
  const int level = ctl->ls.level;
  sparse_count_phase<WORDS>(p, gb, &ctl->par[level & 1], level, make_team(blockIdx.x, gridDim.x));
}

__global__ void k_dl_sparse_decide(Params p, int g, CondH, CondH) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Ctl* ctl = p.groups[g].ctl;
  LoopState& ls = ctl->ls;
  if (!ls.sparse_try) return;
  const Par& pr = ctl->par[ls.level & 1];
  const int nsrc = ls.nb;
  unsigned long long tot = 0;
  for (int i = 0; i < nsrc; i++) tot += pr.scnt[i];
  uint32_t sm[kMaxWords];
#pragma unroll
  for (int k = 0; k < kMaxWords; k++) sm[k] = 0u;
  for (int i = 0; i < nsrc; i++) {
    const unsigned long long c = pr.scnt[i];
    if (c > 0 && c * (unsigned long long)p.sparse_div * (unsigned long long)nsrc < tot)
      sm[i >> 5] |= 1u << (i & 31);
  }
#pragma unroll
  for (int k = 0; k < kMaxWords; k++) ls.smask[k] = sm[k];
}

__device__ __forceinline__ bool dl_sparse(const LoopState& ls, int words) {
  bool any = false;
  for (int k = 0; k < words; k++) any |= ls.smask[k] != 0u;
  return any;
}

// After the bottom-up pass, its deferred hubs and their inspect work: the
// sparse sources' bits, top-down (small pushers by warps, large ones queued
// in chunks), then the chunks over all CTAs.
template <int WORDS>
__global__ void __launch_bounds__(512) k_dl_push_queue(Params p, int g, CondH, CondH) {
  const GroupBufs gb = dl_bufs(p, g);
  Ctl* ctl = gb.ctl;
  const LoopState& ls = ctl->ls;
  if (!dl_sparse(ls, WORDS)) return;  // uniform
  const int level = ls.level;
  push_queue_phase<WORDS>(p, gb, &ctl->par[level & 1], dl_batch_size(p, ls, ls.batch), level,
                          level <= depth_limit(p.db), ls.smask,
                          make_team(blockIdx.x, gridDim.x));
}

template <int WORDS>
__global__ void __launch_bounds__(512) k_dl_push_run(Params p, int g, CondH, CondH) {
  const GroupBufs gb = dl_bufs(p, g);
  Ctl* ctl = gb.ctl;
  const LoopState& ls = ctl->ls;
  if (!dl_sparse(ls, WORDS)) return;  // uniform
  const int level = ls.level;
  if (ctl->par[level & 1].pq_cnt == 0) return;  // uniform
  push_run_phase<WORDS>(p, gb, &ctl->par[level & 1], dl_batch_size(p, ls, ls.batch), level,
                        level <= depth_limit(p.db), ls.smask, make_team(blockIdx.x, gridDim.x));
}

// After the push: clear the level+1 bitmap that the hub epilogue left
// (it was the push's frontier); the next bottom-up pass ORs into it.
template <int WORDS>
__global__ void __launch_bounds__(512) k_dl_clear_next(Params p, int g, CondH, CondH) {
  const GroupBufs gb = dl_bufs(p, g);
  const LoopState& ls = gb.ctl->ls;
  if (!dl_sparse(ls, WORDS)) return;  // uniform: the hub epilogue cleared it
  zero_words(chg_at(gb, p, ls.level + 1), p.chg_stride, make_team(blockIdx.x, gridDim.x));
}

// threads per CTA and CTAs per SM of the output pass (R-MAT scale 24, one
// batch at a time, output per 1024-source run: 512 x 1 10.6 ms, 512 x 2
// (64 registers, spills) 15.9 ms, 256 x 3 17.0 ms)
#ifndef IBFS_DL_OUT_THREADS
#define IBFS_DL_OUT_THREADS 512
#endif
#ifndef IBFS_DL_OUT_MINB
#define IBFS_DL_OUT_MINB 1
#endif
template <int WORDS>
__global__ void __launch_bounds__(IBFS_DL_OUT_THREADS, IBFS_DL_OUT_MINB) k_dl_output(Params p, int g, CondH, CondH) {
  __shared__ int32_t s_rows[kMaxWords * 32];
  const GroupBufs gb = dl_bufs(p, g);
  const LoopState& ls = gb.ctl->ls;
  if (ls.err) return;  // uniform
  const int b = ls.batch, n_b = dl_batch_size(p, ls, b);
  load_rows(p, b, n_b, s_rows);
  output_phase<WORDS>(p, gb, batch_depth(p, b), s_rows, n_b, ls.max_level,
                      make_team(blockIdx.x, gridDim.x));
}

// The records of a batch that finished without error (one thread).
__device__ void dl_batch_record(const Params& p, LoopState& ls, int b) {
  if (ls.level + 1 < p.lrec_cap) {
    LevelRec r;  // dir 2: the batch's output pass
    r.batch = b; r.level = ls.level + 1; r.dir = 2; r.pad = 0;
    r.frontier = 0; r.frontier_edges = 0;
    r.expand_ns = (long long)(global_ns() - ls.t_lvl);
    r.inspect_ns = 0;
    p.lrec[(size_t)b * p.lrec_cap + ls.level + 1] = r;
  }
  BatchRec r;
  r.levels = ls.level;
  r.max_level = ls.max_level;
  r.td = ls.td;
  r.bu = ls.bu;
  r.teps = ls.teps;
  r.err = 0;
  r.pad = 0;
  p.brec[b] = r;
  if (p.done_flags) {
    // the output kernel of batch b has finished (graph edge): tell the host,
    // whose depth sink starts copying the batch's rows out
    __threadfence_system();
    *reinterpret_cast<volatile int32_t*>(p.done_flags + b) = 1;
  }
  if (p.q_slots > 0) {
    // serving: the slot's depths are in their rows and its record (host
    // memory) is written before the state says so
    __threadfence_system();
    reinterpret_cast<volatile int32_t*>(p.q_state)[b] = 2;
  }
}

// End of a batch: its record (or the group's error), then the next batch of
// the group; the batch loop ends after the last one or on an error (in the
// serving queue: when no published batch is left; an error there is the
// batch's own and goes into its record).
__global__ void k_dl_batch_end(Params p, int g, CondH h_batch, CondH) {
  if (blockIdx.x != 0) return;
  Ctl* ctl = p.groups[g].ctl;
  LoopState& ls = ctl->ls;
  const int b = ls.batch;
  // the batch's sources from v_reach on were the only nonzero status words
  // there: clear them for the group's next batch
  if (p.v_reach < p.V) {
    const GroupBufs& gb = p.groups[g];
    const long long words = p.plane_stride / ((p.V + 31) & ~31LL);  // status words per vertex
    for (int j = threadIdx.x; j < ls.nb; j += blockDim.x) {
      const int32_t v = p.src[(size_t)b * p.C + j];
      if (v < p.v_reach) continue;
      for (long long k = 0; k < words; k++) {
        gb.last[(size_t)v * words + k] = 0u;
        gb.curr[(size_t)v * words + k] = 0u;
      }
    }
  }
  __shared__ int s_stop;
  __syncthreads();
  if (threadIdx.x == 0) {
    ls.tail_clean = 1;
    s_stop = 0;
    if (ls.err && p.q_slots > 0) {
      // serving: the error belongs to this batch's queries alone; report it
      // in the slot's record and go on with the next batch
      BatchRec r;
      memset(&r, 0, sizeof(r));
      r.err = ls.err;
      p.brec[b] = r;
      __threadfence_system();
      reinterpret_cast<volatile int32_t*>(p.q_state)[b] = 2;
      ls.err = 0;
    } else if (ls.err) {
      atomicCAS(&ctl->err, 0, ls.err);
      p.brec[b].err = ls.err;
      cudaGraphSetConditional(h_batch, 0u);
      s_stop = 1;
    } else {
      dl_batch_record(p, ls, b);
    }
  }
  __syncthreads();
  if (s_stop) return;
  const bool go = dl_next_batch(p, ctl, g, b);
  if (threadIdx.x == 0) cudaGraphSetConditional(h_batch, go ? 1u : 0u);
}

// ---- device-driven schedule: graph construction ------------------------
using DlKernel = void (*)(Params, int, CondH, CondH);

static cudaError_t dl_kernel(cudaGraph_t gr, cudaGraphNode_t* out, cudaGraphNode_t dep,
                             DlKernel fn, int grid, int threads, const Params& p, int g,
                             CondH h0, CondH h1) {
  Params pp = p;
  int gg = g;
  CondH a = h0, b = h1;
  void* args[] = {&pp, &gg, &a, &b};
  cudaKernelNodeParams kp;
  std::memset(&kp, 0, sizeof(kp));
  kp.func = reinterpret_cast<void*>(fn);
  kp.gridDim = dim3((unsigned)grid);
  kp.blockDim = dim3((unsigned)threads);
  kp.kernelParams = args;
  return cudaGraphAddKernelNode(out, gr, dep ? &dep : nullptr, dep ? 1 : 0, &kp);
}

static cudaError_t dl_cond(cudaGraph_t gr, cudaGraphNode_t* out, cudaGraphNode_t dep, CondH h,
                           cudaGraphConditionalNodeType type, unsigned size, cudaGraph_t* bodies) {
  cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
  np.conditional.handle = h;
  np.conditional.type = type;
  np.conditional.size = size;
  cudaError_t e = cudaGraphAddNode(out, gr, dep ? &dep : nullptr, dep ? 1 : 0, &np);
  if (e == cudaSuccess)
    for (unsigned i = 0; i < size; i++) bodies[i] = np.conditional.phGraph_out[i];
  return e;
}

// One branch per group g:
//   start -> WHILE(batch) { init -> seed -> inspect(0) -> WHILE(level) {
//              decide -> SWITCH(dir) { 0: qbuild -> td -> inspect,
//                                      1: bu -> bu_defer -> inspect } }
//            -> output -> batch_end }
// Every loop ends: decide stops at an empty level or past max_levels, and
// batch_end stops after the group's last batch or on an error.
template <int WORDS>
static cudaError_t build_device_loop(const Params& p, int G, int sms, int threads,
                                     cudaGraph_t* out) {
  *out = nullptr;
  cudaGraph_t top = nullptr;
  cudaError_t e = cudaGraphCreate(&top, 0);
  if (e != cudaSuccess) return e;
  const int gz = occ_grid((const void*)k_dl_batch_init<WORDS>, threads, sms);
  const int gi = occ_grid((const void*)k_dl_inspect<WORDS>, threads, sms);
  const int gq = occ_grid((const void*)k_dl_qbuild<WORDS>, threads, sms);
  const int gh = occ_grid((const void*)k_dl_bu_hubs<WORDS>, threads, sms);
  const int gt = occ_grid((const void*)k_dl_td<WORDS>, threads, sms);
  const int gu = occ_grid((const void*)k_dl_bu<WORDS>, IBFS_DL_BU_THREADS, sms);
  const int gd = occ_grid((const void*)k_dl_bu_defer<WORDS>, threads, sms);
  const int go = occ_grid((const void*)k_dl_output<WORDS>, IBFS_DL_OUT_THREADS, sms);
  const int gpq = occ_grid((const void*)k_dl_push_queue<WORDS>, threads, sms);
  const int gpr = occ_grid((const void*)k_dl_push_run<WORDS>, threads, sms);
  const int gsc = occ_grid((const void*)k_dl_sparse_count<WORDS>, threads, sms);
#define DL_TRY(call)                   \
  do {                                 \
    e = (call);                        \
    if (e != cudaSuccess) {            \
      cudaGraphDestroy(top);           \
      return e;                        \
    }                                  \
  } while (0)
  for (int g = 0; g < G; g++) {
    CondH hb = 0, hl = 0, hd = 0;
    DL_TRY(cudaGraphConditionalHandleCreate(&hb, top, 0, cudaGraphCondAssignDefault));
    cudaGraphNode_t n0, n1;
    DL_TRY(dl_kernel(top, &n0, nullptr, k_dl_start, 1, kDlLoopThreads, p, g, hb, 0));
    cudaGraph_t B = nullptr;
    DL_TRY(dl_cond(top, &n1, n0, hb, cudaGraphCondTypeWhile, 1, &B));
    DL_TRY(cudaGraphConditionalHandleCreate(&hl, B, 0, cudaGraphCondAssignDefault));
    cudaGraphNode_t b0, b1, b2, b3, b4, b5;
    DL_TRY(dl_kernel(B, &b0, nullptr, k_dl_batch_init<WORDS>, gz, threads, p, g, hl, 0));
    DL_TRY(dl_kernel(B, &b1, b0, k_dl_seed<WORDS>, 1, 512, p, g, 0, 0));
    DL_TRY(dl_kernel(B, &b2, b1, k_dl_inspect<WORDS>, gi, threads, p, g, 0, 0));
    cudaGraph_t L = nullptr;
    DL_TRY(dl_cond(B, &b3, b2, hl, cudaGraphCondTypeWhile, 1, &L));
    DL_TRY(dl_kernel(B, &b4, b3, k_dl_output<WORDS>, go, IBFS_DL_OUT_THREADS, p, g, 0, 0));
    DL_TRY(dl_kernel(B, &b5, b4, k_dl_batch_end, 1, kDlLoopThreads, p, g, hb, 0));
    DL_TRY(cudaGraphConditionalHandleCreate(&hd, L, 2, cudaGraphCondAssignDefault));
    cudaGraphNode_t l0, l1;
    DL_TRY(dl_kernel(L, &l0, nullptr, k_dl_decide, 1, 32, p, g, hl, hd));
    cudaGraph_t S[2] = {nullptr, nullptr};
    DL_TRY(dl_cond(L, &l1, l0, hd, cudaGraphCondTypeSwitch, 2, S));
    cudaGraphNode_t t0, t1, t2, u0, u1, u2, u3, u4;
    DL_TRY(dl_kernel(S[0], &t0, nullptr, k_dl_qbuild<WORDS>, gq, threads, p, g, 0, 0));
    DL_TRY(dl_kernel(S[0], &t1, t0, k_dl_td<WORDS>, gt, threads, p, g, 0, 0));
    DL_TRY(dl_kernel(S[0], &t2, t1, k_dl_inspect<WORDS>, gi, threads, p, g, 0, 0));
    cudaGraphNode_t bu_dep = nullptr;
    if (IBFS_DL_FUSED_BU && p.sparse_div > 0) {
      cudaGraphNode_t s0, s1;
      DL_TRY(dl_kernel(S[1], &s0, nullptr, k_dl_sparse_count<WORDS>, gsc, threads, p, g, 0, 0));
      DL_TRY(dl_kernel(S[1], &s1, s0, k_dl_sparse_decide, 1, 32, p, g, 0, 0));
      bu_dep = s1;
    }
    DL_TRY(dl_kernel(S[1], &u0, bu_dep, k_dl_bu<WORDS>, gu, IBFS_DL_BU_THREADS, p, g, 0, 0));
    DL_TRY(dl_kernel(S[1], &u1, u0, k_dl_bu_defer<WORDS>, gd, threads, p, g, 0, 0));
    if (IBFS_DL_FUSED_BU) {
      DL_TRY(dl_kernel(S[1], &u2, u1, k_dl_bu_hubs<WORDS>, gh, threads, p, g, 0, 0));
      if (p.sparse_div > 0) {
        cudaGraphNode_t u5;
        DL_TRY(dl_kernel(S[1], &u3, u2, k_dl_push_queue<WORDS>, gpq, threads, p, g, 0, 0));
        DL_TRY(dl_kernel(S[1], &u4, u3, k_dl_push_run<WORDS>, gpr, threads, p, g, 0, 0));
        DL_TRY(dl_kernel(S[1], &u5, u4, k_dl_clear_next<WORDS>, gz, threads, p, g, 0, 0));
      }
    } else {
      DL_TRY(dl_kernel(S[1], &u2, u1, k_dl_inspect<WORDS>, gi, threads, p, g, 0, 0));
    }
  }
#undef DL_TRY
  *out = top;
  return cudaSuccess;
}

cudaError_t build_device_loop_graph(const Params& p, int words, int G, int sms, int threads,
                                    cudaGraph_t* out) {
  return DISPATCH_WORDS(words, build_device_loop, p, G, sms, threads, out);
}

}  // namespace ibfs
