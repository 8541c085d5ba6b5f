// bfs_device.cuh -- device side of the concurrent multi-source BFS.
//
// One batch = up to W sources (W = 32*WORDS status bits per vertex).  Per
// vertex v the status word holds bit s when source s has reached v.  Two
// copies are kept: `last` (status after the previous level) and `curr` (the
// status being built); after every level the vertices whose word changed
// are fixed up (last = curr) so that curr == last holds for every vertex at
// the start of a level.  Reference: comp_t status words and
// depth_comp_last/curr (comm.h:44, allocator.cuh:51-52).
//
// A level is three phases, separated by barriers (grid barriers inside the
// persistent kernel, kernel boundaries in the plain schedule):
//   expand   top-down push over the joint frontier queues (expander.cuh:
//            140-331) or bottom-up pull over all vertices (expander.cuh:
//            341-489); both mark changed vertices in a 1-bit-per-vertex
//            bitmap (V/8 bytes, L2 resident), double-buffered by level parity
//            so that the bottom-up pull can skip neighbours outside the
//            previous frontier;
//   inspect  walks the bitmap only: new bits = curr & ~last, last = curr,
//            ORs the new bits into the depth bit-planes of the level number,
//            and accumulates the direction-switch counters.  Replaces the
//            O(V) count/scan/gather passes of inspector.cuh:63-525,
//            scan.cuh:455-655 and the per-level depth_merge writes of
//            inspector.cuh:8-56,113-120;
//   qbuild   (only before a top-down level) turns the bitmap into the
//            small/medium/large queues with warp-ballot compaction
//            (replaces td_frontier_count/td_frontier_gather).
// After the last level one pass turns the bit-planes into the depth output
// (either layout), writing every output byte exactly once.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ibfs {

constexpr int kDirTD = 0;
constexpr int kDirBU = 1;
constexpr int kMaxWords = 8;   // W = 256
constexpr int kMaxPlanes = 16; // two-byte depths

// Per-level counters, double-buffered by level parity.
struct Par {
  unsigned long long changed;  // vertices whose status changed
  unsigned long long mf;       // sum of their degrees (frontier edges)
  unsigned long long cdeg;     // sum of degrees of vertices that became complete
  unsigned long long teps;     // sum over new (v, s) pairs of deg(v)
  uint32_t fmask[kMaxWords];   // OR of all new bits (sources still expanding)
  int32_t range_err;           // a level did not fit the depth type
  int32_t hq_cnt;              // deferred bottom-up hub chunks of this level
  int32_t pq_cnt;              // queued sparse-source push chunks of this level
  int32_t pad;
  uint32_t scnt[kMaxWords * 32];  // per source: vertices it reached at the
                                  // previous level (sparse_count_phase)
};

// State of the level loop when it runs as kernels inside a CUDA graph (the
// device-driven schedule): what the persistent kernel keeps in registers
// lives here between kernels.
struct LoopState {
  long long n_total;  // sources of the run (set by the host before the launch)
  int32_t nbatches;   // batches of the run (set by the host before the launch)
  int32_t batch;      // batch the group is traversing
  int32_t level;      // level being expanded / inspected
  int32_t dir;        // direction of `level`
  int32_t max_level;
  int32_t td, bu;
  int32_t err;
  int32_t flip;       // 1: the status "last" lives in GroupBufs::curr and vice versa
  int32_t sync;       // the next top-down level first copies new statuses over old ones
  int32_t nb;         // sources of `batch`
  uint32_t smask[kMaxWords];  // bottom-up level: sources pushed top-down instead
  int32_t tail_clean;         // both status buffers are zero from v_reach on
                              // (batch_end clears its unreachable sources' words)
  int32_t sparse_try;         // this bottom-up level follows a top-down one: count
                              // the sources' frontiers and pick the sparse ones
  unsigned long long m_u, teps, prev_changed;
  unsigned long long t_lvl, t_mid;  // %globaltimer at the level start / inspect start
};

// Control block of one group (one batch at a time).  256-byte aligned.
struct __align__(256) Ctl {
  unsigned int bar_count;
  unsigned int bar_gen;
  int err;
  int pad0;
  Par par[2];
  int32_t qc[2][4];  // [consumer level parity][small, medium, large-chunks]
  unsigned long long pad1[4];
  LoopState ls;
};

struct BatchRec {
  int32_t levels;     // levels expanded (incl. the last empty one)
  int32_t max_level;  // deepest level with a new vertex
  int32_t td, bu;
  unsigned long long teps;
  int32_t err;
  int32_t pad;
};

struct LevelRec {
  int32_t batch, level, dir, pad;
  long long frontier, frontier_edges;
  long long expand_ns, inspect_ns;  // device time of the level's phases (persistent)
};

struct GroupBufs {
  uint32_t* last;    // [Vpad][WORDS]
  uint32_t* curr;    // [Vpad][WORDS]
  uint32_t* chg;     // 2 bitmaps of chg_stride words (level parity)
  uint32_t* planes;  // depth bit-planes, plane b at b*plane_stride words
  int32_t* qs;
  int32_t* qm;
  int2* ql;
  int2* hq;          // deferred bottom-up hub chunks (v, chunk)
  Ctl* ctl;
};

struct Params {
  const int64_t* beg;
  const int32_t* col;
  int64_t V, E, nchg;
  long long chg_stride;    // words per bitmap (nchg rounded up to 4)
  long long plane_stride;  // words per bit-plane (Vpad * WORDS)
  const int32_t* src;      // ordered sources [n_total]
  const int32_t* out_row;  // output row of ordered source k (source-major)
  int64_t n_total;
  int C, nbatches, G, cpg;
  int db;                  // depth bytes
  int layout;              // 0 source-major, 1 vertex-major
  uint8_t* out;            // device output
  int sml, lrg, chunk, but;
  int switch_level;
  float alpha, beta;
  int max_levels;
  unsigned long long timeout_ns;
  int withhold;
  GroupBufs* groups;
  BatchRec* brec;
  LevelRec* lrec;
  int lrec_cap;
  int vec_out;  // vertex-major rows allow 4-byte stores (n_b*db % 4 == 0, aligned base)
  int vec_sm;   // source-major rows allow vector stores of this many bytes: 16 (V % 16
                // == 0, 16-byte aligned base), 4 (V % 4 == 0, 4-byte aligned) or 0
  int td_stage;     // top-down stages large vertices' chunks by bulk copies
  int sparse_div;   // device loop: a bottom-up level pushes, top-down, the sources
                    // whose previous frontier is below 1/sparse_div of the average
                    // (0: off; see sparse_count_phase)
  int bu_filter;    // bottom-up skips neighbours outside the previous frontier:
                    // 1 always, 0 never, -1 on levels whose previous frontier
                    // is small (bu_filter_level)
  int col_vec;      // col is 16-byte aligned and padded by 4 entries (vector reads)
  int hub_t;        // bottom-up: a warp scans at most hub_t neighbours of a vertex;
                    // a hub still missing bits defers the rest in chunks
  const int32_t* vmap;  // caller id -> internal id of the resident graph (null:
                        // identical); the output pass reads statuses through it
  long long v_nz;       // bottom-up sweeps [0, v_nz): in the degree order the
                        // vertices from v_nz on have no edges (v_nz a multiple
                        // of 32, or V); a bottom-up pass cannot change them and
                        // a top-down level (a directed graph's sinks) writes
                        // both status buffers through inspect, so they agree
  long long v_reach;    // v_nz when no edge points into [v_nz, V) (symmetric
                        // graphs), else V: vertices from v_reach on are reached
                        // only as sources, at depth 0
  long long big_prefix; // bottom-up: vertices [0, big_prefix) take one warp each
                        // (degree-ordered graphs: the vertices above the
                        // thread-path limit; a multiple of 32; 0 otherwise)
  int32_t* done_flags;  // per batch, in mapped host memory: 1 once the batch's
                        // depths are complete in `out` (device loop), so that
                        // the host can stream them out while later batches run
  // Serving queue (device loop, q_slots > 0): batches are not a fixed list
  // but slots of a ring that the host fills while the graph runs.  The host
  // writes a slot's sources (internal ids), output rows and count, then
  // raises q_tail; a group that finishes a batch claims the next published
  // one (q_head, compare-and-swap), copies the slot into src/out_row (device
  // arrays of q_slots * C entries) and marks it 1 in q_state; after its
  // output pass it writes brec[slot] and marks it 2.  A group that finds no
  // published batch ends its batch loop; the host relaunches the graph for
  // batches published after every group ended.
  int q_slots;
  const long long* q_tail;      // mapped host memory: batches published
  const int32_t* q_n;           // mapped host memory [q_slots]: sources per slot
  const int32_t* q_src;         // mapped host memory [q_slots * C]
  const int32_t* q_rows;        // mapped host memory [q_slots * C]
  int32_t* q_state;             // mapped host memory [q_slots]: 1 claimed, 2 done
  unsigned long long* q_head;   // device memory: batches claimed
  unsigned long long q_wait_ns; // a group that finds no published batch waits this
                                // long for one (%globaltimer) before ending
};

// Neighbours one thread of the bottom-up thread path has in flight per step
// (4 or 8).
#ifndef IBFS_BU_STEP
#define IBFS_BU_STEP 4
#endif
constexpr int kBuStep = IBFS_BU_STEP;
// Steps of kBuStep neighbours a big vertex (degree above the thread-path
// limit) scans on its own lane before the warp takes it (0: none).
#ifndef IBFS_BU_PEEK
#define IBFS_BU_PEEK 2
#endif
constexpr int kBuPeek = IBFS_BU_PEEK;

// Bottom-up frontier filter.  A neighbour u that did not change at level L-1
// cannot give v a bit it lacks at level L: every bit u held before L-1
// reached v by L-1 already (BFS distances of adjacent vertices differ by at
// most one).  So the scan may skip, exactly, every neighbour outside the
// level-(L-1) changed bitmap.  The bitmap test costs a lookup per neighbour;
// it can pay off when the previous frontier is a small part of the graph
// (the tail levels of a traversal), not when it is a large part.
constexpr long long kFilterDiv = 16;  // auto: filter when prev frontier < V / 16
__host__ __device__ inline bool bu_filter_level(int mode, unsigned long long prev_changed,
                                                long long V) {
  if (mode >= 0) return mode > 0;
  return (long long)prev_changed * kFilterDiv < V;
}

// Whether u is in the previous level's changed bitmap; through L1 when the
// pass runs as a kernel of its own (RO: nothing writes that bitmap while it
// runs), else through L2 (the persistent kernel rewrites it at later levels).
template <bool RO>
__device__ __forceinline__ bool in_front(const uint32_t* front, int32_t u) {
  const uint32_t w = RO ? __ldg(front + (u >> 5)) : __ldcg(front + (u >> 5));
  return (w >> (u & 31)) & 1u;
}

constexpr int kHubScan = 1024;   // neighbours one warp scans before deferring
constexpr int kHubChunk = 2048;  // edges per deferred chunk (one CTA each)

// Neighbour statuses of a bottom-up pass that runs as a kernel of its own
// (RO: nothing writes `last` while it runs) are read through L1 (ld.global.nc):
// most gathers hit the few hub words that the degree order packs into the
// first lines of `last`, and L1 serves them instead of L2.  Measured on
// R-MAT scale 24, one batch at a time: bottom-up 25.1 -> 19.4 ms per
// 1024-source run; the persistent kernel, whose other phases write `last`
// within the same launch, keeps L2 reads.
#ifndef IBFS_BU_NC
#define IBFS_BU_NC 1
#endif

// A team is the set of threads that share one batch: the whole grid in the
// plain schedule, the CTAs of one group in the persistent kernel.
struct Team {
  int block, nblocks;  // CTA index inside the team, team size in CTAs
  long long tid, nthreads;
  long long warp, nwarps;
  int lane;
};

__host__ __device__ inline uint32_t* chg_at(const GroupBufs& gb, const Params& p, int level) {
  return gb.chg + (level & 1) * p.chg_stride;
}

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
template <int WORDS>
__device__ __forceinline__ void ld_status(const uint32_t* p, uint32_t (&x)[WORDS]) {
  if constexpr (WORDS == 1) {
    x[0] = __ldcg(p);
  } else if constexpr (WORDS == 2) {
    uint2 t = __ldcg(reinterpret_cast<const uint2*>(p));
    x[0] = t.x; x[1] = t.y;
  } else if constexpr (WORDS == 4) {
    uint4 t = __ldcg(reinterpret_cast<const uint4*>(p));
    x[0] = t.x; x[1] = t.y; x[2] = t.z; x[3] = t.w;
  } else {
    uint4 a = __ldcg(reinterpret_cast<const uint4*>(p));
    uint4 b = __ldcg(reinterpret_cast<const uint4*>(p) + 1);
    x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
  }
}

template <int WORDS>
__device__ __forceinline__ void st_status(uint32_t* p, const uint32_t (&x)[WORDS]) {
  if constexpr (WORDS == 1) {
    __stcg(p, x[0]);
  } else if constexpr (WORDS == 2) {
    __stcg(reinterpret_cast<uint2*>(p), make_uint2(x[0], x[1]));
  } else if constexpr (WORDS == 4) {
    __stcg(reinterpret_cast<uint4*>(p), make_uint4(x[0], x[1], x[2], x[3]));
  } else {
    __stcg(reinterpret_cast<uint4*>(p), make_uint4(x[0], x[1], x[2], x[3]));
    __stcg(reinterpret_cast<uint4*>(p) + 1, make_uint4(x[4], x[5], x[6], x[7]));
  }
}

// Status read through the non-coherent (L1) path: only for buffers that no
// thread writes while the kernel runs (`last` during a fused bottom-up pass).
template <int WORDS>
__device__ __forceinline__ void ld_status_nc(const uint32_t* p, uint32_t (&x)[WORDS]) {
  if constexpr (WORDS == 1) {
    x[0] = __ldg(p);
  } else if constexpr (WORDS == 2) {
    uint2 t = __ldg(reinterpret_cast<const uint2*>(p));
    x[0] = t.x; x[1] = t.y;
  } else if constexpr (WORDS == 4) {
    uint4 t = __ldg(reinterpret_cast<const uint4*>(p));
    x[0] = t.x; x[1] = t.y; x[2] = t.z; x[3] = t.w;
  } else {
    uint4 a = __ldg(reinterpret_cast<const uint4*>(p));
    uint4 b = __ldg(reinterpret_cast<const uint4*>(p) + 1);
    x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
  }
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile_i32(const int* p) {
  return *reinterpret_cast<const volatile int*>(p);
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bit mask of the sources of a batch of n inside word k.
__host__ __device__ __forceinline__ uint32_t full_word(int n, int k) {
  const int lo = k * 32;
  if (n >= lo + 32) return 0xFFFFFFFFu;
  if (n <= lo) return 0u;
  return (1u << (n - lo)) - 1u;
}

// Number of depth bit-planes that levels 0..max_level use.
__host__ __device__ __forceinline__ int planes_for(int max_level) {
  int p = 0;
  while (p < 31 && (max_level >> p) != 0) p++;
  return p;
}

// Bounded team barrier.  All waits end: after timeout_ns the waiting CTA
// records IBFS_ERR_TIMEOUT (6) in ctl->err and every other CTA leaves on
// seeing a non-zero err.  Returns false when the team must stop.
static __device__ __noinline__ bool team_barrier(Ctl* ctl, unsigned nblocks,
                                                 unsigned long long timeout_ns,
                                                 bool withhold) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned gen = ld_acquire_u32(&ctl->bar_gen);
    if (!withhold) {
      __threadfence();
      const unsigned prev = atomicAdd(&ctl->bar_count, 1u);
      if (prev == nblocks - 1) {
        atomicExch(&ctl->bar_count, 0u);
        __threadfence();
        st_release_u32(&ctl->bar_gen, gen + 1);
      }
    }
    if (ld_acquire_u32(&ctl->bar_gen) == gen) {
      const unsigned long long t0 = global_ns();
      while (ld_acquire_u32(&ctl->bar_gen) == gen) {
        if (ld_volatile_i32(&ctl->err) != 0) { ok = 0; break; }
        if (global_ns() - t0 > timeout_ns) {
          atomicCAS(&ctl->err, 0, 6);
          ok = 0;
          break;
        }
        __nanosleep(100);
      }
    }
    __threadfence();
    if (ld_volatile_i32(&ctl->err) != 0) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// CTA-wide sum of a 64-bit value, then one atomicAdd by thread 0.
__device__ __forceinline__ void cta_add_u64(unsigned long long* dst, unsigned long long x) {
  __shared__ unsigned long long s_red[32];
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) s_red[w] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += s_red[i];
    if (t) atomicAdd(dst, t);
  }
}

__device__ __forceinline__ void cta_or_u32(uint32_t* dst, uint32_t x) {
  __shared__ uint32_t s_or[32];
  x = __reduce_or_sync(0xFFFFFFFFu, x);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) s_or[w] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) t |= s_or[i];
    if (t) atomicOr(dst, t);
  }
}

// Per-source counts of a level's new bits, for the sparse-source decision:
// shared-memory counters per CTA (every thread calls scnt_begin and
// scnt_flush), one atomic add per counted (vertex, source) pair.
__device__ __forceinline__ void scnt_begin(uint32_t* s_cnt) {
  for (int i = threadIdx.x; i < kMaxWords * 32; i += blockDim.x) s_cnt[i] = 0u;
  __syncthreads();
}
template <int WORDS>
__device__ __forceinline__ void scnt_flush(const uint32_t* s_cnt, Par* par) {
  __syncthreads();
  for (int i = threadIdx.x; i < WORDS * 32; i += blockDim.x)
    if (s_cnt[i]) atomicAdd(&par->scnt[i], s_cnt[i]);
}

__device__ __forceinline__ void zero_words(uint32_t* p, long long nwords, const Team& t) {
  // nwords is a multiple of 4 and p 16-byte aligned (allocation padding)
  uint4* q = reinterpret_cast<uint4*>(p);
  const uint4 z = make_uint4(0, 0, 0, 0);
  for (long long i = t.tid; i < nwords / 4; i += t.nthreads) __stcg(q + i, z);
}

// ---------------------------------------------------------------------------
// Direction choice for the next level (host and device use the same rule).
//   fixed (switch_level >= 0): top-down while level <= switch_level, then
//     bottom-up -- the reference's CLI switch level (expander.cuh:687-723);
//   alpha/beta (Beamer et al., SC'12): top-down -> bottom-up when the
//     frontier's edges exceed unexplored_edges/alpha and the frontier is
//     growing; bottom-up -> top-down when the frontier holds fewer than
//     V/beta vertices and is shrinking.  Without the growing/shrinking
//     tests a long shrinking tail (high-diameter graphs) flips direction
//     every level once the unexplored edges run low, paying a full
//     bottom-up sweep for a handful of frontier vertices.
// ---------------------------------------------------------------------------
__host__ __device__ inline int choose_dir(int next_level, int prev_dir,
                                          int switch_level, float alpha,
                                          float beta, unsigned long long changed,
                                          unsigned long long prev_changed,
                                          unsigned long long mf,
                                          unsigned long long m_u, long long V) {
  if (switch_level >= 0) return next_level <= switch_level ? kDirTD : kDirBU;
  if (prev_dir == kDirTD)
    return ((double)mf * (double)alpha > (double)m_u && changed > prev_changed) ? kDirBU
                                                                                : kDirTD;
  return ((double)changed * (double)beta < (double)V && changed < prev_changed) ? kDirTD
                                                                                : kDirBU;
}

// ---------------------------------------------------------------------------
// Phase: seed the sources of one batch (curr bits + level-0 changed bits).
// ---------------------------------------------------------------------------
template <int WORDS>
__device__ void seed_phase(const Params& p, const GroupBufs& gb,
                           const int32_t* src_b, int n_b, const Team& t) {
  uint32_t* chg0 = chg_at(gb, p, 0);
  for (long long i = t.tid; i < n_b; i += t.nthreads) {
    const int32_t v = src_b[i];
    atomicOr(gb.curr + (size_t)v * WORDS + (i >> 5), 1u << (i & 31));
    atomicOr(chg0 + (v >> 5), 1u << (v & 31));
  }
}

// Zero depth bit-plane b when `level` = 2^b, the first level that uses it.
__device__ __forceinline__ void zero_plane_if_first(const Params& p, const GroupBufs& gb,
                                                    int level, const Team& t) {
  if (level > 0 && (level & (level - 1)) == 0) {
    const int b = __ffs(level) - 1;
    zero_words(gb.planes + (size_t)b * p.plane_stride, p.plane_stride, t);
  }
}

// ---------------------------------------------------------------------------
// Phase: inspect level L (reads the level-L bitmap, fixes last, updates the
// depth bit-planes, counters).
// ---------------------------------------------------------------------------
// Per changed vertex v of level L: new bits, last = curr, counters, planes.
template <int WORDS>
__device__ __forceinline__ void inspect_vertex(const Params& p, const GroupBufs& gb, long long v,
                                               int level, bool depth_ok,
                                               const uint32_t (&full)[WORDS], uint32_t (&fm)[WORDS],
                                               unsigned long long& mf, unsigned long long& cnt,
                                               unsigned long long& cdeg,
                                               unsigned long long& teps,
                                               uint32_t (&nb)[WORDS]) {
  uint32_t c[WORDS], l[WORDS];
  ld_status<WORDS>(gb.curr + (size_t)v * WORDS, c);
  ld_status<WORDS>(gb.last + (size_t)v * WORDS, l);
  bool comp = true;
  uint32_t pop = 0;
#pragma unroll
  for (int k = 0; k < WORDS; k++) {
    nb[k] = c[k] & ~l[k];
    comp = comp && (c[k] == full[k]);
    pop += __popc(nb[k]);
    fm[k] |= nb[k];
  }
  st_status<WORDS>(gb.last + (size_t)v * WORDS, c);
  const long long deg = p.beg[v + 1] - p.beg[v];
  mf += deg;
  cnt += 1;
  teps += (unsigned long long)deg * pop;
  if (comp) cdeg += deg;
  if (depth_ok) {
    // depth(v, s) = level for the new bits: OR them into the planes of the
    // level's set bits (one coalesced read-modify-write per plane), two
    // planes at a time so that their loads are in flight together.
    uint32_t* q0 = gb.planes + (size_t)v * WORDS;
    unsigned rest = (unsigned)level;
    while (rest) {
      const int b0 = __ffs(rest) - 1;
      rest &= rest - 1;
      uint32_t* qa = q0 + (size_t)b0 * p.plane_stride;
      uint32_t xa[WORDS];
      ld_status<WORDS>(qa, xa);
      if (rest) {
        const int b1 = __ffs(rest) - 1;
        rest &= rest - 1;
        uint32_t* qb = q0 + (size_t)b1 * p.plane_stride;
        uint32_t xb[WORDS];
        ld_status<WORDS>(qb, xb);
#pragma unroll
        for (int k = 0; k < WORDS; k++) xb[k] |= nb[k];
        st_status<WORDS>(qb, xb);
      }
#pragma unroll
      for (int k = 0; k < WORDS; k++) xa[k] |= nb[k];
      st_status<WORDS>(qa, xa);
    }
  }
}

// ---------------------------------------------------------------------------
// Phase: inspect level L (reads the level-L bitmap, fixes last, updates the
// depth bit-planes, counters).  Every warp step takes 32 bitmap words (1024
// vertices) and compacts their set bits across the warp: lane j of round k
// inspects the (32k + j)-th changed vertex of the chunk, found by a binary
// search over the warp's inclusive bit counts (per-lane shuffles) and
// __fns within the owning word.  All 32 lanes work on a changed vertex in
// every full round whatever the density or the spread of the changed set,
// so a frontier scattered thinly over the whole graph (a grid late in a
// traversal, a power-law graph's tail) costs rounds of 32 vertices, not
// one mostly idle round per non-empty word.
//
// LEAN selects the walk of the persistent kernel instead, whose budget of
// 64 registers per thread (2 x 512 threads per SM) has no room for the
// compaction: lanes map to the bits of one word, one word per warp step
// (`dense`, many changed vertices) or the non-empty words of 128-word
// blocks (few changed vertices).
// ---------------------------------------------------------------------------
template <int WORDS, bool LEAN>
__device__ void inspect_phase(const Params& p, const GroupBufs& gb, Par* par, int n_b,
                              int level, bool depth_ok, bool dense, const Team& t) {
  uint32_t full[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) full[k] = full_word(n_b, k);
  unsigned long long mf = 0, cnt = 0, cdeg = 0, teps = 0;
  uint32_t fm[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) fm[k] = 0;
  const uint32_t* chg = chg_at(gb, p, level);
  // the bitmap of level+1 (last used by level-1's expand) must start empty:
  // bottom-up merges into it with atomics
  zero_words(chg_at(gb, p, level + 1), p.chg_stride, t);
  const int lane = t.lane;
  uint32_t nbx[WORDS];  // the new bits of the vertex a lane inspected (unused here)
  if (LEAN && dense) {
    for (long long w = t.warp; w < p.nchg; w += t.nwarps) {
      const uint32_t bits = __ldcg(chg + w);
      if (!bits) continue;
      const long long v = w * 32 + lane;
      if ((bits >> lane) & 1u)
        inspect_vertex<WORDS>(p, gb, v, level, depth_ok, full, fm, mf, cnt, cdeg, teps, nbx);
    }
  } else if (LEAN) {
    const long long nblk = (p.nchg + 127) / 128;
    for (long long blk = t.warp; blk < nblk; blk += t.nwarps) {
      const uint4 q4 = __ldcg(reinterpret_cast<const uint4*>(chg) + blk * 32 + lane);
      uint32_t nzl = __ballot_sync(0xFFFFFFFFu, (q4.x | q4.y | q4.z | q4.w) != 0u);
      while (nzl) {
        const int src = __ffs(nzl) - 1;
        nzl &= nzl - 1;
        const uint32_t b0 = __shfl_sync(0xFFFFFFFFu, q4.x, src);
        const uint32_t b1 = __shfl_sync(0xFFFFFFFFu, q4.y, src);
        const uint32_t b2 = __shfl_sync(0xFFFFFFFFu, q4.z, src);
        const uint32_t b3 = __shfl_sync(0xFFFFFFFFu, q4.w, src);
        const long long w0 = blk * 128 + src * 4;
        if ((b0 >> lane) & 1u)
          inspect_vertex<WORDS>(p, gb, (w0 + 0) * 32 + lane, level, depth_ok, full, fm, mf, cnt, cdeg, teps, nbx);
        if ((b1 >> lane) & 1u)
          inspect_vertex<WORDS>(p, gb, (w0 + 1) * 32 + lane, level, depth_ok, full, fm, mf, cnt, cdeg, teps, nbx);
        if ((b2 >> lane) & 1u)
          inspect_vertex<WORDS>(p, gb, (w0 + 2) * 32 + lane, level, depth_ok, full, fm, mf, cnt, cdeg, teps, nbx);
        if ((b3 >> lane) & 1u)
          inspect_vertex<WORDS>(p, gb, (w0 + 3) * 32 + lane, level, depth_ok, full, fm, mf, cnt, cdeg, teps, nbx);
      }
    }
  } else {
  const long long nchunk = (p.nchg + 31) / 32;  // whole chunks lie inside chg_stride
  for (long long c = t.warp; c < nchunk; c += t.nwarps) {
    const uint32_t word = __ldcg(chg + c * 32 + lane);
    if (__ballot_sync(0xFFFFFFFFu, word != 0u) == 0u) continue;
    const int own = __popc(word);
    int incl = own;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    const int excl = incl - own;
    const int total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    for (int base = 0; base < total; base += 32) {
      const int r = base + lane;
      // owner = number of lanes whose inclusive count is <= r
      int lo = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const int probe = __shfl_sync(0xFFFFFFFFu, incl, lo + step - 1);
        if (probe <= r) lo += step;
      }
      const uint32_t w = __shfl_sync(0xFFFFFFFFu, word, lo);
      const int e = __shfl_sync(0xFFFFFFFFu, excl, lo);
      if (r < total) {
        const int bit = (int)__fns(w, 0u, r - e + 1);
        const long long v = (c * 32 + lo) * 32 + bit;
        inspect_vertex<WORDS>(p, gb, v, level, depth_ok, full, fm, mf, cnt, cdeg, teps, nbx);
      }
    }
  }
  }
  if (!depth_ok && cnt) par->range_err = 1;
  cta_add_u64(&par->changed, cnt);
  cta_add_u64(&par->mf, mf);
  cta_add_u64(&par->cdeg, cdeg);
  cta_add_u64(&par->teps, teps);
#pragma unroll
  for (int k = 0; k < WORDS; k++) cta_or_u32(&par->fmask[k], fm[k]);
}

// Whether the lean inspect of the next level should use the dense walk: its
// changed set is at most the previous frontier's neighbourhood.
__host__ __device__ inline bool inspect_dense(unsigned long long prev_mf, long long V) {
  return prev_mf * 16ull > (unsigned long long)V;
}

// ---------------------------------------------------------------------------
// Phase: build the joint frontier queues for top-down level L from the
// level-(L-1) bitmap (warp-ballot compaction, degree classes as td_inspect,
// inspector.cuh:534-626: deg < sml -> small, deg > lrg -> large, else
// medium, deg 0 dropped).  Large vertices are cut into chunks of p.chunk
// edges.  Clears the level-L bitmap that the top-down pass will fill.
// ---------------------------------------------------------------------------
// With `sync` (a top-down level right after a fused bottom-up level, which
// left the new statuses in `last` and the previous ones in `curr`) every
// changed vertex also copies last -> curr, restoring curr == last.
template <int WORDS = 4>
__device__ inline void qbuild_phase(const Params& p, const GroupBufs& gb, int level,
                                    int32_t* qc, const Team& t, bool sync = false) {
  const int lane = t.lane;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t* prev = chg_at(gb, p, level - 1);
  uint32_t* next = chg_at(gb, p, level);
  const long long nblk = (p.nchg + 127) / 128;
  for (long long blk = t.warp; blk < nblk; blk += t.nwarps) {
   const uint4 q4 = __ldcg(reinterpret_cast<const uint4*>(prev) + blk * 32 + lane);
   __stcg(reinterpret_cast<uint4*>(next) + blk * 32 + lane, make_uint4(0, 0, 0, 0));
   uint32_t nzl = __ballot_sync(0xFFFFFFFFu, (q4.x | q4.y | q4.z | q4.w) != 0u);
   while (nzl) {
    const int src_lane = __ffs(nzl) - 1;
    nzl &= nzl - 1;
    const uint32_t qw[4] = {__shfl_sync(0xFFFFFFFFu, q4.x, src_lane),
                            __shfl_sync(0xFFFFFFFFu, q4.y, src_lane),
                            __shfl_sync(0xFFFFFFFFu, q4.z, src_lane),
                            __shfl_sync(0xFFFFFFFFu, q4.w, src_lane)};
    for (int kk = 0; kk < 4; kk++) {
    const uint32_t bits = qw[kk];
    if (!bits) continue;
    const long long w = blk * 128 + src_lane * 4 + kk;
    const long long v = w * 32 + lane;
    const bool mine = (bits >> lane) & 1u;
    long long deg = 0;
    if (mine) deg = p.beg[v + 1] - p.beg[v];
    if (sync && mine) {
      uint32_t x[WORDS];
      ld_status<WORDS>(gb.last + (size_t)v * WORDS, x);
      st_status<WORDS>(gb.curr + (size_t)v * WORDS, x);
    }
    const int cls = (!mine || deg == 0) ? -1 : deg < p.sml ? 0 : deg <= p.lrg ? 1 : 2;
    const uint32_t m0 = __ballot_sync(0xFFFFFFFFu, cls == 0);
    if (m0) {
      const int leader = __ffs(m0) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(&qc[0], __popc(m0));
      base = __shfl_sync(0xFFFFFFFFu, base, leader);
      if (cls == 0) gb.qs[base + __popc(m0 & lt)] = (int32_t)v;
    }
    const uint32_t m1 = __ballot_sync(0xFFFFFFFFu, cls == 1);
    if (m1) {
      const int leader = __ffs(m1) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(&qc[1], __popc(m1));
      base = __shfl_sync(0xFFFFFFFFu, base, leader);
      if (cls == 1) gb.qm[base + __popc(m1 & lt)] = (int32_t)v;
    }
    const uint32_t m2 = __ballot_sync(0xFFFFFFFFu, cls == 2);
    if (m2) {
      int nch = cls == 2 ? (int)((deg + p.chunk - 1) / p.chunk) : 0;
      int incl = nch;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      const int total = __shfl_sync(0xFFFFFFFFu, incl, 31);
      int base = 0;
      if (lane == 0) base = atomicAdd(&qc[2], total);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      const int first = base + incl - nch;
      for (int c = 0; c < nch; c++) gb.ql[first + c] = make_int2((int)v, c);
    }
    }
   }
  }
}

// Fire-and-forget ORs (red: no value comes back, so nothing waits on them).
__device__ __forceinline__ void red_or_u32(uint32_t* p, uint32_t x) {
  asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(p), "r"(x) : "memory");
}
__device__ __forceinline__ void red_or_u64(unsigned long long* p, unsigned long long x) {
  asm volatile("red.relaxed.gpu.global.or.b64 [%0], %1;" ::"l"(p), "l"(x) : "memory");
}

// Top-down edges: push the frontier word P of v into neighbours u[0..cnt).
// The status reads of all cnt neighbours are issued before any of them is
// used, so one thread has cnt gathers in flight instead of one.
// The status read s (through L2) decides everything: every level starts
// with curr == last, so bits of P missing from s are missing from last[u],
// and once ORed in (by this thread or a concurrent one) u has changed at
// this level.  So the ORs into curr[u] and into the changed bitmap are
// reductions whose old value is never needed: the thread issues them and
// goes on instead of waiting for L2 round trips.  A stale s (fewer bits)
// costs at most one redundant OR.
constexpr int kTdStep = 4;  // edges one thread has in flight
template <int WORDS>
__device__ __forceinline__ void td_push_n(const GroupBufs& gb, uint32_t* chg,
                                          const int32_t (&u)[kTdStep], int cnt,
                                          const uint32_t (&P)[WORDS]) {
  uint32_t s[kTdStep][WORDS];
#pragma unroll
  for (int i = 0; i < kTdStep; i++) {
    if (i < cnt) {
      ld_status<WORDS>(gb.curr + (size_t)u[i] * WORDS, s[i]);
    } else {
#pragma unroll
      for (int k = 0; k < WORDS; k++) s[i][k] = 0xFFFFFFFFu;
    }
  }
#pragma unroll
  for (int i = 0; i < kTdStep; i++) {
    bool need = false;
#pragma unroll
    for (int k = 0; k < WORDS; k++) need |= (P[k] & ~s[i][k]) != 0u;
    if (!need) continue;
    if constexpr (WORDS == 1) {
      red_or_u32(gb.curr + u[i], P[0]);
    } else {
      unsigned long long* q = reinterpret_cast<unsigned long long*>(gb.curr + (size_t)u[i] * WORDS);
#pragma unroll
      for (int k = 0; k < WORDS / 2; k++) {
        const uint32_t n0 = P[2 * k] & ~s[i][2 * k], n1 = P[2 * k + 1] & ~s[i][2 * k + 1];
        if (n0 | n1) red_or_u64(q + k, ((unsigned long long)P[2 * k + 1] << 32) | P[2 * k]);
      }
    }
    red_or_u32(chg + (u[i] >> 5), 1u << (u[i] & 31));
  }
}

// ---- bulk-copy (TMA) staging of large vertices' adjacency chunks ---------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// One untiled bulk copy global -> shared (both addresses 16-byte aligned,
// bytes a multiple of 16), completing on `bar`.  The source is this GPU's
// own CSR; no multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of `bar` (each try_wait suspends the
// thread for a while in hardware; kMbarTries of them is seconds).
constexpr long long kMbarTries = 1LL << 22;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  for (long long i = 0; i < kMbarTries; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

constexpr int kStageInts = 2048 + 8;  // one chunk (threads*4 <= 2048) plus alignment slack

// The column-id range [a0, a1) that covers chunk c of a large vertex with
// 16-byte aligned ends (col is 16-byte aligned and padded by 4 entries).
__device__ __forceinline__ void td_chunk(const Params& p, const GroupBufs& gb, int c, int32_t* v,
                                         long long* b0, long long* b1, long long* a0,
                                         long long* a1) {
  const int2 d = gb.ql[c];
  *v = d.x;
  const long long e_end = p.beg[d.x + 1];
  *b0 = p.beg[d.x] + (long long)d.y * p.chunk;
  *b1 = min(e_end, *b0 + (long long)p.chunk);
  *a0 = *b0 & ~3LL;
  *a1 = (*b1 + 3) & ~3LL;
}

// ---------------------------------------------------------------------------
// Phase: top-down expansion of level L over the three queues: one CTA per
// chunk of a large vertex (td_expand_cta, expander.cuh:276-331), one warp
// per medium vertex (td_expand_warp, expander.cuh:208-267), one thread per
// small vertex (td_expand_thd, expander.cuh:140-199).  Every thread takes
// kTdStep edges at a time: their column ids first, then their statuses.
// STAGE (the phase's own kernel, chunk <= 2048) with Params::td_stage: the
// large vertices' chunks -- the hubs' adjacency -- are staged through shared
// memory by bulk copies (TMA, cp.async.bulk), double-buffered: while the CTA
// pushes one chunk's edges, the next chunk's column ids are already on
// their way, so the pushes never wait for a column read.  Off by default:
// on R-MAT scale 24 the top-down levels are bound by the random status
// gathers, not by the column reads, and staging measured ~1 % slower.
// ---------------------------------------------------------------------------
template <int WORDS, bool STAGE = false>
__device__ void td_phase(const Params& p, const GroupBufs& gb, int level, const int32_t* qc,
                         const Team& t) {
  uint32_t* chg = chg_at(gb, p, level);
  const int nS = __ldcg(qc + 0), nM = __ldcg(qc + 1), nL = __ldcg(qc + 2);
  if (STAGE && p.td_stage) {
    __shared__ __align__(128) int32_t s_col[2][kStageInts];
    __shared__ __align__(8) unsigned long long s_bar[2];
    __shared__ int s_fail;
    if (threadIdx.x == 0) {
      mbar_init(&s_bar[0], 1);
      mbar_init(&s_bar[1], 1);
      mbar_init_fence();
      s_fail = 0;
    }
    __syncthreads();
    auto issue = [&](int i) {  // thread 0: chunk i of this CTA into buffer i & 1
      int32_t v;
      long long b0, b1, a0, a1;
      td_chunk(p, gb, t.block + i * t.nblocks, &v, &b0, &b1, &a0, &a1);
      const unsigned bytes = (unsigned)((a1 - a0) * 4);
      mbar_expect_tx(&s_bar[i & 1], bytes);
      bulk_g2s(s_col[i & 1], p.col + a0, bytes, &s_bar[i & 1]);
    };
    int issued = 0;  // chunks whose copy thread 0 has started
    if (threadIdx.x == 0 && t.block < nL) {
      issue(0);
      issued = 1;
    }
    for (int i = 0;; i++) {
      const int c = t.block + i * t.nblocks;
      if (c >= nL) break;
      if (threadIdx.x == 0 && c + t.nblocks < nL) {
        issue(i + 1);
        issued = i + 2;
      }
      int32_t v;
      long long b0, b1, a0, a1;
      td_chunk(p, gb, c, &v, &b0, &b1, &a0, &a1);
      uint32_t P[WORDS];
      ld_status<WORDS>(gb.last + (size_t)v * WORDS, P);
      if (!mbar_wait(&s_bar[i & 1], (unsigned)((i >> 1) & 1))) s_fail = 1;
      __syncthreads();
      if (s_fail) break;  // uniform
      const int32_t* sc = s_col[i & 1] + (b0 - a0);
      const int n = (int)(b1 - b0);
      for (int j = threadIdx.x; j < n; j += kTdStep * blockDim.x) {
        int32_t u[kTdStep];
        int cnt = 0;
#pragma unroll
        for (int q = 0; q < kTdStep; q++) {
          const int jq = j + q * (int)blockDim.x;
          u[q] = jq < n ? sc[jq] : 0;
          cnt += jq < n ? 1 : 0;
        }
        td_push_n<WORDS>(gb, chg, u, cnt, P);
      }
      __syncthreads();  // buffer i & 1 is read: the copy of chunk i + 2 may reuse it
    }
    if (s_fail && threadIdx.x == 0) {
      // a copy did not complete in time: report it, and before the CTA's
      // shared memory goes away, wait (bounded) for every copy it started
      atomicCAS(&gb.ctl->err, 0, 6);
      for (int i = 0; i < issued; i++) (void)mbar_wait(&s_bar[i & 1], (unsigned)((i >> 1) & 1));
    }
  } else {
    for (int c = t.block; c < nL; c += t.nblocks) {
      int32_t v;
      long long b0, b1, a0, a1;
      td_chunk(p, gb, c, &v, &b0, &b1, &a0, &a1);
      uint32_t P[WORDS];
      ld_status<WORDS>(gb.last + (size_t)v * WORDS, P);
      for (long long e = b0 + threadIdx.x; e < b1; e += (long long)kTdStep * blockDim.x) {
        int32_t u[kTdStep];
        int cnt = 0;
#pragma unroll
        for (int i = 0; i < kTdStep; i++) {
          const long long ei = e + (long long)i * blockDim.x;
          u[i] = ei < b1 ? __ldg(p.col + ei) : 0;
          cnt += ei < b1 ? 1 : 0;
        }
        td_push_n<WORDS>(gb, chg, u, cnt, P);
      }
    }
  }
  for (long long i = t.warp; i < nM; i += t.nwarps) {
    const int32_t v = gb.qm[i];
    uint32_t P[WORDS];
    ld_status<WORDS>(gb.last + (size_t)v * WORDS, P);
    const long long b1 = p.beg[v + 1];
    for (long long e = p.beg[v] + t.lane; e < b1; e += 32 * kTdStep) {
      int32_t u[kTdStep];
      int cnt = 0;
#pragma unroll
      for (int j = 0; j < kTdStep; j++) {
        const long long ej = e + 32LL * j;
        u[j] = ej < b1 ? __ldg(p.col + ej) : 0;
        cnt += ej < b1 ? 1 : 0;
      }
      td_push_n<WORDS>(gb, chg, u, cnt, P);
    }
  }
  for (long long i = t.tid; i < nS; i += t.nthreads) {
    const int32_t v = gb.qs[i];
    uint32_t P[WORDS];
    ld_status<WORDS>(gb.last + (size_t)v * WORDS, P);
    const long long b1 = p.beg[v + 1];
    for (long long e = p.beg[v]; e < b1; e += kTdStep) {
      int32_t u[kTdStep];
      const int cnt = (int)min((long long)kTdStep, b1 - e);
#pragma unroll
      for (int j = 0; j < kTdStep; j++) u[j] = j < cnt ? __ldg(p.col + e + j) : 0;
      td_push_n<WORDS>(gb, chg, u, cnt, P);
    }
  }
}

// Second bottom-up stage: the hubs that were still missing frontier bits
// after their first hub_t neighbours.  One CTA per chunk of kHubChunk edges
// (frontier neighbours only); a chunk is skipped when curr[v], which the
// other chunks of the same hub merge into with atomics, already covers
// every frontier bit.  So one hub's long scan is spread over many CTAs
// instead of holding one warp -- and the whole level -- for its adjacency.
template <int WORDS, bool RO = false>
__device__ void bu_defer_phase(const Params& p, const GroupBufs& gb, int level,
                               const uint32_t* fmask_g, const int32_t* hq_cnt, const Team& t,
                               bool filt = false, const uint32_t* smask = nullptr) {
  __shared__ uint32_t s_acc[32][kMaxWords];
  __shared__ uint32_t s_cur[kMaxWords];
  __shared__ int s_skip;
  uint32_t fm[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) fm[k] = __ldcg(fmask_g + k) & (smask ? ~__ldcg(smask + k) : ~0u);
  const uint32_t* front = chg_at(gb, p, level - 1);
  uint32_t* out = chg_at(gb, p, level);
  const int n = __ldcg(hq_cnt);
  const int lane = t.lane, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c = t.block; c < n; c += t.nblocks) {
    const int2 hc = gb.hq[c];
    const int32_t v = hc.x;
    if (threadIdx.x == 0) {  // one read, so that the skip decision is uniform
      uint32_t cur[WORDS];
      ld_status<WORDS>(gb.curr + (size_t)v * WORDS, cur);
      bool need = false;
#pragma unroll
      for (int k = 0; k < WORDS; k++) {
        s_cur[k] = cur[k];
        need |= (fm[k] & ~cur[k]) != 0u;
      }
      s_skip = need ? 0 : 1;
    }
    __syncthreads();
    if (s_skip) {
      __syncthreads();
      continue;
    }
    const long long e_end = p.beg[v + 1];
    const long long b0 = p.beg[v] + p.hub_t + (long long)hc.y * kHubChunk;
    const long long b1 = min(e_end, b0 + (long long)kHubChunk);
    uint32_t acc[WORDS];
#pragma unroll
    for (int k = 0; k < WORDS; k++) acc[k] = 0;
    for (long long e = b0 + threadIdx.x; e < b1; e += blockDim.x) {
      const int32_t u = p.col[e];
      if (filt && !in_front<RO>(front, u)) continue;
      uint32_t x[WORDS];
      if constexpr (RO && IBFS_BU_NC) ld_status_nc<WORDS>(gb.last + (size_t)u * WORDS, x);
      else ld_status<WORDS>(gb.last + (size_t)u * WORDS, x);
#pragma unroll
      for (int k = 0; k < WORDS; k++) acc[k] |= x[k];
    }
#pragma unroll
    for (int k = 0; k < WORDS; k++) {
      const uint32_t r = __reduce_or_sync(0xFFFFFFFFu, acc[k]);
      if (lane == 0) s_acc[wid][k] = r;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t nb[WORDS];
      bool any = false;
#pragma unroll
      for (int k = 0; k < WORDS; k++) {
        uint32_t r = 0;
        for (int i = 0; i < nw; i++) r |= s_acc[i][k];
        nb[k] = r & ~s_cur[k];
        any |= nb[k] != 0u;
      }
      if (any) {
        if constexpr (WORDS == 1) {
          atomicOr(gb.curr + v, nb[0]);
        } else {
          unsigned long long* q = reinterpret_cast<unsigned long long*>(gb.curr + (size_t)v * WORDS);
#pragma unroll
          for (int k = 0; k < WORDS / 2; k++) {
            const unsigned long long w2 = ((unsigned long long)nb[2 * k + 1] << 32) | nb[2 * k];
            if (w2) atomicOr(q + k, w2);
          }
        }
        atomicOr(out + (v >> 5), 1u << (v & 31));
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Phase: bottom-up level L.  Every vertex that still lacks a bit of the
// previous level's frontier mask ORs the `last` words of those neighbours
// that were in the previous frontier (a bit can only come from a vertex
// that gained it at level L-1; the level-(L-1) bitmap, L2 resident, filters
// the others before their status word is read) and stops as soon as no
// frontier bit is missing -- the early exit of expander.cu:298,348,
// generalised from "all bits" to "all bits any frontier vertex carries".
// Low-degree vertices scan with one thread (sw_expand_thd, expander.cuh:
// 431-489), the rest with the whole warp and a warp OR-reduction
// (sw_expand_warp, expander.cuh:341-422).
// ---------------------------------------------------------------------------
//
// FUSED (device loop only) also does the inspect work of the level in the
// same pass, so that bottom-up levels need no inspect pass: every vertex's
// new status goes to `curr` (for all vertices, changed or not: `curr` then
// holds the complete status of the level while `last` keeps the previous
// one, and the caller swaps their roles), the new bits update the depth
// planes and the counters directly (the whole plane b is written at level
// 2^b, so it needs no zeroing), and the changed bitmap is still marked for a
// following top-down level.  Hubs deferred to bu_defer_phase get their
// planes and counters in bu_hub_epilogue.
// Status of neighbour u for a bottom-up scan: from the CTA's shared-memory
// copy of the hubs' statuses when u is one of the first hk vertices, else
// from `last` (through L1 when NC: `last` is read-only during a fused pass).
template <int WORDS, int HK, bool NC>
__device__ __forceinline__ void ld_nbr(const uint32_t* last, const uint32_t* s_hub, long long hk,
                                       int32_t u, uint32_t (&x)[WORDS]) {
  if (HK > 0 && u < hk) {
    if constexpr (WORDS >= 4) {
#pragma unroll
      for (int q = 0; q < WORDS / 4; q++) {
        const uint4 t = reinterpret_cast<const uint4*>(s_hub + (size_t)u * WORDS)[q];
        x[4 * q] = t.x; x[4 * q + 1] = t.y; x[4 * q + 2] = t.z; x[4 * q + 3] = t.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < WORDS; k++) x[k] = s_hub[(size_t)u * WORDS + k];
    }
    return;
  }
  if constexpr (NC) ld_status_nc<WORDS>(last + (size_t)u * WORDS, x);
  else ld_status<WORDS>(last + (size_t)u * WORDS, x);
}

// smask (device loop, sparse-source levels): bits pushed top-down after this
// pass (push_queue_phase / push_run_phase); the scan's early exit ignores them.
template <int WORDS, bool FUSED = false, bool RO = FUSED, int HK = 0>
__device__ void bu_phase(const Params& p, const GroupBufs& gb, int level,
                         const uint32_t* fmask_g, int32_t* hq_cnt, const Team& t,
                         Par* par = nullptr, int n_b = 0, bool depth_ok = true,
                         bool filt = false, const uint32_t* smask = nullptr) {
  constexpr bool NC = RO && IBFS_BU_NC;
  // Hub status cache (HK > 0, passes that run as their own kernel: `last` is
  // not written while they run).  The degree order puts the highest-degree vertices at
  // internal ids 0..HK-1 and every adjacency list is ascending, so the first
  // neighbours a scan reads -- the ones that usually complete it -- are these
  // hubs: every CTA copies their previous-level statuses into shared memory
  // once and reads them from there instead of from L2.
  __shared__ __align__(16) uint32_t s_hub[HK > 0 ? HK * WORDS : 4];
  long long hk = 0;
  if constexpr (HK > 0) {
    hk = min((long long)HK, (long long)p.V);
    for (long long i = threadIdx.x; i < hk * WORDS; i += blockDim.x) s_hub[i] = __ldcg(gb.last + i);
    __syncthreads();
  }
  uint32_t fm[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) fm[k] = __ldcg(fmask_g + k) & (smask ? ~__ldcg(smask + k) : ~0u);
  const uint32_t* front = chg_at(gb, p, level - 1);
  uint32_t* out = chg_at(gb, p, level);
  const int lane = t.lane;
  // FUSED counters (as inspect_phase); degree sums of one thread's vertices
  // are below E < 2^31, so 32 bits hold them
  uint32_t f_mf = 0, f_cnt = 0, f_cdeg = 0;
  unsigned long long f_teps = 0;
  uint32_t full[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) full[k] = full_word(n_b, k);
  // the OR of the level's new bits: per warp step a warp OR-reduction into
  // shared memory (fewer live registers than a per-thread accumulator)
  __shared__ uint32_t s_fm[kMaxWords];
  if (FUSED) {
    if (threadIdx.x < kMaxWords) s_fm[threadIdx.x] = 0u;
    __syncthreads();
  }
  const bool first_plane = (level & (level - 1)) == 0;
  const int pb = __ffs(level) - 1;
  bool range = false;
  // The degree order puts every vertex above the thread-path limit into the
  // prefix [0, p.big_prefix): one warp per vertex there, so that the hubs,
  // which that order packs into a few warps, are spread over all of them.
  for (long long v = t.warp; v < p.big_prefix; v += t.nwarps) {
    uint32_t l[WORDS];
    ld_status<WORDS>(gb.last + (size_t)v * WORDS, l);
    const long long e0 = p.beg[v], e1 = p.beg[v + 1];
    bool need = false;
#pragma unroll
    for (int k = 0; k < WORDS; k++) need |= (fm[k] & ~l[k]) != 0u;
    need = need && e1 > e0;  // uniform across the warp
    uint32_t a[WORDS];
#pragma unroll
    for (int k = 0; k < WORDS; k++) a[k] = l[k];
    bool defer = false;
    if (need) {
      const long long e_lim = (e1 - e0 > p.hub_t) ? e0 + p.hub_t : e1;
      bool miss = true;
      for (long long e = e0; e < e_lim; e += 32) {
        uint32_t x[WORDS];
#pragma unroll
        for (int k = 0; k < WORDS; k++) x[k] = 0;
        if (e + lane < e_lim) {
          const int32_t u = p.col[e + lane];
          if (!filt || in_front<RO>(front, u))
            ld_nbr<WORDS, HK, NC>(gb.last, s_hub, hk, u, x);
        }
        miss = false;
#pragma unroll
        for (int k = 0; k < WORDS; k++) {
          a[k] |= __reduce_or_sync(0xFFFFFFFFu, x[k]);
          miss |= (fm[k] & ~a[k]) != 0u;
        }
        if (!miss) break;
      }
      defer = miss && e_lim < e1;
      if (defer && lane == 0) {
        const int nch = (int)((e1 - e_lim + kHubChunk - 1) / kHubChunk);
        const int base0 = atomicAdd(hq_cnt, nch);
        for (int c = 0; c < nch; c++) gb.hq[base0 + c] = make_int2((int)v, c);
      }
    }
    bool ch = false;
#pragma unroll
    for (int k = 0; k < WORDS; k++) ch |= a[k] != l[k];
    if (lane == 0) {
      if constexpr (!FUSED) {
        if (ch) {
          st_status<WORDS>(gb.curr + (size_t)v * WORDS, a);
          atomicOr(out + (v >> 5), 1u << (v & 31));
        }
      } else {
        st_status<WORDS>(gb.curr + (size_t)v * WORDS, a);  // every vertex: curr = new status
        const bool epi = ch && !defer;
        uint32_t nb[WORDS];
        uint32_t pop = 0;
        bool comp = true;
#pragma unroll
        for (int k = 0; k < WORDS; k++) {
          nb[k] = epi ? (a[k] & ~l[k]) : 0u;
          pop += __popc(nb[k]);
          comp = comp && a[k] == full[k];
          if (nb[k]) atomicOr(&s_fm[k], nb[k]);
        }
        if (epi) {
          const uint32_t deg = (uint32_t)(e1 - e0);
          f_cnt += 1;
          f_mf += deg;
          f_teps += (unsigned long long)deg * pop;
          if (comp) f_cdeg += deg;
          if (!depth_ok) range = true;
          atomicOr(out + (v >> 5), 1u << (v & 31));
        }
        uint32_t* q0 = gb.planes + (size_t)v * WORDS;
        if (first_plane) {
          st_status<WORDS>(q0 + (size_t)pb * p.plane_stride, nb);
        } else if (epi && depth_ok) {
          unsigned rest = (unsigned)level;
          while (rest) {
            const int b0p = __ffs(rest) - 1;
            rest &= rest - 1;
            uint32_t* qa = q0 + (size_t)b0p * p.plane_stride;
            uint32_t xa[WORDS];
            ld_status<WORDS>(qa, xa);
#pragma unroll
            for (int k = 0; k < WORDS; k++) xa[k] |= nb[k];
            st_status<WORDS>(qa, xa);
          }
        }
      }
    }
  }
  const long long start = p.big_prefix;  // a multiple of 32
  const long long rstep = t.nwarps * 32;
  if (FUSED && first_plane) {
    // the pass writes its first-used plane whole; the edgeless tail it does
    // not sweep gets zeros (an edgeless source keeps depth 0)
    const long long n4 = (p.V - p.v_nz) * WORDS / 4;
    uint4* q = reinterpret_cast<uint4*>(gb.planes + (size_t)pb * p.plane_stride +
                                        (size_t)p.v_nz * WORDS);
    for (long long i = t.tid; i < n4 + ((p.V - p.v_nz) * WORDS % 4 ? 1 : 0); i += t.nthreads)
      __stcg(q + i, make_uint4(0, 0, 0, 0));
  }
  for (long long base = start + t.warp * 32; base < p.v_nz; base += rstep) {
    const long long v = base + lane;
    const bool valid = v < p.V;
    uint32_t l[WORDS], acc[WORDS];
    long long b0 = 0, b1 = 0;
    if (valid) {
      ld_status<WORDS>(gb.last + (size_t)v * WORDS, l);
      b0 = p.beg[v];
      b1 = p.beg[v + 1];
    } else {
#pragma unroll
      for (int k = 0; k < WORDS; k++) l[k] = 0;
    }
    bool need = false;
#pragma unroll
    for (int k = 0; k < WORDS; k++) {
      acc[k] = l[k];
      need |= (fm[k] & ~l[k]) != 0u;
    }
    need = need && valid && (b1 > b0);
    const bool small = need && (b1 - b0) <= p.but;
    // Every vertex that needs bits scans on its own lane first: a small one
    // its whole list, a big one only its first kBuPeek steps -- its
    // highest-degree neighbours, which in the degree order usually cover
    // the frontier bits already.  Only big vertices still missing bits go on
    // to the warp scan below, which takes them one at a time.
    bool covered = false;
    long long e_big = b0;  // where a big vertex's warp scan starts
    if (need) {
      // kBuStep neighbours in flight per step; with col_vec their ids come as
      // aligned 16-byte vectors (col is padded by 4 entries at its end, and
      // a vector is only read when it starts before b1)
      constexpr int S = kBuStep;
      const int4* col4 = reinterpret_cast<const int4*>(p.col);
      const long long a0 = p.col_vec ? (b0 & ~3LL) : b0;
      const long long a_end = small ? b1 : min(b1, a0 + (long long)kBuPeek * S);
      if (!small) e_big = max(b0, a_end);
      for (long long a = a0; a < a_end; a += S) {
        int32_t u[S];
        if (p.col_vec) {
#pragma unroll
          for (int q = 0; q < S / 4; q++) {
            int4 c4 = make_int4(0, 0, 0, 0);
            if (q == 0 || a + 4 * q < b1) c4 = __ldg(col4 + ((a >> 2) + q));
            u[4 * q] = c4.x; u[4 * q + 1] = c4.y; u[4 * q + 2] = c4.z; u[4 * q + 3] = c4.w;
          }
        } else {
#pragma unroll
          for (int i = 0; i < S; i++) u[i] = a + i < b1 ? __ldg(p.col + a + i) : 0;
        }
        bool f[S];
#pragma unroll
        for (int i = 0; i < S; i++) {
          const bool in = (a + i >= b0) && (a + i < b1);
          f[i] = in && (!filt || in_front<RO>(front, u[i]));
        }
        uint32_t x[S][WORDS];
#pragma unroll
        for (int i = 0; i < S; i++) {
          if (f[i]) {
            ld_nbr<WORDS, HK, NC>(gb.last, s_hub, hk, u[i], x[i]);
          } else {
#pragma unroll
            for (int k = 0; k < WORDS; k++) x[i][k] = 0;
          }
        }
        bool miss = false;
#pragma unroll
        for (int k = 0; k < WORDS; k++) {
#pragma unroll
          for (int i = 0; i < S; i++) acc[k] |= x[i][k];
          miss |= (fm[k] & ~acc[k]) != 0u;
        }
        if (!miss) {
          covered = true;
          break;
        }
      }
    }
    bool deferred = false;  // this lane's vertex left chunks to bu_defer_phase
    uint32_t big = __ballot_sync(0xFFFFFFFFu, need && !small && !covered);
    while (big) {
      const int j = __ffs(big) - 1;
      big &= big - 1;
      const long long e0 = __shfl_sync(0xFFFFFFFFu, b0, j);
      const long long e1 = __shfl_sync(0xFFFFFFFFu, b1, j);
      const long long es = __shfl_sync(0xFFFFFFFFu, e_big, j);
      uint32_t a[WORDS];
#pragma unroll
      for (int k = 0; k < WORDS; k++) a[k] = __shfl_sync(0xFFFFFFFFu, acc[k], j);
      // a warp scans at most hub_t neighbours; the rest of a hub that is
      // still missing frontier bits is deferred to bu_defer_phase
      // (the limit counts from the list's start, as bu_defer_phase does)
      const long long e_lim = (e1 - e0 > p.hub_t) ? e0 + p.hub_t : e1;
      bool miss = true;
      for (long long e = es; e < e_lim; e += 32) {
        uint32_t x[WORDS];
#pragma unroll
        for (int k = 0; k < WORDS; k++) x[k] = 0;
        if (e + lane < e_lim) {
          const int32_t u = p.col[e + lane];
          if (!filt || in_front<RO>(front, u))
            ld_nbr<WORDS, HK, NC>(gb.last, s_hub, hk, u, x);
        }
        miss = false;
#pragma unroll
        for (int k = 0; k < WORDS; k++) {
          a[k] |= __reduce_or_sync(0xFFFFFFFFu, x[k]);
          miss |= (fm[k] & ~a[k]) != 0u;
        }
        if (!miss) break;
      }
      const bool defer = miss && e_lim < e1;
      if (defer && lane == 0) {
        const int nch = (int)((e1 - e_lim + kHubChunk - 1) / kHubChunk);
        const int base0 = atomicAdd(hq_cnt, nch);
        for (int c = 0; c < nch; c++) gb.hq[base0 + c] = make_int2((int)(base + j), c);
      }
      if (lane == j) {
#pragma unroll
        for (int k = 0; k < WORDS; k++) acc[k] = a[k];
        deferred = defer;
      }
    }
    bool ch = false;
#pragma unroll
    for (int k = 0; k < WORDS; k++) ch |= acc[k] != l[k];
    ch = ch && need;
    uint32_t nb[WORDS];
#pragma unroll
    for (int k = 0; k < WORDS; k++) nb[k] = 0u;
    if constexpr (!FUSED) {
      if (ch) st_status<WORDS>(gb.curr + (size_t)v * WORDS, acc);
    } else if (valid) {
      st_status<WORDS>(gb.curr + (size_t)v * WORDS, acc);  // every vertex: curr = new status
      const bool epi = ch && !deferred;  // deferred hubs: bu_hub_epilogue
      uint32_t pop = 0;
      bool comp = true;
#pragma unroll
      for (int k = 0; k < WORDS; k++) {
        nb[k] = epi ? (acc[k] & ~l[k]) : 0u;
        pop += __popc(nb[k]);
        comp = comp && acc[k] == full[k];
      }
      if (epi) {
        const uint32_t deg = (uint32_t)(b1 - b0);
        f_cnt += 1;
        f_mf += deg;
        f_teps += (unsigned long long)deg * pop;
        if (comp) f_cdeg += deg;
        if (!depth_ok) range = true;
      }
      uint32_t* q0 = gb.planes + (size_t)v * WORDS;
      if (first_plane) {
        // level 2^b is the first to use plane b: write it whole (0 where no bit is new)
        st_status<WORDS>(q0 + (size_t)pb * p.plane_stride, nb);
      } else if (epi && depth_ok) {
        unsigned rest = (unsigned)level;
        while (rest) {
          const int b0p = __ffs(rest) - 1;
          rest &= rest - 1;
          uint32_t* qa = q0 + (size_t)b0p * p.plane_stride;
          uint32_t xa[WORDS];
          ld_status<WORDS>(qa, xa);
#pragma unroll
          for (int k = 0; k < WORDS; k++) xa[k] |= nb[k];
          st_status<WORDS>(qa, xa);
        }
      }
      ch = epi;
    }
    if constexpr (FUSED) {
#pragma unroll
      for (int k = 0; k < WORDS; k++) {
        const uint32_t r = __reduce_or_sync(0xFFFFFFFFu, nb[k]);
        if (lane == 0 && r) atomicOr(&s_fm[k], r);
      }
    }
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, ch);
    if (lane == 0 && bal) atomicOr(out + (base >> 5), bal);
  }
  if constexpr (FUSED) {
    if (range) par->range_err = 1;
    cta_add_u64(&par->changed, f_cnt);
    cta_add_u64(&par->mf, f_mf);
    cta_add_u64(&par->cdeg, f_cdeg);
    cta_add_u64(&par->teps, f_teps);
    __syncthreads();
    if (threadIdx.x < WORDS && s_fm[threadIdx.x]) atomicOr(&par->fmask[threadIdx.x], s_fm[threadIdx.x]);
  }
}

// FUSED bottom-up, after bu_defer_phase: the inspect work of the hubs whose
// scan was deferred (one entry per hub: chunk 0), from their final status
// in `curr` and the previous one in `last`; and the level+1 bitmap cleared
// for the next expand (what inspect_phase does on other levels).
// keep_next: a sparse-source push follows and still reads the level-(L-1)
// bitmap, which is the same buffer as level L+1's (level parity); the push
// kernel's successor clears it then.
template <int WORDS>
__device__ void bu_hub_epilogue(const Params& p, const GroupBufs& gb, Par* par, int n_b,
                                int level, bool depth_ok, const Team& t, bool keep_next = false) {
  if (!keep_next) zero_words(chg_at(gb, p, level + 1), p.chg_stride, t);
  uint32_t full[WORDS], fm[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) {
    full[k] = full_word(n_b, k);
    fm[k] = 0;
  }
  unsigned long long mf = 0, cnt = 0, cdeg = 0, teps = 0;
  uint32_t* out = chg_at(gb, p, level);
  const int n = __ldcg(&par->hq_cnt);
  for (long long i = t.tid; i < n; i += t.nthreads) {
    const int2 hc = gb.hq[i];
    if (hc.y != 0) continue;
    const long long v = hc.x;
    uint32_t c[WORDS], l[WORDS], nb[WORDS];
    ld_status<WORDS>(gb.curr + (size_t)v * WORDS, c);
    ld_status<WORDS>(gb.last + (size_t)v * WORDS, l);
    bool any = false, comp = true;
    uint32_t pop = 0;
#pragma unroll
    for (int k = 0; k < WORDS; k++) {
      nb[k] = c[k] & ~l[k];
      any |= nb[k] != 0u;
      comp = comp && c[k] == full[k];
      pop += __popc(nb[k]);
      fm[k] |= nb[k];
    }
    if (!any) continue;
    const unsigned long long deg = (unsigned long long)(p.beg[v + 1] - p.beg[v]);
    cnt += 1;
    mf += deg;
    teps += deg * pop;
    if (comp) cdeg += deg;
    if (!depth_ok) par->range_err = 1;
    atomicOr(out + (v >> 5), 1u << (v & 31));
    if (depth_ok) {
      unsigned rest = (unsigned)level;
      while (rest) {
        const int b = __ffs(rest) - 1;
        rest &= rest - 1;
        uint32_t* q = gb.planes + (size_t)b * p.plane_stride + (size_t)v * WORDS;
        uint32_t x[WORDS];
        ld_status<WORDS>(q, x);
#pragma unroll
        for (int k = 0; k < WORDS; k++) x[k] |= nb[k];
        st_status<WORDS>(q, x);
      }
    }
  }
  cta_add_u64(&par->changed, cnt);
  cta_add_u64(&par->mf, mf);
  cta_add_u64(&par->cdeg, cdeg);
  cta_add_u64(&par->teps, teps);
#pragma unroll
  for (int k = 0; k < WORDS; k++) cta_or_u32(&par->fmask[k], fm[k]);
}

// ---------------------------------------------------------------------------
// Sparse sources (device loop, a bottom-up level L that follows a top-down
// level).  A bottom-up scan stops once a vertex holds every bit of the
// previous frontier.  A source whose level-(L-1) frontier holds only a
// handful of vertices (it started far from the hubs) has not reached most
// vertices yet, so with its bit in the mask almost no vertex can stop early
// and most scan their whole neighbour lists.  So at such a level:
//   sparse_count_phase  counts every source's level-(L-1) frontier;
//   (k_dl_sparse_decide) the sources below 1/sparse_div of the average go
//                       into LoopState::smask, and the bottom-up pass's
//                       early exit ignores their bits;
//   push_queue_phase /  after the pass (and its deferred hubs), those bits
//   push_run_phase      are delivered exactly as a top-down level would:
//                       every vertex that gained a sparse bit at level L-1
//                       pushes it to all its neighbours -- a warp per small
//                       vertex, 2048-edge chunks spread over all CTAs for a
//                       vertex above the large-queue threshold (a hub can be
//                       in a sparse source's frontier).
// Each push takes its new bits from the atomic OR's old value, so the
// level's edge count, its depth planes (OR reductions: other pushes may hit
// the same vertex) and fmask stay exact; the changed count, the frontier-edge
// sum and the completed-degree sum (which only steer the direction choice)
// count a vertex when a push is the first change to it at this level.  The
// result is the BFS of every source: a bit reaches each vertex at its
// distance either way.
// ---------------------------------------------------------------------------
// The bits of `mask` that v gained at level L-1 (`last` holds the statuses
// after level L-1; a bit's depth is L-1 when the planes spell L-1: the planes
// of bits already in `last` no longer change).
template <int WORDS>
__device__ __forceinline__ bool gained_at(const Params& p, const GroupBufs& gb, long long v,
                                          int lp, const uint32_t (&mask)[WORDS],
                                          uint32_t (&P)[WORDS]) {
  ld_status<WORDS>(gb.last + (size_t)v * WORDS, P);
  bool has = false;
#pragma unroll
  for (int k = 0; k < WORDS; k++) {
    P[k] &= mask[k];
    has |= P[k] != 0u;
  }
  if (!has) return false;
  const int np = planes_for(lp);
  for (int b = 0; b < np; b++) {
    uint32_t x[WORDS];
    ld_status<WORDS>(gb.planes + (size_t)b * p.plane_stride + (size_t)v * WORDS, x);
    const bool one = (lp >> b) & 1;
#pragma unroll
    for (int k = 0; k < WORDS; k++) P[k] &= one ? x[k] : ~x[k];
  }
  has = false;
#pragma unroll
  for (int k = 0; k < WORDS; k++) has |= P[k] != 0u;
  return has;
}

template <int WORDS>
__device__ void sparse_count_phase(const Params& p, const GroupBufs& gb, Par* par, int level,
                                   const Team& t) {
  __shared__ uint32_t s_scnt[kMaxWords * 32];
  scnt_begin(s_scnt);
  uint32_t all[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) all[k] = 0xFFFFFFFFu;
  const uint32_t* front = chg_at(gb, p, level - 1);
  for (long long v = t.tid; v < p.V; v += t.nthreads) {
    if (!((__ldcg(front + (v >> 5)) >> (v & 31)) & 1u)) continue;
    uint32_t P[WORDS];
    if (!gained_at<WORDS>(p, gb, v, level - 1, all, P)) continue;
#pragma unroll
    for (int k = 0; k < WORDS; k++) {
      uint32_t r = P[k];
      while (r) {
        atomicAdd(&s_scnt[k * 32 + __ffs(r) - 1], 1u);
        r &= r - 1;
      }
    }
  }
  scnt_flush<WORDS>(s_scnt, par);
}

struct PushAcc {
  unsigned long long mf = 0, cnt = 0, cdeg = 0, teps = 0;
  uint32_t fm[kMaxWords] = {0, 0, 0, 0, 0, 0, 0, 0};
  bool range = false;
};

// One pushed edge: OR the bits P into u's status and account for the ones
// that were new (see above).
template <int WORDS>
__device__ __forceinline__ void push_edge(const Params& p, const GroupBufs& gb, uint32_t* out,
                                          int level, bool depth_ok, const uint32_t (&full)[WORDS],
                                          int32_t u, const uint32_t (&P)[WORDS], PushAcc& acc) {
  uint32_t s[WORDS];
  ld_status<WORDS>(gb.curr + (size_t)u * WORDS, s);
  bool need = false;
#pragma unroll
  for (int k = 0; k < WORDS; k++) need |= (P[k] & ~s[k]) != 0u;
  if (!need) return;
  uint32_t old[WORDS], nb[WORDS];
  if constexpr (WORDS == 1) {
    old[0] = atomicOr(gb.curr + u, P[0]);
  } else {
    unsigned long long* q = reinterpret_cast<unsigned long long*>(gb.curr + (size_t)u * WORDS);
#pragma unroll
    for (int k = 0; k < WORDS / 2; k++) {
      const unsigned long long pw = ((unsigned long long)P[2 * k + 1] << 32) | P[2 * k];
      const unsigned long long o =
          pw ? atomicOr(q + k, pw) : (((unsigned long long)s[2 * k + 1] << 32) | s[2 * k]);
      old[2 * k] = (uint32_t)o;
      old[2 * k + 1] = (uint32_t)(o >> 32);
    }
  }
  bool any = false;
  uint32_t pop = 0;
#pragma unroll
  for (int k = 0; k < WORDS; k++) {
    nb[k] = P[k] & ~old[k];
    any |= nb[k] != 0u;
    pop += __popc(nb[k]);
  }
  if (!any) return;
  uint32_t l[WORDS];
  ld_status<WORDS>(gb.last + (size_t)u * WORDS, l);
  bool first = true, was_full = true, now_full = true;
#pragma unroll
  for (int k = 0; k < WORDS; k++) {
    first = first && (old[k] & ~l[k]) == 0u;
    was_full = was_full && old[k] == full[k];
    now_full = now_full && (old[k] | nb[k]) == full[k];
    acc.fm[k] |= nb[k];
  }
  const unsigned long long deg = (unsigned long long)(p.beg[u + 1] - p.beg[u]);
  acc.teps += deg * pop;
  if (first) {
    acc.cnt += 1;
    acc.mf += deg;
  }
  if (now_full && !was_full) acc.cdeg += deg;
  red_or_u32(out + (u >> 5), 1u << (u & 31));
  if (!depth_ok) {
    acc.range = true;
    return;
  }
  unsigned rest = (unsigned)level;
  while (rest) {
    const int b = __ffs(rest) - 1;
    rest &= rest - 1;
    uint32_t* q = gb.planes + (size_t)b * p.plane_stride + (size_t)u * WORDS;
#pragma unroll
    for (int k = 0; k < WORDS; k++)
      if (nb[k]) red_or_u32(q + k, nb[k]);
  }
}

template <int WORDS>
__device__ __forceinline__ void push_acc_flush(const PushAcc& acc, Par* par) {
  if (acc.range) par->range_err = 1;
  cta_add_u64(&par->changed, acc.cnt);
  cta_add_u64(&par->mf, acc.mf);
  cta_add_u64(&par->cdeg, acc.cdeg);
  cta_add_u64(&par->teps, acc.teps);
#pragma unroll
  for (int k = 0; k < WORDS; k++) cta_or_u32(&par->fmask[k], acc.fm[k]);
}

template <int WORDS>
__device__ void push_queue_phase(const Params& p, const GroupBufs& gb, Par* par, int n_b,
                                 int level, bool depth_ok, const uint32_t* smask,
                                 const Team& t) {
  uint32_t sm[WORDS], full[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) {
    sm[k] = __ldcg(smask + k);
    full[k] = full_word(n_b, k);
  }
  const uint32_t* front = chg_at(gb, p, level - 1);
  uint32_t* out = chg_at(gb, p, level);
  PushAcc acc;
  const int lane = t.lane;
  for (long long w = t.warp; w < p.nchg; w += t.nwarps) {
    const uint32_t bits = __ldcg(front + w);
    if (!bits) continue;  // uniform
    const long long v0 = w * 32 + lane;
    uint32_t P[WORDS];
    bool has = false;
#pragma unroll
    for (int k = 0; k < WORDS; k++) P[k] = 0u;
    long long deg = 0;
    if ((bits >> lane) & 1u) {
      has = gained_at<WORDS>(p, gb, v0, level - 1, sm, P);
      if (has) deg = p.beg[v0 + 1] - p.beg[v0];
    }
    // a vertex above the large-queue threshold goes to the chunk queue
    if (has && deg > p.lrg) {
      const int nch = (int)((deg + p.chunk - 1) / p.chunk);
      const int base0 = atomicAdd(&par->pq_cnt, nch);
      for (int c = 0; c < nch; c++) gb.ql[base0 + c] = make_int2((int)v0, c);
      has = false;
    }
    uint32_t pushers = __ballot_sync(0xFFFFFFFFu, has);
    while (pushers) {
      const int j = __ffs(pushers) - 1;
      pushers &= pushers - 1;
      uint32_t Pj[WORDS];
#pragma unroll
      for (int k = 0; k < WORDS; k++) Pj[k] = __shfl_sync(0xFFFFFFFFu, P[k], j);
      const long long v = w * 32 + j;
      const long long e1 = p.beg[v + 1];
      for (long long e = p.beg[v] + lane; e < e1; e += 32)
        push_edge<WORDS>(p, gb, out, level, depth_ok, full, __ldg(p.col + e), Pj, acc);
    }
  }
  push_acc_flush<WORDS>(acc, par);
}

template <int WORDS>
__device__ void push_run_phase(const Params& p, const GroupBufs& gb, Par* par, int n_b,
                               int level, bool depth_ok, const uint32_t* smask, const Team& t) {
  uint32_t sm[WORDS], full[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) {
    sm[k] = __ldcg(smask + k);
    full[k] = full_word(n_b, k);
  }
  uint32_t* out = chg_at(gb, p, level);
  PushAcc acc;
  const int n = __ldcg(&par->pq_cnt);
  for (int c = t.block; c < n; c += t.nblocks) {
    const int2 d = gb.ql[c];
    uint32_t P[WORDS];
    (void)gained_at<WORDS>(p, gb, d.x, level - 1, sm, P);
    const long long e_end = p.beg[d.x + 1];
    const long long b0 = p.beg[d.x] + (long long)d.y * p.chunk;
    const long long b1 = min(e_end, b0 + (long long)p.chunk);
    for (long long e = b0 + threadIdx.x; e < b1; e += blockDim.x)
      push_edge<WORDS>(p, gb, out, level, depth_ok, full, __ldg(p.col + e), P, acc);
  }
  push_acc_flush<WORDS>(acc, par);
}

// ---------------------------------------------------------------------------
// Phase: write one batch's depths from the bit-planes.  Depth of (v, s) =
// the number whose bit b is bit s of plane b, INFTY (255 / 65535,
// comm.h:120) when bit s of the final status is clear.  Every output byte is
// written once, in whole sectors.
//   source-major: rows out_row[...] of V depths;
//   vertex-major: the batch block [V][n_b] (depth_merge, inspector.cuh:48).
// ---------------------------------------------------------------------------

// 4 bits -> the low bit of 4 bytes (bit i -> bit 8i).
__device__ __forceinline__ uint32_t nib_to_bytes(uint32_t nib) {
  return (nib * 0x00204081u) & 0x01010101u;
}
// 8 bits -> every 4th bit of a word (bit r -> bit 4r).
__device__ __forceinline__ uint32_t spread8(uint32_t b8) {
  uint32_t x = b8 & 0xFFu;
  x = (x | (x << 12)) & 0x000F000Fu;
  x = (x | (x << 6)) & 0x03030303u;
  x = (x | (x << 3)) & 0x11111111u;
  return x;
}
// Interleave the words of 4 vertices: bit 4r+i of y[q] = bit 8q+r of x[i],
// so nibble r of y[q] holds source 8q+r for the 4 vertices.
__device__ __forceinline__ void interleave4(const uint32_t (&x)[4], uint32_t (&y)[4]) {
#pragma unroll
  for (int q = 0; q < 4; q++)
    y[q] = spread8(x[0] >> (8 * q)) | (spread8(x[1] >> (8 * q)) << 1) |
           (spread8(x[2] >> (8 * q)) << 2) | (spread8(x[3] >> (8 * q)) << 3);
}

// In-register transpose of a 32 x 32 bit matrix, LSB-first: afterwards
// bit r of A[j] is what bit j of A[r] was.  Five rounds of block swaps
// (16, 8, 4, 2, 1), 16 masked delta swaps each; rows that are zero at
// compile time fold away.
__device__ __forceinline__ void transpose32(uint32_t (&A)[32]) {
#pragma unroll
  for (int lv = 0; lv < 5; lv++) {
    const int j = 16 >> lv;
    const uint32_t m = lv == 0 ? 0x0000FFFFu : lv == 1 ? 0x00FF00FFu : lv == 2 ? 0x0F0F0F0Fu
                     : lv == 3 ? 0x33333333u : 0x55555555u;
#pragma unroll
    for (int r = 0; r < 32; r++) {
      if (r & j) continue;
      const uint32_t t = ((A[r] >> j) ^ A[r + j]) & m;
      A[r + j] ^= t;
      A[r] ^= t << j;
    }
  }
}

#ifndef IBFS_OUT_PRMT
#define IBFS_OUT_PRMT 1
#endif
#ifndef IBFS_OUT_FASTST
#define IBFS_OUT_FASTST 1
#endif
#ifndef IBFS_OUT_STCS
#define IBFS_OUT_STCS 1
#endif

// A 4-byte piece of a depth row.  The rows are written once and not read
// again on the device: with IBFS_OUT_STCS they are streaming stores (evict
// first), so that they do not push the gathered statuses and planes out of
// L2.
__device__ __forceinline__ void st_row4(uint8_t* a, uint32_t x) {
#if IBFS_OUT_STCS
  __stcs(reinterpret_cast<unsigned int*>(a), x);
#else
  *reinterpret_cast<uint32_t*>(a) = x;
#endif
}

// The same transpose with its first two rounds (whole 16- and 8-bit blocks)
// as byte permutes, two per row pair instead of a five-instruction masked
// delta swap.  Z: bit r set = row r is zero on entry (a compile-time
// constant), so that pairs of zero rows are skipped; the rounds commute, so
// the order of the five does not matter.
template <uint32_t Z>
__device__ __forceinline__ void transpose32_z(uint32_t (&A)[32]) {
#pragma unroll
  for (int r = 0; r < 16; r++) {
    if (((Z >> r) & 1u) && ((Z >> (r + 16)) & 1u)) continue;
    const uint32_t a = A[r], b = A[r + 16];
    A[r] = __byte_perm(a, b, 0x5410);       // low halves
    A[r + 16] = __byte_perm(a, b, 0x7632);  // high halves
  }
  constexpr uint32_t Z1 = (Z & (Z >> 16) & 0xFFFFu) * 0x10001u;
#pragma unroll
  for (int r = 0; r < 32; r++) {
    if (r & 8) continue;
    if (((Z1 >> r) & 1u) && ((Z1 >> (r + 8)) & 1u)) continue;
    const uint32_t a = A[r], b = A[r + 8];
    A[r] = __byte_perm(a, b, 0x6240);      // bytes 0 and 2 of both
    A[r + 8] = __byte_perm(a, b, 0x7351);  // bytes 1 and 3 of both
  }
#pragma unroll
  for (int lv = 2; lv < 5; lv++) {
    const int j = 16 >> lv;
    const uint32_t m = lv == 2 ? 0x0F0F0F0Fu : lv == 3 ? 0x33333333u : 0x55555555u;
#pragma unroll
    for (int r = 0; r < 32; r++) {
      if (r & j) continue;
      // m << j == ~m: each row keeps its own half and takes the partner's
      // other half, a shift and a three-input select each
      const uint32_t a = A[r], b = A[r + j];
      A[r] = (a & m) | ((b << j) & ~m);
      A[r + j] = ((a >> j) & m) | (b & ~m);
    }
  }
}

// Rows known zero in output_sm_u8's matrix: 8i + b for NP <= b <= 6.
template <int NP>
__host__ __device__ constexpr uint32_t out_zero_rows() {
  uint32_t z = 0u;
  for (int i = 0; i < 4; i++)
    for (int b = NP; b < 7; b++) z |= 1u << (8 * i + b);
  return z;
}

// Source-major, one-byte depths, NP (<= 8) planes known at compile time:
// lane = 4 consecutive vertices, one 4-byte store per source row.  The
// depth byte of (vertex i, source s) has bit b = bit s of plane b of vertex
// i, or is 0xFF when bit s of the final status is clear: the 32 words
// A[8i + b] form a 32 x 32 bit matrix whose transpose is exactly the 32
// output words, one per source, byte i = vertex i.  With NP <= 7 (depths
// below 128) A[8i + b] = plane_b(i) for b < NP, 0 up to b = 6 and ~status(i)
// for b = 7, and one sign-replicating byte permute per word turns bit 7
// into 0xFF; the zero rows are compile-time constants that fold out of the
// transpose.  With NP = 8, A[8i + b] = plane_b(i) | ~status(i).
template <int WORDS, int NP>
__device__ void output_sm_u8(const Params& p, const GroupBufs& gb, const int32_t* rows, int n_b,
                             const Team& t) {
  static_assert(NP <= 8, "one-byte depths use at most 8 planes");
  const int lane = t.lane;
  for (long long base = t.warp * 128; base < p.V; base += t.nwarps * 128) {
    const long long v0 = base + 4 * lane;
    const bool full4 = p.vec_sm >= 4 && v0 + 3 < p.V;
    // rows are in the caller's vertex order; statuses in the graph's
    uint32_t vis[4];
#pragma unroll
    for (int i = 0; i < 4; i++)
      vis[i] = v0 + i < p.V ? (uint32_t)(p.vmap ? p.vmap[v0 + i] : v0 + i) : 0u;
#pragma unroll 1
    for (int k = 0; k < WORDS && k * 32 < n_b; k++) {
      uint32_t A[32];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const bool in = v0 + i < p.V;
        const size_t vi = vis[i];
        // a vertex from v_reach on is reached only as a source, at depth 0:
        // its plane words are zeros (every plane was first written whole
        // during the batch), so they are not gathered
        const bool edged = in && (long long)vi < p.v_reach;
        const uint32_t nst = in ? ~gb.last[vi * WORDS + k] : 0xFFFFFFFFu;
        if constexpr (NP <= 7) {
          // planes in rows 0..NP-1, zero rows up to 6 (folded away by the
          // compiler), the unreached flag in row 7
#pragma unroll
          for (int b = 0; b < 7; b++)
            A[8 * i + b] = (b < NP && edged)
                               ? gb.planes[(size_t)b * p.plane_stride + vi * WORDS + k]
                               : 0u;
          A[8 * i + 7] = nst;
        } else {
#pragma unroll
          for (int b = 0; b < 8; b++) {
            uint32_t x = 0u;
            if (edged) x = gb.planes[(size_t)b * p.plane_stride + vi * WORDS + k];
            A[8 * i + b] = x | nst;
          }
        }
      }
#if IBFS_OUT_PRMT
      transpose32_z<out_zero_rows<NP>()>(A);
#else
      transpose32(A);
#endif
      if constexpr (NP <= 7) {
        // byte i = depth (< 128) with bit 7 = unreached: widen bit 7 to the
        // whole byte (prmt in sign-replicating mode), 0xFF = INFTY
#pragma unroll
        for (int j = 0; j < 32; j++) {
          uint32_t m;
          asm("prmt.b32 %0, %1, 0, 0xBA98;" : "=r"(m) : "r"(A[j]));
          A[j] |= m;
        }
      }
      const int js = min(32, n_b - k * 32);
#if IBFS_OUT_FASTST
      if (full4 && js == 32) {
        // the common case: 32 whole rows, 4 in-range vertices per lane
#pragma unroll
        for (int j = 0; j < 32; j++)
          st_row4(p.out + (size_t)rows[k * 32 + j] * (size_t)p.V + v0, A[j]);
        continue;
      }
#endif
#pragma unroll
      for (int j = 0; j < 32; j++) {
        if (j < js) {
          uint8_t* row = p.out + (size_t)rows[k * 32 + j] * (size_t)p.V;
          if (full4) {
            st_row4(row + v0, A[j]);
          } else {
            for (int i = 0; i < 4; i++)
              if (v0 + i < p.V) row[v0 + i] = (uint8_t)(A[j] >> (8 * i));
          }
        }
      }
    }
  }
}

// Vertex-major, one-byte depths: lane = vertex, 4 sources per store.
template <int WORDS, int NP>
__device__ void output_vm_u8(const Params& p, const GroupBufs& gb, uint8_t* depth_vm, int n_b,
                             const Team& t) {
  const bool vec = p.vec_out && (n_b % 4 == 0);
  for (long long v = t.tid; v < p.V; v += t.nthreads) {
    uint8_t* row = depth_vm + (size_t)v * n_b;
    const size_t vi = (size_t)(p.vmap ? p.vmap[v] : v);
#pragma unroll 1
    for (int k = 0; k < WORDS && k * 32 < n_b; k++) {
      const uint32_t st = gb.last[vi * WORDS + k];
      uint32_t pw[NP > 0 ? NP : 1];
#pragma unroll
      for (int b = 0; b < NP; b++) pw[b] = gb.planes[(size_t)b * p.plane_stride + vi * WORDS + k];
      const int js = min(32, n_b - k * 32);
#pragma unroll
      for (int j4 = 0; j4 < 8; j4++) {
        if (j4 * 4 < js) {
          uint32_t w = nib_to_bytes(~(st >> (4 * j4)) & 0xFu) * 0xFFu;
#pragma unroll
          for (int b = 0; b < NP; b++) w |= nib_to_bytes((pw[b] >> (4 * j4)) & 0xFu) << b;
          if (vec && j4 * 4 + 4 <= js) {
            *reinterpret_cast<uint32_t*>(row + k * 32 + j4 * 4) = w;
          } else {
            for (int i = 0; i < 4 && j4 * 4 + i < js; i++) row[k * 32 + j4 * 4 + i] = (uint8_t)(w >> (8 * i));
          }
        }
      }
    }
  }
}

// Any depth width and plane count (two-byte depths): lane = vertex.
template <int WORDS>
__device__ void output_generic(const Params& p, const GroupBufs& gb, uint8_t* depth_vm,
                               const int32_t* rows, int n_b, int P, const Team& t) {
  const uint32_t inf = p.db == 1 ? 0xFFu : 0xFFFFu;
  for (long long v = t.tid; v < p.V; v += t.nthreads) {
    const size_t vi = (size_t)(p.vmap ? p.vmap[v] : v);
#pragma unroll 1
    for (int k = 0; k < WORDS && k * 32 < n_b; k++) {
      const uint32_t st = gb.last[vi * WORDS + k];
      const int js = min(32, n_b - k * 32);
      for (int j = 0; j < js; j++) {
        uint32_t d = inf;
        if ((st >> j) & 1u) {
          d = 0;
          for (int b = 0; b < P; b++)
            d |= ((gb.planes[(size_t)b * p.plane_stride + vi * WORDS + k] >> j) & 1u) << b;
        }
        uint8_t* dst = p.layout == 0
                           ? p.out + ((size_t)rows[k * 32 + j] * (size_t)p.V + (size_t)v) * p.db
                           : depth_vm + ((size_t)v * n_b + k * 32 + j) * p.db;
        if (p.db == 1) *dst = (uint8_t)d;
        else *reinterpret_cast<uint16_t*>(dst) = (uint16_t)d;
      }
    }
  }
}

template <int WORDS, int NP>
__device__ __forceinline__ void output_u8(const Params& p, const GroupBufs& gb, uint8_t* depth_vm,
                                          const int32_t* rows, int n_b, const Team& t) {
  if (p.layout == 0) output_sm_u8<WORDS, NP>(p, gb, rows, n_b, t);
  else output_vm_u8<WORDS, NP>(p, gb, depth_vm, n_b, t);
}

template <int WORDS>
__device__ void output_phase(const Params& p, const GroupBufs& gb, uint8_t* depth_vm,
                             const int32_t* rows, int n_b, int max_level, const Team& t) {
  const int P = planes_for(max_level);
  if (p.db == 1) {
    switch (P) {
      case 0: output_u8<WORDS, 0>(p, gb, depth_vm, rows, n_b, t); return;
      case 1: output_u8<WORDS, 1>(p, gb, depth_vm, rows, n_b, t); return;
      case 2: output_u8<WORDS, 2>(p, gb, depth_vm, rows, n_b, t); return;
      case 3: output_u8<WORDS, 3>(p, gb, depth_vm, rows, n_b, t); return;
      case 4: output_u8<WORDS, 4>(p, gb, depth_vm, rows, n_b, t); return;
      case 5: output_u8<WORDS, 5>(p, gb, depth_vm, rows, n_b, t); return;
      case 6: output_u8<WORDS, 6>(p, gb, depth_vm, rows, n_b, t); return;
      case 7: output_u8<WORDS, 7>(p, gb, depth_vm, rows, n_b, t); return;
      case 8: output_u8<WORDS, 8>(p, gb, depth_vm, rows, n_b, t); return;
      default: break;
    }
  }
  output_generic<WORDS>(p, gb, depth_vm, rows, n_b, P, t);
}

}  // namespace ibfs
