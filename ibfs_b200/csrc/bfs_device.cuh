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
//            bitmap `chg` (V/8 bytes, L2 resident);
//   inspect  walks the bitmap only: new bits = curr & ~last, writes the
//            depth bytes of the new bits, last = curr, and accumulates the
//            direction-switch counters.  Replaces the O(V) count/scan/gather
//            passes of inspector.cuh:63-525 and scan.cuh:455-655;
//   qbuild   (only before a top-down level) turns the bitmap into the
//            small/medium/large queues with warp-ballot compaction
//            (replaces td_frontier_count/td_frontier_gather).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ibfs {

constexpr int kDirTD = 0;
constexpr int kDirBU = 1;
constexpr int kMaxWords = 8;  // W = 256

// Per-level counters, double-buffered by level parity.
struct Par {
  unsigned long long changed;  // vertices whose status changed
  unsigned long long mf;       // sum of their degrees (frontier edges)
  unsigned long long cdeg;     // sum of degrees of vertices that became complete
  unsigned long long teps;     // sum over new (v, s) pairs of deg(v)
  uint32_t fmask[kMaxWords];   // OR of all new bits (sources still expanding)
  int32_t range_err;           // a level did not fit the depth type
  int32_t pad[3];
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
};

struct GroupBufs {
  uint32_t* last;
  uint32_t* curr;
  uint32_t* chg;
  int32_t* qs;
  int32_t* qm;
  int2* ql;
  Ctl* ctl;
  uint8_t* stage;  // vertex-major depth staging [V][C] (db bytes each)
};

struct Params {
  const int64_t* beg;
  const int32_t* col;
  int64_t V, E, nchg;
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
  int vec_out;  // output rows allow 4-vertex vector stores (V % 4 == 0, aligned base)
};

// A team is the set of threads that share one batch: the whole grid in the
// plain schedule, the CTAs of one group in the persistent kernel.
struct Team {
  int block, nblocks;  // CTA index inside the team, team size in CTAs
  long long tid, nthreads;
  long long warp, nwarps;
  int lane;
};

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
__device__ __forceinline__ uint32_t full_word(int n, int k) {
  const int lo = k * 32;
  if (n >= lo + 32) return 0xFFFFFFFFu;
  if (n <= lo) return 0u;
  return (1u << (n - lo)) - 1u;
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

__device__ __forceinline__ void store_depth(uint8_t* row, int idx, int db, int level) {
  if (db == 1) row[idx] = (uint8_t)level;
  else reinterpret_cast<uint16_t*>(row)[idx] = (uint16_t)level;
}

// ---------------------------------------------------------------------------
// Direction choice for the next level (host and device use the same rule).
//   fixed (switch_level >= 0): top-down while level <= switch_level, then
//     bottom-up -- the reference's CLI switch level (expander.cuh:687-723);
//   alpha/beta (Beamer et al., SC'12): top-down -> bottom-up when the
//     frontier's edges exceed unexplored_edges/alpha; bottom-up -> top-down
//     when the frontier holds fewer than V/beta vertices.
// ---------------------------------------------------------------------------
__host__ __device__ inline int choose_dir(int next_level, int prev_dir,
                                          int switch_level, float alpha,
                                          float beta, unsigned long long changed,
                                          unsigned long long mf,
                                          unsigned long long m_u, long long V) {
  if (switch_level >= 0) return next_level <= switch_level ? kDirTD : kDirBU;
  if (prev_dir == kDirTD)
    return ((double)mf * (double)alpha > (double)m_u) ? kDirBU : kDirTD;
  return ((double)changed * (double)beta < (double)V) ? kDirTD : kDirBU;
}

// ---------------------------------------------------------------------------
// Phase: seed the sources of one batch (curr bits + changed bits).
// ---------------------------------------------------------------------------
template <int WORDS>
__device__ void seed_phase(const Params& p, const GroupBufs& gb,
                           const int32_t* src_b, int n_b, const Team& t) {
  for (long long i = t.tid; i < n_b; i += t.nthreads) {
    const int32_t v = src_b[i];
    atomicOr(gb.curr + (size_t)v * WORDS + (i >> 5), 1u << (i & 31));
    atomicOr(gb.chg + (v >> 5), 1u << (v & 31));
  }
}

// ---------------------------------------------------------------------------
// Phase: inspect level L (reads chg, fixes last, writes depth, counters).
// ---------------------------------------------------------------------------
template <int WORDS>
__device__ void inspect_phase(const Params& p, const GroupBufs& gb, Par* par,
                              uint8_t* depth, int n_b, int level, bool depth_ok,
                              const Team& t) {
  uint32_t full[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) full[k] = full_word(n_b, k);
  unsigned long long mf = 0, cnt = 0, cdeg = 0, teps = 0;
  uint32_t fm[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) fm[k] = 0;
  const int lane = t.lane;
  const size_t row_bytes = (size_t)n_b * p.db;
  for (long long w = t.warp; w < p.nchg; w += t.nwarps) {
    const uint32_t bits = __ldcg(gb.chg + w);
    if (!bits) continue;
    const long long v = w * 32 + lane;
    const bool mine = (bits >> lane) & 1u;
    uint32_t nb[WORDS];
#pragma unroll
    for (int k = 0; k < WORDS; k++) nb[k] = 0;
    if (mine) {
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
    }
    if (!depth_ok) continue;
    // Depth bytes: the warp writes one changed vertex's row at a time; lane
    // l owns sources l, l+32, ... so every store instruction is one
    // coalesced (byte-masked) 32-source segment of the row.
    uint32_t rem = bits;
    while (rem) {
      const int j = __ffs(rem) - 1;
      rem &= rem - 1;
      uint8_t* row = depth + (size_t)(w * 32 + j) * row_bytes;
#pragma unroll
      for (int k = 0; k < WORDS; k++) {
        const uint32_t x = __shfl_sync(0xFFFFFFFFu, nb[k], j);
        if ((x >> lane) & 1u) store_depth(row, k * 32 + lane, p.db, level);
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

// ---------------------------------------------------------------------------
// Phase: build the joint frontier queues for a top-down level from chg
// (warp-ballot compaction, degree classes as td_inspect, inspector.cuh:
// 534-626: deg < sml -> small, deg > lrg -> large, else medium, deg 0
// dropped).  Large vertices are cut into chunks of p.chunk edges.  Clears
// the bitmap words it reads.
// ---------------------------------------------------------------------------
__device__ inline void qbuild_phase(const Params& p, const GroupBufs& gb,
                                    int32_t* qc, const Team& t) {
  const int lane = t.lane;
  const uint32_t lt = (1u << lane) - 1u;
  for (long long w = t.warp; w < p.nchg; w += t.nwarps) {
    const uint32_t bits = __ldcg(gb.chg + w);
    if (!bits) continue;
    const long long v = w * 32 + lane;
    const bool mine = (bits >> lane) & 1u;
    long long deg = 0;
    if (mine) deg = p.beg[v + 1] - p.beg[v];
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
    if (lane == 0) __stcg(gb.chg + w, 0u);
  }
}

// One top-down edge: push the frontier word P of v into neighbour u.
// The status read goes to L2 (ld.cg): it only filters atomics, a stale
// value has fewer bits and just costs one more atomic.
template <int WORDS>
__device__ __forceinline__ void td_push(const GroupBufs& gb, int32_t u,
                                        const uint32_t (&P)[WORDS]) {
  uint32_t s[WORDS];
  ld_status<WORDS>(gb.curr + (size_t)u * WORDS, s);
  bool need = false;
#pragma unroll
  for (int k = 0; k < WORDS; k++) need |= (P[k] & ~s[k]) != 0u;
  if (!need) return;
  bool changed = false;
  if constexpr (WORDS == 1) {
    const uint32_t old = atomicOr(gb.curr + u, P[0]);
    changed = (old & P[0]) != P[0];
  } else {
    unsigned long long* q = reinterpret_cast<unsigned long long*>(gb.curr + (size_t)u * WORDS);
#pragma unroll
    for (int k = 0; k < WORDS / 2; k++) {
      const uint32_t n0 = P[2 * k] & ~s[2 * k], n1 = P[2 * k + 1] & ~s[2 * k + 1];
      if (n0 | n1) {
        const unsigned long long pw = ((unsigned long long)P[2 * k + 1] << 32) | P[2 * k];
        const unsigned long long old = atomicOr(q + k, pw);
        changed |= (old & pw) != pw;
      }
    }
  }
  if (changed) {
    uint32_t* cw = gb.chg + (u >> 5);
    const uint32_t bit = 1u << (u & 31);
    if (!(__ldcg(cw) & bit)) atomicOr(cw, bit);
  }
}

// ---------------------------------------------------------------------------
// Phase: top-down expansion of level L over the three queues: one CTA per
// chunk of a large vertex (td_expand_cta, expander.cuh:276-331), one warp
// per medium vertex (td_expand_warp, expander.cuh:208-267), one thread per
// small vertex (td_expand_thd, expander.cuh:140-199).
// ---------------------------------------------------------------------------
template <int WORDS>
__device__ void td_phase(const Params& p, const GroupBufs& gb, const int32_t* qc,
                         const Team& t) {
  const int nS = __ldcg(qc + 0), nM = __ldcg(qc + 1), nL = __ldcg(qc + 2);
  for (int c = t.block; c < nL; c += t.nblocks) {
    const int2 d = gb.ql[c];
    const int32_t v = d.x;
    const long long e_end = p.beg[v + 1];
    const long long b0 = p.beg[v] + (long long)d.y * p.chunk;
    const long long b1 = min(e_end, b0 + (long long)p.chunk);
    uint32_t P[WORDS];
    ld_status<WORDS>(gb.last + (size_t)v * WORDS, P);
    for (long long e = b0 + threadIdx.x; e < b1; e += blockDim.x) td_push<WORDS>(gb, p.col[e], P);
  }
  for (long long i = t.warp; i < nM; i += t.nwarps) {
    const int32_t v = gb.qm[i];
    uint32_t P[WORDS];
    ld_status<WORDS>(gb.last + (size_t)v * WORDS, P);
    const long long b1 = p.beg[v + 1];
    for (long long e = p.beg[v] + t.lane; e < b1; e += 32) td_push<WORDS>(gb, p.col[e], P);
  }
  for (long long i = t.tid; i < nS; i += t.nthreads) {
    const int32_t v = gb.qs[i];
    uint32_t P[WORDS];
    ld_status<WORDS>(gb.last + (size_t)v * WORDS, P);
    const long long b1 = p.beg[v + 1];
    for (long long e = p.beg[v]; e < b1; e++) td_push<WORDS>(gb, p.col[e], P);
  }
}

// ---------------------------------------------------------------------------
// Phase: bottom-up level L.  Every vertex that still lacks a bit of the
// previous level's frontier mask ORs the `last` words of its neighbours and
// stops as soon as no frontier bit is missing (the early exit of
// expander.cu:298,348, generalised from "all bits" to "all bits any frontier
// vertex carries").  Low-degree vertices scan with one thread
// (sw_expand_thd, expander.cuh:431-489), the rest with the whole warp and a
// warp OR-reduction (sw_expand_warp, expander.cuh:341-422).
// ---------------------------------------------------------------------------
template <int WORDS>
__device__ void bu_phase(const Params& p, const GroupBufs& gb,
                         const uint32_t* fmask_g, const Team& t) {
  uint32_t fm[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) fm[k] = __ldcg(fmask_g + k);
  const int lane = t.lane;
  for (long long base = t.warp * 32; base < p.V; base += t.nwarps * 32) {
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
    if (small) {
      for (long long e = b0; e < b1; e++) {
        uint32_t x[WORDS];
        ld_status<WORDS>(gb.last + (size_t)p.col[e] * WORDS, x);
        bool miss = false;
#pragma unroll
        for (int k = 0; k < WORDS; k++) {
          acc[k] |= x[k];
          miss |= (fm[k] & ~acc[k]) != 0u;
        }
        if (!miss) break;
      }
    }
    uint32_t big = __ballot_sync(0xFFFFFFFFu, need && !small);
    while (big) {
      const int j = __ffs(big) - 1;
      big &= big - 1;
      const long long e0 = __shfl_sync(0xFFFFFFFFu, b0, j);
      const long long e1 = __shfl_sync(0xFFFFFFFFu, b1, j);
      uint32_t a[WORDS];
#pragma unroll
      for (int k = 0; k < WORDS; k++) a[k] = __shfl_sync(0xFFFFFFFFu, acc[k], j);
      for (long long e = e0; e < e1; e += 32) {
        uint32_t x[WORDS];
        if (e + lane < e1) {
          ld_status<WORDS>(gb.last + (size_t)p.col[e + lane] * WORDS, x);
        } else {
#pragma unroll
          for (int k = 0; k < WORDS; k++) x[k] = 0;
        }
        bool miss = false;
#pragma unroll
        for (int k = 0; k < WORDS; k++) {
          a[k] |= __reduce_or_sync(0xFFFFFFFFu, x[k]);
          miss |= (fm[k] & ~a[k]) != 0u;
        }
        if (!miss) break;
      }
      if (lane == j) {
#pragma unroll
        for (int k = 0; k < WORDS; k++) acc[k] = a[k];
      }
    }
    bool ch = false;
#pragma unroll
    for (int k = 0; k < WORDS; k++) ch |= acc[k] != l[k];
    ch = ch && need;
    if (ch) st_status<WORDS>(gb.curr + (size_t)v * WORDS, acc);
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, ch);
    if (lane == 0) __stcg(gb.chg + (base >> 5), bal);
  }
}

// ---------------------------------------------------------------------------
// Phase: finish one batch's depth output.  Depth bytes of (v, s) were
// written only at the level s reached v; unreached pairs are filled with
// INFTY here (255 / 65535, comm.h:120) from the final status bits, so no
// byte is written twice and there is no up-front fill pass.
//   vertex-major: in place in `stage` ([V][n_b]);
//   source-major: transpose `stage` into out rows out_row[k0 + j] through a
//   shared-memory tile of 128 vertices.
// ---------------------------------------------------------------------------
template <int WORDS>
__device__ void finish_vertex_major(const Params& p, const GroupBufs& gb,
                                    uint8_t* depth, int n_b, const Team& t) {
  const int lane = t.lane;
  const size_t row_bytes = (size_t)n_b * p.db;
  const uint16_t inf = p.db == 1 ? 0xFFu : 0xFFFFu;
  for (long long base = t.warp * 32; base < p.V; base += t.nwarps * 32) {
    const long long v = base + lane;
    uint32_t l[WORDS];
    bool incomplete = false;
    if (v < p.V) {
      ld_status<WORDS>(gb.last + (size_t)v * WORDS, l);
#pragma unroll
      for (int k = 0; k < WORDS; k++) incomplete |= (full_word(n_b, k) & ~l[k]) != 0u;
    }
    uint32_t todo = __ballot_sync(0xFFFFFFFFu, incomplete);
    while (todo) {
      const int j = __ffs(todo) - 1;
      todo &= todo - 1;
      uint8_t* row = depth + (size_t)(base + j) * row_bytes;
#pragma unroll
      for (int k = 0; k < WORDS; k++) {
        const uint32_t x = __shfl_sync(0xFFFFFFFFu, l[k], j);
        const int s = k * 32 + lane;
        if (s < n_b && !((x >> lane) & 1u)) store_depth(row, s, p.db, inf);
      }
    }
  }
}

constexpr int kTileV = 128;

// Shared-memory bytes finish_source_major needs for a batch of n_b sources.
__host__ __device__ inline size_t transpose_smem_bytes(int n_b, int db, int words) {
  const size_t rs = (size_t)n_b * db + (db == 1 ? 1 : 2);
  return (((size_t)kTileV * rs + 15) & ~(size_t)15) + (size_t)kTileV * words * 4;
}

template <int WORDS>
__device__ void finish_source_major(const Params& p, const GroupBufs& gb,
                                    const uint8_t* stage, int n_b, long long k0,
                                    uint8_t* smem, const Team& t) {
  const int db = p.db;
  const int rb = n_b * db;                 // row bytes in the staging array
  const int rs = rb + (db == 1 ? 1 : 2);   // odd word stride: no bank conflicts
  uint32_t* sst = reinterpret_cast<uint32_t*>(smem + (((size_t)kTileV * rs + 15) & ~(size_t)15));
  const long long ntiles = (p.V + kTileV - 1) / kTileV;
  const bool vec_out = p.vec_out != 0;
  for (long long tile = t.block; tile < ntiles; tile += t.nblocks) {
    const long long v0 = tile * kTileV;
    const int nv = (int)min((long long)kTileV, p.V - v0);
    __syncthreads();
    // The tile's rows are one contiguous run of nv*rb bytes (16-byte aligned:
    // v0 is a multiple of 128 and the staging base is 256-byte aligned).
    const uint8_t* src = stage + (size_t)v0 * rb;
    const int tot = nv * rb;
    const int nvec = tot >> 4;
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) {
      const uint4 x = __ldcs(reinterpret_cast<const uint4*>(src) + i);
      const uint32_t wv[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
      for (int b = 0; b < 16; b++) {
        const int o = i * 16 + b, r = o / rb, c = o - r * rb;
        smem[r * rs + c] = (uint8_t)(wv[b >> 2] >> (8 * (b & 3)));
      }
    }
    for (int o = nvec * 16 + threadIdx.x; o < tot; o += blockDim.x) {
      const int r = o / rb, c = o - r * rb;
      smem[r * rs + c] = src[o];
    }
    for (int i = threadIdx.x; i < nv * WORDS; i += blockDim.x)
      sst[i] = __ldcg(gb.last + (size_t)v0 * WORDS + i);
    __syncthreads();
    // item = (source j, quad of 4 vertices q)
    const int nq = (nv + 3) / 4;
    for (int i = threadIdx.x; i < n_b * nq; i += blockDim.x) {
      const int j = i / nq, q = i - j * nq;
      uint8_t* orow = p.out + (size_t)p.out_row[k0 + j] * (size_t)p.V * db;
      const uint32_t bitw = (uint32_t)j >> 5, bit = 1u << (j & 31);
      uint32_t val[4];
#pragma unroll
      for (int r4 = 0; r4 < 4; r4++) {
        const int r = q * 4 + r4;
        val[r4] = db == 1 ? 0xFFu : 0xFFFFu;
        if (r < nv && (sst[r * WORDS + bitw] & bit))
          val[r4] = db == 1 ? (uint32_t)smem[r * rs + j]
                            : (uint32_t)(smem[r * rs + 2 * j] | (smem[r * rs + 2 * j + 1] << 8));
      }
      if (vec_out && q * 4 + 4 <= nv) {
        if (db == 1) {
          *reinterpret_cast<uint32_t*>(orow + v0 + q * 4) =
              val[0] | (val[1] << 8) | (val[2] << 16) | (val[3] << 24);
        } else {
          *reinterpret_cast<uint2*>(orow + 2 * (v0 + q * 4)) =
              make_uint2(val[0] | (val[1] << 16), val[2] | (val[3] << 16));
        }
      } else {
        for (int r = q * 4; r < min(q * 4 + 4, nv); r++) {
          if (db == 1) orow[v0 + r] = (uint8_t)val[r - q * 4];
          else reinterpret_cast<uint16_t*>(orow)[v0 + r] = (uint16_t)val[r - q * 4];
        }
      }
    }
  }
}

}  // namespace ibfs
