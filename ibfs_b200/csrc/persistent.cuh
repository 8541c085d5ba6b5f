// persistent.cuh -- the persistent kernel (IBFS_MODE_PERSISTENT): one
// cooperative launch runs every level of every batch; the grid is cut into
// G groups of CTAs, each group owns one batch at a time and synchronises with
// a bounded team barrier, and the direction decision is taken on the device.
// Each status width is instantiated in a translation unit of its own
// (persistent_w32/64/128/256.cu), which exports the kernels' addresses per
// occupancy level through persistent_fn_w<W>().
#pragma once
#include <cstring>

#include <cuda_runtime.h>

#include "bfs_device.cuh"
#include "launch_common.cuh"

namespace ibfs {

// THREADS x MINB fixes the register budget (65536 / (THREADS * MINB)) and
// hence how many warps per SM hide the latency of the random gathers.
template <int WORDS, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) persistent_kernel(Params p) {
  __shared__ int s_dir, s_stop, s_err, s_maxl, s_dense;
  __shared__ int32_t s_rows[kMaxWords * 32];
  const int g = blockIdx.x / p.cpg;
  const Team t = make_team(blockIdx.x % p.cpg, p.cpg);
  const GroupBufs gb = p.groups[g];
  Ctl* ctl = gb.ctl;
  const unsigned nb = (unsigned)p.cpg;
  const bool lead = (t.block == 0 && threadIdx.x == 0);
  bool withhold = p.withhold && t.block == 0 && g == 0;
  const long long vpad = (p.V + 31) & ~31LL;

#define BARRIER()                                                   \
  do {                                                              \
    if (!team_barrier(ctl, nb, p.timeout_ns, withhold)) return;     \
    withhold = false;                                               \
  } while (0)

  for (int b = g; b < p.nbatches; b += p.G) {
    const long long k0 = (long long)b * p.C;
    const int n_b = (int)min((long long)p.C, p.n_total - k0);
    zero_words(gb.last, vpad * WORDS, t);
    zero_words(gb.curr, vpad * WORDS, t);
    zero_words(gb.chg, 2 * p.chg_stride, t);
    load_rows(p, b, n_b, s_rows);
    if (lead) {
      memset(&ctl->par[0], 0, sizeof(Par) * 2);
      memset(&ctl->qc[0][0], 0, sizeof(ctl->qc));
    }
    BARRIER();
    seed_phase<WORDS>(p, gb, p.src + k0, n_b, t);
    BARRIER();
    inspect_phase<WORDS, true>(p, gb, &ctl->par[0], n_b, 0, true, false, t);
    BARRIER();
    int level = 0, cur_dir = kDirTD, max_level = 0, td = 0, bu = 0;
    unsigned long long m_u = (unsigned long long)p.E, teps = 0, prev_changed = 0;
    unsigned long long t_lvl = global_ns(), t_mid = t_lvl;
    int err = 0;
    while (true) {
      if (threadIdx.x == 0) {
        const volatile Par* pr = &ctl->par[level & 1];
        const unsigned long long changed = pr->changed, mf = pr->mf, cdeg = pr->cdeg;
        teps += pr->teps;
        m_u = m_u > cdeg ? m_u - cdeg : 0ull;
        int stop = 0;
        if (pr->range_err) { stop = 1; err = 3; }
        else if (changed == 0) stop = 1;
        else if (level + 1 > p.max_levels) { stop = 1; err = 3; }
        if (changed && !pr->range_err) max_level = level;
        const int nd = choose_dir(level + 1, cur_dir, p.switch_level, p.alpha, p.beta,
                                  changed, prev_changed, mf, m_u, p.V);
        prev_changed = changed;
        if (t.block == 0) {
          if (level < p.lrec_cap) {
            LevelRec r;
            r.batch = b; r.level = level; r.dir = level == 0 ? -1 : cur_dir; r.pad = 0;
            r.frontier = (long long)changed; r.frontier_edges = (long long)mf;
            const unsigned long long t_now = global_ns();
            r.expand_ns = (long long)(t_mid - t_lvl);
            r.inspect_ns = (long long)(t_now - t_mid);
            t_lvl = t_now;
            p.lrec[(size_t)b * p.lrec_cap + level] = r;
          }
          if (!stop) {
            memset((void*)&ctl->par[(level + 1) & 1], 0, sizeof(Par));
            ctl->qc[level & 1][0] = ctl->qc[level & 1][1] = ctl->qc[level & 1][2] = 0;
          }
        }
        s_dir = nd;
        s_stop = stop;
        s_err = err;
        s_maxl = max_level;
        s_dense = inspect_dense(mf, p.V) ? 1 : 0;
      }
      __syncthreads();
      const int stop = s_stop;
      cur_dir = s_dir;
      err = s_err;
      const bool dense = s_dense != 0;
      __syncthreads();
      if (stop) break;
      level++;
      bool continue_inspect = false;
      zero_plane_if_first(p, gb, level, t);
      if (cur_dir == kDirTD) {
        td++;
        qbuild_phase(p, gb, level, ctl->qc[level & 1], t);
        BARRIER();
        td_phase<WORDS>(p, gb, level, ctl->qc[level & 1], t);
      } else {
        bu++;
        const bool filt =
            bu_filter_level(p.bu_filter, __ldcg(&ctl->par[(level - 1) & 1].changed), p.V);
        bu_phase<WORDS>(p, gb, level, ctl->par[(level - 1) & 1].fmask,
                        &ctl->par[level & 1].hq_cnt, t, nullptr, 0, true, filt);
        BARRIER();
        if (__ldcg(&ctl->par[level & 1].hq_cnt) > 0) {  // same value in every CTA
          bu_defer_phase<WORDS>(p, gb, level, ctl->par[(level - 1) & 1].fmask,
                                &ctl->par[level & 1].hq_cnt, t, filt);
          BARRIER();
        }
        if (lead) t_mid = global_ns();
        continue_inspect = true;
      }
      if (!continue_inspect) {
        BARRIER();
        if (lead) t_mid = global_ns();
      }
      inspect_phase<WORDS, true>(p, gb, &ctl->par[level & 1], n_b, level,
                                 level <= depth_limit(p.db), dense, t);
      BARRIER();
    }
    if (err) {
      if (lead) {
        atomicCAS(&ctl->err, 0, err);
        p.brec[b].err = err;
      }
      return;
    }
    output_phase<WORDS>(p, gb, batch_depth(p, b), s_rows, n_b, s_maxl, t);
    if (lead && level + 1 < p.lrec_cap) {
      // one extra record per batch: dir 2 = the output pass
      LevelRec r;
      r.batch = b; r.level = level + 1; r.dir = 2; r.pad = 0;
      r.frontier = 0; r.frontier_edges = 0;
      r.expand_ns = (long long)(global_ns() - t_lvl);
      r.inspect_ns = 0;
      p.lrec[(size_t)b * p.lrec_cap + level + 1] = r;
    }
    if (lead) {
      BatchRec r;
      r.levels = level;
      r.max_level = max_level;
      r.td = td;
      r.bu = bu;
      r.teps = teps;
      r.err = 0;
      r.pad = 0;
      p.brec[b] = r;
    }
    BARRIER();
  }
#undef BARRIER
}

// Occupancy levels of the persistent kernel: 512 x 2 (default), 256 x 6,
// 256 x 8 and 512 x 1 threads x CTAs per SM (the register budget).
template <int WORDS>
const void* persistent_fn(int level) {
  switch (level) {
    case 1: return (const void*)persistent_kernel<WORDS, 256, 6>;
    case 2: return (const void*)persistent_kernel<WORDS, 256, 8>;
    case 3: return (const void*)persistent_kernel<WORDS, 512, 1>;
    default: return (const void*)persistent_kernel<WORDS, 512, 2>;
  }
}

}  // namespace ibfs
