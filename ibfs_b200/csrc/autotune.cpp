// autotune.cpp -- per-graph tuning of the traversal options.
//
// Coordinate descent over the knobs of one run: status width W (32, 64,
// 128, 256 bits; batches of W sources), the direction-switch alpha/beta, the
// small/large queue degree thresholds, the persistent kernel's occupancy
// level (persistent schedule only) and the number of concurrently running
// batches.  Every trial is the real run, in the base options' schedule
// (device loop or persistent kernel), on the caller's sample of sources with
// the depths left on the device; the score is aggregate traversed edges per
// device second.  The reference has
// no tuner (its constants are fixed: comm.h:25-30, ibfs.cu:71-72).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "internal.h"

namespace {

struct Trial {
  ibfs_opts o;
  double gteps = 0;
  double ms = 0;
};

ibfs_status time_run(ibfs_graph* g, const int32_t* src, int64_t n, const ibfs_opts& o,
                     void* dout, int reps, Trial* t) {
  ibfs_stats st;
  double best = 1e30;
  int64_t edges = 0;
  for (int r = 0; r < reps + 1; r++) {  // first run warms up (and captures the graph)
    std::memset(&st, 0, sizeof(st));
    ibfs_status s = ibfs_run(g, src, n, &o, dout, IBFS_LAYOUT_SOURCE_MAJOR, IBFS_OUT_DEVICE, &st);
    if (s != IBFS_OK) return s;
    if (r > 0 && st.device_ms > 0) best = std::min(best, st.device_ms);
    edges = st.traversed_edges;
  }
  t->o = o;
  t->ms = best;
  t->gteps = best < 1e29 ? (double)edges / (best * 1e-3) / 1e9 : 0.0;
  return IBFS_OK;
}

}  // namespace

extern "C" ibfs_status ibfs_autotune(ibfs_graph* g, const int32_t* src, int64_t n,
                                     const ibfs_opts* base, int32_t reps, ibfs_opts* best,
                                     double* best_gteps, char* log, int32_t log_cap) {
  if (!g || !src || n <= 0 || !best) return IBFS_ERR_INVALID_ARG;
  ibfs_opts o0;
  if (base) o0 = *base;
  else ibfs_opts_default(&o0);
  int64_t V = 0, E = 0;
  ibfs_graph_info(g, &V, &E, nullptr);
  if (o0.mode == IBFS_MODE_PLAIN || o0.mode == IBFS_MODE_AUTO)  // fix the schedule for all trials
    o0.mode = (double)V * (o0.width / 8) <= 32.0 * 1024 * 1024 ? IBFS_MODE_PERSISTENT
                                                                 : IBFS_MODE_DEVICE_LOOP;
  const bool persistent = o0.mode == IBFS_MODE_PERSISTENT;
  o0.use_graph = 1;
  if (o0.depth_bytes == 0) o0.depth_bytes = 1;
  if (reps < 1) reps = 2;
  void* dout = nullptr;
  if (cudaMalloc(&dout, (size_t)n * (size_t)V * o0.depth_bytes) != cudaSuccess) {
    (void)cudaGetLastError();
    return IBFS_ERR_OOM;
  }
  std::string text;
  auto note = [&](const Trial& t) {
    char buf[256];
    std::snprintf(buf, sizeof(buf),
                  "{\"width\":%d,\"concurrent\":%d,\"sml\":%d,\"lrg\":%d,\"occupancy\":%d,"
                  "\"alpha\":%g,\"beta\":%g,\"groups\":%d,\"ms\":%.4f,\"gteps\":%.2f}\n",
                  t.o.width, t.o.concurrent, t.o.sml_shed, t.o.lrg_shed, t.o.occupancy, t.o.alpha,
                  t.o.beta, t.o.groups, t.ms, t.gteps);
    text += buf;
  };
  Trial cur;
  ibfs_status s = time_run(g, src, n, o0, dout, reps, &cur);
  if (s != IBFS_OK) {
    cudaFree(dout);
    return s;
  }
  note(cur);
  // A knob moves off its current value only for a gain above kMinGain: two
  // timings of the same options differ by up to about 1 %, and chasing that
  // noise can leave a choice that is slower on the full workload.
  constexpr double kMinGain = 0.01;
  auto try_set = [&](auto mutate, int count) -> ibfs_status {
    Trial bestt = cur;
    bestt.gteps = cur.gteps * (1.0 + kMinGain);
    bool moved = false;
    for (int i = 0; i < count; i++) {
      ibfs_opts o = cur.o;
      if (!mutate(o, i)) continue;
      Trial t;
      ibfs_status st = time_run(g, src, n, o, dout, reps, &t);
      if (st == IBFS_ERR_OOM || st == IBFS_ERR_UNSUPPORTED || st == IBFS_ERR_INVALID_ARG)
        continue;  // a combination that does not fit: skip it
      if (st != IBFS_OK) return st;
      note(t);
      if (t.gteps > bestt.gteps) {
        bestt = t;
        moved = true;
      }
    }
    if (moved) cur = bestt;
    return IBFS_OK;
  };
  const int widths[] = {32, 64, 128, 256};
  const float alphas[] = {1.0f, 2.0f, 4.0f, 8.0f, 14.0f, 32.0f};
  const float betas[] = {8.0f, 24.0f, 64.0f, 256.0f};
  const int thr[][2] = {{16, 256}, {32, 512}, {64, 1024}, {32, 4096}, {8, 128}};
  const int occ[] = {0, 1, 2};
  const int groups_p[] = {0, 1, 2, 4};
  const int groups_d[] = {1, 2, 4, 8};
  const int* groups = persistent ? groups_p : groups_d;
  s = try_set([&](ibfs_opts& o, int i) {
        o.width = widths[i];
        o.concurrent = 0;
        return true;
      }, 4);
  if (s == IBFS_OK)
    s = try_set([&](ibfs_opts& o, int i) { o.alpha = alphas[i]; return true; }, 6);
  if (s == IBFS_OK)
    s = try_set([&](ibfs_opts& o, int i) { o.beta = betas[i]; return true; }, 4);
  if (s == IBFS_OK)
    s = try_set([&](ibfs_opts& o, int i) {
          o.sml_shed = thr[i][0];
          o.lrg_shed = thr[i][1];
          return true;
        }, 5);
  if (s == IBFS_OK && persistent)
    s = try_set([&](ibfs_opts& o, int i) { o.occupancy = occ[i]; return true; }, 3);
  if (s == IBFS_OK)
    s = try_set([&](ibfs_opts& o, int i) { o.groups = groups[i]; return true; }, 4);
  cudaFree(dout);
  if (s != IBFS_OK) return s;
  *best = cur.o;
  best->use_graph = base ? base->use_graph : 0;
  if (best_gteps) *best_gteps = cur.gteps;
  if (log && log_cap > 0) {
    std::snprintf(log, (size_t)log_cap, "%s", text.c_str());
  }
  return IBFS_OK;
}
