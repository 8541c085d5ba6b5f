// server.cu -- continuous-batching BFS query server over a resident graph.
//
// Queries of 1..N sources arrive at any time (ibfs_server_submit, thread
// safe).  A worker thread
//   1. admits queries in arrival order as device memory allows: each query
//      owns k contiguous rows of V depths in a device arena (its per-query
//      state; a query that can never fit is refused, a full waiting queue
//      refuses with IBFS_ERR_BUSY);
//   2. cuts the admitted, not yet traversed sources of ALL queries into
//      batches of `concurrent` sources (first come first served), regrouping
//      up to `round_batches` batches' worth at a time with GroupBy
//      (GroupBy.cuh:19-84) so that sources sharing hubs share a batch, and
//      publishes them to the serving schedule's work queue (serve_loop.cu)
//      whenever a group would otherwise run dry (publish_locked);
//   3. keeps the device-loop graph of `round_batches` concurrent groups
//      running while published batches wait; a group that finishes a batch
//      takes the next published one, so a query that arrives while others
//      are on the GPU starts on the first group that frees up;
//   4. completes a query as soon as its last batch reports done.
// A query's depths are the same alone or in a mix because every source owns
// its own status bit and output row.  Results stay in the arena until the
// client polls them (host or device copy, outside the server's lock), which
// frees the rows and admits waiting queries.
//
// The reference has no serving path (it runs one fixed source list,
// bfs_gpu_opt.cuh:182-262); this is the serving pattern added beside it.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "internal.h"

namespace {

using clock_t_ = std::chrono::steady_clock;

double ms_between(clock_t_::time_point a, clock_t_::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Query {
  std::vector<int32_t> src;
  int64_t row0 = -1;  // first arena row, -1 until admitted
  int64_t remaining = 0;
  int32_t status = IBFS_OK;
  bool done = false;
  bool started = false;
  clock_t_::time_point t_submit, t_start, t_done;
};

// First-fit allocator of contiguous row ranges.
struct RowArena {
  std::map<int64_t, int64_t> free_;  // start -> length
  int64_t rows = 0, used = 0;
  void init(int64_t r) {
    rows = r;
    used = 0;
    free_.clear();
    if (r > 0) free_[0] = r;
  }
  int64_t alloc(int64_t k) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= k) {
        const int64_t s = it->first, len = it->second;
        free_.erase(it);
        if (len > k) free_[s + k] = len - k;
        used += k;
        return s;
      }
    }
    return -1;
  }
  void release(int64_t s, int64_t k) {
    used -= k;
    auto it = free_.emplace(s, k).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

}  // namespace

struct ibfs_server {
  ibfs_graph* g = nullptr;
  ibfs_server_opts so;
  int64_t V = 0;
  int db = 1;
  int64_t C = 128;
  void* arena = nullptr;
  RowArena rows;
  ibfs::ServeLoop loop;  // driven by the worker thread only
  // per queue slot: the (query, source index) of every source of its batch
  std::vector<std::vector<std::pair<uint64_t, int64_t>>> slot_src;
  std::mutex mu;
  std::condition_variable cv;
  std::thread worker;
  bool stop = false;
  ibfs_status fatal = IBFS_OK;  // a launch failed: every later query fails with it
  uint64_t next_id = 1;
  std::unordered_map<uint64_t, Query> q;
  std::deque<uint64_t> waiting;                          // not admitted yet
  std::deque<std::pair<uint64_t, int64_t>> pending;      // admitted sources (query, index)
  clock_t_::time_point t_create;
  ibfs_server_stats st;
};

using namespace ibfs;

static void admit_locked(ibfs_server* s) {
  while (!s->waiting.empty()) {
    const uint64_t id = s->waiting.front();
    Query& qq = s->q[id];
    const int64_t r = s->rows.alloc((int64_t)qq.src.size());
    if (r < 0) break;  // head of line waits for memory (first come, first served)
    qq.row0 = r;
    for (int64_t i = 0; i < (int64_t)qq.src.size(); i++) s->pending.emplace_back(id, i);
    s->waiting.pop_front();
  }
}

// GroupBy over `src` (n sources); `rows` and `who` travel with their source.
static void regroup(ibfs_server* s, std::vector<int32_t>& src, std::vector<int32_t>& rows,
                    std::vector<std::pair<uint64_t, int64_t>>& who) {
  const int64_t n = (int64_t)src.size();
  if (!s->so.groupby || n < 2) return;
  std::vector<int32_t> tmp((size_t)n);
  groupby_host(graph_host_beg(s->g), graph_host_col(s->g), s->V, src.data(), n, tmp.data());
  // map the reordered ids back to positions, stable for repeated ids
  std::vector<std::pair<int32_t, int64_t>> a((size_t)n), b((size_t)n);
  for (int64_t i = 0; i < n; i++) a[i] = {src[i], i};
  for (int64_t k = 0; k < n; k++) b[k] = {tmp[k], k};
  std::stable_sort(a.begin(), a.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
  std::stable_sort(b.begin(), b.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
  std::vector<int32_t> s2((size_t)n), r2((size_t)n);
  std::vector<std::pair<uint64_t, int64_t>> w2((size_t)n);
  for (int64_t i = 0; i < n; i++) {
    s2[b[i].second] = src[a[i].second];
    r2[b[i].second] = rows[a[i].second];
    w2[b[i].second] = who[a[i].second];
  }
  src.swap(s2);
  rows.swap(r2);
  who.swap(w2);
}

// Finished batches complete their sources; a query is done with its last.
static bool complete_locked(ibfs_server* s, const std::vector<ServeLoop::Done>& done) {
  if (done.empty()) return false;
  const auto now = clock_t_::now();
  for (const ServeLoop::Done& d : done) {
    auto& who = s->slot_src[(size_t)d.slot];
    s->st.rounds++;
    s->st.sources += (int64_t)who.size();
    if (d.err == 0) s->st.traversed_edges += (int64_t)d.teps;
    for (const auto& w : who) {
      auto it = s->q.find(w.first);
      if (it == s->q.end()) continue;
      Query& qq = it->second;
      if (d.err != 0 && qq.status == IBFS_OK) qq.status = d.err;
      if (--qq.remaining == 0) {
        qq.done = true;
        qq.t_done = now;
        s->st.completed++;
      }
    }
    who.clear();
  }
  return true;
}

// Publish batches from the pending sources, oldest first, each time as one
// GroupBy'd set so that sources sharing hubs share a batch:
//   - never while every group already has a published batch waiting;
//   - a whole round (round_batches batches) once that many sources wait;
//   - the full batches that wait, when no published batch is left unclaimed
//     (a group frees up soon and would find nothing);
//   - a partial batch once its oldest source has waited max_wait_us and no
//     published batch is left unclaimed.
static bool publish_locked(ibfs_server* s, std::vector<int32_t>& src, std::vector<int32_t>& rows,
                           std::vector<std::pair<uint64_t, int64_t>>& who) {
  ServeLoop& L = s->loop;
  const int G = L.groups();
  const int64_t round = (int64_t)std::max(1, s->so.round_batches) * s->C;
  bool any = false;
  while (!s->pending.empty() && L.can_publish()) {
    const int unclaimed = L.unclaimed();
    if (unclaimed >= G) break;
    const int64_t np = (int64_t)s->pending.size();
    int64_t take = 0;
    if (np >= round) {
      take = round;
    } else if (unclaimed == 0 && np >= s->C) {
      take = np / s->C * s->C;
    } else if (unclaimed == 0) {
      const auto oldest = s->q[s->pending.front().first].t_submit;
      if (clock_t_::now() - oldest >= std::chrono::microseconds(s->so.max_wait_us))
        take = np;
    }
    if (take == 0) break;
    src.resize((size_t)take);
    rows.resize((size_t)take);
    who.assign(s->pending.begin(), s->pending.begin() + take);
    s->pending.erase(s->pending.begin(), s->pending.begin() + take);
    const auto now = clock_t_::now();
    for (int64_t i = 0; i < take; i++) {
      Query& qq = s->q[who[(size_t)i].first];
      src[(size_t)i] = qq.src[(size_t)who[(size_t)i].second];
      rows[(size_t)i] = (int32_t)(qq.row0 + who[(size_t)i].second);
      if (!qq.started) {
        qq.started = true;
        qq.t_start = now;
      }
    }
    regroup(s, src, rows, who);
    for (int64_t b0 = 0; b0 < take; b0 += s->C) {
      const int nb = (int)std::min<int64_t>(s->C, take - b0);
      int slot = L.publish(src.data() + b0, rows.data() + b0, nb);
      if (slot < 0) {
        // no slot in publishing order is free: the rest goes back to the
        // head of the pending queue, in order
        s->pending.insert(s->pending.begin(), who.begin() + b0, who.end());
        return any;
      }
      s->slot_src[(size_t)slot].assign(who.begin() + b0, who.begin() + b0 + nb);
      any = true;
    }
  }
  return any;
}

static void fail_all_locked(ibfs_server* s, ibfs_status rc) {
  s->fatal = rc;
  const auto now = clock_t_::now();
  for (auto& kv : s->q) {
    Query& qq = kv.second;
    if (qq.done || qq.row0 < 0) continue;
    qq.status = rc;
    qq.done = true;
    qq.t_done = now;
    s->st.completed++;
  }
  s->pending.clear();
}

static void worker_loop(ibfs_server* s) {
  cudaSetDevice(graph_device(s->g));
  ServeLoop& L = s->loop;
  std::vector<int32_t> src, rows;
  std::vector<std::pair<uint64_t, int64_t>> who;
  std::vector<ServeLoop::Done> done;
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    if (s->stop) break;
    admit_locked(s);
    L.harvest(&done);
    bool progress = complete_locked(s, done);
    if (s->fatal == IBFS_OK) {
      progress |= publish_locked(s, src, rows, who);
      bool launched = false;
      const ibfs_status rc = L.pump(&launched);
      if (rc != IBFS_OK) fail_all_locked(s, rc);
      progress |= launched;
    } else {
      fail_all_locked(s, s->fatal);
    }
    if (progress) s->cv.notify_all();
    if (L.in_flight() > 0) {
      // batches on the GPU: poll their states often
      s->cv.wait_for(lk, std::chrono::microseconds(30));
    } else if (!s->pending.empty()) {
      const auto oldest = s->q[s->pending.front().first].t_submit;
      s->cv.wait_until(lk, oldest + std::chrono::microseconds(s->so.max_wait_us));
    } else if (!progress) {
      s->cv.wait_for(lk, std::chrono::milliseconds(20));
    }
  }
  lk.unlock();
  L.drain();
}

// Rows of row_bytes that an arena of `bytes` holds, at most INT32_MAX: the
// kernels receive output rows as int32 indices (row * V is computed in
// 64 bits), so a larger count would wrap and write outside the arena.
static int64_t server_arena_rows(size_t bytes, size_t row_bytes) {
  if (row_bytes == 0) return 0;
  const size_t r = bytes / row_bytes;
  return r > (size_t)INT32_MAX ? (int64_t)INT32_MAX : (int64_t)r;
}

extern "C" int64_t ibfs_server_arena_rows(int64_t arena_bytes, int64_t V, int32_t depth_bytes) {
  if (arena_bytes <= 0 || V <= 0 || (depth_bytes != 1 && depth_bytes != 2)) return 0;
  return server_arena_rows((size_t)arena_bytes, (size_t)V * (size_t)depth_bytes);
}

extern "C" void ibfs_server_opts_default(ibfs_server_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  ibfs_opts_default(&o->run);
  o->arena_bytes = 0;
  o->max_waiting = 4096;
  o->round_batches = 4;
  o->max_wait_us = 200;
  o->groupby = 1;
}

extern "C" ibfs_status ibfs_server_create(ibfs_graph* g, const ibfs_server_opts* opts,
                                          ibfs_server** out) {
  if (!g || !out) return IBFS_ERR_INVALID_ARG;
  *out = nullptr;
  ibfs_server* s = new (std::nothrow) ibfs_server();
  if (!s) return IBFS_ERR_OOM;
  if (opts) s->so = *opts;
  else ibfs_server_opts_default(&s->so);
  if (s->so.max_waiting <= 0) s->so.max_waiting = 4096;
  if (s->so.round_batches <= 0) s->so.round_batches = 4;
  if (s->so.max_wait_us < 0) s->so.max_wait_us = 0;
  s->g = g;
  int64_t E = 0;
  ibfs_graph_info(g, &s->V, &E, nullptr);
  s->db = s->so.run.depth_bytes == 2 ? 2 : 1;
  s->C = s->so.run.concurrent ? s->so.run.concurrent : s->so.run.width;
  if (s->C <= 0 || s->C > 256) {
    delete s;
    return IBFS_ERR_INVALID_ARG;
  }
  cudaSetDevice(graph_device(g));
  size_t bytes = (size_t)s->so.arena_bytes;
  if (bytes == 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      (void)cudaGetLastError();
      delete s;
      return IBFS_ERR_CUDA;
    }
    bytes = fr / 4;
  }
  const size_t row_bytes = (size_t)s->V * s->db;
  // rows travel to the kernel as int32 output-row indices
  const int64_t nrows = server_arena_rows(bytes, row_bytes);
  if (nrows < 1) {
    delete s;
    return IBFS_ERR_OOM;
  }
  if (cudaMalloc(&s->arena, (size_t)nrows * row_bytes) != cudaSuccess) {
    (void)cudaGetLastError();
    delete s;
    return IBFS_ERR_OOM;
  }
  s->rows.init(nrows);
  // the serving schedule: round_batches concurrent groups, a queue of slots
  // deep enough that publishing never waits on a slot in normal operation
  const int G = std::max(1, s->so.round_batches);
  ibfs_opts ro = s->so.run;
  ro.depth_bytes = s->db;
  const ibfs_status ls = s->loop.init(g, ro, G, std::max(64, 8 * G), s->arena, s->db);
  if (ls != IBFS_OK) {
    cudaFree(s->arena);
    delete s;
    return ls;
  }
  s->slot_src.resize((size_t)std::max(64, 8 * G));
  std::memset(&s->st, 0, sizeof(s->st));
  s->st.arena_rows = nrows;
  s->t_create = clock_t_::now();
  try {
    s->worker = std::thread(worker_loop, s);
  } catch (...) {
    s->loop.release();
    cudaFree(s->arena);
    delete s;
    return IBFS_ERR_OOM;
  }
  *out = s;
  return IBFS_OK;
}

extern "C" ibfs_status ibfs_server_submit(ibfs_server* s, const int32_t* src, int64_t n,
                                          uint64_t* qid) {
  if (!s || !src || n <= 0 || !qid) return IBFS_ERR_INVALID_ARG;
  for (int64_t i = 0; i < n; i++)
    if (src[i] < 0 || src[i] >= s->V) return IBFS_ERR_RANGE;
  std::lock_guard<std::mutex> lk(s->mu);
  if (n > s->rows.rows) {
    s->st.refused++;
    return IBFS_ERR_RANGE;  // can never fit the arena
  }
  if ((int64_t)s->waiting.size() >= s->so.max_waiting) {
    s->st.refused++;
    return IBFS_ERR_BUSY;
  }
  const uint64_t id = s->next_id++;
  Query& qq = s->q[id];
  qq.src.assign(src, src + n);
  qq.remaining = n;
  qq.t_submit = clock_t_::now();
  s->waiting.push_back(id);
  s->st.submitted++;
  *qid = id;
  s->cv.notify_all();
  return IBFS_OK;
}

// Hand a finished query to the caller: its rows are copied (host or device)
// outside the server's lock, on this thread's own stream, so that the copy
// never holds up the worker; the query leaves the table first, so no other
// thread can collect it meanwhile, and its rows are freed after the copy.
static ibfs_status collect(ibfs_server* s, std::unique_lock<std::mutex>& lk, uint64_t qid,
                           void* out, uint32_t flags, ibfs_query_info* info) {
  auto it = s->q.find(qid);
  Query qq = std::move(it->second);
  s->q.erase(it);
  ibfs_status rc = (ibfs_status)qq.status;
  const size_t bytes = qq.src.size() * (size_t)s->V * s->db;
  if (rc == IBFS_OK && out) {
    const uint8_t* from = static_cast<uint8_t*>(s->arena) + (size_t)qq.row0 * s->V * s->db;
    lk.unlock();
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(graph_device(s->g));
    cudaError_t e = cudaMemcpyAsync(out, from, bytes,
                                    (flags & IBFS_OUT_DEVICE) ? cudaMemcpyDeviceToDevice
                                                              : cudaMemcpyDeviceToHost,
                                    cudaStreamPerThread);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      rc = IBFS_ERR_CUDA;
    }
    if (prev >= 0) cudaSetDevice(prev);
    lk.lock();
  }
  const auto t_out = clock_t_::now();
  if (info) {
    info->n_sources = (int64_t)qq.src.size();
    info->latency_ms = ms_between(qq.t_submit, qq.t_done);
    info->queue_ms = qq.started ? ms_between(qq.t_submit, qq.t_start) : 0.0;
    info->status = qq.status;
    info->depth_bytes = s->db;
    info->delivered_ms = ms_between(qq.t_submit, t_out);
  }
  s->rows.release(qq.row0, (int64_t)qq.src.size());
  s->cv.notify_all();  // rows freed: the worker may admit waiting queries
  return rc;
}

extern "C" ibfs_status ibfs_server_poll(ibfs_server* s, uint64_t qid, void* out, uint32_t flags,
                                        int32_t* done, ibfs_query_info* info) {
  if (!s || !done) return IBFS_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->q.find(qid);
  if (it == s->q.end()) return IBFS_ERR_NOT_FOUND;
  *done = it->second.done ? 1 : 0;
  if (!it->second.done) return IBFS_OK;
  return collect(s, lk, qid, out, flags, info);
}

extern "C" ibfs_status ibfs_server_wait(ibfs_server* s, uint64_t qid, int32_t timeout_ms,
                                        void* out, uint32_t flags, ibfs_query_info* info) {
  if (!s) return IBFS_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->q.find(qid);
  if (it == s->q.end()) return IBFS_ERR_NOT_FOUND;
  const auto deadline = clock_t_::now() + std::chrono::milliseconds(timeout_ms);
  // look the query up afresh after every wake-up: another thread may have
  // polled and collected it meanwhile
  for (;;) {
    it = s->q.find(qid);
    if (it == s->q.end()) return IBFS_ERR_NOT_FOUND;
    if (it->second.done) break;
    if (s->cv.wait_until(lk, deadline) == std::cv_status::timeout) {
      it = s->q.find(qid);
      if (it == s->q.end()) return IBFS_ERR_NOT_FOUND;
      if (!it->second.done) return IBFS_ERR_TIMEOUT;
      break;
    }
  }
  return collect(s, lk, qid, out, flags, info);
}

extern "C" ibfs_status ibfs_server_stats_get(ibfs_server* s, ibfs_server_stats* out) {
  if (!s || !out) return IBFS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->busy_ms = s->loop.busy_ms();
  out->launches = s->loop.launches();
  out->wall_ms = ms_between(s->t_create, clock_t_::now());
  out->arena_rows_used = s->rows.used;
  return IBFS_OK;
}

extern "C" ibfs_status ibfs_server_destroy(ibfs_server* s) {
  if (!s) return IBFS_ERR_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(graph_device(s->g));
  s->loop.release();
  if (s->arena) cudaFree(s->arena);
  delete s;
  return IBFS_OK;
}
