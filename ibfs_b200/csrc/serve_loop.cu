// serve_loop.cu -- the serving schedule: the device-loop graph (devloop.cu)
// fed from a work queue in mapped host memory instead of a fixed batch list.
//
// The host publishes batches (up to C already grouped sources each, with the
// arena rows their depths go to) into slots of a ring and raises the ring's
// tail; every group of the running graph claims the next published batch
// when it finishes one (compare-and-swap on a device counter), so a batch
// published while the graph runs starts on the first group that frees up
// instead of waiting for the graph to end.  A group that finds the ring empty
// waits for a publication (at most kServeWaitNs), then ends its batch loop;
// once every group has, the graph launch is over and the host relaunches it
// for the batches published since.  Each finished
// batch reports itself through its slot's state word (2) and record, both in
// mapped host memory, so the host completes queries batch by batch while
// later batches still run.
//
// The reference has no serving path: it runs one fixed source list batch
// after batch (bfs_gpu_opt.cuh:182-262, batches of num_agg_bfs sources); this
// replaces that fixed loop with a queue that grows while the GPU works.
#include <algorithm>
#include <atomic>
#include <cstring>

#include <cuda_runtime.h>

#include "bfs_device.cuh"
#include "internal.h"

namespace ibfs {

namespace {
size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
// How long a group of the running graph waits for a new batch before it
// ends its loop (the graph ends once every group has): long enough to bridge
// the host's publication gaps under load, short enough that an idle server's
// graph ends soon after its last batch.
constexpr unsigned long long kServeWaitNs = 2000000ull;
}  // namespace

ServeLoop::~ServeLoop() { release(); }

void* ServeLoop::dalloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(bytes, 256)) != cudaSuccess) {
    (void)cudaGetLastError();
    return nullptr;
  }
  dev_.push_back(p);
  return p;
}

void ServeLoop::release() {
  if (stream_) {
    cudaStreamSynchronize(stream_);
    (void)cudaGetLastError();
  }
  if (exec_) cudaGraphExecDestroy(exec_);
  exec_ = nullptr;
  for (void* p : dev_) cudaFree(p);
  dev_.clear();
  if (host_) cudaFreeHost(host_);
  host_ = nullptr;
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  ev0_ = ev1_ = nullptr;
  if (stream_) cudaStreamDestroy(stream_);
  stream_ = nullptr;
  live_ = false;
}

ibfs_status ServeLoop::init(ibfs_graph* g, const ibfs_opts& o, int G, int slots, void* arena,
                            int db) {
  release();
  g_ = g;
  device_ = graph_device(g);
  if (cudaSetDevice(device_) != cudaSuccess) return IBFS_ERR_CUDA;
  words_ = o.width / 32;
  C_ = o.concurrent ? o.concurrent : o.width;
  G_ = std::max(1, G);
  slots_ = std::max(slots, 2 * G_);
  db_ = db;
  const int threads = o.threads ? o.threads : 512;
  int64_t V = 0, E = 0;
  ibfs_graph_info(g, &V, &E, nullptr);
  if (cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&ev0_) != cudaSuccess || cudaEventCreate(&ev1_) != cudaSuccess) {
    (void)cudaGetLastError();
    release();
    return IBFS_ERR_CUDA;
  }
  // ---- mapped host memory: the ring the host writes and the device reads
  const size_t o_n = 64;
  const size_t o_state = o_n + round_up(sizeof(int32_t) * slots_, 64);
  const size_t o_brec = o_state + round_up(sizeof(int32_t) * slots_, 64);
  const size_t o_src = o_brec + round_up(sizeof(BatchRec) * slots_, 64);
  const size_t o_rows = o_src + round_up(sizeof(int32_t) * slots_ * C_, 64);
  const size_t hbytes = o_rows + round_up(sizeof(int32_t) * slots_ * C_, 64);
  if (cudaHostAlloc(&host_, hbytes, cudaHostAllocMapped) != cudaSuccess) {
    (void)cudaGetLastError();
    host_ = nullptr;
    release();
    return IBFS_ERR_OOM;
  }
  std::memset(host_, 0, hbytes);
  uint8_t* hb = static_cast<uint8_t*>(host_);
  uint8_t* db_base = nullptr;
  if (cudaHostGetDevicePointer(reinterpret_cast<void**>(&db_base), host_, 0) != cudaSuccess) {
    (void)cudaGetLastError();
    release();
    return IBFS_ERR_CUDA;
  }
  h_tail_ = reinterpret_cast<long long*>(hb);
  h_n_ = reinterpret_cast<int32_t*>(hb + o_n);
  h_state_ = reinterpret_cast<int32_t*>(hb + o_state);
  h_brec_ = hb + o_brec;
  h_src_ = reinterpret_cast<int32_t*>(hb + o_src);
  h_rows_ = reinterpret_cast<int32_t*>(hb + o_rows);
  // ---- device memory: G group workspaces, the slots' copies, the claim counter
  const size_t vpad = (size_t)((V + 31) & ~31LL);
  const size_t nchg = (size_t)(((V + 31) / 32 + 127) & ~127LL);
  const int chunk = threads * 4;
  const size_t capl = (size_t)(E / chunk + std::min<int64_t>(V, E / std::max(o.lrg_shed, 1)) + 16);
  std::vector<GroupBufs> hgb((size_t)G_);
  for (int i = 0; i < G_; i++) {
    GroupBufs& b = hgb[(size_t)i];
    b.last = static_cast<uint32_t*>(dalloc(vpad * words_ * 4));
    b.curr = static_cast<uint32_t*>(dalloc(vpad * words_ * 4));
    b.chg = static_cast<uint32_t*>(dalloc(2 * nchg * 4));
    b.planes = static_cast<uint32_t*>(dalloc((size_t)(db == 1 ? 8 : 16) * vpad * words_ * 4));
    b.qs = static_cast<int32_t*>(dalloc((size_t)V * 4));
    b.qm = static_cast<int32_t*>(dalloc((size_t)V * 4));
    b.ql = static_cast<int2*>(dalloc(capl * 8));
    b.hq = static_cast<int2*>(dalloc((size_t)graph_defer_cap(g) * 8));
    b.ctl = static_cast<Ctl*>(dalloc(sizeof(Ctl)));
    if (!b.last || !b.curr || !b.chg || !b.planes || !b.qs || !b.qm || !b.ql || !b.hq || !b.ctl) {
      release();
      return IBFS_ERR_OOM;
    }
  }
  GroupBufs* d_groups = static_cast<GroupBufs*>(dalloc(sizeof(GroupBufs) * G_));
  int32_t* d_src = static_cast<int32_t*>(dalloc(sizeof(int32_t) * slots_ * C_));
  int32_t* d_rows = static_cast<int32_t*>(dalloc(sizeof(int32_t) * slots_ * C_));
  unsigned long long* d_head = static_cast<unsigned long long*>(dalloc(sizeof(unsigned long long)));
  if (!d_groups || !d_src || !d_rows || !d_head) {
    release();
    return IBFS_ERR_OOM;
  }
  bool ok = cudaMemcpy(d_groups, hgb.data(), sizeof(GroupBufs) * G_, cudaMemcpyHostToDevice) ==
                cudaSuccess &&
            cudaMemset(d_head, 0, sizeof(unsigned long long)) == cudaSuccess;
  for (int i = 0; ok && i < G_; i++)
    ok = cudaMemset(hgb[(size_t)i].ctl, 0, sizeof(Ctl)) == cudaSuccess;
  if (!ok) {
    (void)cudaGetLastError();
    release();
    return IBFS_ERR_CUDA;
  }
  Params p;
  fill_graph_params(g, o, words_, threads, &p);
  p.src = d_src;
  p.out_row = d_rows;
  p.C = C_;
  p.G = G_;
  p.cpg = graph_sms(g);
  p.db = db;
  p.layout = IBFS_LAYOUT_SOURCE_MAJOR;
  set_output_params(g, C_, static_cast<uint8_t*>(arena), &p);
  p.groups = d_groups;
  p.brec = reinterpret_cast<BatchRec*>(db_base + o_brec);
  p.lrec = nullptr;
  p.lrec_cap = 0;
  p.q_slots = slots_;
  p.q_tail = reinterpret_cast<const long long*>(db_base);
  p.q_n = reinterpret_cast<const int32_t*>(db_base + o_n);
  p.q_state = reinterpret_cast<int32_t*>(db_base + o_state);
  p.q_src = reinterpret_cast<const int32_t*>(db_base + o_src);
  p.q_rows = reinterpret_cast<const int32_t*>(db_base + o_rows);
  p.q_head = d_head;
  p.q_wait_ns = kServeWaitNs;
  cudaGraph_t graph = nullptr;
  cudaError_t e = build_device_loop_graph(p, words_, G_, graph_sms(g), threads, &graph);
  if (e == cudaSuccess) {
    e = cudaGraphInstantiate(&exec_, graph, 0);
    cudaGraphDestroy(graph);
  }
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    exec_ = nullptr;
    release();
    return IBFS_ERR_CUDA;
  }
  free_.clear();
  busy_.clear();
  for (int i = 0; i < slots_; i++) free_.push_back(i);
  published_ = 0;
  busy_ms_ = 0.0;
  launches_ = 0;
  return IBFS_OK;
}

int ServeLoop::unclaimed() const {
  int k = 0;
  for (int s : busy_)
    if (reinterpret_cast<const volatile int32_t*>(h_state_)[s] == 0) k++;
  return k;
}

int ServeLoop::publish(const int32_t* src, const int32_t* rows, int n) {
  if (n < 1 || n > C_) return -1;
  // the device maps claim number h to slot h % slots: publish in that order
  const int slot = (int)(published_ % slots_);
  auto it = std::find(free_.begin(), free_.end(), slot);
  if (it == free_.end()) return -1;  // still in flight
  free_.erase(it);
  const int32_t* noo = graph_new_of_old(g_);
  int32_t* s = h_src_ + (size_t)slot * C_;
  int32_t* r = h_rows_ + (size_t)slot * C_;
  for (int j = 0; j < n; j++) {
    s[j] = noo[(size_t)src[j]];
    r[j] = rows[j];
  }
  h_n_[slot] = n;
  reinterpret_cast<volatile int32_t*>(h_state_)[slot] = 0;
  // the slot's contents are globally visible before the tail that publishes it
  std::atomic_thread_fence(std::memory_order_seq_cst);
  published_++;
  *reinterpret_cast<volatile long long*>(h_tail_) = published_;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  busy_.push_back(slot);
  return slot;
}

bool ServeLoop::running() {
  if (!live_) return false;
  const cudaError_t q = cudaEventQuery(ev1_);
  if (q == cudaErrorNotReady) return true;
  if (q == cudaSuccess) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, ev0_, ev1_) == cudaSuccess) busy_ms_ += ms;
  }
  (void)cudaGetLastError();
  live_ = false;
  return false;
}

ibfs_status ServeLoop::pump(bool* launched) {
  *launched = false;
  if (running() || unclaimed() == 0) return IBFS_OK;
  if (cudaEventRecord(ev0_, stream_) != cudaSuccess || cudaGraphLaunch(exec_, stream_) != cudaSuccess ||
      cudaEventRecord(ev1_, stream_) != cudaSuccess) {
    (void)cudaGetLastError();
    return IBFS_ERR_CUDA;
  }
  live_ = true;
  launches_++;
  *launched = true;
  return IBFS_OK;
}

void ServeLoop::harvest(std::vector<Done>* out) {
  out->clear();
  for (size_t i = 0; i < busy_.size();) {
    const int s = busy_[i];
    if (reinterpret_cast<const volatile int32_t*>(h_state_)[s] != 2) {
      i++;
      continue;
    }
    // the record was written before the state (system-scope fence on the device)
    std::atomic_thread_fence(std::memory_order_acquire);
    BatchRec r;
    std::memcpy(&r, static_cast<const uint8_t*>(h_brec_) + sizeof(BatchRec) * s, sizeof(r));
    Done d;
    d.slot = s;
    d.err = r.err;
    d.teps = r.teps;
    d.max_level = r.max_level;
    out->push_back(d);
    busy_[i] = busy_.back();
    busy_.pop_back();
    free_.push_back(s);
  }
}

ibfs_status ServeLoop::drain() {
  if (!stream_) return IBFS_OK;
  const cudaError_t e = cudaStreamSynchronize(stream_);
  (void)running();
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return IBFS_ERR_CUDA;
  }
  return IBFS_OK;
}

}  // namespace ibfs
