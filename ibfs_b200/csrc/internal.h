// internal.h -- declarations shared by the host C++ and CUDA sources of libibfs.
#pragma once
#include <cstdint>
#include <algorithm>
#include <cstddef>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ibfs.h"

namespace ibfs {

// Counter-based 64-bit hash (splitmix64 finaliser, Steele/Lea/Flood 2014):
// every generator draws value i of stream `stream` as rnd(seed, stream, i),
// so generation is parallel and independent of the thread count.
static inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static inline uint64_t rnd(uint64_t seed, uint64_t stream, uint64_t i) {
  return mix64(mix64(seed ^ (stream * 0xD1B54A32D192ED03ull)) + i);
}

// Host CSR (int64 offsets, int32 column ids).
struct HostCsr {
  int64_t V = 0, E = 0;
  std::vector<int64_t> beg;
  std::vector<int32_t> col;
};

// Symmetrise, drop self-loops, sort and dedupe every adjacency list.
ibfs_status build_csr(const int32_t* u, const int32_t* v, int64_t m, int64_t V,
                      HostCsr* out);
ibfs_status load_csr_files(const char* beg_path, const char* csr_path,
                           HostCsr* out);
ibfs_status validate_csr(const int64_t* beg, const int32_t* col, int64_t V,
                         int64_t E);
void groupby_host(const int64_t* beg, const int32_t* col, int64_t V,
                  const int32_t* src, int64_t n, int32_t* out);
void groupby_host_maxhub(const int64_t* beg, const int32_t* col, int64_t V,
                         const int32_t* src, int64_t n, int32_t* out);

}  // namespace ibfs

namespace ibfs {
struct Params;
// persistent_w*.cu: the persistent kernel's address for a status width and an
// occupancy level (0: 512 x 2, 1: 256 x 6, 2: 256 x 8, 3: 512 x 1).
const void* persistent_fn_w32(int level);
const void* persistent_fn_w64(int level);
const void* persistent_fn_w128(int level);
const void* persistent_fn_w256(int level);
// engine.cu: launch helpers shared with the static-scratch entry point.
cudaError_t launch_persistent_params(const Params& p, int words, int grid, int threads,
                                     size_t smem, cudaStream_t s);
cudaError_t persistent_occupancy(int words, int threads, size_t smem, int* per_sm);
// groupby_dev.cu: GroupBy on the device (keys sized groupby_dev_pad(n)).
int64_t groupby_dev_pad(int64_t n);
cudaError_t groupby_dev_run(const int32_t* gb_hub, const int32_t* src, int64_t n,
                            unsigned long long* keys, int32_t* ord, int32_t* pos,
                            cudaStream_t s, const int32_t* idmap = nullptr);
// devloop.cu: the device-loop CUDA graph of one run (not instantiated).
cudaError_t build_device_loop_graph(const Params& p, int words, int G, int sms, int threads,
                                    cudaGraph_t* out);
}  // namespace ibfs

namespace ibfs {
// engine.cu: already-ordered sources into explicit rows of a device array.
ibfs_status run_rows(ibfs_graph* g, const int32_t* src, const int32_t* rows, int64_t n,
                     const ibfs_opts& o, void* dev_out, ibfs_stats* st);
int graph_device(const ibfs_graph* g);
const int64_t* graph_host_beg(const ibfs_graph* g);
const int32_t* graph_host_col(const ibfs_graph* g);
int graph_sms(const ibfs_graph* g);
int64_t graph_defer_cap(const ibfs_graph* g);
const int32_t* graph_new_of_old(const ibfs_graph* g);  // caller id -> internal id (host)
// Launch parameters that depend only on the graph and the options, and the
// output pointer with the store widths its alignment allows.
void fill_graph_params(const ibfs_graph* g, const ibfs_opts& o, int words, int threads,
                       Params* p);
void set_output_params(const ibfs_graph* g, int C, uint8_t* dout, Params* p);
}  // namespace ibfs

namespace ibfs {
// serve_loop.cu: the serving schedule -- the device-loop graph of G groups
// fed from a work queue in mapped host memory (Params::q_*).  The host
// publishes batches of already grouped sources whose depths go to rows of a
// device arena while the graph runs; each group claims the next published
// batch when it finishes one.  Not thread safe: one host thread drives it.
class ServeLoop {
 public:
  struct Done {
    int slot;
    int32_t err;         // 0, or the batch's ibfs_status
    uint64_t teps;       // traversed edges of the batch
    int32_t max_level;
  };
  ~ServeLoop();
  // G groups, `slots` queue slots of C sources each, depths (db bytes) to
  // source-major rows of `arena` (V * db bytes per row).
  ibfs_status init(ibfs_graph* g, const ibfs_opts& o, int G, int slots, void* arena, int db);
  int capacity() const { return C_; }
  int groups() const { return G_; }
  // whether the next slot in publishing order is free
  bool can_publish() const {
    return std::find(free_.begin(), free_.end(), (int)(published_ % slots_)) != free_.end();
  }
  // published batches that no group has claimed yet
  int unclaimed() const;
  // slots published and not yet reported done
  int in_flight() const { return (int)busy_.size(); }
  // Publish one batch (caller ids, 1..C sources, their arena rows); returns
  // the slot, or -1 when no slot is free.
  int publish(const int32_t* src, const int32_t* rows, int n);
  // Launch the graph when it is not running and a published batch waits.
  // Returns true when a launch was issued.
  ibfs_status pump(bool* launched);
  // Batches finished since the last call.
  void harvest(std::vector<Done>* out);
  // Whether the graph is running.
  bool running();
  // Wait for the running graph to end (every group finds the queue empty).
  ibfs_status drain();
  double busy_ms() const { return busy_ms_; }
  int64_t launches() const { return launches_; }
  void release();

 private:
  ibfs_graph* g_ = nullptr;
  int device_ = 0, C_ = 0, slots_ = 0, G_ = 0, words_ = 0, db_ = 1;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  bool live_ = false;
  double busy_ms_ = 0.0;
  int64_t launches_ = 0;
  long long published_ = 0;
  // mapped host memory: tail, n, src, rows, state, records
  void* host_ = nullptr;
  long long* h_tail_ = nullptr;
  int32_t *h_n_ = nullptr, *h_src_ = nullptr, *h_rows_ = nullptr, *h_state_ = nullptr;
  void* h_brec_ = nullptr;
  // device memory: workspace of the G groups, slot copies, claim counter
  std::vector<void*> dev_;
  std::vector<int> free_;   // free slots
  std::vector<int> busy_;   // published, not yet harvested
  void* dalloc(size_t bytes);
};
}  // namespace ibfs

namespace ibfs {
// sink.cpp: streams finished batches' depth rows (byte ranges of the device
// output) to a host buffer on a copy stream of its own; pinned destinations
// take direct copies, pageable ones a pinned staging ring.
class DepthSink {
 public:
  ~DepthSink();
  cudaError_t begin(int device, void* dst_host, const uint8_t* src_dev);
  // the next copies wait for `ev` (recorded on the compute stream)
  cudaError_t wait_for(cudaEvent_t ev);
  // copy bytes [off, off + bytes) of the output to the same offset on the host
  cudaError_t push(size_t off, size_t bytes);
  // wait until every pushed range is in the host buffer
  cudaError_t finish();
  void release();
  size_t copied() const { return copied_; }
  bool pinned() const { return pinned_; }

 private:
  static constexpr int kSlots = 4;
  static constexpr size_t kSlotBytes = 32u << 20;
  struct Piece {
    size_t off, at, bytes;  // output offset, offset in the slot, length
  };
  struct Slot {
    void* buf = nullptr;
    cudaEvent_t ev = nullptr;
    std::vector<Piece> pieces;
  };
  cudaError_t drain_one();
  cudaError_t close_open();
  int device_ = -1;
  cudaStream_t stream_ = nullptr;
  std::vector<Slot> slots_;
  std::vector<int> pending_;  // closed slots in copy order
  int next_ = 0;
  int open_ = -1;             // slot being filled (-1: none)
  size_t fill_ = 0;
  bool pinned_ = false;
  uint8_t* dst_ = nullptr;
  const uint8_t* src_ = nullptr;
  size_t copied_ = 0;
};
}  // namespace ibfs
