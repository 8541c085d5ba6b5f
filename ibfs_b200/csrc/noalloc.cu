// noalloc.cu -- concurrent BFS that performs no memory allocation.
//
// Some callers cannot call cudaMalloc: plug-ins hosted by a process whose
// own allocator (a framework's caching allocator or a fixed pool) owns all
// device memory, latency-critical request paths that may not stall in
// cudaMalloc's implicit device synchronisation, and embedded deployments
// that forbid allocation after start-up.  For them ibfs_run_static_scratch runs the persistent BFS kernel
// with its scratch (status words, changed-vertex bitmap, frontier queues,
// control block and per-batch records) carved out of one file-scope device
// array of fixed size, kScratchBytes = 64 MiB.  Every GPU that loads this
// library holds that array until the process exits.
//
// The array is shared by every call on a device and keeps the last call's
// contents; the kernel clears the status words and the bitmap at the start
// of every batch and this file clears the control block and the records
// before each launch.  Calls whose work overlaps on the same GPU (two
// streams, two host threads) race on the array: callers must serialise them.
#include <cstring>

#include <cuda_runtime.h>

#include "bfs_device.cuh"
#include "internal.h"

namespace {

constexpr size_t kScratchBytes = 64ull << 20;  // the fixed maximum
constexpr int kMaxBatches = 16;
constexpr int kLrecCap = 64;
constexpr int kMaxSources = kMaxBatches * 256;

// The scratch.  In host code `g_scratch` is only a stand-in symbol: its
// device address comes from cudaGetSymbolAddress (scratch_base below).
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Device address of g_scratch in the current device's context.  Looked up
// on every call (a cheap runtime query next to the launch), so that a new
// context -- after cudaDeviceReset, say -- never receives a stale address.
// The first call on a device also loads this library's device code there,
// so that first call should come before any stream capture.
ibfs_status scratch_base(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
  if (e != cudaSuccess || p == nullptr) {
    (void)cudaGetLastError();
    return IBFS_ERR_CUDA;
  }
  *out = static_cast<unsigned char*>(p);
  return IBFS_OK;
}

}  // namespace

using namespace ibfs;

#define NA_CU(call)                  \
  do {                               \
    if ((call) != cudaSuccess) {     \
      (void)cudaGetLastError();      \
      return IBFS_ERR_CUDA;          \
    }                                \
  } while (0)

extern "C" ibfs_status ibfs_run_static_scratch(const int64_t* beg_dev, const int32_t* col_dev,
                                               int64_t V, int64_t E, const int32_t* src_dev,
                                               int64_t n, int32_t width, void* depth_dev,
                                               void* cuda_stream, int64_t* traversed_edges) {
  if (!beg_dev || (!col_dev && E > 0) || !src_dev || !depth_dev || V <= 0 || E < 0 || n <= 0)
    return IBFS_ERR_INVALID_ARG;
  if (width != 32 && width != 64 && width != 128 && width != 256) return IBFS_ERR_INVALID_ARG;
  if (V >= INT32_MAX) return IBFS_ERR_RANGE;
  const int words = width / 32;
  const int nbatches = (int)((n + width - 1) / width);
  if (nbatches > kMaxBatches || n > kMaxSources) return IBFS_ERR_RANGE;

  // scratch layout (256-byte aligned pieces)
  const int threads = 512;
  const int chunk = threads * 4;
  const int lrg = 512;
  const size_t vpad = (size_t)((V + 31) & ~31LL);
  const size_t nchg = (size_t)(((V + 31) / 32 + 127) & ~127LL);
  const size_t capl = (size_t)(E / chunk + (V < E / lrg ? V : E / lrg) + 16);
  size_t off = 0;
  const size_t o_gb = off; off = align256(off + sizeof(GroupBufs));
  const size_t o_ctl = off; off = align256(off + sizeof(Ctl));
  const size_t o_brec = off; off = align256(off + sizeof(BatchRec) * kMaxBatches);
  const size_t o_lrec = off; off = align256(off + sizeof(LevelRec) * kMaxBatches * kLrecCap);
  const size_t o_last = off; off = align256(off + vpad * words * 4);
  const size_t o_curr = off; off = align256(off + vpad * words * 4);
  const size_t o_chg = off; off = align256(off + 2 * nchg * 4);
  const size_t o_planes = off; off = align256(off + 8 * vpad * words * 4);
  const size_t o_qs = off; off = align256(off + (size_t)V * 4);
  const size_t o_qm = off; off = align256(off + (size_t)V * 4);
  const size_t o_ql = off; off = align256(off + capl * 8);
  if (off > kScratchBytes) return IBFS_ERR_RANGE;  // graph too large for the fixed scratch

  int dev = 0;
  NA_CU(cudaGetDevice(&dev));
  unsigned char* base = nullptr;
  ibfs_status st = scratch_base(&base);
  if (st != IBFS_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);

  // The sources must be vertex ids: check them on the host (stack buffer).
  int32_t hsrc[kMaxSources];
  NA_CU(cudaMemcpyAsync(hsrc, src_dev, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, s));
  NA_CU(cudaStreamSynchronize(s));
  for (int64_t i = 0; i < n; i++)
    if (hsrc[i] < 0 || hsrc[i] >= V) return IBFS_ERR_RANGE;

  GroupBufs gb;
  gb.last = reinterpret_cast<uint32_t*>(base + o_last);
  gb.curr = reinterpret_cast<uint32_t*>(base + o_curr);
  gb.chg = reinterpret_cast<uint32_t*>(base + o_chg);
  gb.planes = reinterpret_cast<uint32_t*>(base + o_planes);
  gb.qs = reinterpret_cast<int32_t*>(base + o_qs);
  gb.qm = reinterpret_cast<int32_t*>(base + o_qm);
  gb.ql = reinterpret_cast<int2*>(base + o_ql);
  gb.hq = nullptr;
  gb.ctl = reinterpret_cast<Ctl*>(base + o_ctl);
  // What must start at zero: the control block (barrier, error, counters)
  // and the batch records.  Status words and bitmap are cleared per batch by
  // the kernel itself.
  NA_CU(cudaMemcpyAsync(base + o_gb, &gb, sizeof(gb), cudaMemcpyHostToDevice, s));
  NA_CU(cudaMemsetAsync(base + o_ctl, 0, sizeof(Ctl), s));
  NA_CU(cudaMemsetAsync(base + o_brec, 0, sizeof(BatchRec) * kMaxBatches, s));

  int sms = 0, per_sm = 0;
  NA_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  NA_CU(persistent_occupancy(words, threads, 0, &per_sm));
  if (per_sm < 1) return IBFS_ERR_UNSUPPORTED;

  Params p;
  std::memset(&p, 0, sizeof(p));
  p.beg = beg_dev;
  p.col = col_dev;
  p.V = V;
  p.v_nz = V;  // the caller's CSR is not degree-ordered: sweep every vertex
  p.v_reach = V;
  p.E = E;
  p.nchg = (V + 31) / 32;
  p.chg_stride = (long long)nchg;
  p.plane_stride = (long long)vpad * words;
  p.src = src_dev;
  p.out_row = nullptr;
  p.n_total = n;
  p.C = width;
  p.nbatches = nbatches;
  p.G = 1;
  p.cpg = sms * per_sm;
  p.db = 1;
  p.layout = IBFS_LAYOUT_VERTEX_MAJOR;
  p.out = static_cast<uint8_t*>(depth_dev);
  p.sml = 32;
  p.lrg = lrg;
  p.chunk = chunk;
  p.but = 32;
  p.switch_level = -1;
  p.alpha = 14.0f;
  p.beta = 24.0f;
  p.max_levels = 254;
  p.timeout_ns = 10000ull * 1000000ull;
  p.withhold = 0;
  p.groups = reinterpret_cast<GroupBufs*>(base + o_gb);
  p.brec = reinterpret_cast<BatchRec*>(base + o_brec);
  p.lrec = reinterpret_cast<LevelRec*>(base + o_lrec);
  p.lrec_cap = kLrecCap;
  p.vec_out = ((reinterpret_cast<uintptr_t>(depth_dev) & 3) == 0) ? 1 : 0;
  p.hub_t = INT32_MAX;  // no deferred hub chunks here: the sweep scans whole lists
  p.bu_filter = 0;
  p.col_vec = 0;  // the caller's col is neither known to be padded nor aligned
  p.vec_sm = 0;
  NA_CU(launch_persistent_params(p, words, p.cpg, threads, 0, s));

  int err = 0;
  BatchRec br[kMaxBatches];
  NA_CU(cudaMemcpyAsync(&err, &gb.ctl->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  NA_CU(cudaMemcpyAsync(br, base + o_brec, sizeof(BatchRec) * nbatches, cudaMemcpyDeviceToHost, s));
  NA_CU(cudaStreamSynchronize(s));
  if (err) return (ibfs_status)err;
  if (traversed_edges) {
    int64_t t = 0;
    for (int b = 0; b < nbatches; b++) t += (int64_t)br[b].teps;
    *traversed_edges = t;
  }
  return IBFS_OK;
}
