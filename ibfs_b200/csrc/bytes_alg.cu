// bytes_alg.cu -- the algorithmic byte model of one batch, on the GPU.
//
// Implementation independent: a function of the graph and the per-source
// depths only (the same definition as oracle_bytes_alg in oracle/oracle.c,
// which the tests compare against bit for bit):
//   F_l  = { v : some source s has depth[s][v] == l-1 }
//   U_l  = { v : deg(v) > 0 and some source s has depth[s][v] >= l }
//   TD_l = sum_{v in F_l} (8 + w + deg(v)(4 + w))
//   BU_l = sum_{v in U_l} (8 + 2w + k_v (4 + w)), k_v = neighbours scanned in
//          CSR order until the OR of their level-(l-1) bits covers every bit
//          v gains at level l
//   bytes = sum_l min(TD_l, BU_l) + 2 w V + V n b_d
// Measurement tooling: runs outside any timed region.
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "bfs_device.cuh"
#include "internal.h"

struct ibfs_graph;
extern "C" ibfs_status ibfs_graph_device_csr(const ibfs_graph* g, const int64_t** beg,
                                             const int32_t** col);
namespace ibfs {
const int32_t* graph_host_col(const ibfs_graph* g);
const int64_t* graph_host_beg(const ibfs_graph* g);
}
extern "C" ibfs_status ibfs_graph_info(const ibfs_graph* g, int64_t* V, int64_t* E,
                                       int64_t* max_degree);

namespace ibfs {

__device__ __forceinline__ uint32_t depth_at(const void* d, int db, long long idx) {
  return db == 1 ? (uint32_t)static_cast<const uint8_t*>(d)[idx]
                 : (uint32_t)static_cast<const uint16_t*>(d)[idx];
}

__global__ void k_maxlevel(const void* depth, int db, long long total, unsigned* out) {
  const uint32_t inf = db == 1 ? 0xFFu : 0xFFFFu;
  unsigned m = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const uint32_t d = depth_at(depth, db, i);
    if (d != inf && d > m) m = d;
  }
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// mask[v] bit s = depth[s][v] <= l-1 (source s reached v before level l)
__global__ void k_mask(const void* depth, int db, long long V, int n, int words, int l,
                       uint32_t* mask) {
  const uint32_t inf = db == 1 ? 0xFFu : 0xFFFFu;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x) {
    uint32_t m[kMaxWords] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int s = 0; s < n; s++) {
      const uint32_t d = depth_at(depth, db, (long long)s * V + v);
      if (d != inf && (int)d <= l - 1) m[s >> 5] |= 1u << (s & 31);
    }
    for (int k = 0; k < words; k++) mask[v * words + k] = m[k];
  }
}

__global__ void k_level_bytes(const void* depth, int db, const int64_t* beg, const int32_t* col,
                              long long V, int n, int words, int l, const uint32_t* mask,
                              unsigned long long* td_bu) {
  const uint32_t inf = db == 1 ? 0xFFu : 0xFFFFu;
  const long long w = words * 4;
  unsigned long long td = 0, bu = 0;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x) {
    const long long deg = beg[v + 1] - beg[v];
    bool in_f = false, in_u = false;
    uint32_t need[kMaxWords] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool any = false;
    for (int s = 0; s < n; s++) {
      const uint32_t d = depth_at(depth, db, (long long)s * V + v);
      if (d == (uint32_t)(l - 1)) in_f = true;
      if (d == inf || (int)d >= l) in_u = true;
      if (d == (uint32_t)l) {
        need[s >> 5] |= 1u << (s & 31);
        any = true;
      }
    }
    if (in_f) td += 8 + w + deg * (4 + w);
    if (in_u && deg > 0) {
      long long k = 0;
      if (any) {
        uint32_t acc[kMaxWords] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (long long e = beg[v]; e < beg[v + 1]; e++) {
          const int32_t u = col[e];
          k++;
          bool covered = true;
          for (int q = 0; q < words; q++) {
            acc[q] |= mask[(long long)u * words + q];
            covered = covered && !(need[q] & ~acc[q]);
          }
          if (covered) break;
        }
      }
      bu += 8 + 2 * w + k * (4 + w);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    td += __shfl_xor_sync(0xFFFFFFFFu, td, o);
    bu += __shfl_xor_sync(0xFFFFFFFFu, bu, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (td) atomicAdd(&td_bu[0], td);
    if (bu) atomicAdd(&td_bu[1], bu);
  }
}

}  // namespace ibfs

using namespace ibfs;

extern "C" ibfs_status ibfs_bytes_alg(ibfs_graph* g, const void* depth_dev, int64_t n,
                                      int32_t depth_bytes, int32_t width, int64_t* bytes) {
  if (!g || !depth_dev || !bytes || n <= 0 || n > width ||
      (depth_bytes != 1 && depth_bytes != 2) ||
      (width != 32 && width != 64 && width != 128 && width != 256))
    return IBFS_ERR_INVALID_ARG;
  const int64_t *beg = nullptr;
  const int32_t* col = nullptr;
  int64_t V = 0, E = 0;
  ibfs_graph_device_csr(g, &beg, &col);
  ibfs_graph_info(g, &V, &E, nullptr);
  const int words = width / 32;
  // the model works on the caller's CSR (the device copy is in the graph's
  // internal vertex order), so upload that for the measurement
  int32_t* col_in = nullptr;
  int64_t* beg_in = nullptr;
  if (cudaMalloc(&beg_in, sizeof(int64_t) * (size_t)(V + 1)) != cudaSuccess) {
    (void)cudaGetLastError();
    return IBFS_ERR_OOM;
  }
  cudaMemcpy(beg_in, graph_host_beg(g), sizeof(int64_t) * (size_t)(V + 1), cudaMemcpyHostToDevice);
  beg = beg_in;
  if (E > 0) {
    if (cudaMalloc(&col_in, sizeof(int32_t) * (size_t)E) != cudaSuccess) {
      cudaFree(beg_in);
      (void)cudaGetLastError();
      return IBFS_ERR_OOM;
    }
    cudaMemcpy(col_in, graph_host_col(g), sizeof(int32_t) * (size_t)E, cudaMemcpyHostToDevice);
    col = col_in;
  }
  uint32_t* mask = nullptr;
  unsigned long long* acc = nullptr;
  unsigned* maxl = nullptr;
  if (cudaMalloc(&mask, sizeof(uint32_t) * (size_t)V * words) != cudaSuccess) {
    cudaFree(col_in);
    cudaFree(beg_in);
    (void)cudaGetLastError();
    return IBFS_ERR_OOM;
  }
  if (cudaMalloc(&acc, sizeof(unsigned long long) * 2) != cudaSuccess ||
      cudaMalloc(&maxl, sizeof(unsigned)) != cudaSuccess) {
    cudaFree(mask);
    cudaFree(acc);
    cudaFree(col_in);
    cudaFree(beg_in);
    (void)cudaGetLastError();
    return IBFS_ERR_OOM;
  }
  ibfs_status st = IBFS_OK;
  cudaMemset(maxl, 0, sizeof(unsigned));
  k_maxlevel<<<1184, 256>>>(depth_dev, depth_bytes, (long long)n * V, maxl);
  unsigned ml = 0;
  cudaMemcpy(&ml, maxl, sizeof(unsigned), cudaMemcpyDeviceToHost);
  long long total = 2LL * (width / 8) * V + V * n * depth_bytes;
  for (int l = 1; l <= (int)ml + 1; l++) {
    k_mask<<<1184, 256>>>(depth_dev, depth_bytes, V, (int)n, words, l, mask);
    cudaMemset(acc, 0, sizeof(unsigned long long) * 2);
    k_level_bytes<<<1184, 256>>>(depth_dev, depth_bytes, beg, col, V, (int)n, words, l, mask, acc);
    unsigned long long h[2] = {0, 0};
    if (cudaMemcpy(h, acc, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) {
      st = IBFS_ERR_CUDA;
      break;
    }
    total += (long long)std::min(h[0], h[1]);
  }
  if (cudaGetLastError() != cudaSuccess) st = IBFS_ERR_CUDA;
  cudaFree(mask);
  cudaFree(acc);
  cudaFree(maxl);
  cudaFree(col_in);
  cudaFree(beg_in);
  *bytes = total;
  return st;
}
