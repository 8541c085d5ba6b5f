// groupby_dev.cu -- GroupBy on the GPU (ibfs_opts.groupby = 2,
// ibfs_groupby_device).
//
// Same order as GroupBy (GroupBy.cuh:19-84, restated on the host in
// host_graph.cpp groupby_host): sources of degree <= 128 that have a
// neighbour of degree > 128 come first, ordered by the id of their FIRST
// such neighbour in the caller's CSR order (stable: input order among equal
// hubs), then every other source in input order.  The per-vertex hub is a
// property of the graph, computed once when the graph is uploaded
// (`gb_hub[v]`, -1 when v is not eligible), so one regroup costs a key per
// source and a sort of n 64-bit keys: key = hub << 32 | input position, with
// hub = 0xFFFFFFFF for the ineligible ones.  Positions make every key
// distinct, so any sort of the keys is the stable order; a bitonic network
// sorts them (one CTA in shared memory up to 4096 keys, global passes
// above).  The sorted keys give both the ordered sources and, for every
// ordered source, its input position (the caller's output row).
#include <algorithm>
#include <cstdint>

#include <cuda_runtime.h>

#include "internal.h"

namespace ibfs {

constexpr int kGbSmemKeys = 4096;   // keys sorted by one CTA in shared memory (32 KB)
constexpr int kGbThreads = 1024;

__global__ void k_gb_keys(const int32_t* __restrict__ gb_hub, const int32_t* __restrict__ src,
                          int64_t n, int64_t npad, unsigned long long* keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npad;
       i += (int64_t)gridDim.x * blockDim.x) {
    unsigned long long k = ~0ull;  // padding sorts last
    if (i < n) {
      const int32_t h = gb_hub[src[i]];
      k = ((unsigned long long)(h < 0 ? 0xFFFFFFFFu : (uint32_t)h) << 32) | (uint32_t)i;
    }
    keys[i] = k;
  }
}

// Whole bitonic network in one CTA (npad <= kGbSmemKeys, a power of two).
__global__ void __launch_bounds__(kGbThreads) k_gb_sort_smem(unsigned long long* keys,
                                                             int npad) {
  __shared__ unsigned long long s[kGbSmemKeys];
  for (int i = threadIdx.x; i < npad; i += blockDim.x) s[i] = keys[i];
  __syncthreads();
  for (int k = 2; k <= npad; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < npad; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long a = s[i], b = s[ixj];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            s[i] = b;
            s[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < npad; i += blockDim.x) keys[i] = s[i];
}

// One compare-exchange step (k, j) of the network over global memory.
__global__ void k_gb_sort_step(unsigned long long* keys, int64_t npad, int64_t k, int64_t j) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npad;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ixj = i ^ j;
    if (ixj > i) {
      const unsigned long long a = keys[i], b = keys[ixj];
      const bool up = (i & k) == 0;
      if ((a > b) == up) {
        keys[i] = b;
        keys[ixj] = a;
      }
    }
  }
}

__global__ void k_gb_gather(const unsigned long long* __restrict__ keys,
                            const int32_t* __restrict__ src, int64_t n, int32_t* ord,
                            int32_t* pos, const int32_t* __restrict__ idmap) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t p = (int32_t)(keys[i] & 0xFFFFFFFFull);
    ord[i] = idmap ? idmap[src[p]] : src[p];
    if (pos) pos[i] = p;
  }
}

int64_t groupby_dev_pad(int64_t n) {
  int64_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

// src, ord, pos (optional) and keys (groupby_dev_pad(n) entries) are device
// arrays; ord must not alias src.  idmap (optional) renames the ordered ids
// (caller ids -> the graph's internal order).  Asynchronous on `s`.
cudaError_t groupby_dev_run(const int32_t* gb_hub, const int32_t* src, int64_t n,
                            unsigned long long* keys, int32_t* ord, int32_t* pos,
                            cudaStream_t s, const int32_t* idmap) {
  if (n <= 0) return cudaSuccess;
  const int64_t npad = groupby_dev_pad(n);
  const int threads = 256;
  const int blocks = (int)std::min<int64_t>((npad + threads - 1) / threads, 4096);
  k_gb_keys<<<blocks, threads, 0, s>>>(gb_hub, src, n, npad, keys);
  if (npad <= kGbSmemKeys) {
    k_gb_sort_smem<<<1, kGbThreads, 0, s>>>(keys, (int)npad);
  } else {
    for (int64_t k = 2; k <= npad; k <<= 1)
      for (int64_t j = k >> 1; j > 0; j >>= 1)
        k_gb_sort_step<<<blocks, threads, 0, s>>>(keys, npad, k, j);
  }
  k_gb_gather<<<blocks, threads, 0, s>>>(keys, src, n, ord, pos, idmap);
  return cudaGetLastError();
}

}  // namespace ibfs
