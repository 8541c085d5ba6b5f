// launch_common.cuh -- helpers shared by the kernels of the three schedules
// (engine.cu: persistent and plain; devloop.cu: the device loop).
#pragma once
#include <algorithm>
#include <cuda_runtime.h>

#include "bfs_device.cuh"

namespace ibfs {

__device__ __forceinline__ Team make_team(int block, int nblocks) {
  Team t;
  t.block = block;
  t.nblocks = nblocks;
  t.tid = (long long)block * blockDim.x + threadIdx.x;
  t.nthreads = (long long)nblocks * blockDim.x;
  t.warp = t.tid >> 5;
  t.nwarps = t.nthreads >> 5;
  t.lane = threadIdx.x & 31;
  return t;
}

__device__ __forceinline__ int depth_limit(int db) { return db == 1 ? 254 : 65534; }

__device__ __forceinline__ uint8_t* batch_depth(const Params& p, int b) {
  return p.layout == 1 ? p.out + (size_t)b * (size_t)p.V * p.C * p.db : nullptr;
}

// Output rows of batch b (source-major) into shared memory.
__device__ __forceinline__ void load_rows(const Params& p, int b, int n_b, int32_t* s_rows) {
  if (p.layout == 0)
    for (int j = threadIdx.x; j < n_b; j += blockDim.x) s_rows[j] = p.out_row[(long long)b * p.C + j];
  __syncthreads();
}

// Plain and device-loop schedules: every kernel gets as many CTAs as fit on
// the GPU for its own register and shared-memory use (a grid-stride team
// over the whole grid).
static inline int occ_grid(const void* fn, int threads, int sms) {
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, 0) != cudaSuccess) {
    (void)cudaGetLastError();
    per = 1;
  }
  return sms * std::max(per, 1);
}

#define DISPATCH_WORDS(words, fn, ...)                  \
  ((words) == 1   ? fn<1>(__VA_ARGS__)                  \
   : (words) == 2 ? fn<2>(__VA_ARGS__)                  \
   : (words) == 4 ? fn<4>(__VA_ARGS__)                  \
                  : fn<8>(__VA_ARGS__))

}  // namespace ibfs
