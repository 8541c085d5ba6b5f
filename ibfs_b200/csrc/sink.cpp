// sink.cpp -- the depth sink: finished batches' depth rows stream from HBM
// to the caller's host buffer while later batches are still traversing.
//
// Replaces the reference's result writer (write_result.cuh:5-36, commented
// out at its call site bfs_gpu_opt.cuh:89), which would have copied every
// depth array to the host after the whole run.  Here a batch's rows are
// handed to the sink as soon as its output pass has finished (a device flag
// in the device-loop schedule, an event in the plain one) and go down on a
// copy stream of their own, so the PCIe transfer of early batches overlaps
// the traversal of later ones:
//   * pinned destination (cudaMallocHost / cudaHostRegister memory): one
//     cudaMemcpyAsync per row straight into the caller's buffer;
//   * pageable destination: a ring of four 32 MiB pinned staging slots that
//     rows are packed into -- later slots copy in while the host spreads the
//     oldest into the caller's buffer with a parallel memcpy.
#include <algorithm>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "internal.h"

namespace ibfs {

static bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Parallel host memcpy (the pageable path's spread from a staging slot).
static void par_memcpy(void* dst, const void* src, size_t bytes) {
  constexpr size_t kPiece = 1 << 20;
  const long long pieces = (long long)((bytes + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(static) if (pieces > 4)
  for (long long i = 0; i < pieces; i++) {
    const size_t o = (size_t)i * kPiece;
    std::memcpy(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o,
                std::min(kPiece, bytes - o));
  }
}

DepthSink::~DepthSink() { release(); }

void DepthSink::release() {
  for (auto& s : slots_) {
    if (s.buf) cudaFreeHost(s.buf);
    if (s.ev) cudaEventDestroy(s.ev);
  }
  slots_.clear();
  if (stream_) cudaStreamDestroy(stream_);
  stream_ = nullptr;
  device_ = -1;
}

cudaError_t DepthSink::begin(int device, void* dst_host, const uint8_t* src_dev) {
  dst_ = static_cast<uint8_t*>(dst_host);
  src_ = src_dev;
  next_ = 0;
  open_ = -1;
  fill_ = 0;
  pending_.clear();
  for (auto& sl : slots_) sl.pieces.clear();
  copied_ = 0;
  if (stream_ && device_ != device) release();
  device_ = device;
  if (!stream_) {
    const cudaError_t e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
  }
  pinned_ = is_pinned(dst_host);
  if (!pinned_ && slots_.empty()) {
    slots_.resize(kSlots);
    for (auto& sl : slots_) {
      cudaError_t e = cudaMallocHost(&sl.buf, kSlotBytes);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming);
      if (e != cudaSuccess) {
        release();
        return e;
      }
    }
  }
  return cudaSuccess;
}

cudaError_t DepthSink::wait_for(cudaEvent_t ev) {
  if (!ev) return cudaSuccess;
  return cudaStreamWaitEvent(stream_, ev, 0);
}

// Spread the oldest closed staging slot into the caller's buffer once its
// copies have landed.
cudaError_t DepthSink::drain_one() {
  Slot& sl = slots_[pending_.front()];
  const cudaError_t e = cudaEventSynchronize(sl.ev);
  if (e != cudaSuccess) return e;
  for (const Piece& pc : sl.pieces)
    par_memcpy(dst_ + pc.off, static_cast<const uint8_t*>(sl.buf) + pc.at, pc.bytes);
  sl.pieces.clear();
  pending_.erase(pending_.begin());
  return cudaSuccess;
}

// Close the open slot: its copies are queued, an event marks their end.
cudaError_t DepthSink::close_open() {
  if (open_ < 0) return cudaSuccess;
  const cudaError_t e = cudaEventRecord(slots_[open_].ev, stream_);
  if (e != cudaSuccess) return e;
  pending_.push_back(open_);
  open_ = -1;
  return cudaSuccess;
}

cudaError_t DepthSink::push(size_t off, size_t bytes) {
  copied_ += bytes;
  if (pinned_)
    return cudaMemcpyAsync(dst_ + off, src_ + off, bytes, cudaMemcpyDeviceToHost, stream_);
  // pack pieces into staging slots; a full slot is closed and the next one
  // opened (after spreading the oldest when all are in flight)
  while (bytes > 0) {
    if (open_ >= 0 && fill_ == kSlotBytes) {
      const cudaError_t e = close_open();
      if (e != cudaSuccess) return e;
    }
    if (open_ < 0) {
      if ((int)pending_.size() == kSlots) {
        const cudaError_t e = drain_one();
        if (e != cudaSuccess) return e;
      }
      open_ = next_;
      next_ = (next_ + 1) % kSlots;
      fill_ = 0;
    }
    const size_t n = std::min(bytes, kSlotBytes - fill_);
    Slot& sl = slots_[open_];
    const cudaError_t e = cudaMemcpyAsync(static_cast<uint8_t*>(sl.buf) + fill_, src_ + off, n,
                                          cudaMemcpyDeviceToHost, stream_);
    if (e != cudaSuccess) return e;
    sl.pieces.push_back({off, fill_, n});
    fill_ += n;
    off += n;
    bytes -= n;
  }
  return cudaSuccess;
}

cudaError_t DepthSink::finish() {
  cudaError_t e = pinned_ ? cudaSuccess : close_open();
  while (e == cudaSuccess && !pending_.empty()) e = drain_one();
  const cudaError_t e2 = stream_ ? cudaStreamSynchronize(stream_) : cudaSuccess;
  return e != cudaSuccess ? e : e2;
}

}  // namespace ibfs
