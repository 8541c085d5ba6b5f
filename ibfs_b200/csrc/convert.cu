// convert.cu -- edge-list text -> binary CSR on the GPU (ibfs_convert_text).
//
// Replaces the reference's converter tuple_text_to_bin.cpp:56-310:
//   * the text (after `skip` header lines, skipped as tuple_text_to_bin.cpp:
//     79-96 does) is a run of integer tokens separated by ' ', '\t' or '\n';
//     a token begins at offset 0 and after every run of separators, and its
//     value is what atol() reads there (tuple_text_to_bin.cpp:103-130);
//   * tokens pair up into edges (u, v) in order; ids are shifted by the
//     smallest token so that V = max - min + 1 (:133-147);
//   * reference mode: every edge u->v (and v->u with `reverse`) is appended
//     to its source's list in file order -- no sorting, no deduplication,
//     self loops kept (:201-266) -- so the files are byte-identical to the
//     reference's _beg_pos.bin/_csr.bin.  That includes its self-loop quirk
//     with `reverse`: both directions are written before either count
//     moves (:248-262), so a loop u-u fills one slot of u's list with u and
//     leaves the next one 0;
//   * clean mode (what the reference lacks): symmetrised, self loops
//     dropped, every list sorted and deduplicated.
// On the device: token starts are flags, a scan numbers them, a kernel
// parses each; the half-edges are put in source order by a stable LSD radix
// sort written here (8-bit digits; per block a digit histogram, one global
// scan, then a stable scatter whose in-block ranks come from warp
// match/ballot); list offsets are a degree histogram and a scan.
// Differences from the reference, by design: an odd token count is an
// IBFS_ERR_FORMAT (the reference writes an inconsistent CSR), and the
// _head/_deg/_weight side files are not written (the weights come from an
// unseeded rand(); iBFS reads only _beg_pos and _csr).
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "internal.h"

namespace ibfs {
namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 2 * kScanThreads;
constexpr int kRsThreads = 256;                  // radix sort CTA
constexpr int kRsItems = 8;                      // items per thread per tile
constexpr int kRsTile = kRsThreads * kRsItems;   // 2048 items per tile
constexpr int kRsWarps = kRsThreads / 32;

__device__ __forceinline__ bool is_sep(uint8_t c) { return c == ' ' || c == '\t' || c == '\n'; }
__device__ __forceinline__ bool is_space(uint8_t c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

// ---- exclusive scan of unsigned long long (multi-level) ----------------------
__global__ void __launch_bounds__(kScanThreads) k_scan_chunk(const unsigned long long* in,
                                                             unsigned long long* out,
                                                             unsigned long long* sums,
                                                             int64_t n) {
  __shared__ unsigned long long s[kScanItems];
  const int64_t base = (int64_t)blockIdx.x * kScanItems;
  for (int i = threadIdx.x; i < kScanItems; i += blockDim.x)
    s[i] = base + i < n ? in[base + i] : 0ull;
  __syncthreads();
  // Blelloch up-sweep / down-sweep over kScanItems entries
  for (int d = 1; d < kScanItems; d <<= 1) {
    const int i = (threadIdx.x + 1) * (d << 1) - 1;
    if (i < kScanItems) s[i] += s[i - d];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (sums) sums[blockIdx.x] = s[kScanItems - 1];
    s[kScanItems - 1] = 0;
  }
  __syncthreads();
  for (int d = kScanItems >> 1; d >= 1; d >>= 1) {
    const int i = (threadIdx.x + 1) * (d << 1) - 1;
    if (i < kScanItems) {
      const unsigned long long t = s[i - d];
      s[i - d] = s[i];
      s[i] += t;
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < kScanItems; i += blockDim.x)
    if (base + i < n) out[base + i] = s[i];
}

__global__ void k_scan_add(unsigned long long* out, const unsigned long long* offs, int64_t n) {
  const int64_t base = (int64_t)blockIdx.x * kScanItems;
  for (int i = threadIdx.x; i < kScanItems; i += blockDim.x)
    if (base + i < n) out[base + i] += offs[blockIdx.x];
}

struct Scratch {
  std::vector<void*> bufs;
  ~Scratch() {
    for (void* p : bufs) cudaFree(p);
  }
  template <class T>
  cudaError_t get(T** p, size_t count) {
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return e;
    bufs.push_back(q);
    *p = reinterpret_cast<T*>(q);
    return cudaSuccess;
  }
};

// out may alias in.
cudaError_t exclusive_scan(const unsigned long long* in, unsigned long long* out, int64_t n,
                           Scratch& sc, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int64_t chunks = (n + kScanItems - 1) / kScanItems;
  unsigned long long* sums = nullptr;
  cudaError_t e;
  if (chunks > 1 && (e = sc.get(&sums, (size_t)chunks)) != cudaSuccess) return e;
  k_scan_chunk<<<(unsigned)chunks, kScanThreads, 0, s>>>(in, out, sums, n);
  if (chunks > 1) {
    if ((e = exclusive_scan(sums, sums, chunks, sc, s)) != cudaSuccess) return e;
    k_scan_add<<<(unsigned)chunks, kScanThreads, 0, s>>>(out, sums, n);
  }
  return cudaGetLastError();
}

// ---- text -> tokens --------------------------------------------------------
__global__ void k_token_flags(const uint8_t* t, int64_t len, unsigned long long* flag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = (i == 0 || (is_sep(t[i - 1]) && !is_sep(t[i]))) ? 1ull : 0ull;
}

// value of the token at i as atol() reads it: leading white space, a sign,
// decimal digits (it may run past the token, as atol does)
__device__ long long atol_at(const uint8_t* t, int64_t len, int64_t i) {
  while (i < len && is_space(t[i])) i++;
  bool neg = false;
  if (i < len && (t[i] == '+' || t[i] == '-')) neg = t[i++] == '-';
  long long v = 0;
  while (i < len && t[i] >= '0' && t[i] <= '9') v = v * 10 + (t[i++] - '0');
  return neg ? -v : v;
}

__global__ void k_tokens(const uint8_t* t, int64_t len, const unsigned long long* flag,
                         const unsigned long long* idx, long long* tok, long long* mn,
                         long long* mx) {
  long long lo = LLONG_MAX, hi = LLONG_MIN;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    const long long v = atol_at(t, len, i);
    tok[idx[i]] = v;
    lo = min(lo, v);
    hi = max(hi, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mn, lo);
    atomicMax(mx, hi);
  }
}

// half-edges in insertion order: edge i gives 2i (u->v) and, with reverse,
// 2i+1 (v->u); clean mode drops self loops later
__global__ void k_half_edges(const long long* tok, int64_t lines, long long vmin, int reverse,
                             int clean, uint32_t* key, uint32_t* val) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < lines;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t u = (uint32_t)(tok[2 * i] - vmin), v = (uint32_t)(tok[2 * i + 1] - vmin);
    if (reverse) {
      key[2 * i] = u; val[2 * i] = v;
      key[2 * i + 1] = v; val[2 * i + 1] = (u != v || clean) ? u : 0u;  // the reference's hole
    } else {
      key[i] = u; val[i] = v;
    }
  }
}

// ---- stable LSD radix sort of (key, value) by key -----------------------------
__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const uint32_t* key, int64_t n,
                                                        int shift, int64_t ntiles,
                                                        unsigned long long* hist) {
  __shared__ unsigned int h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kRsTile;
  for (int j = 0; j < kRsItems; j++) {
    const int64_t i = base + (int64_t)j * kRsThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(key[i] >> shift) & 0xFFu], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x)
    hist[(int64_t)d * ntiles + blockIdx.x] = h[d];  // digit-major: scan gives global offsets
}

// Item order inside a tile is j-major (j * kRsThreads + thread), the order of
// the input; ranks among equal digits follow it, so the pass is stable.
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const uint32_t* key,
                                                           const uint32_t* val, int64_t n,
                                                           int shift, int64_t ntiles,
                                                           const unsigned long long* offs,
                                                           uint32_t* key_out, uint32_t* val_out) {
  __shared__ unsigned int cnt[kRsWarps][256];
  __shared__ unsigned long long run[256];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < 256; d += blockDim.x)
    run[d] = offs[(int64_t)d * ntiles + blockIdx.x];
  const int64_t base = (int64_t)blockIdx.x * kRsTile;
  for (int j = 0; j < kRsItems; j++) {
    for (int i = threadIdx.x; i < kRsWarps * 256; i += blockDim.x) (&cnt[0][0])[i] = 0;
    __syncthreads();
    const int64_t i = base + (int64_t)j * kRsThreads + threadIdx.x;
    const bool ok = i < n;
    const uint32_t k = ok ? key[i] : 0u;
    const int d = ok ? (int)((k >> shift) & 0xFFu) : 256 + lane;  // invalid: unique, unmatched
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (ok && rank == 0) cnt[w][d] = __popc(peers);
    __syncthreads();
    unsigned long long before = 0;
    if (ok) {
      before = run[d];
      for (int ww = 0; ww < w; ww++) before += cnt[ww][d];
      before += rank;
    }
    __syncthreads();
    for (int dd = threadIdx.x; dd < 256; dd += blockDim.x) {
      unsigned int tot = 0;
      for (int ww = 0; ww < kRsWarps; ww++) tot += cnt[ww][dd];
      run[dd] += tot;
    }
    if (ok) {
      key_out[before] = k;
      val_out[before] = val[i];
    }
    __syncthreads();
  }
}

cudaError_t radix_sort(uint32_t*& key, uint32_t*& val, uint32_t* key_alt, uint32_t* val_alt,
                       int64_t n, int bits, Scratch& sc, cudaStream_t s) {
  if (n <= 1) return cudaSuccess;
  const int64_t ntiles = (n + kRsTile - 1) / kRsTile;
  unsigned long long* hist = nullptr;
  cudaError_t e;
  if ((e = sc.get(&hist, (size_t)(256 * ntiles))) != cudaSuccess) return e;
  uint32_t *ka = key, *va = val, *kb = key_alt, *vb = val_alt;
  for (int shift = 0; shift < bits; shift += 8) {
    k_rs_hist<<<(unsigned)ntiles, kRsThreads, 0, s>>>(ka, n, shift, ntiles, hist);
    if ((e = exclusive_scan(hist, hist, 256 * ntiles, sc, s)) != cudaSuccess) return e;
    k_rs_scatter<<<(unsigned)ntiles, kRsThreads, 0, s>>>(ka, va, n, shift, ntiles, hist, kb, vb);
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  key = ka;
  val = va;
  return cudaGetLastError();
}

// ---- CSR assembly ------------------------------------------------------------
__global__ void k_clean_flags(const uint32_t* key, const uint32_t* val, int64_t n,
                              unsigned long long* keep) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    keep[i] = (key[i] != val[i] && (i == 0 || key[i] != key[i - 1] || val[i] != val[i - 1]))
                  ? 1ull : 0ull;
}

__global__ void k_compact(const uint32_t* key, const uint32_t* val, int64_t n,
                          const unsigned long long* keep, const unsigned long long* pos,
                          uint32_t* key_out, uint32_t* val_out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (keep[i]) {
      key_out[pos[i]] = key[i];
      val_out[pos[i]] = val[i];
    }
}

__global__ void k_degree(const uint32_t* key, int64_t n, unsigned long long* deg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&deg[key[i]], 1ull);
}

int bits_for(int64_t V) {
  int b = 0;
  while (b < 32 && (1LL << b) < V) b += 8;
  return std::max(b, 8);
}

// Skip `skip` header lines exactly as tuple_text_to_bin.cpp:79-96 does
// (its first step moves past offset 0 before looking for '\n').
bool skip_header(const std::vector<uint8_t>& t, int64_t skip, size_t* off) {
  size_t h = 0;
  int64_t k = 0;
  while (true) {
    if (k == skip) break;
    if (h >= t.size()) return false;
    h++;
    if (h < t.size() && t[h] == '\n') {
      h++;
      k++;
      if (k == skip) break;
    }
  }
  *off = h;
  return true;
}

}  // namespace
}  // namespace ibfs

using namespace ibfs;

extern "C" ibfs_status ibfs_convert_text(const char* text_path, int32_t reverse,
                                         int64_t skip_lines, int32_t clean,
                                         const char* beg_path, const char* csr_path,
                                         int32_t device, int64_t* V_out, int64_t* E_out) {
  if (!text_path || !beg_path || !csr_path || skip_lines < 0) return IBFS_ERR_INVALID_ARG;
  FILE* f = std::fopen(text_path, "rb");
  if (!f) return IBFS_ERR_IO;
  std::vector<uint8_t> text;
  {
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (sz < 0) {
      std::fclose(f);
      return IBFS_ERR_IO;
    }
    text.resize((size_t)sz);
    const bool ok = std::fread(text.data(), 1, text.size(), f) == text.size();
    std::fclose(f);
    if (!ok) return IBFS_ERR_IO;
  }
  size_t off = 0;
  if (!skip_header(text, skip_lines, &off)) return IBFS_ERR_FORMAT;
  const int64_t len = (int64_t)(text.size() - std::min(off, text.size()));
  if (len <= 0) return IBFS_ERR_FORMAT;
  if (cudaSetDevice(device) != cudaSuccess) {
    (void)cudaGetLastError();
    return IBFS_ERR_CUDA;
  }
  cudaStream_t s = nullptr;
  Scratch sc;
#define CV(call)                                                   \
  do {                                                             \
    const cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) {                                       \
      (void)cudaGetLastError();                                    \
      return e_ == cudaErrorMemoryAllocation ? IBFS_ERR_OOM : IBFS_ERR_CUDA; \
    }                                                              \
  } while (0)
  const int threads = 256, blocks = 4096;
  uint8_t* dt = nullptr;
  unsigned long long *flag = nullptr, *idx = nullptr;
  CV(sc.get(&dt, (size_t)len));
  CV(sc.get(&flag, (size_t)len));
  CV(sc.get(&idx, (size_t)len));
  CV(cudaMemcpyAsync(dt, text.data() + off, (size_t)len, cudaMemcpyHostToDevice, s));
  k_token_flags<<<blocks, threads, 0, s>>>(dt, len, flag);
  CV(cudaGetLastError());
  CV(exclusive_scan(flag, idx, len, sc, s));
  unsigned long long last_idx = 0, last_flag = 0;
  CV(cudaMemcpyAsync(&last_idx, idx + len - 1, 8, cudaMemcpyDeviceToHost, s));
  CV(cudaMemcpyAsync(&last_flag, flag + len - 1, 8, cudaMemcpyDeviceToHost, s));
  CV(cudaStreamSynchronize(s));
  const int64_t ntok = (int64_t)(last_idx + last_flag);
  if (ntok < 2 || (ntok & 1)) return IBFS_ERR_FORMAT;
  long long* tok = nullptr;
  long long* mm = nullptr;
  CV(sc.get(&tok, (size_t)ntok));
  CV(sc.get(&mm, 2));
  const long long init[2] = {LLONG_MAX, LLONG_MIN};
  CV(cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, s));
  k_tokens<<<blocks, threads, 0, s>>>(dt, len, flag, idx, tok, mm, mm + 1);
  CV(cudaGetLastError());
  long long mmh[2];
  CV(cudaMemcpyAsync(mmh, mm, sizeof(mmh), cudaMemcpyDeviceToHost, s));
  CV(cudaStreamSynchronize(s));
  const long long vmin = mmh[0], vmax = mmh[1];
  const int64_t V = (int64_t)(vmax - vmin + 1);
  if (vmin < 0 || V <= 0 || V >= (1LL << 31)) return IBFS_ERR_RANGE;
  const int64_t lines = ntok / 2;
  const bool both = reverse || clean;  // clean mode always symmetrises
  int64_t n = both ? 2 * lines : lines;
  if (n >= (1LL << 31)) return IBFS_ERR_RANGE;
  uint32_t *k0 = nullptr, *v0 = nullptr, *k1 = nullptr, *v1 = nullptr;
  CV(sc.get(&k0, (size_t)n));
  CV(sc.get(&v0, (size_t)n));
  CV(sc.get(&k1, (size_t)n));
  CV(sc.get(&v1, (size_t)n));
  k_half_edges<<<blocks, threads, 0, s>>>(tok, lines, vmin, both ? 1 : 0, clean ? 1 : 0, k0, v0);
  CV(cudaGetLastError());
  uint32_t *key = k0, *val = v0;
  const int bits = bits_for(V);
  if (clean) {
    // by (source, neighbour): a pass keyed by the neighbour, then a stable
    // pass keyed by the source
    uint32_t *ka = v0, *va = k0;
    CV(radix_sort(ka, va, k1, v1, n, bits, sc, s));
    const bool in0 = ka == v0 || ka == k0;  // which buffer pair holds the result
    uint32_t *kb = va, *vb = ka;
    CV(radix_sort(kb, vb, in0 ? k1 : k0, in0 ? v1 : v0, n, bits, sc, s));
    key = kb;
    val = vb;
    unsigned long long *keep = nullptr, *pos = nullptr;
    CV(sc.get(&keep, (size_t)n));
    CV(sc.get(&pos, (size_t)n));
    k_clean_flags<<<blocks, threads, 0, s>>>(key, val, n, keep);
    CV(cudaGetLastError());
    CV(exclusive_scan(keep, pos, n, sc, s));
    unsigned long long lp = 0, lk = 0;
    CV(cudaMemcpyAsync(&lp, pos + n - 1, 8, cudaMemcpyDeviceToHost, s));
    CV(cudaMemcpyAsync(&lk, keep + n - 1, 8, cudaMemcpyDeviceToHost, s));
    CV(cudaStreamSynchronize(s));
    uint32_t *ck = nullptr, *cvv = nullptr;
    CV(sc.get(&ck, (size_t)(lp + lk)));
    CV(sc.get(&cvv, (size_t)(lp + lk)));
    k_compact<<<blocks, threads, 0, s>>>(key, val, n, keep, pos, ck, cvv);
    CV(cudaGetLastError());
    key = ck;
    val = cvv;
    n = (int64_t)(lp + lk);
  } else {
    CV(radix_sort(key, val, k1, v1, n, bits, sc, s));
  }
  unsigned long long* deg = nullptr;
  CV(sc.get(&deg, (size_t)(V + 1)));
  CV(cudaMemsetAsync(deg, 0, sizeof(unsigned long long) * (size_t)(V + 1), s));
  k_degree<<<blocks, threads, 0, s>>>(key, n, deg);
  CV(cudaGetLastError());
  CV(exclusive_scan(deg, deg, V + 1, sc, s));
  std::vector<int64_t> beg((size_t)V + 1);
  std::vector<int32_t> col((size_t)std::max<int64_t>(n, 1));
  CV(cudaMemcpyAsync(beg.data(), deg, sizeof(int64_t) * (size_t)(V + 1), cudaMemcpyDeviceToHost,
                     s));
  if (n) CV(cudaMemcpyAsync(col.data(), val, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, s));
  CV(cudaStreamSynchronize(s));
#undef CV
  if (beg[(size_t)V] != n) return IBFS_ERR_CUDA;
  const ibfs_status ws = ibfs_write_csr(beg_path, csr_path, beg.data(), col.data(), V);
  if (ws != IBFS_OK) return ws;
  if (V_out) *V_out = V;
  if (E_out) *E_out = n;
  return IBFS_OK;
}
