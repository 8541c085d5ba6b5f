// host_graph.cpp -- CSR files, synthetic graph generators, source files and
// GroupBy on the host.  No CUDA here; OpenMP for the O(E) passes.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <new>
#include <numeric>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "internal.h"

namespace ibfs {

// ---------------------------------------------------------------------------
// CSR construction.
// ---------------------------------------------------------------------------
ibfs_status build_csr(const int32_t* u, const int32_t* v, int64_t m, int64_t V,
                      HostCsr* out) {
  if (V <= 0 || V >= INT32_MAX || m < 0) return IBFS_ERR_RANGE;
  try {
    std::vector<int64_t> deg(V + 1, 0);
    // Count both directions of every non-loop edge.
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; i++) {
      int32_t a = u[i], b = v[i];
      if (a == b) continue;
      __atomic_fetch_add(&deg[a], 1, __ATOMIC_RELAXED);
      __atomic_fetch_add(&deg[b], 1, __ATOMIC_RELAXED);
    }
    std::vector<int64_t> off(V + 1, 0);
    for (int64_t i = 0; i < V; i++) off[i + 1] = off[i] + deg[i];
    const int64_t total = off[V];
    std::vector<int32_t> adj((size_t)total);
    std::vector<int64_t> cur(off.begin(), off.end() - 1);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; i++) {
      int32_t a = u[i], b = v[i];
      if (a == b) continue;
      int64_t pa = __atomic_fetch_add(&cur[a], 1, __ATOMIC_RELAXED);
      adj[pa] = b;
      int64_t pb = __atomic_fetch_add(&cur[b], 1, __ATOMIC_RELAXED);
      adj[pb] = a;
    }
    // Sort + dedupe each list in place; record the unique length.
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t x = 0; x < V; x++) {
      int32_t* s = adj.data() + off[x];
      int32_t* e = adj.data() + off[x + 1];
      std::sort(s, e);
      deg[x] = std::unique(s, e) - s;
    }
    out->V = V;
    out->beg.assign(V + 1, 0);
    for (int64_t i = 0; i < V; i++) out->beg[i + 1] = out->beg[i] + deg[i];
    out->E = out->beg[V];
    out->col.resize((size_t)out->E);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t x = 0; x < V; x++)
      std::memcpy(out->col.data() + out->beg[x], adj.data() + off[x],
                  sizeof(int32_t) * (size_t)deg[x]);
  } catch (const std::bad_alloc&) {
    return IBFS_ERR_OOM;
  }
  return IBFS_OK;
}

ibfs_status validate_csr(const int64_t* beg, const int32_t* col, int64_t V,
                         int64_t E) {
  if (V <= 0 || V >= INT32_MAX || E < 0) return IBFS_ERR_RANGE;
  if (beg[0] != 0 || beg[V] != E) return IBFS_ERR_FORMAT;
  std::atomic<int> bad{0};
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < V; i++)
    if (beg[i + 1] < beg[i]) bad.store(1, std::memory_order_relaxed);
  if (bad.load()) return IBFS_ERR_FORMAT;
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < E; j++)
    if (col[j] < 0 || col[j] >= V) bad.store(1, std::memory_order_relaxed);
  return bad.load() ? IBFS_ERR_FORMAT : IBFS_OK;
}

// ---------------------------------------------------------------------------
// Binary CSR files: the reference's format (tuple_text_to_bin.cpp:149-152,
// 175-179, 220-228; read at graph_reader.cuh:63-119).  V = size(beg)/8 - 1,
// E = size(csr)/8, both little-endian uint64, beg[V] = E.  The reference
// asserts on short reads and narrows to int32 without checks; this loader
// returns a status instead and rejects ids >= 2^31.
// ---------------------------------------------------------------------------
static int64_t file_size(const char* p) {
  struct stat st;
  if (stat(p, &st) != 0) return -1;
  return (int64_t)st.st_size;
}

static ibfs_status read_u64_file(const char* path, std::vector<uint64_t>* buf) {
  int64_t sz = file_size(path);
  if (sz < 0) return IBFS_ERR_IO;
  if (sz % 8 != 0) return IBFS_ERR_FORMAT;
  FILE* f = std::fopen(path, "rb");
  if (!f) return IBFS_ERR_IO;
  try {
    buf->resize((size_t)(sz / 8));
  } catch (const std::bad_alloc&) {
    std::fclose(f);
    return IBFS_ERR_OOM;
  }
  size_t got = buf->empty() ? 0 : std::fread(buf->data(), 8, buf->size(), f);
  std::fclose(f);
  return got == buf->size() ? IBFS_OK : IBFS_ERR_IO;
}

ibfs_status load_csr_files(const char* beg_path, const char* csr_path,
                           HostCsr* out) {
  if (!beg_path || !csr_path || !out) return IBFS_ERR_INVALID_ARG;
  std::vector<uint64_t> b, c;
  ibfs_status s = read_u64_file(beg_path, &b);
  if (s != IBFS_OK) return s;
  s = read_u64_file(csr_path, &c);
  if (s != IBFS_OK) return s;
  if (b.size() < 2) return IBFS_ERR_FORMAT;
  const int64_t V = (int64_t)b.size() - 1, E = (int64_t)c.size();
  if (V >= INT32_MAX) return IBFS_ERR_RANGE;
  try {
    out->V = V;
    out->E = E;
    out->beg.resize(V + 1);
    out->col.resize((size_t)E);
  } catch (const std::bad_alloc&) {
    return IBFS_ERR_OOM;
  }
  std::atomic<int> bad{0};
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i <= V; i++) {
    if (b[i] > (uint64_t)INT64_MAX) bad.store(1, std::memory_order_relaxed);
    out->beg[i] = (int64_t)b[i];
  }
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < E; j++) {
    if (c[j] >= (uint64_t)V) bad.store(1, std::memory_order_relaxed);
    out->col[j] = (int32_t)c[j];
  }
  if (bad.load()) return IBFS_ERR_FORMAT;
  return validate_csr(out->beg.data(), out->col.data(), V, E);
}

// ---------------------------------------------------------------------------
// GroupBy on the host: exact restatement of GroupBy.cuh:19-84 (see the
// header comment of ibfs_groupby).  Degree limit 128 (GroupBy.cuh:25,30).
// ---------------------------------------------------------------------------
void groupby_host(const int64_t* beg, const int32_t* col, int64_t V,
                  const int32_t* src, int64_t n, int32_t* out) {
  const int64_t kHub = 128;
  std::vector<int32_t> hub_of((size_t)n, -1);
  std::vector<int64_t> count;  // per hub id, sparse through a sort below
  // Eligible: deg(src) <= 128 and a neighbour with deg > 128; the hub is the
  // first such neighbour in CSR order.
  for (int64_t i = 0; i < n; i++) {
    const int32_t s = src[i];
    if (beg[s + 1] - beg[s] > kHub) continue;
    for (int64_t j = beg[s]; j < beg[s + 1]; j++) {
      const int32_t h = col[j];
      if (beg[h + 1] - beg[h] > kHub) {
        hub_of[i] = h;
        break;
      }
    }
  }
  // Counting sort by hub id, stable in input order; O(n log n) over the
  // eligible sources instead of the reference's two V-sized arrays, same order.
  std::vector<int64_t> idx;
  idx.reserve((size_t)n);
  for (int64_t i = 0; i < n; i++)
    if (hub_of[i] >= 0) idx.push_back(i);
  std::stable_sort(idx.begin(), idx.end(),
                   [&](int64_t a, int64_t b) { return hub_of[a] < hub_of[b]; });
  int64_t k = 0;
  for (int64_t i : idx) out[k++] = src[i];
  for (int64_t i = 0; i < n; i++)
    if (hub_of[i] < 0) out[k++] = src[i];
  (void)V;
}

// A GroupBy variant (ibfs_opts.groupby = 3, not in the reference): the same
// eligibility (degree <= 128 with a neighbour of degree > 128), but the hub
// of a source is its HIGHEST-degree neighbour (ties: smaller id) instead of
// the first one in CSR order, and the groups come largest hub first.  Sources
// that share the biggest hubs then share batches whatever the CSR order.
void groupby_host_maxhub(const int64_t* beg, const int32_t* col, int64_t V,
                         const int32_t* src, int64_t n, int32_t* out) {
  const int64_t kHub = 128;
  std::vector<int32_t> hub_of((size_t)n, -1);
  for (int64_t i = 0; i < n; i++) {
    const int32_t s = src[i];
    if (beg[s + 1] - beg[s] > kHub) continue;
    int64_t best = kHub;
    for (int64_t j = beg[s]; j < beg[s + 1]; j++) {
      const int32_t h = col[j];
      const int64_t d = beg[h + 1] - beg[h];
      if (d > best || (d == best && d > kHub && h < hub_of[i])) {
        best = d;
        hub_of[i] = h;
      }
    }
  }
  std::vector<int64_t> idx;
  idx.reserve((size_t)n);
  for (int64_t i = 0; i < n; i++)
    if (hub_of[i] >= 0) idx.push_back(i);
  std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) {
    const int32_t ha = hub_of[a], hb = hub_of[b];
    const int64_t da = beg[ha + 1] - beg[ha], db = beg[hb + 1] - beg[hb];
    return da != db ? da > db : ha < hb;
  });
  int64_t k = 0;
  for (int64_t i : idx) out[k++] = src[i];
  for (int64_t i = 0; i < n; i++)
    if (hub_of[i] < 0) out[k++] = src[i];
  (void)V;
}

}  // namespace ibfs

using namespace ibfs;

// ---------------------------------------------------------------------------
// Generators.
// ---------------------------------------------------------------------------
static ibfs_status export_csr(HostCsr& h, int64_t** beg, int32_t** col,
                              int64_t* V, int64_t* E) {
  *beg = (int64_t*)std::malloc(sizeof(int64_t) * (size_t)(h.V + 1));
  *col = (int32_t*)std::malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(h.E, 1));
  if (!*beg || !*col) {
    std::free(*beg);
    std::free(*col);
    *beg = nullptr;
    *col = nullptr;
    return IBFS_ERR_OOM;
  }
  std::memcpy(*beg, h.beg.data(), sizeof(int64_t) * (size_t)(h.V + 1));
  if (h.E) std::memcpy(*col, h.col.data(), sizeof(int32_t) * (size_t)h.E);
  *V = h.V;
  *E = h.E;
  return IBFS_OK;
}

// Seeded bijection on `bits`-bit integers (odd multiply, add, xorshift
// rounds): relabels R-MAT vertices so ids carry no degree order.
static inline uint32_t perm_bits(uint32_t x, int bits, const uint64_t* mul,
                                 const uint64_t* add) {
  const uint64_t mask = (bits >= 32) ? 0xFFFFFFFFull : ((1ull << bits) - 1);
  uint64_t y = x;
  const int sh = bits / 2 + 1;
  for (int r = 0; r < 4; r++) {
    y = (y * mul[r] + add[r]) & mask;
    y ^= (y >> sh);
  }
  return (uint32_t)y;
}

extern "C" ibfs_status ibfs_gen_rmat(int32_t scale, int32_t edge_factor,
                                     double a, double b, double c,
                                     uint64_t seed, int64_t** beg,
                                     int32_t** col, int64_t* V, int64_t* E) {
  if (!beg || !col || !V || !E) return IBFS_ERR_INVALID_ARG;
  if (scale < 1 || scale > 30 || edge_factor < 1) return IBFS_ERR_RANGE;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return IBFS_ERR_INVALID_ARG;
  const int64_t nv = 1ll << scale;
  const int64_t m = nv * (int64_t)edge_factor;
  const double two32 = 4294967296.0;
  const uint64_t ta = (uint64_t)std::min(a * two32, two32);
  const uint64_t tab = (uint64_t)std::min((a + b) * two32, two32);
  const uint64_t tabc = (uint64_t)std::min((a + b + c) * two32, two32);
  uint64_t mul[4], add[4];
  for (int r = 0; r < 4; r++) {
    mul[r] = rnd(seed, 2, r) | 1ull;
    add[r] = rnd(seed, 3, r);
  }
  const int64_t draws = (scale + 1) / 2;
  std::vector<int32_t> us, vs;
  try {
    us.resize((size_t)m);
    vs.resize((size_t)m);
  } catch (const std::bad_alloc&) {
    return IBFS_ERR_OOM;
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; i++) {
    uint32_t x = 0, y = 0;
    int k = 0;
    for (int64_t d = 0; d < draws; d++) {
      const uint64_t h = rnd(seed, 1, (uint64_t)i * (uint64_t)draws + (uint64_t)d);
      for (int half = 0; half < 2 && k < scale; half++, k++) {
        const uint64_t r = (h >> (32 * half)) & 0xFFFFFFFFull;
        const uint32_t q = r < ta ? 0u : r < tab ? 1u : r < tabc ? 2u : 3u;
        x = (x << 1) | (q >> 1);
        y = (y << 1) | (q & 1u);
      }
    }
    us[i] = (int32_t)perm_bits(x, scale, mul, add);
    vs[i] = (int32_t)perm_bits(y, scale, mul, add);
  }
  HostCsr h;
  ibfs_status s = build_csr(us.data(), vs.data(), m, nv, &h);
  if (s != IBFS_OK) return s;
  return export_csr(h, beg, col, V, E);
}

extern "C" ibfs_status ibfs_gen_grid(int32_t rows, int32_t cols,
                                     double delete_frac, double shortcut_frac,
                                     uint64_t seed, int64_t** beg,
                                     int32_t** col, int64_t* V, int64_t* E) {
  if (!beg || !col || !V || !E) return IBFS_ERR_INVALID_ARG;
  if (rows < 1 || cols < 1 || (int64_t)rows * cols >= INT32_MAX)
    return IBFS_ERR_RANGE;
  if (delete_frac < 0 || delete_frac > 1 || shortcut_frac < 0)
    return IBFS_ERR_INVALID_ARG;
  const int64_t nv = (int64_t)rows * cols;
  const int64_t nh = (int64_t)rows * (cols - 1);
  const int64_t nvv = (int64_t)(rows - 1) * cols;
  const int64_t base = nh + nvv;
  const int64_t nsc = (int64_t)std::llround(shortcut_frac * (double)base);
  const uint64_t cut = (uint64_t)(delete_frac * 18446744073709551616.0 >= 18446744073709551615.0
                                      ? UINT64_MAX
                                      : delete_frac * 18446744073709551616.0);
  std::vector<int32_t> us, vs;
  try {
    us.resize((size_t)(base + nsc));
    vs.resize((size_t)(base + nsc));
  } catch (const std::bad_alloc&) {
    return IBFS_ERR_OOM;
  }
  // Deleted edges become self-loops, which build_csr drops.
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < base; e++) {
    int64_t x, y;
    if (e < nh) {
      const int64_t r = e / (cols - 1), cc = e % (cols - 1);
      x = r * cols + cc;
      y = x + 1;
    } else {
      const int64_t f = e - nh;
      x = f;
      y = f + cols;
    }
    const bool keep = rnd(seed, 5, (uint64_t)e) >= cut;
    us[e] = (int32_t)x;
    vs[e] = (int32_t)(keep ? y : x);
  }
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < nsc; j++) {
    us[base + j] = (int32_t)(rnd(seed, 6, 2 * (uint64_t)j) % (uint64_t)nv);
    vs[base + j] = (int32_t)(rnd(seed, 6, 2 * (uint64_t)j + 1) % (uint64_t)nv);
  }
  HostCsr h;
  ibfs_status s = build_csr(us.data(), vs.data(), base + nsc, nv, &h);
  if (s != IBFS_OK) return s;
  return export_csr(h, beg, col, V, E);
}

extern "C" ibfs_status ibfs_gen_chung_lu(int64_t n, int64_t m, double gamma,
                                         double max_degree, uint64_t seed,
                                         int64_t** beg, int32_t** col,
                                         int64_t* V, int64_t* E) {
  if (!beg || !col || !V || !E) return IBFS_ERR_INVALID_ARG;
  if (n < 2 || n >= INT32_MAX || m < 0 || gamma <= 1.0 || max_degree <= 0)
    return IBFS_ERR_RANGE;
  // Expected degrees w_i = C (i + i0)^(-p), p = 1/(gamma-1), with w_0 =
  // max_degree and mean 2m/n; i0 found by bisection.
  const double p = 1.0 / (gamma - 1.0);
  const double target = 2.0 * (double)m / (double)n;
  auto mean_for = [&](double i0) {
    const double C = max_degree * std::pow(i0, p);
    double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int64_t i = 0; i < n; i++) s += C * std::pow((double)i + i0, -p);
    return s / (double)n;
  };
  double lo = 1e-9, hi = (double)n * 1e3;
  if (mean_for(hi) < target) return IBFS_ERR_RANGE;
  for (int it = 0; it < 200; it++) {
    const double mid = std::sqrt(lo * hi);
    if (mean_for(mid) < target) lo = mid; else hi = mid;
  }
  const double i0 = hi, C = max_degree * std::pow(i0, p);
  std::vector<double> cum;
  std::vector<int32_t> us, vs, relabel;
  try {
    cum.resize((size_t)n);
    us.resize((size_t)m);
    vs.resize((size_t)m);
    relabel.resize((size_t)n);
  } catch (const std::bad_alloc&) {
    return IBFS_ERR_OOM;
  }
  double acc = 0;
  for (int64_t i = 0; i < n; i++) {
    acc += C * std::pow((double)i + i0, -p);
    cum[i] = acc;
  }
  const double total = acc;
  // Random relabelling so that vertex ids carry no degree order.
  {
    std::vector<std::pair<uint64_t, int32_t>> key((size_t)n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) key[i] = {rnd(seed, 7, (uint64_t)i), (int32_t)i};
    std::sort(key.begin(), key.end());
    for (int64_t i = 0; i < n; i++) relabel[key[i].second] = (int32_t)i;
  }
  auto draw = [&](uint64_t h) {
    const double r = (double)(h >> 11) * (1.0 / 9007199254740992.0) * total;
    int64_t k = std::upper_bound(cum.begin(), cum.end(), r) - cum.begin();
    if (k >= n) k = n - 1;
    return relabel[k];
  };
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < m; j++) {
    us[j] = draw(rnd(seed, 9, 2 * (uint64_t)j));
    vs[j] = draw(rnd(seed, 9, 2 * (uint64_t)j + 1));
  }
  HostCsr h;
  ibfs_status s = build_csr(us.data(), vs.data(), m, n, &h);
  if (s != IBFS_OK) return s;
  return export_csr(h, beg, col, V, E);
}

extern "C" ibfs_status ibfs_csr_read(const char* beg_path, const char* csr_path, int64_t** beg,
                                     int32_t** col, int64_t* V, int64_t* E) {
  if (!beg || !col || !V || !E) return IBFS_ERR_INVALID_ARG;
  HostCsr h;
  ibfs_status s = load_csr_files(beg_path, csr_path, &h);
  if (s != IBFS_OK) return s;
  return export_csr(h, beg, col, V, E);
}

extern "C" ibfs_status ibfs_csr_from_edges(const int32_t* src,
                                           const int32_t* dst, int64_t m,
                                           int64_t V, int64_t** beg,
                                           int32_t** col, int64_t* E) {
  if (!src || !dst || !beg || !col || !E) return IBFS_ERR_INVALID_ARG;
  for (int64_t i = 0; i < m; i++)
    if (src[i] < 0 || src[i] >= V || dst[i] < 0 || dst[i] >= V)
      return IBFS_ERR_RANGE;
  HostCsr h;
  ibfs_status s = build_csr(src, dst, m, V, &h);
  if (s != IBFS_OK) return s;
  int64_t v2;
  return export_csr(h, beg, col, &v2, E);
}

extern "C" ibfs_status ibfs_write_csr(const char* beg_path, const char* csr_path,
                                      const int64_t* beg, const int32_t* col,
                                      int64_t V) {
  if (!beg_path || !csr_path || !beg || (!col && beg[V] > 0) || V <= 0)
    return IBFS_ERR_INVALID_ARG;
  const int64_t E = beg[V];
  FILE* f = std::fopen(beg_path, "wb");
  if (!f) return IBFS_ERR_IO;
  std::vector<uint64_t> buf((size_t)std::min<int64_t>(V + 1, 1 << 20));
  bool ok = true;
  for (int64_t i = 0; i <= V && ok; i += (int64_t)buf.size()) {
    const int64_t k = std::min<int64_t>((int64_t)buf.size(), V + 1 - i);
    for (int64_t j = 0; j < k; j++) buf[j] = (uint64_t)beg[i + j];
    ok = std::fwrite(buf.data(), 8, (size_t)k, f) == (size_t)k;
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return IBFS_ERR_IO;
  f = std::fopen(csr_path, "wb");
  if (!f) return IBFS_ERR_IO;
  for (int64_t i = 0; i < E && ok; i += (int64_t)buf.size()) {
    const int64_t k = std::min<int64_t>((int64_t)buf.size(), E - i);
    for (int64_t j = 0; j < k; j++) buf[j] = (uint64_t)(uint32_t)col[i + j];
    ok = std::fwrite(buf.data(), 8, (size_t)k, f) == (size_t)k;
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? IBFS_OK : IBFS_ERR_IO;
}

// read_src_v (graph.cuh:99-133): one decimal vertex id per line.  Blank lines
// are skipped; anything else that is not an integer is a format error.
extern "C" ibfs_status ibfs_read_sources(const char* path, int32_t* ids,
                                         int64_t cap, int64_t* n) {
  if (!path || !n) return IBFS_ERR_INVALID_ARG;
  std::ifstream f(path);
  if (!f.good()) return IBFS_ERR_IO;
  std::string line;
  int64_t k = 0;
  while (std::getline(f, line)) {
    const char* p = line.c_str();
    while (*p == ' ' || *p == '\t' || *p == '\r') p++;
    if (!*p) continue;
    char* end = nullptr;
    errno = 0;
    long long x = std::strtoll(p, &end, 10);
    while (end && (*end == ' ' || *end == '\t' || *end == '\r')) end++;
    if (errno || end == p || (end && *end)) return IBFS_ERR_FORMAT;
    if (x < 0 || x >= INT32_MAX) return IBFS_ERR_RANGE;
    if (ids) {
      if (k >= cap) return IBFS_ERR_RANGE;
      ids[k] = (int32_t)x;
    }
    k++;
  }
  *n = k;
  return IBFS_OK;
}

extern "C" ibfs_status ibfs_write_sources(const char* path, const int32_t* ids,
                                          int64_t n) {
  if (!path || (!ids && n > 0)) return IBFS_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "w");
  if (!f) return IBFS_ERR_IO;
  for (int64_t i = 0; i < n; i++) std::fprintf(f, "%d\n", ids[i]);
  return std::fclose(f) == 0 ? IBFS_OK : IBFS_ERR_IO;
}

// Largest connected component by label propagation over a union-find.
static int32_t uf_find(std::vector<int32_t>& p, int32_t x) {
  while (p[x] != x) {
    p[x] = p[p[x]];
    x = p[x];
  }
  return x;
}

extern "C" ibfs_status ibfs_sample_sources(const int64_t* beg,
                                           const int32_t* col, int64_t V,
                                           int64_t n, uint64_t seed,
                                           int32_t component, int32_t* out) {
  if (!beg || !out || V <= 0 || n < 0) return IBFS_ERR_INVALID_ARG;
  std::vector<int32_t> cand;
  if (component < 0) {
    for (int64_t v = 0; v < V; v++)
      if (beg[v + 1] > beg[v]) cand.push_back((int32_t)v);
  } else {
    std::vector<int32_t> p((size_t)V);
    std::iota(p.begin(), p.end(), 0);
    for (int64_t v = 0; v < V; v++)
      for (int64_t j = beg[v]; j < beg[v + 1]; j++) {
        int32_t a = uf_find(p, (int32_t)v), b = uf_find(p, col[j]);
        if (a != b) p[std::max(a, b)] = std::min(a, b);
      }
    std::vector<int64_t> size((size_t)V, 0);
    for (int64_t v = 0; v < V; v++) size[uf_find(p, (int32_t)v)]++;
    int64_t best = 0;
    for (int64_t v = 1; v < V; v++)
      if (size[v] > size[best]) best = v;
    for (int64_t v = 0; v < V; v++)
      if (uf_find(p, (int32_t)v) == best) cand.push_back((int32_t)v);
  }
  if ((int64_t)cand.size() < n) return IBFS_ERR_RANGE;
  // Seeded partial Fisher-Yates: n distinct draws.
  const uint64_t cs = cand.size();
  for (int64_t i = 0; i < n; i++) {
    const uint64_t j = (uint64_t)i + rnd(seed, 8, (uint64_t)i) % (cs - (uint64_t)i);
    std::swap(cand[i], cand[j]);
    out[i] = cand[i];
  }
  return IBFS_OK;
}

extern "C" ibfs_status ibfs_groupby_csr(const int64_t* beg, const int32_t* col, int64_t V,
                                        const int32_t* src, int64_t n, int32_t* out) {
  if (!beg || (!col && beg[V] > 0) || V <= 0 || n < 0 || (n > 0 && (!src || !out)))
    return IBFS_ERR_INVALID_ARG;
  for (int64_t i = 0; i < n; i++)
    if (src[i] < 0 || src[i] >= V) return IBFS_ERR_RANGE;
  groupby_host(beg, col, V, src, n, out);
  return IBFS_OK;
}

// The largest-hub GroupBy variant (ibfs_opts.groupby = 3) on host arrays.
extern "C" ibfs_status ibfs_groupby_csr_maxhub(const int64_t* beg, const int32_t* col, int64_t V,
                                               const int32_t* src, int64_t n, int32_t* out) {
  if (!beg || (!col && beg[V] > 0) || V <= 0 || n < 0 || (n > 0 && (!src || !out)))
    return IBFS_ERR_INVALID_ARG;
  for (int64_t i = 0; i < n; i++)
    if (src[i] < 0 || src[i] >= V) return IBFS_ERR_RANGE;
  groupby_host_maxhub(beg, col, V, src, n, out);
  return IBFS_OK;
}

extern "C" void ibfs_free(void* p) { std::free(p); }

extern "C" ibfs_status ibfs_teps(const ibfs_graph* g, const void* depth_host,
                                 int64_t n, int32_t depth_bytes,
                                 int64_t* edges);
