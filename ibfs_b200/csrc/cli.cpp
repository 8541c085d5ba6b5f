// cli.cpp -- gpu_ibfs: the drop-in command line of the reference
// (ibfs.cu:52-105, main.cpp:7-20) over the C ABI of libibfs.
//
//   gpu_ibfs <beg_pos.bin> <csr.bin> <concurrent-count> <switch-level> <bfs_count> [options]
//
// Positional arguments keep the reference's meaning (ibfs.cu:58-67):
//   concurrent-count  sources per batch (1..width; the reference requires 128)
//   switch-level      top-down while level <= switch-level, bottom-up after
//                     (-1: alpha/beta switching, not in the reference)
//   bfs_count         number of sources
// A wrong argument count prints the usage and exits with -1 like the
// reference (ibfs.cu:63).  Each batch prints "Traversal-iter-<i>: <t>
// second(s)" (reporter.cpp:10).
//
// Options:
//   --sources FILE     read_src_v file (graph.cuh:99-133); default: seeded
//                      sample of non-isolated vertices (--seed)
//   --depth-out FILE   binary depths, [bfs_count][V] in source-file order,
//                      uint8 (INFTY 255) or uint16 when a level exceeds 254
//   --width W          status bits per vertex: 32, 64, 128, 256 (default 128)
//   --alpha A --beta B direction-switch parameters (with switch-level -1)
//   --thresholds S,L   degree thresholds of the small/large queues (32,512)
//   --groupby          reorder sources with GroupBy before batching
//   --groupby-device   the same order, computed on the GPU
//   --plain            host-driven level loop (default: the library's AUTO
//                      schedule -- the persistent kernel on small graphs,
//                      the device loop on large ones)
//   --device-loop      kernel per phase, level loop on the device (CUDA graph
//                      conditional nodes)
//   --batched          all batches in one launch (CUDA graph), one report
//   --bu-filter M      bottom-up frontier filter: 1 every level, 0 off,
//                      -1 per level (default)
//   --td-stage         stage large vertices' chunks in shared memory (TMA)
//   --sparse-push D    push sources below 1/D of the average frontier
//                      top-down on a bottom-up level (default off)
//   --repeat K         run the whole set K times (timing)
//   --device D, --seed S, --depth-bytes 1|2, --vertex-major
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ibfs.h"

static void usage() {
  std::printf("Input: /path/to/exe /path/to/beg /path/to/csr concurrent-count switch-level "
              "bfs_count [--sources F] [--depth-out F] [--width W] [--alpha A] [--beta B] "
              "[--thresholds S,L] [--groupby] [--groupby-device] [--plain] [--device-loop] [--batched] "
              "[--bu-filter M] [--td-stage] [--sparse-push D] [--repeat K] [--device D] "
              "[--seed S] [--depth-bytes 1|2] [--vertex-major]\n");
}

static int fail(const char* what, ibfs_status s) {
  std::fprintf(stderr, "%s: %s\n", what, ibfs_strerror(s));
  return 1;
}

int main(int argc, char** argv) {
  usage();
  if (argc < 6) {
    std::printf("Wrong input\n");
    return -1;
  }
  const char* beg_file = argv[1];
  const char* csr_file = argv[2];
  const int concurrent = std::atoi(argv[3]);
  const int switch_level = std::atoi(argv[4]);
  const long long bfs_count = std::atoll(argv[5]);
  std::string sources, depth_out;
  ibfs_opts o;
  ibfs_opts_default(&o);
  o.switch_level = switch_level;
  int device = 0, repeat = 1, layout = IBFS_LAYOUT_SOURCE_MAJOR;
  bool batched = false;
  unsigned long long seed = 1;
  for (int i = 6; i < argc; i++) {
    const std::string a = argv[i];
    auto next = [&](const char* name) -> const char* {
      if (i + 1 >= argc) {
        std::printf("Wrong input: %s needs a value\n", name);
        std::exit(-1);
      }
      return argv[++i];
    };
    if (a == "--sources") sources = next("--sources");
    else if (a == "--depth-out") depth_out = next("--depth-out");
    else if (a == "--width") o.width = std::atoi(next("--width"));
    else if (a == "--alpha") o.alpha = (float)std::atof(next("--alpha"));
    else if (a == "--beta") o.beta = (float)std::atof(next("--beta"));
    else if (a == "--thresholds") {
      const char* v = next("--thresholds");
      if (std::sscanf(v, "%d,%d", &o.sml_shed, &o.lrg_shed) != 2) {
        std::printf("Wrong input: --thresholds S,L\n");
        return -1;
      }
    } else if (a == "--groupby") o.groupby = 1;
    else if (a == "--groupby-device") o.groupby = 2;
    else if (a == "--plain") o.mode = IBFS_MODE_PLAIN;
    else if (a == "--device-loop") o.mode = IBFS_MODE_DEVICE_LOOP;
    else if (a == "--batched") batched = true;
    else if (a == "--bu-filter") o.bu_filter = std::atoi(next("--bu-filter"));
    else if (a == "--td-stage") o.td_stage = 1;
    else if (a == "--sparse-push") o.sparse_push = std::atoi(next("--sparse-push"));
    else if (a == "--repeat") repeat = std::atoi(next("--repeat"));
    else if (a == "--device") device = std::atoi(next("--device"));
    else if (a == "--seed") seed = std::strtoull(next("--seed"), nullptr, 10);
    else if (a == "--depth-bytes") o.depth_bytes = std::atoi(next("--depth-bytes"));
    else if (a == "--vertex-major") layout = IBFS_LAYOUT_VERTEX_MAJOR;
    else {
      std::printf("Wrong input: unknown option %s\n", a.c_str());
      return -1;
    }
  }
  if (concurrent < 1 || concurrent > o.width || bfs_count < 1) {
    std::printf("Wrong input: concurrent-count must be 1..%d and bfs_count >= 1\n", o.width);
    return -1;
  }
  o.concurrent = concurrent;
  if (batched) o.use_graph = 1;

  const auto t0 = std::chrono::steady_clock::now();
  ibfs_graph* g = nullptr;
  ibfs_status s = ibfs_graph_open(beg_file, csr_file, device, &g);
  if (s != IBFS_OK) return fail("graph load", s);
  int64_t V = 0, E = 0, maxd = 0;
  ibfs_graph_info(g, &V, &E, &maxd);
  std::printf("Graph load (success): %lld verts, %lld edges %.3f second(s)\n", (long long)V,
              (long long)E,
              std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());

  std::vector<int32_t> src;
  if (!sources.empty()) {
    int64_t n = 0;
    if ((s = ibfs_read_sources(sources.c_str(), nullptr, 0, &n)) != IBFS_OK)
      return fail("source file", s);
    src.resize((size_t)n);
    if ((s = ibfs_read_sources(sources.c_str(), src.data(), n, &n)) != IBFS_OK)
      return fail("source file", s);
    if ((long long)src.size() < bfs_count) {
      std::printf("Wrong input: %s holds %zu sources, bfs_count is %lld\n", sources.c_str(),
                  src.size(), bfs_count);
      return -1;
    }
    src.resize((size_t)bfs_count);
  } else {
    int64_t *hb = nullptr;
    int32_t* hc = nullptr;
    int64_t v2 = 0, e2 = 0;
    if ((s = ibfs_csr_read(beg_file, csr_file, &hb, &hc, &v2, &e2)) != IBFS_OK)
      return fail("graph read", s);
    src.resize((size_t)bfs_count);
    s = ibfs_sample_sources(hb, hc, v2, bfs_count, seed, -1, src.data());
    ibfs_free(hb);
    ibfs_free(hc);
    if (s != IBFS_OK) return fail("source sampling", s);
  }
  for (int32_t x : src)
    if (x < 0 || x >= V) {
      std::printf("Wrong input: source %d out of range\n", x);
      return -1;
    }

  // Output buffer: the whole set, source-major in source-file order.
  int db = o.depth_bytes ? o.depth_bytes : 1;
  std::vector<uint8_t> depth;
  const int64_t n = (int64_t)src.size();
  double total_s = 0;
  int64_t edges = 0;
  int max_level = 0;
  for (int rep = 0; rep < repeat; rep++) {
    for (;;) {
      depth.assign((size_t)n * (size_t)V * db, 0);
      ibfs_opts ob = o;
      ob.depth_bytes = db;
      s = IBFS_OK;
      edges = 0;
      total_s = 0;
      max_level = 0;
      const int64_t step = batched ? n : concurrent;
      for (int64_t b0 = 0; b0 < n && s == IBFS_OK; b0 += step) {
        const int64_t nb = std::min<int64_t>(step, n - b0);
        ibfs_stats st;
        std::memset(&st, 0, sizeof(st));
        const auto tb = std::chrono::steady_clock::now();
        s = ibfs_run(g, src.data() + b0, nb, &ob, depth.data() + (size_t)b0 * V * db, layout, 0,
                     &st);
        const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - tb)
                              .count();
        if (s != IBFS_OK) break;
        total_s += dt;
        edges += st.traversed_edges;
        max_level = std::max(max_level, st.max_level);
        if (batched)
          std::printf("Traversal-all-%lld-batches: %.6f second(s) (device %.6f)\n",
                      (long long)st.n_batches, dt, st.device_ms / 1e3);
        else
          std::printf("Traversal-iter-%lld: %.6f second(s)\n", (long long)(b0 / concurrent), dt);
      }
      if (s == IBFS_ERR_RANGE && o.depth_bytes == 0 && db == 1) {
        db = 2;  // a level exceeded 254: widen the depth type
        continue;
      }
      break;
    }
    if (s != IBFS_OK) return fail("traversal", s);
  }
  std::printf("Sources: %lld  max level: %d  traversed edges: %lld  time: %.6f s  "
              "TEPS (Billion): %.3f\n",
              (long long)n, max_level, (long long)edges, total_s,
              total_s > 0 ? edges / total_s / 1e9 : 0.0);
  if (!depth_out.empty()) {
    FILE* f = std::fopen(depth_out.c_str(), "wb");
    if (!f) return fail("depth-out", IBFS_ERR_IO);
    const size_t w = std::fwrite(depth.data(), 1, depth.size(), f);
    if (std::fclose(f) != 0 || w != depth.size()) return fail("depth-out", IBFS_ERR_IO);
    std::printf("Depths (%s, %d byte(s) each, [%lld][%lld]) written to %s\n",
                layout == IBFS_LAYOUT_SOURCE_MAJOR ? "source-major" : "vertex-major", db,
                (long long)n, (long long)V, depth_out.c_str());
  }
  ibfs_graph_close(g);
  return 0;
}
