// ref_harness.cu -- runs the reference's own host-side code on our inputs.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/build_ref.sh from the reference
// sources where they lie (never copied into this repository) into
// oracle/_ref/ref_harness.  It exposes the reference functions that have a
// CPU implementation, so that the oracle restatement (oracle/oracle.c) and
// the library's host code can be checked against the real thing:
//
//   load   <beg.bin> <csr.bin> <out_beg.i32> <out_csr.i32>
//          graph_reader::graph_reader (graph_reader.cuh:63-119): the uint64
//          files narrowed to int32, dumped raw
//   groupby <beg.bin> <csr.bin> <src.txt> <out.txt>
//          GroupBy<int,int> (GroupBy.cuh:6-115) on the reader's CSR
//   report  <beg.bin> <csr.bin> <depth.u8> <n>
//          report<> (validate.h:59-76) per source row of a [n][V] uint8
//          depth file; prints "<traversed_vertices> <traversed_edges>" per row
//   validate <beg.bin> <csr.bin> <depth.u8> <n>
//          validate<> (validate.h:2-56) per row; prints its return code
//   deep2   <beg.bin> <csr.bin> <src.txt>
//          deep_than_two (graph.cuh:28-70, the level-1-limited queue BFS);
//          prints 1/0 per source
//
// The reference's GPU kernels are compiled along (the headers include them)
// but never launched: nothing here touches a GPU.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "graph.h"
#include "graph_reader.h"

static std::vector<int> read_ids(const char* path) {
  std::vector<int> v;
  std::ifstream f(path);
  long long x;
  while (f >> x) v.push_back((int)x);
  return v;
}

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: ref_harness <cmd> <beg.bin> <csr.bin> ...\n");
    return 2;
  }
  const std::string cmd = argv[1];
  graph_reader* g = new graph_reader(argv[2], argv[3], 1);
  const index_t V = g->vert_count;
  std::vector<index_t> card(V);
  for (index_t i = 0; i < V; i++) card[i] = g->beg_pos[i + 1] - g->beg_pos[i];

  if (cmd == "load" && argc >= 6) {
    FILE* fb = std::fopen(argv[4], "wb");
    FILE* fc = std::fopen(argv[5], "wb");
    std::fwrite(g->beg_pos, sizeof(index_t), (size_t)V + 1, fb);
    std::fwrite(g->csr, sizeof(vertex_t), (size_t)g->edge_count, fc);
    std::fclose(fb);
    std::fclose(fc);
    return 0;
  }
  if (cmd == "groupby" && argc >= 6) {
    std::vector<int> src = read_ids(argv[4]);
    std::vector<int> out(src.size());
    CSR_Graph cg;
    std::memset(&cg, 0, sizeof(cg));
    cg.vert_count = V;
    cg.edge_count = g->edge_count;
    cg.beg_pos = g->beg_pos;
    cg.adj_list = g->csr;
    cg.adj_card = card.data();
    GroupBy<vertex_t, index_t>((index_t)src.size(), src.data(), out.data(), &cg);
    FILE* fo = std::fopen(argv[5], "w");
    for (int x : out) std::fprintf(fo, "%d\n", x);
    std::fclose(fo);
    return 0;
  }
  if ((cmd == "report" || cmd == "validate") && argc >= 6) {
    const long long n = std::atoll(argv[5]);
    std::vector<depth_t> d((size_t)V * n);
    FILE* fd = std::fopen(argv[4], "rb");
    if (!fd || std::fread(d.data(), 1, d.size(), fd) != d.size()) return 3;
    std::fclose(fd);
    for (long long i = 0; i < n; i++) {
      depth_t* row = d.data() + (size_t)i * V;
      if (cmd == "report") {
        index_t edges = 0, verts = 0;
        report<vertex_t, index_t, depth_t>(edges, verts, row, card.data(), V);
        std::printf("%d %d\n", (int)verts, (int)edges);
      } else {
        std::printf("%d\n", (int)validate<index_t, vertex_t, depth_t>(row, g->csr, card.data(),
                                                                     g->beg_pos, V));
      }
    }
    return 0;
  }
  if (cmd == "deep2" && argc >= 5) {
    std::vector<int> src = read_ids(argv[4]);
    std::vector<vertex_t> qa(V), qb(V);
    std::vector<depth_t> depth(V);
    for (int s : src) {
      std::memset(depth.data(), INFTY, (size_t)V);
      const bool r = deep_than_two<vertex_t, index_t>(s, qa.data(), qb.data(), depth.data(),
                                                      card.data(), g->beg_pos, g->csr);
      std::printf("%d\n", r ? 1 : 0);
    }
    return 0;
  }
  std::fprintf(stderr, "bad command\n");
  return 2;
}
