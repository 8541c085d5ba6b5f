// convert_cli.cpp -- tuple_text_to_bin: the reference's edge-list converter
// command line (tuple_text_to_bin.cpp:56-70) over ibfs_convert_text.
//
//   tuple_text_to_bin <tuple_file> <reverse 1|0> <lines_to_skip> [--clean] [--device D]
//
// Writes <tuple_file>_beg_pos.bin and <tuple_file>_csr.bin next to the input,
// as the reference does.  --clean symmetrises, drops self loops and
// deduplicates (the reference keeps the file's edges as they are).
#include <cstdio>
#include <cstdlib>
#include <string>

#include "ibfs.h"

int main(int argc, char** argv) {
  std::printf("Input: ./exe tuple_file(text) reverse_the_edge(1 reverse, 0 not reverse) "
              "lines_to_skip [--clean] [--device D]\n");
  if (argc < 4) {
    std::printf("Wrong input\n");
    return -1;
  }
  int clean = 0, device = 0;
  for (int i = 4; i < argc; i++) {
    const std::string a = argv[i];
    if (a == "--clean") clean = 1;
    else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
    else {
      std::printf("Wrong input: unknown option %s\n", a.c_str());
      return -1;
    }
  }
  const std::string in = argv[1];
  const int reverse = std::atol(argv[2]) == 1;
  const long long skip = std::atoll(argv[3]);
  int64_t V = 0, E = 0;
  const ibfs_status s = ibfs_convert_text(in.c_str(), reverse, skip, clean,
                                          (in + "_beg_pos.bin").c_str(), (in + "_csr.bin").c_str(),
                                          device, &V, &E);
  if (s != IBFS_OK) {
    std::printf("error: %s\n", ibfs_strerror(s));
    return -1;
  }
  std::printf("edge count: %lld\nvert count: %lld\n", (long long)E, (long long)V);
  return 0;
}
