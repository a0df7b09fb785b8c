// A GSAP-style caller (GSAP.cu:7-34) built against include/: reads a TSV
// with readTsv, calls partition(g) and writes g.partitions.
#include <cstdio>
#include <fstream>
#include <string>

#include "load.hpp"
#include "partition.hpp"

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  auto g = readTsv<int, int, unsigned>(argv[1], "");
  partition(g);
  std::ofstream o(argv[2], std::ios::binary);
  o.write((const char*)g.partitions.data(), sizeof(int) * g.partitions.size());
  int B = 0;
  for (int v : g.partitions) B = v + 1 > B ? v + 1 : B;
  std::printf("N=%d E=%d B=%d\n", g.N, g.E, B);
  return 0;
}
