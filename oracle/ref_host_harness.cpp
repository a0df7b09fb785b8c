// Test infrastructure: runs the reference's host code (GSAP/load.hpp and
// GSAP/evaluate/eval.hpp, included from the reference tree by
// oracle/build_ref.sh) to produce golden vectors.
//
//   ref_host load <LL|LH|HL|HH> <1k|5k> <out.bin>
//       run from GSAP/ so that load.hpp's "../Dataset/static/" resolves;
//       writes N, E and the CSR arrays (int32 / uint32, little endian)
//   ref_host eval <n> <truth.bin> <given.bin>
//       prints the three figures evaluate.hpp prints (recall, precision, NMI)
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>
#include <chrono>

#include "graph.hpp"
#include "load.hpp"
#include "evaluate/eval.hpp"

template <typename X>
static void put(std::ofstream& f, const std::vector<X>& v) {
  int64_t n = (int64_t)v.size();
  f.write((const char*)&n, sizeof(n));
  f.write((const char*)v.data(), sizeof(X) * v.size());
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  std::string cmd = argv[1];
  if (cmd == "load" && argc == 5) {
    std::string cat = argv[2], size = argv[3];
    auto g = readFile<int, int, unsigned>(cat, size);
    std::ofstream f(argv[4], std::ios::binary);
    int32_t hdr[2] = {g.N, g.E};
    f.write((const char*)hdr, sizeof(hdr));
    put(f, g.csr_out.adj_ptr);
    put(f, g.csr_out.adj_node);
    put(f, g.csr_out.adj_wgt);
    put(f, g.csr_in.adj_ptr);
    put(f, g.csr_in.adj_node);
    put(f, g.csr_in.adj_wgt);
    put(f, g.node_deg_out);
    put(f, g.node_deg_in);
    put(f, g.truePartitions);
    return 0;
  }
  if (cmd == "eval" && argc == 5) {
    int n = std::atoi(argv[2]);
    std::vector<int> truth(n), given(n);
    std::ifstream a(argv[3], std::ios::binary), b(argv[4], std::ios::binary);
    a.read((char*)truth.data(), sizeof(int) * n);
    b.read((char*)given.data(), sizeof(int) * n);
    bf::evaluate<int>(truth, given);
    return 0;
  }
  return 2;
}
