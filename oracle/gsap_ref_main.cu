// Drives the unmodified GSAP GPU path (graph.hpp + partition.hpp from the
// reference tree) on a graph file written by write_graph_bin (oracle/oracle.py
// or gsap_b200/sbp.py, the same format), for the reference arm of bench.py.
// Built by oracle/build_ref.sh into oracle/_ref/gsap_ref; the binary is all
// that later runs need, not the sources of the reference.
//
//   gsap_ref <graph.bin> <runs> <labels_out.bin>
//
// Builds Graph<int,int,unsigned> the way load.hpp:6-133 does (adj_ptr with
// N entries and no end sentinel, node degrees as weighted sums), then times
// partition(g) + cudaDeviceSynchronize() with steady_clock like GSAP.cu:24-30,
// `runs` times, printing one JSON line per run.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "GSAP/graph.hpp"
#include "GSAP/partition.hpp"

template <typename X>
static bool get(std::ifstream& f, std::vector<X>& v, size_t n) {
  v.resize(n);
  f.read((char*)v.data(), sizeof(X) * n);
  return (bool)f;
}

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: gsap_ref <graph.bin> <runs> <labels_out.bin>\n");
    return 2;
  }
  std::ifstream f(argv[1], std::ios::binary);
  int32_t hdr[4];
  f.read((char*)hdr, sizeof(hdr));
  if (!f || hdr[0] != 0x53425047) {
    std::fprintf(stderr, "bad graph file\n");
    return 2;
  }
  int N = hdr[1], E = hdr[2];
  std::vector<int32_t> optr, oidx, iptr, iidx;
  std::vector<uint32_t> ow, iw, dout, din;
  bool ok = get(f, optr, N + 1) && get(f, oidx, E) && get(f, ow, E) && get(f, iptr, N + 1) &&
            get(f, iidx, E) && get(f, iw, E) && get(f, dout, N) && get(f, din, N);
  if (!ok) {
    std::fprintf(stderr, "short graph file\n");
    return 2;
  }
  int runs = std::atoi(argv[2]);
  Graph<int, int, unsigned> g;
  g.N = N;
  g.E = E;
  g.csr_out.adj_ptr.assign(optr.begin(), optr.begin() + N);
  g.csr_out.adj_node.assign(oidx.begin(), oidx.end());
  g.csr_out.adj_wgt.assign(ow.begin(), ow.end());
  g.csr_in.adj_ptr.assign(iptr.begin(), iptr.begin() + N);
  g.csr_in.adj_node.assign(iidx.begin(), iidx.end());
  g.csr_in.adj_wgt.assign(iw.begin(), iw.end());
  g.node_deg_out.assign(dout.begin(), dout.end());
  g.node_deg_in.assign(din.begin(), din.end());
  for (int r = 0; r < runs; ++r) {
    auto begin = std::chrono::steady_clock::now();
    partition(g);
    cudaError_t err = cudaDeviceSynchronize();
    auto end = std::chrono::steady_clock::now();
    double ms = std::chrono::duration<double, std::milli>(end - begin).count();
    int B = 0;
    for (int v : g.partitions) B = v + 1 > B ? v + 1 : B;
    std::printf("{\"run\": %d, \"ms\": %.3f, \"B\": %d, \"cuda\": \"%s\"}\n", r, ms, B,
                cudaGetErrorString(err));
    std::fflush(stdout);
    if (err != cudaSuccess) return 3;
  }
  std::ofstream o(argv[3], std::ios::binary);
  o.write((const char*)g.partitions.data(), sizeof(int) * g.partitions.size());
  return 0;
}
