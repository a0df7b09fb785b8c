// Runs GSAP's own blockmodel builder, calculate_new_csr (GSAP/partition.hpp:
// 707-849, with its bb_segsort, thrust and moderngpu steps), on given
// partitions of a graph and writes the CSR pair it builds, so that the
// oracle's and the partitioner's builders can be pinned to it bit for bit.
// Checker infrastructure: built by oracle/build_ref.sh into oracle/_ref/.
//
//   gsap_csr <graph.bin> <cases.bin> <out.bin>
//
// graph.bin: the file oracle/gsap_ref_main.cu reads.  cases.bin: int32
// count, then per case int32 B and N int32 labels in [0, B).  out.bin, per
// case: int32 B, nnz_out, nnz_in; out ptr (B), out col (nnz_out), out count
// (nnz_out), out degree (B); the same for the in CSR.  GSAP's row pointers
// have B entries (no end sentinel).
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <vector>

#include "GSAP/graph.hpp"
#include "GSAP/partition.hpp"

template <typename X>
static bool get(std::ifstream& f, std::vector<X>& v, size_t n) {
  v.resize(n);
  f.read((char*)v.data(), sizeof(X) * n);
  return (bool)f;
}

template <typename X>
static void put(std::ofstream& o, const X* p, size_t n) {
  o.write((const char*)p, sizeof(X) * n);
}

template <typename X>
static std::vector<X> down(const X* d, size_t n) {
  std::vector<X> h(n);
  if (n) cudaMemcpy(h.data(), d, sizeof(X) * n, cudaMemcpyDeviceToHost);
  return h;
}

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: gsap_csr <graph.bin> <cases.bin> <out.bin>\n");
    return 2;
  }
  std::ifstream f(argv[1], std::ios::binary);
  int32_t hdr[4];
  f.read((char*)hdr, sizeof(hdr));
  if (!f || hdr[0] != 0x53425047) {
    std::fprintf(stderr, "bad graph file\n");
    return 2;
  }
  const int N = hdr[1], E = hdr[2];
  std::vector<int32_t> optr, oidx, iptr, iidx;
  std::vector<uint32_t> ow, iw, dout, din;
  if (!(get(f, optr, N + 1) && get(f, oidx, E) && get(f, ow, E) && get(f, iptr, N + 1) &&
        get(f, iidx, E) && get(f, iw, E) && get(f, dout, N) && get(f, din, N))) {
    std::fprintf(stderr, "short graph file\n");
    return 2;
  }
  // Graph<int,int,unsigned> as load.hpp:86-117 fills it
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

  std::ifstream c(argv[2], std::ios::binary);
  int32_t ncases = 0;
  c.read((char*)&ncases, 4);
  std::ofstream o(argv[3], std::ios::binary);
  cudaStream_t s[15];
  for (int i = 0; i < 15; ++i) cudaStreamCreate(&s[i]);
  cudaStream_t st;
  cudaStreamCreate(&st);
  for (int k = 0; k < ncases; ++k) {
    int32_t B = 0;
    c.read((char*)&B, 4);
    std::vector<int32_t> labels;
    if (!c || B < 1 || B > N || !get(c, labels, N)) {
      std::fprintf(stderr, "bad cases file\n");
      return 2;
    }
    // device state sized as partition() sizes it (partition.hpp:863-888)
    Partition<int, int, unsigned> P;
    P.B = N;
    P.csr_out_node_size = E;
    P.csr_in_node_size = E;
    Gpu<int, int, unsigned> gpu;
    allocate_device_memory<int, int, unsigned>(gpu, g, P, N / 4, s, 10);
    cudaDeviceSynchronize();
    cudaMemcpy(gpu.partitions, labels.data(), sizeof(int) * N, cudaMemcpyHostToDevice);
    P.B = B;
    {
      mgpu::standard_context_t context(false);
      calculate_new_csr<int, int, unsigned>(P, gpu, g, context, s);
    }
    cudaError_t err = cudaDeviceSynchronize();
    if (err != cudaSuccess) {
      std::fprintf(stderr, "case %d: %s\n", k, cudaGetErrorString(err));
      return 3;
    }
    const int no = P.csr_out_node_size, ni = P.csr_in_node_size;
    int32_t head[3] = {B, no, ni};
    put(o, head, 3);
    put(o, down(gpu.csr_out_adj_ptr, B).data(), B);
    put(o, down(gpu.csr_out_adj_node, no).data(), no);
    put(o, down(gpu.csr_out_adj_wgt, no).data(), no);
    put(o, down(gpu.csr_out_deg, B).data(), B);
    put(o, down(gpu.csr_in_adj_ptr, B).data(), B);
    put(o, down(gpu.csr_in_adj_node, ni).data(), ni);
    put(o, down(gpu.csr_in_adj_wgt, ni).data(), ni);
    put(o, down(gpu.csr_in_deg, B).data(), B);
    deallocate_device_memory(gpu, st);
    cudaDeviceSynchronize();
    std::printf("{\"case\": %d, \"B\": %d, \"nnz_out\": %d, \"nnz_in\": %d}\n", k, B, no, ni);
    std::fflush(stdout);
  }
  return 0;
}
