// Test infrastructure: runs GSAP's own kernels (GSAP/kernels.hpp, included
// from the reference tree by oracle/build_ref.sh) on the host, so that the
// oracle's dS restatements can be checked against the reference's code on the
// same inputs.  Blockmodel inputs use the reference layout: row pointers with
// B entries and the nnz count as the end of the last row (kernels.hpp:161-166).
#include "cuda_emul.h"
#include "kernels.hpp"

#include <algorithm>
#include <cstring>
#include <vector>

emu_dim3 threadIdx{0, 0, 0}, blockIdx{0, 0, 0}, blockDim{1, 1, 1};

template <typename F>
static void launch(unsigned n, F f) {
  blockIdx.x = 0;
  blockDim.x = 1;
  for (unsigned i = 0; i < n; ++i) {
    threadIdx.x = i;
    f();
  }
}

typedef int T;
typedef int V;
typedef unsigned W;

extern "C" {

// calculate_dS_out (kernels.hpp:143-182) for every block.
void ref_dS_out(int B, const int* ptr, const int* col, const unsigned* cnt, const unsigned* d_out,
                const unsigned* d_in, long nnz, float* out) {
  launch((unsigned)B, [&] {
    calculate_dS_out<T, V, W>(out, (T*)ptr, (V*)col, (W*)cnt, (W*)d_out, (W*)d_in, B, (size_t)nnz);
  });
}

// One nodal batch through the reference's kernel sequence
// (partition.hpp:537-649): neighbour blocks, per-vertex sort (bb_segsort's
// result), r/s in-weights, the seven dS terms and the accept kernel.  props
// is indexed by vertex (proposed_blocks_nodal).  Writes the seven term
// arrays (BS each, in the order dS_out_nodal[B] first, then in_r, in_s,
// new_r_out, new_s_out, new_r_in, new_s_in) and the accepted dS;
// part is updated in place as the reference does.
void ref_nodal_batch(int N, int E, const int* g_out_ptr, const int* g_out_idx, const unsigned* g_out_w,
                     const int* g_in_ptr, const int* g_in_idx, const unsigned* g_in_w,
                     const unsigned* node_deg_out, const unsigned* node_deg_in, int B,
                     const int* o_ptr, const int* o_col, const unsigned* o_cnt, const int* i_ptr,
                     const int* i_col, const unsigned* i_cnt, long nnz, const unsigned* d_out,
                     const unsigned* d_in, int* part, const int* props, int BS, int itr,
                     float* dS_out_blocks, float* terms7, float* dS_acc) {
  // buffers sized one past their data: the reference reads one element past
  // a row (kernels.hpp:1224 and similar; 1351)
  std::vector<int> gob(E + 1, -1), gib(E + 1, -1);
  std::vector<unsigned> gow(g_out_w, g_out_w + E), giw(g_in_w, g_in_w + E);
  gow.push_back(0);
  giw.push_back(0);
  std::vector<int> optr(o_ptr, o_ptr + B), iptr(i_ptr, i_ptr + B);
  std::vector<int> ocol(o_col, o_col + nnz), icol(i_col, i_col + nnz);
  std::vector<unsigned> ocnt(o_cnt, o_cnt + nnz), icnt(i_cnt, i_cnt + nnz);
  ocol.push_back(-1); icol.push_back(-1); ocnt.push_back(0); icnt.push_back(0);
  std::vector<int> gop(g_out_ptr, g_out_ptr + N), gip(g_in_ptr, g_in_ptr + N);
  std::vector<int> goi(g_out_idx, g_out_idx + E), gii(g_in_idx, g_in_idx + E);
  std::vector<unsigned> dout(d_out, d_out + B), din(d_in, d_in + B);
  std::vector<unsigned> kdo(node_deg_out, node_deg_out + N), kdi(node_deg_in, node_deg_in + N);
  std::vector<int> pr(props, props + N);
  std::vector<unsigned> rw(N, 0), sw(N, 0);
  float* t_in_r = terms7 + 0 * (size_t)BS;
  float* t_in_s = terms7 + 1 * (size_t)BS;
  float* t_r_out = terms7 + 2 * (size_t)BS;
  float* t_s_out = terms7 + 3 * (size_t)BS;
  float* t_r_in = terms7 + 4 * (size_t)BS;
  float* t_s_in = terms7 + 5 * (size_t)BS;
  launch((unsigned)N, [&] {
    match_neighbored_block_out<T, V, W>(gop.data(), goi.data(), (size_t)E, gob.data(), part, N);
  });
  launch((unsigned)N, [&] {
    match_neighbored_block_in<T, V, W>(gip.data(), gii.data(), (size_t)E, gib.data(), part, N);
  });
  // bb_segsort(keys=blocks, vals=weights) per vertex segment (partition.hpp:546-547)
  auto segsort = [&](std::vector<int>& ptr, std::vector<int>& key, std::vector<unsigned>& val) {
    for (int v = 0; v < N; ++v) {
      int b = ptr[v], e = v + 1 < N ? ptr[v + 1] : E;
      std::vector<std::pair<int, unsigned>> kv;
      for (int j = b; j < e; ++j) kv.push_back({key[j], val[j]});
      std::sort(kv.begin(), kv.end());
      for (int j = b; j < e; ++j) { key[j] = kv[j - b].first; val[j] = kv[j - b].second; }
    }
  };
  segsort(gop, gob, gow);
  segsort(gip, gib, giw);
  launch((unsigned)B, [&] {
    calculate_dS_out<T, V, W>(dS_out_blocks, optr.data(), ocol.data(), ocnt.data(), dout.data(),
                              din.data(), B, (size_t)nnz);
  });
  launch((unsigned)BS, [&] {
    calculate_dS_in_nodal_r<T, V, W>(t_in_r, iptr.data(), icol.data(), icnt.data(), din.data(),
                                     dout.data(), part, pr.data(), BS, itr, B, N, (size_t)nnz);
  });
  launch((unsigned)BS, [&] {
    calculate_dS_in_nodal_s<T, V, W>(t_in_s, iptr.data(), icol.data(), icnt.data(), din.data(),
                                     dout.data(), part, pr.data(), BS, itr, B, N, (size_t)nnz);
  });
  launch((unsigned)BS, [&] {
    find_csr_in_r_wgt<T, V, W>(rw.data(), part, gip.data(), gib.data(), (size_t)E, giw.data(), BS,
                               itr, B, N);
  });
  launch((unsigned)BS, [&] {
    calculate_dS_new_r_out_nodal_new<T, V, W>(t_r_out, part, pr.data(), optr.data(), ocol.data(),
                                              (size_t)nnz, ocnt.data(), gop.data(), gob.data(),
                                              (size_t)E, gow.data(), kdo.data(), din.data(),
                                              dout.data(), rw.data(), BS, itr, B, N);
  });
  launch((unsigned)BS, [&] {
    find_csr_in_s_wgt<T, V, W>(sw.data(), pr.data(), gip.data(), gib.data(), (size_t)E, giw.data(),
                               BS, itr, B, N);
  });
  launch((unsigned)BS, [&] {
    calculate_dS_new_s_out_nodal_new<T, V, W>(t_s_out, part, pr.data(), optr.data(), ocol.data(),
                                              (size_t)nnz, ocnt.data(), gop.data(), gob.data(),
                                              (size_t)E, gow.data(), kdo.data(), din.data(),
                                              dout.data(), sw.data(), BS, itr, B, N);
  });
  launch((unsigned)BS, [&] {
    calculate_dS_new_r_in_nodal_new<T, V, W>(t_r_in, part, pr.data(), iptr.data(), icol.data(),
                                             (size_t)nnz, icnt.data(), gip.data(), gib.data(),
                                             (size_t)E, giw.data(), kdi.data(), din.data(),
                                             dout.data(), BS, itr, B, N);
  });
  launch((unsigned)BS, [&] {
    calculate_dS_new_s_in_nodal_new<T, V, W>(t_s_in, part, pr.data(), iptr.data(), icol.data(),
                                             (size_t)nnz, icnt.data(), gip.data(), gib.data(),
                                             (size_t)E, giw.data(), kdi.data(), din.data(),
                                             dout.data(), BS, itr, B, N);
  });
  launch((unsigned)BS, [&] {
    calculate_dS_overall_nodal<V, W>(dS_acc, t_r_in, t_s_in, t_s_out, t_r_out, t_in_r, t_in_s,
                                     dS_out_blocks, part, pr.data(), BS, itr, B, N);
  });
}

// Merge dS of all B*np proposals through calculate_dS_out, calculate_dS_in,
// calculate_dS_new_out, calculate_dS_new_in and calculate_dS_overall
// (partition.hpp:392-435).
void ref_merge_delta(int B, int np, const int* o_ptr, const int* o_col, const unsigned* o_cnt,
                     const int* i_ptr, const int* i_col, const unsigned* i_cnt, long nnz,
                     const unsigned* d_out, const unsigned* d_in, const int* props, float* dS) {
  std::vector<int> optr(o_ptr, o_ptr + B), iptr(i_ptr, i_ptr + B);
  std::vector<int> ocol(o_col, o_col + nnz), icol(i_col, i_col + nnz);
  std::vector<unsigned> ocnt(o_cnt, o_cnt + nnz), icnt(i_cnt, i_cnt + nnz);
  std::vector<unsigned> dout(d_out, d_out + B), din(d_in, d_in + B);
  std::vector<int> pr(props, props + (size_t)B * np);
  std::vector<float> dso(B), dsi((size_t)B * np), dno((size_t)B * np), dni((size_t)B * np);
  std::vector<int> best(B);
  launch((unsigned)B, [&] {
    calculate_dS_out<T, V, W>(dso.data(), optr.data(), ocol.data(), ocnt.data(), dout.data(),
                              din.data(), B, (size_t)nnz);
  });
  unsigned tB = (unsigned)(B * np);
  launch(tB, [&] {
    calculate_dS_in<T, V, W>(dsi.data(), iptr.data(), icol.data(), icnt.data(), din.data(),
                             dout.data(), pr.data(), B, (size_t)nnz, np);
  });
  launch(tB, [&] {
    calculate_dS_new_out<T, V, W>(dno.data(), pr.data(), optr.data(), ocol.data(), ocnt.data(),
                                  dout.data(), din.data(), B, (size_t)nnz, np);
  });
  launch(tB, [&] {
    calculate_dS_new_in<T, V, W>(dni.data(), pr.data(), iptr.data(), icol.data(), icnt.data(),
                                 din.data(), dout.data(), B, (size_t)nnz, np);
  });
  launch(tB, [&] {
    calculate_dS_overall<T, V, W>(dS, dso.data(), dsi.data(), dno.data(), dni.data(), optr.data(),
                                  ocol.data(), ocnt.data(), dout.data(), din.data(), pr.data(),
                                  best.data(), B, np);
  });
}

// data_S of compute_overall_entropy_cuda (kernels.hpp:1034-1093), summed in
// index order in double, and the model term of partition.hpp:696-701 in float.
void ref_mdl(int B, int N, int E, const int* o_ptr, const int* o_col, const unsigned* o_cnt, long nnz,
             const unsigned* d_out, const unsigned* d_in, double* data_S, float* S) {
  std::vector<int> optr(o_ptr, o_ptr + B), ocol(o_col, o_col + nnz);
  std::vector<unsigned> ocnt(o_cnt, o_cnt + nnz), dout(d_out, d_out + B), din(d_in, d_in + B);
  std::vector<unsigned> mo(nnz), mi(nnz);
  std::vector<float> terms(nnz);
  launch((unsigned)B, [&] {
    block_deg_mapping<T, V, W>(optr.data(), ocol.data(), (size_t)nnz, ocnt.data(), mo.data(),
                               mi.data(), dout.data(), din.data(), B);
  });
  launch((unsigned)nnz, [&] {
    compute_overall_S_transform<T, V, W>(optr.data(), ocol.data(), (size_t)nnz, ocnt.data(),
                                         terms.data(), mo.data(), mi.data(), B);
  });
  double acc = 0.0;
  for (long i = 0; i < nnz; ++i) acc += terms[i];
  *data_S = acc;
  float model_S_term = (float)B * B / E;
  float model_S = (float)(E * (1 + model_S_term) * std::log(1 + model_S_term)) -
                  (model_S_term * std::log(model_S_term)) + (N * std::log(B));
  *S = model_S - (float)acc;
}

// calculate_accepted_prob (kernels.hpp:709-723).
void ref_accepted_prob(int B, const unsigned* d_out, const unsigned* d_in, float* out) {
  std::vector<unsigned> dout(d_out, d_out + B), din(d_in, d_in + B);
  launch((unsigned)B, [&] { calculate_accepted_prob<W>(out, dout.data(), din.data(), B); });
}

}  // extern "C"
