// Drop-in replacement of GSAP/load.hpp: readFile<T, V, W>(cat, size) reads
// "../Dataset/static/<category>/<size>/<N>_nodes.tsv" and its
// "_truePartition.tsv" relative to the working directory, exactly as
// load.hpp:6-133 does (same parse, N = largest source id, rows in file
// order, weighted degrees).  readFileAt() takes the dataset root instead and
// readTsv() any TSV path.  Errors throw std::runtime_error where GSAP calls
// std::exit.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "graph.hpp"
#include "sbp.h"

template <typename T, typename V, typename W>
Graph<T, V, W> readTsv(const std::string& path, const std::string& truth_path) {
  sbp_edges* e = nullptr;
  sbp_status st = sbp_load_tsv(path.c_str(), truth_path.empty() ? nullptr : truth_path.c_str(), &e);
  if (st != SBP_OK) throw std::runtime_error(std::string("readTsv: ") + sbp_last_error());
  int32_t N = 0, E = 0;
  sbp_edges_size(e, &N, &E);
  std::vector<int32_t> src(E), dst(E), truth(N);
  std::vector<uint32_t> w(E);
  sbp_edges_copy(e, src.data(), dst.data(), w.data(), truth.data());
  sbp_edges_free(e);
  Graph<T, V, W> g;
  g.N = N;
  g.E = E;
  for (int32_t j = 0; j < E; ++j) g.edges.emplace_back(src[j] + 1, dst[j] + 1, w[j]);
  std::vector<int32_t> optr(N + 1), iptr(N + 1);
  g.csr_out.adj_node.resize(E);
  g.csr_out.adj_wgt.resize(E);
  g.csr_in.adj_node.resize(E);
  g.csr_in.adj_wgt.resize(E);
  g.node_deg_out.resize(N);
  g.node_deg_in.resize(N);
  st = sbp_csr_from_edges(N, E, src.data(), dst.data(), w.data(), optr.data(),
                          reinterpret_cast<int32_t*>(g.csr_out.adj_node.data()),
                          reinterpret_cast<uint32_t*>(g.csr_out.adj_wgt.data()), iptr.data(),
                          reinterpret_cast<int32_t*>(g.csr_in.adj_node.data()),
                          reinterpret_cast<uint32_t*>(g.csr_in.adj_wgt.data()),
                          reinterpret_cast<uint32_t*>(g.node_deg_out.data()),
                          reinterpret_cast<uint32_t*>(g.node_deg_in.data()));
  if (st != SBP_OK) throw std::runtime_error(std::string("readTsv: ") + sbp_last_error());
  g.csr_out.adj_ptr.assign(optr.begin(), optr.end() - 1);
  g.csr_in.adj_ptr.assign(iptr.begin(), iptr.end() - 1);
  g.out_neighbors.resize(N);
  g.in_neighbors.resize(N);
  for (int32_t j = 0; j < E; ++j) {
    g.out_neighbors[src[j]].emplace_back(dst[j], w[j]);
    g.in_neighbors[dst[j]].emplace_back(src[j], w[j]);
  }
  if (!truth_path.empty()) g.truePartitions.assign(truth.begin(), truth.end());
  return g;
}

inline std::string sbp_dataset_base(const std::string& ca, const std::string& num) {
  std::string f;
  if (ca == "LL") f = "lowOverlap_lowBlockSizeVar/";
  else if (ca == "LH") f = "lowOverlap_highBlockSizeVar/";
  else if (ca == "HL") f = "highOverlap_lowBlockSizeVar/";
  else if (ca == "HH") f = "highOverlap_highBlockSizeVar/";
  else throw std::runtime_error("usage: [LL/LH/HL/HH] [1k/5k/20k/50k/200k/1m]");
  if (num == "1k") f += "1k/1000_nodes";
  else if (num == "5k") f += "5k/5000_nodes";
  else if (num == "20k") f += "20k/20000_nodes";
  else if (num == "50k") f += "50k/50000_nodes";
  else if (num == "200k") f += "200k/200000_nodes";
  else if (num == "1m") f += "1m/1000000_nodes";
  else throw std::runtime_error("usage: [LL/LH/HL/HH] [1k/5k/20k/50k/200k/1m]");
  return f;
}

template <typename T, typename V, typename W>
Graph<T, V, W> readFileAt(const std::string& root, const std::string& ca, const std::string& num) {
  std::string base = root + "/" + sbp_dataset_base(ca, num);
  return readTsv<T, V, W>(base + ".tsv", base + "_truePartition.tsv");
}

template <typename T, typename V, typename W>
Graph<T, V, W> readFile(std::string& ca, std::string& num) {
  return readFileAt<T, V, W>("../Dataset/static", ca, num);
}
