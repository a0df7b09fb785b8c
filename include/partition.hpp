// Drop-in replacement of GSAP/partition.hpp for the SBP path.
//
//   template <typename T, typename V, typename W>
//   void partition(Graph<T, V, W>& g);                 // partition.hpp:852-954
//
// keeps its signature and its effect (g.partitions resized to N and filled
// with labels 0..B-1) and runs the B200 partitioner through sbp_partition()
// (include/sbp.h).  T, V must be 32-bit integers and W a 32-bit unsigned
// type, as in GSAP's instantiation <int, int, unsigned> (GSAP.cu:20).  GSAP
// ignores errors; this version throws std::runtime_error with the library's
// message.  partition_with(g, options, report) exposes the options and the
// run report.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "graph.hpp"
#include "sbp.h"

template <typename T, typename V, typename W>
void partition_with(Graph<T, V, W>& g, const sbp_options& o, sbp_report* report) {
  static_assert(sizeof(T) == 4 && sizeof(V) == 4 && sizeof(W) == 4 &&
                    std::is_unsigned<W>::value,
                "partition(): GSAP's <int, int, unsigned> graph types are required");
  const int N = g.N;
  // GSAP's adj_ptr has N entries; the ABI takes N+1
  std::vector<int32_t> optr(g.csr_out.adj_ptr.begin(), g.csr_out.adj_ptr.end());
  std::vector<int32_t> iptr(g.csr_in.adj_ptr.begin(), g.csr_in.adj_ptr.end());
  optr.push_back((int32_t)g.csr_out.adj_node.size());
  iptr.push_back((int32_t)g.csr_in.adj_node.size());
  sbp_graph_csr c;
  c.N = N;
  c.E = (int32_t)g.csr_out.adj_node.size();
  c.out_ptr = optr.data();
  c.out_idx = reinterpret_cast<const int32_t*>(g.csr_out.adj_node.data());
  c.out_w = reinterpret_cast<const uint32_t*>(g.csr_out.adj_wgt.data());
  c.in_ptr = iptr.data();
  c.in_idx = reinterpret_cast<const int32_t*>(g.csr_in.adj_node.data());
  c.in_w = reinterpret_cast<const uint32_t*>(g.csr_in.adj_wgt.data());
  c.deg_out = reinterpret_cast<const uint32_t*>(g.node_deg_out.data());
  c.deg_in = reinterpret_cast<const uint32_t*>(g.node_deg_in.data());
  g.partitions.resize(N);
  sbp_status st =
      sbp_partition(&c, &o, reinterpret_cast<int32_t*>(g.partitions.data()), report);
  if (st != SBP_OK)
    throw std::runtime_error(std::string("sbp_partition: ") + sbp_status_string(st) + ": " +
                             sbp_last_error());
}

template <typename T, typename V, typename W>
void partition(Graph<T, V, W>& g) {
  sbp_options o;
  sbp_default_options(&o);
  partition_with(g, o, nullptr);
}
