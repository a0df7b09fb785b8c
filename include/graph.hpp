// Host graph types of GSAP's SBP path (GSAP/graph.hpp:8-45), kept so that a
// GSAP caller compiles unchanged against this library: Edge, Csr, Graph with
// the same members and meanings (adj_ptr holds N row starts with no end
// sentinel; node degrees are weighted sums; partitions is filled by
// partition(g)).  The device-side Gpu struct of GSAP (graph.hpp:97-220) has
// no counterpart: the device state lives behind include/sbp.h.
#pragma once

#include <set>
#include <utility>
#include <vector>

template <typename V, typename W>
struct Edge {
  V from;
  V to;
  W wgt;
  Edge(V f, V t, W w) : from(f), to(t), wgt(w) {}
};

template <typename T, typename V, typename W>
struct Csr {
  std::vector<T> adj_ptr;   // N row starts, no end sentinel
  std::vector<V> adj_node;
  std::vector<W> adj_wgt;
  std::vector<W> deg;
  void reset(int B) {
    adj_ptr.clear();
    adj_node.clear();
    adj_wgt.clear();
    deg.clear();
    deg.resize(B);
  }
};

template <typename T, typename V, typename W>
struct Graph {
  std::vector<V> partitions;      // output of partition(g): labels 0..B-1
  std::vector<V> truePartitions;  // planted labels, when known
  int N;
  int E;
  std::vector<Edge<V, W>> edges;
  std::vector<std::vector<std::pair<V, W>>> out_neighbors;
  std::vector<std::vector<std::pair<V, W>>> in_neighbors;
  Csr<T, V, W> csr_out;
  Csr<T, V, W> csr_in;
  std::vector<W> node_deg_out;
  std::vector<W> node_deg_in;
};
