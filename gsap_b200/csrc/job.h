// One partition job's device state and the host helpers shared by the
// one-shot entry points (driver.cu) and the multi-job engine (engine.cu).
#pragma once

#include "../../include/sbp.h"
#include "kernels.h"

#include <chrono>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

namespace sbp {

sbp_status fail(sbp_status st, const std::string& msg);

#define SBP_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e__ = (call);                                                           \
    if (e__ != cudaSuccess)                                                             \
      return fail(SBP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
  } while (0)

struct Arena {
  char* base = nullptr;
  size_t cap = 0, off = 0;
  template <typename T>
  T* take(size_t n) {
    size_t bytes = ((n * sizeof(T)) + 255) & ~size_t(255);
    if (off + bytes > cap) return nullptr;
    T* p = (T*)(base + off);
    off += bytes;
    return p;
  }
};

// Everything one partition job keeps in HBM.  A full job owns two streams
// (the one-shot entry points launch on them); a lean job (admitted by the
// engine) has only its arena, from the stream-ordered pool, and works on the
// engine's stream.
struct Job {
  int device = 0;
  bool lean = false;
  cudaStream_t st = nullptr;
  cudaStream_t pool_stream = nullptr;  // arena from the stream-ordered allocator
  int32_t N = 0, E = 0, np = 10, max_itr = 100;
  void* mem = nullptr;
  size_t mem_bytes = 0;
  DevGraph g;
  DevBM m;
  RebuildScratch rs;
  int32_t *part = nullptr, *newlab = nullptr, *props = nullptr, *best = nullptr, *map = nullptr;
  int32_t* snap[3] = {nullptr, nullptr, nullptr};
  double *rec = nullptr, *mdS = nullptr, *best_dS = nullptr;
  double* mdsin = nullptr;      // merge in-row terms by proposal slot (MergeGrid)
  MergeApplyBufs ma;            // merge application scratch (mergeapply.cu)
  int32_t* ma_out = nullptr;    // new block count, target-out-of-range flag
  int32_t* lists = nullptr;     // batch indices by nodal kernel path (classify_batch)
  int32_t* err = nullptr;       // nodal error counter (hash-table overflow)
  int32_t* ctl = nullptr;       // sweep control: sweeps done in the outer step, stop flag
  CommitScratch cs;
  int32_t dense_cap = 0;        // largest B the dense arrays can hold
  int32_t dense_eff = 0;        // largest B kept in dense form in this run
  cudaStream_t side = nullptr;  // heavy vertices run here, next to the warp kernel
  cudaEvent_t fork = nullptr, join = nullptr;
  double* dsum = nullptr;       // per nodal iteration (or batch): sum of recorded dS
  double* dataS = nullptr;      // per nodal iteration: MDL data term
  long long* acc = nullptr;     // per nodal iteration (or batch): applied moves
  // pinned host mirrors (the one-shot merge step)
  int32_t* h_best = nullptr;
  double* h_best_dS = nullptr;
  int32_t* h_map = nullptr;
  std::vector<int32_t> h_optr, h_iptr;  // host copies of the graph's row pointers

  Job() = default;
  Job(const Job&) = delete;
  Job& operator=(const Job&) = delete;
  ~Job() { release(); }
  void release();
};

sbp_status validate_graph(const sbp_graph_csr* g);
// The DCSBM generator's planted labels and out-degree CDF (host.cpp), the
// stages the host and device generators share.
sbp_status dcsbm_labels(const sbp_dcsbm_params* p, std::vector<int32_t>& truth,
                        std::vector<double>& cdf);
sbp_status validate_part(const int32_t* part, int32_t N, int32_t B);
int resolve_device(int32_t d);
// Device arena bytes of a job (the engine's HBM admission test uses it).
size_t job_bytes(int32_t N, int32_t E, int32_t np, int32_t max_itr, int32_t dense_cap);
sbp_status job_create(Job& J, int device, int32_t N, int32_t E, int32_t np, int32_t max_itr,
                      int32_t dense_max, bool lean = false, cudaStream_t engine_stream = nullptr);
// Copies the graph to the job's arena (on J.st) and keeps host row pointers.
sbp_status job_upload(Job& J, const sbp_graph_csr* h);
// The process-wide x log2 x table of a device (filled once).
sbp_status device_xlx_table(int device, const double** out);
// Returns the new block count, or -1 when a target lies outside [0, B).
int32_t apply_merges_host(int32_t B, int32_t B_to_merge, const int32_t* best,
                          const double* best_dS, int32_t* map_out);
// Model term of the MDL: GSAP's (partition.hpp:696-699, Q6) or, exact = 1,
// the standard description length's in bits (exact mode searches B on it).
double model_S(int32_t B, int32_t N, int32_t E, int32_t exact = 0);

// Largest B kept in the dense B x B form: dense_max when it is >= 0, else
// (the default) max(4096, sqrt(32 E)), so that above B = 4096 the two
// matrices take at most about 256 bytes per edge; never more than N.  A
// rebuild of the CSR form after every batch costs O(E); the dense form's
// per-sweep terms cost O(B^2), so the crossover grows with E.
int32_t dense_limit(int32_t N, int32_t E, int32_t dense_max);

// Whether GSAP's merge grid is reproduced (sbp_options.ref_grid).
inline bool ref_grid_on(const sbp_options& o) {
  return o.ref_grid < 0 ? o.exact == 0 : o.ref_grid != 0;
}
// The persistent merge buffers of a job as a MergeGrid.
inline MergeGrid merge_grid(const Job& J, const sbp_options& o) {
  MergeGrid g;
  g.on = ref_grid_on(o) ? 1 : 0;
  g.dS = J.mdS;
  g.dsin = J.mdsin;
  return g;
}

inline ScoreMode score_mode(const sbp_options& o) {
  ScoreMode m;
  m.exact = o.exact;
  m.mh = o.mh;
  m.beta = o.beta;
  return m;
}
bool heavy_vertex(const Job& J, int32_t v);
// Appends the batch indices i in [0, count) of vertices lo + i (verts[i]
// when verts is given) to `out`, grouped by nodal kernel path: small, mid,
// heavy (NodalAux); n[k] receives the group sizes.
void classify_batch(const Job& J, const int32_t* verts, int32_t lo, int32_t count,
                    std::vector<int32_t>& out, int32_t n[3]);
// The NodalAux of groups of sizes n[3] stored back to back at `dev`.
NodalAux nodal_lists(Job& J, const int32_t* dev, const int32_t n[3]);
sbp_status check_options(const sbp_options* o);

struct Timer {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
        .count();
  }
};

struct Bracket {
  int32_t B = 0;
  int32_t B_to_merge = 0;
  double S = std::numeric_limits<double>::infinity();
  int slot = -1;  // snapshot buffer holding its labels
};

// partition() of one job through the engine (engine.cu); the job holds the
// uploaded graph.
sbp_status run_solo(Job& J, const sbp_options& o, int32_t* labels_out, sbp_report* rep);
// sbp_nodal_sweeps through the engine: `sweeps` sweeps at a fixed B from the
// job's current labels, per-batch dS sums into sums[].
sbp_status run_sweeps(Job& J, int32_t B, uint64_t seed, uint32_t seq0, int32_t num_batches,
                      int32_t sweeps, double* sums);

}  // namespace sbp
