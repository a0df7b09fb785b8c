// Host-side declarations of the partitioner's kernels and the device state
// they work on.  All launches go to one stream; nothing here synchronises.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <vector>

namespace sbp {

// Kernels launched by this thread through the launchers below (the bench's
// launch count).
extern thread_local long long g_launches;

// The graph in HBM (uploaded once per job).
struct DevGraph {
  int32_t N = 0, E = 0;
  int32_t *optr = nullptr, *oidx = nullptr, *iptr = nullptr, *iidx = nullptr;
  uint32_t *ow = nullptr, *iw = nullptr, *kdo = nullptr, *kdi = nullptr;
  int32_t *osrc = nullptr, *isrc = nullptr;  // owning vertex of each CSR entry
};

// Blockmodel M (out CSR rows = source block, in CSR rows = destination
// block), weighted block degrees and their log2, and the per-block sums the
// dS kernels start from.  Capacities: rows N+1, entries E.
struct DevBM {
  int32_t *optr = nullptr, *ocol = nullptr, *iptr = nullptr, *icol = nullptr;
  uint32_t *ocnt = nullptr, *icnt = nullptr, *d_out = nullptr, *d_in = nullptr;
  double *ld_out = nullptr, *ld_in = nullptr;
  double *dSout = nullptr;    // sum over out-row b of M (log2 M - log2 d_out[b] - log2 d_in[c])
  double *ambout = nullptr;   // sum over out-row b of M log2 M - M log2 d_in[c]
  double *ambin = nullptr;    // sum over in-row b of M log2 M - M log2 d_out[c]
  double *sinfull = nullptr;  // ambin[b] - d_in[b] log2 d_in[b]
  int32_t* nbr_s = nullptr;   // per-block second-hop sample of a nodal batch
  uint8_t* use_rand = nullptr;
  // dense form for small B: Md[r*B + c] = M[r][c], MTd[c*B + r] = M[r][c]
  uint32_t* Md = nullptr;
  uint32_t* MTd = nullptr;
  // chunk sums of the dense rows, 32 columns a chunk, K = ceil(B/32):
  // Sd[b*2K + j] = sum of Md[b][32j..32j+31], Sd[b*2K + K + j] the same
  // over MTd[b] (the in-row); kept with Md and MTd by the same atomics
  uint32_t* Sd = nullptr;
  // xlx[x] = x log2 x and xlx[kXlxTable + x] = log2 x for x < kXlxTable
  // (filled by fill_xlx_table)
  double* xlx = nullptr;
};

// Fills the x log2 x table of a job.
void fill_xlx_table(double* tab, cudaStream_t st);

// Scratch of the multi-CTA commit (partial sums of each CTA, a ticket).
struct CommitScratch {
  double* part_sum = nullptr;
  long long* part_cnt = nullptr;
  unsigned* ticket = nullptr;  // must be 0 between commits
};
constexpr int kCommitCtas = 256;

// Scratch of one rebuild direction.
struct RebuildDir {
  int32_t *cnt = nullptr, *seg = nullptr, *vofs = nullptr, *tcol = nullptr, *uniq = nullptr;
  uint32_t* tw = nullptr;
  int32_t* ucol = nullptr;
  uint32_t* uw = nullptr;
  int32_t* big = nullptr;
};

struct RebuildScratch {
  RebuildDir d[2];
  int32_t* big_count = nullptr;  // 2 ints
  int32_t* tile = nullptr;       // scan tile sums (capacity >= 2 * tiles)
  int32_t tile_cap = 0;
};

// Launch shape of a rebuild (the autotuner's choice; results never depend
// on it): segments longer than warp_cap entries are reduced by a CTA,
// big_ctas CTAs per direction (0: 296 at most) take one per big_entries graph
// entries.
struct RebuildTune {
  int32_t warp_cap = 256;
  int32_t big_ctas = 0;
  int32_t big_entries = 2048;
};

// How a nodal move is scored and accepted.  exact = 0: GSAP's dS terms
// (kernels.hpp:494-643, 1153-1726, quirks kept); 1: the exact change of the
// MDL.  mh = 0: accept iff dS < 0 (kernels.hpp:634-640); 1: Metropolis-
// Hastings with inverse temperature beta (dS in bits) and the Hastings
// ratio of GSAP's proposal.  Anything but (0, 0) runs the general-mode
// kernels; the merge phase reads only `exact`.
struct ScoreMode {
  int32_t exact = 0, mh = 0;
  double beta = 3.0;
  bool general() const { return exact != 0 || mh != 0; }
  int slot(bool dense) const { return (dense ? 1 : 0) + (general() ? 2 : 0); }
};

// ------------------------------------------------------ multi-job launches --
// One launch of a kernel body over many jobs: `args` holds njobs argument
// records back to back, job j owns virtual blocks [cta0[j], cta0[j+1]).
struct MultiSpan {
  const void* args = nullptr;
  const int32_t* cta0 = nullptr;
  int32_t njobs = 0, total = 0;
};

struct MultiKernel {
  size_t rec_bytes;
  void (*launch)(const MultiSpan&, cudaStream_t);
  void (*launch_one)(const void* rec, int32_t vctas, cudaStream_t);
  const char* name;
};

// A multi-job launch being assembled on the host: records and offsets.
struct Slot {
  const MultiKernel* k = nullptr;
  bool mismatch = false;  // records of two different kernels were added
  std::vector<unsigned char> recs;
  std::vector<int32_t> cta0 = std::vector<int32_t>(1, 0);
  bool empty() const { return cta0.size() <= 1; }
  int32_t njobs() const { return (int32_t)cta0.size() - 1; }
  int32_t total() const { return cta0.back(); }
  void clear() {
    k = nullptr;
    mismatch = false;
    recs.clear();
    cta0.assign(1, 0);
  }
};

inline Slot& slot_bind(Slot& s, const MultiKernel& k) {
  if (s.k && s.k != &k) s.mismatch = true;
  s.k = &k;
  return s;
}

// The launches of a blockmodel rebuild, in order.
struct RebuildSlots {
  Slot zero, count, scan1[3], scatter, rows_small, rows_big, scan2[3], compact;
  Slot dense_count, dense_fill;  // the CSR form from a fresh dense form instead
  void clear();
  std::vector<Slot*> all();
};

// The launches of a dense-form build, in order.
struct DenseBuildSlots {
  Slot zero, edges, mapped, degrees, logs;
  void clear();
  std::vector<Slot*> all();
};

// Record builders: each adds one job's launch record(s) to the slot(s), with
// a virtual grid that depends on that job's sizes only.  `ctl` (optional)
// is the job's sweep control (int32 pair in device memory: sweeps done in
// the outer step, stop flag): a gated launch does nothing once the stop
// flag is set, and takes its RNG sequence as seq + ctl[0] * seq_mul and its
// result slot as slot + ctl[0] * slot_mul.
void add_rebuild(RebuildSlots& s, const DevGraph& g, const int32_t* part, int32_t B, DevBM& m,
                 RebuildScratch& rs, const int32_t* ctl = nullptr,
                 const RebuildTune& t = RebuildTune{});
// The CSR form of the current labels from their dense form (which must hold
// them): the rebuild's outputs from O(B^2) cells instead of the edges.
void add_csr_from_dense(RebuildSlots& s, int32_t B, DevBM& m, RebuildScratch& rs);
// The dense form right after a merge step: from the CSR blockmodel of the
// labels before it (B_old blocks, still in m's CSR arrays) and the merge map.
void add_dense_build_mapped(DenseBuildSlots& s, const DevGraph& g, const int32_t* part,
                            int32_t B, DevBM& m, int32_t B_old, const int32_t* map);
void add_dense_build(DenseBuildSlots& s, const DevGraph& g, const int32_t* part, int32_t B,
                     DevBM& m);
void add_dense_update(Slot& s, const DevGraph& g, const int32_t* part, int32_t lo, int32_t count,
                      const int32_t* newlab, int32_t B, DevBM& m, const int32_t* ctl = nullptr);
void add_block_terms(Slot& s, DevBM& m, int32_t B, int draws, uint64_t seed, uint32_t seq,
                     const int32_t* ctl = nullptr, uint32_t seq_mul = 0);
void add_block_terms_dense(Slot& s, DevBM& m, int32_t B, int draws, uint64_t seed,
                           uint32_t seq, const int32_t* ctl = nullptr, uint32_t seq_mul = 0);
// data_S into out[ctl[0]] (out[0] without ctl).
void add_mdl_sum(Slot& s, const DevBM& m, int32_t B, double* out, const int32_t* ctl = nullptr);
// The stop test after a queued sweep (window 0: count sweeps to max_itr).
void add_sweep_ctl(Slot& s, int32_t* ctl, const double* dsum, const double* dataS,
                   double model_S, double thr, int32_t window, int32_t max_itr);
void add_zero(Slot& s, void* p, size_t words, const int32_t* ctl = nullptr);
void add_copy(Slot& s, void* dst, const void* src, size_t words);
void add_iota(Slot& s, int32_t* p, int32_t n);
// Nodal batch of one job: the warp kernel's record goes to `warp`, the
// CTA-per-vertex kernel's (heavy vertices) to `heavy`.  Use separate slots
// per md.slot(dense): dense and CSR jobs, GSAP-mode and general-mode jobs
// run different kernels.
struct NodalAux;
void add_nodal(Slot& warp, Slot& heavy, bool dense, const ScoreMode& md, const DevGraph& g,
               const int32_t* part,
               const DevBM& m, int32_t B, uint64_t seed, uint32_t seq, int32_t lo, int32_t count,
               int32_t* newlab, double* rec, int32_t* props, const NodalAux& lists,
               const int32_t* ctl = nullptr, uint32_t seq_mul = 0);
// With draw_next (dense mode), the commit's extra CTAs also make the next
// batch's per-block draws (the block-terms kernel's draws == 1 work) with RNG
// sequence draw_seq + ctl[0] * draw_seq_mul, from M after the batch's moves.
void add_commit(Slot& s, int32_t* part, int32_t lo, int32_t count, const int32_t* newlab,
                const double* rec, double* slot_sum, long long* slot_acc, const DevBM* dense_m,
                int32_t B, const CommitScratch& cs, const int32_t* ctl = nullptr,
                int32_t slot_mul = 0, bool draw_next = false, uint64_t seed = 0,
                uint32_t draw_seq = 0, uint32_t draw_seq_mul = 0);
// GSAP's merge grid (Q16, partition.hpp:335-336): when `on`, only the
// proposal slots below the nnz of the out CSR, rounded up to 256, are drawn
// and scored; the others keep the targets, dS (dS) and in-row terms (dsin)
// their slots hold from earlier merge steps of the run (zero at its start).
// Arrays of N * np entries that persist over the run.
struct MergeGrid {
  int32_t on = 0;
  double* dS = nullptr;
  double* dsin = nullptr;
};

void add_merge_props(Slot& s, const DevBM& m, int32_t B, int32_t np, uint64_t seed, uint32_t seq,
                     int32_t* props, const MergeGrid& grid = MergeGrid());
// E: the graph's edge count, which picks the dS kernel: jobs with short
// blockmodel rows go to slot s8 (a warp per block, groups of 8 lanes per
// proposal), the others to s32 (a warp per proposal, into grid.dS) and
// sbest (each block's best).  Without grid.dS, dS is the scratch.
void add_merge_delta(Slot& s32, Slot& s8, Slot& sbest, const DevBM& m, int32_t B, int32_t E,
                     int32_t np,
                     const int32_t* props, double* dS, int32_t* best, double* best_dS,
                     int32_t exact = 0, const MergeGrid& grid = MergeGrid());
void add_relabel(Slot& s, int32_t* part, int32_t N, const int32_t* map);

// Merge application on the device (mergeapply.cu): the scratch of one job
// (merge_apply_bytes(N) bytes, carved by merge_apply_carve), the launches of
// one merge application in order, and the one-shot form.  map[b] receives
// the new label of block b, out[0] the new block count and out[1] = 1 when a
// target lay outside [0, B) (out[] must start at zero).
struct MergeApplyBufs {
  uint64_t *key = nullptr, *mkA = nullptr, *mkB = nullptr;
  int32_t *jA = nullptr, *jB = nullptr, *miA = nullptr, *miB = nullptr;
  uint8_t* onc = nullptr;
  int32_t *pA = nullptr, *pB = nullptr, *root = nullptr, *newid = nullptr, *tile = nullptr;
  uint32_t* hist = nullptr;
  int32_t* sel = nullptr;
};
constexpr int kMaRounds = 31, kMaSelPasses = 8;
struct MergeApplySlots {
  Slot fused;  // the whole application in one CTA (small B)
  Slot keys, cyc[kMaRounds], mark, hist[kMaSelPasses], pick[kMaSelPasses], parent,
      rootj[kMaRounds], scan[3], map;
  void clear();
  std::vector<Slot*> all();
};
size_t merge_apply_bytes(int32_t N);
MergeApplyBufs merge_apply_carve(void* base, int32_t N);
void add_merge_apply(MergeApplySlots& s, const MergeApplyBufs& w, int32_t B, int32_t K,
                     const int32_t* best, const double* best_dS, int32_t* map, int32_t* out);
void merge_apply(const MergeApplyBufs& w, int32_t B, int32_t K, const int32_t* best,
                 const double* best_dS, int32_t* map, int32_t* out, cudaStream_t st);
// Exclusive scan records (three slots: tile sums, one-CTA scan, apply);
// out[n] receives the total; tile needs 2 * ceil(n / 2048) + 2 entries.
void add_exclusive_scan(Slot* sl, const int32_t* in, int32_t* out, int32_t n, int32_t* tile);

// Tuned shape for a device and a blockmodel size class, if known.
bool rebuild_tuned(int device, int32_t E, int32_t B, RebuildTune* out);
// Times the candidate shapes on this blockmodel (labels `part` must be in
// [0, B)), caches and returns the fastest.  Synchronises the stream.
cudaError_t tune_rebuild(int device, const DevGraph& g, const int32_t* part, int32_t B, DevBM& m,
                         RebuildScratch& rs, cudaStream_t st, RebuildTune* out);

// Opt-in shared-memory sizes; call once per device before the first launch.
cudaError_t init_kernel_attributes();

// Exclusive scan of n int32 counts into out[0..n] (out[n] = total).
void scan_exclusive(const int32_t* in, int32_t* out, int32_t n, int32_t* tile, cudaStream_t st);

// ---------------------------------------------------------------- ingest --
// Stable sort of n non-negative keys (at most max_key): keys_out ascending,
// vals_out[p] = input position of the p-th key, equal keys in input order.
// scratch: sort_scratch_bytes(n).
size_t sort_scratch_bytes(int32_t n);
cudaError_t sort_by_key_stable(const int32_t* keys, int32_t n, int32_t max_key,
                               int32_t* keys_out, int32_t* vals_out, void* scratch,
                               cudaStream_t st);
// The CSR pair of an edge list in device memory, as sbp_csr_from_edges
// builds it (rows in input edge order, w == nullptr for unit weights), into
// g's arrays (row pointers, entries, weights, degrees, owners).  Bits of
// *err (device): 1 endpoint outside [0, N), 2 weight 0, 4 degree above
// 2^32 - 1.  scratch: csr_build_scratch_bytes(N, E).
size_t csr_build_scratch_bytes(int32_t N, int32_t E);
cudaError_t csr_from_device_edges(int32_t N, int32_t E, const int32_t* src, const int32_t* dst,
                                  const uint32_t* w, DevGraph& g, int32_t* err, void* scratch,
                                  cudaStream_t st);
// The device stages of the DCSBM generator: degrees, block members, edges.
struct DcsbmDeviceIn {
  const int32_t* truth;  // host: the N planted labels (dcsbm_labels)
  const double* cdf;     // host: ncdf running out-degree weights
  uint64_t seed, pin_scaled;
  int32_t N, B, ncdf, deg_min;
  long long max_edges;   // N * deg_max: the edge slots the sources may fill
};
struct DcsbmDeviceOut {
  int32_t *src, *dst;  // device, max_edges entries each: the edges, source-major
  int32_t* E_host;     // the edge count, once the stream has run
};
cudaError_t dcsbm_device_edges(const DcsbmDeviceIn& in, DcsbmDeviceOut& out, cudaStream_t st);

// calculate_new_csr (partition.hpp:707-849): rebuild M from the labels.
void rebuild_blockmodel(const DevGraph& g, const int32_t* part, int32_t B, DevBM& m,
                        RebuildScratch& rs, cudaStream_t st,
                        const RebuildTune& t = RebuildTune{});

// Per-block work: draws == 0 computes the per-block sums (dSout, ambout,
// ambin, sinfull; the MDL and the merge phase read them), draws == 1 only
// the per-block draws of nodal batch `seq` (choose_neighbored_block and the
// per-block uniform, kernels.hpp:942-997, 1024), draws == 2 both.
void block_terms(DevBM& m, int32_t B, int draws, uint64_t seed, uint32_t seq, cudaStream_t st);

// Dense form (B*B counts and their transpose, degrees and their log2) of the
// labels' blockmodel, built from scratch.
void dense_build(const DevGraph& g, const int32_t* part, int32_t B, DevBM& m, cudaStream_t st);
// Applies a batch's moves to the dense form: `part` still holds the old
// labels, newlab[i] the new label of vertex lo+i.  Degrees are updated; their
// log2 are refreshed by nodal_commit (dense mode).
void dense_update(const DevGraph& g, const int32_t* part, int32_t lo, int32_t count,
                  const int32_t* newlab, int32_t B, DevBM& m, cudaStream_t st);
// block_terms for the dense form.
void block_terms_dense(DevBM& m, int32_t B, int draws, uint64_t seed, uint32_t seq,
                       cudaStream_t st);

// data_S = sum of dSout over blocks, written to *out (deterministic order).
void mdl_data_sum(const DevBM& m, int32_t B, double* out, cudaStream_t st);

cudaError_t init_nodal_attributes();
// Vertices with more than this many entries in a direction go to the
// CTA-per-vertex kernel.
int nodal_heavy_threshold();

// A batch's vertices (indices into the batch) by kernel path: small ones
// (at most kSmallEntries neighbour entries) go two to a warp, mid ones one to
// a warp, heavy ones (more than nodal_heavy_threshold() entries in a
// direction) one to a CTA on the side stream.  err counts hash-table
// overflows (should stay 0).
constexpr int32_t kSmallEntries = 16;
struct NodalAux {
  const int32_t* small = nullptr;
  int32_t nsmall = 0;
  const int32_t* mid = nullptr;
  int32_t nmid = 0;
  const int32_t* heavy = nullptr;
  int32_t nheavy = 0;
  int32_t* err = nullptr;
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

// Nodal batch of vertices [lo, lo+count): proposal, dS, accept flag.
// newlab[i] = new label of vertex lo+i, rec[i] = recorded dS (0 if rejected),
// props[i] (optional) = proposal.  dense: read M from its dense form.
void nodal_batch_sample(const DevGraph& g, const int32_t* part, const DevBM& m, int32_t B,
                        bool dense, uint64_t seed, uint32_t seq, int32_t lo, int32_t count,
                        int32_t* newlab, double* rec, int32_t* props, const NodalAux& aux,
                        cudaStream_t st, const ScoreMode& md = ScoreMode());
// dS of given (vertex, proposal) pairs, no accept; with md.mh, logH[i] (if
// given) receives the log Hastings ratio of move i.
void nodal_delta_given(const DevGraph& g, const int32_t* part, const DevBM& m, int32_t B,
                       bool dense, int32_t nv, const int32_t* verts, const int32_t* props,
                       double* dS, const NodalAux& aux, cudaStream_t st,
                       const ScoreMode& md = ScoreMode(), double* logH = nullptr);
// Apply a batch: part[lo+i] = newlab[i]; slot_sum[0] += sum(rec) in a fixed
// order, slot_acc[0] += number of moves.  With dense_m, also recomputes the
// log2 of its block degrees.
void nodal_commit(int32_t* part, int32_t lo, int32_t count, const int32_t* newlab,
                  const double* rec, double* slot_sum, long long* slot_acc, const DevBM* dense_m,
                  int32_t B, const CommitScratch& cs, cudaStream_t st);

// Merge proposals (kernels.hpp:726-856) and their dS with the per-block best
// (kernels.hpp:143-491).
void merge_proposals(const DevBM& m, int32_t B, int32_t np, uint64_t seed, uint32_t seq,
                     int32_t* props, cudaStream_t st, const MergeGrid& grid = MergeGrid());
void merge_delta(const DevBM& m, int32_t B, int32_t E, int32_t np, const int32_t* props,
                 double* dS, int32_t* best, double* best_dS, cudaStream_t st, int32_t exact = 0,
                 const MergeGrid& grid = MergeGrid());
// part[v] = map[part[v]] (update_partitions, kernels.hpp:1728-1740).
void relabel(int32_t* part, int32_t N, const int32_t* map, cudaStream_t st);

}  // namespace sbp
