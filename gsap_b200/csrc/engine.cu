// The multi-job engine: GSAP's partition() loop (partition.hpp:852-954) for
// many jobs at once.
//
// Each job is a Run: the loop's host state (block count, golden-section
// bracket, stop test, RNG sequence) as a state machine that is advanced one
// step per engine tick.  A step is either one merge step (proposals, dS,
// the merge application and the relabel, all on the device) or queued nodal
// sweeps (num_batches batches plus the MDL each), preceded by the device work
// the last host decision left pending (golden-section snapshot and restore
// copies, the blockmodel build).
//
// A tick gathers the device work of every active Run and issues it as
// multi-job launches: one launch per kernel body covers all jobs that need
// it (multi.cuh), so a tick costs about the same number of launches for one
// job as for hundreds.  Argument records and heavy-vertex lists go up in two
// host-to-device copies per tick, every result the host needs (new block
// counts, sweep sums, MDL terms, final labels) comes back in one
// device-to-host copy, and the host synchronises once per tick.
//
// sbp_partition is a batch of one.  sbp_partition_batch and the server
// (server.cu) admit jobs against an HBM budget as earlier jobs finish.
#include "../../include/sbp.h"
#include "common.cuh"
#include "engine.h"
#include "job.h"
#include "kernels.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>

namespace sbp {

// ------------------------------------------------------------------- Run --
void Run::setup_batches() {
  const int nb = o.num_batches;
  BS = J->N / nb;
  batch_entries.assign(nb, 0.0);
  lists_all.clear();
  list_off.assign(nb + 1, 0);
  list_n.assign(3 * (size_t)nb, 0);
  for (int32_t b = 0; b < nb; ++b) {
    int32_t lo = b * BS, hi = (b + 1) * BS;
    batch_entries[b] = (double)(J->h_optr[hi] - J->h_optr[lo]) +
                       (double)(J->h_iptr[hi] - J->h_iptr[lo]);
    classify_batch(*J, nullptr, lo, BS, lists_all, &list_n[3 * (size_t)b]);
    list_off[b + 1] = (int32_t)lists_all.size();
  }
}

void Run::start_partition() {
  const int32_t N = J->N;
  J->dense_eff = std::min(J->dense_cap, dense_limit(J->N, J->E, o.dense_max));
  B = N;
  B_to_merge = (int32_t)((float)B * o.reduction_rate);
  itr_dS.assign(o.max_nodal_itr, 0.0);
  nnz_now = (double)J->E;
  setup_batches();
  stage = kMerge;
  init = true;
  upload_lists = !lists_all.empty();
}

void Run::start_sweeps(int32_t B0, uint32_t seq0, int32_t sweeps) {
  sweeps_only = true;
  sweeps_total = sweeps;
  J->dense_eff = J->dense_cap;
  B = B0;
  seq = seq0;
  nnz_now = (double)J->E;
  setup_batches();
  stage = kSweep;
  init = false;
  build = true;
  build_from_merge = false;
  zero_itr = true;
  upload_lists = !lists_all.empty();
}

bool Run::dense() const { return B <= J->dense_eff; }

// The stop test and golden-section bookkeeping after a sweep
// (partition.hpp:920-934, prepare_for_partition_next :80-322).
void Run::after_sweep(double dsum, double dataS, long long acc) {
  ++R.nodal_itrs;
  itr_dS[itr] = dsum;
  R.accepted_moves += acc;
  S = model_S(B, J->N, J->E, o.exact) - dataS;
  bool stop = false;
  if (itr >= o.window - 1) {
    bool isf = std::isfinite(large.S) && std::isfinite(med.S) && std::isfinite(small.S);
    double mean = 0.0;
    for (int32_t i = itr - o.window + 1; i < itr; ++i) mean += itr_dS[i];
    mean /= (double)(o.window - 1);
    stop = !isf ? (-mean < (double)o.threshold1 * S) : (-mean < (double)o.threshold2 * S);
  }
  if (!stop && itr + 1 < o.max_nodal_itr) {
    ++itr;
    return;
  }
  if (o.verbose)
    std::fprintf(stderr, "[sbp] step %d B=%d S=%.17g itrs=%d\n", R.outer_steps, B, S,
                 R.nodal_itrs);
  Bracket P;
  P.B = B;
  P.B_to_merge = B_to_merge;
  P.S = S;
  auto take_slot = [&](Bracket& x) {
    // the slot of whichever bracket point is being replaced is reused
    bool used[3] = {false, false, false};
    for (Bracket* q : {&large, &med, &small})
      if (q != &x && q->slot >= 0) used[q->slot] = true;
    for (int i = 0; i < 3; ++i)
      if (!used[i]) return i;
    return -1;
  };
  if (P.S <= med.S) {
    if (med.B > P.B) large = med;
    else small = med;
    med = P;
    med.slot = take_slot(med);
    snap_slot = med.slot;
  } else {
    Bracket& tgt = med.B > P.B ? small : large;
    tgt = P;
    tgt.slot = take_slot(tgt);
    snap_slot = tgt.slot;
  }
  const Bracket* restore = nullptr;
  bool optimal = false;
  if (std::isinf(small.S)) {
    restore = &med;
    B_to_merge = (int32_t)((float)med.B * o.reduction_rate);
    if (B_to_merge == 0) optimal = true;
  } else if (large.B - small.B == 2) {
    optimal = true;
    restore = &med;
  } else if ((large.B - med.B) >= (med.B - small.B)) {
    int32_t next_B = med.B + (int32_t)std::round((large.B - med.B) * 0.618);
    restore = &large;
    B_to_merge = large.B - next_B;
  } else {
    int32_t next_B = small.B + (int32_t)std::round((med.B - small.B) * 0.618);
    restore = &med;
    B_to_merge = med.B - next_B;
  }
  if (snap_slot < 0 || restore->slot < 0) {
    set_error(SBP_ERR_INTERNAL, "bracket point without a snapshot");
    return;
  }
  restore_slot = restore->slot;
  // restoring the snapshot just taken of this step leaves the labels as they
  // are, and with them a dense form, which the merge step then reads its CSR
  // form from
  dense_kept = dense() && restore->slot == snap_slot;
  B = restore->B;
  S = restore->S;
  csr_fresh = false;
  stage = optimal ? kFinish : kMerge;
}

void Run::set_error(sbp_status st, const std::string& msg) {
  if (status == SBP_OK) {
    status = st;
    error = msg;
  }
  stage = kDone;
}

// ---------------------------------------------------------------- Engine --
Engine::~Engine() {
  if (!st) return;
  cudaSetDevice(device);
  cudaStreamSynchronize(st);
  runs.clear();  // runs belong to the caller
  cudaFree(up_dev);
  cudaFree(desc_dev);
  cudaFree(rd_dev);
  cudaFreeHost(up_host);
  cudaFreeHost(desc_host);
  cudaFreeHost(rd_host);
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  if (ev_first) cudaEventDestroy(ev_first);
  if (fork) cudaEventDestroy(fork);
  if (join) cudaEventDestroy(join);
  if (side) cudaStreamDestroy(side);
  cudaStreamDestroy(st);
}

sbp_status Engine::init(int dev) {
  device = dev;
  SBP_CUDA(cudaSetDevice(device));
  SBP_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  SBP_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
  SBP_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  SBP_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
  return SBP_OK;
}

// Grows a pinned host + device buffer pair to at least `need` bytes (only
// between ticks, when nothing in flight uses them).
static sbp_status grow(size_t need, size_t& cap, void*& host, void*& dev) {
  if (need <= cap) return SBP_OK;
  size_t n = std::max(need, cap * 2);
  n = std::max<size_t>(n, 1 << 16);
  cudaFreeHost(host);
  cudaFree(dev);
  host = nullptr;
  dev = nullptr;
  cap = 0;
  SBP_CUDA(cudaMallocHost(&host, n));
  SBP_CUDA(cudaMalloc(&dev, n));
  cap = n;
  return SBP_OK;
}

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

void Engine::ensure_slots(int K, int nb) {
  if ((int)sw.size() < K * nb) sw.resize(K * nb);
  if ((int)ends.size() < K) ends.resize(K);
}

void Engine::clear_slots() {
  for (Slot* s : {&s_iota, &s_lists, &s_snap, &s_restore, &s_zero, &m_bt, &m_props, &m_delta,
                  &m_delta8, &m_best, &m_relabel, &s_gather})
    s->clear();
  m_apply.clear();
  pre_dense.clear();
  pre_rebuild.clear();
  for (auto& b : sw) {
    for (Slot* s : {&b.bt_csr, &b.bt_dense, &b.dupd, &b.commit}) s->clear();
    for (Slot& s : b.heavy) s.clear();
    for (Slot& s : b.nodal) s.clear();
    b.rebuild.clear();
  }
  for (auto& e : ends)
    for (Slot* s : {&e.bt_csr, &e.bt_dense, &e.mdl, &e.ctl}) s->clear();
}

// Sweeps queued for a run this tick: the first `window` sweeps of an outer
// step cannot end it, later ticks queue kSweepsAhead; queued sweeps after
// the stop test fires do nothing.
static int32_t sweeps_to_queue(const Run& r) {
  static const int32_t ahead = [] {
    const char* e = std::getenv("SBP_SWEEPS_AHEAD");
    int v = e ? std::atoi(e) : 3;
    return std::max(1, std::min(v, 16));
  }();
  if (r.sweeps_only) return std::min(ahead, r.sweeps_total - r.itr);
  const int32_t left = r.o.max_nodal_itr - r.itr;
  const int32_t k = r.itr == 0 ? std::max(ahead, r.o.window) : ahead;
  return std::max(1, std::min(k, left));
}

// The rebuild launch shape for a job's size class: the autotuner's choice
// when it has one, else the defaults.
static RebuildTune tune_for(const Job& J, int32_t B) {
  RebuildTune t;
  rebuild_tuned(J.device, J.E, B, &t);
  return t;
}

static bool tuning_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("SBP_TUNE");
    return !(e && e[0] == '0');
  }();
  return on;
}

// Readback layout of a sweeping run: ctl pair, err, nnz, then dsum, dataS
// and acc of the queued sweeps.
static size_t sweep_rd_bytes(int32_t K) { return (16 + 24 * (size_t)K + 255) & ~size_t(255); }

// Device work of one run for this tick, as records in the slots.
void Engine::add_run_work(Run& r) {
  Job& J = *r.J;
  const int32_t N = J.N;
  if (r.init) add_iota(s_iota, J.part, N);
  if (r.init && ref_grid_on(r.o)) {
    // GSAP's merge buffers start at zero in a fresh process; the slots its
    // grid leaves out read them (MergeGrid)
    const size_t slots = (size_t)N * J.np;
    add_zero(s_zero, J.props, slots);
    add_zero(s_zero, J.mdS, 2 * slots);
    add_zero(s_zero, J.mdsin, 2 * slots);
  }
  if (r.upload_lists)
    add_copy(s_lists, J.lists, up_dev_ptr(r.up_lists), r.lists_all.size());
  if (r.snap_slot >= 0) add_copy(s_snap, J.snap[r.snap_slot], J.part, (size_t)N);
  if (r.restore_slot >= 0) add_copy(s_restore, J.part, J.snap[r.restore_slot], (size_t)N);
  if (r.zero_itr) {
    const size_t n = r.sweeps_only ? (size_t)r.sweeps_total * r.o.num_batches
                                   : (size_t)r.o.max_nodal_itr;
    add_zero(s_zero, J.dsum, 2 * n);
    add_zero(s_zero, J.acc, 2 * n);
    add_zero(s_zero, J.ctl, 2);
  }
  const bool dense = r.dense();
  if (r.stage == Run::kMerge) {
    // the merge kernels read the CSR form
    if (!r.csr_fresh && r.dense_kept && r.dense()) {
      add_csr_from_dense(pre_rebuild, r.B, J.m, J.rs);
      r.pre_bytes += 8.0 * r.B * (double)r.B + 8.0 * r.nnz_now + 8.0 * r.B;
    } else if (!r.csr_fresh) {
      add_rebuild(pre_rebuild, J.g, J.part, r.B, J.m, J.rs, nullptr, tune_for(J, r.B));
      r.pre_bytes += 4.0 * N + 24.0 * J.E + 16.0 * r.nnz_now + 8.0 * r.B;
    }
    add_block_terms(m_bt, J.m, r.B, 0, r.o.seed, 0);
    const MergeGrid grid = merge_grid(J, r.o);
    add_merge_props(m_props, J.m, r.B, J.np, r.o.seed, r.seq, J.props, grid);
    add_merge_delta(m_delta, m_delta8, m_best, J.m, r.B, J.E, J.np, J.props, nullptr, J.best,
                    J.best_dS, r.o.exact, grid);
    // carry_out_best_merges on the device, then the relabel: the host reads
    // back only the new block count
    add_zero(s_zero, J.ma_out, 2);
    add_merge_apply(m_apply, J.ma, r.B, r.B_to_merge, J.best, J.best_dS, J.map, J.ma_out);
    add_relabel(m_relabel, J.part, N, J.map);
    add_copy(s_gather, rd_dev_ptr(r.rd_off), J.ma_out, 2);
    return;
  }
  if (r.stage == Run::kSweep) {
    if (r.build) {
      if (dense && r.build_from_merge) {
        // from the merge step's CSR blockmodel and its map: nnz entries, not E edges
        add_dense_build_mapped(pre_dense, J.g, J.part, r.B, J.m, r.B_merged_from, J.map);
        r.pre_bytes += 8.0 * r.B * (double)r.B +
                       12.0 * std::min((double)J.E, (double)r.B_merged_from * r.B_merged_from);
      } else if (dense) {
        add_dense_build(pre_dense, J.g, J.part, r.B, J.m);
        r.pre_bytes += 8.0 * r.B * (double)r.B + 12.0 * J.E;  // zero M, M^T; add the edges
      } else {
        add_rebuild(pre_rebuild, J.g, J.part, r.B, J.m, J.rs, nullptr, tune_for(J, r.B));
        r.pre_bytes += 4.0 * N + 24.0 * J.E + 16.0 * r.nnz_now + 8.0 * r.B;
      }
    }
    const int nb = r.o.num_batches;
    const RebuildTune tune = tune_for(J, r.B);
    const int32_t* ctl = J.ctl;
    const bool isf = std::isfinite(r.large.S) && std::isfinite(r.med.S) && std::isfinite(r.small.S);
    const double thr = isf ? (double)r.o.threshold2 : (double)r.o.threshold1;
    const double mS = model_S(r.B, J.N, J.E, r.o.exact);
    const ScoreMode md = score_mode(r.o);
    for (int32_t k = 0; k < r.sweep_k; ++k) {
      for (int32_t b = 0; b < nb; ++b) {
        SweepSlots& s = sw[k * nb_slots_ + b];
        const uint32_t seq = r.seq_sweep0 + (uint32_t)b;  // + ctl[0] * nb on the device
        double* slot_sum = r.sweeps_only ? J.dsum + b : J.dsum;
        long long* slot_acc = r.sweeps_only ? J.acc + b : J.acc;
        const int32_t slot_mul = r.sweeps_only ? nb : 1;
        const int32_t lo = b * r.BS;
        // dense form: the tick's first batch draws here, every later one in
        // the commit of the batch before it (its seq is always one more)
        if (dense) {
          if (k == 0 && b == 0)
            add_block_terms_dense(s.bt_dense, J.m, r.B, 1, r.o.seed, seq, ctl, nb);
        } else {
          add_block_terms(s.bt_csr, J.m, r.B, 1, r.o.seed, seq, ctl, nb);
        }
        const int ms = md.slot(dense);
        add_nodal(s.nodal[ms], s.heavy[ms], dense, md, J.g, J.part, J.m, r.B, r.o.seed, seq, lo,
                  r.BS, J.newlab, J.rec, nullptr,
                  nodal_lists(J, J.lists + r.list_off[b], &r.list_n[3 * (size_t)b]), ctl, nb);
        if (dense) {
          // the moved vertices' edges, applied to the dense form before the
          // labels change (it reads old and new labels)
          add_dense_update(s.dupd, J.g, J.part, lo, r.BS, J.newlab, r.B, J.m, ctl);
          const bool last = k == r.sweep_k - 1 && b == nb - 1;
          add_commit(s.commit, J.part, lo, r.BS, J.newlab, J.rec, slot_sum, slot_acc, &J.m,
                     r.B, J.cs, ctl, slot_mul, !last, r.o.seed, seq + 1, nb);
        } else {
          add_commit(s.commit, J.part, lo, r.BS, J.newlab, J.rec, slot_sum, slot_acc, nullptr,
                     0, J.cs, ctl, slot_mul);
          add_rebuild(s.rebuild, J.g, J.part, r.B, J.m, J.rs, ctl, tune);
        }
      }
      SweepEndSlots& e = ends[k];
      if (r.sweeps_only) {
        add_sweep_ctl(e.ctl, J.ctl, J.dsum, J.dataS, 0.0, 0.0, 0, r.sweeps_total);
      } else {
        if (dense) add_block_terms_dense(e.bt_dense, J.m, r.B, 0, r.o.seed, 0, ctl, 0);
        else add_block_terms(e.bt_csr, J.m, r.B, 0, r.o.seed, 0, ctl, 0);
        add_mdl_sum(e.mdl, J.m, r.B, J.dataS, ctl);
        add_sweep_ctl(e.ctl, J.ctl, J.dsum, J.dataS, mS, thr, r.o.window, r.o.max_nodal_itr);
      }
    }
    add_copy(s_gather, rd_dev_ptr(r.rd_off), J.ctl, 2);
    add_copy(s_gather, rd_dev_ptr(r.rd_off + 8), J.err, 1);
    add_copy(s_gather, rd_dev_ptr(r.rd_off + 12), J.m.optr + r.B, 1);
    if (!r.sweeps_only) {
      const size_t K = (size_t)r.sweep_k;
      add_copy(s_gather, rd_dev_ptr(r.rd_off + 16), J.dsum + r.itr, 2 * K);
      add_copy(s_gather, rd_dev_ptr(r.rd_off + 16 + 8 * K), J.dataS + r.itr, 2 * K);
      add_copy(s_gather, rd_dev_ptr(r.rd_off + 16 + 16 * K), J.acc + r.itr, 2 * K);
    }
    return;
  }
  if (r.stage == Run::kFinish) {
    add_copy(s_gather, rd_dev_ptr(r.rd_off), J.part, (size_t)N);
    if (r.sweeps_only) {
      const size_t n = (size_t)r.sweeps_total * r.o.num_batches;
      add_copy(s_gather, rd_dev_ptr(r.rd_off + align256(4 * (size_t)N)), J.dsum, 2 * n);
    }
  }
}

// Readback bytes of one run this tick.
static size_t rd_bytes(const Run& r) {
  switch (r.stage) {
    case Run::kMerge:
      return 256;
    case Run::kSweep:
      return sweep_rd_bytes(r.sweep_k);
    case Run::kFinish:
      return align256(4 * (size_t)r.J->N) +
             (r.sweeps_only ? align256(8 * (size_t)r.sweeps_total * r.o.num_batches) : 0);
    default:
      return 0;
  }
}

sbp_status Engine::launch_slot(Slot& s, size_t off, cudaStream_t stream) {
  if (s.empty()) return SBP_OK;
  if (s.mismatch || !s.k) return fail(SBP_ERR_INTERNAL, "engine slot with mixed kernels");
  if (s.njobs() == 1) {
    s.k->launch_one(s.recs.data(), s.total(), stream);
    return SBP_OK;
  }
  MultiSpan sp;
  sp.args = (const char*)desc_dev + off;
  sp.cta0 = (const int32_t*)((const char*)desc_dev + off + align256(s.recs.size()));
  sp.njobs = s.njobs();
  sp.total = s.total();
  s.k->launch(sp, stream);
  return SBP_OK;
}

// Engines in different host threads (the server's lanes) hand their CUDA
// calls to the driver one thread at a time, so a tick's launches (and a
// graph capture) stay contiguous; only the wait for a tick's end runs
// outside this lock, so the lanes' device work still overlaps.
std::mutex& cuda_submit_mutex() {
  static std::mutex mu;
  return mu;
}

sbp_status Engine::tick() {
  std::unique_lock<std::mutex> submit(cuda_submit_mutex());
  const double t_start = now_ms();
  int trace = 0;  // verbose >= 2: one line per tick on stderr
  for (Run* r : runs)
    if (r->stage != Run::kDone) trace = std::max(trace, r->o.verbose);
  SBP_CUDA(cudaSetDevice(device));
  // runs that reach the outer-step limit stop at their next merge
  for (Run* r : runs) {
    if (r->stage != Run::kMerge) continue;
    if (++r->R.outer_steps > r->o.max_outer) {
      r->R.status = SBP_ERR_INTERNAL;
      r->stage = Run::kFinish;
    }
  }
  // graphs only when every active run asks for them
  use_graphs = true;
  for (Run* r : runs)
    if (r->stage != Run::kDone && !r->o.use_graphs) use_graphs = false;
  // per-batch phase events when any active run asks for them (an event node
  // costs a few microseconds of device time, five of them every batch)
  bool timing = trace >= 3;
  for (Run* r : runs)
    if (r->stage != Run::kDone && r->o.phase_timing) timing = true;
  // pass 1: sweeps to queue, uploads (maps, batch lists) and readbacks
  size_t up = 0, rd = 0;
  int nb_max = 0, k_max = 0;
  for (Run* r : runs) {
    if (r->stage == Run::kDone) continue;
    r->sweep_k = 0;
    if (r->stage == Run::kSweep) {
      r->sweep_k = sweeps_to_queue(*r);
      if (r->itr == 0) r->seq_sweep0 = r->seq;
      nb_max = std::max(nb_max, r->o.num_batches);
      k_max = std::max(k_max, r->sweep_k);
    }
    if (r->upload_lists) {
      r->up_lists = up;
      up += align256(4 * r->lists_all.size());
    }
    r->rd_off = rd;
    rd += rd_bytes(*r);
  }
  sbp_status s = grow(up, up_cap, up_host, up_dev);
  if (s != SBP_OK) return s;
  s = grow(rd, rd_cap, rd_host, rd_dev);
  if (s != SBP_OK) return s;
  // pass 2: records
  ensure_slots(k_max, nb_max);
  nb_slots_ = nb_max;
  clear_slots();
  for (Run* r : runs) {
    if (r->stage == Run::kDone) continue;
    if (r->upload_lists)
      std::memcpy((char*)up_host + r->up_lists, r->lists_all.data(), 4 * r->lists_all.size());
    add_run_work(*r);
  }
  // pass 3: pack the slots' records and offsets
  std::vector<Slot*> order = {&s_iota, &s_lists, &s_snap, &s_restore, &s_zero};
  for (Slot* x : pre_dense.all()) order.push_back(x);
  for (Slot* x : pre_rebuild.all()) order.push_back(x);
  for (Slot* x : {&m_bt, &m_props, &m_delta, &m_delta8, &m_best}) order.push_back(x);
  for (Slot* x : m_apply.all()) order.push_back(x);
  order.push_back(&m_relabel);
  for (int k = 0; k < k_max; ++k) {
    for (int b = 0; b < nb_max; ++b) {
      SweepSlots& w = sw[k * nb_max + b];
      order.push_back(&w.bt_csr);
      order.push_back(&w.bt_dense);
      for (Slot& x : w.heavy) order.push_back(&x);
      for (Slot& x : w.nodal) order.push_back(&x);
      order.push_back(&w.dupd);
      order.push_back(&w.commit);
      for (Slot* x : w.rebuild.all()) order.push_back(x);
    }
    SweepEndSlots& e = ends[k];
    for (Slot* x : {&e.bt_csr, &e.bt_dense, &e.mdl, &e.ctl}) order.push_back(x);
  }
  order.push_back(&s_gather);
  // Only multi-job launches read their records from device memory (a
  // one-job launch takes its record as the kernel argument), so a tick of
  // one-job slots packs and uploads nothing.
  bool multi = false;
  for (const Slot* x : order) multi = multi || x->njobs() > 1;
  size_t desc = 0;
  std::vector<size_t> off(order.size(), 0);
  for (size_t i = 0; i < order.size() && multi; ++i) {
    if (order[i]->empty()) continue;
    off[i] = desc;
    desc += align256(order[i]->recs.size()) + align256(4 * order[i]->cta0.size());
  }
  s = grow(desc, desc_cap, desc_host, desc_dev);
  if (s != SBP_OK) return s;
  for (size_t i = 0; i < order.size() && multi; ++i) {
    Slot* x = order[i];
    if (x->empty()) continue;
    std::memcpy((char*)desc_host + off[i], x->recs.data(), x->recs.size());
    std::memcpy((char*)desc_host + off[i] + align256(x->recs.size()), x->cta0.data(),
                4 * x->cta0.size());
  }
  auto slot_off = [&](Slot* x) {
    for (size_t i = 0; i < order.size(); ++i)
      if (order[i] == x) return off[i];
    return (size_t)0;
  };
  // pass 4: issue
  const int nbatch = k_max * nb_max;
  const int n_ev = 4 + 5 * nbatch;
  while ((int)ev.size() < n_ev) {
    cudaEvent_t e;
    SBP_CUDA(cudaEventCreate(&e));
    ev.push_back(e);
  }
  if (!ev_first) {
    SBP_CUDA(cudaEventCreate(&ev_first));
    SBP_CUDA(cudaEventRecord(ev_first, st));
  }
  for (Run* r : runs)
    if (r->stage != Run::kDone && !r->ev_begin) {
      SBP_CUDA(cudaEventCreate(&r->ev_begin));
      SBP_CUDA(cudaEventRecord(r->ev_begin, st));
    }
  SBP_CUDA(cudaEventRecord(ev[0], st));
  if (up) SBP_CUDA(cudaMemcpyAsync(up_dev, up_host, up, cudaMemcpyHostToDevice, st));
  if (desc) SBP_CUDA(cudaMemcpyAsync(desc_dev, desc_host, desc, cudaMemcpyHostToDevice, st));
  size_t i = 0;
  auto emit_until = [&](Slot* last) -> sbp_status {
    for (; i < order.size(); ++i) {
      sbp_status q = launch_slot(*order[i], off[i], st);
      if (q != SBP_OK) return q;
      if (order[i] == last) {
        ++i;
        break;
      }
    }
    return SBP_OK;
  };
  s = emit_until(pre_rebuild.all().back());
  if (s != SBP_OK) return s;
  SBP_CUDA(cudaEventRecord(ev[1], st));
  s = emit_until(&m_relabel);
  if (s != SBP_OK) return s;
  SBP_CUDA(cudaEventRecord(ev[2], st));
  // the queued sweeps; timing events are external records so that they
  // also time a replayed graph
  const size_t sweep_first = i;
  bool capturing = false;
  auto record = [&](cudaEvent_t e) {
    return capturing ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal)
                     : cudaEventRecord(e, st);
  };
  auto issue_sweeps = [&]() -> sbp_status {
    for (int k = 0; k < k_max; ++k) {
      for (int b = 0; b < nb_max; ++b) {
        SweepSlots& w = sw[k * nb_max + b];
        cudaEvent_t* be = &ev[4 + 5 * (k * nb_max + b)];
        if (timing) SBP_CUDA(record(be[0]));
        sbp_status q = emit_until(&w.bt_dense);
        if (q != SBP_OK) return q;
        if (timing) SBP_CUDA(record(be[1]));
        bool heavy = false;
        for (const Slot& x : w.heavy) heavy = heavy || !x.empty();
        if (heavy) {
          // heavy vertices on the side stream, next to the warp kernels
          SBP_CUDA(cudaEventRecord(fork, st));
          SBP_CUDA(cudaStreamWaitEvent(side, fork, 0));
          for (Slot& x : w.heavy) {
            q = launch_slot(x, slot_off(&x), side);
            if (q != SBP_OK) return q;
          }
          SBP_CUDA(cudaEventRecord(join, side));
        }
        i += 4;  // the heavy slots
        q = emit_until(&w.nodal[3]);
        if (q != SBP_OK) return q;
        if (heavy) SBP_CUDA(cudaStreamWaitEvent(st, join, 0));
        if (timing) SBP_CUDA(record(be[2]));
        q = emit_until(&w.commit);
        if (q != SBP_OK) return q;
        if (timing) SBP_CUDA(record(be[3]));
        q = emit_until(w.rebuild.all().back());
        if (q != SBP_OK) return q;
        if (timing) SBP_CUDA(record(be[4]));
      }
      sbp_status q = emit_until(&ends[k].ctl);
      if (q != SBP_OK) return q;
    }
    return SBP_OK;
  };
  // A tick of queued sweeps only (no pending build, copy or merge) is one
  // CUDA graph: its launches and arguments repeat tick after tick within an
  // outer step (RNG sequence and result slots come from the device-side
  // sweep control), so it is captured once and replayed; a changed step
  // (new B) updates the executable graph in place.
  bool graphable = use_graphs && k_max > 0;
  for (size_t q = 0; q < sweep_first && graphable; ++q)
    if (!order[q]->empty()) graphable = false;
  if (!graphable) {
    s = issue_sweeps();
    if (s != SBP_OK) return s;
  } else {
    // the sweeps' launches, byte for byte: kernels, records, grids, offsets
    std::vector<unsigned char>& key = key_scratch;
    key.clear();
    auto mix = [&](const void* p, size_t n) {
      const unsigned char* c = (const unsigned char*)p;
      key.insert(key.end(), c, c + n);
    };
    mix(&k_max, sizeof(k_max));
    mix(&nb_max, sizeof(nb_max));
    mix(&timing, sizeof(timing));
    for (size_t q = sweep_first; q < order.size(); ++q) {
      const Slot* x = order[q];
      if (x == &s_gather || x->empty()) continue;
      mix(&q, sizeof(q));
      mix(&x->k, sizeof(x->k));
      mix(x->recs.data(), x->recs.size());
      mix(x->cta0.data(), 4 * x->cta0.size());
      mix(&off[q], sizeof(off[q]));
    }
    mix(&desc_dev, sizeof(desc_dev));
    if (graph_exec && key.size() == graph_key.size() &&
        std::memcmp(key.data(), graph_key.data(), key.size()) == 0) {
      // replay: skip the slots the graph holds
      i = sweep_first;
      while (i < order.size() && order[i] != &s_gather) ++i;
      ++graph_replays;
      g_launches += graph_kernels;
    } else {
      SBP_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      const long long l0 = g_launches;
      capturing = true;
      sbp_status q = issue_sweeps();
      capturing = false;
      graph_kernels = g_launches - l0;
      cudaGraph_t g = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(st, &g);
      if (q != SBP_OK) {
        if (g) cudaGraphDestroy(g);
        return q;
      }
      if (ce != cudaSuccess) return fail(SBP_ERR_CUDA, cudaGetErrorString(ce));
      if (graph_exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(graph_exec, g, &info) != cudaSuccess) {
          cudaGetLastError();
          cudaGraphExecDestroy(graph_exec);
          graph_exec = nullptr;
        }
      }
      if (!graph_exec) {
        const cudaError_t ie = cudaGraphInstantiate(&graph_exec, g, 0);
        if (ie != cudaSuccess) {
          cudaGraphDestroy(g);
          graph_exec = nullptr;
          return fail(SBP_ERR_CUDA, cudaGetErrorString(ie));
        }
      }
      cudaGraphDestroy(g);
      graph_key.swap(key);
      ++graph_captures;
    }
    SBP_CUDA(cudaGraphLaunch(graph_exec, st));
  }
  s = emit_until(&s_gather);
  if (s != SBP_OK) return s;
  if (rd) SBP_CUDA(cudaMemcpyAsync(rd_host, rd_dev, rd, cudaMemcpyDeviceToHost, st));
  SBP_CUDA(cudaEventRecord(ev[3], st));
  const double t_issued = now_ms();
  submit.unlock();
  // phase times of this tick (shared by the runs that took part), each
  // batch's read as soon as its last event has passed, so that the queries
  // overlap the later batches instead of following the tick
  float ms_pre = 0.f, ms_merge = 0.f;
  float t_nodal = 0.f, t_kernel = 0.f, t_rebuild = 0.f;
  cudaError_t waited = cudaEventSynchronize(ev[2]);
  if (waited == cudaSuccess) waited = cudaEventElapsedTime(&ms_pre, ev[0], ev[1]);
  if (waited == cudaSuccess) waited = cudaEventElapsedTime(&ms_merge, ev[1], ev[2]);
  std::vector<float> seg;  // verbose >= 3: each batch's four segments
  for (int q = 0; q < nbatch && waited == cudaSuccess && timing; ++q) {
    cudaEvent_t* be = &ev[4 + 5 * q];
    float a = 0.f, b = 0.f, c = 0.f;
    waited = cudaEventSynchronize(be[4]);
    if (waited == cudaSuccess) waited = cudaEventElapsedTime(&a, be[0], be[3]);
    if (waited == cudaSuccess) waited = cudaEventElapsedTime(&b, be[1], be[2]);
    if (waited == cudaSuccess) waited = cudaEventElapsedTime(&c, be[3], be[4]);
    t_nodal += a;
    t_kernel += b;
    t_rebuild += c;
    if (trace >= 3 && waited == cudaSuccess) {
      float d = 0.f, e = 0.f;
      waited = cudaEventElapsedTime(&d, be[0], be[1]);
      if (waited == cudaSuccess) waited = cudaEventElapsedTime(&e, be[2], be[3]);
      seg.insert(seg.end(), {d, b, e, c});
    }
  }
  if (waited == cudaSuccess) waited = cudaEventSynchronize(ev[3]);
  submit.lock();
  const double t_waited = now_ms();
  SBP_CUDA(waited);
  SBP_CUDA(cudaGetLastError());
  ++ticks;
  // host side of each run
  for (Run* r : runs) {
    if (r->stage == Run::kDone) continue;
    r->R.ms_rebuild += ms_pre;
    r->R.bytes_rebuild += r->pre_bytes;
    r->pre_bytes = 0.0;
    const char* rdp = (const char*)rd_host + r->rd_off;
    r->init = false;
    r->upload_lists = false;
    r->snap_slot = -1;
    r->restore_slot = -1;
    r->zero_itr = false;
    if (r->stage == Run::kMerge) {
      Job& J = *r->J;
      r->R.ms_merge += ms_merge;
      r->R.bytes_merge += 320.0 * r->nnz_now + 8.0 * J.N;
      int32_t res[2] = {0, 0};
      std::memcpy(res, rdp, 8);
      const int32_t nb = res[0];
      if (res[1] != 0 || nb < 1 || nb > r->B) {
        r->set_error(SBP_ERR_INTERNAL, "merge target out of range (B=" + std::to_string(r->B) +
                                           ", N=" + std::to_string(J.N) + ")");
        continue;
      }
      ++r->seq;
      r->B_merged_from = r->B;  // the CSR form holds this B's blockmodel
      r->dense_kept = false;
      r->B = nb;
      r->csr_fresh = false;
      r->build = true;
      r->build_from_merge = true;
      r->zero_itr = true;
      r->itr = 0;
      r->stage = Run::kSweep;
      if (r->dense()) r->nnz_now = std::min((double)J.E, (double)r->B * r->B);
      continue;
    }
    if (r->stage == Run::kSweep) {
      Job& J = *r->J;
      const bool dense = r->dense();
      const int nb = r->o.num_batches;
      r->build = false;
      if (!dense) r->csr_fresh = true;
      r->R.ms_nodal += t_nodal;
      r->R.ms_nodal_kernel += t_kernel;
      r->R.ms_rebuild += t_rebuild;
      int32_t ctl[2] = {0, 0}, err = 0, nnz = 0;
      std::memcpy(ctl, rdp, 8);
      std::memcpy(&err, rdp + 8, 4);
      std::memcpy(&nnz, rdp + 12, 4);
      const int32_t done = ctl[0] - r->itr;  // sweeps that ran this tick
      if (err != 0) {
        r->set_error(SBP_ERR_INTERNAL, "neighbour-block table overflow in the nodal kernel");
        continue;
      }
      if (done < 1 || done > r->sweep_k) {
        r->set_error(SBP_ERR_INTERNAL, "sweep control out of step");
        continue;
      }
      for (int32_t q = 0; q < done; ++q)
        for (int b = 0; b < nb; ++b) {
          r->R.nodal_proposals += r->BS;
          r->R.nodal_launches += 1;
          r->R.bytes_nodal += 28.0 * r->BS + 12.0 * r->batch_entries[b] +
                              16.0 * r->nnz_now + 8.0 * r->B;
          // a CSR batch's rebuild; a dense batch's incremental update runs
          // inside the nodal phase and is not counted
          if (!dense) r->R.bytes_rebuild += 4.0 * J.N + 24.0 * J.E + 16.0 * r->nnz_now + 8.0 * r->B;
        }
      r->seq = r->seq_sweep0 + (uint32_t)ctl[0] * (uint32_t)nb;
      if (!dense) r->nnz_now = (double)nnz;
      // the labels are those of this B now: tune the rebuild for its class
      RebuildTune known;
      if (!dense && tuning_enabled() && !rebuild_tuned(J.device, J.E, r->B, &known)) {
        cudaError_t te = tune_rebuild(J.device, J.g, J.part, r->B, J.m, J.rs, st, &known);
        if (te != cudaSuccess) return fail(SBP_ERR_CUDA, cudaGetErrorString(te));
      }
      if (r->sweeps_only) {
        r->itr = ctl[0];
        if (ctl[1]) r->stage = Run::kFinish;
        continue;
      }
      const size_t K = (size_t)r->sweep_k;
      for (int32_t q = 0; q < done && r->stage == Run::kSweep; ++q) {
        double dsum = 0.0, dataS = 0.0;
        long long acc = 0;
        std::memcpy(&dsum, rdp + 16 + 8 * q, 8);
        std::memcpy(&dataS, rdp + 16 + 8 * K + 8 * q, 8);
        std::memcpy(&acc, rdp + 16 + 16 * K + 8 * q, 8);
        const bool last = q == done - 1;
        r->after_sweep(dsum, dataS, acc);
        // the device's stop test and the host's must agree
        const bool host_stopped = r->stage != Run::kSweep;
        if (host_stopped != (last && ctl[1] != 0) && r->status == SBP_OK)
          r->set_error(SBP_ERR_INTERNAL, "device and host stop tests disagree");
      }
      continue;
    }
    if (r->stage == Run::kFinish) {
      if (r->labels_out) std::memcpy(r->labels_out, rdp, 4 * (size_t)r->J->N);
      if (r->sweeps_only && r->sums_out)
        std::memcpy(r->sums_out, rdp + align256(4 * (size_t)r->J->N),
                    8 * (size_t)r->sweeps_total * r->o.num_batches);
      float ms = 0.f;
      SBP_CUDA(cudaEventElapsedTime(&ms, r->ev_begin, ev[3]));
      r->R.ms_device = ms;
      r->R.B = r->B;
      r->R.S = r->S;
      r->stage = Run::kDone;
      // a server request is published (Run::finished) by its lane, under
      // the server's lock, once the engine no longer touches it
    }
  }
  if (trace >= 2) {
    float dev = 0.f;
    cudaEventElapsedTime(&dev, ev[0], ev[3]);
    std::fprintf(stderr,
                 "[sbp] tick %lld runs %zu sweeps %d: host issue %.3f ms, wait %.3f ms, host after "
                 "%.3f ms, device %.3f ms\n",
                 ticks, runs.size(), k_max, t_issued - t_start, t_waited - t_issued,
                 now_ms() - t_waited, (double)dev);
    // per batch: block draws, nodal kernels, dense update + commit, rebuild (us)
    for (size_t q = 0; q + 3 < seg.size(); q += 4)
      std::fprintf(stderr, "[sbp]   batch %zu: draws %.1f us, nodal %.1f us, commit %.1f us, rebuild %.1f us\n",
                   q / 4, 1000.0 * seg[q], 1000.0 * seg[q + 1], 1000.0 * seg[q + 2],
                   1000.0 * seg[q + 3]);
  }
  return SBP_OK;
}

void Engine::reset() {
  runs.clear();
  ticks = 0;
  if (ev_first) cudaEventDestroy(ev_first);
  ev_first = nullptr;
}

double Engine::device_ms() {
  if (!ev_first || ev.size() < 4) return 0.0;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ev_first, ev[3]) != cudaSuccess) return 0.0;
  return ms;
}

void Run::release_events() {
  if (ev_begin) cudaEventDestroy(ev_begin);
  ev_begin = nullptr;
}

Run::~Run() { release_events(); }

void HostGraph::assign(const sbp_graph_csr& g) {
  N = g.N;
  E = g.E;
  optr.assign(g.out_ptr, g.out_ptr + N + 1);
  iptr.assign(g.in_ptr, g.in_ptr + N + 1);
  oidx.assign(g.out_idx, g.out_idx + E);
  iidx.assign(g.in_idx, g.in_idx + E);
  ow.assign(g.out_w, g.out_w + E);
  iw.assign(g.in_w, g.in_w + E);
  kdo.assign(g.deg_out, g.deg_out + N);
  kdi.assign(g.deg_in, g.deg_in + N);
}

sbp_graph_csr HostGraph::csr() const {
  sbp_graph_csr g{};
  g.N = N;
  g.E = E;
  g.out_ptr = optr.data();
  g.out_idx = oidx.data();
  g.out_w = ow.data();
  g.in_ptr = iptr.data();
  g.in_idx = iidx.data();
  g.in_w = iw.data();
  g.deg_out = kdo.data();
  g.deg_in = kdi.data();
  return g;
}

// ------------------------------------------------------------- Scheduler --
sbp_status Scheduler::init(int device, uint64_t hbm_budget, int32_t max_active_jobs,
                           std::shared_ptr<HbmBudget> shared) {
  sbp_status s = eng.init(device);
  if (s != SBP_OK) return s;
  max_active = max_active_jobs;
  if (shared) {
    hbm = shared;
    return SBP_OK;
  }
  // job arenas come from the stream-ordered pool; keep freed memory in it
  cudaMemPool_t pool;
  SBP_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t keep = ~0ull;
  SBP_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  if (hbm_budget == 0) {
    size_t free_b = 0, total_b = 0;
    SBP_CUDA(cudaMemGetInfo(&free_b, &total_b));
    hbm_budget = (uint64_t)(0.9 * (double)free_b);
  }
  hbm = std::make_shared<HbmBudget>();
  hbm->cap = (double)hbm_budget;
  return SBP_OK;
}

static size_t run_bytes(const Run& r) {
  const sbp_graph_csr& g = *r.graph;
  return job_bytes(g.N, g.E, r.o.num_proposals, r.o.max_nodal_itr,
                   dense_limit(g.N, g.E, r.o.dense_max));
}

sbp_status Scheduler::admit(std::vector<Run*>& done) {
  std::lock_guard<std::mutex> submit(cuda_submit_mutex());
  while (queued() > 0) {
    Run* r = queue[queue_head];
    if (max_active > 0 && (int32_t)eng.runs.size() >= max_active) break;
    const double bytes = (double)run_bytes(*r);
    if (bytes > hbm->cap) {
      ++queue_head;
      r->set_error(SBP_ERR_BUDGET, "job arena exceeds the HBM budget");
      done.push_back(r);
      continue;
    }
    if (!hbm->take(bytes)) break;  // waits for running jobs, in order
    ++queue_head;
    r->owned.reset(new Job());
    r->J = r->owned.get();
    const sbp_graph_csr& g = *r->graph;
    sbp_status s = job_create(*r->J, eng.device, g.N, g.E, r->o.num_proposals,
                              r->o.max_nodal_itr, r->o.dense_max, true, eng.st);
    if (s == SBP_OK) s = job_upload(*r->J, &g);
    if (s != SBP_OK) {
      hbm->give(bytes);
      r->set_error(s, sbp_last_error());
      r->owned.reset();
      r->J = nullptr;
      done.push_back(r);
      continue;
    }
    r->admit_bytes = bytes;
    r->t_admit_ms = now_ms();
    r->start_partition();
    eng.runs.push_back(r);
    max_active_seen = std::max(max_active_seen, (int32_t)eng.runs.size());
  }
  if (queue_head > 1024 && queue_head * 2 > queue.size()) {
    queue.erase(queue.begin(), queue.begin() + (long)queue_head);
    queue_head = 0;
  }
  return SBP_OK;
}

sbp_status Scheduler::step(std::vector<Run*>& done) {
  sbp_status s = admit(done);
  if (s != SBP_OK) return s;
  if (eng.runs.empty()) return SBP_OK;
  s = eng.tick();
  if (s != SBP_OK) return s;
  std::lock_guard<std::mutex> submit(cuda_submit_mutex());
  std::vector<Run*> keep;
  keep.reserve(eng.runs.size());
  for (Run* r : eng.runs) {
    if (r->stage != Run::kDone) {
      keep.push_back(r);
      continue;
    }
    r->t_done_ms = now_ms();
    hbm->give(r->admit_bytes);
    r->owned.reset();  // arena back to the pool, in stream order
    r->J = nullptr;
    r->release_events();
    done.push_back(r);
  }
  eng.runs.swap(keep);
  return SBP_OK;
}

Scheduler::~Scheduler() {
  // active jobs give their arenas back while the engine's stream exists
  for (Run* r : eng.runs) {
    if (hbm) hbm->give(r->admit_bytes);
    r->owned.reset();
    r->J = nullptr;
  }
  eng.runs.clear();
}

double now_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Idle engines of one device, reused by single-job calls (streams, events
// and staging buffers are made once).  They live until the process exits.
class EnginePool {
 public:
  Engine* take(int device, sbp_status* st) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      auto& v = idle_[device];
      if (!v.empty()) {
        Engine* e = v.back();
        v.pop_back();
        *st = SBP_OK;
        return e;
      }
    }
    Engine* e = new Engine();
    *st = e->init(device);
    if (*st != SBP_OK) {
      delete e;
      return nullptr;
    }
    return e;
  }
  void give(Engine* e) {
    e->reset();
    std::lock_guard<std::mutex> lk(mu_);
    idle_[e->device].push_back(e);
  }

 private:
  std::mutex mu_;
  std::map<int, std::vector<Engine*>> idle_;
};

static EnginePool& engine_pool() {
  static EnginePool* p = new EnginePool();
  return *p;
}

// Runs one job to the end on an engine of its own.
static sbp_status run_one(Job& J, Run& r) {
  sbp_status s = SBP_OK;
  Engine* eng = engine_pool().take(J.device, &s);
  if (!eng) return s;
  // the job's uploads were issued on its own stream
  cudaError_t e = cudaStreamSynchronize(J.st);
  if (e != cudaSuccess) {
    engine_pool().give(eng);
    return fail(SBP_ERR_CUDA, cudaGetErrorString(e));
  }
  const long long l0 = g_launches;
  const long long c0 = eng->graph_captures, p0 = eng->graph_replays;
  eng->runs.push_back(&r);
  while (r.stage != Run::kDone) {
    s = eng->tick();
    if (s != SBP_OK) break;
  }
  eng->runs.clear();
  // a failed tick leaves the engine's stream in an unknown state: drop it
  if (s != SBP_OK) return s;
  r.R.graph_captures = eng->graph_captures - c0;
  r.R.graph_replays = eng->graph_replays - p0;
  engine_pool().give(eng);
  r.R.kernel_launches = g_launches - l0;
  return SBP_OK;
}

sbp_status run_solo(Job& J, const sbp_options& o, int32_t* labels_out, sbp_report* rep) {
  Timer t;
  Run r;
  r.J = &J;
  r.o = o;
  r.labels_out = labels_out;
  r.start_partition();
  sbp_status s = run_one(J, r);
  if (s != SBP_OK) return s;
  r.R.ms_total = t.ms();
  if (r.status == SBP_OK && r.R.status != 0) r.status = (sbp_status)r.R.status;
  r.R.status = r.status;
  if (rep) *rep = r.R;
  if (r.status != SBP_OK && !r.error.empty()) return fail(r.status, r.error);
  return r.status;
}

sbp_status run_sweeps(Job& J, int32_t B, uint64_t seed, uint32_t seq0, int32_t num_batches,
                      int32_t sweeps, double* sums) {
  Run r;
  r.J = &J;
  sbp_default_options(&r.o);
  r.o.seed = seed;
  r.o.num_batches = num_batches;
  r.sums_out = sums;
  r.start_sweeps(B, seq0, sweeps);
  sbp_status s = run_one(J, r);
  if (s != SBP_OK) return s;
  if (r.status != SBP_OK) return fail(r.status, r.error);
  return SBP_OK;
}

}  // namespace sbp

// ------------------------------------------------------------------ C ABI --
using namespace sbp;

extern "C" uint64_t sbp_job_bytes(int32_t N, int32_t E, const sbp_options* o) {
  if (N < 1 || E < 0 || !o) return 0;
  return job_bytes(N, E, o->num_proposals, o->max_nodal_itr, dense_limit(N, E, o->dense_max));
}

extern "C" sbp_status sbp_partition_batch(const sbp_graph_csr* graphs, int32_t count,
                                          const sbp_options* o, const uint64_t* seeds,
                                          uint64_t hbm_budget, int32_t* const* labels_out,
                                          sbp_report* reports, sbp_batch_report* batch) {
  Timer t;
  if (count < 0 || (count > 0 && (!graphs || !labels_out)))
    return fail(SBP_ERR_INVALID, "bad batch arguments");
  sbp_status s = check_options(o);
  if (s != SBP_OK) return s;
  for (int32_t i = 0; i < count; ++i) {
    s = validate_graph(&graphs[i]);
    if (s != SBP_OK) return fail(s, "graph " + std::to_string(i) + ": " + sbp_last_error());
    if (!labels_out[i]) return fail(SBP_ERR_INVALID, "labels_out entry is NULL");
  }
  // the runs outlive the scheduler (declared first, destroyed last): on an
  // engine failure the scheduler still holds pointers to the active ones
  std::vector<std::unique_ptr<Run>> runs(count);
  Scheduler sch;
  s = sch.init(resolve_device(o->device), hbm_budget, 0);
  if (s != SBP_OK) return s;
  for (int32_t i = 0; i < count; ++i) {
    runs[i].reset(new Run());
    Run& r = *runs[i];
    r.graph = &graphs[i];
    r.o = *o;
    if (seeds) r.o.seed = seeds[i];
    r.labels_out = labels_out[i];
    r.id = i;
    sch.enqueue(&r);
  }
  const long long l0 = g_launches;
  std::vector<Run*> done;
  while (!sch.idle()) {
    s = sch.step(done);
    if (s != SBP_OK) return s;
  }
  sbp_status first = SBP_OK;
  std::string first_msg;
  for (int32_t i = 0; i < count; ++i) {
    Run& r = *runs[i];
    if (r.status == SBP_OK && r.R.status != 0) r.status = (sbp_status)r.R.status;
    r.R.status = r.status;
    r.R.ms_total = r.t_done_ms - r.t_admit_ms;
    if (reports) reports[i] = r.R;
    if (r.status != SBP_OK && first == SBP_OK) {
      first = r.status;
      first_msg = "graph " + std::to_string(i) + ": " + r.error;
    }
  }
  if (batch) {
    std::memset(batch, 0, sizeof(*batch));
    batch->count = count;
    batch->max_active = sch.max_active_seen;
    batch->ticks = sch.eng.ticks;
    batch->kernel_launches = g_launches - l0;
    batch->ms_device = sch.eng.device_ms();
    batch->peak_bytes = sch.hbm->peak;
    batch->ms_total = t.ms();
  }
  if (first != SBP_OK) return fail(first, first_msg);
  return SBP_OK;
}
