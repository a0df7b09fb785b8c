// The multi-job engine (engine.cu): Run is one job's partition() state,
// Engine advances a set of runs one tick at a time with multi-job launches.
#pragma once

#include "job.h"
#include "kernels.h"

#include <algorithm>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace sbp {

// Host clock in milliseconds (steady).
double now_ms();

// Serialises the CUDA calls of engines that run in different host threads.
std::mutex& cuda_submit_mutex();

// A graph held on the host by the engine (server requests are copied).
struct HostGraph {
  int32_t N = 0, E = 0;
  std::vector<int32_t> optr, oidx, iptr, iidx;
  std::vector<uint32_t> ow, iw, kdo, kdi;
  void assign(const sbp_graph_csr& g);
  sbp_graph_csr csr() const;
};

struct Run {
  Job* J = nullptr;
  const sbp_graph_csr* graph = nullptr;  // host graph uploaded at admission
  HostGraph graph_copy;                  // server requests: the copied graph
  sbp_graph_csr graph_view{};
  std::unique_ptr<Job> owned;  // jobs the engine admitted itself
  sbp_options o{};
  int32_t* labels_out = nullptr;  // host labels, written when the run finishes
  double* sums_out = nullptr;     // sweeps-only runs: per-batch dS sums
  sbp_report R{};
  sbp_status status = SBP_OK;
  std::string error;
  enum Stage { kMerge, kSweep, kFinish, kDone } stage = kMerge;
  bool finished = false;  // server requests: set by the lane under the server's lock
  bool sweeps_only = false;
  int32_t sweeps_total = 0;
  // loop state (partition.hpp:852-954)
  int32_t B = 0, B_to_merge = 0, BS = 0, itr = 0;
  uint32_t seq = 0;
  uint32_t seq_sweep0 = 0;  // seq of the outer step's first sweep
  int32_t sweep_k = 0;      // sweeps queued this tick
  Bracket large, med, small;
  double S = 0.0;
  std::vector<double> itr_dS;
  // per batch b, vertices by nodal kernel path (classify_batch): groups of
  // sizes list_n[3b .. 3b+2] starting at list_off[b] in lists_all
  std::vector<int32_t> lists_all, list_off, list_n;
  std::vector<double> batch_entries;
  double nnz_now = 0.0;
  double pre_bytes = 0.0;  // algorithmic bytes of this tick's builds before the merge or sweeps
  // device work left pending by the last host decision
  bool init = false, upload_lists = false, build = false, zero_itr = false;
  bool csr_fresh = false;
  // the pending build follows a merge step: the CSR arrays still hold the
  // blockmodel of the B_merged_from blocks before it, and the job's map the
  // merge, so a dense form is built from them rather than from the edges
  bool build_from_merge = false;
  int32_t B_merged_from = 0;
  // the golden section kept the step's labels, so the dense form still holds
  // their blockmodel (the next merge step reads its CSR form from it)
  bool dense_kept = false;
  int snap_slot = -1, restore_slot = -1;
  // this tick's offsets in the upload and readback buffers
  size_t up_lists = 0, rd_off = 0;
  cudaEvent_t ev_begin = nullptr;
  // scheduler / server bookkeeping
  double admit_bytes = 0.0;
  long long id = -1;
  double t_submit_ms = 0.0, t_admit_ms = 0.0, t_done_ms = 0.0;
  std::vector<int32_t> labels_store;

  Run() = default;
  Run(const Run&) = delete;
  Run& operator=(const Run&) = delete;
  // CUDA events of the run; call on the thread that drives the engine (a
  // server request is destroyed by whichever thread collects it)
  void release_events();
  ~Run();

  void setup_batches();
  void start_partition();
  void start_sweeps(int32_t B0, uint32_t seq0, int32_t sweeps);
  bool dense() const;
  void after_sweep(double dsum, double dataS, long long acc);
  void set_error(sbp_status st, const std::string& msg);
};

// The launches of one nodal batch position across runs.
struct SweepSlots {
  // heavy / nodal indexed by ScoreMode::slot(dense)
  Slot bt_csr, bt_dense, heavy[4], nodal[4], dupd, commit;
  RebuildSlots rebuild;
};

// The launches that end one queued sweep: MDL terms, MDL sum, stop test.
struct SweepEndSlots {
  Slot bt_csr, bt_dense, mdl, ctl;
};

class Engine {
 public:
  int device = 0;
  cudaStream_t st = nullptr, side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  std::vector<Run*> runs;
  long long ticks = 0;
  cudaEvent_t ev_first = nullptr;  // recorded at the first tick
  bool use_graphs = false;         // ticks of queued sweeps as CUDA graphs
  long long graph_captures = 0, graph_replays = 0;

  Engine() = default;
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;
  ~Engine();
  sbp_status init(int dev);
  // One step of every run that is not done; synchronises once.
  sbp_status tick();
  // CUDA-event time from the first tick to the end of the last one.
  double device_ms();
  // Forgets its runs and tick count (an idle engine, ready for reuse).
  void reset();

 private:
  Slot s_iota, s_lists, s_snap, s_restore, s_zero;
  DenseBuildSlots pre_dense;
  RebuildSlots pre_rebuild;
  Slot m_bt, m_props, m_delta, m_delta8, m_best;
  MergeApplySlots m_apply;  // merge application on the device (mergeapply.cu)
  Slot m_relabel;
  std::vector<SweepSlots> sw;     // [queued sweep][batch]
  std::vector<SweepEndSlots> ends;  // [queued sweep]
  Slot s_gather;
  std::vector<cudaEvent_t> ev;
  void *up_host = nullptr, *up_dev = nullptr, *desc_host = nullptr, *desc_dev = nullptr;
  void *rd_host = nullptr, *rd_dev = nullptr;
  size_t up_cap = 0, desc_cap = 0, rd_cap = 0;
  cudaGraphExec_t graph_exec = nullptr;  // the last captured sweep tick
  std::vector<unsigned char> graph_key;    // what the graph's launches were made from
  std::vector<unsigned char> key_scratch;
  long long graph_kernels = 0;            // kernel launches the graph holds
  int nb_slots_ = 0;  // batch positions per queued sweep in this tick's slots

  void* up_dev_ptr(size_t off) { return (char*)up_dev + off; }
  void* rd_dev_ptr(size_t off) { return (char*)rd_dev + off; }
  void ensure_slots(int K, int nb);
  void clear_slots();
  void add_run_work(Run& r);
  sbp_status launch_slot(Slot& s, size_t off, cudaStream_t stream);
};

// Device bytes of admitted job arenas against a cap; shared by the
// schedulers of one server.
struct HbmBudget {
  std::mutex mu;
  double cap = 0.0, used = 0.0, peak = 0.0;
  bool take(double bytes) {
    std::lock_guard<std::mutex> lk(mu);
    if (used + bytes > cap) return false;
    used += bytes;
    peak = std::max(peak, used);
    return true;
  }
  void give(double bytes) {
    std::lock_guard<std::mutex> lk(mu);
    used -= bytes;
  }
};

// Admission against an HBM budget in front of an engine (batched calls and
// the server): queued runs join the engine in order while their arenas fit.
class Scheduler {
 public:
  Engine eng;
  std::shared_ptr<HbmBudget> hbm;
  int32_t max_active = 0;
  std::vector<Run*> queue;  // waiting, in arrival order (front = next)
  size_t queue_head = 0;
  int32_t max_active_seen = 0;

  Scheduler() = default;
  Scheduler(const Scheduler&) = delete;
  Scheduler& operator=(const Scheduler&) = delete;
  ~Scheduler();
  // hbm_budget 0: 90% of the device's free memory.  `shared` (optional)
  // is a budget other schedulers also draw on; it is then used as is.
  sbp_status init(int device, uint64_t hbm_budget, int32_t max_active_jobs,
                  std::shared_ptr<HbmBudget> shared = nullptr);
  void enqueue(Run* r) { queue.push_back(r); }
  size_t queued() const { return queue.size() - queue_head; }
  bool idle() const { return queued() == 0 && eng.runs.empty(); }
  // Admits what fits, runs one tick, hands back the runs that ended.
  sbp_status step(std::vector<Run*>& done);

 private:
  sbp_status admit(std::vector<Run*>& done);
};

}  // namespace sbp
