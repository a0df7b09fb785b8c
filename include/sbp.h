/*
 * sbp.h - C ABI of the B200-native stochastic block partitioner.
 *
 * This is the drop-in boundary for the SBP path of GSAP
 * (chih-chun-chang/GSAP).  GSAP's entry point is the header template
 *     template <typename T, typename V, typename W>
 *     void partition(Graph<T, V, W>& g);          // GSAP/partition.hpp:852-954
 * instantiated with <int, int, unsigned> (GSAP.cu:20,25).  include/partition.hpp
 * keeps that template and forwards to sbp_partition() below.  Everything
 * crosses this boundary as plain pointers and sizes.
 *
 * Graph convention: CSR with an N+1 entry row pointer (GSAP keeps N entries
 * and uses adj_node.size() as the end of the last row, load.hpp:96-116),
 * int32 vertex ids, uint32 edge weights >= 1, node degrees = weighted sums
 * (load.hpp:106,112).  Labels are int32 in [0, B).
 *
 * Errors: every call returns an sbp_status; sbp_last_error() gives a message
 * for the calling thread.  No call aborts the process.  (GSAP returns void
 * and ignores CUDA errors, partition.hpp:852.)
 */
#ifndef SBP_H
#define SBP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum sbp_status {
  SBP_OK = 0,
  SBP_ERR_INVALID = 1,   /* malformed input or option */
  SBP_ERR_CUDA = 2,      /* a CUDA runtime call failed */
  SBP_ERR_NOMEM = 3,     /* device or host allocation failed */
  SBP_ERR_BUDGET = 4,    /* the HBM budget of a server/batch is exceeded */
  SBP_ERR_TIMEOUT = 5,   /* a bounded device wait or a job deadline ran out */
  SBP_ERR_INTERNAL = 6,  /* an internal consistency check failed */
  SBP_ERR_BUSY = 7,      /* queue full / job still running */
  SBP_ERR_NOT_FOUND = 8, /* unknown job id */
  SBP_ERR_CANCELLED = 9  /* the job was cancelled */
} sbp_status;

/* A directed weighted graph in CSR, both directions (GSAP/graph.hpp:32-45). */
typedef struct sbp_graph_csr {
  int32_t N;                /* vertices */
  int32_t E;                /* edges (entries of each CSR) */
  const int32_t* out_ptr;   /* N+1 */
  const int32_t* out_idx;   /* E: destination of each out-edge */
  const uint32_t* out_w;    /* E */
  const int32_t* in_ptr;    /* N+1 */
  const int32_t* in_idx;    /* E: source of each in-edge */
  const uint32_t* in_w;     /* E */
  const uint32_t* deg_out;  /* N: weighted out-degree (node_deg_out) */
  const uint32_t* deg_in;   /* N: weighted in-degree (node_deg_in) */
} sbp_graph_csr;

/* Hyper-parameters of partition.hpp:855-861 plus what the reference fixes
 * implicitly (RNG seed, device). */
typedef struct sbp_options {
  uint64_t seed;           /* Philox key; the reference seeds curand with clock64() */
  int32_t num_proposals;   /* merge proposals per block, 10 (:855) */
  float reduction_rate;    /* 0.35 (:856) */
  int32_t max_nodal_itr;   /* 100 (:857) */
  int32_t num_batches;     /* Jacobi batches per nodal sweep, 4 (:858) */
  float threshold1;        /* 5e-4, bracket incomplete (:859) */
  float threshold2;        /* 1e-4, bracket complete (:860) */
  int32_t window;          /* moving-average window, 3 (:861) */
  int32_t max_outer;       /* cap on merge/golden-section steps (no reference counterpart) */
  int32_t device;          /* CUDA device ordinal, -1 = current device */
  int32_t use_graphs;      /* ticks of queued nodal sweeps as CUDA graphs (default 1) */
  int32_t verbose;         /* 1: one line per outer step on stderr; 2: also one per engine tick;
                              3: also each nodal batch's event-timed segments */
  int32_t dense_max;       /* keep M as dense B x B matrices while B <= dense_max
                              (0 = always CSR); default -1 = automatic:
                              max(4096, sqrt(32 E)), at most N */
  /* Scoring mode (no reference counterpart; defaults reproduce GSAP):
   * exact = 1 scores nodal moves and merges by the exact change of the MDL
   * (merged columns folded, new column degrees, self loops moved with the
   * vertex) instead of GSAP's dS terms, and compares partitions (stop test,
   * golden section, sbp_report.S) by the standard description length
   * (sbp_mdl_mode) instead of GSAP's formula; mh = 1 accepts nodal moves by
   * Metropolis-Hastings, u < exp(-beta dS_nats) p(s->r)/p(r->s) with the
   * Hastings ratio of GSAP's proposal, instead of dS < 0. */
  int32_t exact;           /* 0 (default) or 1 */
  int32_t mh;              /* 0 (default) or 1 */
  double beta;             /* inverse temperature of the MH test, per nat (default 3) */
  /* GSAP's merge grid (partition.hpp:335-336): GSAP launches every merge
   * kernel on nnz threads (nnz = entries of the out CSR) rounded up to 256,
   * so when B * num_proposals is larger (the first merge step, where
   * nnz ~ E < 10 N) the proposals of the last blocks are never drawn: their
   * slots keep what the buffers held, zeros in a fresh process, so those
   * blocks all propose block 0 with dS 0 and merge into it first.  1 does
   * the same (slots start at zero and keep earlier steps' values), 0 draws
   * and scores every proposal; -1 (default) = 1 with GSAP's scoring
   * (exact = 0), 0 in exact mode. */
  int32_t ref_grid;
  /* 1: time every phase with CUDA events around each nodal batch and
   * rebuild, filling sbp_report.ms_nodal, ms_nodal_kernel and ms_rebuild
   * (each event node costs a few microseconds of device time, about 10% of
   * a 200k partition); 0 (default): only ms_device, ms_total and the
   * merge and pre-build parts of ms_merge / ms_rebuild. */
  int32_t phase_timing;
} sbp_options;

/* What one partition run did.  Timings are CUDA-event milliseconds on the
 * run's stream except ms_total (host steady clock around the whole call). */
typedef struct sbp_report {
  int32_t B;                /* final number of blocks */
  double S;                 /* final MDL (partition.hpp:696-701, FP64) */
  int32_t outer_steps;      /* merge + golden-section steps */
  int32_t nodal_itrs;       /* nodal sweeps (each = num_batches batches) */
  int64_t nodal_proposals;  /* vertex moves evaluated */
  int64_t accepted_moves;   /* vertex moves applied */
  double ms_total;
  double ms_merge;          /* proposals, merge dS, merge application */
  double ms_nodal;          /* nodal batches (proposal, dS, accept) */
  double ms_rebuild;        /* blockmodel rebuilds and per-block terms */
  double ms_h2d;            /* graph upload (sbp_partition only) */
  double bytes_nodal;       /* algorithmic bytes, per the roofline model */
  double bytes_rebuild;
  double bytes_merge;
  int32_t status;
  double ms_device;         /* CUDA-event time of the whole run on its stream */
  double ms_nodal_kernel;   /* CUDA-event time of the nodal dS kernels alone */
  int64_t nodal_launches;   /* nodal batches run (one warp-kernel launch each) */
  int64_t kernel_launches;  /* kernels this library launched during the run */
  int64_t graph_captures;   /* sweep ticks captured as CUDA graphs (use_graphs) */
  int64_t graph_replays;    /* sweep ticks replayed from a captured graph */
} sbp_report;

void sbp_default_options(sbp_options* o);
const char* sbp_status_string(sbp_status s);
const char* sbp_last_error(void);

/* ---------------------------------------------------------------- partition
 * Replaces partition(g) (GSAP/partition.hpp:852-954): host graph in, host
 * labels out (N int32).  Uploads the graph, runs the merge / nodal /
 * golden-section loop on the GPU, downloads the labels. */
sbp_status sbp_partition(const sbp_graph_csr* g, const sbp_options* o, int32_t* labels_out,
                         sbp_report* report);

/* The same with the graph already resident in HBM (allocate_device.hpp:
 * 184-191 does this upload inside every partition call). */
typedef struct sbp_graph_dev sbp_graph_dev;
sbp_status sbp_graph_upload(const sbp_graph_csr* g, int32_t device, sbp_graph_dev** out);
sbp_status sbp_graph_release(sbp_graph_dev* g);
sbp_status sbp_partition_resident(sbp_graph_dev* g, const sbp_options* o, int32_t* labels_out,
                                  sbp_report* report);

/* ------------------------------------------------------------ device ingest
 * Resident graphs made on the device, without a host CSR.  GSAP builds the
 * CSR pair on the host (load.hpp:86-117) and uploads it
 * (allocate_device.hpp:184-191); these have no counterpart there.
 *
 * sbp_graph_from_device_edges: the CSR pair of an edge list already in the
 * memory of `device` (src, dst, w: E entries each; w NULL for unit
 * weights), the same arrays sbp_csr_from_edges builds on the host (rows in
 * input edge order).  The handle keeps its own copy of the edges; the
 * caller's arrays may be freed after the call.  SBP_ERR_INVALID for an
 * endpoint outside [0, N), a weight of 0 or a weighted degree above
 * 2^32 - 1.
 *
 * sbp_dcsbm_generate_device: the graph of sbp_dcsbm_generate with the same
 * parameters, edge for edge, generated on `device` (the planted labels and
 * the degree CDF on the host, degrees, block members and edges on the
 * device).  truth_out (N labels, may be NULL) receives the planted labels.
 * Requires N * deg_max < 2^31.
 *
 * sbp_graph_shape / sbp_graph_download: sizes and a host copy of a resident
 * graph's CSR pair (arrays sized as sbp_graph_csr; any pointer may be
 * NULL). */
struct sbp_dcsbm_params; /* defined with the host utilities below */
sbp_status sbp_graph_from_device_edges(int32_t N, int32_t E, const int32_t* src,
                                       const int32_t* dst, const uint32_t* w, int32_t device,
                                       sbp_graph_dev** out);
sbp_status sbp_dcsbm_generate_device(const struct sbp_dcsbm_params* p, int32_t device,
                                     int32_t* truth_out, sbp_graph_dev** out);
sbp_status sbp_graph_shape(const sbp_graph_dev* g, int32_t* N, int32_t* E);
sbp_status sbp_graph_download(const sbp_graph_dev* g, int32_t* out_ptr, int32_t* out_idx,
                              uint32_t* out_w, int32_t* in_ptr, int32_t* in_idx, uint32_t* in_w,
                              uint32_t* deg_out, uint32_t* deg_in);

/* ----------------------------------------------------------------- batched
 * Partitions `count` independent graphs in one call (no GSAP counterpart:
 * GSAP partitions one graph per process).  A multi-job engine advances every
 * admitted job one step per tick (a merge step or a nodal sweep), with one
 * kernel launch per kernel body for all jobs together.  Jobs are admitted in
 * order while their device arenas fit `hbm_budget` bytes (0: 90% of the
 * device's free memory); later jobs join as earlier ones finish.  Each
 * graph's labels and MDL are the same bits as sbp_partition of that graph
 * alone with the same options and seed.
 *   labels_out[i]  N_i labels of graph i
 *   seeds          per-graph seeds (NULL: o->seed for every graph)
 *   reports        one report per graph (optional)
 * Returns SBP_OK when every job succeeded, else the first failing job's
 * status (the other jobs still complete). */
typedef struct sbp_batch_report {
  int32_t count;
  int32_t max_active;       /* most jobs on the device at once */
  int64_t ticks;            /* engine steps */
  int64_t kernel_launches;  /* kernels launched by the call */
  double ms_total;          /* wall time of the call */
  double ms_device;         /* CUDA-event time from the first tick to the last */
  double peak_bytes;        /* largest sum of admitted job arenas */
} sbp_batch_report;

/* Device arena bytes of one job of N vertices and E edges under options o
 * (what the batch and server admission counts against the HBM budget). */
uint64_t sbp_job_bytes(int32_t N, int32_t E, const sbp_options* o);

sbp_status sbp_partition_batch(const sbp_graph_csr* graphs, int32_t count, const sbp_options* o,
                               const uint64_t* seeds, uint64_t hbm_budget,
                               int32_t* const* labels_out, sbp_report* reports,
                               sbp_batch_report* batch);

/* ------------------------------------------------------------------ served
 * A partition server (no GSAP counterpart): a host thread runs the same
 * engine continuously.  Requests are queued by sbp_server_submit (the graph
 * is copied, the caller may free it on return) and admitted in arrival order
 * as soon as the active jobs' device arenas leave room for them under the
 * HBM budget; admitted jobs join the running engine at its next tick, so
 * jobs that arrive while others run overlap on the device with them.  Small
 * and large graphs run in separate lanes (engines with their own stream and
 * host thread, one shared budget), so a small job's steps do not wait for a
 * large job's.  Each job keeps its graph, blockmodel, labels and RNG state
 * resident until it finishes; its result is the same bits as sbp_partition
 * alone. */
typedef struct sbp_server sbp_server;

typedef struct sbp_server_options {
  sbp_options partition;    /* loop options of every job (seed per request) */
  uint64_t hbm_budget;      /* bytes of job arenas at once (0: 90% of free memory) */
  int32_t max_active;       /* jobs on the device at once, per lane (0: no limit) */
  int32_t max_queued;       /* queued requests before submit says BUSY (0: no limit) */
  int32_t lanes;            /* engines by graph size, each on its own stream (0: 2) */
  int32_t lane_split;       /* graphs of N <= lane_split go to the small lane (0: 10000) */
} sbp_server_options;

typedef struct sbp_job_times {
  double ms_queue;          /* submit -> admitted to the device */
  double ms_run;            /* admitted -> result ready */
  double ms_latency;        /* submit -> result ready */
} sbp_job_times;

typedef struct sbp_server_stats {
  int64_t submitted, completed, failed;
  int32_t active, queued, max_active_seen;
  int64_t ticks;
  double bytes_active;      /* device bytes of the active jobs' arenas */
  double peak_bytes;
} sbp_server_stats;

void sbp_server_default_options(sbp_server_options* o);
sbp_status sbp_server_create(const sbp_server_options* o, sbp_server** out);
/* Queues a request; *id identifies it.  SBP_ERR_BUSY when the queue is full,
 * SBP_ERR_BUDGET when the job alone exceeds the HBM budget. */
sbp_status sbp_server_submit(sbp_server* s, const sbp_graph_csr* g, uint64_t seed, int64_t* id);
/* Result of a request: SBP_ERR_BUSY while it is queued or running
 * (timeout_ms = 0), or waits up to timeout_ms (< 0: no limit) for it.  On
 * completion fills labels_out (N ints), rep and times (each optional),
 * releases the request and returns the job's status; SBP_ERR_NOT_FOUND for
 * an unknown or already collected id. */
sbp_status sbp_server_poll(sbp_server* s, int64_t id, int32_t timeout_ms, int32_t* labels_out,
                           sbp_report* rep, sbp_job_times* times);
sbp_status sbp_server_stats_get(sbp_server* s, sbp_server_stats* out);
/* Stops the server thread after the jobs on the device finish; queued
 * requests are cancelled. */
sbp_status sbp_server_destroy(sbp_server* s);

/* ---------------------------------------------------- path pieces (parity)
 * Each runs one phase of the loop on the GPU from host inputs. */

/* calculate_new_csr (partition.hpp:707-849): the blockmodel of `part` as an
 * out CSR (rows = source block) and an in CSR (rows = destination block),
 * ascending columns, uint32 counts, and the weighted block degrees.  Row
 * pointers have B+1 entries; column/count arrays need capacity E.  *nnz
 * receives the number of nonzeros. */
sbp_status sbp_build_blockmodel(const sbp_graph_csr* g, const int32_t* part, int32_t B,
                                int32_t* out_ptr, int32_t* out_col, uint32_t* out_cnt,
                                int32_t* in_ptr, int32_t* in_col, uint32_t* in_cnt,
                                uint32_t* d_out, uint32_t* d_in, int64_t* nnz);

/* dS of moving verts[i] to props[i] (kernels.hpp:494-643, 1153-1726), every
 * move judged against the same `part` (one Jacobi batch without the accept). */
sbp_status sbp_delta_mdl_nodal(const sbp_graph_csr* g, const int32_t* part, int32_t B, int32_t nv,
                               const int32_t* verts, const int32_t* props, double* dS);

/* sbp_delta_mdl_nodal in a scoring mode: exact = 1 gives the exact change
 * of the MDL; logH (optional, nv doubles) receives each move's log Hastings
 * ratio ln(p(s->r)/p(r->s)) of GSAP's proposal (0 for a vertex without
 * edges).  No reference counterpart. */
sbp_status sbp_delta_mdl_nodal_mode(const sbp_graph_csr* g, const int32_t* part, int32_t B,
                                    int32_t nv, const int32_t* verts, const int32_t* props,
                                    int32_t exact, double* dS, double* logH);

/* Merge dS of B*np proposals (props[r*np+k] = target of block r's k-th
 * proposal; kernels.hpp:143-449) and each block's best proposal and its dS
 * (find_best_warp, kernels.hpp:452-491). */
sbp_status sbp_delta_mdl_merge(const sbp_graph_csr* g, const int32_t* part, int32_t B, int32_t np,
                               const int32_t* props, double* dS, int32_t* best, double* best_dS);

/* sbp_delta_mdl_merge in a scoring mode (exact = 1: the exact change of the
 * MDL of each merge; 0 (r = s) for a block proposed to itself).  No
 * reference counterpart. */
sbp_status sbp_delta_mdl_merge_mode(const sbp_graph_csr* g, const int32_t* part, int32_t B,
                                    int32_t np, const int32_t* props, int32_t exact, double* dS,
                                    int32_t* best, double* best_dS);

/* Merge proposals (kernels.hpp:726-856) from the Philox stream (seed, seq). */
sbp_status sbp_merge_proposals(const sbp_graph_csr* g, const int32_t* part, int32_t B, int32_t np,
                               uint64_t seed, uint32_t seq, int32_t* props);

/* One nodal batch over vertices [lo, hi) (propose_nodal_move,
 * partition.hpp:456-662): proposals from the Philox stream (seed, seq), dS,
 * accept if dS < 0, labels updated in place.  dS_rec[i] is the recorded dS
 * (0 when rejected), props[i] the proposal; *sum = sum of dS_rec. */
sbp_status sbp_nodal_batch(const sbp_graph_csr* g, int32_t* part, int32_t B, uint64_t seed,
                           uint32_t seq, int32_t lo, int32_t hi, double* dS_rec, int32_t* props,
                           double* sum);

/* sbp_nodal_batch in a scoring mode (exact, mh, beta as in sbp_options; the
 * MH uniform of vertex v is the third word of its Philox draw).  dS_rec[i]
 * is the dS of an accepted move (positive ones included under MH).  No
 * reference counterpart. */
sbp_status sbp_nodal_batch_mode(const sbp_graph_csr* g, int32_t* part, int32_t B, uint64_t seed,
                                uint32_t seq, int32_t lo, int32_t hi, int32_t exact, int32_t mh,
                                double beta, double* dS_rec, int32_t* props, double* sum);

/* `sweeps` nodal sweeps of `num_batches` Jacobi batches each, as the nodal
 * phase of partition() runs them (partition.hpp:912-916): batch k uses the
 * Philox stream (seed, seq0 + k).  The blockmodel is kept dense while
 * B <= dense_max (updated from the moved vertices' edges after each batch),
 * else rebuilt as CSR.  Labels updated in place; sums[k] = recorded dS sum
 * of batch k (sweeps * num_batches entries). */
sbp_status sbp_nodal_sweeps(const sbp_graph_csr* g, int32_t* part, int32_t B, uint64_t seed,
                            uint32_t seq0, int32_t num_batches, int32_t sweeps, int32_t dense_max,
                            double* sums);

/* One merge step (propose_block_merge + carry_out_best_merges,
 * partition.hpp:26-78, 324-454): labels updated in place; *B_new receives the
 * new block count. */
/* carry_out_best_merges (partition.hpp:26-78) alone, on the host (no GPU
 * is touched): blocks merge in ascending order of best_dS (equal values by
 * block id, NaN last), each into the current label of best[b] unless that
 * label is its own, until B_to_merge merges are made; map[b] receives the
 * new label of block b (surviving blocks renumbered in ascending order) and
 * *B_new the new block count. */
sbp_status sbp_apply_merges(int32_t B, int32_t B_to_merge, const int32_t* best,
                            const double* best_dS, int32_t* map, int32_t* B_new);

/* sbp_apply_merges computed on the GPU (`device`, -1 = current) the way
 * the partition loop applies its merges: the same map and block count
 * (carry_out_best_merges, partition.hpp:26-78), from host arrays. */
sbp_status sbp_apply_merges_device(int32_t B, int32_t B_to_merge, const int32_t* best,
                                   const double* best_dS, int32_t device, int32_t* map,
                                   int32_t* B_new);

sbp_status sbp_merge_step(const sbp_graph_csr* g, int32_t* part, int32_t B, int32_t B_to_merge,
                          int32_t np, uint64_t seed, uint32_t seq, int32_t* best, double* best_dS,
                          int32_t* B_new);

/* sbp_merge_step as the first merge step of a run with sbp_options.ref_grid
 * = ref_grid: with 1, the proposal slots past GSAP's merge grid (the nnz of
 * the out CSR rounded up to 256, partition.hpp:335-336) read the zeros of
 * fresh merge buffers instead of being drawn and scored. */
sbp_status sbp_merge_step_mode(const sbp_graph_csr* g, int32_t* part, int32_t B,
                               int32_t B_to_merge, int32_t np, uint64_t seed, uint32_t seq,
                               int32_t ref_grid, int32_t* best, double* best_dS, int32_t* B_new);

/* The MDL of a partition (compute_overall_entropy_cuda, partition.hpp:665-704). */
sbp_status sbp_mdl(const sbp_graph_csr* g, const int32_t* part, int32_t B, double* S,
                   double* data_S);

/* sbp_mdl with exact = 1: the standard description length of the
 * degree-corrected SBP in bits, (E h(B^2/E) + N ln B) / ln 2 - data_S with
 * h(x) = (1+x) ln(1+x) - x ln x, the objective exact mode searches B on
 * (GSAP's formula scales only part of h by E and mixes nats with bits).
 * exact = 0 is sbp_mdl.  No reference counterpart. */
sbp_status sbp_mdl_mode(const sbp_graph_csr* g, const int32_t* part, int32_t B, int32_t exact,
                        double* S, double* data_S);

/* The MDL of a blockmodel already in device memory (out CSR with B+1 row
 * pointers, block degrees), written to the device doubles *S and *data_S on
 * `stream` (a cudaStream_t; NULL = default stream), without allocating
 * anything: for callers that cannot let a library allocate device memory,
 * such as hosts that own all device memory through their own pool, or
 * serving loops that forbid the synchronisation a cudaMalloc or cudaFree can
 * cost.  The caller passes inputs and outputs; the scratch is a fixed ~1 MB
 * device array of the library, held by every GPU that loads it until the
 * process exits, so B <= 65536 (larger B returns SBP_ERR_INVALID).  The first
 * call on a device looks that array's address up (once per device, with the
 * device current), so make it before any stream capture; the address is not
 * valid after a cudaDeviceReset.  All calls share the array, which keeps the
 * last call's contents: calls that overlap on the GPU race.  This entry
 * point has no counterpart in the reference. */
sbp_status sbp_mdl_device_static(int32_t N, int32_t E, int32_t B, const int32_t* out_ptr,
                                 const int32_t* out_col, const uint32_t* out_cnt,
                                 const uint32_t* d_out, const uint32_t* d_in, double* S,
                                 double* data_S, void* stream);

/* ----------------------------------------------------------- host utilities */

/* Seeded directed DCSBM generator standing in for the GraphChallenge static
 * graphs: Dirichlet(alpha) block sizes, truncated power-law out-degrees,
 * in-block edges with probability p_in, destinations proportional to degree
 * within the chosen block, no self-loops or repeated edges, unit weights. */
typedef struct sbp_dcsbm_params {
  int32_t N;
  int32_t B;
  double alpha;       /* Dirichlet concentration of block sizes */
  double p_in;        /* probability an edge stays in its source block */
  int32_t deg_min;    /* out-degree support [deg_min, deg_max] */
  int32_t deg_max;
  double exponent;    /* P(k) ~ k^-exponent */
  uint64_t seed;
} sbp_dcsbm_params;

typedef struct sbp_edges sbp_edges;
sbp_status sbp_dcsbm_generate(const sbp_dcsbm_params* p, sbp_edges** out);
/* Sizes of an edge list; E may be NULL. */
sbp_status sbp_edges_size(const sbp_edges* e, int32_t* N, int32_t* E);
/* Copies the edge list (src, dst, w: E each) and the planted labels (N). Any
 * pointer may be NULL. */
sbp_status sbp_edges_copy(const sbp_edges* e, int32_t* src, int32_t* dst, uint32_t* w,
                          int32_t* truth);
void sbp_edges_free(sbp_edges* e);

/* The CSR pair of an edge list the way load.hpp:86-117 builds it: out rows
 * in edge order, in rows in edge order, weighted degrees. */
sbp_status sbp_csr_from_edges(int32_t N, int32_t E, const int32_t* src, const int32_t* dst,
                              const uint32_t* w, int32_t* out_ptr, int32_t* out_idx,
                              uint32_t* out_w, int32_t* in_ptr, int32_t* in_idx, uint32_t* in_w,
                              uint32_t* deg_out, uint32_t* deg_in);

/* GraphChallenge TSV ("src\tdst\tweight", 1-based) as load.hpp:6-133 reads
 * it, including its parse of a first field that holds a space (the first
 * line of lowOverlap_lowBlockSizeVar/1k parses as a self-loop).  N is the
 * largest source id, as in the reference.  truth_path (may be NULL) is the
 * "_truePartition.tsv" file ("vertex\tblock", 1-based, load.hpp:119-130);
 * without it the planted labels are -1. */
sbp_status sbp_load_tsv(const char* path, const char* truth_path, sbp_edges** out);

/* Pairwise recall, pairwise precision and NMI of `given` against `truth`
 * (evaluate.hpp:18-265) with 64-bit pair counts.  truth[i] < 0 = unknown. */
sbp_status sbp_evaluate(int32_t n, const int32_t* truth, const int32_t* given, double* recall,
                        double* precision, double* nmi);

#ifdef __cplusplus
}
#endif
#endif /* SBP_H */
