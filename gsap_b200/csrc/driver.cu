// Host driver of the B200 stochastic block partitioner and the C ABI of
// include/sbp.h.
//
// The loop is GSAP's partition() (partition.hpp:852-954): start from B = N,
// then repeat { merge step; nodal sweeps until the moving-average dS test
// stops them; golden-section bookkeeping over B } until the bracket closes.
// Differences in how it runs on the device:
//   * one device arena per job (GSAP: four slabs plus separate buffers and
//     per-call allocations inside bb_segsort / mgpu / thrust);
//   * every kernel on one stream, issued by the engine (engine.cu) in ticks:
//     the host synchronises once per tick of queued nodal sweeps (ended on
//     the device by the stop test; the host reads their dS sums and MDLs)
//     and once per merge step (to apply the merges), where GSAP synchronises
//     after every batch and inside every rebuild;
//   * golden-section snapshots keep only the labels; the blockmodel of a
//     restored point is rebuilt from them (exactly the same matrix);
//   * merges are applied with a union-find pass over the ranked blocks, the
//     same result as GSAP's O(B * B_to_merge) relabel loop
//     (partition.hpp:41-56).
#include "../../include/sbp.h"
#include "common.cuh"
#include "job.h"
#include "kernels.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <future>
#include <memory>
#include <cstring>
#include <limits>
#include <mutex>
#include <numeric>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

namespace sbp {

static thread_local std::string g_last_error;

sbp_status fail(sbp_status st, const std::string& msg) {
  g_last_error = msg;
  return st;
}

sbp_status host_fail(sbp_status st, const char* msg) { return fail(st, msg); }


// ------------------------------------------------------------ validation --
// Sizes, arrays and row pointers (0 .. E, never decreasing): what an upload
// needs before the owner-filling kernels write through the row pointers.
static sbp_status validate_rows(const sbp_graph_csr* g) {
  if (!g) return fail(SBP_ERR_INVALID, "graph is NULL");
  if (g->N < 1 || g->E < 0) return fail(SBP_ERR_INVALID, "need N >= 1 and E >= 0");
  if (!g->out_ptr || !g->in_ptr || !g->deg_out || !g->deg_in)
    return fail(SBP_ERR_INVALID, "graph arrays are NULL");
  if (g->E > 0 && (!g->out_idx || !g->out_w || !g->in_idx || !g->in_w))
    return fail(SBP_ERR_INVALID, "graph arrays are NULL");
  const int32_t N = g->N;
  const int32_t* ptrs[2] = {g->out_ptr, g->in_ptr};
  const int32_t* idxs[2] = {g->out_idx, g->in_idx};
  const uint32_t* ws[2] = {g->out_w, g->in_w};
  const uint32_t* degs[2] = {g->deg_out, g->deg_in};
  // row pointers first: once they run from 0 to E without decreasing, every
  // entry index below is in [0, E)
  for (int d = 0; d < 2; ++d)
    if (ptrs[d][0] != 0 || ptrs[d][N] != g->E)
      return fail(SBP_ERR_INVALID, "row pointers must start at 0 and end at E");
  for (int d = 0; d < 2; ++d)
    for (int32_t v = 0; v < N; ++v)
      if (ptrs[d][v + 1] < ptrs[d][v]) return fail(SBP_ERR_INVALID, "row pointers decrease");
  return SBP_OK;
}

// The entries of a graph whose rows validate_rows accepted: vertex ids in
// range, weights >= 1, degrees equal to the weight sums.  Split by vertex
// over up to 8 threads for large graphs; returns the first error in
// (direction, vertex, entry) order, or nullptr.  Sets no thread's error, so
// that it can run beside the upload on a helper thread.
static const char* graph_entry_error(const sbp_graph_csr* g) {
  const int32_t N = g->N;
  const int32_t* ptrs[2] = {g->out_ptr, g->in_ptr};
  const int32_t* idxs[2] = {g->out_idx, g->in_idx};
  const uint32_t* ws[2] = {g->out_w, g->in_w};
  const uint32_t* degs[2] = {g->deg_out, g->deg_in};
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int T = (int)std::min<int64_t>({8, (int64_t)hw, std::max<int64_t>(1, g->E / 262144)});
  struct Bad {
    int32_t v = -1;
    const char* msg = nullptr;
  };
  std::vector<Bad> bad((size_t)T * 2);
  auto check = [&](int t) {
    const int32_t v0 = (int32_t)((int64_t)N * t / T), v1 = (int32_t)((int64_t)N * (t + 1) / T);
    for (int d = 0; d < 2; ++d) {
      Bad& b = bad[(size_t)t * 2 + d];
      for (int32_t v = v0; v < v1 && !b.msg; ++v) {
        uint64_t s = 0;
        for (int32_t j = ptrs[d][v]; j < ptrs[d][v + 1]; ++j) {
          if (idxs[d][j] < 0 || idxs[d][j] >= N) {
            b = Bad{v, "vertex id out of range"};
            break;
          }
          if (ws[d][j] == 0u) {
            b = Bad{v, "edge weights must be >= 1"};
            break;
          }
          s += ws[d][j];
        }
        if (!b.msg && s != degs[d][v]) b = Bad{v, "node degree differs from the sum of its edge weights"};
      }
      if (b.msg) break;  // a direction-0 error precedes every direction-1 error
    }
  };
  std::vector<std::thread> th;
  int spawned = 1;
  try {
    for (; spawned < T; ++spawned) th.emplace_back(check, spawned);
  } catch (const std::system_error&) {
    // no more threads: the remaining slices run here
  }
  for (int t = spawned; t < T; ++t) check(t);
  check(0);
  for (auto& x : th) x.join();
  for (int d = 0; d < 2; ++d)
    for (int t = 0; t < T; ++t)  // threads hold ascending vertex ranges
      if (bad[(size_t)t * 2 + d].msg) return bad[(size_t)t * 2 + d].msg;
  return nullptr;
}

sbp_status validate_graph(const sbp_graph_csr* g) {
  sbp_status s = validate_rows(g);
  if (s != SBP_OK) return s;
  const char* bad = graph_entry_error(g);
  return bad ? fail(SBP_ERR_INVALID, bad) : SBP_OK;
}

sbp_status validate_part(const int32_t* part, int32_t N, int32_t B) {
  if (!part) return fail(SBP_ERR_INVALID, "labels are NULL");
  if (B < 1 || B > N) return fail(SBP_ERR_INVALID, "need 1 <= B <= N");
  for (int32_t v = 0; v < N; ++v)
    if (part[v] < 0 || part[v] >= B) return fail(SBP_ERR_INVALID, "label out of [0, B)");
  return SBP_OK;
}

// ----------------------------------------------------------------- arena --
static int32_t scan_tiles_cap(int32_t N) { return 2 * (2 * ((N + 1) / 2048 + 2) + 2); }

size_t job_bytes(int32_t N, int32_t E, int32_t np, int32_t max_itr, int32_t dense_cap) {
  const int32_t tiles = scan_tiles_cap(N);
  size_t n1 = (size_t)N + 1, e = (size_t)E > 0 ? (size_t)E : 1;
  size_t b = 0;
  auto add = [&](size_t elems, size_t sz) { b += ((elems * sz) + 255) & ~size_t(255); };
  // graph
  add(n1, 4); add(n1, 4); add(e, 4); add(e, 4); add(e, 4); add(e, 4); add(e, 4); add(e, 4);
  add(N, 4); add(N, 4);
  // labels, snapshots, map
  for (int i = 0; i < 6; ++i) add(n1, 4);
  // blockmodel
  add(n1, 4); add(n1, 4); add(e, 4); add(e, 4); add(e, 4); add(e, 4); add(N, 4); add(N, 4);
  for (int i = 0; i < 6; ++i) add(N, 8);
  add(N, 4); add(N, 1);
  // rebuild scratch
  for (int d = 0; d < 2; ++d) {
    add(n1, 4); add(n1, 4); add(N, 4); add(e, 4); add(e, 4); add(e, 4); add(e, 4); add(n1, 4);
    add(N, 4);
  }
  add(2, 4);
  add((size_t)tiles, 4);
  // nodal / merge
  add(N, 8);
  add((size_t)N * np, 4);
  add((size_t)N * np, 8);
  add((size_t)N * np, 8);
  add(N, 8);
  add((size_t)max_itr, 8); add((size_t)max_itr, 8); add((size_t)max_itr, 8);
  add((size_t)N, 4); add(2, 4); add(2, 4);
  add((size_t)dense_cap * dense_cap, 4); add((size_t)dense_cap * dense_cap, 4);
  add((size_t)2 * dense_cap * ((dense_cap + 31) / 32), 4);
  add(kCommitCtas, 8); add(kCommitCtas, 8); add(1, 4);
  // merge application on the device
  b += merge_apply_bytes(N);
  add(2, 4);
  return b + 4096;
}

void Job::release() {
  if (!mem && !st) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(device);
  if (lean) {
    if (mem) {
      if (pool_stream) cudaFreeAsync(mem, pool_stream);
      else cudaFree(mem);
    }
    mem = nullptr;
    st = nullptr;
    cudaSetDevice(cur);
    return;
  }
  if (mem) cudaFreeAsync(mem, st);
  if (st) cudaStreamSynchronize(st);
  if (fork) cudaEventDestroy(fork);
  if (join) cudaEventDestroy(join);
  fork = join = nullptr;
  if (side) cudaStreamDestroy(side);
  side = nullptr;
  if (st) cudaStreamDestroy(st);
  cudaFreeHost(h_best);
  cudaFreeHost(h_best_dS);
  cudaFreeHost(h_map);
  h_best = nullptr;
  h_best_dS = nullptr;
  h_map = nullptr;
  cudaSetDevice(cur);
  mem = nullptr;
  st = nullptr;
}

sbp_status device_xlx_table(int device, const double** out) {
  static std::mutex mu;
  static double* tab[64] = {};
  if (device < 0 || device >= 64) return fail(SBP_ERR_INVALID, "device ordinal too large");
  std::lock_guard<std::mutex> lk(mu);
  if (!tab[device]) {
    double* t = nullptr;
    SBP_CUDA(cudaMalloc(&t, sizeof(double) * 2 * kXlxTable));
    cudaStream_t st;
    SBP_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    fill_xlx_table(t, st);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) return fail(SBP_ERR_CUDA, cudaGetErrorString(e));
    tab[device] = t;
  }
  *out = tab[device];
  return SBP_OK;
}

sbp_status job_create(Job& J, int device, int32_t N, int32_t E, int32_t np, int32_t max_itr,
                      int32_t dense_max, bool lean, cudaStream_t engine_stream) {
  J.device = device;
  J.lean = lean;
  J.dense_cap = dense_limit(N, E, dense_max);
  J.dense_eff = J.dense_cap;
  J.N = N;
  J.E = E;
  J.np = np;
  J.max_itr = max_itr;
  SBP_CUDA(cudaSetDevice(device));
  static std::once_flag once[64];
  if (device >= 0 && device < 64)
    std::call_once(once[device], [device] {
      init_kernel_attributes();
      init_nodal_attributes();
      // arenas come from the stream-ordered pool; freed ones stay in it, so
      // repeated calls reuse device memory without allocating from the driver
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      }
    });
  const double* xlx = nullptr;
  sbp_status xs = device_xlx_table(device, &xlx);
  if (xs != SBP_OK) return xs;
  int32_t tiles = scan_tiles_cap(N);
  J.mem_bytes = job_bytes(N, E, np, max_itr, J.dense_cap);
  if (lean) {
    J.st = engine_stream;
  } else {
    SBP_CUDA(cudaStreamCreateWithFlags(&J.st, cudaStreamNonBlocking));
    SBP_CUDA(cudaStreamCreateWithFlags(&J.side, cudaStreamNonBlocking));
    SBP_CUDA(cudaEventCreateWithFlags(&J.fork, cudaEventDisableTiming));
    SBP_CUDA(cudaEventCreateWithFlags(&J.join, cudaEventDisableTiming));
  }
  if (cudaMallocAsync(&J.mem, J.mem_bytes, J.st) != cudaSuccess) {
    cudaGetLastError();
    J.mem = nullptr;
    return fail(SBP_ERR_NOMEM, "device arena of " + std::to_string(J.mem_bytes) + " bytes");
  }
  J.pool_stream = J.st;
  Arena A{(char*)J.mem, J.mem_bytes, 0};
  size_t n1 = (size_t)N + 1, e = (size_t)E > 0 ? (size_t)E : 1;
  DevGraph& g = J.g;
  g.N = N;
  g.E = E;
  g.optr = A.take<int32_t>(n1); g.iptr = A.take<int32_t>(n1);
  g.oidx = A.take<int32_t>(e); g.iidx = A.take<int32_t>(e);
  g.ow = A.take<uint32_t>(e); g.iw = A.take<uint32_t>(e);
  g.osrc = A.take<int32_t>(e); g.isrc = A.take<int32_t>(e);
  g.kdo = A.take<uint32_t>(N); g.kdi = A.take<uint32_t>(N);
  J.part = A.take<int32_t>(n1); J.newlab = A.take<int32_t>(n1); J.map = A.take<int32_t>(n1);
  for (int i = 0; i < 3; ++i) J.snap[i] = A.take<int32_t>(n1);
  DevBM& m = J.m;
  m.optr = A.take<int32_t>(n1); m.iptr = A.take<int32_t>(n1);
  m.ocol = A.take<int32_t>(e); m.icol = A.take<int32_t>(e);
  m.ocnt = A.take<uint32_t>(e); m.icnt = A.take<uint32_t>(e);
  m.d_out = A.take<uint32_t>(N); m.d_in = A.take<uint32_t>(N);
  m.ld_out = A.take<double>(N); m.ld_in = A.take<double>(N);
  m.dSout = A.take<double>(N); m.ambout = A.take<double>(N);
  m.ambin = A.take<double>(N); m.sinfull = A.take<double>(N);
  m.nbr_s = A.take<int32_t>(N); m.use_rand = A.take<uint8_t>(N);
  for (int d = 0; d < 2; ++d) {
    RebuildDir& r = J.rs.d[d];
    r.cnt = A.take<int32_t>(n1); r.seg = A.take<int32_t>(n1); r.vofs = A.take<int32_t>(N);
    r.tcol = A.take<int32_t>(e); r.tw = A.take<uint32_t>(e);
    r.ucol = A.take<int32_t>(e); r.uw = A.take<uint32_t>(e);
    r.uniq = A.take<int32_t>(n1); r.big = A.take<int32_t>(N);
  }
  J.rs.big_count = A.take<int32_t>(2);
  J.rs.tile = A.take<int32_t>(tiles);
  J.rs.tile_cap = tiles;
  J.rec = A.take<double>(N);
  J.props = A.take<int32_t>((size_t)N * np);
  J.mdS = A.take<double>((size_t)N * np);
  J.mdsin = A.take<double>((size_t)N * np);
  J.best = J.newlab;  // merge and nodal phases never overlap
  J.best_dS = A.take<double>(N);
  J.dsum = A.take<double>(max_itr);
  J.dataS = A.take<double>(max_itr);
  J.acc = (long long*)A.take<double>(max_itr);
  J.lists = A.take<int32_t>((size_t)N);
  J.err = A.take<int32_t>(2);
  J.ctl = A.take<int32_t>(2);
  if (J.dense_cap > 0) {
    m.Md = A.take<uint32_t>((size_t)J.dense_cap * J.dense_cap);
    m.MTd = A.take<uint32_t>((size_t)J.dense_cap * J.dense_cap);
    m.Sd = A.take<uint32_t>((size_t)2 * J.dense_cap * ((J.dense_cap + 31) / 32));
  }
  m.xlx = const_cast<double*>(xlx);
  J.cs.part_sum = A.take<double>(kCommitCtas);
  J.cs.part_cnt = A.take<long long>(kCommitCtas);
  J.cs.ticket = A.take<unsigned>(1);
  {
    const size_t mab = merge_apply_bytes(N);
    char* base = A.take<char>(mab);
    if (base) J.ma = merge_apply_carve(base, N);
    J.ma_out = A.take<int32_t>(2);
  }
  if (!J.cs.ticket || !J.ma_out || (J.dense_cap > 0 && !m.Sd))
    return fail(SBP_ERR_INTERNAL, "arena sizing");
  SBP_CUDA(cudaMemsetAsync(J.err, 0, 8, J.st));
  SBP_CUDA(cudaMemsetAsync(J.cs.ticket, 0, 4, J.st));
  return SBP_OK;
}

__global__ void fill_src_kernel(const int32_t* __restrict__ ptr, int32_t N, int32_t* src) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  for (int32_t j = ptr[v]; j < ptr[v + 1]; ++j) src[j] = v;
}


sbp_status job_upload(Job& J, const sbp_graph_csr* h) {
  DevGraph& g = J.g;
  size_t n1 = (size_t)J.N + 1, E = (size_t)J.E;
  cudaStream_t st = J.st;
  SBP_CUDA(cudaMemcpyAsync(g.optr, h->out_ptr, 4 * n1, cudaMemcpyHostToDevice, st));
  SBP_CUDA(cudaMemcpyAsync(g.iptr, h->in_ptr, 4 * n1, cudaMemcpyHostToDevice, st));
  if (E) {
    SBP_CUDA(cudaMemcpyAsync(g.oidx, h->out_idx, 4 * E, cudaMemcpyHostToDevice, st));
    SBP_CUDA(cudaMemcpyAsync(g.iidx, h->in_idx, 4 * E, cudaMemcpyHostToDevice, st));
    SBP_CUDA(cudaMemcpyAsync(g.ow, h->out_w, 4 * E, cudaMemcpyHostToDevice, st));
    SBP_CUDA(cudaMemcpyAsync(g.iw, h->in_w, 4 * E, cudaMemcpyHostToDevice, st));
  }
  SBP_CUDA(cudaMemcpyAsync(g.kdo, h->deg_out, 4 * (size_t)J.N, cudaMemcpyHostToDevice, st));
  SBP_CUDA(cudaMemcpyAsync(g.kdi, h->deg_in, 4 * (size_t)J.N, cudaMemcpyHostToDevice, st));
  ++g_launches;
  fill_src_kernel<<<(J.N + 255) / 256, 256, 0, st>>>(g.optr, J.N, g.osrc);
  J.h_optr.assign(h->out_ptr, h->out_ptr + J.N + 1);
  J.h_iptr.assign(h->in_ptr, h->in_ptr + J.N + 1);
  ++g_launches;
  fill_src_kernel<<<(J.N + 255) / 256, 256, 0, st>>>(g.iptr, J.N, g.isrc);
  SBP_CUDA(cudaGetLastError());
  return SBP_OK;
}

int resolve_device(int32_t d) {
  if (d >= 0) return d;
  int cur = 0;
  cudaGetDevice(&cur);
  return cur;
}

// ------------------------------------------------------------ merge apply --
// Block ids 0..n-1 in ascending order of key[id], equal keys by id: an LSD
// radix sort of (key, id) pairs with 8-bit digits (stable, so ids stay
// ascending within equal keys), skipping digits that all keys share.  Large
// inputs are split over up to 8 host threads: each counts the digits of its
// contiguous slice, then writes the slice to the offsets that the counts of
// the slices before it leave, which keeps the pass stable.
static void rank_by_key(std::vector<uint64_t> key, std::vector<int32_t>& order) {
  const size_t n = key.size();
  order.resize(n);
  std::iota(order.begin(), order.end(), 0);
  std::vector<uint64_t> k2(n);
  std::vector<int32_t> o2(n);
  constexpr int kDigits = 256;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  int T = (int)std::min<size_t>({8, (size_t)hw, std::max<size_t>(1, n / 32768)});
  std::vector<uint32_t> cnt((size_t)T * kDigits);
  auto slice = [&](int t, size_t& lo, size_t& hi) {
    lo = n * (size_t)t / (size_t)T;
    hi = n * (size_t)(t + 1) / (size_t)T;
  };
  auto count_pass = [&](int t, int shift) {
    size_t lo, hi;
    slice(t, lo, hi);
    uint32_t* c = cnt.data() + (size_t)t * kDigits;
    std::fill(c, c + kDigits, 0u);
    for (size_t i = lo; i < hi; ++i) ++c[(key[i] >> shift) & 0xff];
  };
  auto scatter_pass = [&](int t, int shift) {
    size_t lo, hi;
    slice(t, lo, hi);
    // start of each digit for this slice: all smaller digits, then this
    // digit in the slices before
    size_t at[kDigits];
    size_t run = 0;
    for (int d = 0; d < kDigits; ++d) {
      size_t before = 0;
      for (int u = 0; u < T; ++u) {
        if (u == t) before = run;
        run += cnt[(size_t)u * kDigits + d];
      }
      at[d] = before;
    }
    for (size_t i = lo; i < hi; ++i) {
      const size_t q = at[(key[i] >> shift) & 0xff]++;
      k2[q] = key[i];
      o2[q] = order[i];
    }
  };
  // every thread runs the same passes; a pass's phases are separated by a
  // barrier (all T threads arrive at each one, so every wait ends)
  std::atomic<int> arrived{0};
  std::atomic<int> phase{0};
  auto barrier = [&](int& my_phase) {
    ++my_phase;
    if (arrived.fetch_add(1) + 1 == T * my_phase) phase.store(my_phase);
    while (phase.load() < my_phase) std::this_thread::yield();
  };
  auto worker = [&](int t) {
    int my_phase = 0;
    for (int shift = 0; shift < 64; shift += 8) {
      count_pass(t, shift);
      barrier(my_phase);
      bool one = false;
      for (int d = 0; d < kDigits && !one; ++d) {
        size_t tot = 0;
        for (int u = 0; u < T; ++u) tot += cnt[(size_t)u * kDigits + d];
        one = tot == n;
      }
      if (one) {
        barrier(my_phase);  // counts are read before the next pass clears them
        continue;
      }
      scatter_pass(t, shift);
      barrier(my_phase);
      if (t == 0) {
        key.swap(k2);
        order.swap(o2);
      }
      barrier(my_phase);
    }
  };
  // the helpers wait at a gate until all of them exist; if one cannot be
  // started, the others are released without work and the sort runs here
  std::atomic<int> gate{0};  // 0: wait, 1: run, -1: cancelled
  auto start = [&](int t) {
    while (gate.load() == 0) std::this_thread::yield();
    if (gate.load() > 0) worker(t);
  };
  std::vector<std::thread> th;
  try {
    for (int t = 1; t < T; ++t) th.emplace_back(start, t);
    gate.store(1);
  } catch (const std::system_error&) {
    gate.store(-1);
    for (auto& x : th) x.join();
    th.clear();
    T = 1;
  }
  worker(0);
  for (auto& x : th) x.join();
}

// carry_out_best_merges (partition.hpp:26-78).  Blocks are ranked by their
// best dS (ascending, ties by block id: thrust::sort_by_key's stable radix
// sort over an id sequence, partition.hpp:442-447; NaN last); then in that
// order each block merges into the current label of its best target unless
// that label is itself.  Union-find gives the same labels as the reference's
// relabel-all loop.  Surviving labels are renumbered in ascending order
// (std::set, :58-68).  Returns the new block count.
int32_t apply_merges_host(int32_t B, int32_t B_to_merge, const int32_t* best,
                                 const double* best_dS, int32_t* map_out) {
  // the targets come from the device: never index with one out of range
  for (int32_t b = 0; b < B; ++b)
    if (best[b] < 0 || best[b] >= B) return -1;
  // order-preserving integer keys of the dS values (NaN last)
  std::vector<uint64_t> key(B);
  for (int32_t b = 0; b < B; ++b) {
    double x = best_dS[b];
    uint64_t k;
    if (std::isnan(x)) {
      k = ~0ull;
    } else {
      if (x == 0.0) x = 0.0;  // -0 ranks with +0
      uint64_t u;
      std::memcpy(&u, &x, 8);
      k = (u >> 63) ? ~u : (u | (1ull << 63));
    }
    key[b] = k;
  }
  std::vector<int32_t> ranked;
  rank_by_key(key, ranked);
  std::vector<int32_t> parent(B);
  std::iota(parent.begin(), parent.end(), 0);
  auto find = [&](int32_t x) {
    int32_t r = x;
    while (parent[r] != r) r = parent[r];
    while (parent[x] != r) {
      int32_t n = parent[x];
      parent[x] = r;
      x = n;
    }
    return r;
  };
  int32_t merged = 0;
  for (int32_t c = 0; c < B && merged < B_to_merge; ++c) {
    int32_t from = ranked[c];
    int32_t to = find(best[from]);
    if (to != from) {
      parent[from] = to;
      ++merged;
    }
  }
  // a block is a root iff it never merged away (roots keep parent == self)
  std::vector<int32_t> rootid(B, -1);
  int32_t next = 0;
  for (int32_t b = 0; b < B; ++b)
    if (parent[b] == b) rootid[b] = next++;
  for (int32_t b = 0; b < B; ++b) map_out[b] = rootid[find(b)];
  return next;
}

int32_t dense_limit(int32_t N, int32_t E, int32_t dense_max) {
  int64_t d = dense_max;
  if (dense_max < 0) d = std::max<int64_t>(4096, (int64_t)std::sqrt(32.0 * (double)E));
  return (int32_t)std::max<int64_t>(0, std::min<int64_t>(N, d));
}

double model_S(int32_t B, int32_t N, int32_t E, int32_t exact) {
  double b = (double)B;
  double x = b * b / (double)E;
  // the standard description length's model term, in bits:
  // (E h(x) + N ln B) / ln 2, h(x) = (1+x) ln(1+x) - x ln x
  if (exact)
    return ((double)E * ((1.0 + x) * std::log(1.0 + x) - x * std::log(x)) +
            (double)N * std::log(b)) / 0.6931471805599453;
  // partition.hpp:696-699 (Q6)
  return (double)E * (1.0 + x) * std::log(1.0 + x) - x * std::log(x) + (double)N * std::log(b);
}

static bool is_dense(const Job& J, int32_t B) { return B <= J.dense_eff; }

// The blockmodel of the current labels, in the form used at this B: dense
// B x B matrices for small B, the CSR pair otherwise.
static void build_model(Job& J, int32_t B, cudaStream_t st) {
  if (is_dense(J, B)) dense_build(J.g, J.part, B, J.m, st);
  else rebuild_blockmodel(J.g, J.part, B, J.m, J.rs, st);
}

static void block_terms_any(Job& J, int32_t B, int draws, uint64_t seed, uint32_t seq,
                            cudaStream_t st) {
  if (is_dense(J, B)) block_terms_dense(J.m, B, draws, seed, seq, st);
  else block_terms(J.m, B, draws, seed, seq, st);
}

bool heavy_vertex(const Job& J, int32_t v) {
  const int32_t t = nodal_heavy_threshold();
  return J.h_optr[v + 1] - J.h_optr[v] > t || J.h_iptr[v + 1] - J.h_iptr[v] > t;
}

void classify_batch(const Job& J, const int32_t* verts, int32_t lo, int32_t count,
                    std::vector<int32_t>& out, int32_t n[3]) {
  const size_t at = out.size();
  out.resize(at + (size_t)std::max(count, 0));
  int32_t* o = out.data() + at;
  n[0] = n[1] = n[2] = 0;
  if (count <= 0) return;
  // The kernels run their items in list order, the larger vertices first: a
  // longest-first schedule, so that a launch does not end on a tail of its
  // slowest items (10% of a 200k partition), and small vertices paired with
  // ones of about their size.  Each class is ordered by entry count, largest
  // first, ties by batch index (a counting sort: the small and mid classes
  // have at most 2 * kWarpList entries); a vertex's result does not depend on
  // where it runs.
  std::vector<int32_t> ent((size_t)count);
  std::vector<uint8_t> cls((size_t)count);
  int32_t emax = 0;
  for (int32_t i = 0; i < count; ++i) {
    const int32_t v = verts ? verts[i] : lo + i;
    const int32_t e = (J.h_optr[v + 1] - J.h_optr[v]) + (J.h_iptr[v + 1] - J.h_iptr[v]);
    ent[i] = e;
    cls[i] = heavy_vertex(J, v) ? 2 : e <= kSmallEntries ? 0 : 1;
    ++n[cls[i]];
    if (cls[i] < 2) emax = std::max(emax, e);
  }
  std::vector<int32_t> start((size_t)emax + 2, 0);
  int32_t base = 0;
  for (int c = 0; c < 2; ++c) {
    // descending entry count: bucket emax first
    std::fill(start.begin(), start.end(), 0);
    for (int32_t i = 0; i < count; ++i)
      if (cls[i] == c) ++start[(size_t)(emax - ent[i]) + 1];
    for (size_t k = 1; k < start.size(); ++k) start[k] += start[k - 1];
    for (int32_t i = 0; i < count; ++i)
      if (cls[i] == c) o[base + start[(size_t)(emax - ent[i])]++] = i;
    base += n[c];
  }
  int32_t* h = o + base;
  int32_t nh = 0;
  for (int32_t i = 0; i < count; ++i)
    if (cls[i] == 2) h[nh++] = i;
  std::stable_sort(h, h + nh, [&](int32_t x, int32_t y) { return ent[x] > ent[y]; });
}

NodalAux nodal_lists(Job& J, const int32_t* dev, const int32_t n[3]) {
  NodalAux a;
  a.small = dev;
  a.nsmall = n[0];
  a.mid = dev + n[0];
  a.nmid = n[1];
  a.heavy = dev + n[0] + n[1];
  a.nheavy = n[2];
  a.err = J.err;
  a.side = J.side;
  a.fork = J.fork;
  a.join = J.join;
  return a;
}

static sbp_status merge_step(Job& J, int32_t& B, int32_t B_to_merge, uint64_t seed, uint32_t seq,
                             bool keep_dS, int32_t ref_grid = 0) {
  cudaStream_t st = J.st;
  if (!J.h_best) {
    SBP_CUDA(cudaMallocHost(&J.h_best, sizeof(int32_t) * (size_t)J.N));
    SBP_CUDA(cudaMallocHost(&J.h_best_dS, sizeof(double) * (size_t)J.N));
    SBP_CUDA(cudaMallocHost(&J.h_map, sizeof(int32_t) * ((size_t)J.N + 1)));
  }
  // the merge kernels read the CSR form, stale after dense nodal sweeps
  if (is_dense(J, B)) rebuild_blockmodel(J.g, J.part, B, J.m, J.rs, st);
  block_terms(J.m, B, 0, seed, 0, st);
  MergeGrid grid;
  grid.dS = J.mdS;  // per-proposal scratch, and the slots' kept dS
  grid.dsin = J.mdsin;
  if (ref_grid) {
    // a fresh run's merge buffers: the slots GSAP's grid leaves out read zeros
    const size_t slots = (size_t)J.N * J.np;
    SBP_CUDA(cudaMemsetAsync(J.props, 0, 4 * slots, st));
    SBP_CUDA(cudaMemsetAsync(J.mdS, 0, 8 * slots, st));
    SBP_CUDA(cudaMemsetAsync(J.mdsin, 0, 8 * slots, st));
    grid.on = 1;
  }
  merge_proposals(J.m, B, J.np, seed, seq, J.props, st, grid);
  merge_delta(J.m, B, J.E, J.np, J.props, keep_dS ? J.mdS : nullptr, J.best, J.best_dS, st, 0,
              grid);
  SBP_CUDA(cudaMemcpyAsync(J.h_best, J.best, 4 * (size_t)B, cudaMemcpyDeviceToHost, st));
  SBP_CUDA(cudaMemcpyAsync(J.h_best_dS, J.best_dS, 8 * (size_t)B, cudaMemcpyDeviceToHost, st));
  SBP_CUDA(cudaStreamSynchronize(st));
  int32_t nb = apply_merges_host(B, B_to_merge, J.h_best, J.h_best_dS, J.h_map);
  if (nb < 0) return fail(SBP_ERR_INTERNAL, "merge target out of range");
  SBP_CUDA(cudaMemcpyAsync(J.map, J.h_map, 4 * (size_t)B, cudaMemcpyHostToDevice, st));
  relabel(J.part, J.N, J.map, st);
  B = nb;
  return SBP_OK;
}

// A job with the graph uploaded, for the one-shot entry points.
int32_t env_dense_max() {
  const char* e = std::getenv("SBP_DENSE_MAX");
  return e ? std::atoi(e) : 4096;
}

// The entries are checked on a helper thread while the host thread creates
// the arena and uploads (the upload only needs valid row pointers); no
// kernel reads an entry before the check has passed.
static sbp_status job_for(Job& J, const sbp_graph_csr* g, int device, int32_t np, int32_t max_itr,
                          int32_t dense_max) {
  sbp_status s = validate_rows(g);
  if (s != SBP_OK) return s;
  std::future<const char*> entries;
  try {
    entries = std::async(std::launch::async, graph_entry_error, g);
  } catch (const std::system_error&) {
    const char* bad = graph_entry_error(g);  // no thread to spare: check first
    if (bad) return fail(SBP_ERR_INVALID, bad);
  }
  s = job_create(J, resolve_device(device), g->N, g->E, np, max_itr, dense_max);
  if (s == SBP_OK) s = job_upload(J, g);
  const char* bad = entries.valid() ? entries.get() : nullptr;
  if (bad) return fail(SBP_ERR_INVALID, bad);
  return s;
}

// Validates the graph and the labels, then creates the job, uploads both
// and builds the blockmodel of the labels.
// Rebuild shape of the one-shot entry points: the defaults, or the one in
// SBP_REBUILD_WARP_CAP / SBP_REBUILD_BIG_ENTRIES (tests check every shape
// the autotuner may pick).
static RebuildTune env_rebuild_shape() {
  RebuildTune t;
  if (const char* e = std::getenv("SBP_REBUILD_WARP_CAP")) t.warp_cap = std::atoi(e);
  if (const char* e = std::getenv("SBP_REBUILD_BIG_ENTRIES")) t.big_entries = std::atoi(e);
  return t;
}

static sbp_status prepare(Job& J, const sbp_graph_csr* g, const int32_t* part, int32_t B,
                          int32_t np, int32_t max_itr) {
  sbp_status s = validate_graph(g);
  if (s != SBP_OK) return s;
  s = validate_part(part, g->N, B);
  if (s != SBP_OK) return s;
  s = job_create(J, resolve_device(-1), g->N, g->E, np, max_itr, env_dense_max());
  if (s != SBP_OK) return s;
  s = job_upload(J, g);
  if (s != SBP_OK) return s;
  SBP_CUDA(cudaMemcpyAsync(J.part, part, 4 * (size_t)J.N, cudaMemcpyHostToDevice, J.st));
  rebuild_blockmodel(J.g, J.part, B, J.m, J.rs, J.st, env_rebuild_shape());
  if (is_dense(J, B)) dense_build(J.g, J.part, B, J.m, J.st);
  return SBP_OK;
}

sbp_status check_options(const sbp_options* o) {
  if (!o) return fail(SBP_ERR_INVALID, "options are NULL");
  if (o->num_proposals < 1 || o->num_proposals > 32)
    return fail(SBP_ERR_INVALID, "num_proposals must be in [1, 32]");
  if (o->num_batches < 1 || o->max_nodal_itr < 1 || o->window < 2 || o->max_outer < 1)
    return fail(SBP_ERR_INVALID, "bad loop options");
  if (!(o->reduction_rate > 0.f && o->reduction_rate < 1.f))
    return fail(SBP_ERR_INVALID, "reduction_rate must be in (0, 1)");
  if ((o->exact != 0 && o->exact != 1) || (o->mh != 0 && o->mh != 1))
    return fail(SBP_ERR_INVALID, "exact and mh must be 0 or 1");
  if (o->mh && !(o->beta >= 0.0 && o->beta < 1e300))
    return fail(SBP_ERR_INVALID, "beta must be finite and >= 0");
  if (o->ref_grid < -1 || o->ref_grid > 1) return fail(SBP_ERR_INVALID, "ref_grid must be -1, 0 or 1");
  if (o->phase_timing != 0 && o->phase_timing != 1)
    return fail(SBP_ERR_INVALID, "phase_timing must be 0 or 1");
  return SBP_OK;
}

}  // namespace sbp

struct sbp_graph_dev {
  sbp::Job job;
  sbp_graph_csr shape;  // host arrays of an uploaded graph (null for device-built ones)
  // a graph built on the device keeps its edges there, to build the CSR
  // pair again when the job's arena has to grow
  int32_t *d_src = nullptr, *d_dst = nullptr;
  uint32_t* d_w = nullptr;
  int dev = -1;
  ~sbp_graph_dev() {
    if (d_src || d_dst || d_w) {
      int cur = 0;
      cudaGetDevice(&cur);
      cudaSetDevice(dev);
      cudaFree(d_src);
      cudaFree(d_dst);
      cudaFree(d_w);
      cudaSetDevice(cur);
    }
  }
};

namespace sbp {

// Creates the job's arena and builds its CSR pair from edges in device
// memory (csr_from_device_edges), with the host row pointers the engine
// reads.
static sbp_status job_from_device_edges(Job& J, int device, int32_t N, int32_t E,
                                        const int32_t* src, const int32_t* dst,
                                        const uint32_t* w, int32_t np, int32_t max_itr,
                                        int32_t dense_max) {
  sbp_status s = job_create(J, device, N, E, np, max_itr, dense_max);
  if (s != SBP_OK) return s;
  const size_t sb = csr_build_scratch_bytes(N, E) + 256;
  char* scratch = nullptr;
  SBP_CUDA(cudaMallocAsync((void**)&scratch, sb, J.st));
  int32_t* err = (int32_t*)(scratch + sb - 256);
  cudaError_t e = csr_from_device_edges(N, E, src, dst, w, J.g, err, scratch, J.st);
  int32_t herr = 0;
  J.h_optr.resize((size_t)N + 1);
  J.h_iptr.resize((size_t)N + 1);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, J.st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(J.h_optr.data(), J.g.optr, 4 * ((size_t)N + 1), cudaMemcpyDeviceToHost,
                        J.st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(J.h_iptr.data(), J.g.iptr, 4 * ((size_t)N + 1), cudaMemcpyDeviceToHost,
                        J.st);
  const cudaError_t f = cudaFreeAsync(scratch, J.st);
  const cudaError_t q = cudaStreamSynchronize(J.st);
  SBP_CUDA(e);
  SBP_CUDA(f);
  SBP_CUDA(q);
  if (herr & 1) return fail(SBP_ERR_INVALID, "edge endpoint out of range");
  if (herr & 2) return fail(SBP_ERR_INVALID, "edge weights must be >= 1");
  if (herr & 4) return fail(SBP_ERR_INVALID, "node degree does not fit 32 bits");
  return SBP_OK;
}

// A resident-graph handle over edges in device memory that the handle owns.
static sbp_status graph_from_owned_edges(sbp_graph_dev* h, int32_t N, int32_t E) {
  h->shape = sbp_graph_csr{};
  h->shape.N = N;
  h->shape.E = E;
  return job_from_device_edges(h->job, h->dev, N, E, h->d_src, h->d_dst, h->d_w, 10, 100, -1);
}

}  // namespace sbp

using namespace sbp;

extern "C" {

void sbp_default_options(sbp_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->seed = 0;
  o->num_proposals = 10;
  o->reduction_rate = 0.35f;
  o->max_nodal_itr = 100;
  o->num_batches = 4;
  o->threshold1 = 5e-4f;
  o->threshold2 = 1e-4f;
  o->window = 3;
  o->max_outer = 1000;
  o->device = -1;
  o->use_graphs = 1;
  o->verbose = 0;
  o->dense_max = -1;
  o->exact = 0;
  o->mh = 0;
  o->beta = 3.0;
  o->ref_grid = -1;
  o->phase_timing = 0;
}

const char* sbp_status_string(sbp_status s) {
  switch (s) {
    case SBP_OK: return "ok";
    case SBP_ERR_INVALID: return "invalid argument";
    case SBP_ERR_CUDA: return "CUDA error";
    case SBP_ERR_NOMEM: return "out of memory";
    case SBP_ERR_BUDGET: return "HBM budget exceeded";
    case SBP_ERR_TIMEOUT: return "timed out";
    case SBP_ERR_INTERNAL: return "internal error";
    case SBP_ERR_BUSY: return "busy";
    case SBP_ERR_NOT_FOUND: return "not found";
    case SBP_ERR_CANCELLED: return "cancelled";
  }
  return "unknown status";
}

const char* sbp_last_error(void) { return g_last_error.c_str(); }

sbp_status sbp_graph_upload(const sbp_graph_csr* g, int32_t device, sbp_graph_dev** out) {
  if (!out) return fail(SBP_ERR_INVALID, "out is NULL");
  *out = nullptr;
  sbp_graph_dev* h = new (std::nothrow) sbp_graph_dev();
  if (!h) return fail(SBP_ERR_NOMEM, "host allocation");
  sbp_status s = job_for(h->job, g, device, 10, 100, -1);
  if (s != SBP_OK) {
    delete h;
    return s;
  }
  h->shape = *g;
  cudaError_t e = cudaStreamSynchronize(h->job.st);
  if (e != cudaSuccess) {
    delete h;
    return fail(SBP_ERR_CUDA, cudaGetErrorString(e));
  }
  *out = h;
  return SBP_OK;
}

sbp_status sbp_graph_release(sbp_graph_dev* g) {
  delete g;
  return SBP_OK;
}

sbp_status sbp_graph_from_device_edges(int32_t N, int32_t E, const int32_t* src,
                                       const int32_t* dst, const uint32_t* w, int32_t device,
                                       sbp_graph_dev** out) {
  if (!out) return fail(SBP_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (N < 1 || E < 0) return fail(SBP_ERR_INVALID, "need N >= 1 and E >= 0");
  if (E > 0 && (!src || !dst)) return fail(SBP_ERR_INVALID, "edge arrays are NULL");
  std::unique_ptr<sbp_graph_dev> h(new (std::nothrow) sbp_graph_dev());
  if (!h) return fail(SBP_ERR_NOMEM, "host allocation");
  h->dev = resolve_device(device);
  SBP_CUDA(cudaSetDevice(h->dev));
  const size_t n = (size_t)std::max(E, 1);
  SBP_CUDA(cudaMalloc(&h->d_src, 4 * n));
  SBP_CUDA(cudaMalloc(&h->d_dst, 4 * n));
  if (w) SBP_CUDA(cudaMalloc(&h->d_w, 4 * n));
  if (E > 0) {
    SBP_CUDA(cudaMemcpy(h->d_src, src, 4 * (size_t)E, cudaMemcpyDeviceToDevice));
    SBP_CUDA(cudaMemcpy(h->d_dst, dst, 4 * (size_t)E, cudaMemcpyDeviceToDevice));
    if (w) SBP_CUDA(cudaMemcpy(h->d_w, w, 4 * (size_t)E, cudaMemcpyDeviceToDevice));
  }
  sbp_status s = graph_from_owned_edges(h.get(), N, E);
  if (s != SBP_OK) return s;
  *out = h.release();
  return SBP_OK;
}

sbp_status sbp_dcsbm_generate_device(const sbp_dcsbm_params* p, int32_t device,
                                     int32_t* truth_out, sbp_graph_dev** out) {
  if (!p || !out) return fail(SBP_ERR_INVALID, "NULL argument");
  *out = nullptr;
  std::vector<int32_t> truth;
  std::vector<double> cdf;
  sbp_status s = dcsbm_labels(p, truth, cdf);
  if (s != SBP_OK) return s;
  const long long slots = (long long)p->N * p->deg_max;
  if (slots >= (1ll << 31))
    return fail(SBP_ERR_INVALID, "N * deg_max must be below 2^31 for the device generator");
  std::unique_ptr<sbp_graph_dev> h(new (std::nothrow) sbp_graph_dev());
  if (!h) return fail(SBP_ERR_NOMEM, "host allocation");
  h->dev = resolve_device(device);
  SBP_CUDA(cudaSetDevice(h->dev));
  cudaStream_t st = nullptr;
  SBP_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  int32_t *src = nullptr, *dst = nullptr;
  int32_t E = 0;
  cudaError_t e = cudaMalloc(&src, 4 * (size_t)std::max(slots, 1ll));
  if (e == cudaSuccess) e = cudaMalloc(&dst, 4 * (size_t)std::max(slots, 1ll));
  if (e == cudaSuccess) {
    DcsbmDeviceIn in{};
    in.truth = truth.data();
    in.cdf = cdf.data();
    in.seed = p->seed;
    in.pin_scaled = (uint64_t)std::llround(p->p_in * 4294967296.0);
    in.N = p->N;
    in.B = p->B;
    in.ncdf = (int32_t)cdf.size();
    in.deg_min = p->deg_min;
    in.max_edges = slots;
    DcsbmDeviceOut o{src, dst, &E};
    e = dcsbm_device_edges(in, o, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  // the handle keeps the edges at their exact size
  if (e == cudaSuccess) e = cudaMalloc(&h->d_src, 4 * (size_t)std::max(E, 1));
  if (e == cudaSuccess) e = cudaMalloc(&h->d_dst, 4 * (size_t)std::max(E, 1));
  if (e == cudaSuccess && E > 0)
    e = cudaMemcpyAsync(h->d_src, src, 4 * (size_t)E, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess && E > 0)
    e = cudaMemcpyAsync(h->d_dst, dst, 4 * (size_t)E, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(src);
  cudaFree(dst);
  cudaStreamDestroy(st);
  SBP_CUDA(e);
  if (truth_out) std::memcpy(truth_out, truth.data(), 4 * (size_t)p->N);
  s = graph_from_owned_edges(h.get(), p->N, E);
  if (s != SBP_OK) return s;
  *out = h.release();
  return SBP_OK;
}

sbp_status sbp_graph_shape(const sbp_graph_dev* g, int32_t* N, int32_t* E) {
  if (!g) return fail(SBP_ERR_INVALID, "graph handle is NULL");
  if (N) *N = g->shape.N;
  if (E) *E = g->shape.E;
  return SBP_OK;
}

sbp_status sbp_graph_download(const sbp_graph_dev* g, int32_t* out_ptr, int32_t* out_idx,
                              uint32_t* out_w, int32_t* in_ptr, int32_t* in_idx, uint32_t* in_w,
                              uint32_t* deg_out, uint32_t* deg_in) {
  if (!g) return fail(SBP_ERR_INVALID, "graph handle is NULL");
  const Job& J = g->job;
  const size_t n1 = (size_t)J.N + 1, E = (size_t)J.E, N = (size_t)J.N;
  SBP_CUDA(cudaSetDevice(J.device));
  struct Copy {
    void* dst;
    const void* src;
    size_t bytes;
  } copies[] = {{out_ptr, J.g.optr, 4 * n1}, {out_idx, J.g.oidx, 4 * E}, {out_w, J.g.ow, 4 * E},
                {in_ptr, J.g.iptr, 4 * n1},  {in_idx, J.g.iidx, 4 * E},  {in_w, J.g.iw, 4 * E},
                {deg_out, J.g.kdo, 4 * N},   {deg_in, J.g.kdi, 4 * N}};
  for (const Copy& c : copies)
    if (c.dst && c.bytes)
      SBP_CUDA(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, J.st));
  SBP_CUDA(cudaStreamSynchronize(J.st));
  return SBP_OK;
}

sbp_status sbp_partition_resident(sbp_graph_dev* gd, const sbp_options* o, int32_t* labels_out,
                                  sbp_report* report) {
  if (!gd) return fail(SBP_ERR_INVALID, "graph handle is NULL");
  sbp_status s = check_options(o);
  if (s != SBP_OK) return s;
  Job& J = gd->job;
  const int32_t want_dense = dense_limit(gd->shape.N, gd->shape.E, o->dense_max);
  if (o->num_proposals > J.np || o->max_nodal_itr > J.max_itr || want_dense > J.dense_cap) {
    // grow the job's arena for these options; the graph is uploaded (or
    // built from its device edges) again
    int dev = J.device;
    int32_t np = std::max(o->num_proposals, J.np), mi = std::max(o->max_nodal_itr, J.max_itr);
    int32_t dm = std::max(want_dense, J.dense_cap);
    J.release();
    if (gd->d_src)
      s = job_from_device_edges(J, dev, gd->shape.N, gd->shape.E, gd->d_src, gd->d_dst, gd->d_w,
                                np, mi, dm);
    else
      s = job_for(J, &gd->shape, dev, np, mi, dm);
    if (s != SBP_OK) return s;
  }
  SBP_CUDA(cudaSetDevice(J.device));
  return run_solo(J, *o, labels_out, report);
}

sbp_status sbp_partition(const sbp_graph_csr* g, const sbp_options* o, int32_t* labels_out,
                         sbp_report* report) {
  sbp_status s = check_options(o);
  if (s != SBP_OK) return s;
  Timer t;
  Job J;
  s = job_for(J, g, o->device, o->num_proposals, o->max_nodal_itr, o->dense_max);
  if (s != SBP_OK) return s;
  SBP_CUDA(cudaStreamSynchronize(J.st));
  double up = t.ms();
  s = run_solo(J, *o, labels_out, report);
  if (report) {
    report->ms_h2d = up;
    report->ms_total += up;
  }
  return s;
}

sbp_status sbp_build_blockmodel(const sbp_graph_csr* g, const int32_t* part, int32_t B,
                                int32_t* out_ptr, int32_t* out_col, uint32_t* out_cnt,
                                int32_t* in_ptr, int32_t* in_col, uint32_t* in_cnt,
                                uint32_t* d_out, uint32_t* d_in, int64_t* nnz) {
  Job J;
  sbp_status s = prepare(J, g, part, B, 1, 1);
  if (s != SBP_OK) return s;
  int32_t n = 0;
  SBP_CUDA(cudaMemcpyAsync(&n, J.m.optr + B, 4, cudaMemcpyDeviceToHost, J.st));
  SBP_CUDA(cudaStreamSynchronize(J.st));
  SBP_CUDA(cudaGetLastError());
  size_t b1 = (size_t)B + 1;
  if (out_ptr) SBP_CUDA(cudaMemcpy(out_ptr, J.m.optr, 4 * b1, cudaMemcpyDeviceToHost));
  if (in_ptr) SBP_CUDA(cudaMemcpy(in_ptr, J.m.iptr, 4 * b1, cudaMemcpyDeviceToHost));
  if (n > 0) {
    if (out_col) SBP_CUDA(cudaMemcpy(out_col, J.m.ocol, 4 * (size_t)n, cudaMemcpyDeviceToHost));
    if (out_cnt) SBP_CUDA(cudaMemcpy(out_cnt, J.m.ocnt, 4 * (size_t)n, cudaMemcpyDeviceToHost));
    if (in_col) SBP_CUDA(cudaMemcpy(in_col, J.m.icol, 4 * (size_t)n, cudaMemcpyDeviceToHost));
    if (in_cnt) SBP_CUDA(cudaMemcpy(in_cnt, J.m.icnt, 4 * (size_t)n, cudaMemcpyDeviceToHost));
  }
  if (d_out) SBP_CUDA(cudaMemcpy(d_out, J.m.d_out, 4 * (size_t)B, cudaMemcpyDeviceToHost));
  if (d_in) SBP_CUDA(cudaMemcpy(d_in, J.m.d_in, 4 * (size_t)B, cudaMemcpyDeviceToHost));
  if (nnz) *nnz = n;
  return SBP_OK;
}

sbp_status sbp_delta_mdl_nodal(const sbp_graph_csr* g, const int32_t* part, int32_t B, int32_t nv,
                               const int32_t* verts, const int32_t* props, double* dS) {
  return sbp_delta_mdl_nodal_mode(g, part, B, nv, verts, props, 0, dS, nullptr);
}

sbp_status sbp_delta_mdl_nodal_mode(const sbp_graph_csr* g, const int32_t* part, int32_t B,
                                    int32_t nv, const int32_t* verts, const int32_t* props,
                                    int32_t exact, double* dS, double* logH) {
  if (!g) return fail(SBP_ERR_INVALID, "graph is NULL");
  if (exact != 0 && exact != 1) return fail(SBP_ERR_INVALID, "exact must be 0 or 1");
  if (nv < 0 || (nv > 0 && (!verts || !props || !dS)))
    return fail(SBP_ERR_INVALID, "bad vertex/proposal arrays");
  for (int32_t i = 0; i < nv; ++i) {
    if (verts[i] < 0 || verts[i] >= g->N) return fail(SBP_ERR_INVALID, "vertex out of range");
    if (props[i] < 0 || props[i] >= B) return fail(SBP_ERR_INVALID, "proposal out of [0, B)");
  }
  Job J;
  sbp_status s = prepare(J, g, part, B, 1, 1);
  if (s != SBP_OK) return s;
  int32_t *dv = nullptr, *dp = nullptr;
  double *dd = nullptr, *dl = nullptr;
  size_t n = (size_t)(nv > 0 ? nv : 1);
  SBP_CUDA(cudaMalloc(&dv, 4 * n));
  SBP_CUDA(cudaMalloc(&dp, 4 * n));
  SBP_CUDA(cudaMalloc(&dd, 8 * n));
  if (logH) SBP_CUDA(cudaMalloc(&dl, 8 * n));
  ScoreMode md;
  md.exact = exact;
  md.mh = logH ? 1 : 0;
  cudaMemcpyAsync(dv, verts, 4 * (size_t)nv, cudaMemcpyHostToDevice, J.st);
  cudaMemcpyAsync(dp, props, 4 * (size_t)nv, cudaMemcpyHostToDevice, J.st);
  std::vector<int32_t> lists;
  int32_t ln[3];
  classify_batch(J, verts, 0, nv, lists, ln);
  if (!lists.empty())
    cudaMemcpyAsync(J.lists, lists.data(), 4 * lists.size(), cudaMemcpyHostToDevice, J.st);
  block_terms_any(J, B, 0, 0, 0, J.st);
  nodal_delta_given(J.g, J.part, J.m, B, is_dense(J, B), nv, dv, dp, dd,
                    nodal_lists(J, J.lists, ln), J.st, md, dl);
  cudaStreamSynchronize(J.st);
  int32_t err_h = 0;
  cudaMemcpy(&err_h, J.err, 4, cudaMemcpyDeviceToHost);
  cudaMemcpyAsync(dS, dd, 8 * (size_t)nv, cudaMemcpyDeviceToHost, J.st);
  if (logH) cudaMemcpyAsync(logH, dl, 8 * (size_t)nv, cudaMemcpyDeviceToHost, J.st);
  cudaError_t e = cudaStreamSynchronize(J.st);
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaFree(dv);
  cudaFree(dp);
  cudaFree(dd);
  if (dl) cudaFree(dl);
  if (e != cudaSuccess) return fail(SBP_ERR_CUDA, cudaGetErrorString(e));
  if (err_h) return fail(SBP_ERR_INTERNAL, "neighbour-block table overflow in the nodal kernel");
  return SBP_OK;
}

sbp_status sbp_delta_mdl_merge(const sbp_graph_csr* g, const int32_t* part, int32_t B, int32_t np,
                               const int32_t* props, double* dS, int32_t* best, double* best_dS) {
  return sbp_delta_mdl_merge_mode(g, part, B, np, props, 0, dS, best, best_dS);
}

sbp_status sbp_delta_mdl_merge_mode(const sbp_graph_csr* g, const int32_t* part, int32_t B,
                                    int32_t np, const int32_t* props, int32_t exact, double* dS,
                                    int32_t* best, double* best_dS) {
  if (np < 1 || np > 32 || !props || B < 1) return fail(SBP_ERR_INVALID, "bad proposals");
  if (exact != 0 && exact != 1) return fail(SBP_ERR_INVALID, "exact must be 0 or 1");
  for (int64_t t = 0; t < (int64_t)B * np; ++t)
    if (props[t] < 0 || props[t] >= B) return fail(SBP_ERR_INVALID, "proposal out of [0, B)");
  Job J;
  sbp_status s = prepare(J, g, part, B, np, 1);
  if (s != SBP_OK) return s;
  size_t nt = (size_t)B * np;
  SBP_CUDA(cudaMemcpyAsync(J.props, props, 4 * nt, cudaMemcpyHostToDevice, J.st));
  block_terms(J.m, B, 0, 0, 0, J.st);
  merge_delta(J.m, B, J.E, np, J.props, J.mdS, J.best, J.best_dS, J.st, exact);
  SBP_CUDA(cudaStreamSynchronize(J.st));
  SBP_CUDA(cudaGetLastError());
  if (dS) SBP_CUDA(cudaMemcpy(dS, J.mdS, 8 * nt, cudaMemcpyDeviceToHost));
  if (best) SBP_CUDA(cudaMemcpy(best, J.best, 4 * (size_t)B, cudaMemcpyDeviceToHost));
  if (best_dS) SBP_CUDA(cudaMemcpy(best_dS, J.best_dS, 8 * (size_t)B, cudaMemcpyDeviceToHost));
  return SBP_OK;
}

sbp_status sbp_merge_proposals(const sbp_graph_csr* g, const int32_t* part, int32_t B, int32_t np,
                               uint64_t seed, uint32_t seq, int32_t* props) {
  if (np < 1 || np > 32 || !props) return fail(SBP_ERR_INVALID, "bad proposal buffer");
  Job J;
  sbp_status s = prepare(J, g, part, B, np, 1);
  if (s != SBP_OK) return s;
  merge_proposals(J.m, B, np, seed, seq, J.props, J.st);
  SBP_CUDA(cudaStreamSynchronize(J.st));
  SBP_CUDA(cudaGetLastError());
  SBP_CUDA(cudaMemcpy(props, J.props, 4 * (size_t)B * np, cudaMemcpyDeviceToHost));
  return SBP_OK;
}

sbp_status sbp_nodal_batch(const sbp_graph_csr* g, int32_t* part, int32_t B, uint64_t seed,
                           uint32_t seq, int32_t lo, int32_t hi, double* dS_rec, int32_t* props,
                           double* sum) {
  return sbp_nodal_batch_mode(g, part, B, seed, seq, lo, hi, 0, 0, 3.0, dS_rec, props, sum);
}

sbp_status sbp_nodal_batch_mode(const sbp_graph_csr* g, int32_t* part, int32_t B, uint64_t seed,
                                uint32_t seq, int32_t lo, int32_t hi, int32_t exact, int32_t mh,
                                double beta, double* dS_rec, int32_t* props, double* sum) {
  if (!g || lo < 0 || hi < lo || hi > g->N) return fail(SBP_ERR_INVALID, "bad batch range");
  if ((exact != 0 && exact != 1) || (mh != 0 && mh != 1) || !(beta >= 0.0 && beta < 1e300))
    return fail(SBP_ERR_INVALID, "bad scoring mode");
  ScoreMode md;
  md.exact = exact;
  md.mh = mh;
  md.beta = beta;
  Job J;
  sbp_status s = prepare(J, g, part, B, 1, 1);
  if (s != SBP_OK) return s;
  int32_t cnt = hi - lo;
  std::vector<int32_t> lists;
  int32_t ln[3];
  classify_batch(J, nullptr, lo, cnt, lists, ln);
  if (!lists.empty())
    SBP_CUDA(cudaMemcpyAsync(J.lists, lists.data(), 4 * lists.size(), cudaMemcpyHostToDevice,
                             J.st));
  const bool dense = is_dense(J, B);
  block_terms_any(J, B, 1, seed, seq, J.st);
  SBP_CUDA(cudaMemsetAsync(J.dsum, 0, 8, J.st));
  SBP_CUDA(cudaMemsetAsync(J.acc, 0, 8, J.st));
  nodal_batch_sample(J.g, J.part, J.m, B, dense, seed, seq, lo, cnt, J.newlab, J.rec, J.props,
                     nodal_lists(J, J.lists, ln), J.st, md);
  nodal_commit(J.part, lo, cnt, J.newlab, J.rec, J.dsum, J.acc, nullptr, 0, J.cs, J.st);
  SBP_CUDA(cudaStreamSynchronize(J.st));
  SBP_CUDA(cudaGetLastError());
  SBP_CUDA(cudaMemcpy(part, J.part, 4 * (size_t)J.N, cudaMemcpyDeviceToHost));
  if (dS_rec && cnt) SBP_CUDA(cudaMemcpy(dS_rec, J.rec, 8 * (size_t)cnt, cudaMemcpyDeviceToHost));
  if (props && cnt) SBP_CUDA(cudaMemcpy(props, J.props, 4 * (size_t)cnt, cudaMemcpyDeviceToHost));
  if (sum) SBP_CUDA(cudaMemcpy(sum, J.dsum, 8, cudaMemcpyDeviceToHost));
  return SBP_OK;
}

sbp_status sbp_nodal_sweeps(const sbp_graph_csr* g, int32_t* part, int32_t B, uint64_t seed,
                            uint32_t seq0, int32_t num_batches, int32_t sweeps, int32_t dense_max,
                            double* sums) {
  if (!g || num_batches < 1 || sweeps < 1 || !sums) return fail(SBP_ERR_INVALID, "bad arguments");
  sbp_status s = validate_graph(g);
  if (s != SBP_OK) return s;
  s = validate_part(part, g->N, B);
  if (s != SBP_OK) return s;
  const int32_t nb = num_batches * sweeps;
  Job J;
  s = job_create(J, resolve_device(-1), g->N, g->E, 1, nb, dense_max);
  if (s != SBP_OK) return s;
  s = job_upload(J, g);
  if (s != SBP_OK) return s;
  SBP_CUDA(cudaMemcpyAsync(J.part, part, 4 * (size_t)J.N, cudaMemcpyHostToDevice, J.st));
  SBP_CUDA(cudaStreamSynchronize(J.st));
  s = run_sweeps(J, B, seed, seq0, num_batches, sweeps, sums);
  if (s != SBP_OK) return s;
  SBP_CUDA(cudaMemcpy(part, J.part, 4 * (size_t)J.N, cudaMemcpyDeviceToHost));
  return SBP_OK;
}

sbp_status sbp_apply_merges(int32_t B, int32_t B_to_merge, const int32_t* best,
                            const double* best_dS, int32_t* map, int32_t* B_new) {
  if (B < 1 || B_to_merge < 0 || !best || !best_dS || !map || !B_new)
    return fail(SBP_ERR_INVALID, "bad merge arguments");
  const int32_t nb = apply_merges_host(B, B_to_merge, best, best_dS, map);
  if (nb < 0) return fail(SBP_ERR_INVALID, "merge target out of [0, B)");
  *B_new = nb;
  return SBP_OK;
}

sbp_status sbp_apply_merges_device(int32_t B, int32_t B_to_merge, const int32_t* best,
                                   const double* best_dS, int32_t device, int32_t* map,
                                   int32_t* B_new) {
  if (B < 1 || B_to_merge < 0 || !best || !best_dS || !map || !B_new)
    return fail(SBP_ERR_INVALID, "bad merge arguments");
  const int dev = resolve_device(device);
  SBP_CUDA(cudaSetDevice(dev));
  const size_t ws = merge_apply_bytes(B);
  const size_t need = ws + 256 * 5 + (size_t)B * (4 + 8 + 4) + 8;
  char* mem = nullptr;
  cudaStream_t st = nullptr;
  SBP_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  if (cudaMalloc(&mem, need) != cudaSuccess) {
    cudaGetLastError();
    cudaStreamDestroy(st);
    return fail(SBP_ERR_NOMEM, "device buffers of the merge application");
  }
  Arena A{mem, need, 0};
  MergeApplyBufs w = merge_apply_carve(A.take<char>(ws), B);
  int32_t* d_best = A.take<int32_t>(B);
  double* d_bds = A.take<double>(B);
  int32_t* d_map = A.take<int32_t>(B);
  int32_t* d_out = A.take<int32_t>(2);
  int32_t out[2] = {0, 0};
  cudaError_t e = cudaMemcpyAsync(d_best, best, 4 * (size_t)B, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_bds, best_dS, 8 * (size_t)B, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_out, 0, 8, st);
  if (e == cudaSuccess) {
    merge_apply(w, B, B_to_merge, d_best, d_bds, d_map, d_out, st);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(map, d_map, 4 * (size_t)B, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(mem);
  cudaStreamDestroy(st);
  if (e != cudaSuccess) return fail(SBP_ERR_CUDA, cudaGetErrorString(e));
  if (out[1]) return fail(SBP_ERR_INVALID, "merge target out of [0, B)");
  *B_new = out[0];
  return SBP_OK;
}

sbp_status sbp_merge_step(const sbp_graph_csr* g, int32_t* part, int32_t B, int32_t B_to_merge,
                          int32_t np, uint64_t seed, uint32_t seq, int32_t* best, double* best_dS,
                          int32_t* B_new) {
  return sbp_merge_step_mode(g, part, B, B_to_merge, np, seed, seq, 0, best, best_dS, B_new);
}

sbp_status sbp_merge_step_mode(const sbp_graph_csr* g, int32_t* part, int32_t B,
                               int32_t B_to_merge, int32_t np, uint64_t seed, uint32_t seq,
                               int32_t ref_grid, int32_t* best, double* best_dS, int32_t* B_new) {
  if (np < 1 || np > 32) return fail(SBP_ERR_INVALID, "bad np");
  if (ref_grid != 0 && ref_grid != 1) return fail(SBP_ERR_INVALID, "ref_grid must be 0 or 1");
  Job J;
  sbp_status s = prepare(J, g, part, B, np, 1);
  if (s != SBP_OK) return s;
  int32_t b = B;
  s = merge_step(J, b, B_to_merge, seed, seq, false, ref_grid);
  if (s != SBP_OK) return s;
  SBP_CUDA(cudaStreamSynchronize(J.st));
  if (best) std::memcpy(best, J.h_best, 4 * (size_t)B);
  if (best_dS) std::memcpy(best_dS, J.h_best_dS, 8 * (size_t)B);
  SBP_CUDA(cudaMemcpy(part, J.part, 4 * (size_t)J.N, cudaMemcpyDeviceToHost));
  if (B_new) *B_new = b;
  return SBP_OK;
}

sbp_status sbp_mdl(const sbp_graph_csr* g, const int32_t* part, int32_t B, double* S,
                   double* data_S) {
  return sbp_mdl_mode(g, part, B, 0, S, data_S);
}

sbp_status sbp_mdl_mode(const sbp_graph_csr* g, const int32_t* part, int32_t B, int32_t exact,
                        double* S, double* data_S) {
  if (exact != 0 && exact != 1) return fail(SBP_ERR_INVALID, "exact must be 0 or 1");
  Job J;
  sbp_status s = prepare(J, g, part, B, 1, 1);
  if (s != SBP_OK) return s;
  block_terms(J.m, B, 0, 0, 0, J.st);
  mdl_data_sum(J.m, B, J.dataS, J.st);
  double ds = 0.0;
  SBP_CUDA(cudaMemcpyAsync(&ds, J.dataS, 8, cudaMemcpyDeviceToHost, J.st));
  SBP_CUDA(cudaStreamSynchronize(J.st));
  SBP_CUDA(cudaGetLastError());
  if (data_S) *data_S = ds;
  if (S) *S = model_S(B, g->N, g->E, exact) - ds;
  return SBP_OK;
}

}  // extern "C"
