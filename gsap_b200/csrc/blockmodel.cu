// Blockmodel rebuild, per-block terms and the MDL sum.
//
// GSAP rebuilds M after every merge step and every nodal batch with
// thrust::sort_by_key over vertices, four thrust scans, a scatter of
// neighbour blocks, bb_segsort over block segments, six memsets, two
// remove_if compactions with a host read-back and mgpu::segreduce
// (calculate_new_csr, partition.hpp:707-849; about 30 launches and ten hidden
// allocations or synchronisations per call).  Here it is seven launches
// with no host round trip, both directions (out rows / in rows) in each:
//
//   count    per vertex: entries of its row segment, slot inside the segment
//   scan     segment offsets
//   scatter  per graph entry: (neighbour block, weight) into its segment
//   rows     per segment: sort by column and sum runs; a warp per short
//            segment (bitonic sort in shared memory), a CTA per long one
//            (shared-memory histogram when B fits, else bitonic sort, else a
//            windowed histogram)
//   scan     compacted row pointers
//   compact  per row: copy the unique (column, count) pairs into place, the
//            row sum (weighted block degree) and its log2
//
// The result is exact integer work and identical to the oracle's builder.
#include "common.cuh"
#include "kernels.h"
#include "multi.cuh"
#include "dense.cuh"

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

namespace sbp {

thread_local long long g_launches = 0;

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 2048

// Exclusive scan across the CTA (any blockDim multiple of 32 up to 1024).
// `sh` needs 33 ints.  Returns the exclusive prefix; *total gets the sum.
__device__ __forceinline__ int cta_excl_scan(int x, int* sh, int* total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) sh[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int v = lane < nw ? sh[lane] : 0;
    int vi = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(kFull, vi, o);
      if (lane >= o) vi += y;
    }
    if (lane < nw) sh[lane] = vi - v;
    if (lane == 31) sh[32] = vi;
  }
  __syncthreads();
  int res = incl - x + sh[wid];
  *total = sh[32];
  __syncthreads();
  return res;
}

// Scan of one array in three steps when it spans more than one CTA's tiles:
// per-tile sums, a one-CTA scan of those sums, then each tile applies its
// offset.  Short arrays take the one-CTA scan directly.
struct ScanArgs {
  const int32_t* in;
  int32_t* out;
  int32_t* tile;  // tile sums (tile body), offsets (apply body)
  const int32_t* ctl;
  int32_t n, pad;
};

struct ScanTileBody {
  using Args = ScanArgs;
  static constexpr int kThreads = kScanThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int) {
    if (ctl_stopped(a.ctl)) return;
    __shared__ int sh[33];
    int base = vb * kScanTile + threadIdx.x * kScanItems;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
      if (base + k < a.n) s += a.in[base + k];
    int tot;
    cta_excl_scan(s, sh, &tot);
    if (threadIdx.x == 0) a.tile[vb] = tot;
  }
};

// Exclusive scan of `n` values (in place allowed), one CTA, tile by tile with
// a carry; out[n] = total.
struct ScanSingleBody {
  using Args = ScanArgs;
  static constexpr int kThreads = kScanThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int, int) {
    if (ctl_stopped(a.ctl)) return;
    __shared__ int sh[33];
    int carry = 0;
    for (int t0 = 0; t0 < a.n; t0 += kScanTile) {
      int base = t0 + threadIdx.x * kScanItems;
      int v[kScanItems];
      int s = 0;
#pragma unroll
      for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < a.n ? a.in[base + k] : 0;
        s += v[k];
      }
      int tot;
      int pre = cta_excl_scan(s, sh, &tot) + carry;
#pragma unroll
      for (int k = 0; k < kScanItems; ++k) {
        if (base + k < a.n) a.out[base + k] = pre;
        pre += v[k];
      }
      carry += tot;
    }
    if (threadIdx.x == 0) a.out[a.n] = carry;
  }
};

struct ScanApplyBody {
  using Args = ScanArgs;
  static constexpr int kThreads = kScanThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    if (ctl_stopped(a.ctl)) return;
    __shared__ int sh[33];
    int base = vb * kScanTile + threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      v[k] = base + k < a.n ? a.in[base + k] : 0;
      s += v[k];
    }
    int tot;
    int pre = cta_excl_scan(s, sh, &tot) + a.tile[vb];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      if (base + k < a.n) a.out[base + k] = pre;
      pre += v[k];
    }
    if (vb == vg - 1 && threadIdx.x == blockDim.x - 1) a.out[a.n] = pre;
  }
};

constexpr int kScanSingleMax = 8 * kScanTile;

// ------------------------------------------------------------ rebuild ------
struct RbSide {
  const int32_t* gptr;
  const int32_t* gidx;
  const uint32_t* gw;
  const int32_t* gsrc;
  int32_t* cnt;
  int32_t* seg;
  int32_t* vofs;
  int32_t* tcol;
  uint32_t* tw;
  int32_t* ucol;  // unique (column, count) pairs of each segment, at its offset
  uint32_t* uw;
  int32_t* uniq;
  int32_t* big;
  int32_t* big_count;
  int32_t* bptr;
  int32_t* bcol;
  uint32_t* bcnt;
  uint32_t* bdeg;
  double* bld;
};

struct RbArgs {
  RbSide s[2];
  const int32_t* part;
  const int32_t* ctl;
  int32_t N, E, B;
  int32_t warp_cap;  // longest segment a warp reduces; longer ones go to a CTA
};

// The rebuild bodies work on both directions: virtual block vb serves
// direction vb & 1 with the direction's own virtual block vb >> 1.

// Per vertex: its entries form one run inside its block's segment.
struct RbCountBody {
  using Args = RbArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int) {
  if (ctl_stopped(a.ctl)) return;
  const RbSide& d = a.s[vb & 1];
  int v = (vb >> 1) * blockDim.x + threadIdx.x;
  const bool live = v < a.N;
  const unsigned active = __ballot_sync(kFull, live);
  if (!live) return;
  int b = a.part[v];
  int len = d.gptr[v + 1] - d.gptr[v];
  // warp-aggregated: lanes with the same block reserve one range together
  unsigned peers = __match_any_sync(active, b);
  int lane = threadIdx.x & 31;
  int leader = __ffs(peers) - 1;
  int pre = 0, tot = 0;
  for (unsigned m = peers; m; m &= m - 1) {
    int j = __ffs(m) - 1;
    int x = __shfl_sync(peers, len, j);
    tot += x;
    if (j < lane) pre += x;
  }
  int base = 0;
  if (lane == leader) base = atomicAdd(d.cnt + b, tot);
  base = __shfl_sync(peers, base, leader);
  d.vofs[v] = base + pre;
  }
};

// Per graph entry: (block of the neighbour, weight) into the owner's run.
struct RbScatterBody {
  using Args = RbArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int) {
    if (ctl_stopped(a.ctl)) return;
    const RbSide& d = a.s[vb & 1];
    int j = (vb >> 1) * blockDim.x + threadIdx.x;
    if (j >= a.E) return;
    int v = __ldg(d.gsrc + j);
    int b = __ldg(a.part + v);
    int pos = __ldg(d.seg + b) + __ldg(d.vofs + v) + (j - __ldg(d.gptr + v));
    d.tcol[pos] = __ldg(a.part + __ldg(d.gidx + j));
    d.tw[pos] = __ldg(d.gw + j);
  }
};

constexpr int kWarpCap = 256;  // longest segment sorted by one warp
constexpr int kRowsWarps = 8;

__device__ __forceinline__ void warp_bitonic(unsigned long long* key, int P, int lane) {
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < P; i += 32) {
        int ixj = i ^ j;
        if (ixj > i) {
          unsigned long long x = key[i], y = key[ixj];
          bool asc = (i & k) == 0;
          if ((x > y) == asc) {
            key[i] = y;
            key[ixj] = x;
          }
        }
      }
      __syncwarp();
    }
  }
}

// Short segments: one warp each.  Long ones are listed for rb_rows_big.
struct RbRowsSmallBody {
  using Args = RbArgs;
  static constexpr int kThreads = kRowsWarps * 32, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
  if (ctl_stopped(a.ctl)) return;
  __shared__ unsigned long long sk[kRowsWarps][kWarpCap];
  const RbSide& d = a.s[vb & 1];
  vb >>= 1;
  vg >>= 1;
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned long long* key = sk[wid];
  for (int b = vb * kRowsWarps + wid; b < a.B; b += vg * kRowsWarps) {
    int base = d.seg[b];
    int n = d.seg[b + 1] - base;
    if (n > a.warp_cap) {
      if (lane == 0) d.big[atomicAdd(d.big_count, 1)] = b;
      continue;
    }
    if (n == 0) {
      if (lane == 0) d.uniq[b] = 0;
      continue;
    }
    if (n <= 32) {
      // one entry per lane: lanes with equal columns group and sum in
      // registers; each group's leader writes at its column's rank among
      // the distinct columns (ascending order, as a sort would give)
      const bool valid = lane < n;
      const uint32_t c = valid ? (uint32_t)d.tcol[base + lane] : 0xffffffffu;
      const uint32_t w = valid ? d.tw[base + lane] : 0u;
      const unsigned peers = __match_any_sync(kFull, c);
      const uint32_t sum = __reduce_add_sync(peers, w);
      const bool leader = valid && __ffs(peers) - 1 == lane;
      const unsigned leaders = __ballot_sync(kFull, leader);
      int rank = 0;
      for (unsigned m = leaders; m; m &= m - 1) {
        const uint32_t cj = __shfl_sync(kFull, c, __ffs(m) - 1);
        rank += cj < c ? 1 : 0;
      }
      if (leader) {
        d.ucol[base + rank] = (int32_t)c;
        d.uw[base + rank] = sum;
      }
      if (lane == 0) d.uniq[b] = __popc(leaders);
      continue;
    }
    int P = 32;
    while (P < n) P <<= 1;
    for (int i = lane; i < P; i += 32)
      key[i] = i < n ? ((unsigned long long)(uint32_t)d.tcol[base + i] << 32) | d.tw[base + i]
                     : ~0ull;
    __syncwarp();
    warp_bitonic(key, P, lane);
    int running = 0;
    for (int i0 = 0; i0 < n; i0 += 32) {
      int i = i0 + lane;
      bool valid = i < n;
      uint32_t c = valid ? (uint32_t)(key[i] >> 32) : 0u;
      bool head = valid && (i == 0 || (uint32_t)(key[i - 1] >> 32) != c);
      unsigned mask = __ballot_sync(kFull, head);
      if (head) {
        int pos = running + __popc(mask & ((1u << lane) - 1));
        uint32_t s = 0;
        for (int j = i; j < n && (uint32_t)(key[j] >> 32) == c; ++j) s += (uint32_t)key[j];
        d.ucol[base + pos] = (int32_t)c;
        d.uw[base + pos] = s;
      }
      running += __popc(mask);
    }
    if (lane == 0) d.uniq[b] = running;
    __syncwarp();
  }
  }
};

constexpr int kBigThreads = 512;
constexpr int kHistCap = 16384;  // columns counted in shared memory at once
constexpr int kSortCap = 8192;   // longest segment sorted in shared memory
constexpr int kMaxWindows = 256; // column windows a long segment is bucketed into
constexpr size_t kBigSmem = 65536;

struct RbRowsBigBody {
  using Args = RbArgs;
  static constexpr int kThreads = kBigThreads, kMinBlocks = 2;
  static constexpr size_t kSmem = kBigSmem;
  static __device__ void run(const Args& a, int vb, int vg) {
  if (ctl_stopped(a.ctl)) return;
  extern __shared__ unsigned long long big_sm[];
  __shared__ int sh[33];
  __shared__ uint32_t touched[kHistCap / 32];  // bitmap of the histogram's nonzero columns
  __shared__ int wstart[kMaxWindows + 1];      // a long segment's entries by column window
  const RbSide& d = a.s[vb & 1];
  vb >>= 1;
  vg >>= 1;
  uint32_t* hist = (uint32_t*)big_sm;
  int nbig = *d.big_count;
  int T = blockDim.x, tid = threadIdx.x;
  const int nwords = (a.B + 31) >> 5;
  if (a.B <= kHistCap && vb < nbig) {
    // every row fits one histogram: it and the bitmap start zero and each
    // row's extraction clears what the row touched
    for (int i = tid; i < a.B; i += T) hist[i] = 0u;
    for (int i = tid; i < nwords; i += T) touched[i] = 0u;
    __syncthreads();
  }
  for (int idx = vb; idx < nbig; idx += vg) {
    int b = d.big[idx];
    int base = d.seg[b];
    int n = d.seg[b + 1] - base;
    int running = 0;
    if (a.B <= kHistCap) {
      // histogram of the row plus a bitmap of its columns; the extraction
      // walks B/32 bitmap words, not B bins, so a row costs O(n + B/32)
      for (int i = tid; i < n; i += T) {
        const int c = d.tcol[base + i];
        atomicAdd(hist + c, d.tw[base + i]);
        atomicOr(touched + (c >> 5), 1u << (c & 31));
      }
      __syncthreads();
      const int per = (nwords + T - 1) / T;
      const int x0 = min(nwords, tid * per), x1 = min(nwords, x0 + per);
      int nz = 0;
      for (int x = x0; x < x1; ++x) nz += __popc(touched[x]);
      int tot;
      int pos = cta_excl_scan(nz, sh, &tot);
      for (int x = x0; x < x1; ++x) {
        uint32_t m = touched[x];
        touched[x] = 0u;
        while (m) {
          const int c = (x << 5) + __ffs(m) - 1;
          m &= m - 1;
          d.ucol[base + pos] = c;
          d.uw[base + pos] = hist[c];
          hist[c] = 0u;
          ++pos;
        }
      }
      running = tot;
      __syncthreads();
    } else if (n > kSortCap && (a.B + kHistCap - 1) / kHistCap <= kMaxWindows) {
      // Long segment, many columns: bucket the entries by column window of
      // kHistCap (a counting sort into the segment's own output range), then
      // one histogram pass per window over that window's entries only, with
      // the touched-column bitmap.  Window w's results start at or before
      // its bucket (every result consumes an entry of an earlier or the
      // same window) and end at or before the next bucket, and are written
      // after the window's entries are read: the range serves as both.
      const int W = (a.B + kHistCap - 1) / kHistCap;
      uint32_t* cursor = hist;  // W counters, before the histogram use
      for (int i = tid; i < W; i += T) cursor[i] = 0u;
      __syncthreads();
      for (int i = tid; i < n; i += T) atomicAdd(cursor + d.tcol[base + i] / kHistCap, 1u);
      __syncthreads();
      if (tid == 0) {
        int acc = 0;
        for (int w = 0; w < W; ++w) {
          wstart[w] = acc;
          acc += (int)cursor[w];
          cursor[w] = (uint32_t)wstart[w];
        }
        wstart[W] = acc;
      }
      __syncthreads();
      for (int i = tid; i < n; i += T) {
        const int c = d.tcol[base + i];
        const int at = (int)atomicAdd(cursor + c / kHistCap, 1u);
        d.ucol[base + at] = c;
        d.uw[base + at] = d.tw[base + i];
      }
      __syncthreads();
      for (int i = tid; i < kHistCap; i += T) hist[i] = 0u;
      for (int i = tid; i < kHistCap / 32; i += T) touched[i] = 0u;
      __syncthreads();
      for (int w = 0; w < W; ++w) {
        const int w0 = w * kHistCap, e0 = wstart[w], e1 = wstart[w + 1];
        const int nwords_w = (min(kHistCap, a.B - w0) + 31) >> 5;
        for (int i = e0 + tid; i < e1; i += T) {
          const int c = d.ucol[base + i] - w0;
          atomicAdd(hist + c, d.uw[base + i]);
          atomicOr(touched + (c >> 5), 1u << (c & 31));
        }
        __syncthreads();
        const int per = (nwords_w + T - 1) / T;
        const int x0 = min(nwords_w, tid * per), x1 = min(nwords_w, x0 + per);
        int nz = 0;
        for (int x = x0; x < x1; ++x) nz += __popc(touched[x]);
        int tot;
        int pos = cta_excl_scan(nz, sh, &tot) + running;
        for (int x = x0; x < x1; ++x) {
          uint32_t m = touched[x];
          touched[x] = 0u;
          while (m) {
            const int c = (x << 5) + __ffs(m) - 1;
            m &= m - 1;
            d.ucol[base + pos] = w0 + c;
            d.uw[base + pos] = hist[c];
            hist[c] = 0u;
            ++pos;
          }
        }
        running += tot;
        __syncthreads();
      }
    } else if (n > kSortCap) {
      // histogram over column windows of kHistCap
      for (int w0 = 0; w0 < a.B; w0 += kHistCap) {
        int W = min(kHistCap, a.B - w0);
        for (int i = tid; i < W; i += T) hist[i] = 0u;
        __syncthreads();
        for (int i = tid; i < n; i += T) {
          int c = d.tcol[base + i] - w0;
          if (c >= 0 && c < W) atomicAdd(hist + c, d.tw[base + i]);
        }
        __syncthreads();
        int per = (W + T - 1) / T;
        int c0 = min(W, tid * per), c1 = min(W, c0 + per);
        int nz = 0;
        for (int c = c0; c < c1; ++c) nz += hist[c] != 0u;
        int tot;
        int pos = cta_excl_scan(nz, sh, &tot) + running;
        for (int c = c0; c < c1; ++c) {
          uint32_t h = hist[c];
          if (h) {
            d.ucol[base + pos] = w0 + c;
            d.uw[base + pos] = h;
            ++pos;
          }
        }
        running += tot;
        __syncthreads();
      }
    } else {
      // bitonic sort of (column, weight) keys
      unsigned long long* key = big_sm;
      int P = 32;
      while (P < n) P <<= 1;
      for (int i = tid; i < P; i += T)
        key[i] = i < n ? ((unsigned long long)(uint32_t)d.tcol[base + i] << 32) | d.tw[base + i]
                       : ~0ull;
      __syncthreads();
      for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
          for (int i = tid; i < P; i += T) {
            int ixj = i ^ j;
            if (ixj > i) {
              unsigned long long x = key[i], y = key[ixj];
              bool asc = (i & k) == 0;
              if ((x > y) == asc) {
                key[i] = y;
                key[ixj] = x;
              }
            }
          }
          __syncthreads();
        }
      }
      for (int i0 = 0; i0 < n; i0 += T) {
        int i = i0 + tid;
        bool valid = i < n;
        uint32_t c = valid ? (uint32_t)(key[i] >> 32) : 0u;
        bool head = valid && (i == 0 || (uint32_t)(key[i - 1] >> 32) != c);
        int tot;
        int pos = cta_excl_scan(head ? 1 : 0, sh, &tot) + running;
        if (head) {
          uint32_t s = 0;
          for (int j = i; j < n && (uint32_t)(key[j] >> 32) == c; ++j) s += (uint32_t)key[j];
          d.ucol[base + pos] = (int32_t)c;
          d.uw[base + pos] = s;
        }
        running += tot;
      }
      __syncthreads();
    }
    if (tid == 0) d.uniq[b] = running;
    __syncthreads();
  }
  }
};

// Per row: unique entries into place, weighted degree and its log2.
struct RbCompactBody {
  using Args = RbArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
  if (ctl_stopped(a.ctl)) return;
  const RbSide& d = a.s[vb & 1];
  vb >>= 1;
  vg >>= 1;
  int lane = threadIdx.x & 31;
  int w = (vb * blockDim.x + threadIdx.x) >> 5;
  int nw = (vg * blockDim.x) >> 5;
  for (int b = w; b < a.B; b += nw) {
    int src = d.seg[b], dst = d.bptr[b], u = d.uniq[b];
    unsigned long long s = 0;
    for (int i = lane; i < u; i += 32) {
      uint32_t c = d.uw[src + i];
      d.bcol[dst + i] = d.ucol[src + i];
      d.bcnt[dst + i] = c;
      s += c;
    }
    s = warp_sum_ull(s);
    if (lane == 0) {
      uint32_t deg = (uint32_t)s;
      d.bdeg[b] = deg;
      d.bld[b] = log2((double)deg);
    }
  }
  }
};

// ------------------------------------------------------------ block terms --
struct BtArgs {
  const double* xlx;
  const int32_t *optr, *ocol, *iptr, *icol;
  const uint32_t *ocnt, *icnt, *d_out, *d_in;
  const double *ld_out, *ld_in;
  double *dSout, *ambout, *ambin, *sinfull;
  int32_t* nbr_s;
  uint8_t* use_rand;
  const int32_t* ctl;  // sweep control: gate, and seq += ctl[0] * seq_mul
  int32_t B;
  int draws;
  uint64_t seed;
  uint32_t seq, seq_mul;
};

// One cell's share of a row sum, x log2 x - x * ld, with one rounding order
// (a fused multiply-add) wherever the per-block sums are formed, so the CSR
// and the dense form give the same bits.
__device__ __forceinline__ double cell_term(const double* tab, uint32_t m, double ld) {
  return __fma_rn(-(double)m, ld, xlx(tab, m));
}

// Row sum minus its degree term; d == 0 leaves the sum (log2 0 = -inf).
__device__ __forceinline__ double row_total(double s, uint32_t d, double ld) {
  return d ? __dsub_rn(s, __dmul_rn((double)d, ld)) : s;
}

// First entry k of out-row ++ in-row of block b whose running count exceeds
// t; the whole warp returns the column (or -1).
__device__ int warp_pick_row(const BtArgs& a, int b, uint64_t t, int lane) {
  int o0 = a.optr[b], no = a.optr[b + 1] - o0;
  int i0 = a.iptr[b], ni = a.iptr[b + 1] - i0;
  int n = no + ni;
  uint64_t acc = 0;
  for (int k0 = 0; k0 < n; k0 += 32) {
    int k = k0 + lane;
    uint64_t w = 0;
    int col = -1;
    if (k < n) {
      if (k < no) { w = a.ocnt[o0 + k]; col = a.ocol[o0 + k]; }
      else { w = a.icnt[i0 + k - no]; col = a.icol[i0 + k - no]; }
    }
    uint64_t incl = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    unsigned hit = __ballot_sync(kFull, k < n && acc + incl > t);
    if (hit) return __shfl_sync(kFull, col, __ffs(hit) - 1);
    acc += __shfl_sync(kFull, incl, 31);
  }
  return -1;
}

struct BlockTermsBody {
  using Args = BtArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
  if (ctl_stopped(a.ctl)) return;
  const uint32_t seq = a.seq + ctl_itr(a.ctl) * a.seq_mul;
  int lane = threadIdx.x & 31;
  int w = (vb * blockDim.x + threadIdx.x) >> 5;
  int nw = (vg * blockDim.x) >> 5;
  for (int b = w; b < a.B; b += nw) {
    if (a.draws != 1) {
    double acc = 0.0;
    // the row's k-th nonzero is added by lane k % 32, in order of k
    // (unrolled so that several entries' loads are in flight at once)
#pragma unroll 4
    for (int i = a.optr[b] + lane; i < a.optr[b + 1]; i += 32)
      acc += cell_term(a.xlx, a.ocnt[i], a.ld_in[a.ocol[i]]);
    double ao = warp_sum(acc);
    acc = 0.0;
#pragma unroll 4
    for (int i = a.iptr[b] + lane; i < a.iptr[b + 1]; i += 32)
      acc += cell_term(a.xlx, a.icnt[i], a.ld_out[a.icol[i]]);
    double ai = warp_sum(acc);
    if (lane == 0) {
      a.ambout[b] = ao;
      a.dSout[b] = row_total(ao, a.d_out[b], a.ld_out[b]);
      a.ambin[b] = ai;
      a.sinfull[b] = row_total(ai, a.d_in[b], a.ld_in[b]);
    }
    }
    if (a.draws) {
      P4 x = draw(a.seed, kRngNodalBlock, seq, (uint32_t)b);
      uint64_t deg = (uint64_t)a.d_out[b] + a.d_in[b];
      int nb = 0;
      if (deg > 0) {
        int c = warp_pick_row(a, b, scale_draw(x.v[1], deg), lane);
        nb = c >= 0 ? c : 0;
      }
      if (lane == 0) {
        a.use_rand[b] = accept_random(x.v[0], deg, (uint64_t)a.B) ? 1 : 0;
        a.nbr_s[b] = nb;
      }
    }
  }
  }
};


// ------------------------------------------------------------ dense form --
// For small B the blockmodel is kept as two B x B count matrices (rows and
// columns of M both contiguous).  Built once per merge step / golden-section
// restore; after each nodal batch only the edges of the moved vertices are
// applied, with integer atomics (exact, order-independent).

struct DenseArgs {
  const int32_t *osrc, *optr, *oidx, *iptr, *iidx;
  const uint32_t *ow, *iw, *kdo, *kdi;
  const int32_t* part;
  const int32_t* newlab;  // update: new labels of vertices lo..lo+count-1
  uint32_t *Md, *MTd, *Sd, *d_out, *d_in;
  double *ld_out, *ld_in;
  const int32_t* ctl;
  int32_t N, E, B, lo, count, pad;
};

// Chunk sums of a dense cell (r, c): out-row r's chunk of column c and
// in-row c's chunk of row r (DevBM::Sd).
__device__ __forceinline__ uint32_t* sd_out(uint32_t* Sd, int K, int r, int c) {
  return Sd + (size_t)r * 2 * K + (c >> 5);
}
__device__ __forceinline__ uint32_t* sd_in(uint32_t* Sd, int K, int r, int c) {
  return Sd + (size_t)c * 2 * K + K + (r >> 5);
}

// Build step 1: every edge adds its weight to M[r][c] (and the transpose).
struct DenseEdgesBody {
  using Args = DenseArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int) {
    int j = vb * blockDim.x + threadIdx.x;
    if (j >= a.E) return;
    int r = __ldg(a.part + __ldg(a.osrc + j)), c = __ldg(a.part + __ldg(a.oidx + j));
    uint32_t w = __ldg(a.ow + j);
    const int K = (a.B + 31) >> 5;
    atomicAdd(a.Md + (size_t)r * a.B + c, w);
    atomicAdd(a.MTd + (size_t)c * a.B + r, w);
    atomicAdd(sd_out(a.Sd, K, r, c), w);
    atomicAdd(sd_in(a.Sd, K, r, c), w);
  }
};

// Build step 2: block degrees from vertex degrees.
struct DenseDegreesBody {
  using Args = DenseArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int) {
    int v = vb * blockDim.x + threadIdx.x;
    if (v >= a.N) return;
    int b = a.part[v];
    atomicAdd(a.d_out + b, a.kdo[v]);
    atomicAdd(a.d_in + b, a.kdi[v]);
  }
};

// Build step 1 after a merge step: the dense form of the merged labels from
// the CSR blockmodel of the labels before it (rebuilt for the merge) and the
// merge map: entry (r, c, count) adds count at (map[r], map[c]).  The same
// integer sums as adding every edge (the counts are the edges' weight sums),
// from nnz entries instead of E edges; a warp per old block row.
struct DenseMapArgs {
  const int32_t *bop, *boc;
  const uint32_t* bon;
  const int32_t* map;
  uint32_t *Md, *MTd, *Sd;
  int32_t B_old, B;
};

struct DenseFromCsrBody {
  using Args = DenseMapArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    const int lane = threadIdx.x & 31;
    const int K = (a.B + 31) >> 5;
    for (int r = (vb * kThreads + threadIdx.x) >> 5; r < a.B_old; r += (vg * kThreads) >> 5) {
      const int R = a.map[r];
      for (int i = a.bop[r] + lane; i < a.bop[r + 1]; i += 32) {
        const int C = a.map[a.boc[i]];
        const uint32_t w = a.bon[i];
        atomicAdd(a.Md + (size_t)R * a.B + C, w);
        atomicAdd(a.MTd + (size_t)C * a.B + R, w);
        atomicAdd(sd_out(a.Sd, K, R, C), w);
        atomicAdd(sd_in(a.Sd, K, R, C), w);
      }
    }
  }
};

// The CSR blockmodel from a dense form that holds the current labels' M (a
// merge step after sweeps that left the labels as they were): a warp per
// row of M (the out CSR) and of M^T (the in CSR) counts the row's nonzero
// cells, and after the scan writes them in column order with their counts:
// the arrays the rebuild from the edges builds.  Degrees and their log2 are
// the dense form's own.
struct DenseCsrArgs {
  const uint32_t *Md, *MTd;
  int32_t *cnt_o, *cnt_i;  // per row: nonzero cells (the scan's input)
  const int32_t *optr, *iptr;
  int32_t *ocol, *icol;
  uint32_t *ocnt, *icnt;
  int32_t B, fill;  // fill 0: count, 1: write the rows
};

struct DenseCsrBody {
  using Args = DenseCsrArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int B = a.B;
    for (int t = (vb * kThreads + threadIdx.x) >> 5; t < 2 * B; t += (vg * kThreads) >> 5) {
      const bool in = t >= B;
      const int b = in ? t - B : t;
      const uint32_t* row = (in ? a.MTd : a.Md) + (size_t)b * B;
      int k = 0;
      int32_t* col = nullptr;
      uint32_t* cnt = nullptr;
      if (a.fill) {
        k = (in ? a.iptr : a.optr)[b];
        col = in ? a.icol : a.ocol;
        cnt = in ? a.icnt : a.ocnt;
      }
      int n = 0;
      for (int c0 = 0; c0 < B; c0 += 32) {
        const int c = c0 + lane;
        const uint32_t m = c < B ? row[c] : 0u;
        const unsigned nz = __ballot_sync(kFull, m != 0u);
        if (a.fill && m) {
          const int pos = k + n + __popc(nz & lt);
          col[pos] = c;
          cnt[pos] = m;
        }
        n += __popc(nz);
      }
      if (!a.fill && lane == 0) (in ? a.cnt_i : a.cnt_o)[b] = n;
    }
  }
};

// Build step 3: log2 of the block degrees.
struct DenseLogsBody {
  using Args = DenseArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int) {
    int b = vb * blockDim.x + threadIdx.x;
    if (b >= a.B) return;
    a.ld_out[b] = log2((double)a.d_out[b]);
    a.ld_in[b] = log2((double)a.d_in[b]);
  }
};

// The moved vertices of a batch: its out-edges move from (r, old block of
// w) to (s, new block of w); its in-edges from unmoved sources move from
// (b(u), r) to (b(u), s).  Edges between two moved vertices are handled
// once, from the source's out-edges.  A lane per batch vertex finds the
// moved ones (about a tenth of a batch once the first sweeps are done);
// the warp then applies each moved vertex's entries together, lane-strided.
// A warp covers kDuVerts batch vertices, so that the moved ones (a few per
// warp at most) are spread over many warps: their dependent loads are the
// latency of the launch.
constexpr int kDuVerts = 8;
struct DenseUpdateBody {
  using Args = DenseArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
  if (ctl_stopped(a.ctl)) return;
  const int32_t* __restrict__ optr = a.optr;
  const int32_t* __restrict__ oidx = a.oidx;
  const uint32_t* __restrict__ ow = a.ow;
  const int32_t* __restrict__ iptr = a.iptr;
  const int32_t* __restrict__ iidx = a.iidx;
  const uint32_t* __restrict__ iw = a.iw;
  const uint32_t* __restrict__ kdo = a.kdo;
  const uint32_t* __restrict__ kdi = a.kdi;
  const int32_t* __restrict__ part = a.part;
  const int32_t* __restrict__ newlab = a.newlab;
  const int32_t lo = a.lo, count = a.count, B = a.B;
  uint32_t *Md = a.Md, *MTd = a.MTd, *Sd = a.Sd, *d_out = a.d_out, *d_in = a.d_in;
  const int K = (B + 31) >> 5;
  const int lane = threadIdx.x & 31;
  const int nw = (vg * kThreads) >> 5;
  for (int w0 = ((vb * kThreads + threadIdx.x) >> 5) * kDuVerts; w0 < count;
       w0 += nw * kDuVerts) {
    const int i = w0 + lane;
    int32_t r0 = 0, s0 = 0;
    if (lane < kDuVerts && i < count) {
      r0 = part[lo + i];
      s0 = newlab[i];
    }
    unsigned moved = __ballot_sync(kFull, lane < kDuVerts && i < count && r0 != s0);
    while (moved) {
      const int src = __ffs(moved) - 1;
      moved &= moved - 1;
      const int v = lo + w0 + src;
      const int r = __shfl_sync(kFull, r0, src), s = __shfl_sync(kFull, s0, src);
      if (lane == 0) {
        atomicSub(d_out + r, kdo[v]);
        atomicAdd(d_out + s, kdo[v]);
        atomicSub(d_in + r, kdi[v]);
        atomicAdd(d_in + s, kdi[v]);
      }
      for (int j = optr[v] + lane; j < optr[v + 1]; j += 32) {
        const int x = __ldg(oidx + j);
        const uint32_t wt = __ldg(ow + j);
        const int bo = __ldg(part + x);
        const int bn = (x >= lo && x < lo + count) ? newlab[x - lo] : bo;
        atomicSub(Md + (size_t)r * B + bo, wt);
        atomicSub(MTd + (size_t)bo * B + r, wt);
        atomicAdd(Md + (size_t)s * B + bn, wt);
        atomicAdd(MTd + (size_t)bn * B + s, wt);
        atomicSub(sd_out(Sd, K, r, bo), wt);
        atomicSub(sd_in(Sd, K, r, bo), wt);
        atomicAdd(sd_out(Sd, K, s, bn), wt);
        atomicAdd(sd_in(Sd, K, s, bn), wt);
      }
      for (int j = iptr[v] + lane; j < iptr[v + 1]; j += 32) {
        const int u = __ldg(iidx + j);
        const int bu = __ldg(part + u);
        if (u >= lo && u < lo + count && newlab[u - lo] != bu) continue;  // moved source
        const uint32_t wt = __ldg(iw + j);
        atomicSub(Md + (size_t)bu * B + r, wt);
        atomicSub(MTd + (size_t)r * B + bu, wt);
        atomicAdd(Md + (size_t)bu * B + s, wt);
        atomicAdd(MTd + (size_t)s * B + bu, wt);
        atomicSub(sd_out(Sd, K, bu, r), wt);
        atomicSub(sd_in(Sd, K, bu, r), wt);
        atomicAdd(sd_out(Sd, K, bu, s), wt);
        atomicAdd(sd_in(Sd, K, bu, s), wt);
      }
    }
  }
  }
};

// Sum of cell_term over a dense row with the CSR loop's order: each chunk of
// 32 columns hands its nonzeros, by their rank in the row, to lanes
// (rank % 32) through a 32-slot shared buffer of the warp, so every lane adds
// the same terms in the same order as over the row's CSR entries.
// Four chunks at a time: their counts, degrees and cell terms are loaded and
// computed first (independent loads in flight together), then handed out
// chunk by chunk in the same order as one chunk at a time.
__device__ __forceinline__ double dense_row_sum(const double* tab, const uint32_t* row,
                                                const double* ld, int B, int lane,
                                                double* buf) {
  constexpr int U = 4;
  double acc = 0.0;
  int k = 0;  // nonzeros before this chunk
  const unsigned lt = (1u << lane) - 1u;
  for (int c0 = 0; c0 < B; c0 += 32 * U) {
    uint32_t m[U];
    double t[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int c = c0 + 32 * u + lane;
      m[u] = c < B ? row[c] : 0u;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int c = c0 + 32 * u + lane;
      t[u] = m[u] ? cell_term(tab, m[u], ld[c]) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const unsigned nz = __ballot_sync(kFull, m[u] != 0u);
      if (nz == 0u) continue;
      const int n = __popc(nz);
      if (m[u]) buf[(k + __popc(nz & lt)) & 31] = t[u];
      __syncwarp();
      if (((lane - k) & 31) < n) acc += buf[lane];
      __syncwarp();
      k += n;
    }
  }
  return acc;
}

struct BtDenseArgs {
  const double* xlx;
  const uint32_t *Md, *MTd, *Sd, *d_out, *d_in;
  const double *ld_out, *ld_in;
  double *dSout, *ambout, *ambin, *sinfull;
  int32_t* nbr_s;
  uint8_t* use_rand;
  const int32_t* ctl;  // sweep control: gate, and seq += ctl[0] * seq_mul
  int32_t B;
  int draws;
  uint64_t seed;
  uint32_t seq, seq_mul;
};

struct BlockTermsDenseBody {
  using Args = BtDenseArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
  if (ctl_stopped(a.ctl)) return;
  __shared__ double tbuf[kThreads / 32][32];
  const uint32_t seq = a.seq + ctl_itr(a.ctl) * a.seq_mul;
  int lane = threadIdx.x & 31;
  int w = (vb * blockDim.x + threadIdx.x) >> 5;
  int nw = (vg * blockDim.x) >> 5;
  const int B = a.B;
  for (int b = w; b < B; b += nw) {
    const uint32_t* orow = a.Md + (size_t)b * B;
    const uint32_t* irow = a.MTd + (size_t)b * B;
    if (a.draws != 1) {
    double* buf = tbuf[threadIdx.x >> 5];
    double ao = warp_sum(dense_row_sum(a.xlx, orow, a.ld_in, B, lane, buf));
    double ai = warp_sum(dense_row_sum(a.xlx, irow, a.ld_out, B, lane, buf));
    if (lane == 0) {
      a.ambout[b] = ao;
      a.dSout[b] = row_total(ao, a.d_out[b], a.ld_out[b]);
      a.ambin[b] = ai;
      a.sinfull[b] = row_total(ai, a.d_in[b], a.ld_in[b]);
    }
    }
    if (a.draws)
      dense_block_draw(a.Md, a.MTd, a.Sd, a.d_out, a.d_in, B, a.seed, seq, b, lane, a.nbr_s,
                       a.use_rand);
  }
  }
};

__global__ void fill_xlx_kernel(double* tab) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x < kXlxTable) {
    tab[x] = xlog2x(x);
    tab[kXlxTable + x] = log2((double)x);
  }
}

struct MdlArgs {
  const double* dSout;
  double* out;  // written at out[ctl[0]] under sweep control
  const int32_t* ctl;
  int32_t B, pad;
};

// data_S = sum of dSout over the blocks, one CTA per job, fixed order.
struct MdlSumBody {
  using Args = MdlArgs;
  static constexpr int kThreads = 512, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int, int) {
    if (ctl_stopped(a.ctl)) return;
    __shared__ double sh[kThreads];
    double s = 0.0;
    for (int b = threadIdx.x; b < a.B; b += kThreads) s += a.dSout[b];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) a.out[ctl_itr(a.ctl)] = sh[0];
  }
};

// The stop test of a queued sweep (partition.hpp:920-934), one thread per
// job, after the sweep's MDL: ctl[0] = sweeps done so far including this
// one; ctl[1] = 1 once the moving-average dS test or the sweep limit ends
// the outer step.  The arithmetic is the host's, operation for operation.
struct SweepCtlArgs {
  int32_t* ctl;
  const double* dsum;   // per sweep of the outer step
  const double* dataS;  // per sweep of the outer step
  double model_S;       // E(1+x)ln(1+x) - x ln x + N ln B of the step's B
  double thr;           // threshold1 or threshold2 by the bracket's state
  int32_t window;       // 0: no stop test (a fixed number of sweeps)
  int32_t max_itr;
};

struct SweepCtlBody {
  using Args = SweepCtlArgs;
  static constexpr int kThreads = 32, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int, int) {
    if (threadIdx.x != 0 || a.ctl[1] != 0) return;
    const int itr = a.ctl[0];
    bool stop = false;
    if (a.window > 0 && itr >= a.window - 1) {
      double mean = 0.0;
      for (int i = itr - a.window + 1; i < itr; ++i) mean += a.dsum[i];
      mean /= (double)(a.window - 1);
      const double S = a.model_S - a.dataS[itr];
      stop = -mean < a.thr * S;
    }
    a.ctl[0] = itr + 1;
    if (stop || itr + 1 >= a.max_itr) a.ctl[1] = 1;
  }
};

// Small utility bodies of the multi-job engine.
struct WordsArgs {
  uint32_t* dst;
  const uint32_t* src;  // copy source (copy body)
  long long n;          // 32-bit words
  const int32_t* ctl;
};

struct ZeroBody {
  using Args = WordsArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    if (ctl_stopped(a.ctl)) return;
    for (long long i = (long long)vb * kThreads + threadIdx.x; i < a.n;
         i += (long long)vg * kThreads)
      a.dst[i] = 0u;
  }
};

struct CopyBody {
  using Args = WordsArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    if (ctl_stopped(a.ctl)) return;
    for (long long i = (long long)vb * kThreads + threadIdx.x; i < a.n;
         i += (long long)vg * kThreads)
      a.dst[i] = a.src[i];
  }
};

struct IotaBody {
  using Args = WordsArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    if (ctl_stopped(a.ctl)) return;
    for (long long i = (long long)vb * kThreads + threadIdx.x; i < a.n;
         i += (long long)vg * kThreads)
      a.dst[i] = (uint32_t)i;
  }
};

int grid_for(long long items, int per_block, int cap) {
  long long g = (items + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

RbArgs rb_args(const DevGraph& g, const int32_t* part, int32_t B, DevBM& m, RebuildScratch& rs,
               const RebuildTune& t) {
  RbArgs a{};
  a.warp_cap = std::max(32, std::min(kWarpCap, t.warp_cap));
  a.part = part;
  a.N = g.N;
  a.E = g.E;
  a.B = B;
  for (int dir = 0; dir < 2; ++dir) {
    RbSide& s = a.s[dir];
    const RebuildDir& r = rs.d[dir];
    s.gptr = dir == 0 ? g.optr : g.iptr;
    s.gidx = dir == 0 ? g.oidx : g.iidx;
    s.gw = dir == 0 ? g.ow : g.iw;
    s.gsrc = dir == 0 ? g.osrc : g.isrc;
    s.cnt = r.cnt;
    s.seg = r.seg;
    s.vofs = r.vofs;
    s.tcol = r.tcol;
    s.tw = r.tw;
    s.ucol = r.ucol;
    s.uw = r.uw;
    s.uniq = r.uniq;
    s.big = r.big;
    s.big_count = rs.big_count + dir;
    s.bptr = dir == 0 ? m.optr : m.iptr;
    s.bcol = dir == 0 ? m.ocol : m.icol;
    s.bcnt = dir == 0 ? m.ocnt : m.icnt;
    s.bdeg = dir == 0 ? m.d_out : m.d_in;
    s.bld = dir == 0 ? m.ld_out : m.ld_in;
  }
  return a;
}

// Virtual grids: functions of one job's sizes only.
int32_t vg_count(const RbArgs& a) { return 2 * ceil_div(a.N, 256); }
int32_t vg_scatter(const RbArgs& a) { return a.E > 0 ? 2 * ceil_div(a.E, 256) : 0; }
int32_t vg_rows_small(const RbArgs& a) { return 2 * grid_for(a.B, kRowsWarps, 4096); }
int32_t vg_rows_big(const RbArgs& a, const RebuildTune& t) {
  const int32_t per = ceil_div(std::max(a.E, 1), std::max(256, t.big_entries));
  return 2 * std::max(1, std::min(t.big_ctas > 0 ? t.big_ctas : 2 * 148, per));
}
int32_t vg_compact(const RbArgs& a) { return 2 * grid_for((long long)a.B * 32, 256, 4096); }
int32_t vg_words(long long n) {
  return n <= 0 ? 0 : (int32_t)std::min<long long>(4096, (n + 2047) / 2048);
}

BtArgs bt_args(DevBM& m, int32_t B, int draws, uint64_t seed, uint32_t seq) {
  BtArgs a{};
  a.xlx = m.xlx;
  a.optr = m.optr; a.ocol = m.ocol; a.iptr = m.iptr; a.icol = m.icol;
  a.ocnt = m.ocnt; a.icnt = m.icnt; a.d_out = m.d_out; a.d_in = m.d_in;
  a.ld_out = m.ld_out; a.ld_in = m.ld_in;
  a.dSout = m.dSout; a.ambout = m.ambout; a.ambin = m.ambin; a.sinfull = m.sinfull;
  a.nbr_s = m.nbr_s; a.use_rand = m.use_rand;
  a.B = B; a.draws = draws; a.seed = seed; a.seq = seq;
  return a;
}

BtDenseArgs bt_dense_args(DevBM& m, int32_t B, int draws, uint64_t seed, uint32_t seq) {
  BtDenseArgs a{};
  a.xlx = m.xlx;
  a.Md = m.Md; a.MTd = m.MTd; a.Sd = m.Sd; a.d_out = m.d_out; a.d_in = m.d_in;
  a.ld_out = m.ld_out; a.ld_in = m.ld_in;
  a.dSout = m.dSout; a.ambout = m.ambout; a.ambin = m.ambin; a.sinfull = m.sinfull;
  a.nbr_s = m.nbr_s; a.use_rand = m.use_rand;
  a.B = B; a.draws = draws; a.seed = seed; a.seq = seq;
  return a;
}

DenseArgs dense_args(const DevGraph& g, const int32_t* part, int32_t B, DevBM& m) {
  DenseArgs a{};
  a.osrc = g.osrc; a.optr = g.optr; a.oidx = g.oidx; a.iptr = g.iptr; a.iidx = g.iidx;
  a.ow = g.ow; a.iw = g.iw; a.kdo = g.kdo; a.kdi = g.kdi;
  a.part = part;
  a.Md = m.Md; a.MTd = m.MTd; a.Sd = m.Sd; a.d_out = m.d_out; a.d_in = m.d_in;
  a.ld_out = m.ld_out; a.ld_in = m.ld_in;
  a.N = g.N; a.E = g.E; a.B = B;
  return a;
}

int32_t vg_block_terms(int32_t B) { return grid_for((long long)B * 32, 256, 8192); }
int32_t vg_dense_update(int32_t count) {
  return grid_for((long long)count, 256 / 32 * kDuVerts, 148 * 16);
}

const MultiKernel kmScanTile = multi_kernel_desc<ScanTileBody>("scan_tile");
const MultiKernel kmScanSingle = multi_kernel_desc<ScanSingleBody>("scan_single");
const MultiKernel kmScanApply = multi_kernel_desc<ScanApplyBody>("scan_apply");
const MultiKernel kmRbCount = multi_kernel_desc<RbCountBody>("rb_count");
const MultiKernel kmRbScatter = multi_kernel_desc<RbScatterBody>("rb_scatter");
const MultiKernel kmRbRowsSmall = multi_kernel_desc<RbRowsSmallBody>("rb_rows_small");
const MultiKernel kmRbRowsBig = multi_kernel_desc<RbRowsBigBody>("rb_rows_big");
const MultiKernel kmRbCompact = multi_kernel_desc<RbCompactBody>("rb_compact");
const MultiKernel kmBlockTerms = multi_kernel_desc<BlockTermsBody>("block_terms");
const MultiKernel kmBlockTermsDense = multi_kernel_desc<BlockTermsDenseBody>("block_terms_dense");
const MultiKernel kmDenseEdges = multi_kernel_desc<DenseEdgesBody>("dense_edges");
const MultiKernel kmDenseFromCsr = multi_kernel_desc<DenseFromCsrBody>("dense_from_csr");
const MultiKernel kmDenseCsr = multi_kernel_desc<DenseCsrBody>("dense_csr");
const MultiKernel kmDenseDegrees = multi_kernel_desc<DenseDegreesBody>("dense_degrees");
const MultiKernel kmDenseLogs = multi_kernel_desc<DenseLogsBody>("dense_logs");
const MultiKernel kmDenseUpdate = multi_kernel_desc<DenseUpdateBody>("dense_update");
const MultiKernel kmMdlSum = multi_kernel_desc<MdlSumBody>("mdl_sum");
const MultiKernel kmSweepCtl = multi_kernel_desc<SweepCtlBody>("sweep_ctl");
const MultiKernel kmZero = multi_kernel_desc<ZeroBody>("zero");
const MultiKernel kmCopy = multi_kernel_desc<CopyBody>("copy");
const MultiKernel kmIota = multi_kernel_desc<IotaBody>("iota");

// One job's scan records: short arrays in one CTA, longer ones in three steps.
void add_scan(Slot* sl, const int32_t* in, int32_t* out, int32_t n, int32_t* tile,
              const int32_t* ctl) {
  ScanArgs a{};
  a.ctl = ctl;
  if (n <= kScanSingleMax) {
    a.in = in;
    a.out = out;
    a.n = n;
    slot_push(slot_bind(sl[1], kmScanSingle), a, 1);
    return;
  }
  const int32_t tiles = ceil_div(n, kScanTile);
  a.in = in;
  a.out = out;
  a.tile = tile;
  a.n = n;
  slot_push(slot_bind(sl[0], kmScanTile), a, tiles);
  ScanArgs b{};
  b.in = tile;
  b.out = tile + tiles;
  b.n = tiles;
  b.ctl = ctl;
  slot_push(slot_bind(sl[1], kmScanSingle), b, 1);
  a.tile = tile + tiles;
  slot_push(slot_bind(sl[2], kmScanApply), a, tiles);
}

}  // namespace

void add_exclusive_scan(Slot* sl, const int32_t* in, int32_t* out, int32_t n, int32_t* tile) {
  add_scan(sl, in, out, n, tile, nullptr);
}

cudaError_t init_kernel_attributes() {
  cudaError_t e = cudaFuncSetAttribute(single_kernel<RbRowsBigBody>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kBigSmem);
  cudaError_t e2 = cudaFuncSetAttribute(multi_kernel<RbRowsBigBody>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kBigSmem);
  return e != cudaSuccess ? e : e2;
}

void scan_exclusive(const int32_t* in, int32_t* out, int32_t n, int32_t* tile, cudaStream_t st) {
  ScanArgs a{};
  a.in = in;
  a.out = out;
  a.n = n;
  if (n <= kScanSingleMax) {
    launch_single<ScanSingleBody>(a, 1, st);
    return;
  }
  int tiles = ceil_div(n, kScanTile);
  a.tile = tile;
  launch_single<ScanTileBody>(a, tiles, st);
  ScanArgs b{};
  b.in = tile;
  b.out = tile + tiles;
  b.n = tiles;
  launch_single<ScanSingleBody>(b, 1, st);
  a.tile = tile + tiles;
  launch_single<ScanApplyBody>(a, tiles, st);
}

void rebuild_blockmodel(const DevGraph& g, const int32_t* part, int32_t B, DevBM& m,
                        RebuildScratch& rs, cudaStream_t st, const RebuildTune& t) {
  RbArgs a = rb_args(g, part, B, m, rs, t);
  for (int dir = 0; dir < 2; ++dir)
    cudaMemsetAsync(rs.d[dir].cnt, 0, sizeof(int32_t) * (size_t)B, st);
  cudaMemsetAsync(rs.big_count, 0, sizeof(int32_t) * 2, st);
  launch_single<RbCountBody>(a, vg_count(a), st);
  for (int dir = 0; dir < 2; ++dir)
    scan_exclusive(rs.d[dir].cnt, rs.d[dir].seg, B, rs.tile + dir * (rs.tile_cap / 2), st);
  launch_single<RbScatterBody>(a, vg_scatter(a), st);
  launch_single<RbRowsSmallBody>(a, vg_rows_small(a), st);
  launch_single<RbRowsBigBody>(a, vg_rows_big(a, t), st);
  for (int dir = 0; dir < 2; ++dir)
    scan_exclusive(rs.d[dir].uniq, dir == 0 ? m.optr : m.iptr, B,
                   rs.tile + dir * (rs.tile_cap / 2), st);
  launch_single<RbCompactBody>(a, vg_compact(a), st);
}

void block_terms(DevBM& m, int32_t B, int draws, uint64_t seed, uint32_t seq, cudaStream_t st) {
  launch_single<BlockTermsBody>(bt_args(m, B, draws, seed, seq), vg_block_terms(B), st);
}

void fill_xlx_table(double* tab, cudaStream_t st) {
  ++g_launches;
  fill_xlx_kernel<<<kXlxTable / 256, 256, 0, st>>>(tab);
}

void dense_build(const DevGraph& g, const int32_t* part, int32_t B, DevBM& m, cudaStream_t st) {
  size_t bb = (size_t)B * B;
  cudaMemsetAsync(m.Md, 0, bb * sizeof(uint32_t), st);
  cudaMemsetAsync(m.MTd, 0, bb * sizeof(uint32_t), st);
  cudaMemsetAsync(m.Sd, 0, (size_t)2 * B * ((B + 31) / 32) * sizeof(uint32_t), st);
  cudaMemsetAsync(m.d_out, 0, (size_t)B * sizeof(uint32_t), st);
  cudaMemsetAsync(m.d_in, 0, (size_t)B * sizeof(uint32_t), st);
  DenseArgs a = dense_args(g, part, B, m);
  if (g.E > 0) launch_single<DenseEdgesBody>(a, ceil_div(g.E, 256), st);
  launch_single<DenseDegreesBody>(a, ceil_div(g.N, 256), st);
  launch_single<DenseLogsBody>(a, ceil_div(B, 256), st);
}

void dense_update(const DevGraph& g, const int32_t* part, int32_t lo, int32_t count,
                  const int32_t* newlab, int32_t B, DevBM& m, cudaStream_t st) {
  if (count <= 0) return;
  DenseArgs a = dense_args(g, part, B, m);
  a.lo = lo;
  a.count = count;
  a.newlab = newlab;
  launch_single<DenseUpdateBody>(a, vg_dense_update(count), st);
}

void block_terms_dense(DevBM& m, int32_t B, int draws, uint64_t seed, uint32_t seq,
                       cudaStream_t st) {
  launch_single<BlockTermsDenseBody>(bt_dense_args(m, B, draws, seed, seq), vg_block_terms(B),
                                     st);
}

void mdl_data_sum(const DevBM& m, int32_t B, double* out, cudaStream_t st) {
  MdlArgs a{m.dSout, out, nullptr, B, 0};
  launch_single<MdlSumBody>(a, 1, st);
}

// -------------------------------------------------------------- autotuner --
// The rebuild's segment width (the longest segment one warp reduces; longer
// ones go to a CTA) and the CTA grid for the long segments are picked by
// timing rebuilds of a job's own blockmodel, once per device and size class
// (log2 of B and of the mean segment length E/B).  Every candidate builds
// the same matrix, so the choice changes only the time.
namespace {
struct TuneKey {
  int device, lb, ls;
  bool operator<(const TuneKey& o) const {
    return device != o.device ? device < o.device : lb != o.lb ? lb < o.lb : ls < o.ls;
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, RebuildTune> g_tune;

int ilog2(long long x) {
  int l = 0;
  while (x > 1) {
    x >>= 1;
    ++l;
  }
  return l;
}

TuneKey tune_key(int device, int32_t E, int32_t B) {
  return TuneKey{device, ilog2(std::max(B, 1)), ilog2(std::max<long long>(1, (long long)E / std::max(B, 1)))};
}
}  // namespace

bool rebuild_tuned(int device, int32_t E, int32_t B, RebuildTune* out) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(tune_key(device, E, B));
  if (it == g_tune.end()) return false;
  *out = it->second;
  return true;
}

cudaError_t tune_rebuild(int device, const DevGraph& g, const int32_t* part, int32_t B, DevBM& m,
                         RebuildScratch& rs, cudaStream_t st, RebuildTune* out) {
  std::vector<RebuildTune> cands;
  for (int wc : {32, 64, 128, 256})
    for (int be : {2048, 512}) cands.push_back(RebuildTune{wc, 0, be});
  cudaEvent_t e0, e1;
  cudaError_t err = cudaEventCreate(&e0);
  if (err != cudaSuccess) return err;
  err = cudaEventCreate(&e1);
  if (err != cudaSuccess) {
    cudaEventDestroy(e0);
    return err;
  }
  RebuildTune best = RebuildTune{};
  float best_ms = 1e30f;
  for (const RebuildTune& c : cands) {
    rebuild_blockmodel(g, part, B, m, rs, st, c);  // warm
    float ms = 0.f;
    cudaEventRecord(e0, st);
    for (int r = 0; r < 2; ++r) rebuild_blockmodel(g, part, B, m, rs, st, c);
    cudaEventRecord(e1, st);
    err = cudaEventSynchronize(e1);
    if (err != cudaSuccess) break;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return err;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[tune_key(device, g.E, B)] = best;
  *out = best;
  return cudaSuccess;
}

// ------------------------------------------------------ multi-job records --
void RebuildSlots::clear() {
  for (Slot* x : all()) x->clear();
}

std::vector<Slot*> RebuildSlots::all() {
  return {&zero,     &count,     &scan1[0],   &scan1[1], &scan1[2], &scatter,
          &rows_small, &rows_big, &dense_count, &scan2[0], &scan2[1], &scan2[2], &compact,
          &dense_fill};
}

void add_csr_from_dense(RebuildSlots& s, int32_t B, DevBM& m, RebuildScratch& rs) {
  DenseCsrArgs a{m.Md, m.MTd, rs.d[0].uniq, rs.d[1].uniq, m.optr, m.iptr,
                 m.ocol, m.icol, m.ocnt, m.icnt, B, 0};
  const int32_t vg = grid_for((long long)2 * B * 32, 256, 148 * 16);
  slot_push(slot_bind(s.dense_count, kmDenseCsr), a, vg);
  for (int dir = 0; dir < 2; ++dir)
    add_scan(s.scan2, rs.d[dir].uniq, dir == 0 ? m.optr : m.iptr, B,
             rs.tile + dir * (rs.tile_cap / 2), nullptr);
  a.fill = 1;
  slot_push(slot_bind(s.dense_fill, kmDenseCsr), a, vg);
}

void add_rebuild(RebuildSlots& s, const DevGraph& g, const int32_t* part, int32_t B, DevBM& m,
                 RebuildScratch& rs, const int32_t* ctl, const RebuildTune& t) {
  RbArgs a = rb_args(g, part, B, m, rs, t);
  a.ctl = ctl;
  for (int dir = 0; dir < 2; ++dir) add_zero(s.zero, rs.d[dir].cnt, (size_t)B, ctl);
  add_zero(s.zero, rs.big_count, 2, ctl);
  slot_push(slot_bind(s.count, kmRbCount), a, vg_count(a));
  for (int dir = 0; dir < 2; ++dir)
    add_scan(s.scan1, rs.d[dir].cnt, rs.d[dir].seg, B, rs.tile + dir * (rs.tile_cap / 2), ctl);
  slot_push(slot_bind(s.scatter, kmRbScatter), a, vg_scatter(a));
  slot_push(slot_bind(s.rows_small, kmRbRowsSmall), a, vg_rows_small(a));
  slot_push(slot_bind(s.rows_big, kmRbRowsBig), a, vg_rows_big(a, t));
  for (int dir = 0; dir < 2; ++dir)
    add_scan(s.scan2, rs.d[dir].uniq, dir == 0 ? m.optr : m.iptr, B,
             rs.tile + dir * (rs.tile_cap / 2), ctl);
  slot_push(slot_bind(s.compact, kmRbCompact), a, vg_compact(a));
}

void DenseBuildSlots::clear() {
  for (Slot* x : all()) x->clear();
}

std::vector<Slot*> DenseBuildSlots::all() { return {&zero, &edges, &mapped, &degrees, &logs}; }

void add_dense_build(DenseBuildSlots& s, const DevGraph& g, const int32_t* part, int32_t B,
                     DevBM& m) {
  const size_t bb = (size_t)B * B;
  add_zero(s.zero, m.Md, bb);
  add_zero(s.zero, m.MTd, bb);
  add_zero(s.zero, m.Sd, (size_t)2 * B * ((B + 31) / 32));
  add_zero(s.zero, m.d_out, (size_t)B);
  add_zero(s.zero, m.d_in, (size_t)B);
  DenseArgs a = dense_args(g, part, B, m);
  slot_push(slot_bind(s.edges, kmDenseEdges), a, g.E > 0 ? ceil_div(g.E, 256) : 0);
  slot_push(slot_bind(s.degrees, kmDenseDegrees), a, ceil_div(g.N, 256));
  slot_push(slot_bind(s.logs, kmDenseLogs), a, ceil_div(B, 256));
}

void add_dense_build_mapped(DenseBuildSlots& s, const DevGraph& g, const int32_t* part,
                            int32_t B, DevBM& m, int32_t B_old, const int32_t* map) {
  const size_t bb = (size_t)B * B;
  add_zero(s.zero, m.Md, bb);
  add_zero(s.zero, m.MTd, bb);
  add_zero(s.zero, m.Sd, (size_t)2 * B * ((B + 31) / 32));
  add_zero(s.zero, m.d_out, (size_t)B);
  add_zero(s.zero, m.d_in, (size_t)B);
  DenseMapArgs b{m.optr, m.ocol, m.ocnt, map, m.Md, m.MTd, m.Sd, B_old, B};
  slot_push(slot_bind(s.mapped, kmDenseFromCsr), b, grid_for((long long)B_old * 32, 256, 148 * 16));
  DenseArgs a = dense_args(g, part, B, m);
  slot_push(slot_bind(s.degrees, kmDenseDegrees), a, ceil_div(g.N, 256));
  slot_push(slot_bind(s.logs, kmDenseLogs), a, ceil_div(B, 256));
}

void add_dense_update(Slot& s, const DevGraph& g, const int32_t* part, int32_t lo, int32_t count,
                      const int32_t* newlab, int32_t B, DevBM& m, const int32_t* ctl) {
  if (count <= 0) return;
  DenseArgs a = dense_args(g, part, B, m);
  a.ctl = ctl;
  a.lo = lo;
  a.count = count;
  a.newlab = newlab;
  slot_push(slot_bind(s, kmDenseUpdate), a, vg_dense_update(count));
}

void add_block_terms(Slot& s, DevBM& m, int32_t B, int draws, uint64_t seed, uint32_t seq,
                     const int32_t* ctl, uint32_t seq_mul) {
  BtArgs a = bt_args(m, B, draws, seed, seq);
  a.ctl = ctl;
  a.seq_mul = seq_mul;
  slot_push(slot_bind(s, kmBlockTerms), a, vg_block_terms(B));
}

void add_block_terms_dense(Slot& s, DevBM& m, int32_t B, int draws, uint64_t seed,
                           uint32_t seq, const int32_t* ctl, uint32_t seq_mul) {
  BtDenseArgs a = bt_dense_args(m, B, draws, seed, seq);
  a.ctl = ctl;
  a.seq_mul = seq_mul;
  slot_push(slot_bind(s, kmBlockTermsDense), a, vg_block_terms(B));
}

void add_mdl_sum(Slot& s, const DevBM& m, int32_t B, double* out, const int32_t* ctl) {
  MdlArgs a{m.dSout, out, ctl, B, 0};
  slot_push(slot_bind(s, kmMdlSum), a, 1);
}

void add_sweep_ctl(Slot& s, int32_t* ctl, const double* dsum, const double* dataS,
                   double model_S, double thr, int32_t window, int32_t max_itr) {
  SweepCtlArgs a{ctl, dsum, dataS, model_S, thr, window, max_itr};
  slot_push(slot_bind(s, kmSweepCtl), a, 1);
}

void add_zero(Slot& s, void* p, size_t words, const int32_t* ctl) {
  WordsArgs a{(uint32_t*)p, nullptr, (long long)words, ctl};
  slot_push(slot_bind(s, kmZero), a, vg_words((long long)words));
}

void add_copy(Slot& s, void* dst, const void* src, size_t words) {
  WordsArgs a{(uint32_t*)dst, (const uint32_t*)src, (long long)words, nullptr};
  slot_push(slot_bind(s, kmCopy), a, vg_words((long long)words));
}

void add_iota(Slot& s, int32_t* p, int32_t n) {
  WordsArgs a{(uint32_t*)p, nullptr, (long long)n, nullptr};
  slot_push(slot_bind(s, kmIota), a, vg_words(n));
}

}  // namespace sbp
