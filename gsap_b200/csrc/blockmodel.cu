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

#include <algorithm>

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

__global__ void scan_tile_sums(const int32_t* __restrict__ in, int32_t n, int32_t* tile) {
  __shared__ int sh[33];
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) s += in[base + k];
  int tot;
  cta_excl_scan(s, sh, &tot);
  if (threadIdx.x == 0) tile[blockIdx.x] = tot;
}

// Exclusive scan of `n` values in place, one CTA, tile by tile with a carry.
__global__ void scan_single(const int32_t* __restrict__ in, int32_t* out, int32_t n) {
  __shared__ int sh[33];
  int carry = 0;
  for (int t0 = 0; t0 < n; t0 += kScanTile) {
    int base = t0 + threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      v[k] = base + k < n ? in[base + k] : 0;
      s += v[k];
    }
    int tot;
    int pre = cta_excl_scan(s, sh, &tot) + carry;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      if (base + k < n) out[base + k] = pre;
      pre += v[k];
    }
    carry += tot;
  }
  if (threadIdx.x == 0) out[n] = carry;
}

__global__ void scan_apply(const int32_t* __restrict__ in, int32_t* out, int32_t n,
                           const int32_t* __restrict__ tile_off) {
  __shared__ int sh[33];
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : 0;
    s += v[k];
  }
  int tot;
  int pre = cta_excl_scan(s, sh, &tot) + tile_off[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = pre;
    pre += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = pre;
}

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
  int32_t N, E, B;
};

// Per vertex: its entries form one run inside its block's segment.
__global__ void rb_count(RbArgs a) {
  const RbSide& d = a.s[blockIdx.y];
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= a.N) return;
  int b = a.part[v];
  int len = d.gptr[v + 1] - d.gptr[v];
  // warp-aggregated: lanes with the same block reserve one range together
  unsigned active = __activemask();
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

// Per graph entry: (block of the neighbour, weight) into the owner's run.
__global__ void rb_scatter(RbArgs a) {
  const RbSide& d = a.s[blockIdx.y];
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.E) return;
  int v = __ldg(d.gsrc + j);
  int b = __ldg(a.part + v);
  int pos = __ldg(d.seg + b) + __ldg(d.vofs + v) + (j - __ldg(d.gptr + v));
  d.tcol[pos] = __ldg(a.part + __ldg(d.gidx + j));
  d.tw[pos] = __ldg(d.gw + j);
}

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
__global__ void __launch_bounds__(kRowsWarps * 32) rb_rows_small(RbArgs a) {
  __shared__ unsigned long long sk[kRowsWarps][kWarpCap];
  const RbSide& d = a.s[blockIdx.y];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned long long* key = sk[wid];
  for (int b = blockIdx.x * kRowsWarps + wid; b < a.B; b += gridDim.x * kRowsWarps) {
    int base = d.seg[b];
    int n = d.seg[b + 1] - base;
    if (n > kWarpCap) {
      if (lane == 0) d.big[atomicAdd(d.big_count, 1)] = b;
      continue;
    }
    if (n == 0) {
      if (lane == 0) d.uniq[b] = 0;
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

constexpr int kBigThreads = 512;
constexpr int kHistCap = 16384;  // columns counted in shared memory at once
constexpr int kSortCap = 8192;   // longest segment sorted in shared memory
constexpr size_t kBigSmem = 65536;

__global__ void __launch_bounds__(kBigThreads) rb_rows_big(RbArgs a) {
  extern __shared__ unsigned long long big_sm[];
  __shared__ int sh[33];
  const RbSide& d = a.s[blockIdx.y];
  uint32_t* hist = (uint32_t*)big_sm;
  int nbig = *d.big_count;
  int T = blockDim.x, tid = threadIdx.x;
  for (int idx = blockIdx.x; idx < nbig; idx += gridDim.x) {
    int b = d.big[idx];
    int base = d.seg[b];
    int n = d.seg[b + 1] - base;
    int running = 0;
    if (a.B <= kHistCap || n > kSortCap) {
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

// Per row: unique entries into place, weighted degree and its log2.
__global__ void rb_compact(RbArgs a) {
  const RbSide& d = a.s[blockIdx.y];
  int lane = threadIdx.x & 31;
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int nw = (gridDim.x * blockDim.x) >> 5;
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

// ------------------------------------------------------------ block terms --
struct BtArgs {
  const double* xlx;
  const int32_t *optr, *ocol, *iptr, *icol;
  const uint32_t *ocnt, *icnt, *d_out, *d_in;
  const double *ld_out, *ld_in;
  double *dSout, *ambout, *ambin, *sinfull;
  int32_t* nbr_s;
  uint8_t* use_rand;
  int32_t B;
  int draws;
  uint64_t seed;
  uint32_t seq;
};

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

__global__ void block_terms_kernel(BtArgs a) {
  int lane = threadIdx.x & 31;
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int nw = (gridDim.x * blockDim.x) >> 5;
  for (int b = w; b < a.B; b += nw) {
   if (a.draws != 1) {
    double acc = 0.0;
    for (int i = a.optr[b] + lane; i < a.optr[b + 1]; i += 32) {
      uint32_t m = a.ocnt[i];
      acc += xlx(a.xlx, m) - (double)m * a.ld_in[a.ocol[i]];
    }
    double ao = warp_sum(acc);
    acc = 0.0;
    for (int i = a.iptr[b] + lane; i < a.iptr[b + 1]; i += 32) {
      uint32_t m = a.icnt[i];
      acc += xlx(a.xlx, m) - (double)m * a.ld_out[a.icol[i]];
    }
    double ai = warp_sum(acc);
    if (lane == 0) {
      uint32_t dout = a.d_out[b], din = a.d_in[b];
      a.ambout[b] = ao;
      a.dSout[b] = ao - (dout ? (double)dout * a.ld_out[b] : 0.0);
      a.ambin[b] = ai;
      a.sinfull[b] = ai - (din ? (double)din * a.ld_in[b] : 0.0);
    }
   }
    if (a.draws) {
      P4 x = draw(a.seed, kRngNodalBlock, a.seq, (uint32_t)b);
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


// ------------------------------------------------------------ dense form --
// For small B the blockmodel is kept as two B x B count matrices (rows and
// columns of M both contiguous).  Built once per merge step / golden-section
// restore; after each nodal batch only the edges of the moved vertices are
// applied, with integer atomics (exact, order-independent).

__global__ void dense_edges_kernel(const int32_t* __restrict__ osrc,
                                   const int32_t* __restrict__ oidx,
                                   const uint32_t* __restrict__ ow,
                                   const int32_t* __restrict__ part, int32_t E, int32_t B,
                                   uint32_t* Md, uint32_t* MTd) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= E) return;
  int r = __ldg(part + __ldg(osrc + j)), c = __ldg(part + __ldg(oidx + j));
  uint32_t w = __ldg(ow + j);
  atomicAdd(Md + (size_t)r * B + c, w);
  atomicAdd(MTd + (size_t)c * B + r, w);
}

__global__ void dense_degrees_kernel(const int32_t* __restrict__ part,
                                     const uint32_t* __restrict__ kdo,
                                     const uint32_t* __restrict__ kdi, int32_t N,
                                     uint32_t* d_out, uint32_t* d_in) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  int b = part[v];
  atomicAdd(d_out + b, kdo[v]);
  atomicAdd(d_in + b, kdi[v]);
}

__global__ void dense_logs_kernel(const uint32_t* __restrict__ d_out,
                                  const uint32_t* __restrict__ d_in, int32_t B, double* ld_out,
                                  double* ld_in) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  ld_out[b] = log2((double)d_out[b]);
  ld_in[b] = log2((double)d_in[b]);
}

// One warp per batch vertex that moves: its out-edges move from
// (r, old block of w) to (s, new block of w); its in-edges from unmoved
// sources move from (b(u), r) to (b(u), s).  Edges between two moved vertices
// are handled once, from the source's out-edges.
__global__ void dense_update_kernel(const int32_t* __restrict__ optr,
                                    const int32_t* __restrict__ oidx,
                                    const uint32_t* __restrict__ ow,
                                    const int32_t* __restrict__ iptr,
                                    const int32_t* __restrict__ iidx,
                                    const uint32_t* __restrict__ iw,
                                    const uint32_t* __restrict__ kdo,
                                    const uint32_t* __restrict__ kdi,
                                    const int32_t* __restrict__ part, int32_t lo, int32_t count,
                                    const int32_t* __restrict__ newlab, int32_t B, uint32_t* Md,
                                    uint32_t* MTd, uint32_t* d_out, uint32_t* d_in) {
  const int lane = threadIdx.x & 31;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = w0; i < count; i += nw) {
    const int v = lo + i;
    const int r = part[v], s = newlab[i];
    if (r == s) continue;
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
    }
  }
}

// First column k of dense out-row ++ in-row of block b whose running count
// exceeds t (zero columns never advance the count, so this is the same
// entry as in the CSR rows); the whole warp returns it, or -1.
__device__ int warp_pick_dense(const uint32_t* orow, const uint32_t* irow, int B, uint64_t t,
                               int lane) {
  uint64_t acc = 0;
  for (int k0 = 0; k0 < 2 * B; k0 += 32) {
    int k = k0 + lane;
    uint64_t w = 0;
    if (k < 2 * B) w = k < B ? orow[k] : irow[k - B];
    uint64_t incl = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    unsigned hit = __ballot_sync(kFull, k < 2 * B && acc + incl > t);
    if (hit) {
      int kk = k0 + __ffs(hit) - 1;
      return kk < B ? kk : kk - B;
    }
    acc += __shfl_sync(kFull, incl, 31);
  }
  return -1;
}

struct BtDenseArgs {
  const double* xlx;
  const uint32_t *Md, *MTd, *d_out, *d_in;
  const double *ld_out, *ld_in;
  double *dSout, *ambout, *ambin, *sinfull;
  int32_t* nbr_s;
  uint8_t* use_rand;
  int32_t B;
  int draws;
  uint64_t seed;
  uint32_t seq;
};

__global__ void block_terms_dense_kernel(BtDenseArgs a) {
  int lane = threadIdx.x & 31;
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int nw = (gridDim.x * blockDim.x) >> 5;
  const int B = a.B;
  for (int b = w; b < B; b += nw) {
    const uint32_t* orow = a.Md + (size_t)b * B;
    const uint32_t* irow = a.MTd + (size_t)b * B;
   if (a.draws != 1) {
    double ao = 0.0, ai = 0.0;
    for (int c = lane; c < B; c += 32) {
      uint32_t mo = orow[c], mi = irow[c];
      if (mo) ao += xlx(a.xlx, mo) - (double)mo * a.ld_in[c];
      if (mi) ai += xlx(a.xlx, mi) - (double)mi * a.ld_out[c];
    }
    ao = warp_sum(ao);
    ai = warp_sum(ai);
    if (lane == 0) {
      uint32_t dout = a.d_out[b], din = a.d_in[b];
      a.ambout[b] = ao;
      a.dSout[b] = ao - (dout ? (double)dout * a.ld_out[b] : 0.0);
      a.ambin[b] = ai;
      a.sinfull[b] = ai - (din ? (double)din * a.ld_in[b] : 0.0);
    }
   }
    if (a.draws) {
      P4 x = draw(a.seed, kRngNodalBlock, a.seq, (uint32_t)b);
      uint64_t deg = (uint64_t)a.d_out[b] + a.d_in[b];
      int nb = 0;
      if (deg > 0) {
        int c = warp_pick_dense(orow, irow, B, scale_draw(x.v[1], deg), lane);
        nb = c >= 0 ? c : 0;
      }
      if (lane == 0) {
        a.use_rand[b] = accept_random(x.v[0], deg, (uint64_t)B) ? 1 : 0;
        a.nbr_s[b] = nb;
      }
    }
  }
}

__global__ void fill_xlx_kernel(double* tab) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x < kXlxTable) tab[x] = xlog2x(x);
}

__global__ void mdl_sum_kernel(const double* __restrict__ dSout, int32_t B, double* out) {
  __shared__ double sh[1024];
  double s = 0.0;
  for (int b = threadIdx.x; b < B; b += blockDim.x) s += dSout[b];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

int grid_for(long long items, int per_block, int cap) {
  long long g = (items + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

}  // namespace

cudaError_t init_kernel_attributes() {
  return cudaFuncSetAttribute(rb_rows_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)kBigSmem);
}

void scan_exclusive(const int32_t* in, int32_t* out, int32_t n, int32_t* tile, cudaStream_t st) {
  if (n <= 8 * kScanTile) {
    ++g_launches;
    scan_single<<<1, kScanThreads, 0, st>>>(in, out, n);
    return;
  }
  int tiles = (n + kScanTile - 1) / kScanTile;
  ++g_launches;
  scan_tile_sums<<<tiles, kScanThreads, 0, st>>>(in, n, tile);
  ++g_launches;
  scan_single<<<1, kScanThreads, 0, st>>>(tile, tile + tiles, tiles);
  ++g_launches;
  scan_apply<<<tiles, kScanThreads, 0, st>>>(in, out, n, tile + tiles);
}

void rebuild_blockmodel(const DevGraph& g, const int32_t* part, int32_t B, DevBM& m,
                        RebuildScratch& rs, cudaStream_t st) {
  RbArgs a;
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
    cudaMemsetAsync(r.cnt, 0, sizeof(int32_t) * (size_t)B, st);
  }
  cudaMemsetAsync(rs.big_count, 0, sizeof(int32_t) * 2, st);
  ++g_launches;
  rb_count<<<dim3((g.N + 255) / 256, 2), 256, 0, st>>>(a);
  for (int dir = 0; dir < 2; ++dir)
    scan_exclusive(rs.d[dir].cnt, rs.d[dir].seg, B, rs.tile + dir * (rs.tile_cap / 2), st);
  if (g.E > 0) {
    ++g_launches;
    rb_scatter<<<dim3((g.E + 255) / 256, 2), 256, 0, st>>>(a);
  }
  ++g_launches;
  rb_rows_small<<<dim3(grid_for(B, kRowsWarps, 4096), 2), kRowsWarps * 32, 0, st>>>(a);
  ++g_launches;
  rb_rows_big<<<dim3(2 * 148, 2), kBigThreads, kBigSmem, st>>>(a);
  for (int dir = 0; dir < 2; ++dir)
    scan_exclusive(rs.d[dir].uniq, dir == 0 ? m.optr : m.iptr, B,
                   rs.tile + dir * (rs.tile_cap / 2), st);
  ++g_launches;
  rb_compact<<<dim3(grid_for((long long)B * 32, 256, 4096), 2), 256, 0, st>>>(a);
}

void block_terms(DevBM& m, int32_t B, int draws, uint64_t seed, uint32_t seq, cudaStream_t st) {
  BtArgs a;
  a.xlx = m.xlx;
  a.optr = m.optr; a.ocol = m.ocol; a.iptr = m.iptr; a.icol = m.icol;
  a.ocnt = m.ocnt; a.icnt = m.icnt; a.d_out = m.d_out; a.d_in = m.d_in;
  a.ld_out = m.ld_out; a.ld_in = m.ld_in;
  a.dSout = m.dSout; a.ambout = m.ambout; a.ambin = m.ambin; a.sinfull = m.sinfull;
  a.nbr_s = m.nbr_s; a.use_rand = m.use_rand;
  a.B = B; a.draws = draws; a.seed = seed; a.seq = seq;
  ++g_launches;
  block_terms_kernel<<<grid_for((long long)B * 32, 256, 8192), 256, 0, st>>>(a);
}

void fill_xlx_table(double* tab, cudaStream_t st) {
  ++g_launches;
  fill_xlx_kernel<<<kXlxTable / 256, 256, 0, st>>>(tab);
}

void dense_build(const DevGraph& g, const int32_t* part, int32_t B, DevBM& m, cudaStream_t st) {
  size_t bb = (size_t)B * B;
  cudaMemsetAsync(m.Md, 0, bb * sizeof(uint32_t), st);
  cudaMemsetAsync(m.MTd, 0, bb * sizeof(uint32_t), st);
  cudaMemsetAsync(m.d_out, 0, (size_t)B * sizeof(uint32_t), st);
  cudaMemsetAsync(m.d_in, 0, (size_t)B * sizeof(uint32_t), st);
  if (g.E > 0) {
    ++g_launches;
    dense_edges_kernel<<<(g.E + 255) / 256, 256, 0, st>>>(g.osrc, g.oidx, g.ow, part, g.E, B,
                                                          m.Md, m.MTd);
  }
  ++g_launches;
  dense_degrees_kernel<<<(g.N + 255) / 256, 256, 0, st>>>(part, g.kdo, g.kdi, g.N, m.d_out,
                                                          m.d_in);
  ++g_launches;
  dense_logs_kernel<<<(B + 255) / 256, 256, 0, st>>>(m.d_out, m.d_in, B, m.ld_out, m.ld_in);
}

void dense_update(const DevGraph& g, const int32_t* part, int32_t lo, int32_t count,
                  const int32_t* newlab, int32_t B, DevBM& m, cudaStream_t st) {
  if (count <= 0) return;
  ++g_launches;
  dense_update_kernel<<<grid_for((long long)count * 32, 256, 148 * 16), 256, 0, st>>>(
      g.optr, g.oidx, g.ow, g.iptr, g.iidx, g.iw, g.kdo, g.kdi, part, lo, count, newlab, B, m.Md,
      m.MTd, m.d_out, m.d_in);
}

void block_terms_dense(DevBM& m, int32_t B, int draws, uint64_t seed, uint32_t seq,
                       cudaStream_t st) {
  BtDenseArgs a;
  a.xlx = m.xlx;
  a.Md = m.Md; a.MTd = m.MTd; a.d_out = m.d_out; a.d_in = m.d_in;
  a.ld_out = m.ld_out; a.ld_in = m.ld_in;
  a.dSout = m.dSout; a.ambout = m.ambout; a.ambin = m.ambin; a.sinfull = m.sinfull;
  a.nbr_s = m.nbr_s; a.use_rand = m.use_rand;
  a.B = B; a.draws = draws; a.seed = seed; a.seq = seq;
  ++g_launches;
  block_terms_dense_kernel<<<grid_for((long long)B * 32, 256, 8192), 256, 0, st>>>(a);
}

void mdl_data_sum(const DevBM& m, int32_t B, double* out, cudaStream_t st) {
  ++g_launches;
  mdl_sum_kernel<<<1, 1024, 0, st>>>(m.dSout, B, out);
}

}  // namespace sbp
