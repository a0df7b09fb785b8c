// Graph ingest on the device: the CSR pair of an edge list (the arrays
// GSAP/load.hpp:86-117 builds on the host, rows in the input's edge order)
// and the degree and edge stages of the seeded DCSBM generator, so that a
// graph made or loaded into device memory is partitioned without a host
// round trip.
//
// Both rest on one primitive: a stable LSD radix sort of int32 keys that
// carries each key's input position.  Each 8-bit pass counts the digits of
// 4096-item tiles, scans the (digit, tile) counts in digit-major order and
// scatters every tile's items to their digit's offset, ranking equal digits
// in input order (a warp ranks 32 items at a time with __match_any_sync and
// keeps per-digit counts in shared memory; the warps of a tile then add the
// counts of the warps before them).  Row pointers come from the sorted keys
// by binary search, so nothing here depends on the order of atomics.
#include "common.cuh"
#include "kernels.h"
#include "multi.cuh"

#include <algorithm>
#include <vector>

namespace sbp {

namespace {

constexpr int kRsThreads = 256;  // one thread per digit value in the prefix steps
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;  // 4096 items a CTA
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsWarpItems = kRsTile / kRsWarps;  // 512: 16 rounds of 32
static_assert(kRsThreads == 256, "the prefix steps use one thread per 8-bit digit");

struct RsArgs {
  const int32_t* keys_in;  // non-negative
  const int32_t* vals_in;  // nullptr: the value is the input position
  int32_t* keys_out;
  int32_t* vals_out;
  int32_t* hist;  // 256 * tiles + 1 counts, digit-major, scanned between the steps
  int32_t n, tiles, shift, pad;
};

__device__ __forceinline__ int rs_digit(int32_t key, int shift) {
  return (int)(((uint32_t)key >> shift) & 255u);
}

struct RsHistBody {
  using Args = RsArgs;
  static constexpr int kThreads = kRsThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int) {
    __shared__ int cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const int base = vb * kRsTile;
    for (int k = threadIdx.x; k < kRsTile; k += kRsThreads) {
      const int i = base + k;
      if (i < a.n) atomicAdd(&cnt[rs_digit(a.keys_in[i], a.shift)], 1);
    }
    __syncthreads();
    a.hist[threadIdx.x * a.tiles + vb] = cnt[threadIdx.x];
  }
};

struct RsScatterBody {
  using Args = RsArgs;
  static constexpr int kThreads = kRsThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int) {
    __shared__ int wc[kRsWarps][256];
    for (int k = threadIdx.x; k < kRsWarps * 256; k += kRsThreads) (&wc[0][0])[k] = 0;
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int base = vb * kRsTile + w * kRsWarpItems;
    int32_t key[kRsItems], val[kRsItems];
    int rank[kRsItems];
#pragma unroll
    for (int t = 0; t < kRsItems; ++t) {
      const int i = base + t * 32 + lane;
      const bool ok = i < a.n;
      key[t] = ok ? a.keys_in[i] : 0;
      val[t] = ok ? (a.vals_in ? a.vals_in[i] : i) : 0;
      // lanes past the end get digits no real item has
      const int d = ok ? rs_digit(key[t], a.shift) : 256 + lane;
      const unsigned peers = __match_any_sync(kFull, d);
      int r = -1;
      if (ok) r = wc[w][d] + __popc(peers & lt);
      __syncwarp();
      if (ok && (peers >> lane) == 1u) wc[w][d] += __popc(peers);  // the group's last lane
      __syncwarp();
      rank[t] = r;
    }
    __syncthreads();
    {
      const int d = threadIdx.x;
      int run = 0;
      for (int x = 0; x < kRsWarps; ++x) {
        const int c = wc[x][d];
        wc[x][d] = run;
        run += c;
      }
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < kRsItems; ++t) {
      if (rank[t] < 0) continue;
      const int d = rs_digit(key[t], a.shift);
      const int pos = a.hist[d * a.tiles + vb] + wc[w][d] + rank[t];
      a.keys_out[pos] = key[t];
      a.vals_out[pos] = val[t];
    }
  }
};

// ptr[v] = first position whose sorted key is >= v, v in [0, N].
struct RowPtrArgs {
  const int32_t* keys;
  int32_t* ptr;
  int32_t n, N;
};

struct RowPtrBody {
  using Args = RowPtrArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int) {
    const int v = vb * kThreads + threadIdx.x;
    if (v > a.N) return;
    int lo = 0, hi = a.n;
    while (lo < hi) {
      const int mid = (int)(((unsigned)lo + (unsigned)hi) >> 1);
      if (__ldg(a.keys + mid) < v) lo = mid + 1;
      else hi = mid;
    }
    a.ptr[v] = lo;
  }
};

// Entries of one direction in row order: idx[p] = other[perm[p]], and the
// weight of the edge (1 without weights).
struct GatherArgs {
  const int32_t* perm;
  const int32_t* other;
  const uint32_t* w;
  int32_t* idx;
  uint32_t* wout;
  int32_t n, pad;
};

struct GatherBody {
  using Args = GatherArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    for (int p = vb * kThreads + threadIdx.x; p < a.n; p += vg * kThreads) {
      const int j = __ldg(a.perm + p);
      a.idx[p] = __ldg(a.other + j);
      a.wout[p] = a.w ? __ldg(a.w + j) : 1u;
    }
  }
};

// Edge checks: endpoints in [0, N) (bit 0 of err), weights >= 1 (bit 1).
struct EdgeCheckArgs {
  const int32_t *src, *dst;
  const uint32_t* w;
  int32_t* err;
  int32_t n, N;
};

struct EdgeCheckBody {
  using Args = EdgeCheckArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    int bad = 0;
    for (int j = vb * kThreads + threadIdx.x; j < a.n; j += vg * kThreads) {
      const int32_t s = __ldg(a.src + j), d = __ldg(a.dst + j);
      if (s < 0 || s >= a.N || d < 0 || d >= a.N) bad |= 1;
      if (a.w && __ldg(a.w + j) == 0u) bad |= 2;
    }
    bad = __reduce_or_sync(kFull, bad);
    if (bad && (threadIdx.x & 31) == 0) atomicOr(a.err, bad);
  }
};

// Row degrees (sum of the row's weights, one warp a vertex); a sum that
// does not fit 32 bits sets bit 2 of err.
struct DegreeArgs {
  const int32_t* ptr;
  const uint32_t* w;
  uint32_t* deg;
  int32_t* err;
  int32_t N, pad;
};

struct DegreeBody {
  using Args = DegreeArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    const int lane = threadIdx.x & 31;
    for (int v = (vb * kThreads + threadIdx.x) >> 5; v < a.N; v += (vg * kThreads) >> 5) {
      unsigned long long s = 0;
      for (int p = a.ptr[v] + lane; p < a.ptr[v + 1]; p += 32) s += __ldg(a.w + p);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
      if (lane == 0) {
        a.deg[v] = (uint32_t)s;
        if (s > 0xffffffffull) atomicOr(a.err, 4);
      }
    }
  }
};

__global__ void owner_kernel(const int32_t* __restrict__ ptr, int32_t N, int32_t* src) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= N) return;
  for (int p = ptr[v]; p < ptr[v + 1]; ++p) src[p] = v;
}

// ------------------------------------------------------------- generator --
// The stages of sbp_dcsbm_generate after the labels: out-degrees from the
// power-law CDF, each block's members in vertex order with their running
// degree sums, and the edges of every source (own block with probability
// p_in, else a uniform other block; destination by degree; no self-loops
// or repeated edges; up to 64 draws an edge).  The same Philox counters and
// integer/IEEE-double steps as the host code, so the same edges.
struct GenArgs {
  const int32_t* truth;
  const double* cdf;
  int32_t* deg;
  const int32_t* mem;     // members of all blocks, block-major
  const int32_t* bstart;  // B + 1 block starts in mem
  unsigned long long* cum;
  const int32_t* offs;    // exclusive scan of deg: each source's slot range
  int32_t* tgt;           // accepted destinations of each source, in order
  int32_t* cnt;           // accepted destinations per source
  const int32_t* eoff;    // exclusive scan of cnt
  int32_t *src, *dst;
  uint64_t seed;
  uint64_t pin_scaled;
  int32_t N, B, ncdf, deg_min;
};

__device__ __forceinline__ P4 gen_draw_dev(uint64_t seed, uint32_t stream, uint32_t idx,
                                           uint32_t k) {
  return philox4x32_10(idx, kRngGenerate, stream, k, (uint32_t)seed, (uint32_t)(seed >> 32));
}

__device__ __forceinline__ double unit_open_dev(uint32_t x) {
  return ((double)x + 0.5) * (1.0 / 4294967296.0);
}

struct GenDegreeBody {
  using Args = GenArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    for (int v = vb * kThreads + threadIdx.x; v < a.N; v += vg * kThreads) {
      const P4 x = gen_draw_dev(a.seed, 3, (uint32_t)v, 0);
      const double u = unit_open_dev(x.v[0]) * a.cdf[a.ncdf - 1];
      int lo = 0, hi = a.ncdf;  // lower_bound
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a.cdf[mid] < u) lo = mid + 1;
        else hi = mid;
      }
      a.deg[v] = a.deg_min + min(lo, a.ncdf - 1);
    }
  }
};

// Running degree sums of each block's members: one CTA per block.
struct GenCumBody {
  using Args = GenArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    __shared__ unsigned long long sh[kThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int b = vb; b < a.B; b += vg) {
      const int s0 = a.bstart[b], s1 = a.bstart[b + 1];
      unsigned long long carry = 0;
      for (int i0 = s0; i0 < s1; i0 += kThreads) {
        const int i = i0 + threadIdx.x;
        unsigned long long x = i < s1 ? (unsigned long long)a.deg[a.mem[i]] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const unsigned long long y = __shfl_up_sync(kFull, x, o);
          if (lane >= o) x += y;
        }
        if (lane == 31) sh[w] = x;
        __syncthreads();
        unsigned long long before = carry, tot = 0;
        for (int k = 0; k < kThreads / 32; ++k) {
          if (k < w) before += sh[k];
          tot += sh[k];
        }
        if (i < s1) a.cum[i] = before + x;
        carry += tot;
        __syncthreads();
      }
    }
  }
};

struct GenEdgeBody {
  using Args = GenArgs;
  static constexpr int kThreads = 128, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    for (int u = vb * kThreads + threadIdx.x; u < a.N; u += vg * kThreads) {
      const int32_t own = a.truth[u];
      int32_t* out = a.tgt + a.offs[u];
      int c = 0;
      const int du = a.deg[u];
      for (int k = 0; k < du; ++k) {
        for (uint32_t att = 0; att < 64; ++att) {
          const P4 x = gen_draw_dev(a.seed, 4, (uint32_t)u, ((uint32_t)k << 8) | att);
          int32_t b = own;
          if (a.B > 1 && (uint64_t)x.v[0] >= a.pin_scaled) {
            const int32_t cc = (int32_t)(x.v[1] % (uint32_t)(a.B - 1));
            b = cc >= b ? cc + 1 : cc;
          }
          const int s0 = a.bstart[b], s1 = a.bstart[b + 1];
          const uint64_t t = scale_draw(x.v[2], a.cum[s1 - 1]);
          int lo = s0, hi = s1;  // upper_bound
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (a.cum[mid] <= t) lo = mid + 1;
            else hi = mid;
          }
          const int32_t v = a.mem[lo];
          bool dup = v == u;
          for (int q = 0; q < c && !dup; ++q) dup = out[q] == v;
          if (dup) continue;
          out[c++] = v;
          break;
        }
      }
      a.cnt[u] = c;
    }
  }
};

struct GenCompactBody {
  using Args = GenArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    for (int u = vb * kThreads + threadIdx.x; u < a.N; u += vg * kThreads) {
      const int32_t* in = a.tgt + a.offs[u];
      const int32_t e0 = a.eoff[u], c = a.cnt[u];
      for (int k = 0; k < c; ++k) {
        a.src[e0 + k] = u;
        a.dst[e0 + k] = in[k];
      }
    }
  }
};

int key_bits(int32_t max_key) {
  int b = 1;
  while (b < 31 && (max_key >> b) != 0) ++b;
  return b;
}

int32_t grid_for(long long n, int threads) {
  return (int32_t)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148 * 64));
}

}  // namespace

size_t sort_scratch_bytes(int32_t n) {
  const size_t tiles = (size_t)std::max(1, ceil_div(n, kRsTile));
  const size_t hist = 256 * tiles + 1;
  const size_t scan = 2 * ((hist + 2047) / 2048) + 8;
  return 4 * (2 * (size_t)n + hist + scan) + 256;
}

cudaError_t sort_by_key_stable(const int32_t* keys, int32_t n, int32_t max_key,
                               int32_t* keys_out, int32_t* vals_out, void* scratch,
                               cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int32_t tiles = ceil_div(n, kRsTile);
  int32_t* kb = (int32_t*)scratch;
  int32_t* vbuf = kb + n;
  int32_t* hist = vbuf + n;
  int32_t* scan_tile = hist + 256 * (size_t)tiles + 1;
  const int passes = (key_bits(max_key) + 7) / 8;
  // ping-pong so that the last pass writes keys_out / vals_out
  int32_t* ko[2] = {keys_out, kb};
  int32_t* vo[2] = {vals_out, vbuf};
  int cur = passes % 2 == 1 ? 0 : 1;  // buffer the first pass writes
  const int32_t* kin = keys;
  const int32_t* vin = nullptr;
  for (int p = 0; p < passes; ++p) {
    RsArgs a{};
    a.keys_in = kin;
    a.vals_in = vin;
    a.keys_out = ko[cur];
    a.vals_out = vo[cur];
    a.hist = hist;
    a.n = n;
    a.tiles = tiles;
    a.shift = 8 * p;
    launch_single<RsHistBody>(a, tiles, st);
    scan_exclusive(hist, hist, 256 * tiles, scan_tile, st);
    launch_single<RsScatterBody>(a, tiles, st);
    kin = ko[cur];
    vin = vo[cur];
    cur ^= 1;
  }
  return cudaGetLastError();
}

size_t csr_build_scratch_bytes(int32_t N, int32_t E) {
  (void)N;
  return sort_scratch_bytes(E) + 8 * (size_t)std::max(E, 1) + 256;
}

cudaError_t csr_from_device_edges(int32_t N, int32_t E, const int32_t* src, const int32_t* dst,
                                  const uint32_t* w, DevGraph& g, int32_t* err, void* scratch,
                                  cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(err, 0, 4, st);
  if (e != cudaSuccess) return e;
  int32_t* sk = (int32_t*)scratch;      // sorted keys
  int32_t* perm = sk + std::max(E, 1);  // input position of each sorted entry
  void* ss = perm + std::max(E, 1);
  if (E > 0) {
    EdgeCheckArgs c{src, dst, w, err, E, N};
    launch_single<EdgeCheckBody>(c, grid_for(E, 256), st);
  }
  for (int dir = 0; dir < 2; ++dir) {
    const int32_t* key = dir == 0 ? src : dst;
    const int32_t* other = dir == 0 ? dst : src;
    int32_t* ptr = dir == 0 ? g.optr : g.iptr;
    int32_t* idx = dir == 0 ? g.oidx : g.iidx;
    uint32_t* wout = dir == 0 ? g.ow : g.iw;
    uint32_t* deg = dir == 0 ? g.kdo : g.kdi;
    int32_t* owner = dir == 0 ? g.osrc : g.isrc;
    if (E > 0) {
      e = sort_by_key_stable(key, E, N - 1, sk, perm, ss, st);
      if (e != cudaSuccess) return e;
      GatherArgs ga{perm, other, w, idx, wout, E, 0};
      launch_single<GatherBody>(ga, grid_for(E, 256), st);
    }
    RowPtrArgs ra{sk, ptr, E, N};
    launch_single<RowPtrBody>(ra, ceil_div((long long)N + 1, 256), st);
    DegreeArgs da{ptr, wout, deg, err, N, 0};
    launch_single<DegreeBody>(da, grid_for((long long)N * 32, 256), st);
    ++g_launches;
    owner_kernel<<<ceil_div(N, 256), 256, 0, st>>>(ptr, N, owner);
  }
  return cudaGetLastError();
}

cudaError_t dcsbm_device_edges(const DcsbmDeviceIn& in, DcsbmDeviceOut& out, cudaStream_t st) {
  const int32_t N = in.N, B = in.B;
  // scratch: truth, deg, mem keys, mem, bstart, cum, offs, tgt, cnt, eoff,
  // cdf, sort scratch, scan tiles
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t n1 = (size_t)N + 1;
  const size_t bytes = al(4 * (size_t)N) * 4 + al(4 * ((size_t)B + 1)) + al(8 * (size_t)N) +
                       al(4 * n1) * 3 + al(4 * (size_t)in.max_edges) +
                       al(8 * (size_t)in.ncdf) + al(sort_scratch_bytes(N)) +
                       al(4 * (2 * (n1 / 2048 + 2) + 8));
  char* base = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&base, bytes, st);
  if (e != cudaSuccess) return e;
  char* p = base;
  auto take = [&](size_t n) {
    char* r = p;
    p += al(n);
    return r;
  };
  int32_t* truth = (int32_t*)take(4 * (size_t)N);
  int32_t* deg = (int32_t*)take(4 * (size_t)N);
  int32_t* mkeys = (int32_t*)take(4 * (size_t)N);
  int32_t* mem = (int32_t*)take(4 * (size_t)N);
  int32_t* bstart = (int32_t*)take(4 * ((size_t)B + 1));
  unsigned long long* cum = (unsigned long long*)take(8 * (size_t)N);
  int32_t* offs = (int32_t*)take(4 * n1);
  int32_t* cnt = (int32_t*)take(4 * n1);
  int32_t* eoff = (int32_t*)take(4 * n1);
  int32_t* tgt = (int32_t*)take(4 * (size_t)in.max_edges);
  double* cdf = (double*)take(8 * (size_t)in.ncdf);
  void* ss = take(sort_scratch_bytes(N));
  int32_t* scan_tile = (int32_t*)take(4 * (2 * (n1 / 2048 + 2) + 8));
  auto done = [&](cudaError_t r) {
    cudaError_t f = cudaFreeAsync(base, st);
    return r != cudaSuccess ? r : f;
  };
  e = cudaMemcpyAsync(truth, in.truth, 4 * (size_t)N, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(cdf, in.cdf, 8 * (size_t)in.ncdf, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return done(e);
  GenArgs a{};
  a.truth = truth;
  a.cdf = cdf;
  a.deg = deg;
  a.mem = mem;
  a.bstart = bstart;
  a.cum = cum;
  a.offs = offs;
  a.tgt = tgt;
  a.cnt = cnt;
  a.eoff = eoff;
  a.src = out.src;
  a.dst = out.dst;
  a.seed = in.seed;
  a.pin_scaled = in.pin_scaled;
  a.N = N;
  a.B = B;
  a.ncdf = in.ncdf;
  a.deg_min = in.deg_min;
  launch_single<GenDegreeBody>(a, grid_for(N, 256), st);
  // members of each block in vertex order, and the block starts
  e = sort_by_key_stable(truth, N, B - 1, mkeys, mem, ss, st);
  if (e != cudaSuccess) return done(e);
  RowPtrArgs ra{mkeys, bstart, N, B};
  launch_single<RowPtrBody>(ra, ceil_div((long long)B + 1, 256), st);
  launch_single<GenCumBody>(a, std::min(B, 148 * 8), st);
  scan_exclusive(deg, offs, N, scan_tile, st);
  launch_single<GenEdgeBody>(a, grid_for(N, 128), st);
  scan_exclusive(cnt, eoff, N, scan_tile, st);
  e = cudaMemcpyAsync(out.E_host, eoff + N, 4, cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return done(e);
  launch_single<GenCompactBody>(a, grid_for(N, 256), st);
  e = cudaGetLastError();
  return done(e);
}

}  // namespace sbp
