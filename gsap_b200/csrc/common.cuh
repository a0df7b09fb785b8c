// Shared device/host helpers of the B200 stochastic block partitioner.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sbp {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// ----------------------------------------------------------------- Philox --
// Philox4x32-10 from its published description (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11): ten rounds of two
// 32x32->64 multiplies with the key bumped by the Weyl constants.  It replaces
// GSAP's clock64()-seeded curand XORWOW (kernels.hpp:655-657, 671-673,
// 869-871) so that a run is a pure function of (seed, graph).
struct P4 {
  uint32_t v[4];
};

__host__ __device__ __forceinline__ void mul_hi_lo(uint32_t a, uint32_t b, uint32_t& hi,
                                                   uint32_t& lo) {
#ifdef __CUDA_ARCH__
  hi = __umulhi(a, b);
  lo = a * b;
#else
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
#endif
}

__host__ __device__ __forceinline__ P4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                     uint32_t c3, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    uint32_t hi0, lo0, hi1, lo1;
    mul_hi_lo(0xD2511F53u, c0, hi0, lo0);
    mul_hi_lo(0xCD9E8D57u, c2, hi1, lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return P4{{c0, c1, c2, c3}};
}

// Counter layout: (index, purpose, sequence number, 0), key = seed.
enum : uint32_t { kRngNodalVertex = 1, kRngNodalBlock = 2, kRngMerge = 3, kRngGenerate = 4 };

__host__ __device__ __forceinline__ P4 draw(uint64_t seed, uint32_t purpose, uint32_t seq,
                                            uint32_t idx) {
  return philox4x32_10(idx, purpose, seq, 0u, (uint32_t)seed, (uint32_t)(seed >> 32));
}

// A uniform integer in [0, D): floor(x * D / 2^32).
__host__ __device__ __forceinline__ uint64_t scale_draw(uint32_t x, uint64_t D) {
#ifdef __CUDA_ARCH__
  // D < 2^33 here; split to stay in 64 bits: x*D = x*Dlo + (x*Dhi << 32)
  uint64_t lo = (uint64_t)x * (uint32_t)D;
  uint64_t hi = (uint64_t)x * (uint32_t)(D >> 32);
  return (lo >> 32) + hi;
#else
  return (uint64_t)(((unsigned __int128)x * D) >> 32);
#endif
}

// x / 2^32 < B / (d + B) exactly: the "propose a random block" test of
// kernels.hpp:847 and :1024 with accepted_prob = B/(d+B) (kernels.hpp:720).
__host__ __device__ __forceinline__ bool accept_random(uint32_t x, uint64_t d, uint64_t B) {
  // x*(d+B) < B*2^32  <=>  floor(x*(d+B) / 2^32) < B, computed in 64 bits
  uint64_t m = d + B;
  uint64_t lo = (uint64_t)x * (uint32_t)m;
  uint64_t hi = (uint64_t)x * (uint32_t)(m >> 32);
  return hi + (lo >> 32) < B;
}

// ------------------------------------------------------------ warp helpers --
__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}
__device__ __forceinline__ long long warp_sum_ll(long long x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}
__device__ __forceinline__ unsigned warp_sum_u(unsigned x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}
__device__ __forceinline__ unsigned long long warp_sum_ull(unsigned long long x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}
// inclusive scan over lanes
__device__ __forceinline__ unsigned warp_incl_scan_u(unsigned x, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// w*log2(w) with w a count; 0 for w == 0.
__device__ __forceinline__ double xlog2x(uint32_t w) {
  return w == 0u ? 0.0 : (double)w * log2((double)w);
}

// x*log2(x) and log2(x) of small counts from a table (tab[x] holds exactly
// xlog2x(x), tab[kXlxTable + x] exactly log2(x), both filled on the device
// with the same functions), larger ones computed.
constexpr uint32_t kXlxTable = 1u << 16;
static __device__ __forceinline__ double xlog2x_big(uint32_t w) {
  return (double)w * log2((double)w);
}
__device__ __forceinline__ double xlx(const double* __restrict__ tab, uint32_t w) {
  return w < kXlxTable ? __ldg(tab + w) : xlog2x_big(w);
}
__device__ __forceinline__ double l2x(const double* __restrict__ tab, uint32_t w) {
  return w < kXlxTable ? __ldg(tab + kXlxTable + w) : log2((double)w);
}

// Sweep control of one job, in device memory: ctl[0] = sweeps completed in
// the current outer step, ctl[1] = 1 once the stop test has ended them.
// Kernels of a queued sweep read it: they skip all work once ctl[1] is set
// and take their RNG sequence and result slot from ctl[0].  A null ctl
// means an ungated launch.
__device__ __forceinline__ bool ctl_stopped(const int32_t* ctl) { return ctl && ctl[1] != 0; }
__device__ __forceinline__ uint32_t ctl_itr(const int32_t* ctl) {
  return ctl ? (uint32_t)ctl[0] : 0u;
}

// Binary search of column c in the CSR row [lo, hi); its count, or 0.
__device__ __forceinline__ uint32_t row_lookup(const int32_t* __restrict__ col,
                                               const uint32_t* __restrict__ cnt, int32_t lo,
                                               int32_t hi, int32_t c) {
  int32_t end = hi;
  while (lo < hi) {
    int32_t mid = (lo + hi) >> 1;
    if (__ldg(col + mid) < c) lo = mid + 1;
    else hi = mid;
  }
  return (lo < end && __ldg(col + lo) == c) ? __ldg(cnt + lo) : 0u;
}

}  // namespace sbp
