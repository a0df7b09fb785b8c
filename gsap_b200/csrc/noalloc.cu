// sbp_mdl_device_static: the MDL of a blockmodel that already sits in device
// memory, computed without allocating anything.
//
// Some callers cannot allocate device memory at the point where they need
// the objective: hosts that own all device memory through their own pool and
// do not let a library allocate behind their back, and serving loops that
// forbid the device-wide synchronisation a cudaMalloc or cudaFree can cost.
// For them this entry point keeps its scratch (the log2 of the block degrees
// and the per-CTA partial sums) in one file-scope device array of fixed size,
// created when the library is loaded and held by every GPU that loads it
// until the process exits.  The caller passes the inputs and the outputs.
//
// Limits and rules of use:
//   * at most kStaticMaxBlocks (65,536) blocks; larger B is rejected;
//   * the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress, with that device current) and caches it for the
//     process; make that first call before any stream capture.  A
//     cudaDeviceReset ends the context the cached address belongs to, and
//     the entry point must not be called on that device afterwards;
//   * every call on a device shares the one array, and the array keeps the
//     last call's contents: calls that overlap on the GPU (different
//     streams, or work still running) race on it.  Each call clears what
//     must start at zero (the CTA ticket of the reduction) itself.
#include "../../include/sbp.h"
#include "common.cuh"

#include <cmath>
#include <mutex>
#include <string>

namespace sbp {
sbp_status host_fail(sbp_status st, const char* msg);

namespace {

constexpr int kStaticMaxBlocks = 65536;
constexpr int kStaticCtas = 128;
constexpr int kStaticThreads = 256;

struct StaticScratch {
  double ld_out[kStaticMaxBlocks];
  double ld_in[kStaticMaxBlocks];
  double part[kStaticCtas];
  unsigned ticket;
};

// ~1 MB: the whole scratch of sbp_mdl_device_static.
static __device__ __align__(256) unsigned char g_mdl_scratch[sizeof(StaticScratch)];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
StaticScratch* g_addr[kMaxDevices] = {};

// log2 of the block degrees; also clears the ticket of the reduction.
__global__ void static_logs_kernel(StaticScratch* sc, int32_t B, const uint32_t* __restrict__ d_out,
                                   const uint32_t* __restrict__ d_in) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b == 0) sc->ticket = 0u;
  for (; b < B; b += gridDim.x * blockDim.x) {
    sc->ld_out[b] = log2((double)d_out[b]);
    sc->ld_in[b] = log2((double)d_in[b]);
  }
}

// data_S = sum over blocks b of sum over out-row b of
//   M (log2 M - log2 d_out[b] - log2 d_in[c])
// (compute_overall_S_transform, kernels.hpp:1066-1093), then
// S = model - data_S (partition.hpp:696-701).  Rows are dealt to threads in
// a fixed order, CTA partials land in the scratch and the last CTA (ticket)
// adds them in CTA order: the result does not depend on scheduling.
__global__ void __launch_bounds__(kStaticThreads) static_mdl_kernel(
    StaticScratch* sc, int32_t B, const int32_t* __restrict__ optr,
    const int32_t* __restrict__ ocol, const uint32_t* __restrict__ ocnt,
    const uint32_t* __restrict__ d_out, double model, double* S, double* data_S) {
  __shared__ double sh[kStaticThreads];
  __shared__ bool last;
  const int tid = threadIdx.x;
  double acc = 0.0;
  for (int b = blockIdx.x * kStaticThreads + tid; b < B; b += gridDim.x * kStaticThreads) {
    const double ldo = sc->ld_out[b];
    double row = 0.0;
    for (int i = optr[b]; i < optr[b + 1]; ++i) {
      const uint32_t m = ocnt[i];
      if (m) row += xlog2x(m) - (double)m * sc->ld_in[ocol[i]];
    }
    const uint32_t d = d_out[b];
    acc += row - (d ? (double)d * ldo : 0.0);
  }
  sh[tid] = acc;
  __syncthreads();
  for (int o = kStaticThreads / 2; o > 0; o >>= 1) {
    if (tid < o) sh[tid] += sh[tid + o];
    __syncthreads();
  }
  if (tid == 0) {
    sc->part[blockIdx.x] = sh[0];
    __threadfence();
    last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && tid == 0) {
    __threadfence();
    double t = 0.0;
    for (int k = 0; k < (int)gridDim.x; ++k) t += ((volatile double*)sc->part)[k];
    *data_S = t;
    *S = model - t;
  }
}

// The scratch's device address on the current device, looked up once.
sbp_status scratch_address(StaticScratch** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return host_fail(SBP_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return host_fail(SBP_ERR_INVALID, "device ordinal too large");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_mdl_scratch);
    if (e != cudaSuccess) return host_fail(SBP_ERR_CUDA, cudaGetErrorString(e));
    g_addr[dev] = (StaticScratch*)p;
  }
  *out = g_addr[dev];
  return SBP_OK;
}

}  // namespace
}  // namespace sbp

extern "C" sbp_status sbp_mdl_device_static(int32_t N, int32_t E, int32_t B,
                                            const int32_t* out_ptr, const int32_t* out_col,
                                            const uint32_t* out_cnt, const uint32_t* d_out,
                                            const uint32_t* d_in, double* S, double* data_S,
                                            void* stream) {
  using namespace sbp;
  if (N < 1 || E < 1 || B < 1 || !out_ptr || !out_col || !out_cnt || !d_out || !d_in || !S ||
      !data_S)
    return host_fail(SBP_ERR_INVALID, "sbp_mdl_device_static: bad arguments");
  if (B > kStaticMaxBlocks)
    return host_fail(SBP_ERR_INVALID,
                     "sbp_mdl_device_static: B exceeds its static scratch (65536 blocks)");
  StaticScratch* sc = nullptr;
  sbp_status s = scratch_address(&sc);
  if (s != SBP_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  const double b = (double)B, x = b * b / (double)E;
  const double model =
      (double)E * (1.0 + x) * std::log(1.0 + x) - x * std::log(x) + (double)N * std::log(b);
  // A launch error left pending by earlier, unrelated work is cleared first
  // so that the status below belongs to these two launches (a sticky error,
  // which ends the context, is reported again by the check after them).
  (void)cudaGetLastError();
  static_logs_kernel<<<(B + kStaticThreads - 1) / kStaticThreads, kStaticThreads, 0, st>>>(
      sc, B, d_out, d_in);
  static_mdl_kernel<<<kStaticCtas, kStaticThreads, 0, st>>>(sc, B, out_ptr, out_col, out_cnt,
                                                            d_out, model, S, data_S);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return host_fail(SBP_ERR_CUDA, cudaGetErrorString(e));
  return SBP_OK;
}
