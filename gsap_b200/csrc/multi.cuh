// Multi-job launches.
//
// Every kernel body of the partitioner is written against a virtual grid:
// Body::run(args, vb, vg) does the work of virtual block vb of a job whose
// virtual grid has vg blocks.  Two kernels are generated from each body:
//
//   single_kernel<Body>  one job, arguments by value, vb = blockIdx.x;
//   multi_kernel<Body>   many jobs in one launch.  Job j owns the virtual
//                        blocks [cta0[j], cta0[j+1]); each CTA takes one
//                        virtual block (grid-striding only past 2^22 of
//                        them), finds its job with one warp-wide search of
//                        cta0 and loads the job's argument record into
//                        shared memory.  The hardware block scheduler
//                        balances the jobs' uneven blocks.
//
// A body's result for a job depends only on the job's arguments and its
// virtual grid, never on which physical CTA ran which virtual block, so a
// job computes the same bits alone and inside any mix of other jobs.
#pragma once

#include "common.cuh"
#include "kernels.h"

#include <algorithm>
#include <cstring>

namespace sbp {

template <class Body>
__global__ void __launch_bounds__(Body::kThreads, Body::kMinBlocks)
    single_kernel(typename Body::Args a) {
  Body::run(a, (int)blockIdx.x, (int)gridDim.x);
}

template <class Body>
__global__ void __launch_bounds__(Body::kThreads, Body::kMinBlocks) multi_kernel(MultiSpan sp) {
  using Args = typename Body::Args;
  static_assert(sizeof(Args) % 8 == 0, "argument records are copied in 8-byte words");
  constexpr int kWords = (int)(sizeof(Args) / 8);
  __shared__ unsigned long long raw[kWords];
  __shared__ int s_j, s_vb, s_vg;
  const Args& a = *reinterpret_cast<const Args*>(raw);
  int loaded = -1;
  for (int blk = blockIdx.x; blk < sp.total; blk += gridDim.x) {
    if (threadIdx.x < 32) {
      // job = number of job starts cta0[1..njobs-1] at or below blk (the
      // starts increase strictly: jobs without blocks are not listed)
      const int lane = threadIdx.x;
      int cnt = 0;
      for (int i = 1 + lane; i < sp.njobs; i += 32) cnt += __ldg(sp.cta0 + i) <= blk ? 1 : 0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
      if (lane == 0) {
        const int c0 = __ldg(sp.cta0 + cnt);
        s_j = cnt;
        s_vb = blk - c0;
        s_vg = __ldg(sp.cta0 + cnt + 1) - c0;
      }
    }
    __syncthreads();
    const int j = s_j, vb = s_vb, vg = s_vg;
    if (j != loaded) {
      const unsigned long long* src = reinterpret_cast<const unsigned long long*>(
          static_cast<const char*>(sp.args) + (size_t)j * sizeof(Args));
      for (int k = threadIdx.x; k < kWords; k += blockDim.x) raw[k] = __ldg(src + k);
      loaded = j;
    }
    __syncthreads();
    Body::run(a, vb, vg);
    __syncthreads();
  }
}

constexpr int kMaxMultiGrid = 1 << 22;

template <class Body>
void launch_multi(const MultiSpan& sp, cudaStream_t st) {
  if (sp.total <= 0) return;
  const int grid = std::min(sp.total, kMaxMultiGrid);
  ++g_launches;
  multi_kernel<Body><<<grid, Body::kThreads, Body::kSmem, st>>>(sp);
}

template <class Body>
void launch_single(const typename Body::Args& a, int grid, cudaStream_t st) {
  if (grid <= 0) return;
  ++g_launches;
  single_kernel<Body><<<grid, Body::kThreads, Body::kSmem, st>>>(a);
}

// One job's record through the by-value kernel, same virtual grid: a slot
// holding a single job costs no argument loads.
template <class Body>
void launch_one(const void* rec, int32_t vctas, cudaStream_t st) {
  typename Body::Args a;
  std::memcpy(&a, rec, sizeof(a));
  launch_single<Body>(a, vctas, st);
}

template <class Body>
constexpr MultiKernel multi_kernel_desc(const char* name) {
  return MultiKernel{sizeof(typename Body::Args), &launch_multi<Body>, &launch_one<Body>, name};
}

// Appends one job's record to a slot (nothing when it has no virtual blocks).
template <class Args>
void slot_push(Slot& s, const Args& a, int32_t vctas) {
  if (vctas <= 0) return;
  const size_t off = s.recs.size();
  s.recs.resize(off + sizeof(Args));
  std::memcpy(s.recs.data() + off, &a, sizeof(Args));
  s.cta0.push_back(s.cta0.back() + vctas);
}

inline int32_t ceil_div(long long a, long long b) { return (int32_t)((a + b - 1) / b); }

}  // namespace sbp
