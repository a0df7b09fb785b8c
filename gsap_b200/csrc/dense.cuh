// The per-block draws of a nodal batch from the dense form of M, shared by
// the block-terms kernel and the commit kernel (which draws for the next
// batch once the moved vertices' edges are applied).
#pragma once

#include "common.cuh"

namespace sbp {

// First column k of dense out-row ++ in-row of block b whose running count
// exceeds t (zero columns never advance the count, so this is the same
// entry as in the CSR rows); the whole warp returns it, or -1.  Found
// through the rows' chunk sums (DevBM::Sd, 2K of them: the out-row's K
// chunks, then the in-row's): the chunk whose running count first exceeds
// t, then the column inside it, reading 2K + 32 words instead of up to 2B.
__device__ __forceinline__ int warp_pick_chunked(const uint32_t* orow, const uint32_t* irow,
                                 const uint32_t* srow, int B, int K, uint64_t t, int lane) {
  uint64_t acc = 0;
  for (int k0 = 0; k0 < 2 * K; k0 += 32) {
    const int k = k0 + lane;
    const uint64_t w = k < 2 * K ? __ldg(srow + k) : 0u;
    uint64_t incl = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    const unsigned hit = __ballot_sync(kFull, k < 2 * K && acc + incl > t);
    if (hit) {
      const int j = __ffs(hit) - 1;
      const uint64_t base = acc + __shfl_sync(kFull, incl - w, j);  // count before chunk k0+j
      const int kc = k0 + j;
      const int c0 = (kc < K ? kc : kc - K) * 32;
      const uint32_t* row = kc < K ? orow : irow;
      const int c = c0 + lane;
      uint64_t in2 = c < B ? __ldg(row + c) : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(kFull, in2, o);
        if (lane >= o) in2 += y;
      }
      const unsigned h2 = __ballot_sync(kFull, c < B && base + in2 > t);
      return h2 ? c0 + __ffs(h2) - 1 : -1;
    }
    acc += __shfl_sync(kFull, incl, 31);
  }
  return -1;
}

// Block b's draws for the batch with RNG sequence seq (choose_neighbored_block
// and the per-block uniform, kernels.hpp:942-997, 1024): whether a proposal
// from b takes a uniform random block (use_rand), else the block of a
// neighbour drawn by weight from b's out-row ++ in-row (nbr_s).  The whole
// warp calls it; lane 0 writes.
__device__ __forceinline__ void dense_block_draw(const uint32_t* Md, const uint32_t* MTd,
                                                 const uint32_t* Sd, const uint32_t* d_out,
                                                 const uint32_t* d_in, int32_t B, uint64_t seed,
                                                 uint32_t seq, int b, int lane, int32_t* nbr_s,
                                                 uint8_t* use_rand) {
  const P4 x = draw(seed, kRngNodalBlock, seq, (uint32_t)b);
  const uint64_t deg = (uint64_t)d_out[b] + d_in[b];
  int nb = 0;
  if (deg > 0) {
    const int K = (B + 31) >> 5;
    const int c = warp_pick_chunked(Md + (size_t)b * B, MTd + (size_t)b * B,
                                    Sd + (size_t)b * 2 * K, B, K, scale_draw(x.v[1], deg), lane);
    nb = c >= 0 ? c : 0;
  }
  if (lane == 0) {
    use_rand[b] = accept_random(x.v[0], deg, (uint64_t)B) ? 1 : 0;
    nbr_s[b] = nb;
  }
}

}  // namespace sbp
