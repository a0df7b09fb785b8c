// Nodal batch: proposal, dS and accept for each vertex of a Jacobi batch.
//
// GSAP spends ~25 launches and two bb_segsorts of all E neighbour-block lists
// per batch (partition.hpp:456-662); each of its seven dS kernels has one
// thread walk a whole blockmodel row in a serial sorted merge with the
// vertex's sorted neighbour-block list (kernels.hpp:494-597, 1153-1726).
//
// Here a group of threads owns one vertex: a warp for ordinary vertices, a
// whole CTA for the few with more than kWarpList neighbours in a direction
// (a static per-batch list, run on a second stream next to the warp kernel).
//   * proposal: Philox draws, an exact integer inverse-CDF pick of a
//     neighbour (a warp prefix scan over its out- then in-entries), then the
//     per-block draws of the batch (kernels.hpp:877-1032);
//   * neighbour blocks grouped per distinct block: in registers with
//     __match_any_sync / __reduce_add_sync when a list fits a warp, else
//     sorted in shared memory (bitonic), else hashed in shared memory in
//     passes; GSAP sorts all E entries every batch;
//   * dS: GSAP's seven terms rewritten as "old row sum + changed columns".
//     A row term  sum_c f(x_c)  with  f(x) = x (log2 x - log2 dcol[c] - L)
//     splits into  sum_c (x log2 x - x log2 dcol[c])  -  L * sum_c x ;
//     the first sum over the unchanged columns is the per-block sum computed
//     once per batch (ambout / ambin), so only the columns the vertex touches
//     are visited.  Counts come from the dense B x B form (small B, O(1)) or
//     by binary search in the CSR rows.
//     Quirks of the reference kept: old column degrees (Q2), one term per
//     list entry for blocks missing from the target row
//     (kernels.hpp:1648-1652, 1314-1318), the r/s in-weight corrections and
//     the conditional extra column term (kernels.hpp:1506-1510, 1573-1578,
//     1663-1669, 1718-1723), unsigned count arithmetic.
//   * accept iff dS < 0 (kernels.hpp:634-640); the new label goes to a side
//     buffer so every vertex of the batch sees the same old labels.
// All entropy arithmetic is FP64.
#include "common.cuh"
#include "kernels.h"

namespace sbp {

namespace {

constexpr int kNodalWarps = 8;
constexpr int kWarpList = 128;     // entries per direction a warp sorts in shared memory
constexpr int kHeavyThreads = 256;
constexpr int kHeavyList = 4096;   // entries per direction a CTA sorts in shared memory
constexpr int kHashSlotsCfg = 8192;
// sorted lists (two directions) or the hash table (key, sum, first)
constexpr size_t kHeavySmem =
    2 * kHeavyList * sizeof(unsigned long long) > 3 * kHashSlotsCfg * sizeof(int32_t)
        ? 2 * kHeavyList * sizeof(unsigned long long)
        : 3 * kHashSlotsCfg * sizeof(int32_t);

struct NodalArgs {
  const double* xlx;        // x log2 x table
  const int32_t *optr, *oidx, *iptr, *iidx;
  const uint32_t *ow, *iw, *kdo, *kdi;
  const int32_t* part;
  const int32_t *bop, *boc, *bip, *bic;
  const uint32_t *bon, *bin, *d_out, *d_in;
  const uint32_t *Md, *MTd;
  const double *ld_out, *ld_in, *dSout, *ambout, *ambin, *sinfull;
  const int32_t* nbr_s;
  const uint8_t* use_rand;
  int32_t B;
  uint64_t seed;
  uint32_t seq;
  int32_t lo, count;
  const int32_t* verts;     // given mode
  const int32_t* props_in;  // given mode
  int32_t* newlab;
  double* rec;
  int32_t* props_out;
  double* dS_raw;
  const int32_t* heavy;     // batch indices handled by the CTA kernel
  int32_t nheavy;
  int32_t* err;             // error counter (hash table overflow)
};

// g(x, a) = x log2 x - x a, zero for x == 0
__device__ __forceinline__ double gterm(const double* tab, uint32_t x, double a) {
  return x == 0u ? 0.0 : xlx(tab, x) - (double)x * a;
}

// The four rows a move from r to s reads: out-rows r and s, in-rows r and s.
template <bool DENSE>
struct Rows;

template <>
struct Rows<false> {
  const int32_t *oc, *ic;
  const uint32_t *on, *inn;
  int32_t rO0, rO1, sO0, sO1, rI0, rI1, sI0, sI1;
  __device__ Rows(const NodalArgs& a, int r, int s)
      : oc(a.boc), ic(a.bic), on(a.bon), inn(a.bin), rO0(a.bop[r]), rO1(a.bop[r + 1]),
        sO0(a.bop[s]), sO1(a.bop[s + 1]), rI0(a.bip[r]), rI1(a.bip[r + 1]), sI0(a.bip[s]),
        sI1(a.bip[s + 1]) {}
  __device__ __forceinline__ uint32_t out_r(int c) const { return row_lookup(oc, on, rO0, rO1, c); }
  __device__ __forceinline__ uint32_t out_s(int c) const { return row_lookup(oc, on, sO0, sO1, c); }
  __device__ __forceinline__ uint32_t in_r(int c) const { return row_lookup(ic, inn, rI0, rI1, c); }
  __device__ __forceinline__ uint32_t in_s(int c) const { return row_lookup(ic, inn, sI0, sI1, c); }
};

template <>
struct Rows<true> {
  const uint32_t *orr, *ors, *irr, *irs;
  __device__ Rows(const NodalArgs& a, int r, int s)
      : orr(a.Md + (size_t)r * a.B), ors(a.Md + (size_t)s * a.B), irr(a.MTd + (size_t)r * a.B),
        irs(a.MTd + (size_t)s * a.B) {}
  __device__ __forceinline__ uint32_t out_r(int c) const { return __ldg(orr + c); }
  __device__ __forceinline__ uint32_t out_s(int c) const { return __ldg(ors + c); }
  __device__ __forceinline__ uint32_t in_r(int c) const { return __ldg(irr + c); }
  __device__ __forceinline__ uint32_t in_s(int c) const { return __ldg(irs + c); }
};

// Accumulators of the changed columns of the four new rows (out r, out s,
// in r, in s): a = sum of (x log2 x - x log2 dcol) deltas, m = count deltas.
struct Acc {
  double a4 = 0.0, a5 = 0.0, a6 = 0.0, a7 = 0.0;
  long long m4 = 0, m5 = 0, m6 = 0, m7 = 0;
};

// One out-entry (block c, weight w) of v; `leader` marks one entry per
// distinct block, kc = v's total weight into c (kernels.hpp:1444-1726).
template <bool DENSE>
__device__ __forceinline__ void out_entry(const NodalArgs& a, const Rows<DENSE>& R, int r, int s,
                                          uint32_t niS, int32_t c, uint32_t w, bool leader,
                                          uint32_t kc, Acc& q) {
  const double ldc = a.ld_in[c];
  const uint32_t Msc = R.out_s(c);
  if (leader && c != r && c != s) {
    const uint32_t Mrc = R.out_r(c);
    const uint32_t x = Mrc - kc;
    q.a4 += gterm(a.xlx, x, ldc) - gterm(a.xlx, Mrc, ldc);
    q.m4 += (long long)x - (long long)Mrc;
    if (Msc != 0u) {
      const uint32_t y = Msc + kc;
      q.a5 += gterm(a.xlx, y, ldc) - gterm(a.xlx, Msc, ldc);
      q.m5 += (long long)y - (long long)Msc;
    }
  }
  if (Msc == 0u) {
    // block c absent from row s: one term per list entry
    const uint32_t y = w - (c == r ? niS : 0u) + (c == s ? niS : 0u);
    q.a5 += gterm(a.xlx, y, ldc);
    q.m5 += (long long)y;
  }
}

// One in-entry of v: rows r and s of the in CSR, blocks r and s left out.
template <bool DENSE>
__device__ __forceinline__ void in_entry(const NodalArgs& a, const Rows<DENSE>& R, int r, int s,
                                         int32_t c, uint32_t w, bool leader, uint32_t kc,
                                         Acc& q) {
  if (c == r || c == s) return;
  const double ldc = a.ld_out[c];
  const uint32_t Mcs = R.in_s(c);
  if (leader) {
    const uint32_t Mcr = R.in_r(c);
    const uint32_t x = Mcr - kc;
    q.a6 += gterm(a.xlx, x, ldc) - gterm(a.xlx, Mcr, ldc);
    q.m6 += (long long)x - (long long)Mcr;
    if (Mcs != 0u) {
      const uint32_t y = Mcs + kc;
      q.a7 += gterm(a.xlx, y, ldc) - gterm(a.xlx, Mcs, ldc);
      q.m7 += (long long)y - (long long)Mcs;
    }
  }
  if (Mcs == 0u) {
    q.a7 += gterm(a.xlx, w, ldc);
    q.m7 += (long long)w;
  }
}

// The (r, s) corner, the old terms and the new-row totals.  Every thread
// of the group holds the reduced q and returns the same value; the dozen
// logarithms involved are computed once each, spread over the lanes of each
// warp and broadcast with shuffles.
template <bool DENSE>
__device__ double finish_delta(const NodalArgs& a, const Rows<DENSE>& R, int v, int r, int s,
                               uint32_t koR, uint32_t koS, uint32_t niR, uint32_t niS, Acc q) {
  const int lane = threadIdx.x & 31;
  uint32_t m = 0u;
  if (lane == 0) m = R.out_r(r);
  else if (lane == 1) m = R.out_r(s);
  else if (lane == 2) m = R.out_s(r);
  else if (lane == 3) m = R.out_s(s);
  const uint32_t Mrr = __shfl_sync(kFull, m, 0), Mrs = __shfl_sync(kFull, m, 1);
  const uint32_t Msr = __shfl_sync(kFull, m, 2), Mss = __shfl_sync(kFull, m, 3);
  const uint32_t kO = a.kdo[v], kI = a.kdi[v];
  const uint32_t dor = a.d_out[r], dos = a.d_out[s], dir = a.d_in[r], dis = a.d_in[s];
  // new counts of the corner cells (kernels.hpp:1506-1510, 1573-1578,
  // 1663-1669, 1718-1723); when Mrs (Mss) is 0 the extra column term holds
  // niR (niS)
  const uint32_t xrr = Mrr - koR - niR;
  const uint32_t xrs = Mrs != 0u ? Mrs - koS + niR : niR;
  const uint32_t xsr = Msr + koR - niS;
  const uint32_t xss = Mss != 0u ? Mss + koS + niS : niS;
  uint32_t arg = 0u;
  switch (lane) {
    case 0: arg = Mrr; break;
    case 1: arg = Mrs; break;
    case 2: arg = Msr; break;
    case 3: arg = Mss; break;
    case 4: arg = xrr; break;
    case 5: arg = xrs; break;
    case 6: arg = xsr; break;
    case 7: arg = xss; break;
    case 8: arg = dor - kO; break;
    case 9: arg = dos + kO; break;
    case 10: arg = dir - kI; break;
    case 11: arg = dis + kI; break;
    default: break;
  }
  double val = 0.0;
  if (lane < 8) val = arg == 0u ? 0.0 : xlx(a.xlx, arg);
  else if (lane < 12) val = log2((double)arg);
  const double XMrr = __shfl_sync(kFull, val, 0), XMrs = __shfl_sync(kFull, val, 1);
  const double XMsr = __shfl_sync(kFull, val, 2), XMss = __shfl_sync(kFull, val, 3);
  const double Xrr = __shfl_sync(kFull, val, 4), Xrs = __shfl_sync(kFull, val, 5);
  const double Xsr = __shfl_sync(kFull, val, 6), Xss = __shfl_sync(kFull, val, 7);
  const double L4 = __shfl_sync(kFull, val, 8), L5 = __shfl_sync(kFull, val, 9);
  const double L6 = __shfl_sync(kFull, val, 10), L7 = __shfl_sync(kFull, val, 11);
  const double ldi_r = a.ld_in[r], ldi_s = a.ld_in[s];
  const double ldo_r = a.ld_out[r], ldo_s = a.ld_out[s];
  // g(x, a) = x log2 x - x a from the broadcast x log2 x
  auto g = [](double xl, uint32_t x, double ld) { return x == 0u ? 0.0 : xl - (double)x * ld; };
  // f(M; a, b) = M log2 M - M (a + b)
  auto f = [](double xl, uint32_t x, double l1, double l2) {
    return x == 0u ? 0.0 : xl - (double)x * (l1 + l2);
  };
  if (Mrr != 0u) {
    q.a4 += g(Xrr, xrr, ldi_r) - g(XMrr, Mrr, ldi_r);
    q.m4 += (long long)xrr - (long long)Mrr;
  }
  if (Mrs != 0u) {
    q.a4 += g(Xrs, xrs, ldi_s) - g(XMrs, Mrs, ldi_s);
    q.m4 += (long long)xrs - (long long)Mrs;
  } else if (niR > 0u) {
    q.a4 += g(Xrs, niR, ldi_s);
    q.m4 += (long long)niR;
  }
  if (Msr != 0u) {
    q.a5 += g(Xsr, xsr, ldi_r) - g(XMsr, Msr, ldi_r);
    q.m5 += (long long)xsr - (long long)Msr;
  }
  if (Mss != 0u) {
    q.a5 += g(Xss, xss, ldi_s) - g(XMss, Mss, ldi_s);
    q.m5 += (long long)xss - (long long)Mss;
  } else if (koS == 0u && niS > 0u) {
    q.a5 += g(Xss, niS, ldi_s);
    q.m5 += (long long)niS;
  }
  // old terms (calculate_dS_out, calculate_dS_in_nodal_r/_s)
  double t1 = a.dSout[r] + a.dSout[s];
  double t2 = a.sinfull[r] - f(XMrr, Mrr, ldo_r, ldi_r) - f(XMsr, Msr, ldo_s, ldi_r);
  double t3 = a.sinfull[s] - f(XMrs, Mrs, ldo_r, ldi_s) - f(XMss, Mss, ldo_s, ldi_s);
  // new rows r and s, out and in
  long long mass4 = (long long)dor + q.m4;
  long long mass5 = (long long)dos + q.m5;
  long long mass6 = (long long)dir - (long long)Mrr - (long long)Msr + q.m6;
  long long mass7 = (long long)dis - (long long)Mrs - (long long)Mss + q.m7;
  double t4 = a.ambout[r] + q.a4;
  if (mass4 != 0) t4 -= L4 * (double)mass4;
  double t5 = a.ambout[s] + q.a5;
  if (mass5 != 0) t5 -= L5 * (double)mass5;
  double t6 = a.ambin[r] - g(XMrr, Mrr, ldo_r) - g(XMsr, Msr, ldo_s) + q.a6;
  if (mass6 != 0) t6 -= L6 * (double)mass6;
  double t7 = a.ambin[s] - g(XMrs, Mrs, ldo_r) - g(XMss, Mss, ldo_s) + q.a7;
  if (mass7 != 0) t7 -= L7 * (double)mass7;
  return t1 + t2 + t3 - t4 - t5 - t6 - t7;
}

// A thread group cooperating on one vertex: a warp (G = 32) or a CTA.
template <int G>
struct Group {
  double* red;  // G/32 doubles of shared scratch (CTA only)
  __device__ __forceinline__ int rank() const { return G == 32 ? (threadIdx.x & 31) : threadIdx.x; }
  __device__ __forceinline__ void sync() const {
    if (G == 32) __syncwarp();
    else __syncthreads();
  }
  __device__ double sum(double x) const {
    x = warp_sum(x);
    if (G == 32) return x;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < G / 32; ++i) t += red[i];
    __syncthreads();
    return t;
  }
  __device__ long long sum_ll(long long x) const {
    return (long long)sum((double)x);  // |x| < 2^53: exact
  }
};

template <int G>
__device__ __forceinline__ void reduce_acc(Acc& q, const Group<G>& grp) {
  q.a4 = grp.sum(q.a4);
  q.a5 = grp.sum(q.a5);
  q.a6 = grp.sum(q.a6);
  q.a7 = grp.sum(q.a7);
  q.m4 = grp.sum_ll(q.m4);
  q.m5 = grp.sum_ll(q.m5);
  q.m6 = grp.sum_ll(q.m6);
  q.m7 = grp.sum_ll(q.m7);
}

// Ascending bitonic sort of P (power of two) keys by the group.
template <int G>
__device__ void group_sort(unsigned long long* key, int P, const Group<G>& grp) {
  const int t = grp.rank();
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = t; i < P; i += G) {
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
      grp.sync();
    }
  }
}

__device__ __forceinline__ int32_t kblk(unsigned long long k) { return (int32_t)(k >> 32); }
__device__ __forceinline__ uint32_t kwt(unsigned long long k) { return (uint32_t)k; }

// Stage v's neighbour blocks of one direction as sorted (block, weight) keys.
template <int G>
__device__ void stage_sorted(const int32_t* __restrict__ idx, const uint32_t* __restrict__ w,
                             const int32_t* __restrict__ part, int32_t base, int n,
                             unsigned long long* key, const Group<G>& grp) {
  int P = 32;
  while (P < n) P <<= 1;
  for (int k = grp.rank(); k < P; k += G)
    key[k] = k < n ? ((unsigned long long)(uint32_t)__ldg(part + __ldg(idx + base + k)) << 32) |
                         __ldg(w + base + k)
                   : ~0ull;
  grp.sync();
  group_sort<G>(key, P, grp);
}

// dS from v's sorted neighbour-block lists ko[0..no) (out), ki[0..ni) (in).
template <bool DENSE, int G>
__device__ double delta_sorted(const NodalArgs& a, int v, int r, int s,
                               const unsigned long long* ko, int no,
                               const unsigned long long* ki, int ni, const Group<G>& grp) {
  const int t = grp.rank();
  const Rows<DENSE> R(a, r, s);
  uint32_t koR = 0, koS = 0, niR = 0, niS = 0;
  for (int k = t; k < no; k += G) {
    int32_t c = kblk(ko[k]);
    koR += c == r ? kwt(ko[k]) : 0u;
    koS += c == s ? kwt(ko[k]) : 0u;
  }
  for (int k = t; k < ni; k += G) {
    int32_t c = kblk(ki[k]);
    niR += c == r ? kwt(ki[k]) : 0u;
    niS += c == s ? kwt(ki[k]) : 0u;
  }
  koR = (uint32_t)grp.sum_ll(koR);
  koS = (uint32_t)grp.sum_ll(koS);
  niR = (uint32_t)grp.sum_ll(niR);
  niS = (uint32_t)grp.sum_ll(niS);
  Acc q;
  for (int k = t; k < no; k += G) {
    const int32_t c = kblk(ko[k]);
    const bool leader = k == 0 || kblk(ko[k - 1]) != c;
    uint32_t kc = 0;
    if (leader)
      for (int j = k; j < no && kblk(ko[j]) == c; ++j) kc += kwt(ko[j]);
    out_entry<DENSE>(a, R, r, s, niS, c, kwt(ko[k]), leader, kc, q);
  }
  for (int k = t; k < ni; k += G) {
    const int32_t c = kblk(ki[k]);
    const bool leader = k == 0 || kblk(ki[k - 1]) != c;
    uint32_t kc = 0;
    if (leader)
      for (int j = k; j < ni && kblk(ki[j]) == c; ++j) kc += kwt(ki[j]);
    in_entry<DENSE>(a, R, r, s, c, kwt(ki[k]), leader, kc, q);
  }
  reduce_acc(q, grp);
  return finish_delta<DENSE>(a, R, v, r, s, koR, koS, niR, niS, q);
}

// dS when both lists fit in one warp: each lane holds one out- and one
// in-entry; entries of the same block are grouped with __match_any_sync and
// their weights summed with __reduce_add_sync.
template <bool DENSE>
__device__ double delta_registers(const NodalArgs& a, int v, int r, int s, int32_t o0, int no,
                                  int32_t i0, int ni, int lane) {
  const Rows<DENSE> R(a, r, s);
  const bool vo = lane < no, vi = lane < ni;
  const int32_t co = vo ? __ldg(a.part + __ldg(a.oidx + o0 + lane)) : -1 - lane;
  const uint32_t wo = vo ? __ldg(a.ow + o0 + lane) : 0u;
  const int32_t ci = vi ? __ldg(a.part + __ldg(a.iidx + i0 + lane)) : -1 - lane;
  const uint32_t wi = vi ? __ldg(a.iw + i0 + lane) : 0u;
  const unsigned po = __match_any_sync(kFull, co);
  const unsigned pi = __match_any_sync(kFull, ci);
  const uint32_t kco = __reduce_add_sync(po, wo);
  const uint32_t kci = __reduce_add_sync(pi, wi);
  const uint32_t koR = __reduce_add_sync(kFull, co == r ? wo : 0u);
  const uint32_t koS = __reduce_add_sync(kFull, co == s ? wo : 0u);
  const uint32_t niR = __reduce_add_sync(kFull, ci == r ? wi : 0u);
  const uint32_t niS = __reduce_add_sync(kFull, ci == s ? wi : 0u);
  Acc q;
  if (vo) out_entry<DENSE>(a, R, r, s, niS, co, wo, lane == __ffs(po) - 1, kco, q);
  if (vi) in_entry<DENSE>(a, R, r, s, ci, wi, lane == __ffs(pi) - 1, kci, q);
  q.a4 = warp_sum(q.a4);
  q.a5 = warp_sum(q.a5);
  q.a6 = warp_sum(q.a6);
  q.a7 = warp_sum(q.a7);
  // per-lane count deltas are bounded by the vertex's degree: 32-bit sums
  q.m4 = __reduce_add_sync(kFull, (int)q.m4);
  q.m5 = __reduce_add_sync(kFull, (int)q.m5);
  q.m6 = __reduce_add_sync(kFull, (int)q.m6);
  q.m7 = __reduce_add_sync(kFull, (int)q.m7);
  return finish_delta<DENSE>(a, R, v, r, s, koR, koS, niR, niS, q);
}

// Lists too long for shared memory: per-block totals from a shared-memory
// hash table, built in passes that each take the blocks of one hash class,
// so the table never holds more than a few thousand blocks.  Costs
// O(n * passes) with passes ~ n / 2048.
constexpr int kHashSlots = kHashSlotsCfg;
struct HashTab {
  int32_t* key;    // -1 = empty
  uint32_t* sum;
  int32_t* first;  // smallest entry index of the block
};

__device__ __forceinline__ uint32_t hslot(int32_t c) { return ((uint32_t)c * 2654435761u) >> 19; }
__device__ __forceinline__ uint32_t hclass(int32_t c, uint32_t P) {
  return ((uint32_t)c * 0x85EBCA6Bu ^ ((uint32_t)c >> 13)) % P;
}

// Inserts block c (entry k, weight w); false if the table is full.
__device__ bool hash_add(const HashTab& h, int32_t c, uint32_t w, int k) {
  uint32_t i = hslot(c);
  for (int probe = 0; probe < kHashSlots; ++probe, i = (i + 1) & (kHashSlots - 1)) {
    int32_t cur = atomicCAS(h.key + i, -1, c);
    if (cur == -1 || cur == c) {
      atomicAdd(h.sum + i, w);
      atomicMin(h.first + i, k);
      return true;
    }
  }
  return false;
}

__device__ int hash_find(const HashTab& h, int32_t c) {
  uint32_t i = hslot(c);
  for (int probe = 0; probe < kHashSlots; ++probe, i = (i + 1) & (kHashSlots - 1))
    if (h.key[i] == c) return (int)i;
  return -1;
}

template <bool DENSE, int G>
__device__ double delta_hashed(const NodalArgs& a, int v, int r, int s, HashTab h, int* flag,
                               const Group<G>& grp) {
  const int t = grp.rank();
  const Rows<DENSE> R(a, r, s);
  const int32_t o0 = a.optr[v], no = a.optr[v + 1] - o0;
  const int32_t i0 = a.iptr[v], ni = a.iptr[v + 1] - i0;
  uint32_t koR = 0, koS = 0, niR = 0, niS = 0;
  for (int k = t; k < no; k += G) {
    int32_t c = __ldg(a.part + __ldg(a.oidx + o0 + k));
    uint32_t w = __ldg(a.ow + o0 + k);
    koR += c == r ? w : 0u;
    koS += c == s ? w : 0u;
  }
  for (int k = t; k < ni; k += G) {
    int32_t c = __ldg(a.part + __ldg(a.iidx + i0 + k));
    uint32_t w = __ldg(a.iw + i0 + k);
    niR += c == r ? w : 0u;
    niS += c == s ? w : 0u;
  }
  koR = (uint32_t)grp.sum_ll(koR);
  koS = (uint32_t)grp.sum_ll(koS);
  niR = (uint32_t)grp.sum_ll(niR);
  niS = (uint32_t)grp.sum_ll(niS);
  Acc q;
  for (int dir = 0; dir < 2; ++dir) {
    const int32_t base = dir == 0 ? o0 : i0, n = dir == 0 ? no : ni;
    const int32_t* idx = dir == 0 ? a.oidx : a.iidx;
    const uint32_t* wt = dir == 0 ? a.ow : a.iw;
    uint32_t P = (uint32_t)((n + kHashSlots / 4 - 1) / (kHashSlots / 4));
    for (uint32_t pass = 0; pass < P; ++pass) {
      for (int i = t; i < kHashSlots; i += G) {
        h.key[i] = -1;
        h.sum[i] = 0u;
        h.first[i] = 0x7fffffff;
      }
      if (t == 0) *flag = 0;
      grp.sync();
      for (int k = t; k < n; k += G) {
        int32_t c = __ldg(a.part + __ldg(idx + base + k));
        if (hclass(c, P) == pass && !hash_add(h, c, __ldg(wt + base + k), k)) *flag = 1;
      }
      grp.sync();
      if (*flag) return __longlong_as_double(0x7ff8000000000000ll);  // table overflow
      for (int k = t; k < n; k += G) {
        int32_t c = __ldg(a.part + __ldg(idx + base + k));
        if (hclass(c, P) != pass) continue;
        int slot = hash_find(h, c);
        bool leader = h.first[slot] == k;
        uint32_t kc = h.sum[slot];
        uint32_t w = __ldg(wt + base + k);
        if (dir == 0) out_entry<DENSE>(a, R, r, s, niS, c, w, leader, kc, q);
        else in_entry<DENSE>(a, R, r, s, c, w, leader, kc, q);
      }
      grp.sync();
    }
  }
  reduce_acc(q, grp);
  return finish_delta<DENSE>(a, R, v, r, s, koR, koS, niR, niS, q);
}

// Neighbour of v whose running weight (out-entries, then in-entries) first
// exceeds t (choose_neighbored_node_block, kernels.hpp:877-939).
__device__ int32_t pick_neighbour(const NodalArgs& a, int v, uint64_t t, int lane) {
  const int32_t o0 = a.optr[v], no = a.optr[v + 1] - o0;
  const int32_t i0 = a.iptr[v], ni = a.iptr[v + 1] - i0;
  const int n = no + ni;
  uint64_t acc = 0;
  for (int k0 = 0; k0 < n; k0 += 32) {
    int k = k0 + lane;
    uint32_t w = 0;
    int32_t u = 0;
    if (k < n) {
      if (k < no) { w = __ldg(a.ow + o0 + k); u = __ldg(a.oidx + o0 + k); }
      else { w = __ldg(a.iw + i0 + k - no); u = __ldg(a.iidx + i0 + k - no); }
    }
    uint64_t incl = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    unsigned hit = __ballot_sync(kFull, k < n && acc + incl > t);
    if (hit) return __shfl_sync(kFull, u, __ffs(hit) - 1);
    acc += __shfl_sync(kFull, incl, 31);
  }
  return 0;
}

// Vertex and proposal of batch item i (computed by one warp).
template <bool GIVEN>
__device__ __forceinline__ void item(const NodalArgs& a, int i, int lane, int& v, int& s) {
  if (GIVEN) {
    v = a.verts[i];
    s = a.props_in[i];
    return;
  }
  v = a.lo + i;
  P4 x = draw(a.seed, kRngNodalVertex, a.seq, (uint32_t)v);
  int rnd = (int)(x.v[0] % (uint32_t)a.B);
  uint64_t deg = (uint64_t)a.kdo[v] + a.kdi[v];
  if (deg == 0) {
    s = rnd;
  } else {
    int32_t un = pick_neighbour(a, v, scale_draw(x.v[1], deg), lane);
    int32_t u = a.part[un];
    s = a.use_rand[u] ? rnd : a.nbr_s[u];
  }
}

__device__ __forceinline__ void write_result(const NodalArgs& a, bool given, int i, int r, int s,
                                             double d) {
  if (given) {
    a.dS_raw[i] = d;
  } else {
    bool acc = d < 0.0;
    a.newlab[i] = acc ? s : r;
    a.rec[i] = acc ? d : 0.0;
    if (a.props_out) a.props_out[i] = s;
  }
}

__device__ __forceinline__ bool is_heavy(int no, int ni) {
  return no > kWarpList || ni > kWarpList;
}

template <bool GIVEN, bool DENSE>
__global__ void __launch_bounds__(kNodalWarps * 32, 3) nodal_kernel(NodalArgs a) {
  __shared__ unsigned long long s_ko[kNodalWarps][kWarpList], s_ki[kNodalWarps][kWarpList];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = gridDim.x * kNodalWarps;
  Group<32> grp{nullptr};
  for (int i = blockIdx.x * kNodalWarps + wid; i < a.count; i += nw) {
    const int vv = GIVEN ? a.verts[i] : a.lo + i;
    const int32_t o0 = a.optr[vv], no = a.optr[vv + 1] - o0;
    const int32_t i0 = a.iptr[vv], ni = a.iptr[vv + 1] - i0;
    if (is_heavy(no, ni)) continue;  // the CTA kernel's
    int v, s;
    item<GIVEN>(a, i, lane, v, s);
    const int r = a.part[v];
    double d = 0.0;
    if (r != s) {
      if (no <= 32 && ni <= 32) {
        d = delta_registers<DENSE>(a, v, r, s, o0, no, i0, ni, lane);
      } else {
        stage_sorted<32>(a.oidx, a.ow, a.part, o0, no, s_ko[wid], grp);
        stage_sorted<32>(a.iidx, a.iw, a.part, i0, ni, s_ki[wid], grp);
        d = delta_sorted<DENSE, 32>(a, v, r, s, s_ko[wid], no, s_ki[wid], ni, grp);
      }
    }
    if (lane == 0) write_result(a, GIVEN, i, r, s, d);
    __syncwarp();
  }
}

// Vertices with more than kWarpList entries in a direction: one CTA each,
// lists sorted in shared memory up to kHeavyList entries, longer ones
// through the hashed passes.
template <bool GIVEN, bool DENSE>
__global__ void __launch_bounds__(kHeavyThreads, 2) nodal_heavy_kernel(NodalArgs a) {
  extern __shared__ unsigned long long hsm[];
  __shared__ double red[kHeavyThreads / 32];
  __shared__ int flag, sh_v, sh_s;
  Group<kHeavyThreads> grp{red};
  unsigned long long* ko = hsm;
  unsigned long long* ki = hsm + kHeavyList;
  HashTab ht{(int32_t*)hsm, (uint32_t*)hsm + kHashSlots, (int32_t*)hsm + 2 * kHashSlots};
  for (int h = blockIdx.x; h < a.nheavy; h += gridDim.x) {
    const int i = a.heavy[h];
    if (threadIdx.x < 32) {
      int v, s;
      item<GIVEN>(a, i, threadIdx.x, v, s);
      if (threadIdx.x == 0) {
        sh_v = v;
        sh_s = s;
      }
    }
    __syncthreads();
    const int v = sh_v, s = sh_s;
    const int r = a.part[v];
    const int32_t o0 = a.optr[v], no = a.optr[v + 1] - o0;
    const int32_t i0 = a.iptr[v], ni = a.iptr[v + 1] - i0;
    double d = 0.0;
    if (r != s) {
      if (no <= kHeavyList && ni <= kHeavyList) {
        stage_sorted<kHeavyThreads>(a.oidx, a.ow, a.part, o0, no, ko, grp);
        stage_sorted<kHeavyThreads>(a.iidx, a.iw, a.part, i0, ni, ki, grp);
        d = delta_sorted<DENSE, kHeavyThreads>(a, v, r, s, ko, no, ki, ni, grp);
      } else {
        d = delta_hashed<DENSE, kHeavyThreads>(a, v, r, s, ht, &flag, grp);
        if (threadIdx.x == 0 && d != d) atomicAdd(a.err, 1);
      }
    }
    if (threadIdx.x == 0) write_result(a, GIVEN, i, r, s, d);
    __syncthreads();
  }
}

// Applies the batch's labels and sums its recorded dS.  Each CTA sums a fixed
// slice in a fixed order into its own partial; the last CTA to finish (a
// ticket, no waiting) adds the partials in CTA order, so the result does
// not depend on scheduling.  In dense mode the CTAs also refresh the log2 of
// the block degrees that dense_update changed.
constexpr int kCommitThreads = 512;

__global__ void __launch_bounds__(kCommitThreads) commit_kernel(
    int32_t* part, int32_t lo, int32_t count, const int32_t* __restrict__ newlab,
    const double* __restrict__ rec, double* slot_sum, long long* slot_acc, int32_t B,
    const uint32_t* __restrict__ d_out, const uint32_t* __restrict__ d_in, double* ld_out,
    double* ld_in, double* part_sum, long long* part_cnt, unsigned* ticket) {
  __shared__ double sh[kCommitThreads];
  __shared__ long long shc[kCommitThreads];
  __shared__ bool last;
  const int tid = threadIdx.x;
  double s = 0.0;
  long long c = 0;
  for (int i = blockIdx.x * kCommitThreads + tid; i < count; i += gridDim.x * kCommitThreads) {
    int32_t nl = newlab[i];
    if (part[lo + i] != nl) {
      part[lo + i] = nl;
      ++c;
    }
    s += rec[i];
  }
  if (ld_out)
    for (int b = blockIdx.x * kCommitThreads + tid; b < B; b += gridDim.x * kCommitThreads) {
      ld_out[b] = log2((double)d_out[b]);
      ld_in[b] = log2((double)d_in[b]);
    }
  sh[tid] = s;
  shc[tid] = c;
  __syncthreads();
  for (int o = kCommitThreads / 2; o > 0; o >>= 1) {
    if (tid < o) {
      sh[tid] += sh[tid + o];
      shc[tid] += shc[tid + o];
    }
    __syncthreads();
  }
  if (tid == 0) {
    part_sum[blockIdx.x] = sh[0];
    part_cnt[blockIdx.x] = shc[0];
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && tid == 0) {
    __threadfence();
    double t = 0.0;
    long long n = 0;
    for (int k = 0; k < (int)gridDim.x; ++k) {
      t += ((volatile double*)part_sum)[k];
      n += ((volatile long long*)part_cnt)[k];
    }
    *slot_sum += t;
    *slot_acc += n;
    *ticket = 0u;
  }
}

NodalArgs make_args(const DevGraph& g, const int32_t* part, const DevBM& m, int32_t B,
                    const NodalAux& aux) {
  NodalArgs a{};
  a.xlx = m.xlx;
  a.optr = g.optr; a.oidx = g.oidx; a.iptr = g.iptr; a.iidx = g.iidx;
  a.ow = g.ow; a.iw = g.iw; a.kdo = g.kdo; a.kdi = g.kdi;
  a.part = part;
  a.bop = m.optr; a.boc = m.ocol; a.bip = m.iptr; a.bic = m.icol;
  a.bon = m.ocnt; a.bin = m.icnt; a.d_out = m.d_out; a.d_in = m.d_in;
  a.Md = m.Md; a.MTd = m.MTd;
  a.ld_out = m.ld_out; a.ld_in = m.ld_in; a.dSout = m.dSout; a.ambout = m.ambout;
  a.ambin = m.ambin; a.sinfull = m.sinfull; a.nbr_s = m.nbr_s; a.use_rand = m.use_rand;
  a.B = B;
  a.heavy = aux.heavy;
  a.nheavy = aux.nheavy;
  a.err = aux.err;
  return a;
}

int nodal_grid(int count) {
  int g = (count + kNodalWarps - 1) / kNodalWarps;
  return g < 1 ? 1 : (g > 148 * 64 ? 148 * 64 : g);
}

template <bool GIVEN, bool DENSE>
void launch_pair(const NodalArgs& a, const NodalAux& aux, cudaStream_t st) {
  if (a.nheavy > 0) {
    // heavy vertices on the side stream, next to the warp kernel
    cudaEventRecord(aux.fork, st);
    cudaStreamWaitEvent(aux.side, aux.fork, 0);
    ++g_launches;
    int grid = a.nheavy < 2 * 148 ? a.nheavy : 2 * 148;
    nodal_heavy_kernel<GIVEN, DENSE><<<grid, kHeavyThreads, kHeavySmem, aux.side>>>(a);
    cudaEventRecord(aux.join, aux.side);
  }
  ++g_launches;
  nodal_kernel<GIVEN, DENSE><<<nodal_grid(a.count), kNodalWarps * 32, 0, st>>>(a);
  if (a.nheavy > 0) cudaStreamWaitEvent(st, aux.join, 0);
}

}  // namespace

cudaError_t init_nodal_attributes() {
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* f) {
    cudaError_t x = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kHeavySmem);
    if (x != cudaSuccess) e = x;
  };
  set((const void*)nodal_heavy_kernel<false, false>);
  set((const void*)nodal_heavy_kernel<false, true>);
  set((const void*)nodal_heavy_kernel<true, false>);
  set((const void*)nodal_heavy_kernel<true, true>);
  return e;
}

int nodal_heavy_threshold() { return kWarpList; }

void nodal_batch_sample(const DevGraph& g, const int32_t* part, const DevBM& m, int32_t B,
                        bool dense, uint64_t seed, uint32_t seq, int32_t lo, int32_t count,
                        int32_t* newlab, double* rec, int32_t* props, const NodalAux& aux,
                        cudaStream_t st) {
  NodalArgs a = make_args(g, part, m, B, aux);
  a.seed = seed;
  a.seq = seq;
  a.lo = lo;
  a.count = count;
  a.newlab = newlab;
  a.rec = rec;
  a.props_out = props;
  if (count <= 0) return;
  if (dense) launch_pair<false, true>(a, aux, st);
  else launch_pair<false, false>(a, aux, st);
}

void nodal_delta_given(const DevGraph& g, const int32_t* part, const DevBM& m, int32_t B,
                       bool dense, int32_t nv, const int32_t* verts, const int32_t* props,
                       double* dS, const NodalAux& aux, cudaStream_t st) {
  NodalArgs a = make_args(g, part, m, B, aux);
  a.count = nv;
  a.verts = verts;
  a.props_in = props;
  a.dS_raw = dS;
  if (nv <= 0) return;
  if (dense) launch_pair<true, true>(a, aux, st);
  else launch_pair<true, false>(a, aux, st);
}

void nodal_commit(int32_t* part, int32_t lo, int32_t count, const int32_t* newlab,
                  const double* rec, double* slot_sum, long long* slot_acc, const DevBM* dense_m,
                  int32_t B, const CommitScratch& cs, cudaStream_t st) {
  ++g_launches;
  commit_kernel<<<kCommitCtas, kCommitThreads, 0, st>>>(
      part, lo, count, newlab, rec, slot_sum, slot_acc, dense_m ? B : 0,
      dense_m ? dense_m->d_out : nullptr, dense_m ? dense_m->d_in : nullptr,
      dense_m ? dense_m->ld_out : nullptr, dense_m ? dense_m->ld_in : nullptr, cs.part_sum,
      cs.part_cnt, cs.ticket);
}

}  // namespace sbp
