// Nodal batch: proposal, dS and accept for each vertex of a Jacobi batch.
//
// GSAP spends ~25 launches and two bb_segsorts of all E neighbour-block lists
// per batch (partition.hpp:456-662); each of its seven dS kernels has one
// thread walk a whole blockmodel row in a serial sorted merge with the
// vertex's sorted neighbour-block list (kernels.hpp:494-597, 1153-1726).
//
// Here a group of threads owns one vertex: half a warp for vertices of at
// most kSmallEntries neighbour entries (two per warp), a warp for the other
// ordinary vertices, a whole CTA for the few with more than kWarpList
// neighbours in a direction (run on a second stream next to the warp
// kernel).  The host sorts each batch's vertices into these three lists
// once per job.
//   * proposal: Philox draws, an exact integer inverse-CDF pick of a
//     neighbour (a prefix scan over the group's lanes, out- then
//     in-entries), then the per-block draws of the batch
//     (kernels.hpp:877-1032);
//   * neighbour blocks grouped per distinct block: in registers with
//     __match_any_sync / __reduce_add_sync when a list fits the lane group,
//     else in a per-warp shared-memory hash table (up to kWarpHashEntries),
//     else sorted in shared memory (bitonic), else hashed in shared memory in
//     passes; GSAP sorts all E entries every batch;
//   * dS: GSAP's seven terms rewritten as "changed cells + row degrees".
//     A row term  sum_c f(x_c)  with  f(x) = x (log2 x - log2 dcol[c] - L)
//     splits into  sum_c (x log2 x - x log2 dcol[c])  -  L * sum_c x ;
//     between the old and the new rows the first sums over unchanged columns
//     cancel, so only the columns the vertex touches and the four rows'
//     degree terms remain (see Acc below).  Counts come from the dense B x B
//     form (small B, O(1)) or by binary search in the CSR rows.
//     Quirks of the reference kept: old column degrees (Q2), one term per
//     list entry for blocks missing from the target row
//     (kernels.hpp:1648-1652, 1314-1318), the r/s in-weight corrections and
//     the conditional extra column term (kernels.hpp:1506-1510, 1573-1578,
//     1663-1669, 1718-1723), unsigned count arithmetic.
//   * accept iff dS < 0 (kernels.hpp:634-640), or by the general-mode rules
//     (exact MDL, Metropolis-Hastings) below; the new label goes to a side
//     buffer so every vertex of the batch sees the same old labels.
// All entropy arithmetic is FP64.
#include "common.cuh"
#include "kernels.h"
#include "multi.cuh"
#include "dense.cuh"

namespace sbp {

namespace {

constexpr int kNodalWarps = 4;
constexpr int kWarpList = 128;     // entries per direction a warp sorts in shared memory
constexpr int kHeavyThreads = 256;
constexpr int kHashSlotsCfg = 8192;
// the heavy path's hash table: key, sum, first
constexpr size_t kHeavySmem = 3 * kHashSlotsCfg * sizeof(int32_t);

struct NodalArgs {
  const double* xlx;        // x log2 x table
  const int32_t *optr, *oidx, *iptr, *iidx;
  const uint32_t *ow, *iw, *kdo, *kdi;
  const int32_t* part;
  const int32_t *bop, *boc, *bip, *bic;
  const uint32_t *bon, *bin, *d_out, *d_in;
  const uint32_t *Md, *MTd;
  const double *ld_out, *ld_in;
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
  const int32_t *small, *mid;  // batch indices of the warp kernel: two small ones per warp,
  int32_t nsmall, nmid;        // one mid one per warp
  int32_t* err;             // error counter (hash table overflow)
  const int32_t* ctl;       // sweep control: gate, and seq += ctl[0] * seq_mul
  uint32_t seq_mul;
  // general-mode kernels only (ScoreMode)
  int32_t exact, mh;
  double beta;
  double* logH_raw;         // given mode: log Hastings ratio of each move
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
  __device__ __forceinline__ uint32_t out_at(bool row_s, int c) const {
    return row_lookup(oc, on, row_s ? sO0 : rO0, row_s ? sO1 : rO1, c);
  }
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
  __device__ __forceinline__ uint32_t out_at(bool row_s, int c) const {
    return __ldg((row_s ? ors : orr) + c);
  }
};

// Per-thread partial of a move's dS.  GSAP's seven terms (kernels.hpp:143-182,
// 494-597, 1153-1726) combine, after the per-block row sums cancel, into
//   dS = - sum_X d_X log2 d_X  +  sum_X L_X mass_X
//        - sum over changed cells (g(new) - g(old))  + corner cells
// where X runs over the old/new out- and in-rows of r and s, d_X the old row
// degree, L_X = log2 of the new row degree and mass_X the new row's total
// count; g(x, a) = x log2 x - x a with a = log2 of the old column degree (Q2).
// `acc` collects this thread's terms, m4..m7 the count changes of the new
// out-row r, out-row s, in-row r and in-row s.
struct Acc {
  double acc = 0.0;
  int m4 = 0, m5 = 0, m6 = 0, m7 = 0;
};

// One neighbour entry of v (block c, weight w) in direction `in` (false =
// out-edge, true = in-edge); `leader` marks one entry per distinct block of
// that direction and kc is v's total weight to/from c
// (kernels.hpp:1444-1726 for out, 1153-1362 for in).
template <bool DENSE>
__device__ __forceinline__ void entry(const NodalArgs& a, const Rows<DENSE>& R, int r, int s,
                                      uint32_t niS, bool in, int32_t c, uint32_t w, bool leader,
                                      uint32_t kc, Acc& q) {
  if (in && (c == r || c == s)) return;  // in-rows leave out blocks r and s
  const double ldc = in ? a.ld_out[c] : a.ld_in[c];
  const uint32_t Mt = in ? R.in_s(c) : R.out_s(c);
  int dmo = 0, dmt = 0;
  if (leader && c != r && c != s) {
    const uint32_t Mo = in ? R.in_r(c) : R.out_r(c);
    const uint32_t x = Mo - kc;
    q.acc -= gterm(a.xlx, x, ldc) - gterm(a.xlx, Mo, ldc);
    dmo = (int)((long long)x - (long long)Mo);
    if (Mt != 0u) {
      const uint32_t y = Mt + kc;
      q.acc -= gterm(a.xlx, y, ldc) - gterm(a.xlx, Mt, ldc);
      dmt = (int)((long long)y - (long long)Mt);
    }
  }
  if (Mt == 0u) {
    // block c absent from the target row: one term per list entry
    // (kernels.hpp:1648-1652, 1696-1713; 1314-1318, 1348-1358)
    const uint32_t y = in ? w : w - (c == r ? niS : 0u) + (c == s ? niS : 0u);
    q.acc -= gterm(a.xlx, y, ldc);
    dmt += (int)y;
  }
  if (in) {
    q.m6 += dmo;
    q.m7 += dmt;
  } else {
    q.m4 += dmo;
    q.m5 += dmt;
  }
}

// Adds the corner cells (r,r), (r,s), (s,r), (s,s) of M and the row-degree
// terms to lanes 0..12 of the calling lane group (lane `lane` of the group
// starting at warp lane hb; a warp, or a half-warp with its own vertex; call
// it from one warp of a CTA group, after m4..m7 hold the group totals).
// kernels.hpp:1506-1510, 1573-1578, 1663-1669, 1718-1723 give the new
// corner counts.
template <bool DENSE>
__device__ __forceinline__ void corner_terms(const NodalArgs& a, const Rows<DENSE>& R, int v,
                                             int r, int s, uint32_t koR, uint32_t koS,
                                             uint32_t niR, uint32_t niS, Acc& q, int lane,
                                             int hb) {
  // lane 0: M[r][r], 1: M[r][s], 2: M[s][r], 3: M[s][s]
  const uint32_t mm = lane < 4 ? R.out_at((lane & 2) != 0, (lane & 1) ? s : r) : 0u;
  const uint32_t Mrr = __shfl_sync(kFull, mm, hb), Mrs = __shfl_sync(kFull, mm, hb + 1);
  const uint32_t Msr = __shfl_sync(kFull, mm, hb + 2), Mss = __shfl_sync(kFull, mm, hb + 3);
  const uint32_t xrr = Mrr - koR - niR;
  const uint32_t xrs = Mrs != 0u ? Mrs - koS + niR : niR;
  const uint32_t xsr = Msr + koR - niS;
  const uint32_t xss = Mss != 0u ? Mss + koS + niS : niS;
  const bool use_rs = Mrs != 0u || niR > 0u;                       // cell or extra term
  const bool use_ss = Mss != 0u || (koS == 0u && niS > 0u);
  const long long m4 = q.m4 + (Mrr ? (long long)xrr - Mrr : 0) +
                       (use_rs ? (long long)xrs - (long long)Mrs : 0);
  const long long m5 = q.m5 + (Msr ? (long long)xsr - Msr : 0) +
                       (use_ss ? (long long)xss - (long long)Mss : 0);
  const uint32_t kO = a.kdo[v], kI = a.kdi[v];
  const uint32_t dor = a.d_out[r], dos = a.d_out[s], dir = a.d_in[r], dis = a.d_in[s];
  const long long mass4 = (long long)dor + m4;
  const long long mass5 = (long long)dos + m5;
  const long long mass6 = (long long)dir - (long long)Mrr - (long long)Msr + q.m6;
  const long long mass7 = (long long)dis - (long long)Mrs - (long long)Mss + q.m7;
  const double ldi_r = a.ld_in[r], ldi_s = a.ld_in[s];
  const double ldo_r = a.ld_out[r], ldo_s = a.ld_out[s];
  // Straight-line, no lane branches: every lane evaluates the cell form and
  // the row form of its operands and keeps the one its lane range owns.
  // lanes 0-3: old corner cells, + M log2 M; lanes 4-7: new corner cells,
  // - g(x); lanes 8-11: + L mass of the four new rows; lane 12: the old row
  // degrees.
  const int j = lane & 3;
  const uint32_t Mold = j == 0 ? Mrr : j == 1 ? Mrs : j == 2 ? Msr : Mss;
  const uint32_t xnew = j == 0 ? xrr : j == 1 ? xrs : j == 2 ? xsr : xss;
  const bool on = j == 0 ? Mrr != 0u : j == 1 ? use_rs : j == 2 ? Msr != 0u : use_ss;
  const double ld = (j & 1) ? ldi_s : ldi_r;
  const bool old_cell = lane < 4;
  const uint32_t X = old_cell ? Mold : xnew;
  const bool cell_on = old_cell ? Mold != 0u : on;
  const double cell = old_cell ? xlx(a.xlx, X) : -gterm(a.xlx, X, ld);
  const long long mass = j == 0 ? mass4 : j == 1 ? mass5 : j == 2 ? mass6 : mass7;
  const uint32_t d = j == 0 ? dor - kO : j == 1 ? dos + kO : j == 2 ? dir - kI : dis + kI;
  const double row = mass != 0 ? l2x(a.xlx, d) * (double)mass : 0.0;
  const double deg = -((dor ? (double)dor * ldo_r : 0.0) + (dos ? (double)dos * ldo_s : 0.0) +
                       (dir ? (double)dir * ldi_r : 0.0) + (dis ? (double)dis * ldi_s : 0.0));
  double t = 0.0;
  if (lane < 8) t = cell_on ? cell : 0.0;
  else if (lane < 12) t = row;
  else if (lane == 12) t = deg;
  q.acc += t;
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

// Group sums of the four direction weights v has to/from blocks r and s.
struct RsWeights {
  uint32_t koR, koS, niR, niS;
};

// Finishes a move's dS after every thread of the group has added its
// entries to q: group totals of the count changes, then the corner and
// degree terms on warp 0, then the group sum.
template <bool DENSE, int G>
__device__ double finish(const NodalArgs& a, const Rows<DENSE>& R, int v, int r, int s,
                         const RsWeights& w, Acc q, const Group<G>& grp) {
  q.m4 = (int)grp.sum_ll(q.m4);
  q.m5 = (int)grp.sum_ll(q.m5);
  q.m6 = (int)grp.sum_ll(q.m6);
  q.m7 = (int)grp.sum_ll(q.m7);
  if (G == 32 || threadIdx.x < 32)
    corner_terms<DENSE>(a, R, v, r, s, w.koR, w.koS, w.niR, w.niS, q, threadIdx.x & 31, 0);
  return grp.sum(q.acc);
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
  RsWeights w{(uint32_t)grp.sum_ll(koR), (uint32_t)grp.sum_ll(koS), (uint32_t)grp.sum_ll(niR),
              (uint32_t)grp.sum_ll(niS)};
  Acc q;
  for (int k = t; k < no; k += G) {
    const int32_t c = kblk(ko[k]);
    const bool leader = k == 0 || kblk(ko[k - 1]) != c;
    uint32_t kc = 0;
    if (leader)
      for (int j = k; j < no && kblk(ko[j]) == c; ++j) kc += kwt(ko[j]);
    entry<DENSE>(a, R, r, s, w.niS, false, c, kwt(ko[k]), leader, kc, q);
  }
  for (int k = t; k < ni; k += G) {
    const int32_t c = kblk(ki[k]);
    const bool leader = k == 0 || kblk(ki[k - 1]) != c;
    uint32_t kc = 0;
    if (leader)
      for (int j = k; j < ni && kblk(ki[j]) == c; ++j) kc += kwt(ki[j]);
    entry<DENSE>(a, R, r, s, w.niS, true, c, kwt(ki[k]), leader, kc, q);
  }
  return finish<DENSE, G>(a, R, v, r, s, w, q, grp);
}

// dS from the warp's entries, one per lane and pass (see delta_registers).
template <bool DENSE>
__device__ __forceinline__ double delta_from_entries(const NodalArgs& a, const Rows<DENSE>& R,
                                                     int v, int r, int s, int passes,
                                                     const int32_t* cs, const uint32_t* ws,
                                                     const bool* ins, const bool* valid,
                                                     int lane) {
  Acc q;
  RsWeights w{0u, 0u, 0u, 0u};
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    if (passes == 1 && p == 1) break;
    const bool o = valid[p] && !ins[p], i = valid[p] && ins[p];
    w.koR += __reduce_add_sync(kFull, o && cs[p] == r ? ws[p] : 0u);
    w.koS += __reduce_add_sync(kFull, o && cs[p] == s ? ws[p] : 0u);
    w.niR += __reduce_add_sync(kFull, i && cs[p] == r ? ws[p] : 0u);
    w.niS += __reduce_add_sync(kFull, i && cs[p] == s ? ws[p] : 0u);
  }
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    if (passes == 1 && p == 1) break;
    // direction in the top bit, unique keys for idle lanes
    const unsigned key = valid[p] ? ((unsigned)cs[p] | (ins[p] ? 0x80000000u : 0u))
                                  : (0x7fffffe0u + (unsigned)lane);
    const unsigned peers = __match_any_sync(kFull, key);
    const uint32_t kc = __reduce_add_sync(peers, ws[p]);
    if (valid[p])
      entry<DENSE>(a, R, r, s, w.niS, ins[p], cs[p], ws[p], lane == __ffs(peers) - 1, kc, q);
  }
  q.m4 = __reduce_add_sync(kFull, q.m4);
  q.m5 = __reduce_add_sync(kFull, q.m5);
  q.m6 = __reduce_add_sync(kFull, q.m6);
  q.m7 = __reduce_add_sync(kFull, q.m7);
  corner_terms<DENSE>(a, R, v, r, s, w.koR, w.koS, w.niR, w.niS, q, lane, 0);
  return warp_sum(q.acc);
}

// dS when each direction's list fits in one warp: entries of the same block
// are grouped with __match_any_sync on a direction-tagged key and their
// weights summed with __reduce_add_sync.  When both lists fit together,
// one pass covers both directions.
template <bool DENSE>
__device__ double delta_registers(const NodalArgs& a, int v, int r, int s, int32_t o0, int no,
                                  int32_t i0, int ni, int lane) {
  const Rows<DENSE> R(a, r, s);
  const int passes = no + ni <= 32 ? 1 : 2;
  // pass p, lane l: entry index e; combined pass: out-entries then in-entries
  int32_t cs[2];
  uint32_t ws[2];
  bool ins[2], valid[2];
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    int k;
    bool in;
    if (passes == 1 && p == 1) {
      valid[1] = false;
      ins[1] = false;
      cs[1] = -1;
      ws[1] = 0u;
      break;
    }
    if (passes == 1) {
      in = lane >= no;
      k = in ? lane - no : lane;
      valid[p] = p == 0 && lane < no + ni;
    } else {
      in = p == 1;
      k = lane;
      valid[p] = lane < (in ? ni : no);
    }
    ins[p] = in;
    cs[p] = -1;
    ws[p] = 0u;
    if (valid[p]) {
      cs[p] = in ? __ldg(a.part + __ldg(a.iidx + i0 + k)) : __ldg(a.part + __ldg(a.oidx + o0 + k));
      ws[p] = in ? __ldg(a.iw + i0 + k) : __ldg(a.ow + o0 + k);
    }
  }
  return delta_from_entries<DENSE>(a, R, v, r, s, passes, cs, ws, ins, valid, lane);
}


// Lists of more than kWarpList entries: per-block totals from a shared-memory
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
        entry<DENSE>(a, R, r, s, niS, dir == 1, c, w, leader, kc, q);
      }
      grp.sync();
    }
  }
  return finish<DENSE, G>(a, R, v, r, s, RsWeights{koR, koS, niR, niS}, q, grp);
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
// u2 = the vertex's third draw (the Metropolis-Hastings uniform).
template <bool GIVEN>
__device__ __forceinline__ void item(const NodalArgs& a, int i, int lane, int& v, int& s,
                                     uint32_t& u2) {
  if (GIVEN) {
    v = a.verts[i];
    s = a.props_in[i];
    u2 = 0u;
    return;
  }
  v = a.lo + i;
  P4 x = draw(a.seed, kRngNodalVertex, a.seq + ctl_itr(a.ctl) * a.seq_mul, (uint32_t)v);
  u2 = x.v[2];
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

// Sum over a lane group of W lanes (32: the warp, 16: each half-warp).
template <int W>
__device__ __forceinline__ double group_sum(double x) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}

// dS of a vertex whose entries fit one lane group of W lanes (entry c, wt,
// direction `in` on lane hl of the group; delta_from_entries for one pass).
// The group's masks keep the two half-warps' vertices apart.
template <bool DENSE, int W>
__device__ __forceinline__ double delta_group(const NodalArgs& a, const Rows<DENSE>& R, int v,
                                              int r, int s, int32_t c, uint32_t wt, bool in,
                                              bool valid, int lane) {
  const int hl = lane & (W - 1), hb = lane & (32 - W);
  const unsigned gm = W == 32 ? kFull : (0xFFFFu << hb);
  const bool o = valid && !in, i = valid && in;
  RsWeights w;
  w.koR = __reduce_add_sync(gm, o && c == r ? wt : 0u);
  w.koS = __reduce_add_sync(gm, o && c == s ? wt : 0u);
  w.niR = __reduce_add_sync(gm, i && c == r ? wt : 0u);
  w.niS = __reduce_add_sync(gm, i && c == s ? wt : 0u);
  // direction in the top bit, unique keys for idle lanes
  const unsigned key = valid ? ((unsigned)c | (in ? 0x80000000u : 0u)) : (0x7fffffe0u + (unsigned)lane);
  const unsigned peers = __match_any_sync(gm, key);
  const uint32_t kc = __reduce_add_sync(peers, wt);
  Acc q;
  if (valid) entry<DENSE>(a, R, r, s, w.niS, in, c, wt, lane == __ffs(peers) - 1, kc, q);
  q.m4 = __reduce_add_sync(gm, q.m4);
  q.m5 = __reduce_add_sync(gm, q.m5);
  q.m6 = __reduce_add_sync(gm, q.m6);
  q.m7 = __reduce_add_sync(gm, q.m7);
  corner_terms<DENSE>(a, R, v, r, s, w.koR, w.koS, w.niR, w.niS, q, hl, hb);
  return group_sum<W>(q.acc);
}

// Proposal, dS and accept of batch vertex i when its entries fit one lane
// group of W lanes: one entry per lane, loaded once for the neighbour pick
// (out- then in-entries, pick_neighbour's order) and for the dS.  With
// W = 16 each half-warp takes a vertex of at most 16 entries; both halves
// run every warp-wide step, and a half without a vertex of its own
// (active = false) repeats its partner's and writes nothing.
template <bool DENSE, int W>
__device__ __forceinline__ void fused_group(const NodalArgs& a, int i, bool active, int lane) {
  const int hl = lane & (W - 1), hb = lane & (32 - W);
  const unsigned gm = W == 32 ? kFull : (0xFFFFu << hb);
  const int v = a.lo + i;
  const int32_t o0 = a.optr[v], no = a.optr[v + 1] - o0;
  const int32_t i0 = a.iptr[v], ni = a.iptr[v + 1] - i0;
  const P4 x = draw(a.seed, kRngNodalVertex, a.seq + ctl_itr(a.ctl) * a.seq_mul, (uint32_t)v);
  const int rnd = (int)(x.v[0] % (uint32_t)a.B);
  const bool in = hl >= no;
  const bool valid = hl < no + ni;
  const int k = in ? hl - no : hl;
  int32_t c = -1;
  uint32_t w = 0u;
  if (valid) {
    const int32_t u = in ? __ldg(a.iidx + i0 + k) : __ldg(a.oidx + o0 + k);
    w = in ? __ldg(a.iw + i0 + k) : __ldg(a.ow + o0 + k);
    c = __ldg(a.part + u);
  }
  const int r = a.part[v];
  const uint64_t deg = (uint64_t)a.kdo[v] + a.kdi[v];
  const uint64_t t = scale_draw(x.v[1], deg);
  uint64_t incl = w;
#pragma unroll
  for (int o = 1; o < W; o <<= 1) {
    const uint64_t y = __shfl_up_sync(kFull, incl, o);
    if (hl >= o) incl += y;
  }
  const unsigned hit = __ballot_sync(kFull, valid && incl > t) & gm;
  const int ch = __shfl_sync(kFull, c, hit ? __ffs(hit) - 1 : lane);
  int s = rnd;
  if (deg != 0) {
    const int cu = hit ? ch : a.part[0];
    s = a.use_rand[cu] ? rnd : a.nbr_s[cu];
  }
  double d = 0.0;
  if (__any_sync(kFull, r != s)) {
    const Rows<DENSE> R(a, r, s);
    d = delta_group<DENSE, W>(a, R, v, r, s, c, w, in, valid, lane);
  }
  if (hl == 0 && active) write_result(a, false, i, r, s, r != s ? d : 0.0);
  __syncwarp();
}


// ------------------------------------------------------------ general mode --
// Kernels instantiated with GEN = true score a move by the exact change of
// the MDL (exact = 1) or by GSAP's terms (exact = 0), and accept it by
// Metropolis-Hastings (mh = 1) or iff dS < 0.
//
// Exact dS.  S = model - data_S with
//   data_S = sum_cells M log2 M - sum_rows d_out log2 d_out - sum_cols d_in log2 d_in
// and the model term fixed while B is.  Moving v from r to s, with kout[c]
// and kin[c] v's weight to and from block c (self loops of weight `self`
// apart), moves kout[c] from cell (r,c) to (s,c) and kin[c] from (c,r) to
// (c,s) for every c other than r and s, changes the four corner cells as in
// corner_exact, and moves v's out- and in-degree between the rows and
// columns r and s; dS = -(change of data_S).  Only those cells and four
// degrees enter, each as x log2 x.
//
// Hastings ratio of GSAP's proposal (kernels.hpp:877-1032): v picks an
// incident edge with probability proportional to its weight, the edge's
// other end lies in block t, and s is proposed with probability
// (M_ts + M_st + 1) / (d_t + B), d_t = d_out[t] + d_in[t], so
//   p(r -> s) = sum_t k_t (M_ts + M_st + 1) / (d_t + B) / k_v
// with k_t v's weight to and from t (a self loop counts in both directions)
// and k_v the sum of the k_t.  The reverse move reads the blockmodel after
// the move, in which the self loops sit in block s.  A move is accepted when
//   u < 2^(-beta dS) p(s -> r) / p(r -> s)
// with u the vertex's third draw scaled to [0, 1).

struct Hast {
  double f = 0.0, b = 0.0;  // forward and reverse proposal weights (k_v times p)
};

// Exact dS of the off-corner cells of one neighbour block c (direction
// `in`, v's total weight kc to or from c, counted once per block).
template <bool DENSE>
__device__ __forceinline__ void entry_exact(const NodalArgs& a, const Rows<DENSE>& R, int r, int s,
                                            bool in, int32_t c, bool leader, uint32_t kc,
                                            Acc& q) {
  if (!leader || c == r || c == s) return;
  const uint32_t Mo = in ? R.in_r(c) : R.out_r(c);
  const uint32_t Mt = in ? R.in_s(c) : R.out_s(c);
  q.acc += xlx(a.xlx, Mo) - xlx(a.xlx, Mo - kc) + xlx(a.xlx, Mt) - xlx(a.xlx, Mt + kc);
}

// Corner cells and the four degrees of the exact dS, on lanes 0..15 of the
// calling warp: lanes 0-3 the old cells (r,r), (r,s), (s,r), (s,s), lanes
// 4-7 the same cells after the move, lanes 8-11 the new degrees d_out[r],
// d_out[s], d_in[r], d_in[s], lanes 12-15 the old ones.  koR..niS include
// the self loops (their other end is in r).
template <bool DENSE>
__device__ __forceinline__ void corner_exact(const NodalArgs& a, const Rows<DENSE>& R, int v,
                                             int r, int s, const RsWeights& w, uint32_t self,
                                             Acc& q) {
  const int lane = threadIdx.x & 31;
  if (lane >= 16) return;
  const int j = lane & 3;
  double t;
  if (lane < 8) {
    const uint32_t M = R.out_at((j & 2) != 0, (j & 1) ? s : r);
    // unsigned wrap-around in the middle is fine: the results are >= 0
    const uint32_t x = j == 0   ? M - w.koR - w.niR + self
                       : j == 1 ? M - w.koS + (w.niR - self)
                       : j == 2 ? M + (w.koR - self) - w.niS
                                : M + w.koS + w.niS + self;
    t = lane < 4 ? xlx(a.xlx, M) : -xlx(a.xlx, x);
  } else {
    const uint32_t kO = a.kdo[v], kI = a.kdi[v];
    const uint32_t d0 = j == 0 ? a.d_out[r] : j == 1 ? a.d_out[s] : j == 2 ? a.d_in[r] : a.d_in[s];
    const uint32_t d1 = j == 0 ? d0 - kO : j == 1 ? d0 + kO : j == 2 ? d0 - kI : d0 + kI;
    t = lane < 12 ? xlx(a.xlx, d1) : -xlx(a.xlx, d0);
  }
  q.acc += t;
}

// Proposal weights of a neighbour block t other than r and s, kt = v's
// weight to and from t.
template <bool DENSE>
__device__ __forceinline__ void hast_block(const NodalArgs& a, const Rows<DENSE>& R, int32_t t,
                                           uint32_t kt, Hast& h) {
  const double D = (double)a.d_out[t] + (double)a.d_in[t] + (double)a.B;
  const double k = (double)kt;
  h.f += k * ((double)R.in_s(t) + (double)R.out_s(t) + 1.0) / D;
  h.b += k * ((double)R.in_r(t) + (double)R.out_r(t) - k + 1.0) / D;
}

// Proposal weights of blocks r and s (one thread of the group).
template <bool DENSE>
__device__ __forceinline__ void hast_rs(const NodalArgs& a, const Rows<DENSE>& R, int v, int r,
                                        int s, const RsWeights& w, uint32_t self, Hast& h) {
  const uint32_t Mrr = R.out_at(false, r), Mrs = R.out_at(false, s);
  const uint32_t Msr = R.out_at(true, r), Mss = R.out_at(true, s);
  const uint32_t xrr = Mrr - w.koR - w.niR + self;
  const uint32_t xrs = Mrs - w.koS + (w.niR - self);
  const uint32_t xsr = Msr + (w.koR - self) - w.niS;
  const double kv = (double)a.kdo[v] + (double)a.kdi[v], Bd = (double)a.B;
  const double Dr = (double)a.d_out[r] + (double)a.d_in[r];
  const double Ds = (double)a.d_out[s] + (double)a.d_in[s];
  const double kr = (double)w.koR + (double)w.niR, ks = (double)w.koS + (double)w.niS;
  const double sl = 2.0 * (double)self;
  h.f += kr * ((double)Mrs + (double)Msr + 1.0) / (Dr + Bd);
  h.f += ks * ((double)Mss + (double)Mss + 1.0) / (Ds + Bd);
  h.b += (kr - sl) * ((double)xrr + (double)xrr + 1.0) / (Dr - kv + Bd);
  h.b += (ks + sl) * ((double)xsr + (double)xrs + 1.0) / (Ds + kv + Bd);
}

// v's self-loop weight (group sum over its out-list).
template <int G>
__device__ uint32_t self_weight(const NodalArgs& a, int v, const Group<G>& grp) {
  const int32_t o0 = a.optr[v], no = a.optr[v + 1] - o0;
  uint32_t t = 0u;
  for (int k = grp.rank(); k < no; k += G)
    if (__ldg(a.oidx + o0 + k) == v) t += __ldg(a.ow + o0 + k);
  return (uint32_t)grp.sum_ll(t);
}

// Group totals, then the corner terms (exact or GSAP's) on warp 0, then the
// sums of dS and of the proposal weights.
template <bool DENSE, int G>
__device__ double finish_gen(const NodalArgs& a, const Rows<DENSE>& R, int v, int r, int s,
                             const RsWeights& w, uint32_t self, Acc q, Hast h,
                             const Group<G>& grp, double& logH) {
  if (a.exact) {
    if (G == 32 || threadIdx.x < 32) corner_exact<DENSE>(a, R, v, r, s, w, self, q);
  } else {
    q.m4 = (int)grp.sum_ll(q.m4);
    q.m5 = (int)grp.sum_ll(q.m5);
    q.m6 = (int)grp.sum_ll(q.m6);
    q.m7 = (int)grp.sum_ll(q.m7);
    if (G == 32 || threadIdx.x < 32)
      corner_terms<DENSE>(a, R, v, r, s, w.koR, w.koS, w.niR, w.niS, q, threadIdx.x & 31, 0);
  }
  logH = 0.0;
  if (a.mh) {
    const double f = grp.sum(h.f), b = grp.sum(h.b);
    if ((uint64_t)a.kdo[v] + a.kdi[v] != 0u) logH = log(b) - log(f);
  }
  return grp.sum(q.acc);
}

// Both lists fit one warp together: lane l holds entry l (out-entries,
// then in-entries).
template <bool DENSE>
__device__ double delta_registers_gen(const NodalArgs& a, int v, int r, int s, int32_t o0, int no,
                                      int32_t i0, int ni, int lane, double& logH) {
  const Rows<DENSE> R(a, r, s);
  const bool in = lane >= no, valid = lane < no + ni;
  const int k = in ? lane - no : lane;
  int32_t c = -1;
  uint32_t w = 0u, selfp = 0u;
  if (valid) {
    const int32_t u = in ? __ldg(a.iidx + i0 + k) : __ldg(a.oidx + o0 + k);
    w = in ? __ldg(a.iw + i0 + k) : __ldg(a.ow + o0 + k);
    c = __ldg(a.part + u);
    if (!in && u == v) selfp = w;
  }
  RsWeights rw;
  rw.koR = __reduce_add_sync(kFull, valid && !in && c == r ? w : 0u);
  rw.koS = __reduce_add_sync(kFull, valid && !in && c == s ? w : 0u);
  rw.niR = __reduce_add_sync(kFull, valid && in && c == r ? w : 0u);
  rw.niS = __reduce_add_sync(kFull, valid && in && c == s ? w : 0u);
  const uint32_t self = __reduce_add_sync(kFull, selfp);
  Acc q;
  const unsigned key = valid ? ((unsigned)c | (in ? 0x80000000u : 0u)) : (0x7fffffe0u + (unsigned)lane);
  const unsigned peers = __match_any_sync(kFull, key);
  const uint32_t kc = __reduce_add_sync(peers, w);
  const bool leader = lane == __ffs(peers) - 1;
  if (valid) {
    if (a.exact) entry_exact<DENSE>(a, R, r, s, in, c, leader, kc, q);
    else entry<DENSE>(a, R, r, s, rw.niS, in, c, w, leader, kc, q);
  }
  Hast h;
  if (a.mh) {
    // per block over both directions
    const unsigned pa = __match_any_sync(kFull, valid ? (unsigned)c : 0x7fffffe0u + (unsigned)lane);
    const uint32_t kt = __reduce_add_sync(pa, w);
    if (valid && lane == __ffs(pa) - 1 && c != r && c != s) hast_block<DENSE>(a, R, c, kt, h);
    if (lane == 0) hast_rs<DENSE>(a, R, v, r, s, rw, self, h);
  }
  return finish_gen<DENSE, 32>(a, R, v, r, s, rw, self, q, h, Group<32>{nullptr}, logH);
}

// Weight of block c's run in a sorted list; false when c is absent.
__device__ __forceinline__ bool run_weight(const unsigned long long* key, int n, int32_t c,
                                           uint32_t& w) {
  const unsigned long long k0 = (unsigned long long)(uint32_t)c << 32;
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (key[mid] < k0) lo = mid + 1;
    else hi = mid;
  }
  w = 0u;
  const bool found = lo < n && kblk(key[lo]) == c;
  for (; lo < n && kblk(key[lo]) == c; ++lo) w += kwt(key[lo]);
  return found;
}

template <bool DENSE, int G>
__device__ double delta_sorted_gen(const NodalArgs& a, int v, int r, int s,
                                   const unsigned long long* ko, int no,
                                   const unsigned long long* ki, int ni, const Group<G>& grp,
                                   double& logH) {
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
  const RsWeights w{(uint32_t)grp.sum_ll(koR), (uint32_t)grp.sum_ll(koS),
                    (uint32_t)grp.sum_ll(niR), (uint32_t)grp.sum_ll(niS)};
  const uint32_t self = self_weight<G>(a, v, grp);
  Acc q;
  Hast h;
  for (int k = t; k < no; k += G) {
    const int32_t c = kblk(ko[k]);
    const bool leader = k == 0 || kblk(ko[k - 1]) != c;
    uint32_t kc = 0;
    if (leader)
      for (int j = k; j < no && kblk(ko[j]) == c; ++j) kc += kwt(ko[j]);
    if (a.exact) entry_exact<DENSE>(a, R, r, s, false, c, leader, kc, q);
    else entry<DENSE>(a, R, r, s, w.niS, false, c, kwt(ko[k]), leader, kc, q);
    if (a.mh && leader && c != r && c != s) {
      uint32_t kin;
      run_weight(ki, ni, c, kin);
      hast_block<DENSE>(a, R, c, kc + kin, h);
    }
  }
  for (int k = t; k < ni; k += G) {
    const int32_t c = kblk(ki[k]);
    const bool leader = k == 0 || kblk(ki[k - 1]) != c;
    uint32_t kc = 0;
    if (leader)
      for (int j = k; j < ni && kblk(ki[j]) == c; ++j) kc += kwt(ki[j]);
    if (a.exact) entry_exact<DENSE>(a, R, r, s, true, c, leader, kc, q);
    else entry<DENSE>(a, R, r, s, w.niS, true, c, kwt(ki[k]), leader, kc, q);
    uint32_t kout;
    // blocks on both lists were counted with the out-list
    if (a.mh && leader && c != r && c != s && !run_weight(ko, no, c, kout))
      hast_block<DENSE>(a, R, c, kc, h);
  }
  if (a.mh && t == 0) hast_rs<DENSE>(a, R, v, r, s, w, self, h);
  return finish_gen<DENSE, G>(a, R, v, r, s, w, self, q, h, grp, logH);
}

template <bool DENSE, int G>
__device__ double delta_hashed_gen(const NodalArgs& a, int v, int r, int s, HashTab h, int* flag,
                                   const Group<G>& grp, double& logH) {
  const int t = grp.rank();
  const Rows<DENSE> R(a, r, s);
  const int32_t o0 = a.optr[v], no = a.optr[v + 1] - o0;
  const int32_t i0 = a.iptr[v], ni = a.iptr[v + 1] - i0;
  logH = 0.0;
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
  const RsWeights rw{(uint32_t)grp.sum_ll(koR), (uint32_t)grp.sum_ll(koS),
                     (uint32_t)grp.sum_ll(niR), (uint32_t)grp.sum_ll(niS)};
  const uint32_t self = self_weight<G>(a, v, grp);
  Acc q;
  Hast hs;
  // dS: per direction, one hash class of blocks per pass
  for (int dir = 0; dir < 2; ++dir) {
    const int32_t base = dir == 0 ? o0 : i0, n = dir == 0 ? no : ni;
    const int32_t* idx = dir == 0 ? a.oidx : a.iidx;
    const uint32_t* wt = dir == 0 ? a.ow : a.iw;
    const uint32_t P = (uint32_t)((n + kHashSlots / 4 - 1) / (kHashSlots / 4));
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
        const int slot = hash_find(h, c);
        const bool leader = h.first[slot] == k;
        const uint32_t kc = h.sum[slot];
        if (a.exact) entry_exact<DENSE>(a, R, r, s, dir == 1, c, leader, kc, q);
        else entry<DENSE>(a, R, r, s, rw.niS, dir == 1, c, __ldg(wt + base + k), leader, kc, q);
      }
      grp.sync();
    }
  }
  if (a.mh) {
    // proposal weights: per block over both directions, one hash class per pass
    const int n = no + ni;
    const uint32_t P = (uint32_t)((n + kHashSlots / 4 - 1) / (kHashSlots / 4));
    for (uint32_t pass = 0; pass < P; ++pass) {
      for (int i = t; i < kHashSlots; i += G) {
        h.key[i] = -1;
        h.sum[i] = 0u;
        h.first[i] = 0x7fffffff;
      }
      if (t == 0) *flag = 0;
      grp.sync();
      for (int k = t; k < n; k += G) {
        const bool in = k >= no;
        const int j = in ? k - no : k;
        const int32_t c = __ldg(a.part + __ldg((in ? a.iidx + i0 : a.oidx + o0) + j));
        if (c == r || c == s || hclass(c, P) != pass) continue;
        if (!hash_add(h, c, __ldg((in ? a.iw + i0 : a.ow + o0) + j), k)) *flag = 1;
      }
      grp.sync();
      if (*flag) return __longlong_as_double(0x7ff8000000000000ll);
      for (int i = t; i < kHashSlots; i += G)
        if (h.key[i] != -1) hast_block<DENSE>(a, R, h.key[i], h.sum[i], hs);
      grp.sync();
    }
    if (t == 0) hast_rs<DENSE>(a, R, v, r, s, rw, self, hs);
  }
  return finish_gen<DENSE, G>(a, R, v, r, s, rw, self, q, hs, grp, logH);
}

constexpr double kLn2 = 0.6931471805599453;

// Accept test of a general-mode move (r != s).
__device__ __forceinline__ bool accept_move(const NodalArgs& a, double d, double logH,
                                            uint32_t u) {
  if (!a.mh) return d < 0.0;
  // -beta * dS * ln 2 + logH, rounded step by step (no contraction)
  const double x = __dadd_rn(__dmul_rn(__dmul_rn(-a.beta, d), kLn2), logH);
  if (x >= 0.0) return true;
  return log((double)u * 2.3283064365386963e-10) < x;
}

__device__ __forceinline__ void write_result_gen(const NodalArgs& a, bool given, int i, int r,
                                                 int s, double d, double logH, uint32_t u) {
  if (given) {
    a.dS_raw[i] = d;
    if (a.logH_raw) a.logH_raw[i] = logH;
    return;
  }
  const bool acc = r != s && accept_move(a, d, logH, u);
  a.newlab[i] = acc ? s : r;
  a.rec[i] = acc ? d : 0.0;
  if (a.props_out) a.props_out[i] = s;
}

// Mid vertices (more entries than the warp's registers hold, at most
// kWarpHashEntries in both directions): the entries' (direction, block) keys
// are grouped in a per-warp shared-memory hash table (open addressing, at
// most half full), which gives each group its total weight and its first
// entry, the one that adds the group's terms.  One pass, no sort.
constexpr int kWarpHashEntries = 128;
constexpr int kWarpHashSlots = 256;
constexpr uint32_t kEmptyKey = 0xffffffffu;

struct WarpHash {
  uint32_t* key;  // kWarpHashSlots each
  uint32_t* sum;
  int32_t* first;
};

__device__ __forceinline__ uint32_t wh_slot(uint32_t key) {
  return (key * 2654435761u) >> 24;  // 8 bits: kWarpHashSlots = 256
}

template <bool DENSE>
__device__ double delta_whash(const NodalArgs& a, int v, int r, int s, int32_t o0, int no,
                              int32_t i0, int ni, int lane, const WarpHash& h) {
  constexpr int kPer = kWarpHashEntries / 32;  // entries per lane
  constexpr uint32_t kMask = kWarpHashSlots - 1;
  const Rows<DENSE> R(a, r, s);
  const int n = no + ni;
  for (int i = lane; i < kWarpHashSlots; i += 32) {
    h.key[i] = kEmptyKey;
    h.sum[i] = 0u;
    h.first[i] = 0x7fffffff;
  }
  __syncwarp();
  int32_t cs[kPer];
  uint32_t ws[kPer];
  bool ins[kPer];
  uint32_t koR = 0, koS = 0, niR = 0, niS = 0;
#pragma unroll
  for (int p = 0; p < kPer; ++p) {
    const int k = lane + 32 * p;
    cs[p] = -1;
    ws[p] = 0u;
    ins[p] = false;
    if (k < n) {
      const bool in = k >= no;
      const int j = in ? i0 + k - no : o0 + k;
      const int32_t c = __ldg(a.part + __ldg((in ? a.iidx : a.oidx) + j));
      const uint32_t w = __ldg((in ? a.iw : a.ow) + j);
      cs[p] = c;
      ws[p] = w;
      ins[p] = in;
      koR += !in && c == r ? w : 0u;
      koS += !in && c == s ? w : 0u;
      niR += in && c == r ? w : 0u;
      niS += in && c == s ? w : 0u;
      const uint32_t key = (uint32_t)c | (in ? 0x80000000u : 0u);
      uint32_t sl = wh_slot(key);
      // at most n <= kWarpHashSlots / 2 keys: a free or matching slot is
      // found within the table
      for (int probe = 0; probe < kWarpHashSlots; ++probe, sl = (sl + 1) & kMask) {
        const uint32_t prev = atomicCAS(h.key + sl, kEmptyKey, key);
        if (prev == kEmptyKey || prev == key) {
          atomicAdd(h.sum + sl, w);
          atomicMin(h.first + sl, k);
          break;
        }
      }
    }
  }
  __syncwarp();
  const RsWeights w{__reduce_add_sync(kFull, koR), __reduce_add_sync(kFull, koS),
                    __reduce_add_sync(kFull, niR), __reduce_add_sync(kFull, niS)};
  Acc q;
#pragma unroll
  for (int p = 0; p < kPer; ++p) {
    const int k = lane + 32 * p;
    if (k < n) {
      const uint32_t key = (uint32_t)cs[p] | (ins[p] ? 0x80000000u : 0u);
      uint32_t sl = wh_slot(key);
      for (int probe = 0; probe < kWarpHashSlots && h.key[sl] != key; ++probe)
        sl = (sl + 1) & kMask;
      entry<DENSE>(a, R, r, s, w.niS, ins[p], cs[p], ws[p], h.first[sl] == k, h.sum[sl], q);
    }
  }
  const double d = finish<DENSE, 32>(a, R, v, r, s, w, q, Group<32>{nullptr});
  __syncwarp();  // the warp's next vertex reuses the table
  return d;
}

// One vertex (batch index i) on the whole warp: the fused path when its
// entries fit the warp (sampled proposals, GSAP scoring), else the proposal
// by pick_neighbour and the dS from registers (both lists within a warp),
// from the warp's hash table (GSAP scoring, up to kWarpHashEntries) or from
// sorted shared-memory lists.  buf: the warp's kWarpBufWords words of
// shared memory.
constexpr int kWarpBufWords = 384;  // 3 KB: the hash table, or the two sorted lists
template <bool GIVEN, bool DENSE, bool GEN>
__device__ __forceinline__ void warp_vertex(const NodalArgs& a, int i, int lane,
                                            unsigned long long* buf) {
  const Group<32> grp{nullptr};
  unsigned long long* sko = buf;
  unsigned long long* ski = buf + kWarpList;
  const int vv = GIVEN ? a.verts[i] : a.lo + i;
  const int32_t o0 = a.optr[vv], no = a.optr[vv + 1] - o0;
  const int32_t i0 = a.iptr[vv], ni = a.iptr[vv + 1] - i0;
  if constexpr (GEN) {
    int v, s;
    uint32_t u2;
    item<GIVEN>(a, i, lane, v, s, u2);
    const int r = a.part[v];
    double d = 0.0, lh = 0.0;
    if (r != s) {
      if (no + ni <= 32) {
        d = delta_registers_gen<DENSE>(a, v, r, s, o0, no, i0, ni, lane, lh);
      } else {
        stage_sorted<32>(a.oidx, a.ow, a.part, o0, no, sko, grp);
        stage_sorted<32>(a.iidx, a.iw, a.part, i0, ni, ski, grp);
        d = delta_sorted_gen<DENSE, 32>(a, v, r, s, sko, no, ski, ni, grp, lh);
      }
    }
    if (lane == 0) write_result_gen(a, GIVEN, i, r, s, d, lh, u2);
    __syncwarp();
    return;
  }
  if (!GIVEN && no + ni <= 32) {
    fused_group<DENSE, 32>(a, i, true, lane);
    return;
  }
  int v, s;
  uint32_t u2;
  item<GIVEN>(a, i, lane, v, s, u2);
  const int r = a.part[v];
  double d = 0.0;
  if (r != s) {
    if (no <= 32 && ni <= 32) {
      d = delta_registers<DENSE>(a, v, r, s, o0, no, i0, ni, lane);
    } else if (no + ni <= kWarpHashEntries) {
      uint32_t* t = reinterpret_cast<uint32_t*>(buf);
      const WarpHash h{t, t + kWarpHashSlots, reinterpret_cast<int32_t*>(t + 2 * kWarpHashSlots)};
      d = delta_whash<DENSE>(a, v, r, s, o0, no, i0, ni, lane, h);
    } else {
      stage_sorted<32>(a.oidx, a.ow, a.part, o0, no, sko, grp);
      stage_sorted<32>(a.iidx, a.iw, a.part, i0, ni, ski, grp);
      d = delta_sorted<DENSE, 32>(a, v, r, s, sko, no, ski, ni, grp);
    }
  }
  if (lane == 0) write_result(a, GIVEN, i, r, s, d);
  __syncwarp();
}

// Warp work items of a batch: the mid vertices (largest first, as the host
// lists them), then pairs of small vertices.
__host__ __device__ __forceinline__ int nodal_items(int nsmall, int nmid) {
  return (nsmall + 1) / 2 + nmid;
}

template <bool GIVEN, bool DENSE, bool GEN>
struct NodalBody {
  using Args = NodalArgs;
  static constexpr int kThreads = kNodalWarps * 32, kMinBlocks = GEN ? 4 : DENSE ? 10 : 6;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
  if (ctl_stopped(a.ctl)) return;
  __shared__ unsigned long long s_buf[kNodalWarps][kWarpBufWords];
  static_assert(2 * kWarpList <= kWarpBufWords && 3 * kWarpHashSlots <= 2 * kWarpBufWords,
                "per-warp shared buffer");
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = vg * kNodalWarps;
  const int npairs = (a.nsmall + 1) / 2;
  const int items = npairs + a.nmid;
  for (int it0 = vb * kNodalWarps + wid; it0 < items; it0 += nw) {
    int ia, ib = -1;
    if (it0 < a.nmid) {
      ia = a.mid[it0];
    } else {
      const int it = it0 - a.nmid;
      ia = a.small[2 * it];
      const bool two = 2 * it + 1 < a.nsmall;
      ib = two ? a.small[2 * it + 1] : -1;
      if constexpr (!GIVEN && !GEN) {
        // two vertices of at most 16 entries, one per half-warp
        fused_group<DENSE, 16>(a, lane < 16 || !two ? ia : ib, lane < 16 || two, lane);
        continue;
      }
    }
    // one call site, so that the body stays inline
    for (int q = 0; q < (ib >= 0 ? 2 : 1); ++q)
      warp_vertex<GIVEN, DENSE, GEN>(a, q ? ib : ia, lane, s_buf[wid]);
  }
  }
};

// Vertices with more than kWarpList entries in a direction: one CTA each,
// per-block totals from the shared-memory hash table (one pass up to a few
// thousand distinct blocks, more passes beyond).  Sorting both lists in
// shared memory instead (the warp path's method) made the nodal kernels of a
// 200k-vertex partition about 6 ms slower, for the same dS.
template <bool GIVEN, bool DENSE, bool GEN>
struct NodalHeavyBody {
  using Args = NodalArgs;
  static constexpr int kThreads = kHeavyThreads, kMinBlocks = 2;
  static constexpr size_t kSmem = kHeavySmem;
  static __device__ void run(const Args& a, int vb, int vg) {
  if (ctl_stopped(a.ctl)) return;
  extern __shared__ unsigned long long hsm[];
  __shared__ double red[kHeavyThreads / 32];
  __shared__ int flag, sh_v, sh_s;
  __shared__ uint32_t sh_u2;
  Group<kHeavyThreads> grp{red};
  HashTab ht{(int32_t*)hsm, (uint32_t*)hsm + kHashSlots, (int32_t*)hsm + 2 * kHashSlots};
  for (int h = vb; h < a.nheavy; h += vg) {
    const int i = a.heavy[h];
    if (threadIdx.x < 32) {
      int v, s;
      uint32_t u2;
      item<GIVEN>(a, i, threadIdx.x, v, s, u2);
      if (threadIdx.x == 0) {
        sh_v = v;
        sh_s = s;
        sh_u2 = u2;
      }
    }
    __syncthreads();
    const int v = sh_v, s = sh_s;
    const int r = a.part[v];
    const int32_t o0 = a.optr[v], no = a.optr[v + 1] - o0;
    const int32_t i0 = a.iptr[v], ni = a.iptr[v + 1] - i0;
    double d = 0.0, lh = 0.0;
    if (r != s) {
      if constexpr (GEN)
        d = delta_hashed_gen<DENSE, kHeavyThreads>(a, v, r, s, ht, &flag, grp, lh);
      else
        d = delta_hashed<DENSE, kHeavyThreads>(a, v, r, s, ht, &flag, grp);
      if (threadIdx.x == 0 && d != d) atomicAdd(a.err, 1);
    }
    if (threadIdx.x == 0) {
      if constexpr (GEN) write_result_gen(a, GIVEN, i, r, s, d, lh, sh_u2);
      else write_result(a, GIVEN, i, r, s, d);
    }
    __syncthreads();
  }
  }
};

// Applies the batch's labels and sums its recorded dS.  Each CTA sums a fixed
// slice (one vertex a thread) in a fixed order into its own partial; the
// last CTA to finish (a ticket, no waiting) adds the partials with one warp
// in a fixed order, so the result does not depend on scheduling.  In dense
// mode the CTAs also refresh the log2 of the block degrees that
// dense_update changed, and the virtual blocks past `ncommit` (if any) make
// the next batch's per-block draws: they read only M, its chunk sums and the
// block degrees, all final once dense_update has run, so the draws need no
// launch of their own.
constexpr int kCommitThreads = 256;

struct CommitArgs {
  int32_t* part;
  const int32_t* newlab;
  const double* rec;
  double* slot_sum;
  long long* slot_acc;
  const uint32_t *d_out, *d_in;  // dense mode: refresh ld_out / ld_in
  double *ld_out, *ld_in;
  double* part_sum;
  long long* part_cnt;
  unsigned* ticket;
  const int32_t* ctl;  // sweep control: gate, and slots advance ctl[0] * slot_mul
  // dense mode, draws for the next batch (RNG sequence draw_seq + ctl[0] *
  // draw_seq_mul) by the virtual blocks past ncommit
  const uint32_t *Md, *MTd, *Sd;
  int32_t* nbr_s;
  uint8_t* use_rand;
  uint64_t seed;
  uint32_t draw_seq, draw_seq_mul;
  int32_t lo, count, B, slot_mul;
  int32_t ncommit, pad;
};

struct CommitBody {
  using Args = CommitArgs;
  static constexpr int kThreads = kCommitThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    if (ctl_stopped(a.ctl)) return;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (vb >= a.ncommit) {
      const uint32_t seq = a.draw_seq + ctl_itr(a.ctl) * a.draw_seq_mul;
      const int nw = ((vg - a.ncommit) * kCommitThreads) >> 5;
      for (int b = ((vb - a.ncommit) * kCommitThreads + tid) >> 5; b < a.B; b += nw)
        dense_block_draw(a.Md, a.MTd, a.Sd, a.d_out, a.d_in, a.B, a.seed, seq, b, lane,
                         a.nbr_s, a.use_rand);
      return;
    }
    const int nc = a.ncommit;
    __shared__ double sh[kCommitThreads / 32];
    __shared__ long long shc[kCommitThreads / 32];
    __shared__ bool last;
    double s = 0.0;
    long long c = 0;
    for (int i = vb * kCommitThreads + tid; i < a.count; i += nc * kCommitThreads) {
      const int32_t nl = a.newlab[i];
      const int32_t old = a.part[a.lo + i];
      const double x = a.rec[i];
      if (old != nl) {
        a.part[a.lo + i] = nl;
        ++c;
      }
      s += x;
    }
    if (a.ld_out)
      for (int b = vb * kCommitThreads + tid; b < a.B; b += nc * kCommitThreads) {
        a.ld_out[b] = log2((double)a.d_out[b]);
        a.ld_in[b] = log2((double)a.d_in[b]);
      }
    s = warp_sum(s);
    c = warp_sum_ll(c);
    if (lane == 0) {
      sh[wid] = s;
      shc[wid] = c;
    }
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      long long n = 0;
      for (int k = 0; k < kCommitThreads / 32; ++k) {
        t += sh[k];
        n += shc[k];
      }
      a.part_sum[vb] = t;
      a.part_cnt[vb] = n;
      __threadfence();
      last = atomicAdd(a.ticket, 1u) == (unsigned)nc - 1u;
    }
    __syncthreads();
    if (last && wid == 0) {
      __threadfence();
      double t = 0.0;
      long long n = 0;
      for (int k = lane; k < nc; k += 32) {
        t += ((volatile double*)a.part_sum)[k];
        n += ((volatile long long*)a.part_cnt)[k];
      }
      t = warp_sum(t);
      n = warp_sum_ll(n);
      if (lane == 0) {
        const int k = (int)ctl_itr(a.ctl) * a.slot_mul;
        a.slot_sum[k] += t;
        a.slot_acc[k] += n;
        *a.ticket = 0u;
      }
    }
  }
};

// CTAs of one commit: a function of the batch size only.
int32_t vg_commit(int32_t count) {
  return std::max(1, std::min(kCommitCtas, ceil_div(count, kCommitThreads)));
}

CommitArgs commit_args(int32_t* part, int32_t lo, int32_t count, const int32_t* newlab,
                       const double* rec, double* slot_sum, long long* slot_acc,
                       const DevBM* dense_m, int32_t B, const CommitScratch& cs) {
  CommitArgs a{};
  a.part = part;
  a.newlab = newlab;
  a.rec = rec;
  a.slot_sum = slot_sum;
  a.slot_acc = slot_acc;
  if (dense_m) {
    a.d_out = dense_m->d_out;
    a.d_in = dense_m->d_in;
    a.ld_out = dense_m->ld_out;
    a.ld_in = dense_m->ld_in;
    a.B = B;
  }
  a.part_sum = cs.part_sum;
  a.part_cnt = cs.part_cnt;
  a.ticket = cs.ticket;
  a.lo = lo;
  a.count = count;
  a.ncommit = vg_commit(count);
  return a;
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
  a.ld_out = m.ld_out; a.ld_in = m.ld_in;
  a.nbr_s = m.nbr_s; a.use_rand = m.use_rand;
  a.B = B;
  a.heavy = aux.heavy;
  a.nheavy = aux.nheavy;
  a.small = aux.small;
  a.nsmall = aux.nsmall;
  a.mid = aux.mid;
  a.nmid = aux.nmid;
  a.err = aux.err;
  return a;
}

// CTAs of the warp kernel: one warp per work item.
int nodal_grid(const NodalArgs& a) {
  int g = (nodal_items(a.nsmall, a.nmid) + kNodalWarps - 1) / kNodalWarps;
  return g < 1 ? 1 : (g > 148 * 64 ? 148 * 64 : g);
}

template <bool GIVEN, bool DENSE, bool GEN>
void launch_pair(const NodalArgs& a, const NodalAux& aux, cudaStream_t st) {
  if (a.nheavy > 0) {
    // heavy vertices on the side stream, next to the warp kernel
    cudaEventRecord(aux.fork, st);
    cudaStreamWaitEvent(aux.side, aux.fork, 0);
    launch_single<NodalHeavyBody<GIVEN, DENSE, GEN>>(a, std::min(a.nheavy, 2 * 148), aux.side);
    cudaEventRecord(aux.join, aux.side);
  }
  launch_single<NodalBody<GIVEN, DENSE, GEN>>(a, nodal_grid(a), st);
  if (a.nheavy > 0) cudaStreamWaitEvent(st, aux.join, 0);
}

template <bool GIVEN, bool DENSE>
void launch_mode(const NodalArgs& a, const NodalAux& aux, cudaStream_t st, bool gen) {
  if (gen) launch_pair<GIVEN, DENSE, true>(a, aux, st);
  else launch_pair<GIVEN, DENSE, false>(a, aux, st);
}

// indexed by ScoreMode::slot(dense)
const MultiKernel kmNodal[4] = {
    multi_kernel_desc<NodalBody<false, false, false>>("nodal_csr"),
    multi_kernel_desc<NodalBody<false, true, false>>("nodal_dense"),
    multi_kernel_desc<NodalBody<false, false, true>>("nodal_gen_csr"),
    multi_kernel_desc<NodalBody<false, true, true>>("nodal_gen_dense")};
const MultiKernel kmNodalHeavy[4] = {
    multi_kernel_desc<NodalHeavyBody<false, false, false>>("nodal_heavy_csr"),
    multi_kernel_desc<NodalHeavyBody<false, true, false>>("nodal_heavy_dense"),
    multi_kernel_desc<NodalHeavyBody<false, false, true>>("nodal_heavy_gen_csr"),
    multi_kernel_desc<NodalHeavyBody<false, true, true>>("nodal_heavy_gen_dense")};

void set_mode(NodalArgs& a, const ScoreMode& md) {
  a.exact = md.exact;
  a.mh = md.mh;
  a.beta = md.beta;
}
const MultiKernel kmCommit = multi_kernel_desc<CommitBody>("commit");

}  // namespace

cudaError_t init_nodal_attributes() {
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* f) {
    cudaError_t x = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kHeavySmem);
    if (x != cudaSuccess) e = x;
  };
  set((const void*)single_kernel<NodalHeavyBody<false, false, false>>);
  set((const void*)single_kernel<NodalHeavyBody<false, true, false>>);
  set((const void*)single_kernel<NodalHeavyBody<true, false, false>>);
  set((const void*)single_kernel<NodalHeavyBody<true, true, false>>);
  set((const void*)multi_kernel<NodalHeavyBody<false, false, false>>);
  set((const void*)multi_kernel<NodalHeavyBody<false, true, false>>);
  set((const void*)single_kernel<NodalHeavyBody<false, false, true>>);
  set((const void*)single_kernel<NodalHeavyBody<false, true, true>>);
  set((const void*)single_kernel<NodalHeavyBody<true, false, true>>);
  set((const void*)single_kernel<NodalHeavyBody<true, true, true>>);
  set((const void*)multi_kernel<NodalHeavyBody<false, false, true>>);
  set((const void*)multi_kernel<NodalHeavyBody<false, true, true>>);
  return e;
}

int nodal_heavy_threshold() { return kWarpList; }

void nodal_batch_sample(const DevGraph& g, const int32_t* part, const DevBM& m, int32_t B,
                        bool dense, uint64_t seed, uint32_t seq, int32_t lo, int32_t count,
                        int32_t* newlab, double* rec, int32_t* props, const NodalAux& aux,
                        cudaStream_t st, const ScoreMode& md) {
  NodalArgs a = make_args(g, part, m, B, aux);
  set_mode(a, md);
  a.seed = seed;
  a.seq = seq;
  a.lo = lo;
  a.count = count;
  a.newlab = newlab;
  a.rec = rec;
  a.props_out = props;
  if (count <= 0) return;
  if (dense) launch_mode<false, true>(a, aux, st, md.general());
  else launch_mode<false, false>(a, aux, st, md.general());
}

void nodal_delta_given(const DevGraph& g, const int32_t* part, const DevBM& m, int32_t B,
                       bool dense, int32_t nv, const int32_t* verts, const int32_t* props,
                       double* dS, const NodalAux& aux, cudaStream_t st, const ScoreMode& md,
                       double* logH) {
  NodalArgs a = make_args(g, part, m, B, aux);
  set_mode(a, md);
  a.count = nv;
  a.verts = verts;
  a.props_in = props;
  a.dS_raw = dS;
  a.logH_raw = logH;
  if (nv <= 0) return;
  if (dense) launch_mode<true, true>(a, aux, st, md.general());
  else launch_mode<true, false>(a, aux, st, md.general());
}

void nodal_commit(int32_t* part, int32_t lo, int32_t count, const int32_t* newlab,
                  const double* rec, double* slot_sum, long long* slot_acc, const DevBM* dense_m,
                  int32_t B, const CommitScratch& cs, cudaStream_t st) {
  launch_single<CommitBody>(
      commit_args(part, lo, count, newlab, rec, slot_sum, slot_acc, dense_m, B, cs),
      vg_commit(count), st);
}

void add_nodal(Slot& warp, Slot& heavy, bool dense, const ScoreMode& md, const DevGraph& g,
               const int32_t* part,
               const DevBM& m, int32_t B, uint64_t seed, uint32_t seq, int32_t lo, int32_t count,
               int32_t* newlab, double* rec, int32_t* props, const NodalAux& aux,
               const int32_t* ctl, uint32_t seq_mul) {
  if (count <= 0) return;
  NodalArgs a = make_args(g, part, m, B, aux);
  a.seed = seed;
  a.seq = seq;
  a.lo = lo;
  a.count = count;
  a.newlab = newlab;
  a.rec = rec;
  a.props_out = props;
  a.ctl = ctl;
  a.seq_mul = seq_mul;
  set_mode(a, md);
  slot_push(slot_bind(warp, kmNodal[md.slot(dense)]), a,
            ceil_div(nodal_items(aux.nsmall, aux.nmid), kNodalWarps));
  slot_push(slot_bind(heavy, kmNodalHeavy[md.slot(dense)]), a, aux.nheavy);
}

void add_commit(Slot& s, int32_t* part, int32_t lo, int32_t count, const int32_t* newlab,
                const double* rec, double* slot_sum, long long* slot_acc, const DevBM* dense_m,
                int32_t B, const CommitScratch& cs, const int32_t* ctl, int32_t slot_mul,
                bool draw_next, uint64_t seed, uint32_t draw_seq, uint32_t draw_seq_mul) {
  CommitArgs a = commit_args(part, lo, count, newlab, rec, slot_sum, slot_acc, dense_m, B, cs);
  a.ctl = ctl;
  a.slot_mul = slot_mul;
  int32_t vg = a.ncommit;
  if (draw_next && dense_m) {
    a.Md = dense_m->Md;
    a.MTd = dense_m->MTd;
    a.Sd = dense_m->Sd;
    a.nbr_s = dense_m->nbr_s;
    a.use_rand = dense_m->use_rand;
    a.seed = seed;
    a.draw_seq = draw_seq;
    a.draw_seq_mul = draw_seq_mul;
    // a warp per block, as the block-terms kernel
    vg += std::max(1, std::min(8192, ceil_div((long long)B * 32, kCommitThreads)));
  }
  slot_push(slot_bind(s, kmCommit), a, vg);
}

}  // namespace sbp
