// Merge phase: proposals, merge dS and the best proposal of each block.
//
// GSAP draws proposals with three curand kernels and a float running-sum
// scan (kernels.hpp:645-856), computes dS with four kernels that each walk
// whole rows per proposal thread (kernels.hpp:143-449, grid sized from nnz,
// Q16) and reduces with find_best_warp (kernels.hpp:452-491).
//
// Here: one warp per block draws its proposals (Philox, exact integer picks
// by a running prefix over the row in 32-entry chunks, one ballot per
// proposal per chunk) and one warp per block computes their dS, walking only
// the shorter of the
// two rows being merged and looking the other up by binary search, with the
// unchanged remainder taken from the per-block sums; lanes 0..np-1 then hold
// the proposals' dS and run the same 32-lane halving argmin as
// find_best_warp, ties going to the lane further up.  FP64 throughout.
#include "common.cuh"
#include "kernels.h"
#include "multi.cuh"

#include <cfloat>

namespace sbp {

namespace {

constexpr int kMergeWarps = 8;

int32_t vg_merge_delta(int32_t B);

struct MergeArgs {
  const double* xlx;
  const int32_t *optr, *ocol, *iptr, *icol;
  const uint32_t *ocnt, *icnt, *d_out, *d_in;
  const double *ld_out, *ld_in, *dSout, *ambout, *ambin, *sinfull;
  int32_t B, np;
  uint64_t seed;
  uint32_t seq;
  const int32_t* props_in;
  int32_t* props;
  double* dS;
  int32_t* best;
  double* best_dS;
  int32_t exact;  // 1: exact merge dS (merge_one_exact)
  // GSAP's merge grid (Q16, partition.hpp:335-336): with ref_grid set, only
  // proposals t < T = (nnz of the out CSR, rounded up to 256) are drawn and
  // scored; slots t >= T keep the target (props) and dS (keep_dS) their
  // buffers hold, and a proposal whose partner slot s*np+k lies at or past T
  // reads that slot's in-row term from keep_dsin.
  int32_t ref_grid;
  double* keep_dS;
  double* keep_dsin;
  double* pdS;  // per-proposal dS (B * np) between the warp-per-proposal kernels
};

// First proposal slot GSAP's merge grid leaves out (B*np when none is).
__device__ __forceinline__ long long merge_grid_end(const MergeArgs& a) {
  const long long n = (long long)a.B * a.np;
  if (!a.ref_grid) return n;
  const long long T = ((long long)a.optr[a.B] + 255) / 256 * 256;
  return T < n ? T : n;
}

// Count and column of entry k of out-row ++ in-row of block b (the scan
// order of kernels.hpp:767-783).
__device__ __forceinline__ uint32_t cnt_at(const MergeArgs& a, int b, int k, int no) {
  return k < no ? __ldg(a.ocnt + a.optr[b] + k) : __ldg(a.icnt + a.iptr[b] + k - no);
}
__device__ __forceinline__ int col_at(const MergeArgs& a, int b, int k) {
  int o0 = a.optr[b], no = a.optr[b + 1] - o0;
  return k < no ? __ldg(a.ocol + o0 + k) : __ldg(a.icol + a.iptr[b] + k - no);
}

// Inclusive scan of 64-bit values over the warp's lanes.
__device__ __forceinline__ unsigned long long warp_incl_scan_ull(unsigned long long x, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// The whole warp walks out-row ++ in-row of block b (warp-uniform) in
// chunks of 32 entries with a running prefix of the counts.  Each lane L
// with want set looks for the first entry whose running count exceeds its
// own threshold t; returns that entry's index in the lane that asked, -1
// where none does.  The same picks as a serial running sum.
__device__ int warp_pick(const MergeArgs& a, int b, uint64_t t, bool want, int lane) {
  const int no = a.optr[b + 1] - a.optr[b];
  const int n = no + (a.iptr[b + 1] - a.iptr[b]);
  int found = -1;
  unsigned open = __ballot_sync(kFull, want);
  unsigned long long base = 0;
  for (int c0 = 0; c0 < n && open; c0 += 32) {
    const int k = c0 + lane;
    const unsigned long long incl =
        warp_incl_scan_ull(k < n ? cnt_at(a, b, k, no) : 0u, lane) + base;
    unsigned rest = open;
    while (rest) {
      const int L = __ffs(rest) - 1;
      rest &= rest - 1;
      const unsigned long long tL = __shfl_sync(kFull, (unsigned long long)t, L);
      const unsigned m = __ballot_sync(kFull, k < n && incl > tL);
      if (m) {
        if (lane == L) found = c0 + __ffs(m) - 1;
        open &= ~(1u << L);
      }
    }
    base = __shfl_sync(kFull, incl, 31);
  }
  return found;
}

// choose_neighbors + propose_blocks (kernels.hpp:726-856): one warp per
// block r draws its np proposals, lane k the k-th.  The first hop picks a
// neighbour u of r by weight (all lanes in r's row at once); lanes that do
// not propose a random block then pick in u's row, one walk per lane, and
// take the first entry from there on whose column is not r (block 0 when
// none is).
struct MergePropsBody {
  using Args = MergeArgs;
  static constexpr int kThreads = kMergeWarps * 32, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg);
};

__device__ void MergePropsBody::run(const MergeArgs& a, int vb, int vg) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long T = merge_grid_end(a);
  const uint32_t B = (uint32_t)a.B;
  for (int r = vb * kMergeWarps + wid; r < a.B; r += vg * kMergeWarps) {
    const long long t = (long long)r * a.np + lane;
    const bool mine = lane < a.np && t < T;  // slots GSAP's grid leaves out keep theirs
    if (!__any_sync(kFull, mine)) continue;
    P4 x{};
    if (mine) x = draw(a.seed, kRngMerge, a.seq, (uint32_t)t);
    const int rnd = (int)(x.v[0] % B);
    const uint64_t deg_r = (uint64_t)a.d_out[r] + a.d_in[r];
    int s = rnd;
    // first hop: a neighbour u of r in proportion to weight
    const bool hop = mine && deg_r != 0;
    const int k = warp_pick(a, r, hop ? scale_draw(x.v[1], deg_r) : 0, hop, lane);
    int u = 0;
    bool second = false;
    uint64_t deg_u = 0;
    if (hop) {
      u = k >= 0 ? col_at(a, r, k) : 0;
      deg_u = (uint64_t)a.d_out[u] + a.d_in[u];
      second = !accept_random(x.v[2], deg_u, B);
      if (second) s = 0;
    }
    // second hop: each lane that needs it walks its own u's row with the warp
    unsigned need = __ballot_sync(kFull, second && deg_u > 0);
    while (need) {
      const int L = __ffs(need) - 1;
      need &= need - 1;
      const int uL = __shfl_sync(kFull, u, L);
      const uint64_t tL = __shfl_sync(kFull, (unsigned long long)scale_draw(x.v[3], deg_u), L);
      const int k2 = warp_pick(a, uL, tL, lane == L, lane);
      if (lane == L && k2 >= 0) {
        const int n = (a.optr[u + 1] - a.optr[u]) + (a.iptr[u + 1] - a.iptr[u]);
        for (int q = k2; q < n; ++q) {
          const int c = col_at(a, u, q);
          if (c != r) {
            s = c;
            break;
          }
        }
      }
    }
    if (mine) a.props[t] = s;
  }
}

__device__ __forceinline__ double gterm(const double* tab, uint32_t x, double ld) {
  return x == 0u ? 0.0 : xlx(tab, x) - (double)x * ld;
}
__device__ __forceinline__ double fterm(const double* tab, uint32_t m, double a, double b) {
  return m == 0u ? 0.0 : xlx(tab, m) - (double)m * (a + b);
}

// Sum over a group of G lanes (G = 8 or 32; every lane of the warp calls it).
template <int G>
__device__ __forceinline__ double group_sum(double x) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o, G);
  return x;
}

// Merge dS of block r with s (calculate_dS_overall, kernels.hpp:417-449) by
// a group of G lanes (gl = lane in the group), s2 = the k-th proposal of
// block s (its in-term leaves out s2, Q1).  With given_in_s, block s's
// in-term is in_s_given (a slot GSAP's grid left out); in_r_out receives
// block r's in-term.  An inactive group walks nothing but still takes part
// in the group sums (every lane of the warp must).
template <int G>
__device__ double merge_one(const MergeArgs& a, int r, int s, int s2, int gl, bool active,
                            bool given_in_s, double in_s_given, double* in_r_out) {
  // merged out-rows (calculate_dS_new_out, kernels.hpp:233-320)
  double acc_o = 0.0, acc_i = 0.0;
  const double ldo_r = a.ld_out[r], ldo_s = a.ld_out[s], ldi_r = a.ld_in[r], ldi_s = a.ld_in[s];
  const uint32_t Mrr = row_lookup(a.ocol, a.ocnt, a.optr[r], a.optr[r + 1], r);
  const uint32_t Mrs = row_lookup(a.ocol, a.ocnt, a.optr[r], a.optr[r + 1], s);
  const uint32_t Msr = row_lookup(a.ocol, a.ocnt, a.optr[s], a.optr[s + 1], r);
  const uint32_t Mss = row_lookup(a.ocol, a.ocnt, a.optr[s], a.optr[s + 1], s);
  if (!active) {
  } else if (r == s) {
    for (int i = a.optr[r] + gl; i < a.optr[r + 1]; i += G)
      acc_o += gterm(a.xlx, 2u * a.ocnt[i], a.ld_in[a.ocol[i]]);
    for (int i = a.iptr[r] + gl; i < a.iptr[r + 1]; i += G) {
      int c = a.icol[i];
      if (c != r) acc_i += gterm(a.xlx, 2u * a.icnt[i], a.ld_out[c]);
    }
  } else {
    int x = r, y = s;
    if (a.optr[s + 1] - a.optr[s] < a.optr[r + 1] - a.optr[r]) { x = s; y = r; }
    int y0 = a.optr[y], y1 = a.optr[y + 1];
    for (int i = a.optr[x] + gl; i < a.optr[x + 1]; i += G) {
      int c = a.ocol[i];
      double ld = a.ld_in[c];
      uint32_t my = row_lookup(a.ocol, a.ocnt, y0, y1, c);
      acc_o += gterm(a.xlx, a.ocnt[i] + my, ld) - gterm(a.xlx, my, ld);
    }
    if (gl == 0) acc_o += a.ambout[y];
    x = r; y = s;
    if (a.iptr[s + 1] - a.iptr[s] < a.iptr[r + 1] - a.iptr[r]) { x = s; y = r; }
    y0 = a.iptr[y]; y1 = a.iptr[y + 1];
    for (int i = a.iptr[x] + gl; i < a.iptr[x + 1]; i += G) {
      int c = a.icol[i];
      if (c == r || c == s) continue;
      double ld = a.ld_out[c];
      uint32_t my = row_lookup(a.icol, a.icnt, y0, y1, c);
      acc_i += gterm(a.xlx, a.icnt[i] + my, ld) - gterm(a.xlx, my, ld);
    }
    if (gl == 0) {
      // in-row y's own terms at columns r and s stay out
      uint32_t yr = y == r ? Mrr : Mrs;  // M[r][y]
      uint32_t ys = y == r ? Msr : Mss;  // M[s][y]
      acc_i += a.ambin[y] - gterm(a.xlx, yr, ldo_r) - gterm(a.xlx, ys, ldo_s);
    }
  }
  acc_o = group_sum<G>(acc_o);
  acc_i = group_sum<G>(acc_i);
  const uint32_t dor = a.d_out[r], dos = a.d_out[s], dir = a.d_in[r], dis = a.d_in[s];
  long long mass_o = (long long)dor + (long long)dos;
  long long mass_i = r == s ? 2LL * ((long long)dir - (long long)Mrr)
                            : (long long)dir + (long long)dis - (long long)Mrr - (long long)Msr -
                                  (long long)Mrs - (long long)Mss;
  double new_out = -acc_o;
  if (mass_o != 0) new_out += log2((double)(uint32_t)(dos + dor)) * (double)mass_o;
  double new_in = -acc_i;
  if (mass_i != 0) new_in += log2((double)(uint32_t)(dis + dir)) * (double)mass_i;
  // old in-rows (calculate_dS_in, kernels.hpp:185-231): row r without r, s;
  // row s without s, s2
  double in_r = a.sinfull[r] - fterm(a.xlx, Mrr, ldo_r, ldi_r) - (s != r ? fterm(a.xlx, Msr, ldo_s, ldi_r) : 0.0);
  double in_s;
  if (given_in_s) {
    in_s = in_s_given;
  } else {
    uint32_t Ms2s = s2 == s ? 0u : row_lookup(a.ocol, a.ocnt, a.optr[s2], a.optr[s2 + 1], s);
    in_s = a.sinfull[s] - fterm(a.xlx, Mss, ldo_s, ldi_s) - fterm(a.xlx, Ms2s, a.ld_out[s2], ldi_s);
  }
  *in_r_out = in_r;
  return a.dSout[r] + a.dSout[s] + in_r + in_s + new_out + new_in;
}

// Exact change of the MDL when block r merges into s: rows r and s add up
// into row s, columns r and s into column s.  Of the sum of M log2 M only
// the cells present in both rows (both columns) and the four corner cells,
// which become one, change; of the degree terms the two rows' and the two
// columns'.  dS = -(change of data_S), B fixed.  Group-cooperative: the
// shorter row is walked, the longer one searched.
template <int G>
__device__ double merge_one_exact(const MergeArgs& a, int r, int s, int gl, bool active) {
  active = active && r != s;
  double acc = 0.0;  // - (change of the off-corner cells)
  if (active) {
    int x = r, y = s;
    if (a.optr[s + 1] - a.optr[s] < a.optr[r + 1] - a.optr[r]) { x = s; y = r; }
    int y0 = a.optr[y], y1 = a.optr[y + 1];
    for (int i = a.optr[x] + gl; i < a.optr[x + 1]; i += G) {
      const int c = a.ocol[i];
      if (c == r || c == s) continue;
      const uint32_t b = row_lookup(a.ocol, a.ocnt, y0, y1, c);
      if (b) acc -= xlx(a.xlx, a.ocnt[i] + b) - xlx(a.xlx, a.ocnt[i]) - xlx(a.xlx, b);
    }
    x = r; y = s;
    if (a.iptr[s + 1] - a.iptr[s] < a.iptr[r + 1] - a.iptr[r]) { x = s; y = r; }
    y0 = a.iptr[y]; y1 = a.iptr[y + 1];
    for (int i = a.iptr[x] + gl; i < a.iptr[x + 1]; i += G) {
      const int c = a.icol[i];
      if (c == r || c == s) continue;
      const uint32_t b = row_lookup(a.icol, a.icnt, y0, y1, c);
      if (b) acc -= xlx(a.xlx, a.icnt[i] + b) - xlx(a.xlx, a.icnt[i]) - xlx(a.xlx, b);
    }
    if (gl == 0) {
      const uint32_t Mrr = row_lookup(a.ocol, a.ocnt, a.optr[r], a.optr[r + 1], r);
      const uint32_t Mrs = row_lookup(a.ocol, a.ocnt, a.optr[r], a.optr[r + 1], s);
      const uint32_t Msr = row_lookup(a.ocol, a.ocnt, a.optr[s], a.optr[s + 1], r);
      const uint32_t Mss = row_lookup(a.ocol, a.ocnt, a.optr[s], a.optr[s + 1], s);
      const uint32_t dor = a.d_out[r], dos = a.d_out[s], dir = a.d_in[r], dis = a.d_in[s];
      const double corner = xlx(a.xlx, Mrr + Mrs + Msr + Mss) - xlx(a.xlx, Mrr) -
                            xlx(a.xlx, Mrs) - xlx(a.xlx, Msr) - xlx(a.xlx, Mss);
      const double degs = xlx(a.xlx, dor + dos) - xlx(a.xlx, dor) - xlx(a.xlx, dos) +
                          xlx(a.xlx, dir + dis) - xlx(a.xlx, dir) - xlx(a.xlx, dis);
      acc += degs - corner;
    }
  }
  return group_sum<G>(acc);
}

// One warp per block r: groups of G lanes score the block's proposals, 32/G
// at a time (G = 8 when the blockmodel's rows are short, as at large B;
// else 32, the whole warp on one proposal); lanes 0..np-1 then hold the
// proposals' dS and run find_best_warp's 32-lane halving argmin
// (kernels.hpp:452-491), ties going to the lane further up.
template <int G>
struct MergeDeltaBody {
  using Args = MergeArgs;
  static constexpr int kThreads = kMergeWarps * 32, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
  constexpr int NG = 32 / G;  // groups per warp
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int g = lane / G, gl = lane % G;
  const long long T = merge_grid_end(a);
  for (int r = vb * kMergeWarps + wid; r < a.B; r += vg * kMergeWarps) {
    double mine = DBL_MAX;
    int who = 0;
    for (int k0 = 0; k0 < a.np; k0 += NG) {
      const int k = k0 + g;
      const bool act = k < a.np;
      const long long t = (long long)r * a.np + (act ? k : 0);
      const int s = act ? a.props_in[t] : r;
      const bool stale = act && t >= T;  // a slot GSAP's grid leaves out keeps its values
      const bool comp = act && !stale;
      double d, in_r = 0.0;
      if (a.exact) {
        d = merge_one_exact<G>(a, r, s, gl, comp);
      } else {
        const long long sid = (long long)s * a.np + (act ? k : 0);
        const bool given = comp && sid >= T;
        const int s2 = comp && !given ? a.props_in[sid] : s;
        d = merge_one<G>(a, r, s, s2, gl, comp, given, given ? a.keep_dsin[sid] : 0.0, &in_r);
      }
      if (stale) d = a.keep_dS[t];
      if (comp && gl == 0) {
        if (a.dS) a.dS[t] = d;
        if (a.ref_grid) {
          a.keep_dS[t] = d;
          if (!a.exact) a.keep_dsin[t] = in_r;
        }
      }
      // proposal k0 + j's dS and target from group j's first lane
      const int j = (lane - k0) & (NG - 1);
      const double dj = __shfl_sync(kFull, d, j * G);
      const int sj = __shfl_sync(kFull, s, j * G);
      if (lane >= k0 && lane < k0 + NG && lane < a.np) {
        mine = dj;
        who = sj;
      }
    }
    // find_best_warp's reduction
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_down_sync(kFull, mine, o);
      int ow = __shfl_down_sync(kFull, who, o);
      mine = fmin(mine, ov);
      if (mine == ov) who = ow;
    }
    if (lane == 0) {
      a.best[r] = who;
      a.best_dS[r] = mine;
    }
  }
  }
};

// Long rows (E > 16 B): one warp per proposal, so that the few blocks of a
// small B still fill the GPU; each proposal's dS goes to pdS (slots GSAP's
// grid leaves out keep theirs: pdS is then the persistent keep_dS), and
// MergeBestBody reduces each block's proposals.
struct MergePropDeltaBody {
  using Args = MergeArgs;
  static constexpr int kThreads = kMergeWarps * 32, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const long long n = (long long)a.B * a.np, T = merge_grid_end(a);
    for (long long t = (long long)vb * kMergeWarps + wid; t < n && t < T;
         t += (long long)vg * kMergeWarps) {
      const int r = (int)(t / a.np), k = (int)(t % a.np);
      const int s = a.props_in[t];
      double d, in_r = 0.0;
      if (a.exact) {
        d = merge_one_exact<32>(a, r, s, lane, true);
      } else {
        const long long sid = (long long)s * a.np + k;
        const bool given = sid >= T;
        const int s2 = given ? s : a.props_in[sid];
        d = merge_one<32>(a, r, s, s2, lane, true, given, given ? a.keep_dsin[sid] : 0.0, &in_r);
      }
      if (lane == 0) {
        a.pdS[t] = d;
        if (a.dS && a.dS != a.pdS) a.dS[t] = d;
        if (a.ref_grid && !a.exact) a.keep_dsin[t] = in_r;
      }
    }
  }
};

// find_best_warp (kernels.hpp:452-491) over each block's proposals in pdS.
struct MergeBestBody {
  using Args = MergeArgs;
  static constexpr int kThreads = kMergeWarps * 32, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int r = vb * kMergeWarps + wid; r < a.B; r += vg * kMergeWarps) {
      const long long t = (long long)r * a.np + lane;
      double mine = lane < a.np ? a.pdS[t] : DBL_MAX;
      int who = lane < a.np ? a.props_in[t] : 0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_down_sync(kFull, mine, o);
        int ow = __shfl_down_sync(kFull, who, o);
        mine = fmin(mine, ov);
        if (mine == ov) who = ow;
      }
      if (lane == 0) {
        a.best[r] = who;
        a.best_dS[r] = mine;
      }
    }
  }
};

struct RelabelArgs {
  int32_t* part;
  const int32_t* map;
  int32_t N, pad;
};

struct RelabelBody {
  using Args = RelabelArgs;
  static constexpr int kThreads = 256, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int) {
    int v = vb * kThreads + threadIdx.x;
    if (v < a.N) a.part[v] = __ldg(a.map + a.part[v]);
  }
};


int32_t vg_merge_delta(int32_t B) { return std::min(ceil_div(B, kMergeWarps), 148 * 32); }

const MultiKernel kmMergeProps = multi_kernel_desc<MergePropsBody>("merge_props");
// Groups of 8 lanes score a proposal when rows are short: at most 16
// entries a row on average (nnz <= E).  A function of the job's sizes only.
bool short_rows(int32_t B, int32_t E) { return (long long)E <= 16LL * B; }
int32_t vg_merge_prop(int32_t B, int32_t np) {
  return std::max(1, std::min(ceil_div((long long)B * np, kMergeWarps), 148 * 32));
}

const MultiKernel kmMergeDelta = multi_kernel_desc<MergePropDeltaBody>("merge_delta");
const MultiKernel kmMergeBest = multi_kernel_desc<MergeBestBody>("merge_best");
const MultiKernel kmMergeDelta8 = multi_kernel_desc<MergeDeltaBody<8>>("merge_delta_g8");
const MultiKernel kmRelabel = multi_kernel_desc<RelabelBody>("relabel");

MergeArgs make_args(const DevBM& m, int32_t B, int32_t np, const MergeGrid& grid) {
  MergeArgs a{};
  a.xlx = m.xlx;
  a.optr = m.optr; a.ocol = m.ocol; a.iptr = m.iptr; a.icol = m.icol;
  a.ocnt = m.ocnt; a.icnt = m.icnt; a.d_out = m.d_out; a.d_in = m.d_in;
  a.ld_out = m.ld_out; a.ld_in = m.ld_in; a.dSout = m.dSout; a.ambout = m.ambout;
  a.ambin = m.ambin; a.sinfull = m.sinfull;
  a.B = B;
  a.np = np;
  a.ref_grid = grid.on;
  a.keep_dS = grid.dS;
  a.keep_dsin = grid.dsin;
  a.pdS = grid.dS;
  return a;
}

}  // namespace

void merge_proposals(const DevBM& m, int32_t B, int32_t np, uint64_t seed, uint32_t seq,
                     int32_t* props, cudaStream_t st, const MergeGrid& grid) {
  MergeArgs a = make_args(m, B, np, grid);
  a.seed = seed;
  a.seq = seq;
  a.props = props;
  if (B > 0 && np > 0) launch_single<MergePropsBody>(a, vg_merge_delta(B), st);
}

void merge_delta(const DevBM& m, int32_t B, int32_t E, int32_t np, const int32_t* props,
                 double* dS, int32_t* best, double* best_dS, cudaStream_t st, int32_t exact,
                 const MergeGrid& grid) {
  MergeArgs a = make_args(m, B, np, grid);
  a.exact = exact;
  a.props_in = props;
  a.dS = dS;
  a.best = best;
  a.best_dS = best_dS;
  if (!a.pdS) a.pdS = dS;
  if (B <= 0) return;
  if (short_rows(B, E)) {
    launch_single<MergeDeltaBody<8>>(a, vg_merge_delta(B), st);
  } else if (!a.pdS) {
    launch_single<MergeDeltaBody<32>>(a, vg_merge_delta(B), st);
  } else {
    launch_single<MergePropDeltaBody>(a, vg_merge_prop(B, np), st);
    launch_single<MergeBestBody>(a, vg_merge_delta(B), st);
  }
}

void relabel(int32_t* part, int32_t N, const int32_t* map, cudaStream_t st) {
  RelabelArgs a{part, map, N, 0};
  if (N > 0) launch_single<RelabelBody>(a, ceil_div(N, 256), st);
}

void add_merge_props(Slot& s, const DevBM& m, int32_t B, int32_t np, uint64_t seed, uint32_t seq,
                     int32_t* props, const MergeGrid& grid) {
  MergeArgs a = make_args(m, B, np, grid);
  a.seed = seed;
  a.seq = seq;
  a.props = props;
  slot_push(slot_bind(s, kmMergeProps), a, B > 0 && np > 0 ? vg_merge_delta(B) : 0);
}

void add_merge_delta(Slot& s32, Slot& s8, Slot& sbest, const DevBM& m, int32_t B, int32_t E,
                     int32_t np,
                     const int32_t* props, double* dS, int32_t* best, double* best_dS,
                     int32_t exact, const MergeGrid& grid) {
  MergeArgs a = make_args(m, B, np, grid);
  a.exact = exact;
  a.props_in = props;
  a.dS = dS;
  a.best = best;
  a.best_dS = best_dS;
  if (!a.pdS) a.pdS = dS;
  if (B <= 0) return;
  if (short_rows(B, E) || !a.pdS) {
    slot_push(slot_bind(s8, kmMergeDelta8), a, vg_merge_delta(B));
  } else {
    slot_push(slot_bind(s32, kmMergeDelta), a, vg_merge_prop(B, np));
    slot_push(slot_bind(sbest, kmMergeBest), a, vg_merge_delta(B));
  }
}

void add_relabel(Slot& s, int32_t* part, int32_t N, const int32_t* map) {
  RelabelArgs a{part, map, N, 0};
  slot_push(slot_bind(s, kmRelabel), a, ceil_div(N, 256));
}

}  // namespace sbp
