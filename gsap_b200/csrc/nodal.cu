// Nodal batch: proposal, dS and accept for each vertex of a Jacobi batch.
//
// GSAP spends ~25 launches and two bb_segsorts of all E neighbour-block lists
// per batch (partition.hpp:456-662); each of its seven dS kernels has one
// thread walk a whole blockmodel row in a serial sorted merge with the
// vertex's sorted neighbour-block list (kernels.hpp:494-597, 1153-1726).
//
// Here one warp owns one vertex and does everything in one launch:
//   * proposal: Philox draws, an exact integer inverse-CDF pick of a
//     neighbour (a warp prefix scan over its out- then in-entries), then the
//     per-block draws of the batch (kernels.hpp:877-1032);
//   * dS: GSAP's seven terms rewritten as "old row sum + changed columns".
//     A row term  sum_c f(x_c)  with  f(x) = x (log2 x - log2 dcol[c] - L)
//     splits into  sum_c (x log2 x - x log2 dcol[c])  -  L * sum_c x ;
//     the first sum over the unchanged columns is the per-block sum computed
//     once per batch (ambout / ambin), so only the columns the vertex touches
//     are visited: O(deg(v) log(row)) per vertex instead of O(row nnz).  The
//     changed counts are read with binary searches in the CSR rows.
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
constexpr int kListCap = 64;  // neighbour entries per direction staged in shared memory

struct NodalArgs {
  const int32_t *optr, *oidx, *iptr, *iidx;
  const uint32_t *ow, *iw, *kdo, *kdi;
  const int32_t* part;
  const int32_t *bop, *boc, *bip, *bic;
  const uint32_t *bon, *bin, *d_out, *d_in;
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
};

// g(x, a) = x log2 x - x a, zero for x == 0
__device__ __forceinline__ double gterm(uint32_t x, double a) {
  return x == 0u ? 0.0 : (double)x * log2((double)x) - (double)x * a;
}
// f(M; a, b) = M (log2 M - (a + b)), zero for M == 0 (one old term)
__device__ __forceinline__ double fterm(uint32_t m, double a, double b) {
  return m == 0u ? 0.0 : (double)m * (log2((double)m) - (a + b));
}

struct List {
  const int32_t* idx;
  const uint32_t* w;
  const int32_t* part;
  const int32_t* sc;  // staged blocks
  const uint32_t* sw;
  int32_t base, n;
  __device__ __forceinline__ int32_t blk(int k) const {
    return k < kListCap ? sc[k] : __ldg(part + __ldg(idx + base + k));
  }
  __device__ __forceinline__ uint32_t wt(int k) const {
    return k < kListCap ? sw[k] : __ldg(w + base + k);
  }
};

// dS of moving v from r to s (r != s), computed by the whole warp; every
// lane returns the same value.
__device__ double vertex_delta(const NodalArgs& a, int v, int r, int s, int lane, int32_t* sc_o,
                               uint32_t* sw_o, int32_t* sc_i, uint32_t* sw_i) {
  const int32_t o0 = a.optr[v], no = a.optr[v + 1] - o0;
  const int32_t i0 = a.iptr[v], ni = a.iptr[v + 1] - i0;
  for (int k = lane; k < no && k < kListCap; k += 32) {
    sc_o[k] = __ldg(a.part + __ldg(a.oidx + o0 + k));
    sw_o[k] = __ldg(a.ow + o0 + k);
  }
  for (int k = lane; k < ni && k < kListCap; k += 32) {
    sc_i[k] = __ldg(a.part + __ldg(a.iidx + i0 + k));
    sw_i[k] = __ldg(a.iw + i0 + k);
  }
  __syncwarp();
  List LO{a.oidx, a.ow, a.part, sc_o, sw_o, o0, no};
  List LI{a.iidx, a.iw, a.part, sc_i, sw_i, i0, ni};

  // weights of v's edges into / from blocks r and s
  uint32_t koR = 0, koS = 0, niR = 0, niS = 0;
  for (int k = lane; k < no; k += 32) {
    int32_t c = LO.blk(k);
    uint32_t w = LO.wt(k);
    koR += c == r ? w : 0u;
    koS += c == s ? w : 0u;
  }
  for (int k = lane; k < ni; k += 32) {
    int32_t c = LI.blk(k);
    uint32_t w = LI.wt(k);
    niR += c == r ? w : 0u;
    niS += c == s ? w : 0u;
  }
  koR = warp_sum_u(koR);
  koS = warp_sum_u(koS);
  niR = warp_sum_u(niR);
  niS = warp_sum_u(niS);

  const int32_t rO0 = a.bop[r], rO1 = a.bop[r + 1];
  const int32_t sO0 = a.bop[s], sO1 = a.bop[s + 1];
  const int32_t rI0 = a.bip[r], rI1 = a.bip[r + 1];
  const int32_t sI0 = a.bip[s], sI1 = a.bip[s + 1];

  double a4 = 0.0, a5 = 0.0, a6 = 0.0, a7 = 0.0;
  long long m4 = 0, m5 = 0, m6 = 0, m7 = 0;

  // out-entries: rows r and s of the out CSR (kernels.hpp:1444-1726)
  for (int k = lane; k < no; k += 32) {
    int32_t c = LO.blk(k);
    uint32_t w = LO.wt(k);
    uint32_t Msc = row_lookup(a.boc, a.bon, sO0, sO1, c);
    if (c != r && c != s) {
      bool leader = true;
      uint32_t kc = 0;
      for (int q = 0; q < no; ++q) {
        if (LO.blk(q) == c) {
          kc += LO.wt(q);
          if (q < k) leader = false;
        }
      }
      if (leader) {
        double ldc = a.ld_in[c];
        uint32_t Mrc = row_lookup(a.boc, a.bon, rO0, rO1, c);
        uint32_t x = Mrc - kc;
        a4 += gterm(x, ldc) - gterm(Mrc, ldc);
        m4 += (long long)x - (long long)Mrc;
        if (Msc != 0u) {
          uint32_t y = Msc + kc;
          a5 += gterm(y, ldc) - gterm(Msc, ldc);
          m5 += (long long)y - (long long)Msc;
        }
      }
    }
    if (Msc == 0u) {
      // block c absent from row s: one term per list entry
      uint32_t y = w - (c == r ? niS : 0u) + (c == s ? niS : 0u);
      a5 += gterm(y, a.ld_in[c]);
      m5 += (long long)y;
    }
  }
  // in-entries: rows r and s of the in CSR, blocks r and s left out
  for (int k = lane; k < ni; k += 32) {
    int32_t c = LI.blk(k);
    if (c == r || c == s) continue;
    uint32_t w = LI.wt(k);
    double ldc = a.ld_out[c];
    uint32_t Mcs = row_lookup(a.bic, a.bin, sI0, sI1, c);
    bool leader = true;
    uint32_t kc = 0;
    for (int q = 0; q < ni; ++q) {
      if (LI.blk(q) == c) {
        kc += LI.wt(q);
        if (q < k) leader = false;
      }
    }
    if (leader) {
      uint32_t Mcr = row_lookup(a.bic, a.bin, rI0, rI1, c);
      uint32_t x = Mcr - kc;
      a6 += gterm(x, ldc) - gterm(Mcr, ldc);
      m6 += (long long)x - (long long)Mcr;
      if (Mcs != 0u) {
        uint32_t y = Mcs + kc;
        a7 += gterm(y, ldc) - gterm(Mcs, ldc);
        m7 += (long long)y - (long long)Mcs;
      }
    }
    if (Mcs == 0u) {
      a7 += gterm(w, ldc);
      m7 += (long long)w;
    }
  }
  a4 = warp_sum(a4);
  a5 = warp_sum(a5);
  a6 = warp_sum(a6);
  a7 = warp_sum(a7);
  m4 = warp_sum_ll(m4);
  m5 = warp_sum_ll(m5);
  m6 = warp_sum_ll(m6);
  m7 = warp_sum_ll(m7);

  // the (r, s) corner of M; every lane computes the same scalars
  const uint32_t Mrr = row_lookup(a.boc, a.bon, rO0, rO1, r);
  const uint32_t Mrs = row_lookup(a.boc, a.bon, rO0, rO1, s);
  const uint32_t Msr = row_lookup(a.boc, a.bon, sO0, sO1, r);
  const uint32_t Mss = row_lookup(a.boc, a.bon, sO0, sO1, s);
  const double ldi_r = a.ld_in[r], ldi_s = a.ld_in[s];
  const double ldo_r = a.ld_out[r], ldo_s = a.ld_out[s];
  if (Mrr != 0u) {
    uint32_t x = Mrr - koR - niR;
    a4 += gterm(x, ldi_r) - gterm(Mrr, ldi_r);
    m4 += (long long)x - (long long)Mrr;
  }
  if (Mrs != 0u) {
    uint32_t x = Mrs - koS + niR;
    a4 += gterm(x, ldi_s) - gterm(Mrs, ldi_s);
    m4 += (long long)x - (long long)Mrs;
  } else if (niR > 0u) {
    a4 += gterm(niR, ldi_s);
    m4 += (long long)niR;
  }
  if (Msr != 0u) {
    uint32_t x = Msr + koR - niS;
    a5 += gterm(x, ldi_r) - gterm(Msr, ldi_r);
    m5 += (long long)x - (long long)Msr;
  }
  if (Mss != 0u) {
    uint32_t x = Mss + koS + niS;
    a5 += gterm(x, ldi_s) - gterm(Mss, ldi_s);
    m5 += (long long)x - (long long)Mss;
  } else if (koS == 0u && niS > 0u) {
    a5 += gterm(niS, ldi_s);
    m5 += (long long)niS;
  }

  const uint32_t kO = a.kdo[v], kI = a.kdi[v];
  const uint32_t dor = a.d_out[r], dos = a.d_out[s], dir = a.d_in[r], dis = a.d_in[s];
  // old terms (calculate_dS_out, calculate_dS_in_nodal_r/_s)
  double t1 = a.dSout[r] + a.dSout[s];
  double t2 = a.sinfull[r] - fterm(Mrr, ldo_r, ldi_r) - fterm(Msr, ldo_s, ldi_r);
  double t3 = a.sinfull[s] - fterm(Mrs, ldo_r, ldi_s) - fterm(Mss, ldo_s, ldi_s);
  // new rows r and s, out and in
  long long mass4 = (long long)dor + m4;
  long long mass5 = (long long)dos + m5;
  long long mass6 = (long long)dir - (long long)Mrr - (long long)Msr + m6;
  long long mass7 = (long long)dis - (long long)Mrs - (long long)Mss + m7;
  double t4 = a.ambout[r] + a4;
  if (mass4 != 0) t4 -= log2((double)(uint32_t)(dor - kO)) * (double)mass4;
  double t5 = a.ambout[s] + a5;
  if (mass5 != 0) t5 -= log2((double)(uint32_t)(dos + kO)) * (double)mass5;
  double t6 = a.ambin[r] - gterm(Mrr, ldo_r) - gterm(Msr, ldo_s) + a6;
  if (mass6 != 0) t6 -= log2((double)(uint32_t)(dir - kI)) * (double)mass6;
  double t7 = a.ambin[s] - gterm(Mrs, ldo_r) - gterm(Mss, ldo_s) + a7;
  if (mass7 != 0) t7 -= log2((double)(uint32_t)(dis + kI)) * (double)mass7;
  return t1 + t2 + t3 - t4 - t5 - t6 - t7;
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

template <bool GIVEN>
__global__ void __launch_bounds__(kNodalWarps * 32) nodal_kernel(NodalArgs a) {
  __shared__ int32_t sc_o[kNodalWarps][kListCap], sc_i[kNodalWarps][kListCap];
  __shared__ uint32_t sw_o[kNodalWarps][kListCap], sw_i[kNodalWarps][kListCap];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = gridDim.x * kNodalWarps;
  for (int i = blockIdx.x * kNodalWarps + wid; i < a.count; i += nw) {
    int v, s;
    if (GIVEN) {
      v = a.verts[i];
      s = a.props_in[i];
    } else {
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
    int r = a.part[v];
    double d = 0.0;
    if (r != s) d = vertex_delta(a, v, r, s, lane, sc_o[wid], sw_o[wid], sc_i[wid], sw_i[wid]);
    if (lane == 0) {
      if (GIVEN) {
        a.dS_raw[i] = d;
      } else {
        bool acc = d < 0.0;
        a.newlab[i] = acc ? s : r;
        a.rec[i] = acc ? d : 0.0;
        if (a.props_out) a.props_out[i] = s;
      }
    }
    __syncwarp();
  }
}

// One CTA: applies the batch's labels and sums its recorded dS in a fixed
// order (deterministic across runs).
__global__ void commit_kernel(int32_t* part, int32_t lo, int32_t count,
                              const int32_t* __restrict__ newlab, const double* __restrict__ rec,
                              double* slot_sum, long long* slot_acc) {
  __shared__ double sh[1024];
  __shared__ long long shc[1024];
  double s = 0.0;
  long long c = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    int32_t nl = newlab[i];
    if (part[lo + i] != nl) {
      part[lo + i] = nl;
      ++c;
    }
    s += rec[i];
  }
  sh[threadIdx.x] = s;
  shc[threadIdx.x] = c;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sh[threadIdx.x] += sh[threadIdx.x + o];
      shc[threadIdx.x] += shc[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *slot_sum += sh[0];
    *slot_acc += shc[0];
  }
}

NodalArgs make_args(const DevGraph& g, const int32_t* part, const DevBM& m, int32_t B) {
  NodalArgs a{};
  a.optr = g.optr; a.oidx = g.oidx; a.iptr = g.iptr; a.iidx = g.iidx;
  a.ow = g.ow; a.iw = g.iw; a.kdo = g.kdo; a.kdi = g.kdi;
  a.part = part;
  a.bop = m.optr; a.boc = m.ocol; a.bip = m.iptr; a.bic = m.icol;
  a.bon = m.ocnt; a.bin = m.icnt; a.d_out = m.d_out; a.d_in = m.d_in;
  a.ld_out = m.ld_out; a.ld_in = m.ld_in; a.dSout = m.dSout; a.ambout = m.ambout;
  a.ambin = m.ambin; a.sinfull = m.sinfull; a.nbr_s = m.nbr_s; a.use_rand = m.use_rand;
  a.B = B;
  return a;
}

int nodal_grid(int count) {
  int g = (count + kNodalWarps - 1) / kNodalWarps;
  return g < 1 ? 1 : (g > 148 * 64 ? 148 * 64 : g);
}

}  // namespace

void nodal_batch_sample(const DevGraph& g, const int32_t* part, const DevBM& m, int32_t B,
                        uint64_t seed, uint32_t seq, int32_t lo, int32_t count, int32_t* newlab,
                        double* rec, int32_t* props, cudaStream_t st) {
  NodalArgs a = make_args(g, part, m, B);
  a.seed = seed;
  a.seq = seq;
  a.lo = lo;
  a.count = count;
  a.newlab = newlab;
  a.rec = rec;
  a.props_out = props;
  if (count > 0) nodal_kernel<false><<<nodal_grid(count), kNodalWarps * 32, 0, st>>>(a);
}

void nodal_delta_given(const DevGraph& g, const int32_t* part, const DevBM& m, int32_t B,
                       int32_t nv, const int32_t* verts, const int32_t* props, double* dS,
                       cudaStream_t st) {
  NodalArgs a = make_args(g, part, m, B);
  a.count = nv;
  a.verts = verts;
  a.props_in = props;
  a.dS_raw = dS;
  if (nv > 0) nodal_kernel<true><<<nodal_grid(nv), kNodalWarps * 32, 0, st>>>(a);
}

void nodal_commit(int32_t* part, int32_t lo, int32_t count, const int32_t* newlab,
                  const double* rec, double* slot_sum, long long* slot_acc, cudaStream_t st) {
  commit_kernel<<<1, 1024, 0, st>>>(part, lo, count, newlab, rec, slot_sum, slot_acc);
}

}  // namespace sbp
