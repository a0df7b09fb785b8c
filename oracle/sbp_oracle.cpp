// CPU ORACLE — test infrastructure only.
//
// A sequential, FP64 restatement of the GSAP stochastic block partitioner
// (chih-chun-chang/GSAP).  Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg may load this library; it is the checker, never the
// product.  Each function cites the reference file:line it restates.
//
// Parity pins (see tests/test_oracle_pins.py):
//   * the nodal and merge dS terms are compared with the reference's own
//     kernels (GSAP/kernels.hpp), compiled for the host by oracle/build_ref.sh
//     and run in FP32 on the same inputs;
//   * the evaluator is compared with GSAP/evaluate/evaluate.hpp;
//   * the loader semantics are compared with GSAP/load.hpp on the bundled
//     1k/5k GraphChallenge graphs.
//
// Deliberate differences from the reference, shared with the product:
//   * RNG: Philox4x32-10 (Salmon et al., SC'11) keyed by (seed, purpose,
//     sequence number, index) instead of curand XORWOW seeded by clock64()
//     (kernels.hpp:655-657).  Sampling is an exact integer inverse CDF
//     instead of a float running sum, so the float "scan misses" fallback of
//     kernels.hpp:750,786 never fires (the fallback to block 0 is kept for
//     the second merge hop, which can run out of candidates != r).
//   * Arithmetic: FP64 with log2() instead of FP32 __log2f (fast-math).
//   * Q3 (kernels.hpp:1348-1358) reads csr_in_adj_wgt[i] past the end of the
//     block row; here the tail uses the vertex list's own weight, and the
//     move is flagged so the pin test can leave it out.
//   * Q16 (partition.hpp:335-336): every block gets its proposals.

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <set>
#include <vector>

namespace {

// ---------------------------------------------------------------- Philox ---
// Philox4x32-10, written from the published description (Salmon, Moraes,
// Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11).
struct P4 { uint32_t v[4]; };

inline void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
}

P4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
  uint32_t x0 = c0, x1 = c1, x2 = c2, x3 = c3;
  for (int round = 0; round < 10; ++round) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo(0xD2511F53u, x0, hi0, lo0);
    mulhilo(0xCD9E8D57u, x2, hi1, lo1);
    uint32_t y0 = hi1 ^ x1 ^ k0;
    uint32_t y1 = lo1;
    uint32_t y2 = hi0 ^ x3 ^ k1;
    uint32_t y3 = lo0;
    x0 = y0; x1 = y1; x2 = y2; x3 = y3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return P4{{x0, x1, x2, x3}};
}

// Draw streams.  One Philox call per (purpose, sequence number, index).
enum : uint32_t { RNG_NODAL_VERTEX = 1, RNG_NODAL_BLOCK = 2, RNG_MERGE = 3 };

inline P4 draw(uint64_t seed, uint32_t purpose, uint32_t seq, uint32_t idx) {
  return philox(idx, purpose, seq, 0u, (uint32_t)seed, (uint32_t)(seed >> 32));
}

// floor(x * D / 2^32): a uniform integer in [0, D) from one 32-bit word.
inline uint64_t scale_draw(uint32_t x, uint64_t D) { return ((uint64_t)x * D) >> 32; }

// x / 2^32 < B / (d + B), exactly.  Restates the test
// uniform <= accepted_prob[u] with accepted_prob = B/(d+B)
// (kernels.hpp:709-723, 847, 1024).
inline bool accept_random(uint32_t x, uint64_t d, uint64_t B) {
  return (unsigned __int128)x * (unsigned __int128)(d + B) < ((unsigned __int128)B << 32);
}

// ------------------------------------------------------------- structures ---
struct Graph {
  int32_t N = 0, E = 0;
  const int32_t* out_ptr = nullptr;  // N+1
  const int32_t* out_idx = nullptr;
  const uint32_t* out_w = nullptr;
  const int32_t* in_ptr = nullptr;   // N+1
  const int32_t* in_idx = nullptr;
  const uint32_t* in_w = nullptr;
  const uint32_t* deg_out = nullptr;  // weighted, N
  const uint32_t* deg_in = nullptr;
};

// Blockmodel M as two CSRs with ascending columns (the layout
// calculate_new_csr builds, partition.hpp:707-849).  Row pointers carry a
// B+1 sentinel here; the reference keeps B entries and uses nnz for the end
// of the last row (kernels.hpp:161-166).
struct BM {
  int32_t B = 0;
  std::vector<int32_t> optr, ocol, iptr, icol;
  std::vector<uint32_t> ocnt, icnt, d_out, d_in;
  int64_t nnz() const { return (int64_t)ocol.size(); }
};

// partition.hpp:707-849: the blockmodel of a partition.  Row r of the out
// CSR lists every block c with M[r][c] = sum of weights of edges u->v with
// part[u]=r, part[v]=c, ascending c; the in CSR is its transpose; d_out and
// d_in are the row sums (weighted block degrees, kernels.hpp:69-77).
BM build_bm(const Graph& g, const int32_t* part, int32_t B) {
  BM m;
  m.B = B;
  std::vector<uint64_t> keys;
  std::vector<uint32_t> vals;
  keys.reserve(g.E);
  for (int32_t u = 0; u < g.N; ++u) {
    uint64_t ru = (uint32_t)part[u];
    for (int32_t j = g.out_ptr[u]; j < g.out_ptr[u + 1]; ++j) {
      uint64_t cv = (uint32_t)part[g.out_idx[j]];
      keys.push_back((ru << 32) | cv);
    }
  }
  std::vector<int64_t> order(keys.size());
  std::iota(order.begin(), order.end(), 0);
  // weights follow the edge order of the out CSR
  std::vector<uint32_t> w_edge;
  w_edge.reserve(g.E);
  for (int32_t u = 0; u < g.N; ++u)
    for (int32_t j = g.out_ptr[u]; j < g.out_ptr[u + 1]; ++j) w_edge.push_back(g.out_w[j]);
  std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return keys[a] < keys[b]; });
  std::vector<uint64_t> ukey;
  std::vector<uint32_t> ucnt;
  for (size_t t = 0; t < order.size(); ++t) {
    uint64_t k = keys[order[t]];
    if (ukey.empty() || ukey.back() != k) {
      ukey.push_back(k);
      ucnt.push_back(w_edge[order[t]]);
    } else {
      ucnt.back() += w_edge[order[t]];
    }
  }
  m.optr.assign(B + 1, 0);
  m.iptr.assign(B + 1, 0);
  m.d_out.assign(B, 0);
  m.d_in.assign(B, 0);
  m.ocol.resize(ukey.size());
  m.ocnt.resize(ukey.size());
  for (size_t t = 0; t < ukey.size(); ++t) {
    int32_t r = (int32_t)(ukey[t] >> 32), c = (int32_t)(ukey[t] & 0xffffffffu);
    m.optr[r + 1]++;
    m.iptr[c + 1]++;
    m.ocol[t] = c;
    m.ocnt[t] = ucnt[t];
    m.d_out[r] += ucnt[t];
    m.d_in[c] += ucnt[t];
  }
  for (int32_t b = 0; b < B; ++b) {
    m.optr[b + 1] += m.optr[b];
    m.iptr[b + 1] += m.iptr[b];
  }
  // transpose: entries visited in (r, c) order land in column c's row in
  // ascending r
  m.icol.resize(ukey.size());
  m.icnt.resize(ukey.size());
  std::vector<int32_t> cur(m.iptr.begin(), m.iptr.end() - 1);
  for (size_t t = 0; t < ukey.size(); ++t) {
    int32_t r = (int32_t)(ukey[t] >> 32), c = (int32_t)(ukey[t] & 0xffffffffu);
    int32_t p = cur[c]++;
    m.icol[p] = r;
    m.icnt[p] = ucnt[t];
  }
  return m;
}

inline double L2(double x) { return std::log2(x); }

// kernels.hpp:143-182 (calculate_dS_out): old out-row term of block r.
double dS_out_block(const BM& m, int32_t r) {
  double dS = 0.0;
  double ld_r = L2((double)m.d_out[r]);
  for (int32_t i = m.optr[r]; i < m.optr[r + 1]; ++i) {
    double w = (double)m.ocnt[i];
    double p = L2(w) - (ld_r + L2((double)m.d_in[m.ocol[i]]));
    dS += w * p;
  }
  return dS;
}

// kernels.hpp:185-231 (calculate_dS_in) and 494-597 (calculate_dS_in_nodal_r/_s):
// old in-row term of block r, leaving out rows x and y.
double dS_in_block_excl(const BM& m, int32_t r, int32_t x, int32_t y) {
  double dS = 0.0;
  double ld_r = L2((double)m.d_in[r]);
  for (int32_t i = m.iptr[r]; i < m.iptr[r + 1]; ++i) {
    int32_t n = m.icol[i];
    if (n != x && n != y) {
      double w = (double)m.icnt[i];
      double p = L2(w) - (L2((double)m.d_out[n]) + ld_r);
      dS += w * p;
    }
  }
  return dS;
}

// ---------------------------------------------------------- exact-MDL mode --
// GSAP's dS terms above approximate the change of the MDL (merged columns
// kept apart, Q1; old column degrees, Q2; one term per list entry).  The
// exact mode computes the change of the same data term,
//   data_S = sum_cells M log2 M - sum_b d_out[b] log2 d_out[b]
//            - sum_b d_in[b] log2 d_in[b]
// (each row of sum M log2(M / (d_out d_in)) split by its row and column
// sums), over the cells a move or a merge changes; dS = -(change of data_S),
// as in S = model - data_S.  The Metropolis-Hastings acceptance uses the
// Hastings ratio of the proposal distribution GSAP samples from
// (choose_neighbored_node_block, kernels.hpp:877-1032): a neighbour u of v
// in proportion to edge weight, then, with t = b(u), block s with
// probability (M[t][s] + M[s][t] + 1) / (d[t] + B), d = d_out + d_in; this
// is the standard SBP sampler (Peixoto, Phys. Rev. E 89, 012804, 2014).
// The outer loop of exact mode compares partitions (stop test, golden
// section) by the standard description length (mdl with exact = 1).
struct Mode {
  int exact = 0;     // 0: GSAP's dS terms; 1: the exact change of the MDL
  int mh = 0;        // 0: accept iff dS < 0 (GSAP); 1: Metropolis-Hastings
  double beta = 3.0;  // inverse temperature of the MH acceptance (dS in bits)
};

inline double xl2(double x) { return x > 0.0 ? x * L2(x) : 0.0; }

uint32_t cell_at(const BM& m, int32_t r, int32_t c) {
  auto b = m.ocol.begin() + m.optr[r], e = m.ocol.begin() + m.optr[r + 1];
  auto it = std::lower_bound(b, e, c);
  return (it != e && *it == c) ? m.ocnt[it - m.ocol.begin()] : 0u;
}

// v's edge weight to (out) and from (in) each neighbour block, its
// self-loop weight apart.
struct MoveLists {
  std::map<int32_t, int64_t> kout, kin, ktot;  // ktot: both directions, self loops twice
  int64_t self = 0;
};

MoveLists move_lists(const Graph& g, const int32_t* part, int32_t v) {
  MoveLists L;
  for (int32_t j = g.out_ptr[v]; j < g.out_ptr[v + 1]; ++j) {
    int32_t u = g.out_idx[j];
    L.ktot[part[u]] += g.out_w[j];
    if (u == v) L.self += g.out_w[j];
    else L.kout[part[u]] += g.out_w[j];
  }
  for (int32_t j = g.in_ptr[v]; j < g.in_ptr[v + 1]; ++j) {
    int32_t u = g.in_idx[j];
    L.ktot[part[u]] += g.in_w[j];
    if (u != v) L.kin[part[u]] += g.in_w[j];
  }
  return L;
}

// Cell changes of moving v from r to s.
std::map<std::pair<int32_t, int32_t>, int64_t> move_cells(const MoveLists& L, int32_t r, int32_t s) {
  std::map<std::pair<int32_t, int32_t>, int64_t> dl;
  for (const auto& kv : L.kout) {
    dl[{r, kv.first}] -= kv.second;
    dl[{s, kv.first}] += kv.second;
  }
  for (const auto& kv : L.kin) {
    dl[{kv.first, r}] -= kv.second;
    dl[{kv.first, s}] += kv.second;
  }
  if (L.self) {
    dl[{r, r}] -= L.self;
    dl[{s, s}] += L.self;
  }
  return dl;
}

double nodal_delta_exact(const Graph& g, const BM& m, const int32_t* part, int32_t v, int32_t s) {
  const int32_t r = part[v];
  if (r == s) return 0.0;
  MoveLists L = move_lists(g, part, v);
  double cells = 0.0;
  for (const auto& kv : move_cells(L, r, s)) {
    if (kv.second == 0) continue;
    const double x = cell_at(m, kv.first.first, kv.first.second);
    cells += xl2(x + (double)kv.second) - xl2(x);
  }
  const double kO = g.deg_out[v], kI = g.deg_in[v];
  const double dor = m.d_out[r], dos = m.d_out[s], dir = m.d_in[r], dis = m.d_in[s];
  const double degs = xl2(dor - kO) - xl2(dor) + xl2(dos + kO) - xl2(dos) + xl2(dir - kI) -
                      xl2(dir) + xl2(dis + kI) - xl2(dis);
  return -(cells - degs);
}

// log(p(s -> r) / p(r -> s)) of the move, p as in the comment above.
double hastings_log(const Graph& g, const BM& m, const int32_t* part, int32_t v, int32_t s) {
  const int32_t r = part[v];
  const double kv = (double)g.deg_out[v] + g.deg_in[v];
  if (r == s || kv == 0.0) return 0.0;
  MoveLists L = move_lists(g, part, v);
  auto dl = move_cells(L, r, s);
  auto newcell = [&](int32_t a, int32_t b) {
    auto it = dl.find({a, b});
    return (double)cell_at(m, a, b) + (it == dl.end() ? 0.0 : (double)it->second);
  };
  const double Bd = (double)m.B;
  auto dtot = [&](int32_t t) { return (double)m.d_out[t] + m.d_in[t]; };
  double fwd = 0.0, bwd = 0.0;
  // after the move the self-loop entries point at s
  std::map<int32_t, int64_t> kafter = L.ktot;
  if (L.self) {
    kafter[r] -= 2 * L.self;
    kafter[s] += 2 * L.self;
  }
  for (const auto& kv2 : L.ktot) {
    const int32_t t = kv2.first;
    fwd += (double)kv2.second * ((double)cell_at(m, t, s) + cell_at(m, s, t) + 1.0) /
           (dtot(t) + Bd);
  }
  for (const auto& kv2 : kafter) {
    const int32_t t = kv2.first;
    if (kv2.second == 0) continue;
    double dt = dtot(t);
    if (t == r) dt -= kv;
    if (t == s) dt += kv;
    bwd += (double)kv2.second * (newcell(t, r) + newcell(r, t) + 1.0) / (dt + Bd);
  }
  return std::log(bwd) - std::log(fwd);
}

// Acceptance of a move with dS (bits) and log Hastings ratio, uniform x.
inline bool mh_accept(double dS, double logH, uint32_t x, double beta) {
  const double a = -beta * dS * 0.6931471805599453 + logH;
  if (a >= 0.0) return true;
  return std::log((double)x * 2.3283064365386963e-10) < a;
}

// Exact merge dS of block r into s: rows r, s and columns r, s fold into
// row and column s; only cells present in both rows (both columns) and the
// four corner cells change the sum of M log2 M.
double merge_delta_exact(const BM& m, int32_t r, int32_t s) {
  if (r == s) return 0.0;
  double cells = 0.0;
  for (int32_t i = m.optr[r]; i < m.optr[r + 1]; ++i) {
    const int32_t c = m.ocol[i];
    if (c == r || c == s) continue;
    const double a = m.ocnt[i], b = cell_at(m, s, c);
    if (b != 0.0) cells += xl2(a + b) - xl2(a) - xl2(b);
  }
  for (int32_t i = m.iptr[r]; i < m.iptr[r + 1]; ++i) {
    const int32_t t = m.icol[i];
    if (t == r || t == s) continue;
    const double a = m.icnt[i], b = cell_at(m, t, s);
    if (b != 0.0) cells += xl2(a + b) - xl2(a) - xl2(b);
  }
  const double Mrr = cell_at(m, r, r), Mrs = cell_at(m, r, s), Msr = cell_at(m, s, r),
               Mss = cell_at(m, s, s);
  cells += xl2(Mrr + Mrs + Msr + Mss) - xl2(Mrr) - xl2(Mrs) - xl2(Msr) - xl2(Mss);
  const double dor = m.d_out[r], dos = m.d_out[s], dir = m.d_in[r], dis = m.d_in[s];
  const double degs = xl2(dor + dos) - xl2(dor) - xl2(dos) + xl2(dir + dis) - xl2(dir) - xl2(dis);
  return -(cells - degs);
}

// A vertex's neighbour blocks with weights, sorted by block: what
// match_neighbored_block_{out,in} + bb_segsort leave in
// g_csr_{out,in}_adj_block / _wgt (kernels.hpp:1096-1151, partition.hpp:537-547).
struct Entry { int32_t blk; uint32_t w; };

std::vector<Entry> nbr_blocks(const int32_t* ptr, const int32_t* idx, const uint32_t* w,
                              const int32_t* part, int32_t v) {
  std::vector<Entry> out;
  for (int32_t j = ptr[v]; j < ptr[v + 1]; ++j) out.push_back(Entry{part[idx[j]], w[j]});
  std::sort(out.begin(), out.end(), [](const Entry& a, const Entry& b) {
    return a.blk != b.blk ? a.blk < b.blk : a.w < b.w;
  });
  return out;
}

uint32_t weight_from_block(const std::vector<Entry>& lst, int32_t b) {
  // kernels.hpp:1366-1441 (find_csr_in_{r,s}_wgt)
  uint32_t w = 0;
  for (const Entry& e : lst)
    if (e.blk == b) w += e.w;
  return w;
}

// kernels.hpp:1444-1581 (calculate_dS_new_r_out_nodal_new)
double new_r_out(const BM& m, const std::vector<Entry>& L, int32_t r, int32_t s, uint32_t k_out,
                 uint32_t ni_w) {
  double dS = 0.0;
  uint32_t d_new = m.d_out[r] - k_out;
  double ld_new = L2((double)d_new);
  int32_t i = m.optr[r], ie = m.optr[r + 1];
  size_t j = 0, je = L.size();
  bool find = false;
  auto term = [&](uint32_t w, int32_t n) {
    double p = L2((double)w) - (L2((double)m.d_in[n]) + ld_new);
    dS += (double)w * p;
  };
  while (i < ie && j < je) {
    int32_t n1 = m.ocol[i], n2 = L[j].blk;
    if (n1 < n2) {
      uint32_t w = m.ocnt[i];
      int32_t n = n1;
      ++i;
      if (n == r) w -= ni_w;
      if (n == s) { w += ni_w; find = true; }
      if (w > 0) term(w, n);
    } else if (n1 > n2) {
      ++j;  // the reference drops this entry (kernels.hpp:1521-1525)
    } else {
      uint32_t w = m.ocnt[i] - L[j].w;
      int32_t n = n1;
      ++i;
      ++j;
      while (j < je && L[j].blk == n) { w -= L[j].w; ++j; }
      if (n == r) w -= ni_w;
      if (n == s) { w += ni_w; find = true; }
      if (w > 0) term(w, n);
    }
  }
  for (; i < ie; ++i) {
    uint32_t w = m.ocnt[i];
    int32_t n = m.ocol[i];
    if (n == r) w -= ni_w;
    if (n == s) { w += ni_w; find = true; }
    if (w > 0) term(w, n);
  }
  if (!find && ni_w > 0) term(ni_w, s);
  return dS;
}

// kernels.hpp:1584-1726 (calculate_dS_new_s_out_nodal_new)
double new_s_out(const BM& m, const std::vector<Entry>& L, int32_t r, int32_t s, uint32_t k_out,
                 uint32_t ni_w) {
  double dS = 0.0;
  uint32_t d_new = m.d_out[s] + k_out;
  double ld_new = L2((double)d_new);
  int32_t i = m.optr[s], ie = m.optr[s + 1];
  size_t j = 0, je = L.size();
  bool find = false;
  auto finish = [&](uint32_t w, int32_t n) {
    if (n == r) w -= ni_w;
    if (n == s) { w += ni_w; find = true; }
    if (w != 0) {
      double p = L2((double)w) - (L2((double)m.d_in[n]) + ld_new);
      dS += (double)w * p;
    }
  };
  while (i < ie && j < je) {
    int32_t n1 = m.ocol[i], n2 = L[j].blk;
    if (n1 < n2) {
      finish(m.ocnt[i], n1);
      ++i;
    } else if (n1 > n2) {
      finish(L[j].w, n2);  // one term per list entry (kernels.hpp:1648-1652)
      ++j;
    } else {
      uint32_t w = m.ocnt[i] + L[j].w;
      int32_t n = n1;
      ++i;
      ++j;
      while (j < je && L[j].blk == n) { w += L[j].w; ++j; }
      finish(w, n);
    }
  }
  for (; i < ie; ++i) finish(m.ocnt[i], m.ocol[i]);
  for (; j < je; ++j) finish(L[j].w, L[j].blk);
  if (!find && ni_w > 0) {
    double p = L2((double)ni_w) - (L2((double)m.d_in[s]) + ld_new);
    dS += (double)ni_w * p;
  }
  return dS;
}

// kernels.hpp:1153-1250 (calculate_dS_new_r_in_nodal_new)
double new_r_in(const BM& m, const std::vector<Entry>& L, int32_t r, int32_t s, uint32_t k_in) {
  double dS = 0.0;
  uint32_t d_new = m.d_in[r] - k_in;
  double ld_new = L2((double)d_new);
  int32_t i = m.iptr[r], ie = m.iptr[r + 1];
  size_t j = 0, je = L.size();
  auto term = [&](uint32_t w, int32_t n) {
    double p = L2((double)w) - (L2((double)m.d_out[n]) + ld_new);
    dS += (double)w * p;
  };
  while (i < ie && j < je) {
    int32_t n1 = m.icol[i], n2 = L[j].blk;
    uint32_t w;
    int32_t n;
    if (n1 < n2) {
      w = m.icnt[i]; n = n1; ++i;
    } else if (n1 > n2) {
      w = L[j].w; n = n2; ++j;
    } else {
      w = m.icnt[i] - L[j].w; n = n1; ++i; ++j;
      while (j < je && L[j].blk == n) { w -= L[j].w; ++j; }
    }
    if (n != r && n != s && w != 0) term(w, n);
  }
  for (; i < ie; ++i) {
    int32_t n = m.icol[i];
    if (n != r && n != s) term(m.icnt[i], n);
  }
  return dS;
}

// kernels.hpp:1253-1362 (calculate_dS_new_s_in_nodal_new).  The trailing
// list loop (:1348-1358) reads csr_in_adj_wgt[i] with i one past the block
// row (Q3); it uses the list weight here and raises *q3.
double new_s_in(const BM& m, const std::vector<Entry>& L, int32_t r, int32_t s, uint32_t k_in,
                bool* q3) {
  double dS = 0.0;
  uint32_t d_new = m.d_in[s] + k_in;
  double ld_new = L2((double)d_new);
  int32_t i = m.iptr[s], ie = m.iptr[s + 1];
  size_t j = 0, je = L.size();
  auto term = [&](uint32_t w, int32_t n) {
    double p = L2((double)w) - (L2((double)m.d_out[n]) + ld_new);
    dS += (double)w * p;
  };
  while (i < ie && j < je) {
    int32_t n1 = m.icol[i], n2 = L[j].blk;
    uint32_t w;
    int32_t n;
    if (n1 < n2) {
      w = m.icnt[i]; n = n1; ++i;
    } else if (n1 > n2) {
      w = L[j].w; n = n2; ++j;
    } else {
      w = m.icnt[i] + L[j].w; n = n1; ++i; ++j;
      while (j < je && L[j].blk == n) { w += L[j].w; ++j; }
    }
    if (n != r && n != s && w != 0) term(w, n);
  }
  for (; i < ie; ++i) {
    int32_t n = m.icol[i];
    if (n != r && n != s) term(m.icnt[i], n);
  }
  for (; j < je; ++j) {
    int32_t n = L[j].blk;
    if (n != r && n != s) {
      *q3 = true;
      term(L[j].w, n);
    }
  }
  return dS;
}

// kernels.hpp:600-643 (calculate_dS_overall_nodal): dS of moving v from r to s.
// `mag` (optional) receives the sum of the magnitudes of the eight row sums
// the value is the difference of: its FP64 rounding error grows with them.
double nodal_delta(const Graph& g, const BM& m, const double* dS_out, const int32_t* part,
                   int32_t v, int32_t s, bool* q3, double* mag = nullptr) {
  int32_t r = part[v];
  if (mag) *mag = 0.0;
  if (r == s) return 0.0;
  std::vector<Entry> Lo = nbr_blocks(g.out_ptr, g.out_idx, g.out_w, part, v);
  std::vector<Entry> Li = nbr_blocks(g.in_ptr, g.in_idx, g.in_w, part, v);
  uint32_t ni_r = weight_from_block(Li, r);
  uint32_t ni_s = weight_from_block(Li, s);
  const double t[8] = {dS_out[r],
                       dS_out[s],
                       dS_in_block_excl(m, r, r, s),
                       dS_in_block_excl(m, s, r, s),
                       new_r_out(m, Lo, r, s, g.deg_out[v], ni_r),
                       new_s_out(m, Lo, r, s, g.deg_out[v], ni_s),
                       new_r_in(m, Li, r, s, g.deg_in[v]),
                       new_s_in(m, Li, r, s, g.deg_in[v], q3)};
  double d = 0.0;
  d += t[0] + t[1];
  d += t[2] + t[3];
  d -= t[4];
  d -= t[5];
  d -= t[6];
  d -= t[7];
  if (mag)
    for (double x : t) *mag += std::fabs(x);
  return d;
}

// kernels.hpp:233-320 (calculate_dS_new_out): merged out-rows of r and s.
double merge_new_out(const BM& m, int32_t r, int32_t s) {
  int32_t i = m.optr[r], ie = m.optr[r + 1];
  int32_t j = m.optr[s], je = m.optr[s + 1];
  double dS = 0.0;
  uint32_t d_new = m.d_out[s] + m.d_out[r];
  double ld_new = L2((double)d_new);
  auto term = [&](uint32_t w, int32_t n) {
    double p = L2((double)w) - (L2((double)m.d_in[n]) + ld_new);
    dS -= (double)w * p;
  };
  while (i < ie && j < je) {
    int32_t n1 = m.ocol[i], n2 = m.ocol[j];
    if (n1 < n2) { term(m.ocnt[i], n1); ++i; }
    else if (n1 > n2) { term(m.ocnt[j], n2); ++j; }
    else { term(m.ocnt[i] + m.ocnt[j], n1); ++i; ++j; }
  }
  for (; i < ie; ++i) term(m.ocnt[i], m.ocol[i]);
  for (; j < je; ++j) term(m.ocnt[j], m.ocol[j]);
  return dS;
}

// kernels.hpp:322-414 (calculate_dS_new_in): merged in-rows, rows r, s left out.
double merge_new_in(const BM& m, int32_t r, int32_t s) {
  int32_t i = m.iptr[r], ie = m.iptr[r + 1];
  int32_t j = m.iptr[s], je = m.iptr[s + 1];
  double dS = 0.0;
  uint32_t d_new = m.d_in[s] + m.d_in[r];
  double ld_new = L2((double)d_new);
  auto term = [&](uint32_t w, int32_t n) {
    if (n != r && n != s) {
      double p = L2((double)w) - (L2((double)m.d_out[n]) + ld_new);
      dS -= (double)w * p;
    }
  };
  while (i < ie && j < je) {
    int32_t n1 = m.icol[i], n2 = m.icol[j];
    if (n1 < n2) { term(m.icnt[i], n1); ++i; }
    else if (n1 > n2) { term(m.icnt[j], n2); ++j; }
    else { term(m.icnt[i] + m.icnt[j], n1); ++i; ++j; }
  }
  for (; i < ie; ++i) term(m.icnt[i], m.icol[i]);
  for (; j < je; ++j) term(m.icnt[j], m.icol[j]);
  return dS;
}

// The proposals GSAP's merge kernels compute (Q16, partition.hpp:335-336):
// every merge kernel runs on a grid of nnz threads rounded up to 256 (nnz =
// entries of the out CSR), so when B*np exceeds that count, proposals t >= T
// are never drawn or scored; their slots keep what the buffers held (zeros
// in a fresh process, else an earlier merge step's values), and a proposal
// whose partner slot s*np+k lies past T reads that slot's stale in-row term.
// `keep` holds those persistent buffers across the merge steps of one run.
struct MergeKeep {
  int64_t T = INT64_MAX;         // proposals [0, T) are computed
  std::vector<double> dsin;      // in-row terms by proposal slot (dS_in)
};

inline int64_t merge_grid(const BM& m, int ref_grid) {
  return ref_grid ? (m.nnz() + 255) / 256 * 256 : INT64_MAX;
}

// kernels.hpp:417-449 (calculate_dS_overall) for every proposal, then
// kernels.hpp:452-491 (find_best_warp): per block the minimum over its
// proposals, reduced over 32 lanes by halving offsets; on equal values the
// lane further up wins.  Lanes past num_proposals hold (largest finite, 0).
// With `keep`, proposals t >= keep->T keep the dS and target their slots
// already hold.
void merge_deltas(const BM& m, const int32_t* props, int np, double* dS, int32_t* best,
                  double* best_dS, const Mode& md = Mode(), MergeKeep* keep = nullptr) {
  int32_t B = m.B;
  const int64_t n = (int64_t)B * np;
  const int64_t T = keep ? std::min(keep->T, n) : n;
  std::vector<double> dso(B);
  for (int32_t b = 0; b < B; ++b) dso[b] = dS_out_block(m, b);
  std::vector<double> fresh;
  std::vector<double>& dsin = keep ? keep->dsin : fresh;
  if ((int64_t)dsin.size() < n) dsin.resize(n, 0.0);
  for (int64_t t = 0; t < T; ++t) {
    int32_t r = (int32_t)(t / np);
    dsin[t] = dS_in_block_excl(m, r, r, props[t]);
  }
  for (int64_t t = 0; t < T; ++t) {
    int32_t r = (int32_t)(t / np), s = props[t], k = (int32_t)(t % np);
    int64_t sid = (int64_t)s * np + k;
    double d = 0.0;
    if (md.exact) {
      d = merge_delta_exact(m, r, s);
    } else {
      d += dso[r] + dso[s];
      d += dsin[t] + dsin[sid];
      d += merge_new_out(m, r, s);
      d += merge_new_in(m, r, s);
    }
    dS[t] = d;
  }
  for (int32_t r = 0; r < B; ++r) {
    double val[32];
    int32_t who[32];
    for (int l = 0; l < 32; ++l) {
      if (l < np) { val[l] = dS[(size_t)r * np + l]; who[l] = props[(size_t)r * np + l]; }
      else { val[l] = DBL_MAX; who[l] = 0; }
    }
    for (int off = 16; off > 0; off /= 2) {
      double nv[32];
      int32_t nw[32];
      for (int l = 0; l < 32; ++l) {
        double o = (l + off < 32) ? val[l + off] : val[l];
        int32_t ow = (l + off < 32) ? who[l + off] : who[l];
        double mn = std::fmin(val[l], o);
        nv[l] = mn;
        nw[l] = (mn == o) ? ow : who[l];
      }
      std::memcpy(val, nv, sizeof(val));
      std::memcpy(who, nw, sizeof(who));
    }
    best[r] = who[0];
    best_dS[r] = val[0];
  }
}

// kernels.hpp:1034-1093 + partition.hpp:665-704: the MDL.  data_S uses log2,
// the model term natural logs, and only its first part is scaled by E (Q6).
// exact = 1: the standard description length of the degree-corrected SBP,
// in bits: (E h(B^2/E) + N ln B) / ln 2 - data_S with
// h(x) = (1+x) ln(1+x) - x ln x, every term in one base and the whole of
// h scaled by E.  Exact mode searches B on this objective.
double mdl(const BM& m, int32_t N, int32_t E, double* data_S_out, int exact = 0) {
  double data_S = 0.0;
  for (int32_t r = 0; r < m.B; ++r) data_S += dS_out_block(m, r);
  double B = (double)m.B;
  double x = B * B / (double)E;
  double model = exact ? ((double)E * ((1.0 + x) * std::log(1.0 + x) - x * std::log(x)) +
                          (double)N * std::log(B)) / 0.6931471805599453
                       : (double)E * (1.0 + x) * std::log(1.0 + x) - x * std::log(x) +
                             (double)N * std::log(B);
  if (data_S_out) *data_S_out = data_S;
  return model - data_S;
}

// ---------------------------------------------------------------- sampling --
// Entry k of the concatenation out-row ++ in-row of block b (the scan order
// of kernels.hpp:767-783).
struct RowCat {
  const BM& m;
  int32_t b;
  int32_t n_out() const { return m.optr[b + 1] - m.optr[b]; }
  int32_t n() const { return n_out() + (m.iptr[b + 1] - m.iptr[b]); }
  int32_t col(int32_t k) const {
    return k < n_out() ? m.ocol[m.optr[b] + k] : m.icol[m.iptr[b] + k - n_out()];
  }
  uint32_t cnt(int32_t k) const {
    return k < n_out() ? m.ocnt[m.optr[b] + k] : m.icnt[m.iptr[b] + k - n_out()];
  }
};

// First k with prefix_k > t (prefix inclusive).
int32_t pick_row(const RowCat& rc, uint64_t t) {
  uint64_t acc = 0;
  for (int32_t k = 0; k < rc.n(); ++k) {
    acc += rc.cnt(k);
    if (acc > t) return k;
  }
  return -1;
}

// kernels.hpp:726-856 (choose_neighbors + propose_blocks), one proposal.
int32_t merge_proposal(const BM& m, int32_t r, uint64_t seed, uint32_t seq, uint32_t idx) {
  P4 x = draw(seed, RNG_MERGE, seq, idx);
  uint32_t B = (uint32_t)m.B;
  uint64_t deg_r = (uint64_t)m.d_out[r] + m.d_in[r];
  int32_t rnd = (int32_t)(x.v[0] % B);
  if (deg_r == 0) return rnd;
  RowCat rr{m, r};
  int32_t k = pick_row(rr, scale_draw(x.v[1], deg_r));
  int32_t u = k >= 0 ? rr.col(k) : 0;
  uint64_t deg_u = (uint64_t)m.d_out[u] + m.d_in[u];
  if (accept_random(x.v[2], deg_u, B)) return rnd;
  // second hop: s ~ row of u, skipping r; 0 when nothing qualifies
  RowCat ru{m, u};
  int32_t s = 0;
  if (deg_u > 0) {
    int32_t k2 = pick_row(ru, scale_draw(x.v[3], deg_u));
    for (; k2 >= 0 && k2 < ru.n(); ++k2) {
      if (ru.col(k2) != r) { s = ru.col(k2); break; }
    }
  }
  return s;
}

// Per-block draws of a nodal batch (kernels.hpp:942-997 choose_neighbored_block,
// and the per-block uniform of kernels.hpp:1024).
void nodal_block_draws(const BM& m, uint64_t seed, uint32_t seq, std::vector<int32_t>& nbr_s,
                       std::vector<uint8_t>& use_rand) {
  int32_t B = m.B;
  nbr_s.assign(B, 0);
  use_rand.assign(B, 0);
  for (int32_t b = 0; b < B; ++b) {
    P4 x = draw(seed, RNG_NODAL_BLOCK, seq, (uint32_t)b);
    uint64_t deg = (uint64_t)m.d_out[b] + m.d_in[b];
    use_rand[b] = accept_random(x.v[0], deg, (uint64_t)B) ? 1 : 0;
    if (deg > 0) {
      RowCat rc{m, b};
      int32_t k = pick_row(rc, scale_draw(x.v[1], deg));
      nbr_s[b] = k >= 0 ? rc.col(k) : 0;
    }
  }
}

// kernels.hpp:859-939 + 1000-1032: proposal for batch vertex v.
int32_t nodal_proposal(const Graph& g, const int32_t* part, int32_t B, int32_t v, uint64_t seed,
                       uint32_t seq, const std::vector<int32_t>& nbr_s,
                       const std::vector<uint8_t>& use_rand) {
  P4 x = draw(seed, RNG_NODAL_VERTEX, seq, (uint32_t)v);
  int32_t rnd = (int32_t)(x.v[0] % (uint32_t)B);
  uint64_t deg = (uint64_t)g.deg_out[v] + g.deg_in[v];
  if (deg == 0) return rnd;
  uint64_t t = scale_draw(x.v[1], deg);
  uint64_t acc = 0;
  int32_t u_node = 0;
  bool found = false;
  for (int32_t j = g.out_ptr[v]; j < g.out_ptr[v + 1] && !found; ++j) {
    acc += g.out_w[j];
    if (acc > t) { u_node = g.out_idx[j]; found = true; }
  }
  for (int32_t j = g.in_ptr[v]; j < g.in_ptr[v + 1] && !found; ++j) {
    acc += g.in_w[j];
    if (acc > t) { u_node = g.in_idx[j]; found = true; }
  }
  int32_t u = part[u_node];
  return use_rand[u] ? rnd : nbr_s[u];
}

// One Jacobi batch (partition.hpp:456-662): all vertices in [lo, hi) are
// judged against the same partition and blockmodel, then the accepted moves
// (dS < 0, kernels.hpp:634-640) are applied together.  Returns the sum of
// accepted dS.
double nodal_batch(const Graph& g, std::vector<int32_t>& part, const BM& m, uint64_t seed,
                   uint32_t seq, int32_t lo, int32_t hi, double* dS_out_arr, int32_t* props_out,
                   const Mode& md = Mode()) {
  int32_t B = m.B;
  std::vector<int32_t> nbr_s;
  std::vector<uint8_t> use_rand;
  nodal_block_draws(m, seed, seq, nbr_s, use_rand);
  std::vector<double> dso(B);
  for (int32_t b = 0; b < B; ++b) dso[b] = dS_out_block(m, b);
  std::vector<int32_t> newpart(part);
  double total = 0.0;
  for (int32_t v = lo; v < hi; ++v) {
    int32_t s = nodal_proposal(g, part.data(), B, v, seed, seq, nbr_s, use_rand);
    bool q3 = false;
    double d = md.exact ? nodal_delta_exact(g, m, part.data(), v, s)
                        : nodal_delta(g, m, dso.data(), part.data(), v, s, &q3);
    bool acc = d < 0.0;
    if (md.mh && s != part[v]) {
      P4 x = draw(seed, RNG_NODAL_VERTEX, seq, (uint32_t)v);
      acc = mh_accept(d, hastings_log(g, m, part.data(), v, s), x.v[2], md.beta);
    }
    double rec = 0.0;
    if (acc && s != part[v]) { newpart[v] = s; rec = d; }
    total += rec;
    if (dS_out_arr) dS_out_arr[v - lo] = rec;
    if (props_out) props_out[v - lo] = s;
  }
  part.swap(newpart);
  return total;
}

// partition.hpp:26-78 (carry_out_best_merges).  Blocks are taken in the
// order of their best dS (thrust::sort_by_key over block ids, a stable radix
// sort, partition.hpp:442-447); a merge is skipped when its target already
// maps to the source block.  Labels are then renumbered in ascending order of
// the surviving block ids (std::set, :58-68).  Stops when the ranked list is
// exhausted (the reference would read past it).
int32_t apply_merges(std::vector<int32_t>& part, int32_t B, int32_t B_to_merge,
                     const int32_t* best, const double* best_dS) {
  std::vector<int32_t> ranked(B);
  std::iota(ranked.begin(), ranked.end(), 0);
  std::stable_sort(ranked.begin(), ranked.end(), [&](int32_t a, int32_t b) {
    double x = best_dS[a], y = best_dS[b];
    bool xn = std::isnan(x), yn = std::isnan(y);
    if (xn || yn) return !xn && yn;
    return x < y;
  });
  std::vector<int32_t> block_map(B);
  std::iota(block_map.begin(), block_map.end(), 0);
  int32_t num_merge = 0, counter = 0;
  while (num_merge < B_to_merge && counter < B) {
    int32_t from = ranked[counter];
    int32_t to = block_map[best[from]];
    ++counter;
    if (to != from) {
      for (int32_t i = 0; i < B; ++i)
        if (block_map[i] == from) block_map[i] = to;
      ++num_merge;
    }
  }
  std::set<int32_t> seen(block_map.begin(), block_map.end());
  std::vector<int32_t> reindex(B, B);
  int32_t index = 0;
  for (int32_t b : seen) reindex[b] = index++;
  for (auto& v : part) v = reindex[block_map[v]];
  return index;
}

struct Options {
  uint64_t seed;
  int32_t num_proposals;
  float reduction_rate;
  int32_t max_nodal_itr;
  int32_t num_batches;
  float threshold1;
  float threshold2;
  int32_t window;
  int32_t max_outer;
  Mode mode;
  int32_t ref_grid;  // 1: GSAP's nnz-sized merge grid (Q16), see MergeKeep
};

struct Report {
  int32_t B;
  double S;
  int32_t outer_steps;
  int32_t nodal_itrs;
  int64_t nodal_proposals;
  int64_t accepted;
  double ms_total, ms_merge, ms_nodal, ms_rebuild;
  int32_t status;
};

struct Snapshot {
  int32_t B = 0;
  int32_t B_to_merge = 0;
  double S = std::numeric_limits<double>::infinity();
  std::vector<int32_t> part;
};

using Clock = std::chrono::steady_clock;
inline double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

// One outer step as the golden section sees it: the step's B, its MDL after
// the nodal sweeps, and the sweeps run so far in the whole partition.
struct TraceStep {
  int32_t B;
  double S;
  int32_t itrs;
};

// partition.hpp:852-954 (partition) with the golden-section bookkeeping of
// partition.hpp:80-322 (prepare_for_partition_next).  trace (optional)
// receives one record per outer step.
int run_partition(const Graph& g, const Options& o, int32_t* labels, Report* rep,
                  std::vector<TraceStep>* trace = nullptr) {
  auto t_all = Clock::now();
  Report R{};
  int32_t N = g.N;
  std::vector<int32_t> part(N);
  std::iota(part.begin(), part.end(), 0);
  int32_t B = N;
  int32_t B_to_merge = (int32_t)((float)B * o.reduction_rate);
  auto t0 = Clock::now();
  BM m = build_bm(g, part.data(), B);
  R.ms_rebuild += ms_since(t0);
  uint32_t seq = 0;
  Snapshot large, med, small;
  bool optimal = false;
  double S = 0.0;
  int32_t outer = 0;
  int32_t BS = N / o.num_batches;
  std::vector<double> itr_dS(o.max_nodal_itr);
  // merge buffers persist over the run and start at zero, like GSAP's
  // (allocate_device.hpp:31-73 on a fresh stream-ordered pool)
  std::vector<int32_t> props((size_t)N * o.num_proposals);
  std::vector<double> mdS((size_t)N * o.num_proposals);
  std::vector<int32_t> best(N);
  std::vector<double> best_dS(N);
  MergeKeep keep;
  while (!optimal) {
    if (++outer > o.max_outer) { R.status = 2; break; }
    // merge phase (partition.hpp:900-904)
    t0 = Clock::now();
    keep.T = std::min<int64_t>(merge_grid(m, o.ref_grid), (int64_t)B * o.num_proposals);
    for (int32_t t = 0; t < keep.T; ++t)
      props[t] = merge_proposal(m, t / o.num_proposals, o.seed, seq, (uint32_t)t);
    ++seq;
    merge_deltas(m, props.data(), o.num_proposals, mdS.data(), best.data(), best_dS.data(),
                 o.mode, &keep);
    B = apply_merges(part, B, B_to_merge, best.data(), best_dS.data());
    R.ms_merge += ms_since(t0);
    t0 = Clock::now();
    m = build_bm(g, part.data(), B);
    R.ms_rebuild += ms_since(t0);
    // nodal phase (partition.hpp:906-935)
    std::fill(itr_dS.begin(), itr_dS.end(), 0.0);
    for (int32_t itr = 0; itr < o.max_nodal_itr; ++itr) {
      for (int32_t b = 0; b < o.num_batches; ++b) {
        t0 = Clock::now();
        itr_dS[itr] += nodal_batch(g, part, m, o.seed, seq, b * BS, (b + 1) * BS, nullptr, nullptr,
                                   o.mode);
        ++seq;
        R.nodal_proposals += BS;
        R.ms_nodal += ms_since(t0);
        t0 = Clock::now();
        m = build_bm(g, part.data(), B);
        R.ms_rebuild += ms_since(t0);
      }
      ++R.nodal_itrs;
      S = mdl(m, N, g.E, nullptr, o.mode.exact);
      if (itr >= o.window - 1) {
        bool isf = std::isfinite(large.S) && std::isfinite(med.S) && std::isfinite(small.S);
        double mean = 0.0;
        for (int32_t i = itr - o.window + 1; i < itr; ++i) mean += itr_dS[i];
        mean /= (double)(o.window - 1);
        if (!isf) {
          if (-mean < (double)o.threshold1 * S) break;
        } else {
          if (-mean < (double)o.threshold2 * S) break;
        }
      }
    }
    if (trace) trace->push_back(TraceStep{B, S, R.nodal_itrs});
    // golden section (partition.hpp:80-322)
    Snapshot P;
    P.B = B;
    P.B_to_merge = B_to_merge;
    P.S = S;
    if (P.S <= med.S) {
      if (med.B > P.B) large = med;
      else small = med;
      med = P;
      med.part = part;
    } else {
      if (med.B > P.B) { small = P; small.part = part; }
      else { large = P; large.part = part; }
    }
    const Snapshot* restore = nullptr;
    if (std::isinf(small.S)) {
      restore = &med;
      B_to_merge = (int32_t)((float)med.B * o.reduction_rate);
      if (B_to_merge == 0) optimal = true;
    } else if (large.B - small.B == 2) {
      optimal = true;
      restore = &med;
    } else if ((large.B - med.B) >= (med.B - small.B)) {
      int32_t next_B = med.B + (int32_t)std::round((large.B - med.B) * 0.618);
      restore = &large;
      B_to_merge = large.B - next_B;
    } else {
      int32_t next_B = small.B + (int32_t)std::round((med.B - small.B) * 0.618);
      restore = &med;
      B_to_merge = med.B - next_B;
    }
    bool changed = (restore->part != part) || restore->B != B;
    part = restore->part;
    B = restore->B;
    S = restore->S;
    if (changed) {
      t0 = Clock::now();
      m = build_bm(g, part.data(), B);
      R.ms_rebuild += ms_since(t0);
    }
  }
  R.B = B;
  R.S = S;
  R.outer_steps = outer;
  for (int32_t v = 0; v < N; ++v) labels[v] = part[v];
  R.ms_total = ms_since(t_all);
  if (rep) *rep = R;
  return R.status;
}

// ------------------------------------------------------------ generator ---
// The seeded directed DCSBM graph of the benchmarks and tests, restated from
// its definition so that the reference arm of the benchmark and the tests
// can build the same graph without the product library:
//   * block proportions ~ Dirichlet(alpha): Gamma(alpha, 1) per block by
//     Marsaglia & Tsang, "A simple method for generating gamma variables"
//     (ACM TOMS 26(3), 2000), the normal by Box-Muller, alpha < 1 through
//     Gamma(alpha + 1) * U^(1/alpha);
//   * sizes floor(N p_b), the remainder one vertex each to the largest
//     fractional parts (equal parts: lower block first), every block >= 1
//     (taken from the first largest block);
//   * planted labels block by block, then a Fisher-Yates shuffle;
//   * out-degree k on [deg_min, deg_max] with P(k) ~ k^-exponent, by the
//     first k whose running weight reaches U * total;
//   * each out-edge stays in the source's block with probability p_in,
//     else goes to a uniform other block; the destination is drawn in
//     proportion to degree within that block; self loops and repeated
//     edges are redrawn (64 attempts per edge).
// Philox counter layout (idx, 4, stream, k), key = seed; streams 1 gamma,
// 2 shuffle, 3 degrees, 4 edges.
struct Dcsbm {
  int32_t N, B;
  double alpha, p_in;
  int32_t deg_min, deg_max;
  double exponent;
  uint64_t seed;
};

inline P4 gen(uint64_t seed, uint32_t stream, uint32_t idx, uint32_t k) {
  return philox(idx, 4u, stream, k, (uint32_t)seed, (uint32_t)(seed >> 32));
}
inline double open01(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

double gamma_variate(uint64_t seed, uint32_t block, double alpha) {
  uint32_t k = 0;
  double scale = 1.0;
  if (alpha < 1.0) {
    scale = std::pow(open01(gen(seed, 1, block, k++).v[2]), 1.0 / alpha);
    alpha += 1.0;
  }
  const double d = alpha - 1.0 / 3.0;
  const double c = 1.0 / std::sqrt(9.0 * d);
  while (true) {
    const P4 x = gen(seed, 1, block, k++);
    const double z = std::sqrt(-2.0 * std::log(open01(x.v[0]))) *
                     std::cos(6.283185307179586 * open01(x.v[1]));
    double v = 1.0 + c * z;
    if (!(v > 0.0)) continue;
    v = v * v * v;
    if (std::log(open01(x.v[2])) < 0.5 * z * z + d - d * v + d * std::log(v)) return d * v * scale;
  }
}

// Fills src/dst (capacity cap) and truth (N); returns E, or -1 on bad
// parameters or too small a capacity.
int64_t dcsbm(const Dcsbm& p, int32_t* src, int32_t* dst, int64_t cap, int32_t* truth) {
  const int32_t N = p.N, B = p.B;
  if (N < 2 || B < 1 || B > N || !(p.alpha > 0.0) || p.p_in < 0.0 || p.p_in > 1.0 ||
      p.deg_min < 1 || p.deg_max < p.deg_min || p.deg_max >= N)
    return -1;
  std::vector<double> w(B);
  double wsum = 0.0;
  for (int32_t b = 0; b < B; ++b) wsum += (w[b] = gamma_variate(p.seed, (uint32_t)b, p.alpha));
  std::vector<int64_t> cnt(B);
  std::vector<int32_t> order(B);
  std::vector<double> rest(B);
  int64_t placed = 0;
  for (int32_t b = 0; b < B; ++b) {
    const double share = (double)N * w[b] / wsum;
    cnt[b] = (int64_t)std::floor(share);
    rest[b] = share - (double)cnt[b];
    placed += cnt[b];
    order[b] = b;
  }
  std::sort(order.begin(), order.end(), [&](int32_t a, int32_t c) {
    return rest[a] != rest[c] ? rest[a] > rest[c] : a < c;
  });
  for (int64_t i = 0; placed < N; ++i, ++placed) ++cnt[order[i % B]];
  for (int32_t b = 0; b < B; ++b)
    while (cnt[b] == 0) {
      int32_t big = 0;
      for (int32_t c = 1; c < B; ++c)
        if (cnt[c] > cnt[big]) big = c;
      --cnt[big];
      ++cnt[b];
    }
  int32_t at = 0;
  for (int32_t b = 0; b < B; ++b)
    for (int64_t i = 0; i < cnt[b]; ++i) truth[at++] = b;
  for (int32_t i = N - 1; i > 0; --i) {
    const int32_t j = (int32_t)scale_draw(gen(p.seed, 2, (uint32_t)i, 0).v[0], (uint64_t)i + 1);
    std::swap(truth[i], truth[j]);
  }
  // running weights of the degree law
  std::vector<double> run;
  double acc = 0.0;
  for (int32_t k = p.deg_min; k <= p.deg_max; ++k) run.push_back(acc += std::pow((double)k, -p.exponent));
  std::vector<int32_t> deg(N);
  for (int32_t v = 0; v < N; ++v) {
    const double u = open01(gen(p.seed, 3, (uint32_t)v, 0).v[0]) * run.back();
    int32_t k = 0;
    while (k + 1 < (int32_t)run.size() && run[k] < u) ++k;
    deg[v] = p.deg_min + k;
  }
  std::vector<std::vector<int32_t>> members(B);
  std::vector<std::vector<uint64_t>> upto(B);
  for (int32_t v = 0; v < N; ++v) {
    const int32_t b = truth[v];
    const uint64_t prev = upto[b].empty() ? 0 : upto[b].back();
    members[b].push_back(v);
    upto[b].push_back(prev + (uint64_t)deg[v]);
  }
  const uint64_t stay = (uint64_t)std::llround(p.p_in * 4294967296.0);
  int64_t E = 0;
  std::vector<int32_t> mine;
  for (int32_t u = 0; u < N; ++u) {
    mine.clear();
    for (int32_t k = 0; k < deg[u]; ++k) {
      for (uint32_t att = 0; att < 64; ++att) {
        const P4 x = gen(p.seed, 4, (uint32_t)u, ((uint32_t)k << 8) | att);
        int32_t b = truth[u];
        if (B > 1 && (uint64_t)x.v[0] >= stay) {
          const int32_t c = (int32_t)(x.v[1] % (uint32_t)(B - 1));
          b = c < b ? c : c + 1;
        }
        const uint64_t t = scale_draw(x.v[2], upto[b].back());
        const int32_t i = (int32_t)(std::upper_bound(upto[b].begin(), upto[b].end(), t) -
                                    upto[b].begin());
        const int32_t v = members[b][i];
        if (v == u || std::find(mine.begin(), mine.end(), v) != mine.end()) continue;
        if (E >= cap) return -1;
        mine.push_back(v);
        src[E] = u;
        dst[E] = v;
        ++E;
        break;
      }
    }
  }
  return E;
}

}  // namespace

// ------------------------------------------------------------------ C ABI ---
extern "C" {

// The benchmark DCSBM graph (see dcsbm above): edges into src/dst (capacity
// cap, N * deg_max always suffices), planted labels into truth (N).
// Returns E, or -1 on bad parameters.
int64_t orc_dcsbm(int32_t N, int32_t B, double alpha, double p_in, int32_t deg_min,
                  int32_t deg_max, double exponent, uint64_t seed, int32_t* src, int32_t* dst,
                  int64_t cap, int32_t* truth) {
  Dcsbm p{N, B, alpha, p_in, deg_min, deg_max, exponent, seed};
  return dcsbm(p, src, dst, cap, truth);
}

typedef struct orc_graph {
  int32_t N, E;
  const int32_t* out_ptr;
  const int32_t* out_idx;
  const uint32_t* out_w;
  const int32_t* in_ptr;
  const int32_t* in_idx;
  const uint32_t* in_w;
  const uint32_t* deg_out;
  const uint32_t* deg_in;
} orc_graph;

static Graph to_graph(const orc_graph* x) {
  Graph g;
  g.N = x->N; g.E = x->E;
  g.out_ptr = x->out_ptr; g.out_idx = x->out_idx; g.out_w = x->out_w;
  g.in_ptr = x->in_ptr; g.in_idx = x->in_idx; g.in_w = x->in_w;
  g.deg_out = x->deg_out; g.deg_in = x->deg_in;
  return g;
}

void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  P4 r = philox(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1]);
  std::memcpy(out, r.v, sizeof(r.v));
}

// Blockmodel of a partition; arrays of capacity E (nnz <= E).  Returns nnz.
int64_t orc_build_blockmodel(const orc_graph* xg, const int32_t* part, int32_t B,
                             int32_t* optr, int32_t* ocol, uint32_t* ocnt, int32_t* iptr,
                             int32_t* icol, uint32_t* icnt, uint32_t* d_out, uint32_t* d_in) {
  Graph g = to_graph(xg);
  BM m = build_bm(g, part, B);
  std::copy(m.optr.begin(), m.optr.end(), optr);
  std::copy(m.iptr.begin(), m.iptr.end(), iptr);
  std::copy(m.ocol.begin(), m.ocol.end(), ocol);
  std::copy(m.ocnt.begin(), m.ocnt.end(), ocnt);
  std::copy(m.icol.begin(), m.icol.end(), icol);
  std::copy(m.icnt.begin(), m.icnt.end(), icnt);
  std::copy(m.d_out.begin(), m.d_out.end(), d_out);
  std::copy(m.d_in.begin(), m.d_in.end(), d_in);
  return m.nnz();
}

// dS of moving verts[i] to props[i], every move judged against `part`.
void orc_nodal_delta(const orc_graph* xg, const int32_t* part, int32_t B, int32_t nv,
                     const int32_t* verts, const int32_t* props, double* dS, uint8_t* q3_hit,
                     double* mag) {
  Graph g = to_graph(xg);
  BM m = build_bm(g, part, B);
  std::vector<double> dso(B);
  for (int32_t b = 0; b < B; ++b) dso[b] = dS_out_block(m, b);
  for (int32_t i = 0; i < nv; ++i) {
    bool q3 = false;
    dS[i] = nodal_delta(g, m, dso.data(), part, verts[i], props[i], &q3, mag ? mag + i : nullptr);
    if (q3_hit) q3_hit[i] = q3 ? 1 : 0;
  }
}

// Exact-mode dS (exact = 1) or GSAP's (0) of moving verts[i] to props[i],
// and log Hastings ratios of those moves.
void orc_nodal_delta_mode(const orc_graph* xg, const int32_t* part, int32_t B, int32_t nv,
                          const int32_t* verts, const int32_t* props, int32_t exact,
                          double* dS, double* logH) {
  Graph g = to_graph(xg);
  BM m = build_bm(g, part, B);
  std::vector<double> dso(B);
  for (int32_t b = 0; b < B; ++b) dso[b] = dS_out_block(m, b);
  for (int32_t i = 0; i < nv; ++i) {
    bool q3 = false;
    if (dS)
      dS[i] = exact ? nodal_delta_exact(g, m, part, verts[i], props[i])
                    : nodal_delta(g, m, dso.data(), part, verts[i], props[i], &q3);
    if (logH) logH[i] = hastings_log(g, m, part, verts[i], props[i]);
  }
}

void orc_merge_delta_mode(const orc_graph* xg, const int32_t* part, int32_t B, int32_t np,
                          const int32_t* props, int32_t exact, double* dS, int32_t* best,
                          double* best_dS) {
  Graph g = to_graph(xg);
  BM m = build_bm(g, part, B);
  Mode md;
  md.exact = exact;
  merge_deltas(m, props, np, dS, best, best_dS, md);
}

double orc_nodal_batch_mode(const orc_graph* xg, int32_t* part, int32_t B, uint64_t seed,
                            uint32_t seq, int32_t lo, int32_t hi, int32_t exact, int32_t mh,
                            double beta, double* dS, int32_t* props) {
  Graph g = to_graph(xg);
  std::vector<int32_t> p(part, part + g.N);
  BM m = build_bm(g, p.data(), B);
  Mode md;
  md.exact = exact;
  md.mh = mh;
  md.beta = beta;
  double tot = nodal_batch(g, p, m, seed, seq, lo, hi, dS, props, md);
  std::copy(p.begin(), p.end(), part);
  return tot;
}

// Merge dS of all B*np proposals, best proposal and its dS per block.
void orc_merge_delta(const orc_graph* xg, const int32_t* part, int32_t B, int32_t np,
                     const int32_t* props, double* dS, int32_t* best, double* best_dS) {
  Graph g = to_graph(xg);
  BM m = build_bm(g, part, B);
  merge_deltas(m, props, np, dS, best, best_dS);
}

double orc_mdl(const orc_graph* xg, const int32_t* part, int32_t B, double* data_S) {
  Graph g = to_graph(xg);
  BM m = build_bm(g, part, B);
  return mdl(m, g.N, g.E, data_S);
}

double orc_mdl_mode(const orc_graph* xg, const int32_t* part, int32_t B, int32_t exact,
                    double* data_S) {
  Graph g = to_graph(xg);
  BM m = build_bm(g, part, B);
  return mdl(m, g.N, g.E, data_S, exact);
}

void orc_merge_proposals(const orc_graph* xg, const int32_t* part, int32_t B, int32_t np,
                         uint64_t seed, uint32_t seq, int32_t* props) {
  Graph g = to_graph(xg);
  BM m = build_bm(g, part, B);
  for (int32_t t = 0; t < B * np; ++t) props[t] = merge_proposal(m, t / np, seed, seq, (uint32_t)t);
}

// One nodal batch over [lo, hi): updates part in place, writes the recorded
// dS (0 for rejected moves) and the proposals; returns the accepted sum.
double orc_nodal_batch(const orc_graph* xg, int32_t* part, int32_t B, uint64_t seed, uint32_t seq,
                       int32_t lo, int32_t hi, double* dS, int32_t* props) {
  Graph g = to_graph(xg);
  std::vector<int32_t> p(part, part + g.N);
  BM m = build_bm(g, p.data(), B);
  double tot = nodal_batch(g, p, m, seed, seq, lo, hi, dS, props);
  std::copy(p.begin(), p.end(), part);
  return tot;
}

// One merge step: proposals, dS, best, merges.  Updates part; returns new B.
int32_t orc_merge_step_mode(const orc_graph* xg, int32_t* part, int32_t B, int32_t B_to_merge,
                            int32_t np, uint64_t seed, uint32_t seq, int32_t ref_grid,
                            int32_t* best_out, double* best_dS_out) {
  Graph g = to_graph(xg);
  BM m = build_bm(g, part, B);
  // the first merge step of a run: fresh (zero) merge buffers
  MergeKeep keep;
  keep.T = std::min<int64_t>(merge_grid(m, ref_grid), (int64_t)B * np);
  std::vector<int32_t> props((size_t)B * np, 0);
  for (int64_t t = 0; t < keep.T; ++t)
    props[t] = merge_proposal(m, (int32_t)(t / np), seed, seq, (uint32_t)t);
  std::vector<double> dS((size_t)B * np, 0.0);
  std::vector<int32_t> best(B);
  std::vector<double> bds(B);
  merge_deltas(m, props.data(), np, dS.data(), best.data(), bds.data(), Mode(), &keep);
  if (best_out) std::copy(best.begin(), best.end(), best_out);
  if (best_dS_out) std::copy(bds.begin(), bds.end(), best_dS_out);
  std::vector<int32_t> p(part, part + g.N);
  int32_t nb = apply_merges(p, B, B_to_merge, best.data(), bds.data());
  std::copy(p.begin(), p.end(), part);
  return nb;
}

int32_t orc_merge_step(const orc_graph* xg, int32_t* part, int32_t B, int32_t B_to_merge,
                       int32_t np, uint64_t seed, uint32_t seq, int32_t* best_out,
                       double* best_dS_out) {
  return orc_merge_step_mode(xg, part, B, B_to_merge, np, seed, seq, 0, best_out, best_dS_out);
}

// Merge application alone (for tests of the host merge loop).
int32_t orc_apply_merges(int32_t N, int32_t* part, int32_t B, int32_t B_to_merge,
                         const int32_t* best, const double* best_dS) {
  std::vector<int32_t> p(part, part + N);
  int32_t nb = apply_merges(p, B, B_to_merge, best, best_dS);
  std::copy(p.begin(), p.end(), part);
  return nb;
}

typedef struct orc_options {
  uint64_t seed;
  int32_t num_proposals;
  float reduction_rate;
  int32_t max_nodal_itr;
  int32_t num_batches;
  float threshold1;
  float threshold2;
  int32_t window;
  int32_t max_outer;
  int32_t exact;
  int32_t mh;
  double beta;
  int32_t ref_grid;
} orc_options;

typedef struct orc_report {
  int32_t B;
  double S;
  int32_t outer_steps;
  int32_t nodal_itrs;
  int64_t nodal_proposals;
  int64_t accepted;
  double ms_total, ms_merge, ms_nodal, ms_rebuild;
  int32_t status;
} orc_report;

int orc_partition(const orc_graph* xg, const orc_options* xo, int32_t* labels, orc_report* rep) {
  Graph g = to_graph(xg);
  Options o{xo->seed, xo->num_proposals, xo->reduction_rate, xo->max_nodal_itr, xo->num_batches,
            xo->threshold1, xo->threshold2, xo->window, xo->max_outer, Mode(),
            xo->ref_grid < 0 ? (xo->exact == 0 ? 1 : 0) : xo->ref_grid};
  o.mode.exact = xo->exact;
  o.mode.mh = xo->mh;
  o.mode.beta = xo->beta;
  Report R{};
  int st = run_partition(g, o, labels, &R);
  if (rep) {
    rep->B = R.B; rep->S = R.S; rep->outer_steps = R.outer_steps; rep->nodal_itrs = R.nodal_itrs;
    rep->nodal_proposals = R.nodal_proposals; rep->accepted = R.accepted;
    rep->ms_total = R.ms_total; rep->ms_merge = R.ms_merge; rep->ms_nodal = R.ms_nodal;
    rep->ms_rebuild = R.ms_rebuild; rep->status = R.status;
  }
  return st;
}

// orc_partition with the outer-step trace: up to max_steps records of the
// step's B, MDL and cumulative sweeps; returns the number of steps (or -1
// on a failed run).
int orc_partition_trace(const orc_graph* xg, const orc_options* xo, int32_t* labels,
                        int32_t* steps_B, double* steps_S, int32_t* steps_itrs,
                        int32_t max_steps) {
  Graph g = to_graph(xg);
  Options o{xo->seed, xo->num_proposals, xo->reduction_rate, xo->max_nodal_itr, xo->num_batches,
            xo->threshold1, xo->threshold2, xo->window, xo->max_outer, Mode(),
            xo->ref_grid < 0 ? (xo->exact == 0 ? 1 : 0) : xo->ref_grid};
  o.mode.exact = xo->exact;
  o.mode.mh = xo->mh;
  o.mode.beta = xo->beta;
  std::vector<TraceStep> tr;
  if (run_partition(g, o, labels, nullptr, &tr) != 0) return -1;
  const int32_t n = std::min<int32_t>((int32_t)tr.size(), max_steps);
  for (int32_t i = 0; i < n; ++i) {
    steps_B[i] = tr[i].B;
    steps_S[i] = tr[i].S;
    steps_itrs[i] = tr[i].itrs;
  }
  return (int32_t)tr.size();
}

// Time nodal batches only (the CPU baseline sample): runs `batches` Jacobi
// batches cycling over the batch ranges at the given partition, rebuilding
// the blockmodel after each, and returns the milliseconds spent.
double orc_time_nodal(const orc_graph* xg, int32_t* part, int32_t B, uint64_t seed, int32_t batches,
                      int32_t num_batches) {
  Graph g = to_graph(xg);
  std::vector<int32_t> p(part, part + g.N);
  int32_t BS = g.N / num_batches;
  auto t0 = Clock::now();
  BM m = build_bm(g, p.data(), B);
  for (int32_t k = 0; k < batches; ++k) {
    int32_t b = k % num_batches;
    nodal_batch(g, p, m, seed, (uint32_t)k, b * BS, (b + 1) * BS, nullptr, nullptr);
    m = build_bm(g, p.data(), B);
  }
  double ms = ms_since(t0);
  std::copy(p.begin(), p.end(), part);
  return ms;
}

// evaluate.hpp:18-265 restated with 64-bit pair counts (the reference's int
// counts overflow past N ~ 46k): pairwise recall, pairwise precision, NMI.
void orc_evaluate(int32_t n, const int32_t* truth, const int32_t* given, double* out3) {
  int32_t Bt = 0, Bg = 0;
  for (int32_t i = 0; i < n; ++i) {
    if (truth[i] >= 0) Bt = std::max(Bt, truth[i] + 1);
    Bg = std::max(Bg, given[i] + 1);
  }
  std::vector<int64_t> tab((size_t)Bt * Bg, 0), rows(Bt, 0), cols(Bg, 0);
  int64_t N = 0;
  for (int32_t i = 0; i < n; ++i) {
    if (truth[i] < 0) continue;
    tab[(size_t)truth[i] * Bg + given[i]]++;
    rows[truth[i]]++;
    cols[given[i]]++;
    ++N;
  }
  int64_t same = 0, same1 = 0, same2 = 0;
  for (int64_t c : tab) same += c * (c - 1) / 2;
  for (int64_t c : rows) same1 += c * (c - 1) / 2;
  for (int64_t c : cols) same2 += c * (c - 1) / 2;
  out3[0] = (double)same / (double)same1;
  out3[1] = (double)same / (double)same2;
  double H1 = 0, H2 = 0, MI = 0;
  for (int64_t c : rows)
    if (c) { double p = (double)c / N; H1 -= p * std::log(p); }
  for (int64_t c : cols)
    if (c) { double p = (double)c / N; H2 -= p * std::log(p); }
  for (int32_t i = 0; i < Bt; ++i)
    for (int32_t j = 0; j < Bg; ++j) {
      int64_t c = tab[(size_t)i * Bg + j];
      if (!c) continue;
      double pij = (double)c / N, pi = (double)rows[i] / N, pj = (double)cols[j] / N;
      MI += pij * std::log(pij / (pi * pj));
    }
  out3[2] = (H1 + H2) > 0 ? 2.0 * std::fabs(MI) / (std::fabs(H1) + std::fabs(H2)) : 1.0;
}

}  // extern "C"
