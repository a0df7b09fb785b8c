// Host utilities of the C ABI: the seeded DCSBM generator that stands in for
// the GraphChallenge static graphs, the CSR builder and TSV reader with the
// semantics of GSAP/load.hpp, and the evaluator of GSAP/evaluate.
#include "../../include/sbp.h"
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <string>
#include <vector>

struct sbp_edges {
  int32_t N = 0;
  std::vector<int32_t> src, dst, truth;
  std::vector<uint32_t> w;
};

namespace sbp {
sbp_status host_fail(sbp_status st, const char* msg);
}

namespace {

using sbp::P4;

// Draw k of stream `stream` for item `idx` (key = seed).
inline P4 gen_draw(uint64_t seed, uint32_t stream, uint32_t idx, uint32_t k) {
  return sbp::philox4x32_10(idx, sbp::kRngGenerate, stream, k, (uint32_t)seed,
                            (uint32_t)(seed >> 32));
}
inline double unit_open(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

// Standard normal by Box-Muller from one Philox block.
inline double normal(const P4& x) {
  double u1 = unit_open(x.v[0]), u2 = unit_open(x.v[1]);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

// Gamma(alpha, 1) by Marsaglia & Tsang (2000), "A simple method for
// generating gamma variables"; alpha < 1 through Gamma(alpha+1) U^(1/alpha).
double gamma_draw(uint64_t seed, uint32_t idx, double alpha) {
  double boost = 1.0;
  uint32_t k = 0;
  if (alpha < 1.0) {
    P4 x = gen_draw(seed, 1, idx, k++);
    boost = std::pow(unit_open(x.v[2]), 1.0 / alpha);
    alpha += 1.0;
  }
  double d = alpha - 1.0 / 3.0, c = 1.0 / std::sqrt(9.0 * d);
  for (;;) {
    P4 x = gen_draw(seed, 1, idx, k++);
    double z = normal(x);
    double v = 1.0 + c * z;
    if (v <= 0.0) continue;
    v = v * v * v;
    double u = unit_open(x.v[2]);
    if (std::log(u) < 0.5 * z * z + d - d * v + d * std::log(v)) return d * v * boost;
  }
}

}  // namespace

namespace sbp {

// The generator's first stages, shared by the host generator and the device
// one: the planted labels (block proportions ~ Dirichlet(alpha), sizes, a
// Fisher-Yates shuffle) and the running weights k^-exponent of the
// out-degrees on [deg_min, deg_max].
sbp_status dcsbm_labels(const sbp_dcsbm_params* p, std::vector<int32_t>& truth,
                        std::vector<double>& cdf) {
  const int32_t N = p->N, B = p->B;
  if (N < 2 || B < 1 || B > N || !(p->alpha > 0.0) || p->p_in < 0.0 || p->p_in > 1.0 ||
      p->deg_min < 1 || p->deg_max < p->deg_min || p->deg_max >= N)
    return sbp::host_fail(SBP_ERR_INVALID, "bad DCSBM parameters");
  const uint64_t seed = p->seed;
  // block proportions ~ Dirichlet(alpha)
  std::vector<double> prop(B);
  double tot = 0.0;
  for (int32_t b = 0; b < B; ++b) tot += (prop[b] = gamma_draw(seed, (uint32_t)b, p->alpha));
  // block sizes: floor(N p_b), remainder to the largest fractions, >= 1 each
  std::vector<int64_t> size(B);
  std::vector<std::pair<double, int32_t>> frac(B);
  int64_t used = 0;
  for (int32_t b = 0; b < B; ++b) {
    double x = (double)N * prop[b] / tot;
    size[b] = (int64_t)std::floor(x);
    frac[b] = {x - (double)size[b], b};
    used += size[b];
  }
  std::sort(frac.begin(), frac.end(), [](auto& a, auto& c) {
    return a.first != c.first ? a.first > c.first : a.second < c.second;
  });
  for (int64_t i = 0; used < N; ++i, ++used) size[frac[i % B].second]++;
  for (int32_t b = 0; b < B; ++b) {
    while (size[b] == 0) {
      int32_t big = (int32_t)(std::max_element(size.begin(), size.end()) - size.begin());
      size[big]--;
      size[b]++;
    }
  }
  // labels, shuffled (Fisher-Yates)
  truth.resize(N);
  {
    int32_t v = 0;
    for (int32_t b = 0; b < B; ++b)
      for (int64_t i = 0; i < size[b]; ++i) truth[v++] = b;
    for (int32_t i = N - 1; i > 0; --i) {
      P4 x = gen_draw(seed, 2, (uint32_t)i, 0);
      int32_t j = (int32_t)sbp::scale_draw(x.v[0], (uint64_t)i + 1);
      std::swap(truth[i], truth[j]);
    }
  }
  // out-degrees ~ k^-exponent on [deg_min, deg_max]
  cdf.clear();
  for (int32_t k = p->deg_min; k <= p->deg_max; ++k)
    cdf.push_back((cdf.empty() ? 0.0 : cdf.back()) + std::pow((double)k, -p->exponent));
  return SBP_OK;
}

}  // namespace sbp

extern "C" {

sbp_status sbp_dcsbm_generate(const sbp_dcsbm_params* p, sbp_edges** out) {
  if (!p || !out) return sbp::host_fail(SBP_ERR_INVALID, "NULL argument");
  *out = nullptr;
  std::vector<int32_t> truth;
  std::vector<double> cdf;
  sbp_status st = sbp::dcsbm_labels(p, truth, cdf);
  if (st != SBP_OK) return st;
  const int32_t N = p->N, B = p->B;
  const uint64_t seed = p->seed;
  sbp_edges* g = new (std::nothrow) sbp_edges();
  if (!g) return sbp::host_fail(SBP_ERR_NOMEM, "host allocation");
  g->N = N;
  g->truth.swap(truth);
  std::vector<int32_t> deg(N);
  for (int32_t v = 0; v < N; ++v) {
    P4 x = gen_draw(seed, 3, (uint32_t)v, 0);
    double u = unit_open(x.v[0]) * cdf.back();
    int32_t k = (int32_t)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
    deg[v] = p->deg_min + std::min<int32_t>(k, (int32_t)cdf.size() - 1);
  }
  // members of each block with cumulative degree weights
  std::vector<std::vector<int32_t>> mem(B);
  std::vector<std::vector<uint64_t>> cum(B);
  for (int32_t v = 0; v < N; ++v) {
    int32_t b = g->truth[v];
    mem[b].push_back(v);
    cum[b].push_back((cum[b].empty() ? 0 : cum[b].back()) + (uint64_t)deg[v]);
  }
  // edges: own block with probability p_in, else a uniform other block;
  // destination proportional to degree; no self-loops, no repeated edges
  const uint64_t pin_scaled = (uint64_t)std::llround(p->p_in * 4294967296.0);
  std::vector<int32_t> tgt;
  for (int32_t u = 0; u < N; ++u) {
    tgt.clear();
    for (int32_t k = 0; k < deg[u]; ++k) {
      for (uint32_t att = 0; att < 64; ++att) {
        P4 x = gen_draw(seed, 4, (uint32_t)u, ((uint32_t)k << 8) | att);
        int32_t b = g->truth[u];
        if (B > 1 && (uint64_t)x.v[0] >= pin_scaled) {
          int32_t c = (int32_t)(x.v[1] % (uint32_t)(B - 1));
          b = c >= b ? c + 1 : c;
        }
        uint64_t t = sbp::scale_draw(x.v[2], cum[b].back());
        int32_t i = (int32_t)(std::upper_bound(cum[b].begin(), cum[b].end(), t) - cum[b].begin());
        int32_t v = mem[b][i];
        if (v == u || std::find(tgt.begin(), tgt.end(), v) != tgt.end()) continue;
        tgt.push_back(v);
        g->src.push_back(u);
        g->dst.push_back(v);
        break;
      }
    }
  }
  g->w.assign(g->src.size(), 1u);
  *out = g;
  return SBP_OK;
}

sbp_status sbp_edges_size(const sbp_edges* e, int32_t* N, int32_t* E) {
  if (!e) return sbp::host_fail(SBP_ERR_INVALID, "NULL edges");
  if (N) *N = e->N;
  if (E) *E = (int32_t)e->src.size();
  return SBP_OK;
}

sbp_status sbp_edges_copy(const sbp_edges* e, int32_t* src, int32_t* dst, uint32_t* w,
                          int32_t* truth) {
  if (!e) return sbp::host_fail(SBP_ERR_INVALID, "NULL edges");
  size_t E = e->src.size();
  if (src) std::memcpy(src, e->src.data(), 4 * E);
  if (dst) std::memcpy(dst, e->dst.data(), 4 * E);
  if (w) std::memcpy(w, e->w.data(), 4 * E);
  if (truth) std::memcpy(truth, e->truth.data(), 4 * (size_t)e->N);
  return SBP_OK;
}

void sbp_edges_free(sbp_edges* e) { delete e; }

sbp_status sbp_csr_from_edges(int32_t N, int32_t E, const int32_t* src, const int32_t* dst,
                              const uint32_t* w, int32_t* out_ptr, int32_t* out_idx,
                              uint32_t* out_w, int32_t* in_ptr, int32_t* in_idx, uint32_t* in_w,
                              uint32_t* deg_out, uint32_t* deg_in) {
  if (N < 1 || E < 0) return sbp::host_fail(SBP_ERR_INVALID, "bad sizes");
  std::fill(out_ptr, out_ptr + N + 1, 0);
  std::fill(in_ptr, in_ptr + N + 1, 0);
  std::fill(deg_out, deg_out + N, 0u);
  std::fill(deg_in, deg_in + N, 0u);
  for (int32_t j = 0; j < E; ++j) {
    if (src[j] < 0 || src[j] >= N || dst[j] < 0 || dst[j] >= N)
      return sbp::host_fail(SBP_ERR_INVALID, "edge endpoint out of range");
    out_ptr[src[j] + 1]++;
    in_ptr[dst[j] + 1]++;
  }
  for (int32_t v = 0; v < N; ++v) {
    out_ptr[v + 1] += out_ptr[v];
    in_ptr[v + 1] += in_ptr[v];
  }
  std::vector<int32_t> co(out_ptr, out_ptr + N), ci(in_ptr, in_ptr + N);
  // load.hpp:86-117: rows keep the edge order of the input
  for (int32_t j = 0; j < E; ++j) {
    uint32_t x = w ? w[j] : 1u;
    int32_t po = co[src[j]]++, pi = ci[dst[j]]++;
    out_idx[po] = dst[j];
    out_w[po] = x;
    in_idx[pi] = src[j];
    in_w[pi] = x;
    deg_out[src[j]] += x;
    deg_in[dst[j]] += x;
  }
  return SBP_OK;
}

// load.hpp:50-65 parses each line with 32-bit unsigned positions: a missing
// tab becomes 0xFFFFFFFF, so the next field starts at position 0 again.
static bool parse_line(const std::string& line, long long* from, long long* to, double* wt) {
  try {
    uint32_t start = 0;
    uint32_t tab = (uint32_t)line.find('\t');
    *from = (long long)std::stoul(line.substr(start, (uint32_t)(tab - start)));
    start = tab + 1;
    tab = (uint32_t)line.find('\t', start);
    *to = (long long)std::stoul(line.substr(start, (uint32_t)(tab - start)));
    start = tab + 1;
    tab = (uint32_t)line.find('\t', start);
    *wt = (double)std::stof(line.substr(start, (uint32_t)(tab - start)));
    return true;
  } catch (...) {
    return false;
  }
}

sbp_status sbp_load_tsv(const char* path, const char* truth_path, sbp_edges** out) {
  if (!path || !out) return sbp::host_fail(SBP_ERR_INVALID, "NULL argument");
  *out = nullptr;
  std::ifstream f(path);
  if (!f.is_open()) return sbp::host_fail(SBP_ERR_INVALID, "cannot open graph file");
  sbp_edges* g = new (std::nothrow) sbp_edges();
  if (!g) return sbp::host_fail(SBP_ERR_NOMEM, "host allocation");
  std::string line;
  long long N = 0;
  while (std::getline(f, line)) {
    long long a, b;
    double w;
    if (!parse_line(line, &a, &b, &w)) {
      delete g;
      return sbp::host_fail(SBP_ERR_INVALID, "unparsable line in graph file");
    }
    g->src.push_back((int32_t)(a - 1));
    g->dst.push_back((int32_t)(b - 1));
    g->w.push_back((uint32_t)(float)w);
    if (a > N) N = a;  // load.hpp:76: N is the largest source id
  }
  for (size_t j = 0; j < g->src.size(); ++j) {
    if (g->src[j] < 0 || g->dst[j] < 0 || g->dst[j] >= N) {
      delete g;
      return sbp::host_fail(SBP_ERR_INVALID, "vertex id out of [1, N]");
    }
  }
  g->N = (int32_t)N;
  g->truth.assign((size_t)N, -1);
  if (truth_path) {
    std::ifstream t(truth_path);
    if (!t.is_open()) {
      delete g;
      return sbp::host_fail(SBP_ERR_INVALID, "cannot open truth file");
    }
    size_t i = 0;
    while (std::getline(t, line) && i < (size_t)N) {
      size_t tab = line.find('\t');
      if (tab == std::string::npos) continue;
      try {
        g->truth[i++] = (int32_t)std::stoul(line.substr(tab + 1)) - 1;
      } catch (...) {
        delete g;
        return sbp::host_fail(SBP_ERR_INVALID, "unparsable truth line");
      }
    }
  }
  *out = g;
  return SBP_OK;
}

sbp_status sbp_evaluate(int32_t n, const int32_t* truth, const int32_t* given, double* recall,
                        double* precision, double* nmi) {
  if (n < 1 || !truth || !given) return sbp::host_fail(SBP_ERR_INVALID, "bad arguments");
  int32_t Bt = 0, Bg = 0;
  for (int32_t i = 0; i < n; ++i) {
    if (given[i] < 0) return sbp::host_fail(SBP_ERR_INVALID, "negative label");
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
  if (N == 0) return sbp::host_fail(SBP_ERR_INVALID, "no vertex has a known label");
  int64_t same = 0, same1 = 0, same2 = 0;
  for (int64_t c : tab) same += c * (c - 1) / 2;
  for (int64_t c : rows) same1 += c * (c - 1) / 2;
  for (int64_t c : cols) same2 += c * (c - 1) / 2;
  if (recall) *recall = same1 ? (double)same / (double)same1 : 1.0;
  if (precision) *precision = same2 ? (double)same / (double)same2 : 1.0;
  double H1 = 0, H2 = 0, MI = 0;
  for (int64_t c : rows)
    if (c) { double q = (double)c / N; H1 -= q * std::log(q); }
  for (int64_t c : cols)
    if (c) { double q = (double)c / N; H2 -= q * std::log(q); }
  for (int32_t i = 0; i < Bt; ++i)
    for (int32_t j = 0; j < Bg; ++j) {
      int64_t c = tab[(size_t)i * Bg + j];
      if (!c) continue;
      double pij = (double)c / N;
      MI += pij * std::log(pij / (((double)rows[i] / N) * ((double)cols[j] / N)));
    }
  if (nmi) *nmi = (H1 + H2) > 0 ? 2.0 * std::fabs(MI) / (std::fabs(H1) + std::fabs(H2)) : 1.0;
  return SBP_OK;
}

}  // extern "C"
