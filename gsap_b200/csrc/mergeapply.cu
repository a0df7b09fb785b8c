// Merge application on the device: carry_out_best_merges (partition.hpp:26-78)
// without a host round trip.
//
// GSAP ranks the blocks by their best merge dS (thrust::sort_by_key, ties by
// block id, partition.hpp:442-447) and walks that list on the host: block
// `from` merges into the current label of its best target unless that label
// is `from` itself, until B_to_merge merges are made; the surviving labels
// are then renumbered in ascending order (std::set, :58-68).
//
// The walk is a Kruskal pass over the functional graph b -> best[b]: a merge
// is skipped exactly when its target's group already holds `from`, and in a
// functional graph that happens to one edge per cycle only, the cycle's edge
// that comes last in rank order (a tree edge is a bridge and never closes a
// loop; a self-proposal is a cycle of one).  So, with ranks compared as the
// pair (order-preserving key of dS, block id):
//   1. pointer doubling over b -> best[b] gives every block the largest rank
//      on the path of 2^L edges ahead of it, and marks the blocks on cycles
//      (the image of 2^L jumps, 2^L >= B); the blocks whose own edge holds
//      their cycle's largest rank are the skipped ones;
//   2. a radix select (eight 12-bit digits of the 96-bit pair) finds the
//      B_to_merge-th smallest rank among the merges that are not skipped:
//      exactly the merges up to it are made (all of them when there are
//      fewer);
//   3. the made merges form a forest whose roots are the surviving labels
//      (a group takes the label of the block whose own merge was not made);
//      pointer doubling finds each block's root, an exclusive scan over the
//      roots in id order renumbers them.
// Every step is a function of best, best_dS and B_to_merge only, so the map
// is bit-identical to the host walk (apply_merges_host, the oracle's
// apply_merges).  Each body runs on a virtual grid of one job, so a merge
// step of many jobs is one launch per body (multi.cuh).
#include "common.cuh"
#include "kernels.h"
#include "multi.cuh"

namespace sbp {

namespace {

constexpr int kMaThreads = 256;
constexpr int kSelBits = 12;
constexpr int kSelBins = 1 << kSelBits;  // 4096
constexpr int kSelPasses = 8;            // 96 bits = key (64) : id (32)

// sel[] layout: k (rank still wanted, 1-based), mode, digits[8], successes
enum : int { kSelK = 0, kSelMode = 1, kSelDigit = 2, kSelTotal = 10 };
// mode: 0 searching, 1 threshold found, 2 every merge is made, 3 none is
enum : int { kSearching = 0, kFound = 1, kAll = 2, kNone = 3 };

struct MaArgs {
  const int32_t* best;
  const double* best_dS;
  int32_t* map;
  int32_t* out;  // [0] new block count, [1] 1 when a target was out of range
  MergeApplyBufs w;
  int32_t B, K;  // blocks, merges wanted (B_to_merge)
  int32_t round, pass;
};

__device__ __forceinline__ uint64_t rank_key(double x) {
  if (isnan(x)) return ~0ull;
  if (x == 0.0) x = 0.0;  // -0 ranks with +0
  const uint64_t u = (uint64_t)__double_as_longlong(x);
  return (u >> 63) ? ~u : (u | (1ull << 63));
}

// Larger of two ranks (key, id), lexicographic.
__device__ __forceinline__ bool rank_less(uint64_t ka, int32_t ia, uint64_t kb, int32_t ib) {
  return ka < kb || (ka == kb && ia < ib);
}

// Digit p (from the top) of the 96-bit rank key:id.
__device__ __forceinline__ uint32_t sel_digit(uint64_t key, uint32_t id, int p) {
  const int shift = 84 - kSelBits * p;
  if (shift >= 32) return (uint32_t)(key >> (shift - 32)) & (kSelBins - 1);
  return (uint32_t)((key << (32 - shift)) | ((uint64_t)id >> shift)) & (kSelBins - 1);
}

// Whether block b's merge is one the walk makes if it gets that far (not
// the last-ranked edge of a cycle).
__device__ __forceinline__ bool not_skipped(const MaArgs& a, int b, int fin) {
  const uint64_t* mk = fin ? a.w.mkB : a.w.mkA;
  const int32_t* mi = fin ? a.w.miB : a.w.miA;
  return !(a.w.onc[b] && mk[b] == a.w.key[b] && mi[b] == b);
}

// Keys, the first jump and rank of every block; clears the cycle marks,
// the select state and the histogram.
struct MaKeysBody {
  using Args = MaArgs;
  static constexpr int kThreads = kMaThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    const int tid = vb * kThreads + threadIdx.x, stride = vg * kThreads;
    for (int b = tid; b < a.B; b += stride) {
      int t = a.best[b];
      if (t < 0 || t >= a.B) {
        a.out[1] = 1;  // reported to the host (out[] starts at zero); the
        t = b;         // block is then treated as proposing itself
      }
      const uint64_t k = rank_key(a.best_dS[b]);
      a.w.key[b] = k;
      a.w.jA[b] = t;
      a.w.mkA[b] = k;
      a.w.miA[b] = b;
      a.w.onc[b] = 0;
    }
    for (int i = tid; i < kSelBins; i += stride) a.w.hist[i] = 0u;
    if (tid == 0) {
      a.w.sel[kSelK] = a.K;
      a.w.sel[kSelMode] = kSearching;
      a.w.sel[kSelTotal] = 0;
    }
  }
};

// One pointer-doubling round over b -> best[b] carrying the largest rank
// seen (round r reads buffer r & 1, writes the other).
struct MaCycleJumpBody {
  using Args = MaArgs;
  static constexpr int kThreads = kMaThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    const bool odd = a.round & 1;
    const int32_t* ji = odd ? a.w.jB : a.w.jA;
    const uint64_t* ki = odd ? a.w.mkB : a.w.mkA;
    const int32_t* ii = odd ? a.w.miB : a.w.miA;
    int32_t* jo = odd ? a.w.jA : a.w.jB;
    uint64_t* ko = odd ? a.w.mkA : a.w.mkB;
    int32_t* io = odd ? a.w.miA : a.w.miB;
    for (int b = vb * kThreads + threadIdx.x; b < a.B; b += vg * kThreads) {
      const int j = ji[b];
      uint64_t k = ki[b];
      int32_t i = ii[b];
      const uint64_t k2 = ki[j];
      const int32_t i2 = ii[j];
      if (rank_less(k, i, k2, i2)) {
        k = k2;
        i = i2;
      }
      jo[b] = ji[j];
      ko[b] = k;
      io[b] = i;
    }
  }
};

// Blocks on cycles: the image of 2^L jumps.  a.round = L (the buffer of
// the last round's output is L & 1).
struct MaMarkBody {
  using Args = MaArgs;
  static constexpr int kThreads = kMaThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    const int32_t* j = (a.round & 1) ? a.w.jB : a.w.jA;
    for (int b = vb * kThreads + threadIdx.x; b < a.B; b += vg * kThreads) a.w.onc[j[b]] = 1;
  }
};

// Select pass a.pass: histogram of the next digit over the merges that are
// not skipped and match the digits chosen so far.  a.round = L.
struct MaSelHistBody {
  using Args = MaArgs;
  static constexpr int kThreads = kMaThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    __shared__ uint32_t h[kSelBins];
    if (a.w.sel[kSelMode] != kSearching) return;
    for (int i = threadIdx.x; i < kSelBins; i += kThreads) h[i] = 0u;
    __syncthreads();
    const int fin = a.round & 1;
    for (int b = vb * kThreads + threadIdx.x; b < a.B; b += vg * kThreads) {
      if (!not_skipped(a, b, fin)) continue;
      const uint64_t k = a.w.key[b];
      bool match = true;
      for (int q = 0; q < a.pass && match; ++q)
        match = sel_digit(k, (uint32_t)b, q) == (uint32_t)a.w.sel[kSelDigit + q];
      if (match) atomicAdd(&h[sel_digit(k, (uint32_t)b, a.pass)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kSelBins; i += kThreads)
      if (h[i]) atomicAdd(&a.w.hist[i], h[i]);
  }
};

// Select pass a.pass: the bucket holding the k-th candidate; clears the
// histogram for the next pass.  One CTA per job.
struct MaSelPickBody {
  using Args = MaArgs;
  static constexpr int kThreads = kMaThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int, int) {
    __shared__ int sh[33];
    __shared__ uint32_t part[kThreads + 1];
    if (a.w.sel[kSelMode] != kSearching) return;
    constexpr int per = kSelBins / kThreads;  // 16 bins a thread
    uint32_t c[per];
    uint32_t s = 0;
#pragma unroll
    for (int q = 0; q < per; ++q) {
      c[q] = a.w.hist[threadIdx.x * per + q];
      s += c[q];
    }
    // exclusive prefix of the threads' sums (counts fit in 31 bits: <= B)
    int tot = 0;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = (int)s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) sh[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int v = lane < kThreads / 32 ? sh[lane] : 0, vi = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(kFull, vi, o);
        if (lane >= o) vi += y;
      }
      if (lane < kThreads / 32) sh[lane] = vi - v;
      if (lane == 31) sh[32] = vi;
    }
    __syncthreads();
    const int pre = incl - (int)s + sh[wid];
    tot = sh[32];
    const int k = a.w.sel[kSelK];  // read by every thread before any write
    __syncthreads();
    // pass 0 decides whether there is anything to search: no merge wanted,
    // or at least as many wanted as there are to make
    const bool search = a.pass > 0 || (k > 0 && k < tot);
    if (a.pass == 0 && threadIdx.x == 0) {
      a.w.sel[kSelTotal] = tot;
      if (!search) a.w.sel[kSelMode] = k <= 0 ? kNone : kAll;
    }
    // the thread whose range holds the k-th candidate picks the bucket
    if (search) {
      if (pre < k && k <= pre + (int)s) {
        int run = pre;
#pragma unroll
        for (int q = 0; q < per; ++q) {
          if (run < k && k <= run + (int)c[q]) {
            a.w.sel[kSelDigit + a.pass] = threadIdx.x * per + q;
            a.w.sel[kSelK] = k - run;
            if (a.pass == kSelPasses - 1) a.w.sel[kSelMode] = kFound;
          }
          run += (int)c[q];
        }
      }
    }
#pragma unroll
    for (int q = 0; q < per; ++q) a.w.hist[threadIdx.x * per + q] = 0u;
  }
};

// The merges made: parent = best for them, self otherwise; roots flagged
// for the renumbering scan.  a.round = L.
struct MaParentBody {
  using Args = MaArgs;
  static constexpr int kThreads = kMaThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    const int mode = a.w.sel[kSelMode];
    const int fin = a.round & 1;
    for (int b = vb * kThreads + threadIdx.x; b < a.B; b += vg * kThreads) {
      bool made = false;
      if (mode != kNone && not_skipped(a, b, fin)) {
        if (mode == kAll) {
          made = true;
        } else {
          // rank <= the threshold: compare digit by digit from the top
          const uint64_t k = a.w.key[b];
          made = true;
          for (int q = 0; q < kSelPasses; ++q) {
            const uint32_t d = sel_digit(k, (uint32_t)b, q);
            const uint32_t t = (uint32_t)a.w.sel[kSelDigit + q];
            if (d != t) {
              made = d < t;
              break;
            }
          }
        }
      }
      const int t = a.best[b];
      const bool ok = t >= 0 && t < a.B;
      a.w.pA[b] = made && ok ? t : b;
      a.w.root[b] = made && ok ? 0 : 1;
    }
  }
};

// One pointer-doubling round toward the roots (round r reads buffer r & 1).
struct MaRootJumpBody {
  using Args = MaArgs;
  static constexpr int kThreads = kMaThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    const int32_t* pi = (a.round & 1) ? a.w.pB : a.w.pA;
    int32_t* po = (a.round & 1) ? a.w.pA : a.w.pB;
    for (int b = vb * kThreads + threadIdx.x; b < a.B; b += vg * kThreads) po[b] = pi[pi[b]];
  }
};

// map[b] = new id of b's root; the new block count.  a.round = L.
struct MaMapBody {
  using Args = MaArgs;
  static constexpr int kThreads = kMaThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a, int vb, int vg) {
    const int32_t* p = (a.round & 1) ? a.w.pB : a.w.pA;
    for (int b = vb * kThreads + threadIdx.x; b < a.B; b += vg * kThreads)
      a.map[b] = a.w.newid[p[b]];
    if (vb == 0 && threadIdx.x == 0) a.out[0] = a.w.newid[a.B];
  }
};

// Rounds of pointer doubling that cover B: 2^L >= B.
__host__ __device__ __forceinline__ int ma_rounds(int32_t B) {
  int L = 1;
  while (L < 31 && (1ll << L) < (long long)B) ++L;
  return L;
}

// Every step above in one CTA for B <= kMaFusedMax: the same bodies on a
// virtual grid of one block, in the order the separate launches take, with
// a CTA barrier between them instead of a launch (global writes of one
// body are visible to the whole CTA after the barrier).  At the block counts
// of the golden-section phase this is one launch per merge step instead of
// about forty, with the same bits.
constexpr int kMaFusedMax = 4096;
struct MaFusedBody {
  using Args = MaArgs;
  static constexpr int kThreads = kMaThreads, kMinBlocks = 1;
  static constexpr size_t kSmem = 0;
  static __device__ void run(const Args& a0, int, int) {
    __shared__ int sh[kMaThreads / 32 + 1];
    MaArgs a = a0;
    const int L = ma_rounds(a.B);
    MaKeysBody::run(a, 0, 1);
    __syncthreads();
    for (int r = 0; r < L; ++r) {
      a.round = r;
      MaCycleJumpBody::run(a, 0, 1);
      __syncthreads();
    }
    a.round = L;
    MaMarkBody::run(a, 0, 1);
    __syncthreads();
    for (int q = 0; q < kSelPasses; ++q) {
      a.pass = q;
      MaSelHistBody::run(a, 0, 1);
      __syncthreads();
      MaSelPickBody::run(a, 0, 1);
      __syncthreads();
    }
    MaParentBody::run(a, 0, 1);
    __syncthreads();
    for (int r = 0; r < L; ++r) {
      a.round = r;
      MaRootJumpBody::run(a, 0, 1);
      __syncthreads();
    }
    // exclusive scan of the root flags into new ids, newid[B] = the count:
    // each thread a contiguous run of ceil(B / 256) flags
    {
      const int per = (a.B + kMaThreads - 1) / kMaThreads;
      const int b0 = threadIdx.x * per, b1 = min(a.B, b0 + per);
      int local = 0;
      for (int b = b0; b < b1; ++b) local += a.w.root[b];
      const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
      int incl = local;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) sh[wid] = incl;
      __syncthreads();
      if (threadIdx.x == 0) {
        int run = 0;
        for (int k = 0; k < kMaThreads / 32; ++k) {
          const int c = sh[k];
          sh[k] = run;
          run += c;
        }
        sh[kMaThreads / 32] = run;
      }
      __syncthreads();
      int pre = sh[wid] + incl - local;
      for (int b = b0; b < b1; ++b) {
        const int f = a.w.root[b];
        a.w.newid[b] = pre;
        pre += f;
      }
      if (threadIdx.x == 0) a.w.newid[a.B] = sh[kMaThreads / 32];
      __syncthreads();
    }
    a.round = L;
    MaMapBody::run(a, 0, 1);
  }
};

const MultiKernel kmMaKeys = multi_kernel_desc<MaKeysBody>("ma_keys");
const MultiKernel kmMaCycle = multi_kernel_desc<MaCycleJumpBody>("ma_cycle_jump");
const MultiKernel kmMaMark = multi_kernel_desc<MaMarkBody>("ma_mark");
const MultiKernel kmMaHist = multi_kernel_desc<MaSelHistBody>("ma_select_hist");
const MultiKernel kmMaPick = multi_kernel_desc<MaSelPickBody>("ma_select_pick");
const MultiKernel kmMaParent = multi_kernel_desc<MaParentBody>("ma_parent");
const MultiKernel kmMaRoot = multi_kernel_desc<MaRootJumpBody>("ma_root_jump");
const MultiKernel kmMaMap = multi_kernel_desc<MaMapBody>("ma_map");
const MultiKernel kmMaFused = multi_kernel_desc<MaFusedBody>("ma_fused");

int32_t vg_ma(int32_t B) { return std::max(1, std::min(ceil_div(B, kMaThreads), 148 * 8)); }

// Rounds of pointer doubling that cover B: 2^L >= B.
int rounds_for(int32_t B) { return ma_rounds(B); }

MaArgs ma_args(const MergeApplyBufs& w, int32_t B, int32_t K, const int32_t* best,
               const double* best_dS, int32_t* map, int32_t* out) {
  MaArgs a{};
  a.best = best;
  a.best_dS = best_dS;
  a.map = map;
  a.out = out;
  a.w = w;
  a.B = B;
  a.K = K;
  return a;
}

}  // namespace

size_t merge_apply_bytes(int32_t N) {
  size_t b = 0, n = (size_t)std::max(N, 1);
  auto add = [&](size_t elems, size_t sz) { b += ((elems * sz) + 255) & ~size_t(255); };
  add(n, 8);                           // key
  add(n, 4); add(n, 4);                // jA, jB
  add(n, 8); add(n, 8);                // mkA, mkB
  add(n, 4); add(n, 4);                // miA, miB
  add(n, 1);                           // onc
  add(n, 4); add(n, 4);                // pA, pB
  add(n + 1, 4); add(n + 1, 4);        // root flags, newid
  add(2 * ((n + 2047) / 2048) + 2, 4);  // scan tiles
  add(kSelBins, 4);                    // hist
  add(16, 4);                          // sel
  return b;
}

template <class T>
static T* take(char*& p, size_t n) {
  T* r = (T*)p;
  p += ((n * sizeof(T)) + 255) & ~size_t(255);
  return r;
}

MergeApplyBufs merge_apply_carve(void* base, int32_t N) {
  MergeApplyBufs w;
  char* p = (char*)base;
  size_t n = (size_t)std::max(N, 1);
  w.key = take<uint64_t>(p, n);
  w.jA = take<int32_t>(p, n); w.jB = take<int32_t>(p, n);
  w.mkA = take<uint64_t>(p, n); w.mkB = take<uint64_t>(p, n);
  w.miA = take<int32_t>(p, n); w.miB = take<int32_t>(p, n);
  w.onc = take<uint8_t>(p, n);
  w.pA = take<int32_t>(p, n); w.pB = take<int32_t>(p, n);
  w.root = take<int32_t>(p, n + 1); w.newid = take<int32_t>(p, n + 1);
  w.tile = take<int32_t>(p, 2 * ((n + 2047) / 2048) + 2);
  w.hist = take<uint32_t>(p, kSelBins);
  w.sel = take<int32_t>(p, 16);
  return w;
}

void MergeApplySlots::clear() {
  for (Slot* s : all()) s->clear();
}

std::vector<Slot*> MergeApplySlots::all() {
  std::vector<Slot*> v{&fused, &keys};
  for (Slot& s : cyc) v.push_back(&s);
  v.push_back(&mark);
  for (int p = 0; p < kMaSelPasses; ++p) {
    v.push_back(&hist[p]);
    v.push_back(&pick[p]);
  }
  v.push_back(&parent);
  for (Slot& s : rootj) v.push_back(&s);
  for (Slot& s : scan) v.push_back(&s);
  v.push_back(&map);
  return v;
}

void add_merge_apply(MergeApplySlots& s, const MergeApplyBufs& w, int32_t B, int32_t K,
                     const int32_t* best, const double* best_dS, int32_t* map, int32_t* out) {
  if (B <= 0) return;
  MaArgs a = ma_args(w, B, K, best, best_dS, map, out);
  if (B <= kMaFusedMax) {
    slot_push(slot_bind(s.fused, kmMaFused), a, 1);
    return;
  }
  const int32_t vg = vg_ma(B);
  const int L = rounds_for(B);
  slot_push(slot_bind(s.keys, kmMaKeys), a, vg);
  for (int r = 0; r < L; ++r) {
    a.round = r;
    slot_push(slot_bind(s.cyc[r], kmMaCycle), a, vg);
  }
  a.round = L;
  slot_push(slot_bind(s.mark, kmMaMark), a, vg);
  for (int p = 0; p < kMaSelPasses; ++p) {
    a.pass = p;
    slot_push(slot_bind(s.hist[p], kmMaHist), a, vg);
    slot_push(slot_bind(s.pick[p], kmMaPick), a, 1);
  }
  slot_push(slot_bind(s.parent, kmMaParent), a, vg);
  for (int r = 0; r < L; ++r) {
    a.round = r;
    slot_push(slot_bind(s.rootj[r], kmMaRoot), a, vg);
  }
  add_exclusive_scan(s.scan, w.root, w.newid, B, w.tile);
  a.round = L;
  slot_push(slot_bind(s.map, kmMaMap), a, vg);
}

void merge_apply(const MergeApplyBufs& w, int32_t B, int32_t K, const int32_t* best,
                 const double* best_dS, int32_t* map, int32_t* out, cudaStream_t st) {
  if (B <= 0) return;
  MaArgs a = ma_args(w, B, K, best, best_dS, map, out);
  if (B <= kMaFusedMax) {
    launch_single<MaFusedBody>(a, 1, st);
    return;
  }
  const int32_t vg = vg_ma(B);
  const int L = rounds_for(B);
  launch_single<MaKeysBody>(a, vg, st);
  for (int r = 0; r < L; ++r) {
    a.round = r;
    launch_single<MaCycleJumpBody>(a, vg, st);
  }
  a.round = L;
  launch_single<MaMarkBody>(a, vg, st);
  for (int p = 0; p < kMaSelPasses; ++p) {
    a.pass = p;
    launch_single<MaSelHistBody>(a, vg, st);
    launch_single<MaSelPickBody>(a, 1, st);
  }
  launch_single<MaParentBody>(a, vg, st);
  for (int r = 0; r < L; ++r) {
    a.round = r;
    launch_single<MaRootJumpBody>(a, vg, st);
  }
  scan_exclusive(w.root, w.newid, B, w.tile, st);
  a.round = L;
  launch_single<MaMapBody>(a, vg, st);
}

}  // namespace sbp
