// dense_groups.cu — the candidate-group early-stop replay on the device.
//
// RunDenseGroupExactEarlyStop (common/group_scheduler.cpp:60-239) replays a
// learned proposal schedule over candidate groups (one group per query id)
// against known labels, with no certificates: candidates are ordered by
// (query id, priority desc, cost asc, index) — or by (query id, index) when
// the input order is kept — and each group is walked in that order:
//
//   * a candidate whose uncertainty reaches the threshold sends the rest of
//     the group to full fallback (every candidate from there on at full cost
//     until the first colliding one);
//   * otherwise it costs its narrow cost; a colliding candidate whose
//     predicted interval meets the contact interval is a hit; a colliding
//     one that misses costs the miss penalty and, once the attempt limit is
//     reached, one full fallback call that ends the group as a collision.
//
// The binding parses the rows first (py_module.cpp:1179-1246): the
// predicted interval is the arg-max bin of eight interval scores, the full
// cost is oracle_trace[:, 5], the narrow cost full * cost_target (at least
// 1e-12) when cost_target is finite and positive, the contact interval
// oracle_trace[:, 6:8] and the label oracle_trace[:, 0] > 0.5.
//
// Device layout: one thread per row parses and validates; two stable radix
// sorts give the order; a gather writes the sorted costs and flags and the
// group heads; one warp per group finds the stopping position with ballots
// and folds the group's sums lane by lane in order.  The reference adds its
// work totals one term at a time into double accumulators, so the totals
// depend on the order of the additions: every term goes to a slot whose
// position is its place in the reference's sequence (positive terms only;
// empty slots are +0.0, which adds exactly nothing to a sum that starts at
// +0.0 and only grows), the non-zero slots are compacted in order, and one
// warp per total adds them in sequence from shared-memory tiles that the
// rest of its block streams in.  Every total is therefore the reference's
// to the bit.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include <cmath>

#include "p2c_internal.cuh"

namespace p2c {
namespace {

constexpr int kThreads = 256;
constexpr unsigned char kColl = 1, kOverlap = 2, kHighUnc = 4;

// Integer totals, in p2c_dense_group_stats order of the counters below.
enum {
  kGroups,
  kPositive,
  kCalls,
  kFallback,
  kHit,
  kMiss,
  kTP,
  kTN,
  kFP,
  kFN,
  kReordered,
  kHighUncGroups,
  kRankSum,
  kNumCounters
};

struct DenseAcc {
  unsigned long long ctr[kNumCounters];
  unsigned long long first_error;  // (row << 2) | kind; ~0 none
  int n_groups;                    // DeviceSelect's count of group heads
  int n_terms;                     // DeviceSelect's count of non-zero work terms
};

struct DenseLayout {
  DenseAcc* acc = nullptr;
  unsigned long long* key[2] = {nullptr, nullptr};   // sort A: priority desc | cost asc
  unsigned long long* qkey[2] = {nullptr, nullptr};  // sort B: query id
  unsigned* idx[3] = {nullptr, nullptr, nullptr};
  double* full = nullptr;  // PositiveCost(full, 1), input order
  double* narrow = nullptr;
  unsigned char* flags = nullptr;
  double* s_full = nullptr;  // sorted order
  double* s_narrow = nullptr;
  unsigned char* s_flags = nullptr;
  unsigned char* head = nullptr;
  unsigned* iota = nullptr;
  unsigned* g_start = nullptr;
  double* terms = nullptr;    // 2n + n slots (2 per candidate + 1 per group at most)
  double* compact = nullptr;  // the non-zero terms, in order
  double* g_full = nullptr;   // per group: the summed full costs
  double* g_cost = nullptr;   // per group: the cost before its first positive (0 when none)
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  size_t total = 0;
};

struct NonZeroTerm {
  __host__ __device__ bool operator()(double x) const { return x != 0.0; }
};

size_t cub_bytes(long long n) {
  const int m = (int)(n > 0 ? n : 1);
  size_t a = 0, b = 0, c = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, a, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (const unsigned*)nullptr, (unsigned*)nullptr, m);
  cub::DeviceSelect::Flagged(nullptr, b, (const unsigned*)nullptr, (const unsigned char*)nullptr,
                             (unsigned*)nullptr, (int*)nullptr, m);
  cub::DeviceSelect::If(nullptr, c, (const double*)nullptr, (double*)nullptr, (int*)nullptr, 3 * m, NonZeroTerm{});
  return std::max(a, std::max(b, c));
}

DenseLayout carve(void* base, long long n) {
  DenseLayout L;
  char* p = static_cast<char*>(base);
  size_t off = 0;
  auto take = [&](size_t bytes) -> void* {
    off = (off + 255) & ~size_t(255);
    void* r = p ? p + off : nullptr;
    off += bytes;
    return r;
  };
  const size_t m = (size_t)(n > 0 ? n : 1);
  L.acc = (DenseAcc*)take(sizeof(DenseAcc));
  for (auto& k : L.key) k = (unsigned long long*)take(8 * m);
  for (auto& k : L.qkey) k = (unsigned long long*)take(8 * m);
  for (auto& v : L.idx) v = (unsigned*)take(4 * m);
  L.full = (double*)take(8 * m);
  L.narrow = (double*)take(8 * m);
  L.flags = (unsigned char*)take(m);
  L.s_full = (double*)take(8 * m);
  L.s_narrow = (double*)take(8 * m);
  L.s_flags = (unsigned char*)take(m);
  L.head = (unsigned char*)take(m);
  L.iota = (unsigned*)take(4 * m);
  L.g_start = (unsigned*)take(4 * m);
  L.terms = (double*)take(8 * 3 * m);
  L.compact = (double*)take(8 * 3 * m);
  L.g_full = (double*)take(8 * m);
  L.g_cost = (double*)take(8 * m);
  L.tmp_bytes = cub_bytes(n);
  L.tmp = take(L.tmp_bytes);
  L.total = off;
  return L;
}

__device__ __forceinline__ unsigned float_key_asc(float f) {
  unsigned u = __float_as_uint(f == 0.0f ? 0.0f : f);  // -0 and +0 compare equal
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ double positive_cost(double v, double fallback) {  // group_scheduler.cpp:31-36
  return (!isfinite(v) || v <= 0.0) ? fallback : v;
}

struct ParseIn {
  const unsigned long long* query_id;
  const unsigned long long* candidate_id;
  const float* cost_target;
  const double* oracle_trace;  // n x 8
  const float* interval_scores;  // n x 8
  const float* priority;
  const float* cost_score;
  const float* uncertainty;
};

__global__ void init_kernel(DenseLayout L) {
  if (threadIdx.x < kNumCounters) L.acc->ctr[threadIdx.x] = 0;
  if (threadIdx.x == 0) {
    L.acc->first_error = ~0ull;
    L.acc->n_groups = 0;
    L.acc->n_terms = 0;
  }
}

// One row: the binding's parse (py_module.cpp:1212-1244), the engine's
// validation (group_scheduler.cpp:81-88), the per-candidate costs and flags
// of the walk (:143-150, :170) and the sort keys.
__global__ void __launch_bounds__(kThreads) parse_kernel(ParseIn in, long long n, float threshold, int keep_order,
                                                         DenseLayout L) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long qid = in.query_id[i], cid = in.candidate_id[i];
  const float* sc = in.interval_scores + 8 * i;
  int best = 0;
  float best_score = sc[0];
#pragma unroll
  for (int k = 1; k < 8; ++k) {
    const float v = sc[k];
    if (v > best_score) {
      best_score = v;
      best = k;
    }
  }
  const double width = 1.0 / 8.0;
  const double it0 = width * (double)best;
  const double it0w = it0 + width;
  const double it1 = it0w < 1.0 ? it0w : 1.0;  // std::min(1.0, t0 + width)
  const double* tr = in.oracle_trace + 8 * i;
  const double full = tr[5];
  const float ratio = in.cost_target[i];
  double narrow = full;
  if (isfinite(ratio) && ratio > 0.0f) {
    const double x = full * (double)ratio;
    narrow = 1.0e-12 < x ? x : 1.0e-12;  // std::max(1e-12, x)
  }
  const double c0 = tr[6], c1 = tr[7];
  const float prio = in.priority[i], cost = in.cost_score[i], unc = in.uncertainty[i];
  unsigned kind = 0;
  if (qid == 0 || cid == 0)
    kind = 1;
  else if (!(isfinite(full) && isfinite(narrow) && isfinite(c0) && isfinite(c1) && isfinite(prio) &&
             isfinite(cost) && isfinite(unc)))
    kind = 2;
  if (kind) atomicMin(&L.acc->first_error, ((unsigned long long)i << 2) | kind);
  const double fc = positive_cost(full, 1.0);
  L.full[i] = fc;
  L.narrow[i] = positive_cost(narrow, fc);
  const double lo = it0 < c0 ? c0 : it0;  // std::max(interval_t0, contact_t0)
  const double hi = c1 < it1 ? c1 : it1;  // std::min(interval_t1, contact_t1)
  L.flags[i] = (unsigned char)((tr[0] > 0.5 ? kColl : 0) | (lo <= hi ? kOverlap : 0) |
                               (unc >= threshold ? kHighUnc : 0));
  L.idx[0][i] = (unsigned)i;
  if (keep_order)
    L.qkey[0][i] = qid;
  else
    L.key[0][i] = ((unsigned long long)(~float_key_asc(prio)) << 32) | float_key_asc(cost);
}

__global__ void __launch_bounds__(kThreads) gather_qid_kernel(const unsigned long long* qid, const unsigned* order,
                                                              long long n, unsigned long long* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = qid[order[i]];
}

// Sorted costs and flags, group heads, and the count of moved rows.
__global__ void __launch_bounds__(kThreads) gather_kernel(const unsigned* order, const unsigned long long* sorted_qid,
                                                          long long n, DenseLayout L) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool moved = false;
  if (i < n) {
    const unsigned j = order[i];
    L.s_full[i] = L.full[j];
    L.s_narrow[i] = L.narrow[j];
    L.s_flags[i] = L.flags[j];
    L.head[i] = (i == 0 || sorted_qid[i] != sorted_qid[i - 1]) ? 1 : 0;
    L.iota[i] = (unsigned)i;
    moved = j != (unsigned)i;
  }
  const unsigned m = __ballot_sync(0xffffffffu, moved);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(&L.acc->ctr[kReordered], (unsigned long long)__popc(m));
}

// Adds v of lanes [lo, hi) to s in lane order (every lane returns the same s).
__device__ __forceinline__ double fold_lanes(double s, double v, int lo, int hi) {
  for (int j = lo; j < hi; ++j) s += __shfl_sync(0xffffffffu, v, j);
  return s;
}

// One warp per group: the walk of group_scheduler.cpp:116-232.
__global__ void __launch_bounds__(kThreads) group_kernel(long long n, unsigned limit, double penalty, DenseLayout L) {
  __shared__ unsigned long long s_ctr[kNumCounters];
  if (threadIdx.x < kNumCounters) s_ctr[threadIdx.x] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long G = L.acc->n_groups;
  const long long warps = (long long)gridDim.x * (kThreads / 32);
  unsigned long long c[kNumCounters] = {};
  for (long long g = (long long)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5); g < G; g += warps) {
    const long long begin = L.g_start[g];
    const long long end = g + 1 < G ? (long long)L.g_start[g + 1] : n;
    const long long slot0 = 2 * begin + g;  // this group's 2 * size + 1 term slots
    double gfull = 0.0, wbfp = 0.0, gcost = 0.0;
    bool truth = false, predicted = false;
    int state = 0;  // 0 proposals, 1 full fallback, 2 resolved
    long long rank = 0;
    unsigned long long calls = 0, fallback = 0, hits = 0, misses = 0;
    bool high_group = false;
    for (long long base = begin; base < end; base += 32) {
      const long long pos = base + lane;
      const int nvalid = (int)min(32ll, end - base);
      const bool in = lane < nvalid;
      const double f = in ? L.s_full[pos] : 0.0;
      const double nr = in ? L.s_narrow[pos] : 0.0;
      const unsigned char fl = in ? L.s_flags[pos] : 0;
      const long long my_slot = slot0 + 2 * (pos - begin);
      gfull = fold_lanes(gfull, f, 0, nvalid);
      truth = truth || __any_sync(0xffffffffu, fl & kColl);
      int from = 0;
      if (state == 0) {
        const unsigned attempts = (unsigned)(pos - begin + 1);
        const bool stop = in && ((fl & kHighUnc) || ((fl & kColl) && ((fl & kOverlap) || attempts >= limit)));
        const unsigned m = __ballot_sync(0xffffffffu, stop);
        const int t = m ? __ffs(m) - 1 : nvalid;
        const bool pre = lane < t;
        if (pre) {  // narrow call; a colliding miss adds its penalty
          L.terms[my_slot] = nr;
          if (fl & kColl) L.terms[my_slot + 1] = f * penalty;
        }
        const double wv = (fl & kColl) ? nr + f * penalty : nr;
        wbfp = fold_lanes(wbfp, wv, 0, t);
        calls += (unsigned long long)t;
        misses += (unsigned long long)__popc(__ballot_sync(0xffffffffu, pre && (fl & kColl)));
        if (m) {
          const unsigned char sfl = (unsigned char)__shfl_sync(0xffffffffu, (int)fl, t);
          const double snr = __shfl_sync(0xffffffffu, nr, t);
          const double sf = __shfl_sync(0xffffffffu, f, t);
          const long long sslot = slot0 + 2 * (base + t - begin);
          rank = base + t - begin + 1;
          if (sfl & kHighUnc) {
            state = 1;
            from = t;
            high_group = true;
          } else if (sfl & kOverlap) {  // a hit inside the predicted interval
            if (lane == 0) L.terms[sslot] = snr;
            calls += 1;
            hits += 1;
            gcost = wbfp + snr;
            predicted = true;
            state = 2;
          } else {  // a miss at the attempt limit: penalty, then one full fallback call
            if (lane == 0) {
              L.terms[sslot] = snr;
              L.terms[sslot + 1] = sf * penalty;
              L.terms[slot0 + 2 * (end - begin)] = sf;
            }
            calls += 2;
            fallback += 1;
            misses += 1;
            gcost = (wbfp + snr) + sf;
            predicted = true;
            state = 2;
          }
        }
      }
      if (state == 1) {  // full fallback from lane `from` to the first colliding candidate
        const bool fb = in && lane >= from;
        const unsigned m = __ballot_sync(0xffffffffu, fb && (fl & kColl));
        const int q = m ? __ffs(m) - 1 : nvalid;
        const int last = m ? q + 1 : nvalid;
        if (fb && lane < last) L.terms[my_slot] = f;
        calls += (unsigned long long)(last - from);
        fallback += (unsigned long long)(last - from);
        wbfp = fold_lanes(wbfp, f, from, q);
        if (m) {
          const double qf = __shfl_sync(0xffffffffu, f, q);
          rank = base + q - begin + 1;
          gcost = wbfp + qf;
          predicted = true;
          state = 2;
        }
      }
    }
    if (lane == 0) {
      L.g_full[g] = gfull;
      L.g_cost[g] = predicted ? gcost : 0.0;
      c[kGroups] += 1;
      c[kPositive] += truth ? 1 : 0;
      c[kCalls] += calls;
      c[kFallback] += fallback;
      c[kHit] += hits;
      c[kMiss] += misses;
      c[kTP] += (truth && predicted) ? 1 : 0;
      c[kTN] += (!truth && !predicted) ? 1 : 0;
      c[kFP] += (!truth && predicted) ? 1 : 0;
      c[kFN] += (truth && !predicted) ? 1 : 0;
      c[kHighUncGroups] += high_group ? 1 : 0;
      c[kRankSum] += predicted ? (unsigned long long)rank : 0;
    }
  }
  if (lane == 0)
    for (int k = 0; k < kNumCounters; ++k)
      if (k != kReordered && c[k]) atomicAdd(&s_ctr[k], c[k]);
  __syncthreads();
  if (threadIdx.x < kNumCounters && threadIdx.x != kReordered && s_ctr[threadIdx.x])
    atomicAdd(&L.acc->ctr[threadIdx.x], s_ctr[threadIdx.x]);
}

struct FoldJob {
  const double* src[3];
  const int* count[3];   // device counts, or null: the fixed counts
  long long fixed[3];
  double* out[3];
};

// ---- the ordered fold ------------------------------------------------------
//
// A sum s of non-negative doubles, added one term at a time in a fixed order
// with round-to-nearest-even, reproduced exactly with block-wide scans.
// While s stays below the top of its binade, s = S * u with u its unit in the
// last place and S an integer below 2^53, and adding a term x gives
// S + floor(x / u) + r, where r = 1 when the remainder of x / u is above one
// half, 0 below, and on an exact half the bit that makes the result even:
// r depends on S only through its parity.  Each term is therefore a pair of
// increments (for an even and for an odd S), pairs compose associatively
// ((a then b)[p] = a[p] + b[(p + a[p]) mod 2]), and a block scan gives every
// term the S in front of it.  The first term whose exact sum could reach the
// top of the binade (or an infinite term) is added with the hardware DADD;
// the fold then continues from it in the new binade, with a chunk as long as
// the terms taken so far (steps come every few terms while s is small).
// Each such step at least doubles s, so there are at most a few dozen of
// them.  A zero-start sum takes its first non-zero term exactly.

constexpr int kFoldThreads = 512;
constexpr int kFoldPerThread = 8;  // consecutive terms per thread
constexpr int kFoldChunk = kFoldThreads * kFoldPerThread;
constexpr int kFoldWarps = kFoldThreads / 32;
constexpr int kFoldSmall = 64;  // shortest chunk after a binade step
constexpr unsigned long long kTwo53 = 1ull << 53;

struct IncPair {
  unsigned long long e, o;  // increments of S for an even / an odd S
};

__device__ __forceinline__ IncPair compose(const IncPair& a, const IncPair& b) {  // a, then b
  IncPair c;
  c.e = a.e + ((a.e & 1ull) ? b.o : b.e);
  c.o = a.o + ((a.o & 1ull) ? b.e : b.o);
  return c;
}

__device__ __forceinline__ IncPair shfl_up_pair(const IncPair& v, int o) {
  IncPair r;
  r.e = __shfl_up_sync(0xffffffffu, v.e, o);
  r.o = __shfl_up_sync(0xffffffffu, v.o, o);
  return r;
}

__device__ __forceinline__ IncPair warp_inclusive(IncPair v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const IncPair up = shfl_up_pair(v, o);
    if (lane >= o) v = compose(up, v);
  }
  return v;
}

struct FoldShared {
  unsigned long long we[32], wo[32];
  double s;
  long long pos;
  int first;
  int len;  // terms the next iteration takes
};

// One block per total.
__global__ void __launch_bounds__(kFoldThreads) fold_kernel(FoldJob job) {
  __shared__ FoldShared sh;
  const int b = blockIdx.x;  // selects without indexing the parameter arrays dynamically
  const double* src = b == 0 ? job.src[0] : (b == 1 ? job.src[1] : job.src[2]);
  const int* cp = b == 0 ? job.count[0] : (b == 1 ? job.count[1] : job.count[2]);
  const long long cnt = cp ? (long long)*cp : (b == 0 ? job.fixed[0] : (b == 1 ? job.fixed[1] : job.fixed[2]));
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const IncPair zero{0ull, 0ull};
  if (t == 0) {
    sh.s = 0.0;
    sh.pos = 0;
    sh.len = kFoldSmall;
  }
  __syncthreads();
  double x[kFoldPerThread];
  long long loaded = -1;  // chunk start the registers hold
  while (true) {
    const double s = sh.s;
    const long long pos = sh.pos;
    if (pos >= cnt || isinf(s)) break;
    const int want = sh.len;
    const int len = (int)min((long long)want, cnt - pos);
    const int next_len = min(kFoldChunk, 2 * want);
    if (loaded != pos) {
#pragma unroll
      for (int k = 0; k < kFoldPerThread; ++k) {
        const int i = t * kFoldPerThread + k;
        x[k] = i < len ? src[pos + i] : 0.0;
      }
    }
    double nx[kFoldPerThread];  // the next chunk, in case this one has no binade step
#pragma unroll
    for (int k = 0; k < kFoldPerThread; ++k) {
      const int i = t * kFoldPerThread + k;
      nx[k] = (i < next_len && pos + len + i < cnt) ? src[pos + len + i] : 0.0;
    }
    if (t == 0) sh.first = len;
    __syncthreads();  // everyone read s and pos; first is reset
    if (s == 0.0) {  // 0 + x == x: the first non-zero term starts the sum
#pragma unroll
      for (int k = 0; k < kFoldPerThread; ++k) {
        const int i = t * kFoldPerThread + k;
        if (i < len && x[k] != 0.0) {
          atomicMin(&sh.first, i);
          break;
        }
      }
      __syncthreads();
      const int f = sh.first;
#pragma unroll
      for (int k = 0; k < kFoldPerThread; ++k)
        if (t * kFoldPerThread + k == f) sh.s = x[k];
      if (t == 0) {
        sh.pos = pos + (f < len ? f + 1 : len);
        sh.len = f < len ? kFoldSmall : next_len;
      }
      loaded = -1;
      __syncthreads();
      continue;
    }
    const int ue = max(ilogb(s), -1022) - 52;
    const unsigned long long S = (unsigned long long)ldexp(s, -ue);
    IncPair inc[kFoldPerThread];
    unsigned long long m[kFoldPerThread];
    bool big[kFoldPerThread];
    IncPair local = zero;
#pragma unroll
    for (int k = 0; k < kFoldPerThread; ++k) {
      inc[k] = zero;
      m[k] = 0;
      big[k] = false;
      if (t * kFoldPerThread + k < len) {
        const double q = ldexp(x[k], -ue);
        big[k] = !(q < 9007199254740992.0);
        if (big[k]) {
          inc[k] = IncPair{kTwo53, kTwo53};  // never applied: the binade step comes first
        } else {
          const double mf = floor(q);
          const double f = q - mf;
          m[k] = (unsigned long long)mf;
          const bool above = f > 0.5, tie = f == 0.5;
          inc[k].e = m[k] + (above ? 1ull : (tie ? (m[k] & 1ull) : 0ull));
          inc[k].o = m[k] + (above ? 1ull : (tie ? ((m[k] + 1ull) & 1ull) : 0ull));
        }
      }
      local = compose(local, inc[k]);
    }
    const IncPair incl = warp_inclusive(local, lane);
    if (lane == 31) {
      sh.we[w] = incl.e;
      sh.wo[w] = incl.o;
    }
    __syncthreads();
    if (w == 0) {
      const IncPair v = warp_inclusive(lane < kFoldWarps ? IncPair{sh.we[lane], sh.wo[lane]} : zero, lane);
      IncPair ex = shfl_up_pair(v, 1);
      if (lane == 0) ex = zero;
      __syncwarp();
      sh.we[lane] = ex.e;
      sh.wo[lane] = ex.o;
    }
    __syncthreads();
    IncPair ein = shfl_up_pair(incl, 1);
    if (lane == 0) ein = zero;
    const IncPair wp{sh.we[w], sh.wo[w]};
    const IncPair ex = compose(wp, ein);
    unsigned long long P = S + ((S & 1ull) ? ex.o : ex.e);
    int mine = len;
    unsigned long long P_at = 0;
#pragma unroll
    for (int k = 0; k < kFoldPerThread; ++k) {
      const bool in = t * kFoldPerThread + k < len;
      if (in && mine == len) {
        if (big[k] || P >= kTwo53 || P + m[k] >= kTwo53) {
          mine = t * kFoldPerThread + k;
          P_at = P;
        } else {
          P += (P & 1ull) ? inc[k].o : inc[k].e;
        }
      }
    }
    if (mine < len) atomicMin(&sh.first, mine);
    __syncthreads();
    const int c = sh.first;
    if (c == len) {  // no binade step: the last thread holds the end of the chunk
      if (t == (len - 1) / kFoldPerThread) {
        sh.s = ldexp((double)P, ue);
        sh.pos = pos + len;
        sh.len = next_len;
      }
    } else if (mine == c) {
#pragma unroll
      for (int k = 0; k < kFoldPerThread; ++k)
        if (t * kFoldPerThread + k == c) sh.s = ldexp((double)P_at, ue) + x[k];
      sh.pos = pos + c + 1;
      // s grows about linearly in the terms taken, so the next step is about
      // as many terms away as have been taken so far
      sh.len = (int)max((long long)kFoldSmall, min((long long)kFoldChunk, pos + c + 1));
    }
    __syncthreads();
    if (sh.pos == pos + len) {
#pragma unroll
      for (int k = 0; k < kFoldPerThread; ++k) x[k] = nx[k];
      loaded = pos + len;
    } else {
      loaded = -1;
    }
  }
  if (t == 0) *(b == 0 ? job.out[0] : (b == 1 ? job.out[1] : job.out[2])) = sh.s;
}

__global__ void finish_kernel(long long n, DenseLayout L, p2c_dense_group_stats* st) {
  if (threadIdx.x != 0) return;
  const unsigned long long* c = L.acc->ctr;
  st->candidate_count = (unsigned long long)n;
  st->group_count = c[kGroups];
  st->positive_group_count = c[kPositive];
  st->no_proposal_exact_calls = (unsigned long long)n;
  st->learned_exact_calls = c[kCalls];
  st->learned_fallback_calls = c[kFallback];
  st->learned_interval_hit_count = c[kHit];
  st->learned_interval_miss_count = c[kMiss];
  st->first_positive_rank_sum = (double)c[kRankSum];
  st->tp = c[kTP];
  st->tn = c[kTN];
  st->fp = c[kFP];
  st->fn = c[kFN];
  st->reordered_count = c[kReordered];
  st->high_uncertainty_group_count = c[kHighUncGroups];
  const unsigned long long e = L.acc->first_error;
  st->error_row = e == ~0ull ? -1 : (long long)(e >> 2);
  st->error_kind = e == ~0ull ? 0 : (int)(e & 3);
  st->pad = 0;
}

int grid_for(long long n) { return (int)std::max(1ll, (n + kThreads - 1) / kThreads); }

}  // namespace
}  // namespace p2c

extern "C" {

size_t p2c_dense_group_early_stop_workspace_bytes(int64_t n) {
  if (n < 0) return 0;
  return p2c::carve(nullptr, n).total + 256;
}

int p2c_dense_group_early_stop(int64_t n, const uint64_t* query_id_dev, const uint64_t* candidate_id_dev,
                               const float* cost_target_dev, const double* oracle_trace_dev,
                               const float* interval_scores_dev, const float* priority_score_dev,
                               const float* cost_score_dev, const float* uncertainty_score_dev,
                               const p2c_dense_group_config* config, p2c_dense_group_stats* stats_dev,
                               void* workspace_dev, size_t workspace_bytes, void* stream) {
  using namespace p2c;
  if (config == nullptr) return fail(P2C_ERR_INVALID, "dense group config pointer is null");
  if (stats_dev == nullptr) return fail(P2C_ERR_INVALID, "DenseGroupEarlyStopStats pointer is null");
  if (config->representative_attempt_limit == 0u)
    return fail(P2C_ERR_INVALID, "representative_attempt_limit must be positive");
  if (!std::isfinite(config->uncertainty_fallback_threshold) || config->uncertainty_fallback_threshold < 0.0f)
    return fail(P2C_ERR_INVALID, "uncertainty_fallback_threshold must be finite and non-negative");
  if (!std::isfinite(config->interval_miss_penalty_scale) || config->interval_miss_penalty_scale < 0.0)
    return fail(P2C_ERR_INVALID, "interval_miss_penalty_scale must be finite and non-negative");
  if (n < 0 || n >= (1ll << 29))  // the 3n work-term slots are counted in int by the compaction
    return fail(P2C_ERR_INVALID, "row count must lie in [0, 2^29)");
  if (n > 0 && (query_id_dev == nullptr || candidate_id_dev == nullptr || cost_target_dev == nullptr ||
                oracle_trace_dev == nullptr || interval_scores_dev == nullptr || priority_score_dev == nullptr ||
                cost_score_dev == nullptr || uncertainty_score_dev == nullptr))
    return fail(P2C_ERR_INVALID, "input pointer is null");
  const int qbits = config->query_bits <= 0 || config->query_bits > 64 ? 64 : config->query_bits;
  const size_t need = carve(nullptr, n).total;
  if (workspace_dev == nullptr || workspace_bytes < need)
    return fail(P2C_ERR_INVALID, "dense group workspace too small: %zu < %zu bytes", workspace_bytes, need);
  DenseLayout L = carve(workspace_dev, n);
  cudaStream_t s = as_stream(stream);
  init_kernel<<<1, 32, 0, s>>>(L);
  P2C_CUDA(cudaMemsetAsync(stats_dev, 0, sizeof(p2c_dense_group_stats), s));
  if (n > 0) {
    const ParseIn in{reinterpret_cast<const unsigned long long*>(query_id_dev),
                     reinterpret_cast<const unsigned long long*>(candidate_id_dev),
                     cost_target_dev,
                     oracle_trace_dev,
                     interval_scores_dev,
                     priority_score_dev,
                     cost_score_dev,
                     uncertainty_score_dev};
    const int keep = config->preserve_input_order ? 1 : 0;
    parse_kernel<<<grid_for(n), kThreads, 0, s>>>(in, n, config->uncertainty_fallback_threshold, keep, L);
    size_t tb = L.tmp_bytes;
    const unsigned* order = L.idx[0];
    if (!keep) {  // stable: priority desc, then cost asc, then index
      P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.key[0], L.key[1], L.idx[0], L.idx[1], (int)n, 0, 64, s));
      gather_qid_kernel<<<grid_for(n), kThreads, 0, s>>>(in.query_id, L.idx[1], n, L.qkey[0]);
      order = L.idx[1];
    }
    tb = L.tmp_bytes;  // stable by query id: the final order
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.qkey[0], L.qkey[1], order, L.idx[2], (int)n, 0, qbits, s));
    gather_kernel<<<grid_for(n), kThreads, 0, s>>>(L.idx[2], L.qkey[1], n, L);
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceSelect::Flagged(L.tmp, tb, L.iota, L.head, L.g_start, &L.acc->n_groups, (int)n, s));
    P2C_CUDA(cudaMemsetAsync(L.terms, 0, sizeof(double) * 3 * (size_t)n, s));
    DeviceInfo info;
    if (int rc = current_device_info(&info)) return rc;
    const long long want = (n + (kThreads / 32) - 1) / (kThreads / 32);
    const int grid = (int)std::max(1ll, std::min(want, (long long)info.sm_count * 8));
    group_kernel<<<grid, kThreads, 0, s>>>(n, config->representative_attempt_limit,
                                           config->interval_miss_penalty_scale, L);
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceSelect::If(L.tmp, tb, L.terms, L.compact, &L.acc->n_terms, (int)(3 * n), NonZeroTerm{}, s));
    FoldJob job{{L.compact, L.g_full, L.g_cost},
                {&L.acc->n_terms, &L.acc->n_groups, &L.acc->n_groups},
                {0, 0, 0},
                {&stats_dev->learned_exact_work, &stats_dev->no_proposal_exact_work,
                 &stats_dev->cost_before_first_positive_sum}};
    fold_kernel<<<3, kFoldThreads, 0, s>>>(job);
  }
  finish_kernel<<<1, 32, 0, s>>>(n, L, stats_dev);
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

int p2c_ordered_sum(const double* terms_dev, int64_t n, double* out_dev, void* stream) {
  using namespace p2c;
  if (n < 0) return fail(P2C_ERR_INVALID, "term count must be non-negative");
  if (out_dev == nullptr || (n > 0 && terms_dev == nullptr)) return fail(P2C_ERR_INVALID, "term or output pointer is null");
  FoldJob job{{terms_dev, terms_dev, terms_dev}, {nullptr, nullptr, nullptr}, {n, 0, 0}, {out_dev, out_dev, out_dev}};
  fold_kernel<<<1, kFoldThreads, 0, as_stream(stream)>>>(job);
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

}  // extern "C"
