// groups_batch.cu — scheduled any-hit with fallback replay over the candidate
// groups of many scenes in one launch sequence.
//
// The same procedure as p2c_group_anyhit (the scene tool's
// RunScheduledAnyHitRows, tools/scene_object_envelope_native_ti_walltime.cpp:
// 1283-1410), for every (scene, family) of a batch at once: a group is an
// unordered object pair of one scene and one family (GroupKey :756-770, with
// the scene and family added to the key), so groups of different scenes
// never mix and every scene gets exactly the calls, hits and groups it gets
// alone.  The candidates of all scenes form one index space, segment
// k = family_index * n_scenes + scene; the group and score sorts, the ranks,
// the two certification phases and the call recovery run once over it (about
// twenty launches whatever the number of scenes), and each segment gets its
// own p2c_anyhit_summary.
//
// Proposals are sorted rank-major with the family as the top key bit, so the
// point-triangle proposals precede the edge-edge ones and the engine reads
// them as its two queues (it picks the distance function by queue family).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <cub/block/block_scan.cuh>

#include <algorithm>
#include <vector>

#include "certify_core.cuh"
#include "certify_launch.cuh"
#include "scene_pairs.cuh"

namespace p2c {

namespace {

constexpr unsigned kNone = 0xffffffffu;
constexpr int kThreads = 256;
constexpr int kOffThreads = 1024;
constexpr long long kMaxCandidates = (1ll << 31) - 1;
constexpr long long kMaxGroups = 1ll << 28;
constexpr int kMaxScenes = 1 << 20;

struct Counters {
  unsigned long long n_top[2];    // proposals of each family
  unsigned long long n_fb_vf;     // fallback candidates of family 1 (they precede family 2)
  unsigned long long error_word;  // engine-independent bits shared by all segments (none so far)
  int fb_count;                   // fallback candidates (cub's selection count)
  int pad;
};

constexpr unsigned char kComputedSeparation = 1, kComputedHit = 2;

struct Layout {
  CertifyScratch* sc = nullptr;
  Counters* ctr = nullptr;
  unsigned long long* cand_off = nullptr;   // 2n + 1
  unsigned long long* group_off = nullptr;  // 2n + 1
  unsigned long long* seg_err = nullptr;    // 2n: 4 non-finite geometry, 8 bad id, 16 NaN score
  unsigned long long* seg_spec = nullptr;   // 2n: speculative certificates
  unsigned* seg = nullptr;                  // C: segment of each candidate
  unsigned* grp = nullptr;
  unsigned* rank = nullptr;
  unsigned char* state = nullptr;
  unsigned char* flags = nullptr;
  unsigned long long* skey[2] = {nullptr, nullptr};
  unsigned* val[2] = {nullptr, nullptr};
  unsigned* key32[2] = {nullptr, nullptr};
  unsigned* fb_list = nullptr;
  unsigned* g_size = nullptr;
  unsigned* g_start = nullptr;
  unsigned* g_min_hit = nullptr;
  unsigned* g_min_fb = nullptr;
  unsigned long long* g_fcalls = nullptr;
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  size_t total = 0;
};

size_t cub_temp_bytes(long long cap, long long groups) {
  const int n = (int)std::max(cap, 1ll);
  size_t a = 0, b = 0, c = 0, d = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, a, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (const unsigned*)nullptr, (unsigned*)nullptr, n);
  cub::DeviceRadixSort::SortPairs(nullptr, b, (const unsigned*)nullptr, (unsigned*)nullptr, (const unsigned*)nullptr,
                                  (unsigned*)nullptr, n);
  cub::DeviceScan::ExclusiveSum(nullptr, c, (const unsigned*)nullptr, (unsigned*)nullptr,
                                (int)std::max(groups, 1ll));
  cub::DeviceSelect::Flagged(nullptr, d, (const unsigned*)nullptr, (const unsigned char*)nullptr,
                             (unsigned*)nullptr, (int*)nullptr, n);
  return std::max(std::max(a, b), std::max(c, d));
}

Layout carve(void* base, int n_scenes, long long cap, long long groups) {
  Layout L;
  size_t off = 0;
  char* b = static_cast<char*>(base);
  auto take = [&](size_t bytes) -> void* {
    void* p = b == nullptr ? nullptr : b + off;
    off += (bytes + 255) & ~size_t(255);
    return p;
  };
  const size_t n = (size_t)std::max(cap, 1ll), g = (size_t)std::max(groups, 1ll), k = 2 * (size_t)n_scenes;
  L.sc = static_cast<CertifyScratch*>(take(kScratchHeaderBytes + kPoolBytes));
  L.ctr = static_cast<Counters*>(take(sizeof(Counters)));
  L.cand_off = static_cast<unsigned long long*>(take((k + 1) * 8));
  L.group_off = static_cast<unsigned long long*>(take((k + 1) * 8));
  L.seg_err = static_cast<unsigned long long*>(take(k * 8));
  L.seg_spec = static_cast<unsigned long long*>(take(k * 8));
  L.seg = static_cast<unsigned*>(take(n * 4));
  L.grp = static_cast<unsigned*>(take(n * 4));
  L.rank = static_cast<unsigned*>(take(n * 4));
  L.state = static_cast<unsigned char*>(take(n));
  L.flags = static_cast<unsigned char*>(take(n));
  L.skey[0] = static_cast<unsigned long long*>(take(n * 8));
  L.skey[1] = static_cast<unsigned long long*>(take(n * 8));
  L.val[0] = static_cast<unsigned*>(take(n * 4));
  L.val[1] = static_cast<unsigned*>(take(n * 4));
  L.key32[0] = static_cast<unsigned*>(take(n * 4));
  L.key32[1] = static_cast<unsigned*>(take(n * 4));
  L.fb_list = static_cast<unsigned*>(take(n * 4));
  L.g_size = static_cast<unsigned*>(take(g * 4));
  L.g_start = static_cast<unsigned*>(take(g * 4));
  L.g_min_hit = static_cast<unsigned*>(take(g * 4));
  L.g_min_fb = static_cast<unsigned*>(take(g * 4));
  L.g_fcalls = static_cast<unsigned long long*>(take(g * 8));
  L.tmp_bytes = cub_temp_bytes(cap, groups);
  L.tmp = take(L.tmp_bytes);
  L.total = off;
  return L;
}

// Sizes of the candidate and group spaces from the host table.
struct Sizes {
  long long cap = 0, cap_vf = 0, groups = 0, max_seg_cap = 0;
};

Sizes sizes_of(const p2c_batch_scene* h, int n, unsigned mask) {
  Sizes z;
  for (int f = 0; f < 2; ++f) {
    if ((mask & (1u << f)) == 0u) continue;
    for (int s = 0; s < n; ++s) {
      const long long c = std::max<long long>(0, f == 0 ? h[s].vf_cap : h[s].ee_cap);
      z.cap += c;
      if (f == 0) z.cap_vf += c;
      z.max_seg_cap = std::max(z.max_seg_cap, c);
      z.groups += (long long)h[s].n_obj * h[s].n_obj;
    }
  }
  return z;
}

int bit_width(unsigned long long v) {
  int b = 0;
  while (v != 0ull) {
    ++b;
    v >>= 1;
  }
  return b;
}

unsigned grid_for(long long n, int threads) {
  const long long b = (n + threads - 1) / threads;
  return (unsigned)std::min<long long>(std::max<long long>(b, 1), 1ll << 20);
}

__device__ __forceinline__ long long seg_cap(const p2c_batch_scene& d, int f, unsigned mask) {
  if ((mask & (1u << f)) == 0u) return 0;
  const long long c = f == 0 ? d.vf_cap : d.ee_cap;
  return c > 0 ? c : 0;
}

__device__ __forceinline__ long long seg_count(const p2c_batch_scene& d, int f, unsigned mask) {
  const long long cap = seg_cap(d, f, mask);
  if (cap == 0) return 0;
  const long long c = (long long)d.counts[f];
  return c < cap ? c : cap;
}

// Segment offsets of the candidate and group spaces (one block), the same
// sums the host formed for the sizes.
__global__ void __launch_bounds__(kOffThreads) offsets_kernel(const p2c_batch_scene* scenes, int n, unsigned mask,
                                                            Layout L) {
  using Scan = cub::BlockScan<unsigned long long, kOffThreads>;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ unsigned long long carry[2];
  if (threadIdx.x < 2) carry[threadIdx.x] = 0ull;
  if (threadIdx.x == 0) *L.ctr = Counters{};
  __syncthreads();
  const int k_total = 2 * n;
  for (int base = 0; base < k_total; base += kOffThreads) {
    const int k = base + (int)threadIdx.x;
    unsigned long long c = 0ull, g = 0ull;
    if (k < k_total) {
      const int f = k < n ? 0 : 1, s = k < n ? k : k - n;
      const p2c_batch_scene d = scenes[s];
      c = (unsigned long long)seg_cap(d, f, mask);
      g = (mask & (1u << f)) ? (unsigned long long)d.n_obj * (unsigned long long)d.n_obj : 0ull;
      L.seg_err[k] = 0ull;
      L.seg_spec[k] = 0ull;
    }
    unsigned long long ec = 0ull, tc = 0ull, eg = 0ull, tg = 0ull;
    Scan(tmp).ExclusiveSum(c, ec, tc);
    __syncthreads();
    Scan(tmp).ExclusiveSum(g, eg, tg);
    if (k < k_total) {
      L.cand_off[k] = carry[0] + ec;
      L.group_off[k] = carry[1] + eg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      carry[0] += tc;
      carry[1] += tg;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    L.cand_off[k_total] = carry[0];
    L.group_off[k_total] = carry[1];
  }
}

__global__ void init_groups_kernel(Layout L, long long groups, p2c_anyhit_summary* summaries, int n) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (long long i = g; i < groups; i += (long long)gridDim.x * blockDim.x) {
    L.g_size[i] = 0u;
    L.g_min_hit[i] = kNone;
    L.g_min_fb[i] = kNone;
    L.g_fcalls[i] = 0ull;
  }
  if (summaries != nullptr)
    for (long long i = g; i < 2ll * n; i += (long long)gridDim.x * blockDim.x) summaries[i] = p2c_anyhit_summary{};
}

// Last segment k with off[k] <= v (segments may be empty).
__device__ __forceinline__ int find_seg(const unsigned long long* off, int k_total, unsigned long long v) {
  int lo = 0, hi = k_total - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= v) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ unsigned long long score_key_desc(double s, bool& nan) {
  nan = isnan(s);
  if (nan) return ~0ull - 1ull;
  if (s == 0.0) s = 0.0;
  const unsigned long long b = (unsigned long long)__double_as_longlong(s);
  const unsigned long long asc = (b >> 63) ? ~b : (b | (1ull << 63));
  return ~asc;
}

__device__ __forceinline__ void warp_count(unsigned* table, unsigned key, bool active) {
  const unsigned act = __activemask();
  const unsigned m = __match_any_sync(act, active ? key : kNone);
  if (active && (threadIdx.x & 31) == __ffs((int)m) - 1) atomicAdd(table + key, (unsigned)__popc(m));
}

// Per candidate: segment, group, descending score key; group sizes.
__global__ void prep_kernel(const p2c_batch_scene* scenes, int n, unsigned mask, const double* const* scores,
                            const unsigned long long* seeds, long long cap, unsigned long long groups, Layout L) {
  const int k_total = 2 * n;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < cap;
       c += (long long)gridDim.x * blockDim.x) {
    const int k = find_seg(L.cand_off, k_total, (unsigned long long)c);
    const int f = k < n ? 0 : 1, s = k < n ? k : k - n;
    const p2c_batch_scene& d = scenes[s];
    const long long local = c - (long long)__ldg(L.cand_off + k);
    unsigned g = (unsigned)groups;
    unsigned long long key = ~0ull;
    if (local < seg_count(d, f, mask)) {
      const unsigned long long pair = (f == 0 ? d.vf_pairs : d.ee_pairs)[local];
      const long long a = (long long)(pair >> 32), b = (long long)(pair & 0xffffffffull);
      const long long n_a = f == 0 ? d.nv : d.ne, n_b = f == 0 ? d.nf : d.ne;
      const int* obj_a = f == 0 ? d.v_obj : d.e_obj;
      const int* obj_b = f == 0 ? d.f_obj : d.e_obj;
      const int oa = a < n_a ? __ldg(obj_a + a) : -1, ob = b < n_b ? __ldg(obj_b + b) : -1;
      if (oa >= 0 && ob >= 0 && oa < d.n_obj && ob < d.n_obj) {
        const unsigned lo = (unsigned)min(oa, ob), hi = (unsigned)max(oa, ob);
        g = (unsigned)__ldg(L.group_off + k) + lo * (unsigned)d.n_obj + hi;
        const double sc = scores != nullptr ? scores[2 * s + f][local]
                                            : stub_score(seeds != nullptr ? seeds[s] : 0ull, f + 1, pair);
        bool nan = false;
        key = score_key_desc(sc, nan);
        if (nan) atomicOr(L.seg_err + k, 16ull);
      } else {
        atomicOr(L.seg_err + k, 8ull);
      }
    }
    L.seg[c] = (unsigned)k;
    L.grp[c] = g;
    L.state[c] = 0;
    L.skey[0][c] = key;
    L.val[0][c] = (unsigned)c;
    warp_count(L.g_size, g, g < (unsigned)groups);
  }
}

__global__ void group_key_kernel(long long cap, Layout L) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < cap;
       p += (long long)gridDim.x * blockDim.x)
    L.key32[0][p] = L.grp[L.val[1][p]];
}

// Ranks inside groups and the family-major, rank-major proposal keys.
__global__ void rank_kernel(long long cap, long long cap_vf, unsigned groups, unsigned K, int kbits, Layout L) {
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < cap;
       p += (long long)gridDim.x * blockDim.x) {
    const unsigned c = L.val[0][p];
    const unsigned g = L.grp[c];
    const unsigned fam = (long long)c < cap_vf ? 0u : 1u;
    unsigned r = kNone, key = K;
    if (g < groups) {
      r = (unsigned)p - L.g_start[g];
      key = r < K ? r : K;
    }
    L.rank[c] = r;
    L.key32[0][p] = (fam << kbits) | key;
    const bool top = g < groups && r < K;
    const unsigned act = __activemask();
    const unsigned mv = __ballot_sync(act, top && fam == 0u), me = __ballot_sync(act, top && fam == 1u);
    if ((threadIdx.x & 31) == __ffs((int)act) - 1) {
      if (mv) atomicAdd(&L.ctr->n_top[0], (unsigned long long)__popc(mv));
      if (me) atomicAdd(&L.ctr->n_top[1], (unsigned long long)__popc(me));
    }
  }
}

// Fallback candidates: not a proposal, in a group without a proposal hit.
__global__ void fallback_flags_kernel(long long cap, long long cap_vf, unsigned groups, unsigned K, Layout L) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < cap;
       c += (long long)gridDim.x * blockDim.x) {
    const unsigned g = L.grp[c];
    const bool f = g < groups && L.rank[c] >= K && L.g_min_hit[g] == kNone;
    L.flags[c] = f ? 1 : 0;
    L.key32[0][c] = (unsigned)c;
    const unsigned act = __activemask();
    const unsigned m = __ballot_sync(act, f && c < cap_vf);
    if ((threadIdx.x & 31) == __ffs((int)act) - 1 && m) atomicAdd(&L.ctr->n_fb_vf, (unsigned long long)__popc(m));
  }
}

// One phase over a work list of candidate indices: family 1 entries first.
struct BatchAnyhitProblem {
  const p2c_batch_scene* scenes;
  int n_scenes;
  const unsigned* list;
  const unsigned long long* n_top;       // proposal phase (else null)
  unsigned long long ee_base;            // proposal phase: first family-2 entry of the list
  const int* fb_count;                   // fallback phase (else null)
  const unsigned long long* fb_vf;       // fallback phase: family-1 entries
  const unsigned* seg;
  const unsigned long long* cand_off;
  const unsigned* grp;
  const unsigned* rank;  // null in the fallback phase: the key is the index
  unsigned* min_hit;
  unsigned char* state;
  unsigned long long* seg_err;
  double T0, T1;
  __device__ __forceinline__ long long n(int f) const {
    if (n_top != nullptr) return (long long)n_top[f - 1];
    const long long v = (long long)*fb_vf;
    return f == 1 ? v : (long long)*fb_count - v;
  }
  __device__ __forceinline__ unsigned entry(int f, long long q) const {
    const unsigned long long base = f == 1 ? 0ull : (n_top != nullptr ? ee_base : *fb_vf);
    return __ldg(list + base + (unsigned long long)q);
  }
  __device__ __forceinline__ unsigned order_key(unsigned c) const { return rank != nullptr ? __ldg(rank + c) : c; }
  __device__ __forceinline__ bool skip(int f, long long q) const {
    const unsigned c = entry(f, q);
    return order_key(c) > volatile_load(min_hit + __ldg(grp + c));
  }
  __device__ __forceinline__ void load(int f, long long q, Geo& g, double& t0, double& t1, int& bad) const {
    const unsigned c = entry(f, q);
    const int k = (int)__ldg(seg + c);
    const int s = k < n_scenes ? k : k - n_scenes;
    const p2c_batch_scene& d = scenes[s];
    const long long local = (long long)c - (long long)__ldg(cand_off + k);
    const ScenePairs sp{d.v_t0, d.v_t1, d.faces, d.edges,
                        reinterpret_cast<const unsigned long long*>(f == 1 ? d.vf_pairs : d.ee_pairs), T0, T1};
    bad = load_pair(sp, f, __ldg(sp.pairs + local), g) ? 0 : 2;
    t0 = T0;
    t1 = T1;
  }
  __device__ __forceinline__ void record(int f, long long q, bool hit) const {
    const unsigned c = entry(f, q);
    state[c] = hit ? kComputedHit : kComputedSeparation;
    if (hit) atomicMin(min_hit + grp[c], order_key(c));
  }
  __device__ __forceinline__ void finish(int f, long long q, const Outcome& o) const {
    record(f, q, o.status != P2C_STATUS_SEPARATION);
  }
  __device__ __forceinline__ void invalid(int f, long long q, int, double, double) const {
    atomicOr(seg_err + __ldg(seg + entry(f, q)), 4ull);
    record(f, q, true);  // non-finite geometry is certified undecided: a conservative hit
  }
};

__global__ void __launch_bounds__(kCertifyThreads, kCertifyMinBlocks)
    batch_anyhit_certify_kernel(const __grid_constant__ BatchAnyhitProblem prob, const __grid_constant__ CertParams prm,
                                const __grid_constant__ EnginePools pools, CertifyScratch* scratch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EngineShared& sh = reinterpret_cast<EngineShared*>(smem_raw)[threadIdx.x >> 5];
  WarpStats st;
  const unsigned long long t_start = global_ns();
  const long long warps = (long long)gridDim.x * kCertifyWarps;
  const int f1 = (int)min(32ll, max(1ll, (prob.n(1) + warps - 1) / warps));
  const int f2 = (int)min(32ll, max(1ll, (prob.n(2) + warps - 1) / warps));
  const bool ee_first = ((blockIdx.x * kCertifyWarps + (threadIdx.x >> 5)) & 1u) != 0u;
  const bool ok = run_engine<true, true, false>(prob, prm, f1, f2, ee_first, sh, st, &scratch->engine, pools, t_start);
  flush_stats(st, ok, scratch);
}

// Calls of the sequential procedure from the final minima, per candidate.
__global__ void calls_kernel(const p2c_batch_scene* scenes, int n, unsigned mask, long long cap, unsigned groups,
                             unsigned K, Layout L, unsigned char* evaluated, unsigned char* hit_out) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < cap;
       c += (long long)gridDim.x * blockDim.x) {
    const unsigned g = L.grp[c];
    unsigned char phase = 0;
    bool fb_called = false;
    if (g < groups) {
      const unsigned r = L.rank[c];
      const unsigned mh = L.g_min_hit[g];
      if (r < K) {
        if (r <= mh) phase = 1;
      } else if (mh == kNone && (unsigned)c <= L.g_min_fb[g]) {
        phase = 2;
        fb_called = true;
      }
    }
    const unsigned char st = L.state[c];
    if (evaluated != nullptr) evaluated[c] = phase;
    if (hit_out != nullptr) hit_out[c] = (phase != 0 && st == kComputedHit) ? 1 : 0;
    const unsigned act = __activemask();
    const unsigned m = __match_any_sync(act, fb_called ? g : kNone);
    if (fb_called && (threadIdx.x & 31) == __ffs((int)m) - 1)
      atomicAdd(L.g_fcalls + g, (unsigned long long)__popc(m));
    const bool spec = phase == 0 && st != 0;
    const unsigned k = L.seg[c];
    const unsigned ms = __match_any_sync(act, spec ? k : kNone);
    if (spec && (threadIdx.x & 31) == __ffs((int)ms) - 1) atomicAdd(L.seg_spec + k, (unsigned long long)__popc(ms));
  }
}

__global__ void groups_kernel(int n, unsigned groups, unsigned K, Layout L, unsigned char* detected_out,
                              p2c_anyhit_summary* summaries) {
  const int k_total = 2 * n;
  for (long long gi = (long long)blockIdx.x * blockDim.x + threadIdx.x; gi < (long long)groups;
       gi += (long long)gridDim.x * blockDim.x) {
    const unsigned g = (unsigned)gi;
    const unsigned size = L.g_size[g];
    const unsigned mh = L.g_min_hit[g], mf = L.g_min_fb[g];
    const unsigned long long pc = size == 0u ? 0ull : (mh == kNone ? (unsigned long long)min(size, K) : mh + 1ull);
    const unsigned long long fc = L.g_fcalls[g];
    const bool det = size != 0u && (mh != kNone || mf != kNone);
    if (detected_out != nullptr) detected_out[g] = det ? 1 : 0;
    if (summaries == nullptr || size == 0u) continue;
    const int k = find_seg(L.group_off, k_total, (unsigned long long)g);
    const int s = k < n ? k : k - n, f = k < n ? 0 : 1;
    p2c_anyhit_summary* sm = summaries + 2 * s + f;
    atomicAdd((unsigned long long*)&sm->groups, 1ull);
    if (det) {
      atomicAdd((unsigned long long*)&sm->detected_groups, 1ull);
      atomicAdd((unsigned long long*)&sm->first_hit_rank_sum, pc + fc);
    }
    if (mh == kNone) atomicAdd((unsigned long long*)&sm->fallback_groups, 1ull);
    if (pc) atomicAdd((unsigned long long*)&sm->proposal_calls, pc);
    if (fc) atomicAdd((unsigned long long*)&sm->fallback_calls, fc);
  }
}

// Per segment: candidate count, speculation and error bits.
__global__ void segments_kernel(const p2c_batch_scene* scenes, int n, unsigned mask, Layout L,
                                p2c_anyhit_summary* summaries) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 2 * n; k += gridDim.x * blockDim.x) {
    const int s = k < n ? k : k - n, f = k < n ? 0 : 1;
    p2c_anyhit_summary* sm = summaries + 2 * s + f;
    sm->candidates = (unsigned long long)seg_count(scenes[s], f, mask);
    sm->speculative = L.seg_spec[k];
    sm->error_word = L.seg_err[k] | L.sc->stats.error_word;
  }
}

cudaError_t reset_engine(CertifyScratch* sc, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(&sc->engine, 0, sizeof(EngineState), s);
  if (e != cudaSuccess) return e;
  return cudaMemsetAsync(pools_at(sc).tasks, 0, kTaskCap * sizeof(SubtreeTask), s);
}

int check_sizes(const Sizes& z) {
  if (z.cap > kMaxCandidates) return fail(P2C_ERR_INVALID, "batch any-hit: total candidate capacity must be < 2^31");
  if (z.groups > kMaxGroups) return fail(P2C_ERR_INVALID, "batch any-hit: total groups (sum of n_obj^2) must be <= 2^28");
  return P2C_OK;
}

}  // namespace

int launch_batch_anyhit(const p2c_batch_scene* h, const p2c_batch_scene* scenes, int n, unsigned mask,
                        const double* const* scores, const unsigned long long* seeds, long long top_k, double T0,
                        double T1, const p2c_cert_config& cfg, p2c_anyhit_summary* summaries,
                        unsigned char* group_detected, unsigned char* evaluated, unsigned char* hit_out, void* ws,
                        size_t ws_bytes, cudaStream_t s) {
  const Sizes z = sizes_of(h, n, mask);
  int rc = check_sizes(z);
  if (rc != P2C_OK) return rc;
  const Layout need = carve(nullptr, n, z.cap, z.groups);
  if (ws == nullptr || ws_bytes < need.total)
    return fail(P2C_ERR_INVALID, "batch any-hit workspace too small: %zu < %zu bytes", ws_bytes, need.total);
  Layout L = carve(ws, n, z.cap, z.groups);
  const long long C = z.cap;
  const unsigned G = (unsigned)z.groups;
  const unsigned K = (unsigned)std::min<long long>(top_k, std::max(z.max_seg_cap, 0ll));
  const int kbits = std::max(1, bit_width(K));

  P2C_CUDA(reset_scratch(L.sc, s, true));
  offsets_kernel<<<1, kOffThreads, 0, s>>>(scenes, n, mask, L);
  P2C_CUDA(cudaGetLastError());
  init_groups_kernel<<<grid_for(std::max<long long>(G, 2ll * n), kThreads), kThreads, 0, s>>>(L, G, summaries, n);
  P2C_CUDA(cudaGetLastError());
  LaunchShape shape;
  rc = certify_shape(batch_anyhit_certify_kernel, &shape);
  if (rc != P2C_OK) return rc;
  const CertParams prm = make_params(cfg, shape, 32ll * shape.grid * kCertifyWarps);
  if (C > 0) {
    prep_kernel<<<grid_for(C, kThreads), kThreads, 0, s>>>(scenes, n, mask, scores, seeds, C, G, L);
    P2C_CUDA(cudaGetLastError());
    size_t tb = L.tmp_bytes;
    // (score desc, index)
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.skey[0], L.skey[1], L.val[0], L.val[1], (int)C, 0, 64, s));
    group_key_kernel<<<grid_for(C, kThreads), kThreads, 0, s>>>(C, L);
    P2C_CUDA(cudaGetLastError());
    // (group, score desc, index)
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.key32[0], L.key32[1], L.val[1], L.val[0], (int)C, 0,
                                             std::max(1, bit_width(G)), s));
    if (G > 0) {
      tb = L.tmp_bytes;
      P2C_CUDA(cub::DeviceScan::ExclusiveSum(L.tmp, tb, L.g_size, L.g_start, (int)G, s));
    }
    rank_kernel<<<grid_for(C, kThreads), kThreads, 0, s>>>(C, z.cap_vf, G, K, kbits, L);
    P2C_CUDA(cudaGetLastError());
    if (K > 0) {
      // proposals: family-major, then rank-major: (family, rank, group, score desc, index)
      tb = L.tmp_bytes;
      P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.key32[0], L.key32[1], L.val[0], L.val[1], (int)C, 0,
                                               kbits + 1, s));
      BatchAnyhitProblem prop{scenes, n, L.val[1], L.ctr->n_top, (unsigned long long)z.cap_vf, nullptr, nullptr,
                              L.seg, L.cand_off, L.grp, L.rank, L.g_min_hit, L.state, L.seg_err, T0, T1};
      batch_anyhit_certify_kernel<<<shape.grid, kCertifyThreads, shape.smem, s>>>(prop, prm, pools_at(L.sc), L.sc);
      P2C_CUDA(cudaGetLastError());
    }
    fallback_flags_kernel<<<grid_for(C, kThreads), kThreads, 0, s>>>(C, z.cap_vf, G, K, L);
    P2C_CUDA(cudaGetLastError());
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceSelect::Flagged(L.tmp, tb, L.key32[0], L.flags, L.fb_list, &L.ctr->fb_count, (int)C, s));
    P2C_CUDA(reset_engine(L.sc, s));
    BatchAnyhitProblem fb{scenes, n, L.fb_list, nullptr, 0ull, &L.ctr->fb_count, &L.ctr->n_fb_vf,
                          L.seg, L.cand_off, L.grp, nullptr, L.g_min_fb, L.state, L.seg_err, T0, T1};
    batch_anyhit_certify_kernel<<<shape.grid, kCertifyThreads, shape.smem, s>>>(fb, prm, pools_at(L.sc), L.sc);
    P2C_CUDA(cudaGetLastError());
    calls_kernel<<<grid_for(C, kThreads), kThreads, 0, s>>>(scenes, n, mask, C, G, K, L, evaluated, hit_out);
    P2C_CUDA(cudaGetLastError());
  }
  if (G > 0) {
    groups_kernel<<<grid_for(G, kThreads), kThreads, 0, s>>>(n, G, K, L, group_detected, summaries);
    P2C_CUDA(cudaGetLastError());
  }
  if (summaries != nullptr) {
    segments_kernel<<<grid_for(2ll * n, kThreads), kThreads, 0, s>>>(scenes, n, mask, L, summaries);
    P2C_CUDA(cudaGetLastError());
  }
  return P2C_OK;
}

namespace {
__global__ void stub_scores_kernel(const unsigned long long* pairs, const unsigned long long* count, long long cap,
                                   int family, unsigned long long seed, double* scores) {
  const long long n = count != nullptr ? min((long long)*count, cap) : cap;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < cap;
       i += (long long)gridDim.x * blockDim.x)
    scores[i] = i < n ? stub_score(seed, family, pairs[i]) : 0.0;
}
}  // namespace

}  // namespace p2c

extern "C" {

size_t p2c_batch_anyhit_workspace_bytes(const p2c_batch_scene* scenes_host, int32_t n_scenes, uint32_t family_mask) {
  if (scenes_host == nullptr || n_scenes < 1 || family_mask == 0u || family_mask > 3u) return 0;
  const p2c::Sizes z = p2c::sizes_of(scenes_host, n_scenes, family_mask);
  return p2c::carve(nullptr, n_scenes, z.cap, z.groups).total;
}

int p2c_batch_anyhit(const p2c_batch_scene* scenes_host, const p2c_batch_scene* scenes_dev, int32_t n_scenes,
                     uint32_t family_mask, const double* const* scores_dev, const uint64_t* seeds_dev, int64_t top_k,
                     double interval_t0, double interval_t1, const p2c_cert_config* config,
                     p2c_anyhit_summary* summaries_dev, uint8_t* group_detected_dev, uint8_t* evaluated_dev,
                     uint8_t* hit_dev, void* workspace_dev, size_t workspace_bytes, void* stream) {
  if (scenes_host == nullptr || scenes_dev == nullptr) return p2c::fail(P2C_ERR_INVALID, "scene table pointer is null");
  if (n_scenes < 1 || n_scenes > p2c::kMaxScenes)
    return p2c::fail(P2C_ERR_INVALID, "batch scene count must lie in [1, %d]", p2c::kMaxScenes);
  if (family_mask == 0u || family_mask > 3u)
    return p2c::fail(P2C_ERR_INVALID, "family_mask must be 1 (vf), 2 (ee) or 3 (both)");
  if (config == nullptr) return p2c::fail(P2C_ERR_INVALID, "CertificateEngineConfig pointer is null");
  int rc = p2c::validate_cert_config(*config, interval_t0, interval_t1);
  if (rc != P2C_OK) return rc;
  if (top_k < 0) return p2c::fail(P2C_ERR_INVALID, "proposal top_k must be non-negative");
  for (int s = 0; s < n_scenes; ++s) {
    const p2c_batch_scene& d = scenes_host[s];
    if (d.n_obj < 1 || d.n_obj > 4096)
      return p2c::fail(P2C_ERR_INVALID, "scene %d: n_obj must lie in [1, 4096] for candidate groups", s);
    if (d.vf_cap < 0 || d.ee_cap < 0) return p2c::fail(P2C_ERR_INVALID, "scene %d: negative pair capacity", s);
  }
  return p2c::launch_batch_anyhit(scenes_host, scenes_dev, n_scenes, family_mask, scores_dev,
                                  reinterpret_cast<const unsigned long long*>(seeds_dev), top_k, interval_t0,
                                  interval_t1, *config, summaries_dev, group_detected_dev, evaluated_dev, hit_dev,
                                  workspace_dev, workspace_bytes, p2c::as_stream(stream));
}

int p2c_stub_scores(const uint64_t* pairs_dev, const uint64_t* count_dev, int64_t cap, int family, uint64_t seed,
                    double* scores_dev, void* stream) {
  if (cap < 0) return p2c::fail(P2C_ERR_INVALID, "capacity must be non-negative");
  if (family != 1 && family != 2) return p2c::fail(P2C_ERR_INVALID, "family must be 1 (vf) or 2 (ee)");
  if (cap == 0) return P2C_OK;
  if (pairs_dev == nullptr || scores_dev == nullptr) return p2c::fail(P2C_ERR_INVALID, "pair or score pointer is null");
  p2c::stub_scores_kernel<<<p2c::grid_for(cap, 256), 256, 0, p2c::as_stream(stream)>>>(
      reinterpret_cast<const unsigned long long*>(pairs_dev), reinterpret_cast<const unsigned long long*>(count_dev),
      cap, family, seed, scores_dev);
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

}  // extern "C"
