// groups.cu — scheduled any-hit over candidate groups with conservative
// fallback replay, on the device.
//
// The scene tool's RunScheduledAnyHitRows
// (tools/scene_object_envelope_native_ti_walltime.cpp:1283-1410) is
// sequential: per group (an unordered object pair, GroupKey :756-770) it
// certifies the top-K candidates by score until the first hit, then replays
// every other candidate of each group without a hit, in candidate order,
// until the first hit.  Here both phases run on the persistent certifier:
//
//   1. prep: group id and a descending score key per candidate, group sizes;
//   2. two stable radix sorts order the candidates by (group, score desc,
//      index) and a scan of the group sizes gives every candidate its rank;
//   3. a third stable sort by min(rank, K) lays the proposals out rank-major
//      (all groups' first proposals, then all second ones, ...);
//   4. the engine certifies the proposals in that order; a hit lowers its
//      group's minimum hit rank, and a proposal behind a known hit is dropped
//      before it is evaluated (ones already running finish as speculation);
//   5. the candidates of groups without a proposal hit that are not
//      proposals are compacted in index order and certified the same way,
//      keyed by candidate index;
//   6. the calls of the sequential procedure are recovered exactly from the
//      final per-group minima: a proposal is called iff its rank is at most
//      its group's minimum hit rank, a fallback candidate iff its index is at
//      most its group's minimum fallback hit index.
//
// Every launch takes its sizes from device memory, so the whole sequence
// follows the broad phase without a host sync and captures into a graph.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>

#include "certify_core.cuh"
#include "certify_launch.cuh"
#include "scene_pairs.cuh"

namespace p2c {

int validate_scene(const p2c_scene* sc);

namespace {

constexpr unsigned kNone = 0xffffffffu;  // "no hit" in the per-group minima
constexpr int kMaxGroupObjects = 4096;   // n_obj^2 group table entries
constexpr int kThreads = 256;

struct AnyhitCounters {
  unsigned long long n_top;        // proposals (sum over groups of min(size, K))
  unsigned long long error_word;   // 4: non-finite geometry, 8: bad object id or pair index, 16: NaN score
  unsigned long long speculative;  // certificates computed but not called
  int fb_count;                    // fallback candidates (cub's selection count)
  int pad;
};

// Candidate state written by the engine: 0 not computed, 1 separation, 2 hit.
constexpr unsigned char kComputedSeparation = 1, kComputedHit = 2;

struct AnyhitLayout {
  CertifyScratch* sc = nullptr;
  AnyhitCounters* ctr = nullptr;
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

AnyhitLayout carve(void* base, long long cap, long long groups) {
  AnyhitLayout L;
  size_t off = 0;
  char* b = static_cast<char*>(base);
  auto take = [&](size_t bytes) -> void* {
    void* p = b == nullptr ? nullptr : b + off;
    off += (bytes + 255) & ~size_t(255);
    return p;
  };
  const size_t n = (size_t)std::max(cap, 1ll), g = (size_t)std::max(groups, 1ll);
  L.sc = static_cast<CertifyScratch*>(take(kScratchHeaderBytes + kPoolBytes));
  L.ctr = static_cast<AnyhitCounters*>(take(sizeof(AnyhitCounters)));
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

int bit_width(unsigned long long v) {
  int b = 0;
  while (v != 0ull) {
    ++b;
    v >>= 1;
  }
  return b;
}

__device__ __forceinline__ long long candidate_count(const unsigned long long* count, long long cap) {
  const long long c = (long long)*count;
  return c < cap ? c : cap;
}

// Descending order of scores as an ascending unsigned key: -0 ties with +0,
// NaN ranks after every number.
__device__ __forceinline__ unsigned long long score_key_desc(double s, bool& nan) {
  nan = isnan(s);
  if (nan) return ~0ull - 1ull;
  if (s == 0.0) s = 0.0;
  const unsigned long long b = (unsigned long long)__double_as_longlong(s);
  const unsigned long long asc = (b >> 63) ? ~b : (b | (1ull << 63));
  return ~asc;
}

// Adds 1 to table[key] for every active lane, one atomic per distinct key.
__device__ __forceinline__ void warp_count(unsigned* table, unsigned key, bool active) {
  const unsigned act = __activemask();
  const unsigned m = __match_any_sync(act, active ? key : kNone);
  if (active && (threadIdx.x & 31) == __ffs((int)m) - 1) atomicAdd(table + key, (unsigned)__popc(m));
}

__global__ void init_kernel(AnyhitLayout L, long long groups, p2c_anyhit_summary* summary) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < groups) {
    L.g_size[g] = 0u;
    L.g_min_hit[g] = kNone;
    L.g_min_fb[g] = kNone;
    L.g_fcalls[g] = 0ull;
  }
  if (g == 0) {
    *L.ctr = AnyhitCounters{};
    if (summary != nullptr) *summary = p2c_anyhit_summary{};
  }
}

__global__ void prep_kernel(ScenePairs sp, long long n_a, long long n_b, const int32_t* obj_a, const int32_t* obj_b,
                            int n_obj, const double* scores, const unsigned long long* count, long long cap,
                            AnyhitLayout L) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cap) return;
  const long long n = candidate_count(count, cap);
  const unsigned groups = (unsigned)n_obj * (unsigned)n_obj;
  unsigned g = groups;
  unsigned long long key = ~0ull;
  if (c < n) {
    const unsigned long long pair = sp.pairs[c];
    const long long a = (long long)(pair >> 32), b = (long long)(pair & 0xffffffffull);
    const int oa = a < n_a ? __ldg(obj_a + a) : -1, ob = b < n_b ? __ldg(obj_b + b) : -1;
    if (oa >= 0 && ob >= 0 && oa < n_obj && ob < n_obj) {
      const unsigned lo = (unsigned)min(oa, ob), hi = (unsigned)max(oa, ob);
      g = lo * (unsigned)n_obj + hi;
      bool nan = false;
      key = score_key_desc(scores[c], nan);
      if (nan) atomicOr(&L.ctr->error_word, 16ull);
    } else {
      atomicOr(&L.ctr->error_word, 8ull);
    }
  }
  L.grp[c] = g;
  L.state[c] = 0;
  L.skey[0][c] = key;
  L.val[0][c] = (unsigned)c;
  warp_count(L.g_size, g, g < groups);
}

__global__ void group_key_kernel(long long cap, AnyhitLayout L) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < cap) L.key32[0][p] = L.grp[L.val[1][p]];
}

// Rank of every candidate inside its group (sorted order is group, score
// desc, index) and the rank-major key of the proposal ordering.
__global__ void rank_kernel(long long cap, unsigned groups, unsigned K, AnyhitLayout L) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= cap) return;
  const unsigned c = L.val[0][p];
  const unsigned g = L.grp[c];
  unsigned r = kNone, key = K;
  if (g < groups) {
    r = (unsigned)p - L.g_start[g];
    key = r < K ? r : K;
  }
  L.rank[c] = r;
  L.key32[0][p] = key;
  const unsigned act = __activemask();
  const unsigned top = __ballot_sync(act, g < groups && r < K);
  if ((threadIdx.x & 31) == __ffs((int)act) - 1 && top != 0u)
    atomicAdd(&L.ctr->n_top, (unsigned long long)__popc(top));
}

// Fallback candidates: not a proposal, in a group without a proposal hit.
__global__ void fallback_flags_kernel(const unsigned long long* count, long long cap, unsigned groups, unsigned K,
                                      AnyhitLayout L) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cap) return;
  const long long n = candidate_count(count, cap);
  bool f = false;
  if (c < n) {
    const unsigned g = L.grp[c];
    f = g < groups && L.rank[c] >= K && L.g_min_hit[g] == kNone;
  }
  L.flags[c] = f ? 1 : 0;
  L.key32[0][c] = (unsigned)c;
}

// One phase of the any-hit as an engine problem over a work list of
// candidate indices.  order_key is the candidate's rank (proposals) or its
// index (fallback); min_hit holds the per-group minimum over hits.
struct AnyhitProblem {
  ScenePairs sp;
  int family;
  const unsigned* list;
  const unsigned long long* n_top;  // proposal phase: list length (else null)
  const int* n_fallback;            // fallback phase: list length (else null)
  const unsigned* grp;
  const unsigned* rank;  // null in the fallback phase: the key is the index
  unsigned* min_hit;
  unsigned char* state;
  unsigned long long* error_word;
  __device__ __forceinline__ long long count() const {
    return n_top != nullptr ? (long long)*n_top : (long long)*n_fallback;
  }
  __device__ __forceinline__ long long n(int f) const { return f == family ? count() : 0; }
  __device__ __forceinline__ unsigned order_key(unsigned c) const { return rank != nullptr ? __ldg(rank + c) : c; }
  __device__ __forceinline__ bool skip(int, long long q) const {
    const unsigned c = __ldg(list + q);
    return order_key(c) > volatile_load(min_hit + __ldg(grp + c));
  }
  __device__ __forceinline__ void load(int f, long long q, Geo& g, double& t0, double& t1, int& bad) const {
    const unsigned c = __ldg(list + q);
    bad = load_pair(sp, f, __ldg(sp.pairs + c), g) ? 0 : 2;
    t0 = sp.T0;
    t1 = sp.T1;
  }
  __device__ __forceinline__ void record(long long q, bool hit) const {
    const unsigned c = list[q];
    state[c] = hit ? kComputedHit : kComputedSeparation;
    if (hit) atomicMin(min_hit + grp[c], order_key(c));
  }
  __device__ __forceinline__ void finish(int, long long q, const Outcome& o) const {
    record(q, o.status != P2C_STATUS_SEPARATION);
  }
  __device__ __forceinline__ void invalid(int, long long q, int, double, double) const {
    atomicOr(error_word, 4ull);
    record(q, true);  // non-finite geometry is certified undecided: a conservative hit
  }
};

__global__ void __launch_bounds__(kCertifyThreads, kCertifyMinBlocks)
    anyhit_certify_kernel(const __grid_constant__ AnyhitProblem prob, const __grid_constant__ CertParams prm,
                          const __grid_constant__ EnginePools pools, CertifyScratch* scratch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EngineShared& sh = reinterpret_cast<EngineShared*>(smem_raw)[threadIdx.x >> 5];
  WarpStats st;
  const unsigned long long t_start = global_ns();
  const long long warps = (long long)gridDim.x * kCertifyWarps;
  const int fetch = (int)min(32ll, max(1ll, (prob.count() + warps - 1) / warps));
  const bool ok = run_engine<true, true, false>(prob, prm, fetch, fetch, false, sh, st, &scratch->engine, pools,
                                                t_start);
  flush_stats(st, ok, scratch);
}

// Calls of the sequential procedure from the final minima, per candidate.
__global__ void calls_kernel(const unsigned long long* count, long long cap, unsigned groups, unsigned K,
                             AnyhitLayout L, unsigned char* evaluated, unsigned char* hit_out) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cap) return;
  const long long n = candidate_count(count, cap);
  if (c >= n) return;
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
  if (fb_called && (threadIdx.x & 31) == __ffs((int)m) - 1) atomicAdd(L.g_fcalls + g, (unsigned long long)__popc(m));
  const unsigned spec = __ballot_sync(act, phase == 0 && st != 0);
  if ((threadIdx.x & 31) == __ffs((int)act) - 1 && spec != 0u)
    atomicAdd(&L.ctr->speculative, (unsigned long long)__popc(spec));
}

__global__ void groups_kernel(const unsigned long long* count, long long cap, unsigned groups, unsigned K,
                              AnyhitLayout L, unsigned char* detected_out, long long* pcalls_out,
                              long long* fcalls_out, p2c_anyhit_summary* summary) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= groups) return;
  const unsigned size = L.g_size[g];
  const unsigned mh = L.g_min_hit[g], mf = L.g_min_fb[g];
  const unsigned long long pc = size == 0u ? 0ull : (mh == kNone ? (unsigned long long)min(size, K) : mh + 1ull);
  const unsigned long long fc = L.g_fcalls[g];
  const bool det = size != 0u && (mh != kNone || mf != kNone);
  if (detected_out != nullptr) detected_out[g] = det ? 1 : 0;
  if (pcalls_out != nullptr) pcalls_out[g] = (long long)pc;
  if (fcalls_out != nullptr) fcalls_out[g] = (long long)fc;
  if (summary == nullptr) return;
  if (size != 0u) {
    atomicAdd((unsigned long long*)&summary->groups, 1ull);
    if (det) {
      atomicAdd((unsigned long long*)&summary->detected_groups, 1ull);
      atomicAdd((unsigned long long*)&summary->first_hit_rank_sum, pc + fc);
    }
    if (mh == kNone) atomicAdd((unsigned long long*)&summary->fallback_groups, 1ull);
    if (pc) atomicAdd((unsigned long long*)&summary->proposal_calls, pc);
    if (fc) atomicAdd((unsigned long long*)&summary->fallback_calls, fc);
  }
  if (g == 0) {
    summary->candidates = (unsigned long long)candidate_count(count, cap);
    summary->speculative = L.ctr->speculative;
    summary->error_word = L.ctr->error_word | L.sc->stats.error_word;
  }
}

unsigned grid_for(long long n, int threads) {
  const long long b = (n + threads - 1) / threads;
  return (unsigned)(b > 0 ? b : 1);
}

cudaError_t reset_engine(CertifyScratch* sc, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(&sc->engine, 0, sizeof(EngineState), s);
  if (e != cudaSuccess) return e;
  return cudaMemsetAsync(pools_at(sc).tasks, 0, kTaskCap * sizeof(SubtreeTask), s);
}

}  // namespace

int launch_group_anyhit(const p2c_scene& scene, int family, const unsigned long long* pairs, long long cap,
                        const unsigned long long* count, const double* scores, long long top_k, double T0, double T1,
                        const p2c_cert_config& cfg, unsigned char* evaluated, unsigned char* hit_out,
                        unsigned char* detected_out, long long* pcalls_out, long long* fcalls_out,
                        p2c_anyhit_summary* summary, void* ws, size_t ws_bytes, cudaStream_t s) {
  const long long groups = (long long)scene.n_obj * scene.n_obj;
  const AnyhitLayout need = carve(nullptr, cap, groups);
  if (ws == nullptr || ws_bytes < need.total)
    return fail(P2C_ERR_INVALID, "any-hit workspace too small: %zu < %zu bytes", ws_bytes, need.total);
  AnyhitLayout L = carve(ws, cap, groups);
  const unsigned K = (unsigned)std::min<long long>(top_k, cap);
  const unsigned G = (unsigned)groups;
  const int* obj_a = family == 1 ? scene.v_obj : scene.e_obj;
  const int* obj_b = family == 1 ? scene.f_obj : scene.e_obj;
  ScenePairs sp{scene.v_t0, scene.v_t1, scene.faces, scene.edges, pairs, T0, T1};

  P2C_CUDA(reset_scratch(L.sc, s, true));
  init_kernel<<<grid_for(groups, kThreads), kThreads, 0, s>>>(L, groups, summary);
  P2C_CUDA(cudaGetLastError());
  if (cap > 0) {
    const long long n_a = family == 1 ? scene.nv : scene.ne, n_b = family == 1 ? scene.nf : scene.ne;
    prep_kernel<<<grid_for(cap, kThreads), kThreads, 0, s>>>(sp, n_a, n_b, obj_a, obj_b, scene.n_obj, scores, count,
                                                             cap, L);
    P2C_CUDA(cudaGetLastError());
    size_t tb = L.tmp_bytes;
    // (score desc, index): stable over the index order of the input
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.skey[0], L.skey[1], L.val[0], L.val[1], (int)cap, 0, 64,
                                             s));
    group_key_kernel<<<grid_for(cap, kThreads), kThreads, 0, s>>>(cap, L);
    P2C_CUDA(cudaGetLastError());
    // (group, score desc, index)
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.key32[0], L.key32[1], L.val[1], L.val[0], (int)cap, 0,
                                             bit_width(G), s));
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceScan::ExclusiveSum(L.tmp, tb, L.g_size, L.g_start, (int)groups, s));
    rank_kernel<<<grid_for(cap, kThreads), kThreads, 0, s>>>(cap, G, K, L);
    P2C_CUDA(cudaGetLastError());
  }
  LaunchShape shape;
  int rc = certify_shape(anyhit_certify_kernel, &shape);
  if (rc != P2C_OK) return rc;
  const CertParams prm = make_params(cfg, shape, 32ll * shape.grid * kCertifyWarps);
  if (cap > 0 && K > 0) {
    // proposals rank-major: (rank, group, score desc, index)
    size_t tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.key32[0], L.key32[1], L.val[0], L.val[1], (int)cap, 0,
                                             bit_width(K), s));
    const AnyhitProblem prop{sp, family, L.val[1], &L.ctr->n_top, nullptr, L.grp, L.rank, L.g_min_hit, L.state,
                             &L.ctr->error_word};
    anyhit_certify_kernel<<<shape.grid, kCertifyThreads, shape.smem, s>>>(prop, prm, pools_at(L.sc), L.sc);
    P2C_CUDA(cudaGetLastError());
  }
  if (cap > 0) {
    fallback_flags_kernel<<<grid_for(cap, kThreads), kThreads, 0, s>>>(count, cap, G, K, L);
    P2C_CUDA(cudaGetLastError());
    size_t tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceSelect::Flagged(L.tmp, tb, L.key32[0], L.flags, L.fb_list, &L.ctr->fb_count, (int)cap, s));
    P2C_CUDA(reset_engine(L.sc, s));
    const AnyhitProblem fb{sp, family, L.fb_list, nullptr, &L.ctr->fb_count, L.grp, nullptr, L.g_min_fb, L.state,
                           &L.ctr->error_word};
    anyhit_certify_kernel<<<shape.grid, kCertifyThreads, shape.smem, s>>>(fb, prm, pools_at(L.sc), L.sc);
    P2C_CUDA(cudaGetLastError());
    calls_kernel<<<grid_for(cap, kThreads), kThreads, 0, s>>>(count, cap, G, K, L, evaluated, hit_out);
    P2C_CUDA(cudaGetLastError());
  }
  groups_kernel<<<grid_for(groups, kThreads), kThreads, 0, s>>>(count, cap, G, K, L, detected_out, pcalls_out,
                                                                fcalls_out, summary);
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

}  // namespace p2c

extern "C" {

size_t p2c_group_anyhit_workspace_bytes(int64_t cap, int32_t n_obj) {
  if (cap < 0 || n_obj < 1) return 0;
  return p2c::carve(nullptr, cap, (long long)n_obj * n_obj).total;
}

int p2c_group_anyhit(const p2c_scene* scene, int family, const uint64_t* pairs_dev, int64_t cap,
                     const uint64_t* count_dev, const double* scores_dev, int64_t top_k, double interval_t0,
                     double interval_t1, const p2c_cert_config* config, uint8_t* evaluated_dev, uint8_t* hit_dev,
                     uint8_t* group_detected_dev, int64_t* group_proposal_calls_dev,
                     int64_t* group_fallback_calls_dev, p2c_anyhit_summary* summary_dev, void* workspace_dev,
                     size_t workspace_bytes, void* stream) {
  int rc = p2c::validate_scene(scene);
  if (rc != P2C_OK) return rc;
  if (family != 1 && family != 2) return p2c::fail(P2C_ERR_INVALID, "family must be 1 (vf) or 2 (ee)");
  if (scene->n_obj < 1 || scene->n_obj > p2c::kMaxGroupObjects)
    return p2c::fail(P2C_ERR_INVALID, "scene n_obj must lie in [1, %d] for candidate groups",
                     p2c::kMaxGroupObjects);
  if (config == nullptr) return p2c::fail(P2C_ERR_INVALID, "CertificateEngineConfig pointer is null");
  rc = p2c::validate_cert_config(*config, interval_t0, interval_t1);
  if (rc != P2C_OK) return rc;
  if (cap < 0 || cap >= (1ll << 31)) return p2c::fail(P2C_ERR_INVALID, "candidate capacity must lie in [0, 2^31)");
  if (top_k < 0) return p2c::fail(P2C_ERR_INVALID, "proposal top_k must be non-negative");
  if (count_dev == nullptr) return p2c::fail(P2C_ERR_INVALID, "count pointer is null");
  if (cap > 0 && (pairs_dev == nullptr || scores_dev == nullptr))
    return p2c::fail(P2C_ERR_INVALID, "pair or score pointer is null");
  return p2c::launch_group_anyhit(
      *scene, family, reinterpret_cast<const unsigned long long*>(pairs_dev), cap,
      reinterpret_cast<const unsigned long long*>(count_dev), scores_dev, top_k, interval_t0, interval_t1, *config,
      evaluated_dev, hit_dev, group_detected_dev, reinterpret_cast<long long*>(group_proposal_calls_dev),
      reinterpret_cast<long long*>(group_fallback_calls_dev), summary_dev, workspace_dev, workspace_bytes,
      p2c::as_stream(stream));
}

}  // extern "C"

#ifdef P2C_ENGINE_PROFILE
// Measurement build only: the engine phase clock of this file's kernels (see
// certify_engine.cuh), read and cleared by the host.
extern "C" int p2c_engine_profile_groups(unsigned long long* out16, int clear) {
  if (cudaMemcpyFromSymbol(out16, p2c::g_engine_prof, 16 * sizeof(unsigned long long)) != cudaSuccess) return 2;
  if (clear) {
    static const unsigned long long zero[16] = {};
    if (cudaMemcpyToSymbol(p2c::g_engine_prof, zero, sizeof(zero)) != cudaSuccess) return 2;
  }
  return 0;
}
#endif
