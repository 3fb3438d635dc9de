// features.cu — proposal feature rows of a proxy scene's candidates on the
// device: ComputeCandidateDensityStats (rt_candidate/candidate_stats.cpp:
// 128-170) and ExtractProposalFeatureRows / FillFeatureRow
// (proposal/proposal_features.cpp:122-205, 236-259), the 32-feature rows the
// learned scheduler reads, kept on the device after p2c_proxy_candidates.
//
//   1. density: a sort of the slab ids and one of (object, slab) give the
//      distinct slab and object counts and the cross-object same-slab pair
//      count (pairs in one slab minus pairs in one (slab, object)); each
//      element adds the number of earlier elements of its run;
//   2. the first proxy (in scene order) of each (slab, type, object, patch):
//      two stable sorts order the proxies by that tuple and then by index,
//      and every candidate side finds its proxy by binary search;
//   3. one thread per candidate forms the row with the reference's double
//      arithmetic (bit-identical with --fmad=false) and float clamps.
// p2c_runtime_feature_rows is the runtime form without a scene
// (BuildProposalFeatureRowsFromRuntimeCandidates, proposal_policy.cpp:568-592).
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>

#include "p2c_internal.cuh"

namespace p2c {
namespace {

constexpr int kThreads = 256;

unsigned grid_for(long long n) {
  const long long b = (n + kThreads - 1) / kThreads;
  return (unsigned)(b > 0 ? b : 1);
}

__host__ __device__ inline int id_bits(uint32_t hint) { return hint > 0 && hint < 32 ? (int)hint : 32; }

struct FeatureLayout {
  unsigned long long* acc;       // [0] same-slab pairs, [1] same-(slab, object) pairs, [2] slabs, [3] objects
  unsigned long long* key[2];    // n
  unsigned* val[2];              // n
  unsigned long long* k2;        // n: (slab << 8 | type) of the lookup order
  unsigned long long* ko;        // n: (object << patch_bits | patch) of the lookup order
  unsigned* idx;                 // n: proxy index of the lookup order
  void* tmp;
  size_t tmp_bytes;
  size_t total;
};

FeatureLayout carve(void* base, long long n) {
  FeatureLayout L{};
  size_t off = 0;
  char* b = static_cast<char*>(base);
  auto take = [&](size_t bytes) -> void* {
    void* p = b == nullptr ? nullptr : b + off;
    off += (std::max<size_t>(bytes, 1) + 255) & ~size_t(255);
    return p;
  };
  const size_t N = (size_t)std::max(n, 1ll);
  L.acc = static_cast<unsigned long long*>(take(32));
  for (int k = 0; k < 2; ++k) {
    L.key[k] = static_cast<unsigned long long*>(take(8 * N));
    L.val[k] = static_cast<unsigned*>(take(4 * N));
  }
  L.k2 = static_cast<unsigned long long*>(take(8 * N));
  L.ko = static_cast<unsigned long long*>(take(8 * N));
  L.idx = static_cast<unsigned*>(take(4 * N));
  size_t t = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, t, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (const unsigned*)nullptr, (unsigned*)nullptr, (int)N);
  L.tmp_bytes = t;
  L.tmp = take(t);
  L.total = off;
  return L;
}

// keys of the density sorts: which = 0 slab, 1 (object << slab_bits | slab)
__global__ void density_keys_kernel(p2c_proxy_scene sc, FeatureLayout L, int which, int slab_bits) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sc.n) return;
  L.key[0][i] = which == 0 ? (unsigned long long)sc.slab_id[i]
                           : ((unsigned long long)sc.object_id[i] << slab_bits) | sc.slab_id[i];
  L.val[0][i] = (unsigned)i;
}

// First position in [0, n) whose key is >= k.
__device__ __forceinline__ long long lower_bound(const unsigned long long* __restrict__ keys, long long n,
                                                 unsigned long long k) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long m = (lo + hi) >> 1;
    if (keys[m] < k) lo = m + 1;
    else hi = m;
  }
  return lo;
}

// Over sorted keys: every element adds the count of earlier elements of its
// run (sum over runs of C(run, 2)) to acc[pair_slot]; every run head adds 1
// to acc[head_slot] (with head_shift, runs of key >> head_shift).
__global__ void runs_kernel(FeatureLayout L, long long n, int pair_slot, int head_slot, int head_shift) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long pairs = 0, heads = 0;
  if (p < n) {
    const unsigned long long k = L.key[1][p];
    pairs = (unsigned long long)(p - lower_bound(L.key[1], n, k));
    heads = (p == 0 || (L.key[1][p - 1] >> head_shift) != (k >> head_shift)) ? 1ull : 0ull;
  }
  for (int o = 16; o > 0; o >>= 1) {
    pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    heads += __shfl_xor_sync(0xffffffffu, heads, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (pairs) atomicAdd(L.acc + pair_slot, pairs);
    if (heads) atomicAdd(L.acc + head_slot, heads);
  }
}

__device__ __forceinline__ double safe_ratio(unsigned long long num, unsigned long long den) {  // SafeRatio
  return den == 0 ? 0.0 : (double)num / (double)den;
}

// CandidateDensityStats from the counts (raw hits, candidates) of
// p2c_proxy_candidates and the run sums.  The sum of the candidates' hit
// counts is the raw hit count (every hit lands in one candidate).
__global__ void density_kernel(p2c_proxy_scene sc, FeatureLayout L, const uint64_t* counts,
                               p2c_candidate_density* out) {
  if (threadIdx.x != 0) return;
  p2c_candidate_density d{};
  d.query_id = sc.query_id;
  d.proxy_count = (unsigned long long)sc.n;
  d.slab_count = L.acc[2];
  d.object_count = L.acc[3];
  d.cross_object_same_slab_pair_count = L.acc[0] - L.acc[1];
  d.raw_hit_count = counts[0];
  d.compact_candidate_count = counts[1];
  d.raw_hits_per_proxy = safe_ratio(d.raw_hit_count, d.proxy_count);
  d.candidates_per_proxy = safe_ratio(d.compact_candidate_count, d.proxy_count);
  d.candidates_per_slab = safe_ratio(d.compact_candidate_count, d.slab_count);
  d.aabb_overlap_ratio = safe_ratio(d.raw_hit_count, d.cross_object_same_slab_pair_count);
  d.avg_rt_hits_per_candidate = safe_ratio(d.raw_hit_count, d.compact_candidate_count);
  *out = d;
}

__global__ void lookup_keys_kernel(p2c_proxy_scene sc, FeatureLayout L, int patch_bits) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sc.n) return;
  L.key[0][i] = ((unsigned long long)sc.object_id[i] << patch_bits) | sc.patch_id[i];
  L.val[0][i] = (unsigned)i;
}

// second (stable) pass key: (slab << 8 | type) of the proxies in (object, patch) order
__global__ void lookup_keys2_kernel(p2c_proxy_scene sc, FeatureLayout L) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= sc.n) return;
  const unsigned i = L.val[1][p];
  L.key[0][p] = ((unsigned long long)sc.slab_id[i] << 8) | sc.proxy_type[i];
}

__global__ void lookup_gather_kernel(p2c_proxy_scene sc, FeatureLayout L, int patch_bits) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= sc.n) return;
  const unsigned i = L.val[0][p];  // after the second pass
  L.idx[p] = i;
  L.ko[p] = ((unsigned long long)sc.object_id[i] << patch_bits) | sc.patch_id[i];
}

// Packed lookup key (all width hints set and fitting 64 bits): slab, type,
// object, patch in one word.  Ids past their hints flag bit 4 (the packing
// would alias them).
struct PackedKey {
  int ob, pb;  // bits of the object and patch fields (slab above type above object above patch)
  __device__ __forceinline__ unsigned long long make(unsigned slab, unsigned type, unsigned object,
                                                    unsigned patch) const {
    return ((((((unsigned long long)slab << 8) | type) << ob) | object) << pb) | patch;
  }
  __device__ __forceinline__ bool fits(unsigned slab, unsigned object, unsigned patch, int sb) const {
    return (sb >= 32 || !(slab >> sb)) && (ob >= 32 || !(object >> ob)) && (pb >= 32 || !(patch >> pb));
  }
};

__global__ void packed_keys_kernel(p2c_proxy_scene sc, FeatureLayout L, PackedKey pk, int sb,
                                   unsigned long long* err) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sc.n) return;
  const unsigned slab = sc.slab_id[i], obj = sc.object_id[i], patch = sc.patch_id[i];
  if (!pk.fits(slab, obj, patch, sb)) atomicOr(err, 4ull);
  L.key[0][i] = pk.make(slab, sc.proxy_type[i], obj, patch);
  L.val[0][i] = (unsigned)i;
}

__device__ __forceinline__ long long find_proxy_packed(const FeatureLayout& L, long long n, unsigned long long k) {
  const long long lo = lower_bound(L.k2, n, k);
  return (lo < n && L.k2[lo] == k) ? (long long)L.val[1][lo] : -1;
}

// FindCandidatePrimitive (:103-112): the smallest proxy index whose
// (slab, type, object, patch) equals the candidate side's; -1 if none.
__device__ __forceinline__ long long find_proxy(const FeatureLayout& L, long long n, unsigned long long k2,
                                                unsigned long long ko) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long m = (lo + hi) >> 1;
    const unsigned long long a = L.k2[m];
    if (a < k2 || (a == k2 && L.ko[m] < ko)) lo = m + 1;
    else hi = m;
  }
  return (lo < n && L.k2[lo] == k2 && L.ko[lo] == ko) ? (long long)L.idx[lo] : -1;
}

__device__ __forceinline__ double dmax0(double x) { return 0.0 < x ? x : 0.0; }     // std::max(0.0, x)
__device__ __forceinline__ double dmin_(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double dmax_(double a, double b) { return (a < b) ? b : a; }  // std::max

// ClampFeature (:82-88)
__device__ __forceinline__ float clamp_feature(double v) {
  if (!isfinite(v)) return 0.0f;
  const double c = v < -1.0e6 ? -1.0e6 : (1.0e6 < v ? 1.0e6 : v);
  return __double2float_rn(c);
}

__device__ __forceinline__ double extent(const double* b, int k) { return dmax0(b[3 + k] - b[k]); }  // AabbExtent
__device__ __forceinline__ double volume(const double* b) { return extent(b, 0) * extent(b, 1) * extent(b, 2); }
__device__ __forceinline__ double surface(const double* b) {  // AabbSurfaceArea
  const double x = extent(b, 0), y = extent(b, 1), z = extent(b, 2);
  return 2.0 * (x * y + y * z + z * x);
}
__device__ __forceinline__ double overlap(const double* l, const double* r, int k) {  // OverlapExtent
  return dmax0(dmin_(l[3 + k], r[3 + k]) - dmax_(l[k], r[k]));
}

__global__ void rows_kernel(p2c_proxy_scene sc, FeatureLayout L, const p2c_candidate_record* cand, long long cap,
                            const uint64_t* counts, const p2c_candidate_density* density,
                            p2c_proposal_feature_row* rows, unsigned long long* err, bool packed, PackedKey pk,
                            int sb) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long m = (long long)min((unsigned long long)counts[1], (unsigned long long)cap);
  if (c >= m) return;
  const p2c_candidate_record r = cand[c];
  p2c_proposal_feature_row row{};
  // ValidateCandidateRecord (common/validators.cpp:160-181)
  bool ok = r.schema_version == 1u && r.candidate_id != 0 && r.query_id != 0 &&
            (r.proxy_type_a == 1 || r.proxy_type_a == 2) && (r.proxy_type_b == 1 || r.proxy_type_b == 2) &&
            r.rt_hit_count != 0;
  for (int k = 0; k < 4; ++k) ok = ok && isfinite(r.motion_bound[k]) && !(r.motion_bound[k] < 0.0f);
  const long long n = sc.n;
  const int pb = id_bits(sc.patch_bits);
  long long ia, ib;
  if (packed) {  // a side with ids past the hints matches no proxy (all proxies fit them)
    ia = pk.fits(r.slab_id, r.object_a_id, r.patch_a_id, sb)
             ? find_proxy_packed(L, n, pk.make(r.slab_id, r.proxy_type_a, r.object_a_id, r.patch_a_id))
             : -1;
    ib = pk.fits(r.slab_id, r.object_b_id, r.patch_b_id, sb)
             ? find_proxy_packed(L, n, pk.make(r.slab_id, r.proxy_type_b, r.object_b_id, r.patch_b_id))
             : -1;
  } else {
    ia = find_proxy(L, n, ((unsigned long long)r.slab_id << 8) | r.proxy_type_a,
                    ((unsigned long long)r.object_a_id << pb) | r.patch_a_id);
    ib = find_proxy(L, n, ((unsigned long long)r.slab_id << 8) | r.proxy_type_b,
                    ((unsigned long long)r.object_b_id << pb) | r.patch_b_id);
  }
  if (!ok || ia < 0 || ib < 0) {
    atomicOr(err, (!ok ? 1ull : 0ull) | (ia < 0 || ib < 0 ? 2ull : 0ull));
    rows[c] = row;
    return;
  }
  const double* A = sc.bounds + 6 * ia;
  const double* B = sc.bounds + 6 * ib;
  const double* ma = sc.motion_bound + 4 * ia;
  const double* mb = sc.motion_bound + 4 * ib;
  const double t0 = sc.t0[ia], t1 = sc.t1[ia];
  const double va = volume(A), vb = volume(B);
  const double ov = overlap(A, B, 0) * overlap(A, B, 1) * overlap(A, B, 2);
  const double uv = dmax0(va + vb - ov);  // UnionVolume
  double dc[3];
  for (int k = 0; k < 3; ++k) dc[k] = 0.5 * (A[k] + A[3 + k]) - 0.5 * (B[k] + B[3 + k]);
  const p2c_candidate_density d = *density;
  float* f = row.features;
  f[0] = clamp_feature(t0);
  f[1] = clamp_feature(t1);
  f[2] = clamp_feature(dmax0(t1 - t0));
  f[3] = clamp_feature((double)r.rt_hit_count);
  f[4] = clamp_feature((double)r.proxy_type_a);
  f[5] = clamp_feature((double)r.proxy_type_b);
  for (int k = 0; k < 4; ++k) f[6 + k] = clamp_feature((double)r.motion_bound[k]);
  for (int k = 0; k < 3; ++k) {
    f[10 + k] = clamp_feature(extent(A, k));
    f[13 + k] = clamp_feature(extent(B, k));
  }
  f[16] = clamp_feature(va);
  f[17] = clamp_feature(vb);
  f[18] = clamp_feature(ov);
  f[19] = clamp_feature(uv > 0.0 ? ov / uv : 0.0);
  f[20] = clamp_feature(sqrt(dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2]));
  f[21] = clamp_feature(surface(A));
  f[22] = clamp_feature(surface(B));
  f[23] = clamp_feature(ma[3]);  // conservative radius
  f[24] = clamp_feature(mb[3]);
  f[25] = clamp_feature(ma[0]);  // translation bound
  f[26] = clamp_feature(mb[0]);
  f[27] = clamp_feature(ma[1]);  // rotation angle
  f[28] = clamp_feature(mb[1]);
  f[29] = clamp_feature(d.candidates_per_proxy);
  f[30] = clamp_feature(d.aabb_overlap_ratio);
  f[31] = clamp_feature(d.avg_rt_hits_per_candidate);
  row.schema_version = 1u;
  row.query_id = r.query_id;
  row.candidate_id = r.candidate_id;
  row.slab_id = r.slab_id;
  row.object_a_id = r.object_a_id;
  row.patch_a_id = r.patch_a_id;
  row.object_b_id = r.object_b_id;
  row.patch_b_id = r.patch_b_id;
  // IntervalBin (:90-94): the centre clamped to [0, nextafter(1, 0)], times 8
  double centre = 0.5 * (t0 + t1);
  const double below_one = 0x1.fffffffffffffp-1;
  centre = centre < 0.0 ? 0.0 : (below_one < centre ? below_one : centre);
  row.interval_targets[(unsigned)(centre * 8.0)] = 1.0f;
  row.family_targets[0] = 1.0f;
  row.family_targets[1] = 1.0f;
  row.priority_target = clamp_feature(0.5 * (double)r.rt_hit_count + 0.5 * d.candidates_per_proxy);
  row.cost_target = clamp_feature(1.0 + (double)r.motion_bound[3]);
  const double f19 = (double)f[19];
  row.uncertainty_target = clamp_feature(1.0 - (f19 < 1.0 ? f19 : 1.0));
  row.target_mask = 31u;
  rows[c] = row;
}

// BuildRuntimeFeatureRowFromDerived (proposal/proposal_policy.cpp:184-226):
// a row from the candidate alone, the three density ratios and the query's
// conservative family mask (sorted query ids with their masks; absent or 0:
// both families).
struct RuntimeDerived {
  double candidates_per_proxy, aabb_overlap_ratio, avg_hits;
};

__global__ void runtime_rows_kernel(const p2c_candidate_record* cand, long long n, RuntimeDerived dv,
                                    const unsigned long long* mask_query_ids, const unsigned* masks, long long n_masks,
                                    p2c_proposal_feature_row* rows, unsigned long long* err) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const p2c_candidate_record r = cand[c];
  p2c_proposal_feature_row row{};
  bool ok = r.schema_version == 1u && r.candidate_id != 0 && r.query_id != 0 &&
            (r.proxy_type_a == 1 || r.proxy_type_a == 2) && (r.proxy_type_b == 1 || r.proxy_type_b == 2) &&
            r.rt_hit_count != 0;
  for (int k = 0; k < 4; ++k) ok = ok && isfinite(r.motion_bound[k]) && !(r.motion_bound[k] < 0.0f);
  if (!ok) {
    atomicOr(err, 1ull);
    rows[c] = row;
    return;
  }
  unsigned mask = 3u;  // kFeatureFamilyPointTriangle | kFeatureFamilyEdgeEdge
  long long lo = 0, hi = n_masks;
  while (lo < hi) {
    const long long m = (lo + hi) >> 1;
    if (mask_query_ids[m] < r.query_id) lo = m + 1;
    else hi = m;
  }
  if (lo < n_masks && mask_query_ids[lo] == r.query_id && masks[lo] != 0u) mask = masks[lo];
  row.schema_version = 1u;
  row.query_id = r.query_id;
  row.candidate_id = r.candidate_id;
  row.slab_id = r.slab_id;
  row.object_a_id = r.object_a_id;
  row.patch_a_id = r.patch_a_id;
  row.object_b_id = r.object_b_id;
  row.patch_b_id = r.patch_b_id;
  float* f = row.features;
  f[1] = 1.0f;
  f[2] = 1.0f;
  f[3] = clamp_feature((double)r.rt_hit_count);
  f[4] = clamp_feature((double)r.proxy_type_a);
  f[5] = clamp_feature((double)r.proxy_type_b);
  for (int k = 0; k < 4; ++k) f[6 + k] = clamp_feature((double)r.motion_bound[k]);
  f[19] = clamp_feature(dv.aabb_overlap_ratio < 1.0 ? dv.aabb_overlap_ratio : 1.0);
  f[29] = clamp_feature(dv.candidates_per_proxy);
  f[30] = clamp_feature(dv.aabb_overlap_ratio);
  f[31] = clamp_feature(dv.avg_hits);
  row.interval_targets[0] = 1.0f;
  row.family_targets[0] = (mask & 1u) ? 1.0f : 0.0f;
  row.family_targets[1] = (mask & 2u) ? 1.0f : 0.0f;
  const double pr = 0.5 * (double)r.rt_hit_count + 0.5 * dv.candidates_per_proxy;
  row.priority_target = clamp_feature(pr < 1.0 ? pr : 1.0);
  const double cost = 1.0 + (double)r.rt_hit_count;
  row.cost_target = clamp_feature(1.0 < cost ? cost : 1.0);
  row.uncertainty_target = mask == 3u ? 0.25f : 0.0f;
  row.target_mask = 31u;
  rows[c] = row;
}

}  // namespace
}  // namespace p2c

extern "C" {

int p2c_runtime_feature_rows(const p2c_candidate_record* candidates_dev, int64_t n, uint64_t primitive_count,
                             uint64_t raw_hit_count, uint64_t compact_candidate_count,
                             const uint64_t* mask_query_ids_dev, const uint32_t* masks_dev, int64_t n_masks,
                             p2c_proposal_feature_row* rows_dev, uint64_t* error_word_dev, void* stream) {
  using namespace p2c;
  if (primitive_count == 0) return fail(P2C_ERR_INVALID, "CandidateDensityStats.proxy_count must be non-zero");
  if (n < 0 || n >= (1ll << 31) || n_masks < 0) return fail(P2C_ERR_INVALID, "row or mask count out of range");
  if (error_word_dev == nullptr || (n > 0 && (candidates_dev == nullptr || rows_dev == nullptr)) ||
      (n_masks > 0 && (mask_query_ids_dev == nullptr || masks_dev == nullptr)))
    return fail(P2C_ERR_INVALID, "candidate, row, mask or error word pointer is null");
  // MakeRuntimeDensityDerivedStats (proposal_policy.cpp:44-58)
  auto ratio = [](uint64_t num, uint64_t den) { return den == 0 ? 0.0 : (double)num / (double)den; };
  RuntimeDerived dv;
  dv.candidates_per_proxy = ratio(compact_candidate_count, primitive_count);
  dv.aabb_overlap_ratio = ratio(raw_hit_count, primitive_count >= 2 ? primitive_count / 2 : 1);
  dv.avg_hits = ratio(raw_hit_count, compact_candidate_count);
  cudaStream_t s = as_stream(stream);
  P2C_CUDA(cudaMemsetAsync(error_word_dev, 0, sizeof(uint64_t), s));
  if (n > 0)
    runtime_rows_kernel<<<grid_for(n), kThreads, 0, s>>>(candidates_dev, n, dv,
                                                         reinterpret_cast<const unsigned long long*>(mask_query_ids_dev),
                                                         masks_dev, n_masks, rows_dev,
                                                         reinterpret_cast<unsigned long long*>(error_word_dev));
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}


size_t p2c_proposal_feature_rows_workspace_bytes(int64_t n_proxies) {
  if (n_proxies < 0) return 0;
  return p2c::carve(nullptr, n_proxies).total + 256;
}

int p2c_proposal_feature_rows(const p2c_proxy_scene* scene, const p2c_candidate_record* candidates_dev,
                              int64_t cap, const uint64_t* counts_dev, p2c_candidate_density* density_dev,
                              p2c_proposal_feature_row* rows_dev, uint64_t* error_word_dev, void* workspace_dev,
                              size_t workspace_bytes, void* stream) {
  using namespace p2c;
  if (scene == nullptr) return fail(P2C_ERR_INVALID, "proxy scene pointer is null");
  if (scene->query_id == 0) return fail(P2C_ERR_INVALID, "ProxyScene.query_id is required");
  if (scene->n < 0 || scene->n >= (1ll << 31)) return fail(P2C_ERR_INVALID, "proxy count must lie in [0, 2^31)");
  if (cap < 0 || cap >= (1ll << 31)) return fail(P2C_ERR_INVALID, "candidate capacity must lie in [0, 2^31)");
  if (counts_dev == nullptr || density_dev == nullptr || error_word_dev == nullptr)
    return fail(P2C_ERR_INVALID, "counts, density or error word pointer is null");
  if (cap > 0 && (candidates_dev == nullptr || rows_dev == nullptr))
    return fail(P2C_ERR_INVALID, "candidate or row pointer is null");
  const long long n = scene->n;
  if (n > 0 && (scene->object_id == nullptr || scene->patch_id == nullptr || scene->slab_id == nullptr ||
                scene->proxy_type == nullptr || scene->t0 == nullptr || scene->t1 == nullptr ||
                scene->bounds == nullptr || scene->motion_bound == nullptr))
    return fail(P2C_ERR_INVALID, "proxy scene arrays are null");
  const size_t need = carve(nullptr, n).total;
  if (workspace_dev == nullptr || workspace_bytes < need)
    return fail(P2C_ERR_INVALID, "feature row workspace too small: %zu < %zu bytes", workspace_bytes, need);
  FeatureLayout L = carve(workspace_dev, n);
  cudaStream_t s = as_stream(stream);
  const p2c_proxy_scene sc = *scene;
  const int sb = id_bits(sc.slab_bits), ob = id_bits(sc.object_bits), pb = id_bits(sc.patch_bits);
  P2C_CUDA(cudaMemsetAsync(L.acc, 0, 32, s));
  P2C_CUDA(cudaMemsetAsync(error_word_dev, 0, sizeof(uint64_t), s));
  if (n > 0) {
    size_t tb;
    // density: runs of slab ids, then of (object, slab)
    density_keys_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L, 0, sb);
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.key[0], L.key[1], L.val[0], L.val[1], (int)n, 0, sb, s));
    runs_kernel<<<grid_for(n), kThreads, 0, s>>>(L, n, 0, 2, 0);
    density_keys_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L, 1, sb);
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.key[0], L.key[1], L.val[0], L.val[1], (int)n, 0, ob + sb,
                                             s));
    runs_kernel<<<grid_for(n), kThreads, 0, s>>>(L, n, 1, 3, sb);
  }
  const bool packed = sc.slab_bits > 0 && sc.object_bits > 0 && sc.patch_bits > 0 && sb + 8 + ob + pb <= 64;
  PackedKey pk{ob, pb};
  if (n > 0 && packed) {
    // lookup order in one sort of (slab, type, object, patch) words, ties by proxy index (stable)
    size_t tb = L.tmp_bytes;
    packed_keys_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L, pk, sb,
                                                         reinterpret_cast<unsigned long long*>(error_word_dev));
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.key[0], L.k2, L.val[0], L.val[1], (int)n, 0,
                                             sb + 8 + ob + pb, s));
  } else if (n > 0) {
    size_t tb;
    // lookup order: (slab, type, object, patch), ties by proxy index (stable passes)
    lookup_keys_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L, pb);
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.key[0], L.key[1], L.val[0], L.val[1], (int)n, 0, ob + pb,
                                             s));
    lookup_keys2_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L);
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.key[0], L.k2, L.val[1], L.val[0], (int)n, 0, sb + 8, s));
    lookup_gather_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L, pb);
  }
  density_kernel<<<1, 32, 0, s>>>(sc, L, counts_dev, density_dev);
  if (cap > 0)
    rows_kernel<<<grid_for(cap), kThreads, 0, s>>>(sc, L, candidates_dev, cap, counts_dev, density_dev, rows_dev,
                                                  reinterpret_cast<unsigned long long*>(error_word_dev), packed, pk,
                                                  sb);
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

}  // extern "C"
