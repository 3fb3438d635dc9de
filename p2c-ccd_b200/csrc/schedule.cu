// schedule.cu — the runtime exact work queue from proposals on the device:
// ScheduleRuntimeExactWorkItemsFromProposals (proposal/proposal_policy.cpp:
// 595-742), and the binding's aligned-array form
// (bindings/py_module.cpp:1088-1174).
//
// Per candidate: its feature row and proposal output (mode 0: found by
// candidate id through sorted copies; mode 1: the row and output at the same
// position), the fallback decision (missing, invalid, out-of-distribution or
// uncertain proposal), and one ExactWorkItem; then a stable radix sort by
// priority, descending (the reference's std::stable_sort with `>`: equal
// priorities keep candidate order, -0 and +0 are equal), work item ids in
// queue order, the reorder count and the checks.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>

#include "p2c_internal.cuh"

namespace p2c {
namespace {

constexpr int kThreads = 256;
constexpr unsigned kFull = 0xffffffffu;
constexpr uint8_t kSourceRefined = 1, kSourceFallback = 2;

// error word bits
constexpr unsigned long long kErrCandidate = 1, kErrRowId = 2, kErrOutputId = 4, kErrDuplicateCandidate = 8,
                             kErrWorkItem = 16, kErrNoFamily = 32, kErrUnknownFamily = 64, kErrOrder = 128;

unsigned grid_for(long long n) {
  const long long b = (n + kThreads - 1) / kThreads;
  return (unsigned)(b > 0 ? b : 1);
}

struct SchedLayout {
  unsigned long long* acc;   // [0..9] stats, [10] error word, [11] / [12] first position of a family fault
  unsigned long long* ids;   // scratch ids (max n)
  unsigned* idx;             // scratch positions
  unsigned long long* row_ids;
  unsigned* row_idx;
  unsigned long long* out_ids;
  unsigned* out_idx;
  unsigned long long* cand_ids;
  unsigned* pkey[2];
  unsigned* order[2];
  p2c_exact_work_item* staged;
  void* tmp;
  size_t tmp_bytes;
  size_t total;
};

SchedLayout carve(void* base, long long nc, long long nr, long long no) {
  SchedLayout L{};
  size_t off = 0;
  char* b = static_cast<char*>(base);
  auto take = [&](size_t bytes) -> void* {
    void* p = b == nullptr ? nullptr : b + off;
    off += (std::max<size_t>(bytes, 1) + 255) & ~size_t(255);
    return p;
  };
  const size_t C = (size_t)std::max(nc, 1ll), R = (size_t)std::max(nr, 1ll), O = (size_t)std::max(no, 1ll);
  const size_t M = std::max(C, std::max(R, O));
  L.acc = static_cast<unsigned long long*>(take(16 * 8));
  L.ids = static_cast<unsigned long long*>(take(8 * M));
  L.idx = static_cast<unsigned*>(take(4 * M));
  L.row_ids = static_cast<unsigned long long*>(take(8 * R));
  L.row_idx = static_cast<unsigned*>(take(4 * R));
  L.out_ids = static_cast<unsigned long long*>(take(8 * O));
  L.out_idx = static_cast<unsigned*>(take(4 * O));
  L.cand_ids = static_cast<unsigned long long*>(take(8 * C));
  for (int k = 0; k < 2; ++k) {
    L.pkey[k] = static_cast<unsigned*>(take(4 * C));
    L.order[k] = static_cast<unsigned*>(take(4 * C));
  }
  L.staged = static_cast<p2c_exact_work_item*>(take(sizeof(p2c_exact_work_item) * C));
  size_t a = 0, c = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, a, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (const unsigned*)nullptr, (unsigned*)nullptr, (int)M);
  cub::DeviceRadixSort::SortPairs(nullptr, c, (const unsigned*)nullptr, (unsigned*)nullptr,
                                  (const unsigned*)nullptr, (unsigned*)nullptr, (int)C);
  L.tmp_bytes = std::max(a, c);
  L.tmp = take(L.tmp_bytes);
  L.total = off;
  return L;
}

__global__ void row_ids_kernel(const p2c_proposal_feature_row* rows, long long n, SchedLayout L) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  L.ids[i] = rows[i].candidate_id;
  L.idx[i] = (unsigned)i;
}

__global__ void output_ids_kernel(const p2c_proposal_output* outs, long long n, SchedLayout L) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  L.ids[i] = outs[i].candidate_id;
  L.idx[i] = (unsigned)i;
}

__global__ void candidate_ids_kernel(const p2c_candidate_record* cand, long long n, SchedLayout L) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  L.ids[i] = cand[i].candidate_id;
}

// Sorted ids: a zero or a repeated id sets `bit`.
__global__ void id_check_kernel(const unsigned long long* sorted, long long n, unsigned long long bit,
                                bool zero_is_error, SchedLayout L) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if ((zero_is_error && sorted[i] == 0) || (i > 0 && sorted[i] == sorted[i - 1])) atomicOr(L.acc + 10, bit);
}

__device__ __forceinline__ long long find_id(const unsigned long long* sorted, const unsigned* idx, long long n,
                                             unsigned long long id) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long m = (lo + hi) >> 1;
    if (sorted[m] < id) lo = m + 1;
    else hi = m;
  }
  return (lo < n && sorted[lo] == id) ? (long long)idx[lo] : -1;
}

__device__ __forceinline__ bool finite_f(float v) { return isfinite(v); }

// HasNonFiniteProposal (:322-335) or ValidateProposalOutput failing
// (common/validators.cpp:183-206)
__device__ __forceinline__ bool invalid_output(const p2c_proposal_output& o) {
  bool bad = o.candidate_id == 0;
  for (int k = 0; k < 8; ++k) bad = bad || !finite_f(o.interval_scores[k]) || !finite_f(o.family_scores[k]);
  bad = bad || !finite_f(o.priority_score) || !finite_f(o.cost_score) || !finite_f(o.uncertainty_score);
  return bad || o.cost_score < 0.0f || o.uncertainty_score < 0.0f;
}

// IsProposalFeatureRowOod (:420-428)
__device__ __forceinline__ bool row_ood(const p2c_proposal_feature_row& r, float threshold) {
  bool ood = false;
  for (int k = 0; k < 32; ++k) ood = ood || !finite_f(r.features[k]) || fabsf(r.features[k]) > threshold;
  return ood;
}

// ValidateCandidateRecord (common/validators.cpp:160-181)
__device__ __forceinline__ bool candidate_ok(const p2c_candidate_record& r) {
  bool ok = r.schema_version == 1u && r.candidate_id != 0 && r.query_id != 0 &&
            (r.proxy_type_a == 1 || r.proxy_type_a == 2) && (r.proxy_type_b == 1 || r.proxy_type_b == 2) &&
            r.rt_hit_count != 0;
  for (int k = 0; k < 4; ++k) ok = ok && finite_f(r.motion_bound[k]) && !(r.motion_bound[k] < 0.0f);
  return ok;
}

// Descending, stable radix key of a float priority; -0 and +0 share a key.
__device__ __forceinline__ unsigned priority_key(float p) {
  const float q = p + 0.0f;  // -0 -> +0
  const unsigned b = __float_as_uint(q);
  const unsigned asc = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  return ~asc;
}

struct SchedParams {
  int mode;  // 0: candidates with lookups, 1: aligned rows / outputs, 2: dummy proposals, 3: raw bypass
  p2c_scheduling_config cfg;
  long long n, n_rows, n_outputs, n_masks;
  double candidates_per_proxy, aabb_overlap_ratio, avg_hits;  // mode 2: RuntimeDensityDerivedStats
};

// ClampRuntimeFeature (proposal_policy.cpp:30-35)
__device__ __forceinline__ float runtime_clamp(double v) {
  if (!isfinite(v)) return 0.0f;
  const double c = v < -1.0e6 ? -1.0e6 : (1.0e6 < v ? 1.0e6 : v);
  return __double2float_rn(c);
}

// The query's conservative mask from the sorted (query id, mask) table:
// BaseFamilyMaskForRuntimeQuery's two-argument form (:135-144) when
// `nonzero_only` (a zero mask counts as absent), else unordered_map::at.
__device__ __forceinline__ unsigned query_mask(const unsigned long long* qids, const unsigned* masks, long long n,
                                               unsigned long long q, bool nonzero_only) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long m = (lo + hi) >> 1;
    if (qids[m] < q) lo = m + 1;
    else hi = m;
  }
  if (lo < n && qids[lo] == q && (!nonzero_only || masks[lo] != 0u)) return masks[lo];
  return 3u;
}

// NormalizedDummyFamilyScores (:156-175): equal weights over the mask's families.
__device__ __forceinline__ void dummy_family_scores(unsigned base, float* s0, float* s1) {
  bool a0 = (base & 1u) != 0u, a1 = (base & 2u) != 0u;
  if (!a0 && !a1) a0 = a1 = true;
  const float w = 1.0f / (float)((a0 ? 1 : 0) + (a1 ? 1 : 0));
  *s0 = a0 ? w : 0.0f;
  *s1 = a1 ? w : 0.0f;
}

// IsRuntimeCandidateOod (:245-270)
__device__ __forceinline__ bool runtime_ood(const p2c_candidate_record& r, const SchedParams& P) {
  const double thr = (double)P.cfg.ood_abs_feature_threshold;
  const double capped = P.aabb_overlap_ratio < 1.0 ? P.aabb_overlap_ratio : 1.0;
  const double v[8] = {1.0, (double)r.rt_hit_count, (double)r.proxy_type_a, (double)r.proxy_type_b,
                       capped, P.candidates_per_proxy, P.aabb_overlap_ratio, P.avg_hits};
  bool ood = false;
  for (int k = 0; k < 8; ++k) ood = ood || !isfinite(v[k]) || fabs(v[k]) > thr;
  for (int k = 0; k < 4; ++k)
    ood = ood || !isfinite(r.motion_bound[k]) || fabsf(r.motion_bound[k]) > P.cfg.ood_abs_feature_threshold;
  return ood;
}

// RuntimePriorityTarget (:237-241)
__device__ __forceinline__ float runtime_priority(const p2c_candidate_record& r, const SchedParams& P) {
  const double x = 0.5 * (double)r.rt_hit_count + 0.5 * P.candidates_per_proxy;
  return runtime_clamp(x < 1.0 ? x : 1.0);
}

__device__ __forceinline__ void warp_add(unsigned long long* dst, unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

__global__ void decide_kernel(SchedParams P, const p2c_candidate_record* cand, const p2c_proposal_feature_row* rows,
                              const p2c_proposal_output* outs, const unsigned long long* mask_qids,
                              const unsigned* masks, SchedLayout L) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < P.n;
  unsigned long long f_missing = 0, f_invalid = 0, f_ood = 0, f_unc = 0, f_any = 0;
  if (live && P.mode >= 2) {  // RunDummyProposalScheduleFromRuntimeCandidates (:744-858) / the raw bypass
    const p2c_candidate_record r = cand[i];
    if (!candidate_ok(r)) atomicOr(L.acc + 10, kErrCandidate);
    p2c_exact_work_item it{};
    it.parent_candidate_id = r.candidate_id;
    it.query_id = r.query_id;
    it.slab_id = r.slab_id;
    it.patch_a_id = r.patch_a_id;
    it.patch_b_id = r.patch_b_id;
    it.interval_t0 = P.cfg.fallback_interval_t0;
    it.interval_t1 = P.cfg.fallback_interval_t1;
    const unsigned base = query_mask(mask_qids, masks, P.n_masks, r.query_id, P.mode == 2);
    it.feature_family_mask = base;
    it.priority_score = (float)r.rt_hit_count;
    it.source = 0;  // ProposalSource::kRaw
    if (P.mode == 2) {
      const bool ood = runtime_ood(r, P);
      f_any = f_ood = ood;
      it.source = kSourceFallback;
      if (!ood) {
        float s0, s1;
        dummy_family_scores(base, &s0, &s1);
        unsigned m = base;
        if (s0 >= P.cfg.family_score_threshold) m |= 1u;
        if (s1 >= P.cfg.family_score_threshold) m |= 2u;
        it.feature_family_mask = m;
        const float pr = runtime_priority(r, P);
        it.priority_score = 0.0f < pr ? pr : 0.0f;  // std::max(0.0F, ...)
        it.source = kSourceRefined;
      }
    }
    L.staged[i] = it;
    L.pkey[0][i] = priority_key(it.priority_score);
    L.order[0][i] = (unsigned)i;
  } else if (live) {
    const p2c_scheduling_config& c = P.cfg;
    long long ir = -1, io = -1;
    p2c_exact_work_item it{};
    float fallback_priority = 0.0f;
    if (P.mode == 0) {
      const p2c_candidate_record r = cand[i];
      if (!candidate_ok(r)) atomicOr(L.acc + 10, kErrCandidate);
      ir = find_id(L.row_ids, L.row_idx, P.n_rows, r.candidate_id);
      io = find_id(L.out_ids, L.out_idx, P.n_outputs, r.candidate_id);
      it.parent_candidate_id = r.candidate_id;
      it.query_id = r.query_id;
      it.slab_id = r.slab_id;
      it.patch_a_id = r.patch_a_id;
      it.patch_b_id = r.patch_b_id;
      fallback_priority = (float)r.rt_hit_count;
    } else {
      const p2c_proposal_feature_row& row = rows[i];
      if (row.candidate_id == 0 || outs[i].candidate_id != row.candidate_id) atomicOr(L.acc + 10, kErrOrder);
      ir = io = i;
      it.parent_candidate_id = row.candidate_id;
      it.query_id = row.query_id;
      it.slab_id = row.slab_id;
      it.patch_a_id = row.patch_a_id;
      it.patch_b_id = row.patch_b_id;
      fallback_priority = row.features[3];
    }
    const bool missing = io < 0;
    const bool invalid = !missing && invalid_output(outs[io]);
    const bool ood = ir < 0 || row_ood(rows[ir], c.ood_abs_feature_threshold);
    const bool unc = !missing && finite_f(outs[io].uncertainty_score) &&
                     outs[io].uncertainty_score >= c.uncertainty_fallback_threshold;
    const bool fallback = missing || invalid || ood || unc;
    f_missing = missing;
    f_invalid = invalid;
    f_ood = ood;
    f_unc = unc;
    f_any = fallback;
    // BaseFamilyMaskForRuntimeQuery (:137-146): the query's mask if present and non-zero
    unsigned base = c.conservative_feature_family_mask;
    long long lo = 0, hi = P.n_masks;
    while (lo < hi) {
      const long long m = (lo + hi) >> 1;
      if (mask_qids[m] < it.query_id) lo = m + 1;
      else hi = m;
    }
    if (lo < P.n_masks && mask_qids[lo] == it.query_id && masks[lo] != 0u) base = masks[lo];
    it.interval_t0 = c.fallback_interval_t0;
    it.interval_t1 = c.fallback_interval_t1;
    it.feature_family_mask = base;
    it.priority_score = fallback_priority;
    it.source = kSourceFallback;
    if (!fallback) {  // PredictedFamilyMaskFromScores (:298-308)
      const p2c_proposal_output& o = outs[io];
      unsigned predicted = 0;
      if (o.family_scores[0] >= c.family_score_threshold) predicted |= 1u;
      if (o.family_scores[1] >= c.family_score_threshold) predicted |= 2u;
      it.feature_family_mask = base | predicted;
      it.priority_score = o.priority_score;
      it.source = kSourceRefined;
    }
    L.staged[i] = it;
    L.pkey[0][i] = priority_key(it.priority_score);
    L.order[0][i] = (unsigned)i;
  }
  warp_add(L.acc + 3, f_any);
  warp_add(L.acc + 4, f_missing);
  warp_add(L.acc + 5, f_invalid);
  warp_add(L.acc + 6, f_ood);
  warp_add(L.acc + 7, f_unc);
}

// Work item ids in queue order, reorder count and ValidateExactWorkItem
// (common/validators.cpp:207-230) plus the family checks (:718-736).
__global__ void write_kernel(SchedParams P, const unsigned* order, const p2c_candidate_record* cand,
                             const p2c_proposal_feature_row* rows, p2c_exact_work_item* items, SchedLayout L) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long reordered = 0;
  if (p < P.n) {
    p2c_exact_work_item it = L.staged[order[p]];
    it.work_item_id = P.cfg.first_work_item_id + (unsigned long long)p;
    const unsigned long long original = P.mode == 1 ? rows[p].candidate_id : cand[p].candidate_id;
    reordered = it.parent_candidate_id != original ? 1ull : 0ull;
    const bool interval_ok = isfinite(it.interval_t0) && isfinite(it.interval_t1) && !(it.interval_t0 < 0.0) &&
                             !(it.interval_t1 > 1.0) && !(it.interval_t0 > it.interval_t1);  // ValidateUnitInterval
    const bool ok = it.work_item_id != 0 && it.parent_candidate_id != 0 && it.query_id != 0 && interval_ok &&
                    it.feature_family_mask != 0 && finite_f(it.priority_score);
    unsigned long long e = ok ? 0ull : kErrWorkItem;
    if (P.mode == 0) {  // per item the reference checks a missing family first, then unknown bits
      if ((it.feature_family_mask & 3u) == 0u) {
        e |= kErrNoFamily;
        atomicMin(L.acc + 11, (unsigned long long)p);
      } else if (it.feature_family_mask & ~3u) {
        e |= kErrUnknownFamily;
        atomicMin(L.acc + 12, (unsigned long long)p);
      }
    }
    if (e) atomicOr(L.acc + 10, e);
    items[p] = it;
  }
  warp_add(L.acc + 8, reordered);
}

__global__ void stats_kernel(SchedParams P, SchedLayout L, p2c_schedule_stats* stats, uint64_t* err) {
  if (threadIdx.x != 0) return;
  p2c_schedule_stats s{};
  s.raw_candidate_count = (unsigned long long)P.n;
  s.proposal_output_count = (unsigned long long)P.n_outputs;
  s.work_item_count = (unsigned long long)P.n;
  s.fallback_count = L.acc[3];
  s.missing_proposal_fallback_count = L.acc[4];
  s.invalid_proposal_fallback_count = L.acc[5];
  s.ood_fallback_count = L.acc[6];
  s.high_uncertainty_fallback_count = L.acc[7];
  s.reordered_count = L.acc[8];
  s.monotonic_safe = L.acc[10] == 0 ? 1ull : 0ull;
  *stats = s;
  err[0] = L.acc[10];
  err[1] = L.acc[11];
  err[2] = L.acc[12];
}

// The dummy proposal outputs of materialized rows (:787-800): the row's
// interval targets, the normalized family scores, non-negative priority and
// cost targets, uncertainty 1 for an out-of-distribution candidate.
__global__ void dummy_outputs_kernel(SchedParams P, const p2c_candidate_record* cand,
                                     const p2c_proposal_feature_row* rows, const unsigned long long* mask_qids,
                                     const unsigned* masks, p2c_proposal_output* outs) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const p2c_candidate_record r = cand[i];
  const p2c_proposal_feature_row& row = rows[i];
  p2c_proposal_output o{};
  o.candidate_id = r.candidate_id;
  for (int k = 0; k < 8; ++k) o.interval_scores[k] = row.interval_targets[k];
  dummy_family_scores(query_mask(mask_qids, masks, P.n_masks, r.query_id, true), &o.family_scores[0],
                      &o.family_scores[1]);
  o.priority_score = 0.0f < row.priority_target ? row.priority_target : 0.0f;
  o.cost_score = 0.0f < row.cost_target ? row.cost_target : 0.0f;
  o.uncertainty_score = runtime_ood(r, P) ? 1.0f : (0.0f < row.uncertainty_target ? row.uncertainty_target : 0.0f);
  outs[i] = o;
}

__global__ void init_acc_kernel(SchedLayout L) {
  if (threadIdx.x == 0) L.acc[11] = L.acc[12] = ~0ull;
}

// IsValidSchedulingConfig (:88-122), with the reference's messages.
int check_config(const p2c_scheduling_config& c) {
  if (c.first_work_item_id == 0)
    return fail(P2C_ERR_INVALID, "ProposalSchedulingConfig.first_work_item_id must be non-zero");
  if (c.conservative_feature_family_mask == 0)
    return fail(P2C_ERR_INVALID, "ProposalSchedulingConfig.conservative_feature_family_mask must be non-zero");
  if (c.conservative_feature_family_mask & ~3u)
    return fail(P2C_ERR_INVALID, "ProposalSchedulingConfig.conservative_feature_family_mask has unknown bits");
  if (!std::isfinite(c.fallback_interval_t0) || !std::isfinite(c.fallback_interval_t1) ||
      c.fallback_interval_t0 < 0.0 || c.fallback_interval_t1 > 1.0 || c.fallback_interval_t0 > c.fallback_interval_t1)
    return fail(P2C_ERR_INVALID, "ProposalSchedulingConfig fallback interval must lie in [0, 1]");
  if (!std::isfinite(c.family_score_threshold))
    return fail(P2C_ERR_INVALID, "ProposalSchedulingConfig.family_score_threshold must be finite");
  if (!std::isfinite(c.uncertainty_fallback_threshold) || c.uncertainty_fallback_threshold < 0.0f)
    return fail(P2C_ERR_INVALID, "ProposalSchedulingConfig.uncertainty_fallback_threshold must be non-negative");
  if (!std::isfinite(c.ood_abs_feature_threshold) || c.ood_abs_feature_threshold <= 0.0f)
    return fail(P2C_ERR_INVALID, "ProposalSchedulingConfig.ood_abs_feature_threshold must be positive");
  return P2C_OK;
}

}  // namespace
}  // namespace p2c

extern "C" {

size_t p2c_schedule_work_items_workspace_bytes(int64_t n_candidates, int64_t n_rows, int64_t n_outputs) {
  if (n_candidates < 0 || n_rows < 0 || n_outputs < 0) return 0;
  return p2c::carve(nullptr, n_candidates, n_rows, n_outputs).total + 256;
}

int p2c_schedule_work_items(int mode, const p2c_candidate_record* candidates_dev, int64_t n_candidates,
                            const p2c_proposal_feature_row* rows_dev, int64_t n_rows,
                            const p2c_proposal_output* outputs_dev, int64_t n_outputs,
                            const uint64_t* mask_query_ids_dev, const uint32_t* masks_dev, int64_t n_masks,
                            const p2c_scheduling_config* config, p2c_exact_work_item* items_dev,
                            p2c_schedule_stats* stats_dev, uint64_t* error_dev, void* workspace_dev,
                            size_t workspace_bytes, void* stream) {
  using namespace p2c;
  if (config == nullptr) return fail(P2C_ERR_INVALID, "scheduling config pointer is null");
  if (int rc = check_config(*config)) return rc;
  if (mode != 0 && mode != 1) return fail(P2C_ERR_INVALID, "mode must be 0 (candidates) or 1 (aligned arrays)");
  if (n_candidates < 0 || n_rows < 0 || n_outputs < 0 || n_masks < 0 || n_candidates >= (1ll << 31) ||
      n_rows >= (1ll << 31) || n_outputs >= (1ll << 31))
    return fail(P2C_ERR_INVALID, "counts must lie in [0, 2^31)");
  if (mode == 1 && n_rows != n_outputs)
    return fail(P2C_ERR_INVALID, "feature row and proposal output array lengths must match");
  const long long n = mode == 0 ? n_candidates : n_rows;
  if (stats_dev == nullptr || error_dev == nullptr || (n > 0 && items_dev == nullptr) ||
      (mode == 0 && n > 0 && candidates_dev == nullptr) || (n_rows > 0 && rows_dev == nullptr) ||
      (n_outputs > 0 && outputs_dev == nullptr) || (n_masks > 0 && (mask_query_ids_dev == nullptr ||
                                                                    masks_dev == nullptr)))
    return fail(P2C_ERR_INVALID, "input or output pointer is null");
  const size_t need = carve(nullptr, n, n_rows, n_outputs).total;
  if (workspace_dev == nullptr || workspace_bytes < need)
    return fail(P2C_ERR_INVALID, "scheduling workspace too small: %zu < %zu bytes", workspace_bytes, need);
  SchedLayout L = carve(workspace_dev, n, n_rows, n_outputs);
  cudaStream_t s = as_stream(stream);
  SchedParams P{mode, *config, n, n_rows, n_outputs, n_masks};
  P2C_CUDA(cudaMemsetAsync(L.acc, 0, 16 * 8, s));
  init_acc_kernel<<<1, 32, 0, s>>>(L);
  size_t tb;
  if (mode == 0) {
    if (n_rows > 0) {  // candidate id -> row, in id order; zero or repeated ids are errors
      row_ids_kernel<<<grid_for(n_rows), kThreads, 0, s>>>(rows_dev, n_rows, L);
      tb = L.tmp_bytes;
      P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.ids, L.row_ids, L.idx, L.row_idx, (int)n_rows, 0, 64, s));
      id_check_kernel<<<grid_for(n_rows), kThreads, 0, s>>>(L.row_ids, n_rows, kErrRowId, true, L);
    }
    if (n_outputs > 0) {
      output_ids_kernel<<<grid_for(n_outputs), kThreads, 0, s>>>(outputs_dev, n_outputs, L);
      tb = L.tmp_bytes;
      P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.ids, L.out_ids, L.idx, L.out_idx, (int)n_outputs, 0, 64,
                                               s));
      id_check_kernel<<<grid_for(n_outputs), kThreads, 0, s>>>(L.out_ids, n_outputs, kErrOutputId, true, L);
    }
    if (n > 0) {
      candidate_ids_kernel<<<grid_for(n), kThreads, 0, s>>>(candidates_dev, n, L);
      tb = L.tmp_bytes;
      P2C_CUDA(cub::DeviceRadixSort::SortKeys(L.tmp, tb, L.ids, L.cand_ids, (int)n, 0, 64, s));
      id_check_kernel<<<grid_for(n), kThreads, 0, s>>>(L.cand_ids, n, kErrDuplicateCandidate, false, L);
    }
  }
  const unsigned* order = L.order[0];
  if (n > 0) {
    decide_kernel<<<grid_for(n), kThreads, 0, s>>>(P, candidates_dev, rows_dev, outputs_dev,
                                                   reinterpret_cast<const unsigned long long*>(mask_query_ids_dev),
                                                   masks_dev, L);
    if (!config->preserve_candidate_order) {  // stable: equal priorities keep candidate order
      tb = L.tmp_bytes;
      P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.pkey[0], L.pkey[1], L.order[0], L.order[1], (int)n, 0,
                                               32, s));
      order = L.order[1];
    }
    write_kernel<<<grid_for(n), kThreads, 0, s>>>(P, order, candidates_dev, rows_dev, items_dev, L);
  }
  stats_kernel<<<1, 32, 0, s>>>(P, L, stats_dev, error_dev);
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

int p2c_dummy_schedule(int bypass, const p2c_candidate_record* candidates_dev, int64_t n, uint64_t primitive_count,
                       uint64_t raw_hit_count, uint64_t compact_candidate_count, const uint64_t* mask_query_ids_dev,
                       const uint32_t* masks_dev, int64_t n_masks, const p2c_scheduling_config* config,
                       p2c_proposal_feature_row* rows_dev, p2c_proposal_output* outputs_dev,
                       p2c_exact_work_item* items_dev, p2c_schedule_stats* stats_dev, uint64_t* error_dev,
                       void* workspace_dev, size_t workspace_bytes, void* stream) {
  using namespace p2c;
  if (config == nullptr) return fail(P2C_ERR_INVALID, "scheduling config pointer is null");
  if (!bypass) {
    if (int rc = check_config(*config)) return rc;
    if (primitive_count == 0) return fail(P2C_ERR_INVALID, "CandidateDensityStats.proxy_count must be non-zero");
  }
  if (n < 0 || n >= (1ll << 31) || n_masks < 0) return fail(P2C_ERR_INVALID, "counts must lie in [0, 2^31)");
  if (stats_dev == nullptr || error_dev == nullptr || (n > 0 && (items_dev == nullptr || candidates_dev == nullptr)) ||
      (n_masks > 0 && (mask_query_ids_dev == nullptr || masks_dev == nullptr)) ||
      ((rows_dev == nullptr) != (outputs_dev == nullptr)))
    return fail(P2C_ERR_INVALID, "input or output pointer is null");
  const size_t need = carve(nullptr, n, 0, 0).total;
  if (workspace_dev == nullptr || workspace_bytes < need)
    return fail(P2C_ERR_INVALID, "scheduling workspace too small: %zu < %zu bytes", workspace_bytes, need);
  SchedLayout L = carve(workspace_dev, n, 0, 0);
  cudaStream_t s = as_stream(stream);
  const double P_ = (double)primitive_count;
  const unsigned long long overlap_den = primitive_count >= 2 ? primitive_count / 2 : 1;  // :44-58
  SchedParams P{bypass ? 3 : 2, *config, n, 0, bypass ? 0 : n, n_masks,
                primitive_count == 0 ? 0.0 : (double)compact_candidate_count / P_,
                (double)raw_hit_count / (double)overlap_den,
                compact_candidate_count == 0 ? 0.0 : (double)raw_hit_count / (double)compact_candidate_count};
  P2C_CUDA(cudaMemsetAsync(L.acc, 0, 16 * 8, s));
  init_acc_kernel<<<1, 32, 0, s>>>(L);
  const auto* mq = reinterpret_cast<const unsigned long long*>(mask_query_ids_dev);
  if (n > 0) {
    if (!bypass && rows_dev != nullptr) {  // the artifacts: runtime feature rows, then the dummy outputs
      if (int rc = p2c_runtime_feature_rows(candidates_dev, n, primitive_count, raw_hit_count,
                                            compact_candidate_count, mask_query_ids_dev, masks_dev, n_masks,
                                            rows_dev, reinterpret_cast<uint64_t*>(L.acc + 13), stream))
        return rc;
      dummy_outputs_kernel<<<grid_for(n), kThreads, 0, s>>>(P, candidates_dev, rows_dev, mq, masks_dev, outputs_dev);
    }
    decide_kernel<<<grid_for(n), kThreads, 0, s>>>(P, candidates_dev, nullptr, nullptr, mq, masks_dev, L);
    const unsigned* order = L.order[0];
    if (!bypass && !config->preserve_candidate_order) {
      size_t tb = L.tmp_bytes;
      P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.pkey[0], L.pkey[1], L.order[0], L.order[1], (int)n, 0,
                                               32, s));
      order = L.order[1];
    }
    write_kernel<<<grid_for(n), kThreads, 0, s>>>(P, order, candidates_dev, nullptr, items_dev, L);
  }
  stats_kernel<<<1, 32, 0, s>>>(P, L, stats_dev, error_dev);
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

}  // extern "C"
