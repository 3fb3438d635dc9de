// ref_proxy.cpp — C ABI over the reference's proxy-scene build, candidate
// generation and proposal feature rows (rt_candidate/proxy_scene.cpp:
// BuildProxyScene, ValidateProxyScene; rt_candidate/candidate_buffer.cpp:
// GenerateRawCandidatesCpu, CompactRawCandidates; rt_candidate/
// candidate_stats.cpp: ComputeCandidateDensityStats; proposal/
// proposal_features.cpp: ExtractProposalFeatureRows), compiled unchanged into
// oracle/_ref/libp2c_ref.so.
//
// TEST INFRASTRUCTURE ONLY: tests pin the device proxy candidates and the
// restated checker to it; the product never loads it.
#include "proposal/proposal_features.h"
#include "proposal/proposal_policy.h"
#include "rt_candidate/candidate_buffer.h"
#include "rt_candidate/candidate_stats.h"
#include "common/group_scheduler.h"
#include "geometry/mesh_io.h"
#include "common/validators.h"
#include "rt_candidate/external_batch_candidate.h"
#include "rt_candidate/proxy_scene.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../include/p2c_b200.h"

static_assert(sizeof(p2cccd::RawCandidateHit) == sizeof(p2c_raw_candidate_hit));
static_assert(sizeof(p2cccd::CandidateRecord) == sizeof(p2c_candidate_record));
static_assert(offsetof(p2cccd::CandidateRecord, candidate_id) == offsetof(p2c_candidate_record, candidate_id));
static_assert(offsetof(p2cccd::CandidateRecord, proxy_type_a) == offsetof(p2c_candidate_record, proxy_type_a));
static_assert(offsetof(p2cccd::CandidateRecord, rt_hit_count) == offsetof(p2c_candidate_record, rt_hit_count));
static_assert(offsetof(p2cccd::CandidateRecord, flags) == offsetof(p2c_candidate_record, flags));
static_assert(offsetof(p2cccd::RawCandidateHit, motion_bound) == offsetof(p2c_raw_candidate_hit, motion_bound));
static_assert(sizeof(p2cccd::ProposalFeatureRow) == sizeof(p2c_proposal_feature_row));
static_assert(sizeof(p2cccd::ProposalOutput) == sizeof(p2c_proposal_output));
static_assert(offsetof(p2cccd::ProposalOutput, uncertainty_score) == offsetof(p2c_proposal_output, uncertainty_score));
static_assert(sizeof(p2cccd::ExactWorkItem) == sizeof(p2c_exact_work_item));
static_assert(offsetof(p2cccd::ExactWorkItem, source) == offsetof(p2c_exact_work_item, source));
static_assert(offsetof(p2cccd::ExactWorkItem, priority_score) == offsetof(p2c_exact_work_item, priority_score));
static_assert(offsetof(p2cccd::ProposalFeatureRow, features) == offsetof(p2c_proposal_feature_row, features));
static_assert(offsetof(p2cccd::ProposalFeatureRow, target_mask) == offsetof(p2c_proposal_feature_row, target_mask));

namespace {
thread_local std::string g_proxy_error;
}

static p2cccd::ProxyScene make_scene(uint64_t query_id, int64_t n, const uint32_t* object_id,
                                     const uint32_t* patch_id, const uint32_t* slab_id, const uint8_t* proxy_type,
                                     const double* t0, const double* t1, const double* bounds,
                                     const double* motion_bound) {

  p2cccd::ProxyScene scene;
  scene.query_id = query_id;
  scene.primitives.resize(static_cast<std::size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    p2cccd::ProxyPrimitive& p = scene.primitives[static_cast<std::size_t>(i)];
    p.proxy_id = static_cast<std::uint32_t>(i);
    p.object_id = object_id[i];
    p.patch_id = patch_id[i];
    p.slab_id = slab_id[i];
    p.proxy_type = static_cast<p2cccd::ProxyType>(proxy_type[i]);
    p.t0 = t0[i];
    p.t1 = t1[i];
    for (int a = 0; a < 3; ++a) {
      p.bounds.min[a] = bounds[6 * i + a];
      p.bounds.max[a] = bounds[6 * i + 3 + a];
    }
    p.motion_bound.translation_bound = motion_bound[4 * i + 0];
    p.motion_bound.rotation_angle = motion_bound[4 * i + 1];
    p.motion_bound.radial_motion_bound = motion_bound[4 * i + 2];
    p.motion_bound.conservative_radius = motion_bound[4 * i + 3];
  }
  return scene;
}

extern "C" {

const char* ref_proxy_last_error(void) { return g_proxy_error.c_str(); }

// Proxy arrays as p2c_proxy_scene lays them out (host memory).  Returns 0 and
// the counts, or 1 with the reference's error message.  Outputs (may be NULL
// for a sizing call) receive min(count, cap) records.
int ref_proxy_candidates(uint64_t query_id, int64_t n, const uint32_t* object_id, const uint32_t* patch_id,
                         const uint32_t* slab_id, const uint8_t* proxy_type, const double* t0, const double* t1,
                         const double* bounds, const double* motion_bound, p2c_raw_candidate_hit* raw_out,
                         int64_t raw_cap, p2c_candidate_record* cand_out, int64_t cand_cap, int64_t* n_raw,
                         int64_t* n_cand) {
  p2cccd::ProxyScene scene =
      make_scene(query_id, n, object_id, patch_id, slab_id, proxy_type, t0, t1, bounds, motion_bound);
  p2cccd::RawCandidateBuffer raw;
  p2cccd::Status st = p2cccd::GenerateRawCandidatesCpu(scene, query_id, &raw);
  if (!st.ok) {
    g_proxy_error = st.message;
    return 1;
  }
  std::vector<p2cccd::CandidateRecord> cands;
  st = p2cccd::CompactRawCandidates(scene, raw, &cands);
  if (!st.ok) {
    g_proxy_error = st.message;
    return 1;
  }
  *n_raw = static_cast<int64_t>(raw.hits.size());
  *n_cand = static_cast<int64_t>(cands.size());
  if (raw_out != nullptr)
    for (int64_t k = 0; k < *n_raw && k < raw_cap; ++k)
      std::memcpy(&raw_out[k], &raw.hits[static_cast<std::size_t>(k)], sizeof(p2c_raw_candidate_hit));
  if (cand_out != nullptr)
    for (int64_t k = 0; k < *n_cand && k < cand_cap; ++k) {
      std::memset(&cand_out[k], 0, sizeof(p2c_candidate_record));
      const p2cccd::CandidateRecord& c = cands[static_cast<std::size_t>(k)];
      p2c_candidate_record& o = cand_out[k];
      o.schema_version = c.schema_version;
      o.candidate_id = c.candidate_id;
      o.query_id = c.query_id;
      o.slab_id = c.slab_id;
      o.object_a_id = c.object_a_id;
      o.patch_a_id = c.patch_a_id;
      o.object_b_id = c.object_b_id;
      o.patch_b_id = c.patch_b_id;
      o.proxy_type_a = static_cast<uint8_t>(c.proxy_type_a);
      o.proxy_type_b = static_cast<uint8_t>(c.proxy_type_b);
      o.rt_hit_count = c.rt_hit_count;
      for (int a = 0; a < 4; ++a) o.motion_bound[a] = c.motion_bound[a];
      o.proxy_features_offset = c.proxy_features_offset;
      o.flags = c.flags;
    }
  return 0;
}

// BuildProxyScene over a flattened ProxySceneBuildInput: per object its id,
// type, slabs per segment, eps, and the ranges [patch_offset, +n_patches) of
// the patch arrays and [segment_offset, +n_segments) of the segment array
// (p2c_motion_segment layout).  Outputs n x {object, patch, slab, segment
// ids, type, t0, t1, bounds[6], motion_bound[4] (translation, rotation,
// radial, conservative), detail[8] (centre t0, centre t1, centre and surface
// rotation bounds), capsule radius}; NULL outputs make it a sizing call.
int ref_build_proxy_scene(uint64_t query_id, int64_t n_objects, const uint32_t* object_id,
                          const uint32_t* proxy_type, const uint32_t* slabs_per_segment, const double* eps,
                          const int64_t* patch_offset, const int64_t* n_patches, const int64_t* segment_offset,
                          const int64_t* n_segments, const uint32_t* patch_id, const double* patch_center,
                          const double* patch_radius, const p2c_motion_segment* segments, int64_t cap,
                          uint32_t* o_object, uint32_t* o_patch, uint32_t* o_slab, uint32_t* o_segment,
                          uint8_t* o_type, double* o_t0, double* o_t1, double* o_bounds, double* o_motion,
                          double* o_detail, double* o_capsule_radius, int64_t* n_out) {
  p2cccd::ProxySceneBuildInput in;
  in.query_id = query_id;
  for (int64_t k = 0; k < n_objects; ++k) {
    p2cccd::ProxyObjectBuildInput o;
    o.object_id = object_id[k];
    o.proxy_type = static_cast<p2cccd::ProxyType>(proxy_type[k]);
    o.slabs_per_motion_segment = slabs_per_segment[k];
    o.eps_proxy = eps[k];
    for (int64_t i = patch_offset[k]; i < patch_offset[k] + n_patches[k]; ++i) {
      p2cccd::Patch pt;
      pt.patch_id = patch_id[i];
      pt.local_center = {patch_center[3 * i], patch_center[3 * i + 1], patch_center[3 * i + 2]};
      pt.radius = patch_radius[i];
      o.patches.push_back(pt);
    }
    for (int64_t i = segment_offset[k]; i < segment_offset[k] + n_segments[k]; ++i) {
      const p2c_motion_segment& s = segments[i];
      p2cccd::MotionSegment m;
      m.t0 = s.t0;
      m.t1 = s.t1;
      for (int a = 0; a < 3; ++a) {
        m.pose_t0.translation[a] = s.translation_t0[a];
        m.pose_t1.translation[a] = s.translation_t1[a];
      }
      for (int a = 0; a < 4; ++a) {
        m.pose_t0.rotation_xyzw[a] = s.rotation_t0[a];
        m.pose_t1.rotation_xyzw[a] = s.rotation_t1[a];
      }
      o.motion_segments.push_back(m);
    }
    in.objects.push_back(std::move(o));
  }
  p2cccd::ProxyScene scene;
  const p2cccd::Status st = p2cccd::BuildProxyScene(in, &scene);
  if (!st.ok) {
    g_proxy_error = st.message;
    return 1;
  }
  *n_out = static_cast<int64_t>(scene.primitives.size());
  if (o_object == nullptr) return 0;
  const int64_t n = std::min<int64_t>(*n_out, cap);
  for (int64_t i = 0; i < n; ++i) {
    const p2cccd::ProxyPrimitive& p = scene.primitives[i];
    o_object[i] = p.object_id;
    o_patch[i] = p.patch_id;
    o_slab[i] = p.slab_id;
    o_segment[i] = p.motion_segment_id;
    o_type[i] = static_cast<uint8_t>(p.proxy_type);
    o_t0[i] = p.t0;
    o_t1[i] = p.t1;
    for (int a = 0; a < 3; ++a) {
      o_bounds[6 * i + a] = p.bounds.min[a];
      o_bounds[6 * i + 3 + a] = p.bounds.max[a];
      o_detail[8 * i + a] = p.motion_bound.center_t0[a];
      o_detail[8 * i + 3 + a] = p.motion_bound.center_t1[a];
    }
    o_motion[4 * i + 0] = p.motion_bound.translation_bound;
    o_motion[4 * i + 1] = p.motion_bound.rotation_angle;
    o_motion[4 * i + 2] = p.motion_bound.radial_motion_bound;
    o_motion[4 * i + 3] = p.motion_bound.conservative_radius;
    o_detail[8 * i + 6] = p.motion_bound.center_rotation_bound;
    o_detail[8 * i + 7] = p.motion_bound.surface_rotation_bound;
    o_capsule_radius[i] = p.capsule.radius;
  }
  return 0;
}

// The reference's density stats (ComputeCandidateDensityStats, zero timing)
// and ExtractProposalFeatureRows for the candidates GenerateRawCandidatesCpu
// + CompactRawCandidates give on the same proxy arrays.  rows may be NULL (a
// sizing call); *n_rows receives the candidate count.
int ref_proposal_feature_rows(uint64_t query_id, int64_t n, const uint32_t* object_id, const uint32_t* patch_id,
                              const uint32_t* slab_id, const uint8_t* proxy_type, const double* t0,
                              const double* t1, const double* bounds, const double* motion_bound,
                              p2c_candidate_density* density, p2c_proposal_feature_row* rows, int64_t rows_cap,
                              int64_t* n_rows) {
  p2cccd::ProxyScene scene =
      make_scene(query_id, n, object_id, patch_id, slab_id, proxy_type, t0, t1, bounds, motion_bound);
  p2cccd::CandidateGenerationResult gen;
  gen.backend_name = "cpu_reference";
  p2cccd::Status st = p2cccd::GenerateRawCandidatesCpu(scene, query_id, &gen.raw_buffer);
  if (st.ok) st = p2cccd::CompactRawCandidates(scene, gen.raw_buffer, &gen.candidates);
  if (st.ok)
    st = p2cccd::ComputeCandidateDensityStats(scene, gen.raw_buffer, gen.candidates, gen.timing, gen.backend_name,
                                              &gen.density);
  std::vector<p2cccd::ProposalFeatureRow> out;
  if (st.ok) st = p2cccd::ExtractProposalFeatureRows(scene, gen, &out);
  if (!st.ok) {
    g_proxy_error = st.message;
    return 1;
  }
  const p2cccd::CandidateDensityStats& d = gen.density;
  *density = p2c_candidate_density{d.query_id, d.proxy_count, d.object_count, d.slab_count,
                                   d.cross_object_same_slab_pair_count, d.raw_hit_count, d.compact_candidate_count,
                                   d.raw_hits_per_proxy, d.candidates_per_proxy, d.candidates_per_slab,
                                   d.aabb_overlap_ratio, d.avg_rt_hits_per_candidate};
  *n_rows = static_cast<int64_t>(out.size());
  if (rows != nullptr) {
    const int64_t m = std::min<int64_t>(*n_rows, rows_cap);
    for (int64_t i = 0; i < m; ++i) {
      std::memcpy(rows + i, &out[static_cast<std::size_t>(i)], sizeof(p2c_proposal_feature_row));
      rows[i].pad0 = rows[i].pad1 = 0;  // padding bytes of the reference struct are indeterminate
    }
  }
  return 0;
}

// BuildProposalFeatureRowsFromRuntimeCandidates with the density of
// MakeRuntimeDensityStats (the binding's, py_module.cpp:508-531) and a
// query id -> family mask map.
int ref_runtime_feature_rows(const p2c_candidate_record* cands, int64_t n, uint64_t primitive_count,
                             uint64_t raw_hit_count, uint64_t compact_candidate_count, const uint64_t* mask_query_ids,
                             const uint32_t* masks, int64_t n_masks, p2c_proposal_feature_row* rows) {
  std::vector<p2cccd::CandidateRecord> cand(static_cast<std::size_t>(n));
  for (int64_t i = 0; i < n; ++i) std::memcpy(&cand[static_cast<std::size_t>(i)], cands + i, sizeof(p2c_candidate_record));
  p2cccd::CandidateDensityStats density;
  density.query_id = cand.empty() ? 1U : cand.front().query_id;
  density.proxy_count = primitive_count;
  density.raw_hit_count = raw_hit_count;
  density.compact_candidate_count = compact_candidate_count;
  std::unordered_map<std::uint64_t, std::uint32_t> mask_map;
  for (int64_t i = 0; i < n_masks; ++i) mask_map[mask_query_ids[i]] = masks[i];
  std::vector<p2cccd::ProposalFeatureRow> out;
  const p2cccd::Status st = p2cccd::BuildProposalFeatureRowsFromRuntimeCandidates(cand, density, mask_map, &out);
  if (!st.ok) {
    g_proxy_error = st.message;
    return 1;
  }
  for (int64_t i = 0; i < n; ++i) {
    std::memcpy(rows + i, &out[static_cast<std::size_t>(i)], sizeof(p2c_proposal_feature_row));
    rows[i].pad0 = rows[i].pad1 = 0;
  }
  return 0;
}

// ScheduleRuntimeExactWorkItemsFromProposals on candidate / row / output
// records, a query id -> family mask map and the config fields.
int ref_schedule_runtime(const p2c_candidate_record* cands, int64_t n, const p2c_proposal_feature_row* rows,
                         int64_t n_rows, const p2c_proposal_output* outs, int64_t n_outs, const uint64_t* mask_qids,
                         const uint32_t* masks, int64_t n_masks, uint64_t first_work_item_id, uint32_t conservative,
                         double t0, double t1, float family_threshold, float uncertainty_threshold,
                         float ood_threshold, int preserve, p2c_exact_work_item* items_out, uint64_t* stats_out) {
  std::vector<p2cccd::CandidateRecord> cand(static_cast<std::size_t>(n));
  for (int64_t i = 0; i < n; ++i) std::memcpy(&cand[static_cast<std::size_t>(i)], cands + i, sizeof(p2c_candidate_record));
  std::vector<p2cccd::ProposalFeatureRow> rv(static_cast<std::size_t>(n_rows));
  for (int64_t i = 0; i < n_rows; ++i) std::memcpy(&rv[static_cast<std::size_t>(i)], rows + i, sizeof(p2c_proposal_feature_row));
  std::vector<p2cccd::ProposalOutput> ov(static_cast<std::size_t>(n_outs));
  for (int64_t i = 0; i < n_outs; ++i) std::memcpy(&ov[static_cast<std::size_t>(i)], outs + i, sizeof(p2c_proposal_output));
  std::unordered_map<std::uint64_t, std::uint32_t> mask_map;
  for (int64_t i = 0; i < n_masks; ++i) mask_map[mask_qids[i]] = masks[i];
  p2cccd::ProposalSchedulingConfig cfg;
  cfg.first_work_item_id = first_work_item_id;
  cfg.conservative_feature_family_mask = conservative;
  cfg.fallback_interval_t0 = t0;
  cfg.fallback_interval_t1 = t1;
  cfg.family_score_threshold = family_threshold;
  cfg.uncertainty_fallback_threshold = uncertainty_threshold;
  cfg.ood_abs_feature_threshold = ood_threshold;
  cfg.preserve_candidate_order = preserve != 0;
  std::vector<p2cccd::ExactWorkItem> queue;
  p2cccd::ProposalScheduleStats st;
  const p2cccd::Status status =
      p2cccd::ScheduleRuntimeExactWorkItemsFromProposals(cand, rv, ov, mask_map, cfg, &queue, &st);
  if (!status.ok) {
    g_proxy_error = status.message;
    return 1;
  }
  for (std::size_t i = 0; i < queue.size(); ++i) {
    std::memset(items_out + i, 0, sizeof(p2c_exact_work_item));
    const p2cccd::ExactWorkItem& w = queue[i];
    p2c_exact_work_item& o = items_out[i];
    o.work_item_id = w.work_item_id;
    o.parent_candidate_id = w.parent_candidate_id;
    o.query_id = w.query_id;
    o.slab_id = w.slab_id;
    o.patch_a_id = w.patch_a_id;
    o.patch_b_id = w.patch_b_id;
    o.interval_t0 = w.interval_t0;
    o.interval_t1 = w.interval_t1;
    o.feature_family_mask = w.feature_family_mask;
    o.topk_feature_ids_offset = w.topk_feature_ids_offset;
    o.depth = w.depth;
    o.priority_score = w.priority_score;
    o.source = static_cast<uint8_t>(w.source);
  }
  const uint64_t s[10] = {st.raw_candidate_count, st.proposal_output_count, st.work_item_count, st.fallback_count,
                          st.missing_proposal_fallback_count, st.invalid_proposal_fallback_count,
                          st.ood_fallback_count, st.high_uncertainty_fallback_count, st.reordered_count,
                          st.monotonic_safe ? 1u : 0u};
  std::memcpy(stats_out, s, sizeof(s));
  return 0;
}

namespace {

p2cccd::ProposalSchedulingConfig sched_config(uint64_t first_work_item_id, uint32_t conservative, double t0,
                                              double t1, float family_threshold, float uncertainty_threshold,
                                              float ood_threshold, int preserve) {
  p2cccd::ProposalSchedulingConfig cfg;
  cfg.first_work_item_id = first_work_item_id;
  cfg.conservative_feature_family_mask = conservative;
  cfg.fallback_interval_t0 = t0;
  cfg.fallback_interval_t1 = t1;
  cfg.family_score_threshold = family_threshold;
  cfg.uncertainty_fallback_threshold = uncertainty_threshold;
  cfg.ood_abs_feature_threshold = ood_threshold;
  cfg.preserve_candidate_order = preserve != 0;
  return cfg;
}

void write_schedule(const p2cccd::ProposalRuntimeScheduleResult& r, p2c_exact_work_item* items_out,
                    uint64_t* stats_out, p2c_proposal_feature_row* rows_out, p2c_proposal_output* outs_out,
                    int64_t* sizes_out) {
  for (std::size_t i = 0; i < r.work_queue.size(); ++i) {
    std::memset(items_out + i, 0, sizeof(p2c_exact_work_item));
    const p2cccd::ExactWorkItem& w = r.work_queue[i];
    p2c_exact_work_item& o = items_out[i];
    o.work_item_id = w.work_item_id;
    o.parent_candidate_id = w.parent_candidate_id;
    o.query_id = w.query_id;
    o.slab_id = w.slab_id;
    o.patch_a_id = w.patch_a_id;
    o.patch_b_id = w.patch_b_id;
    o.interval_t0 = w.interval_t0;
    o.interval_t1 = w.interval_t1;
    o.feature_family_mask = w.feature_family_mask;
    o.topk_feature_ids_offset = w.topk_feature_ids_offset;
    o.depth = w.depth;
    o.priority_score = w.priority_score;
    o.source = static_cast<uint8_t>(w.source);
  }
  for (std::size_t i = 0; i < r.feature_rows.size(); ++i)
    std::memcpy(rows_out + i, &r.feature_rows[i], sizeof(p2c_proposal_feature_row));
  for (std::size_t i = 0; i < r.proposal_outputs.size(); ++i)
    std::memcpy(outs_out + i, &r.proposal_outputs[i], sizeof(p2c_proposal_output));
  const p2cccd::ProposalScheduleStats& st = r.stats;
  const uint64_t s[10] = {st.raw_candidate_count, st.proposal_output_count, st.work_item_count, st.fallback_count,
                          st.missing_proposal_fallback_count, st.invalid_proposal_fallback_count,
                          st.ood_fallback_count, st.high_uncertainty_fallback_count, st.reordered_count,
                          st.monotonic_safe ? 1u : 0u};
  std::memcpy(stats_out, s, sizeof(s));
  sizes_out[0] = static_cast<int64_t>(r.work_queue.size());
  sizes_out[1] = static_cast<int64_t>(r.feature_rows.size());
  sizes_out[2] = static_cast<int64_t>(r.proposal_outputs.size());
}

// MakeRuntimeDensityStats (py_module.cpp:508-531)
p2cccd::CandidateDensityStats runtime_density(const std::vector<p2cccd::CandidateRecord>& c, uint64_t primitives,
                                              uint64_t raw, uint64_t compact) {
  p2cccd::CandidateDensityStats d;
  d.query_id = c.empty() ? 1U : c.front().query_id;
  d.proxy_count = primitives;
  d.raw_hit_count = raw;
  d.compact_candidate_count = compact;
  d.candidates_per_proxy = primitives == 0U ? 0.0 : static_cast<double>(compact) / static_cast<double>(primitives);
  const uint64_t den = primitives >= 2U ? primitives / 2U : 1U;
  d.aabb_overlap_ratio = static_cast<double>(raw) / static_cast<double>(den);
  d.avg_rt_hits_per_candidate = compact == 0U ? 0.0 : static_cast<double>(raw) / static_cast<double>(compact);
  return d;
}

}  // namespace

// RunDummyProposalScheduleFromRuntimeCandidates through its binding
// (py_module.cpp:1009-1033).  sizes_out: {items, rows, outputs}.
int ref_dummy_schedule(const p2c_candidate_record* cands, int64_t n, uint64_t primitives, uint64_t raw,
                       uint64_t compact, const uint64_t* mask_qids, const uint32_t* masks, int64_t n_masks,
                       uint64_t first_work_item_id, uint32_t conservative, double t0, double t1,
                       float family_threshold, float uncertainty_threshold, float ood_threshold, int preserve,
                       int materialize, p2c_exact_work_item* items_out, uint64_t* stats_out,
                       p2c_proposal_feature_row* rows_out, p2c_proposal_output* outs_out, int64_t* sizes_out) {
  std::vector<p2cccd::CandidateRecord> cand(static_cast<std::size_t>(n));
  for (int64_t i = 0; i < n; ++i) std::memcpy(&cand[static_cast<std::size_t>(i)], cands + i, sizeof(p2c_candidate_record));
  std::unordered_map<std::uint64_t, std::uint32_t> mask_map;
  for (int64_t i = 0; i < n_masks; ++i) mask_map[mask_qids[i]] = masks[i];
  const auto cfg = sched_config(first_work_item_id, conservative, t0, t1, family_threshold, uncertainty_threshold,
                                ood_threshold, preserve);
  p2cccd::ProposalRuntimeScheduleResult result;
  const p2cccd::Status status = p2cccd::RunDummyProposalScheduleFromRuntimeCandidates(
      cand, runtime_density(cand, primitives, raw, compact), mask_map, cfg, materialize != 0, &result);
  if (!status.ok) {
    g_proxy_error = status.message;
    return 1;
  }
  write_schedule(result, items_out, stats_out, rows_out, outs_out, sizes_out);
  return 0;
}

// GenerateExternalBatchDummyProposalScheduleOrThrow (py_module.cpp:269-361)
// restated over the reference's own functions: the batch's candidates, a
// conservative mask per runtime query id from its family (:213-246), the
// raw bypass when every candidate has its own query and a single-family
// mask (:248-267, :290-318), else the dummy schedule with the binding's
// density (:320-349).  Batch arguments as ref_external_batch; candidates
// (capacity n) are written too.  sizes_out: {items, rows, outputs, cands}.
int ref_external_dummy(int64_t n, const uint64_t* source_id, const uint32_t* source_index, const uint8_t* family,
                       const double* v_t0, const double* v_t1, const int8_t* ground_truth, const uint8_t* has_box,
                       const uint32_t* box_pair, uint64_t first_work_item_id, uint32_t conservative, double t0,
                       double t1, float family_threshold, float uncertainty_threshold, float ood_threshold,
                       int preserve, int materialize, p2c_candidate_record* cand_out, p2c_exact_work_item* items_out,
                       uint64_t* stats_out, p2c_proposal_feature_row* rows_out, p2c_proposal_output* outs_out,
                       int64_t* sizes_out) {
  std::vector<p2cccd::ExternalBatchQuery> queries(static_cast<std::size_t>(n));
  for (int64_t k = 0; k < n; ++k) {
    p2cccd::ExternalBatchQuery& q = queries[static_cast<std::size_t>(k)];
    q.source_query_id = source_id[k];
    q.source_query_index = source_index[k];
    q.family = family[k] ? p2cccd::ExternalQueryFamily::kEdgeEdge : p2cccd::ExternalQueryFamily::kVertexFace;
    for (int v = 0; v < 4; ++v)
      for (int a = 0; a < 3; ++a) {
        q.vertices_t0[v][a] = v_t0[12 * k + 3 * v + a];
        q.vertices_t1[v][a] = v_t1[12 * k + 3 * v + a];
      }
    q.has_ground_truth = ground_truth[k] >= 0;
    q.ground_truth_collides = ground_truth[k] > 0;
    q.has_box_pair = has_box[k] != 0;
    if (q.has_box_pair) q.box_pair = {box_pair[2 * k], box_pair[2 * k + 1]};
  }
  p2cccd::CandidateGeneratorConfig gen_cfg;
  p2cccd::ExternalBatchCandidateResult cr;
  p2cccd::Status status = p2cccd::GenerateCandidatesForExternalBatch(queries, gen_cfg, &cr);
  if (!status.ok) {
    g_proxy_error = status.message;
    return 1;
  }
  std::unordered_map<std::uint64_t, std::uint32_t> source_masks, runtime_masks;
  for (const auto& q : queries)
    source_masks.emplace(q.source_query_id, q.family == p2cccd::ExternalQueryFamily::kVertexFace ? 1u : 2u);
  for (const auto& m : cr.runtime_query_ids) {
    const auto it = source_masks.find(m.source_query_id);
    runtime_masks.emplace(m.runtime_query_id, it != source_masks.end() ? it->second : 3u);
  }
  bool bypass = true;
  {
    std::unordered_map<std::uint64_t, std::uint8_t> seen;
    for (const auto& c : cr.candidates) {
      if (!seen.emplace(c.query_id, 1U).second) {
        bypass = false;
        break;
      }
      const auto it = runtime_masks.find(c.query_id);
      const uint32_t m = it != runtime_masks.end() ? it->second : 3u;
      if (m == 0u || (m & (m - 1u)) != 0u) {
        bypass = false;
        break;
      }
    }
  }
  const auto cfg = sched_config(first_work_item_id, conservative, t0, t1, family_threshold, uncertainty_threshold,
                                ood_threshold, preserve);
  p2cccd::ProposalRuntimeScheduleResult result;
  if (bypass) {
    result.stats.raw_candidate_count = cr.candidates.size();
    result.stats.work_item_count = cr.candidates.size();
    result.stats.monotonic_safe = true;
    for (std::size_t i = 0; i < cr.candidates.size(); ++i) {
      const p2cccd::CandidateRecord& c = cr.candidates[i];
      p2cccd::ExactWorkItem item;
      item.work_item_id = cfg.first_work_item_id + i;
      item.parent_candidate_id = c.candidate_id;
      item.query_id = c.query_id;
      item.slab_id = c.slab_id;
      item.patch_a_id = c.patch_a_id;
      item.patch_b_id = c.patch_b_id;
      item.interval_t0 = cfg.fallback_interval_t0;
      item.interval_t1 = cfg.fallback_interval_t1;
      item.feature_family_mask = runtime_masks.at(c.query_id);
      item.topk_feature_ids_offset = 0U;
      item.depth = 0U;
      item.priority_score = static_cast<float>(c.rt_hit_count);
      item.source = p2cccd::ProposalSource::kRaw;
      status = p2cccd::ValidateExactWorkItem(item);
      if (!status.ok) break;
      result.work_queue.push_back(item);
    }
  } else {
    std::vector<p2cccd::CandidateRecord> cand = cr.candidates;
    p2cccd::CandidateDensityStats d = runtime_density(cand, cr.primitive_count, cr.raw_hit_count,
                                                      cr.compact_candidate_count);
    status = p2cccd::RunDummyProposalScheduleFromRuntimeCandidates(cand, d, runtime_masks, cfg, materialize != 0,
                                                                   &result);
  }
  if (!status.ok) {
    g_proxy_error = status.message;
    return 1;
  }
  for (std::size_t i = 0; i < cr.candidates.size(); ++i)
    std::memcpy(cand_out + i, &cr.candidates[i], sizeof(p2c_candidate_record));
  write_schedule(result, items_out, stats_out, rows_out, outs_out, sizes_out);
  sizes_out[3] = static_cast<int64_t>(cr.candidates.size());
  return 0;
}

// LoadTriangleMesh on a file: counts {vertices, triangles, patch ids} and,
// when the outputs are given, the arrays (vertices n x 3 doubles, triangles
// n x 3 u32, patch ids u32).  With center != NULL also CenterMeshAtAabbCenter
// of the loaded mesh (vertices then centered, center written).
int ref_load_mesh(const char* path, int64_t* counts, double* vertices, uint32_t* triangles, uint32_t* patch_ids,
                  double* center) {
  p2cccd::Mesh mesh;
  p2cccd::Status st = p2cccd::LoadTriangleMesh(path, &mesh);
  if (!st.ok) {
    g_proxy_error = st.message;
    return 1;
  }
  if (center != nullptr) {
    p2cccd::Mesh centered;
    std::array<double, 3> c{};
    st = p2cccd::CenterMeshAtAabbCenter(mesh, &centered, &c);
    if (!st.ok) {
      g_proxy_error = st.message;
      return 1;
    }
    mesh = centered;
    for (int a = 0; a < 3; ++a) center[a] = c[static_cast<std::size_t>(a)];
  }
  counts[0] = static_cast<int64_t>(mesh.vertices_ref.size());
  counts[1] = static_cast<int64_t>(mesh.triangles.size());
  counts[2] = static_cast<int64_t>(mesh.patch_ids.size());
  if (vertices != nullptr)
    for (std::size_t i = 0; i < mesh.vertices_ref.size(); ++i)
      for (int a = 0; a < 3; ++a) vertices[3 * i + static_cast<std::size_t>(a)] = mesh.vertices_ref[i][static_cast<std::size_t>(a)];
  if (triangles != nullptr)
    for (std::size_t i = 0; i < mesh.triangles.size(); ++i)
      for (int a = 0; a < 3; ++a) triangles[3 * i + static_cast<std::size_t>(a)] = mesh.triangles[i][static_cast<std::size_t>(a)];
  if (patch_ids != nullptr)
    for (std::size_t i = 0; i < mesh.patch_ids.size(); ++i) patch_ids[i] = mesh.patch_ids[i];
  return 0;
}

// CompactRawCandidates on n_raw given hits (64-byte records) of the scene.
// Writes the candidates (capacity n_raw) and their count.
int ref_compact_raw(uint64_t query_id, int64_t n, const uint32_t* object_id, const uint32_t* patch_id,
                    const uint32_t* slab_id, const uint8_t* proxy_type, const double* t0, const double* t1,
                    const double* bounds, const double* motion_bound, const p2c_raw_candidate_hit* raw_in,
                    int64_t n_raw, p2c_candidate_record* cand_out, int64_t* n_cand) {
  p2cccd::ProxyScene scene =
      make_scene(query_id, n, object_id, patch_id, slab_id, proxy_type, t0, t1, bounds, motion_bound);
  p2cccd::RawCandidateBuffer raw;
  raw.hits.resize(static_cast<std::size_t>(n_raw));
  for (int64_t k = 0; k < n_raw; ++k)
    std::memcpy(&raw.hits[static_cast<std::size_t>(k)], raw_in + k, sizeof(p2c_raw_candidate_hit));
  std::vector<p2cccd::CandidateRecord> cands;
  const p2cccd::Status st = p2cccd::CompactRawCandidates(scene, raw, &cands);
  if (!st.ok) {
    g_proxy_error = st.message;
    return 1;
  }
  *n_cand = static_cast<int64_t>(cands.size());
  for (std::size_t k = 0; k < cands.size(); ++k) {
    std::memset(&cand_out[k], 0, sizeof(p2c_candidate_record));
    const p2cccd::CandidateRecord& c = cands[k];
    p2c_candidate_record& o = cand_out[k];
    o.schema_version = c.schema_version;
    o.candidate_id = c.candidate_id;
    o.query_id = c.query_id;
    o.slab_id = c.slab_id;
    o.object_a_id = c.object_a_id;
    o.patch_a_id = c.patch_a_id;
    o.object_b_id = c.object_b_id;
    o.patch_b_id = c.patch_b_id;
    o.proxy_type_a = static_cast<uint8_t>(c.proxy_type_a);
    o.proxy_type_b = static_cast<uint8_t>(c.proxy_type_b);
    o.rt_hit_count = c.rt_hit_count;
    for (int m = 0; m < 4; ++m) o.motion_bound[m] = c.motion_bound[static_cast<std::size_t>(m)];
    o.proxy_features_offset = c.proxy_features_offset;
    o.flags = c.flags;
  }
  return 0;
}

// GenerateCandidatesForExternalBatch (CPU reference backend) on n external
// queries: family 0 vertex-face / 1 edge-edge, 4 vertices at t0 and t1
// (n x 12 doubles each), ground truth -1 none / 0 / 1, box pairs (has_box
// 0/1, n x 2 ids).  Outputs: candidates (capacity n), the runtime query id
// of every query, counts {primitives, raw hits, candidates} and the recall.
int ref_external_batch(int64_t n, const uint64_t* source_id, const uint32_t* source_index, const uint8_t* family,
                       const double* v_t0, const double* v_t1, const int8_t* ground_truth, const uint8_t* has_box,
                       const uint32_t* box_pair, p2c_candidate_record* cand_out, uint64_t* runtime_ids,
                       uint64_t* counts, double* recall) {
  std::vector<p2cccd::ExternalBatchQuery> queries(static_cast<std::size_t>(n));
  for (int64_t k = 0; k < n; ++k) {
    p2cccd::ExternalBatchQuery& q = queries[static_cast<std::size_t>(k)];
    q.source_query_id = source_id[k];
    q.source_query_index = source_index[k];
    q.family = family[k] ? p2cccd::ExternalQueryFamily::kEdgeEdge : p2cccd::ExternalQueryFamily::kVertexFace;
    for (int v = 0; v < 4; ++v)
      for (int a = 0; a < 3; ++a) {
        q.vertices_t0[v][a] = v_t0[12 * k + 3 * v + a];
        q.vertices_t1[v][a] = v_t1[12 * k + 3 * v + a];
      }
    q.has_ground_truth = ground_truth[k] >= 0;
    q.ground_truth_collides = ground_truth[k] > 0;
    q.has_box_pair = has_box[k] != 0;
    if (q.has_box_pair) q.box_pair = {box_pair[2 * k], box_pair[2 * k + 1]};
  }
  p2cccd::CandidateGeneratorConfig cfg;
  p2cccd::ExternalBatchCandidateResult res;
  const p2cccd::Status st = p2cccd::GenerateCandidatesForExternalBatch(queries, cfg, &res);
  if (!st.ok) {
    g_proxy_error = st.message;
    return 1;
  }
  for (std::size_t i = 0; i < res.candidates.size(); ++i)
    std::memcpy(cand_out + i, &res.candidates[i], sizeof(p2c_candidate_record));
  for (std::size_t i = 0; i < res.runtime_query_ids.size(); ++i) runtime_ids[i] = res.runtime_query_ids[i].runtime_query_id;
  counts[0] = res.primitive_count;
  counts[1] = res.raw_hit_count;
  counts[2] = res.compact_candidate_count;
  *recall = res.candidate_recall;
  return 0;
}

// RunDenseGroupExactEarlyStop on n rows, parsed as the binding parses its
// arrays (py_module.cpp:1212-1244): arg-max interval bin with strict >,
// full cost trace[5], narrow cost max(1e-12, full * cost_target) for a
// finite positive cost_target, contact trace[6:8], label trace[0] > 0.5.
// Writes 18 totals in p2c_dense_group_stats order (doubles as their bits).
int ref_dense_group(int64_t n, const uint64_t* query_id, const uint64_t* candidate_id, const float* cost_target,
                    const double* trace, const float* interval_scores, const float* priority, const float* cost_score,
                    const float* uncertainty, float threshold, uint32_t limit, double penalty, int preserve,
                    p2c_dense_group_stats* out) {
  std::vector<p2cccd::DenseGroupCandidateInput> rows(static_cast<std::size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    const float* sc = interval_scores + 8 * i;
    int best = 0;
    float best_score = sc[0];
    for (int k = 1; k < 8; ++k)
      if (sc[k] > best_score) {
        best_score = sc[k];
        best = k;
      }
    const double width = 1.0 / 8.0;
    const double full = trace[8 * i + 5];
    const double ratio = cost_target[i];
    p2cccd::DenseGroupCandidateInput& r = rows[static_cast<std::size_t>(i)];
    r.query_id = query_id[i];
    r.candidate_id = candidate_id[i];
    r.full_exact_cost = full;
    r.narrow_exact_cost = std::isfinite(ratio) && ratio > 0.0 ? std::max(1.0e-12, full * ratio) : full;
    r.interval_t0 = width * static_cast<double>(best);
    r.interval_t1 = std::min(1.0, r.interval_t0 + width);
    r.contact_t0 = trace[8 * i + 6];
    r.contact_t1 = trace[8 * i + 7];
    r.priority_score = priority[i];
    r.cost_score = cost_score[i];
    r.uncertainty_score = uncertainty[i];
    r.candidate_collides = trace[8 * i] > 0.5;
  }
  p2cccd::DenseGroupEarlyStopConfig cfg;
  cfg.uncertainty_fallback_threshold = threshold;
  cfg.representative_attempt_limit = limit;
  cfg.interval_miss_penalty_scale = penalty;
  cfg.preserve_input_order = preserve != 0;
  p2cccd::DenseGroupEarlyStopStats st;
  const p2cccd::Status status = p2cccd::RunDenseGroupExactEarlyStop(rows, cfg, &st);
  if (!status.ok) {
    g_proxy_error = status.message;
    return 1;
  }
  std::memset(out, 0, sizeof(*out));
  out->candidate_count = st.candidate_count;
  out->group_count = st.group_count;
  out->positive_group_count = st.positive_group_count;
  out->no_proposal_exact_calls = st.no_proposal_exact_calls;
  out->no_proposal_exact_work = st.no_proposal_exact_work;
  out->learned_exact_calls = st.learned_exact_calls;
  out->learned_fallback_calls = st.learned_fallback_calls;
  out->learned_interval_hit_count = st.learned_interval_hit_count;
  out->learned_interval_miss_count = st.learned_interval_miss_count;
  out->learned_exact_work = st.learned_exact_work;
  out->first_positive_rank_sum = st.first_positive_rank_sum;
  out->cost_before_first_positive_sum = st.cost_before_first_positive_sum;
  out->tp = st.tp;
  out->tn = st.tn;
  out->fp = st.fp;
  out->fn = st.fn;
  out->reordered_count = st.reordered_count;
  out->high_uncertainty_group_count = st.high_uncertainty_group_count;
  out->error_row = -1;
  return 0;
}

}  // extern "C"
