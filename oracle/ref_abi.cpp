// ref_abi.cpp — C ABI over the reference certifier compiled unchanged.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's own sources (read in place from the reference checkout;
// nothing is copied) into oracle/_ref/libp2c_ref.so.  Tests use it to pin the C
// restatement (ccd_oracle.c) and bench.py's CPU-baseline leg times it.  The
// product path never loads it.
#include "certificate/certificate_engine.h"
#include "certificate/mesh_exact_query.h"
#include "geometry/mesh.h"

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../include/p2c_b200.h"

namespace {

using p2cccd::CertificateEngineConfig;
using p2cccd::EdgeEdgeIntervalPrimitive;
using p2cccd::PointTriangleIntervalPrimitive;
using p2cccd::PrimitiveIntervalResult;

// The ABI records are the reference's host structs byte for byte.
static_assert(sizeof(p2cccd::AuditLogRow) == sizeof(p2c_audit_row), "AuditLogRow layout");
static_assert(sizeof(PointTriangleIntervalPrimitive) == sizeof(p2c_point_triangle));
static_assert(sizeof(EdgeEdgeIntervalPrimitive) == sizeof(p2c_edge_edge));
static_assert(sizeof(PrimitiveIntervalResult) == sizeof(p2c_interval_result));
static_assert(offsetof(PrimitiveIntervalResult, covered_feature_mask) ==
              offsetof(p2c_interval_result, covered_feature_mask));
static_assert(offsetof(PrimitiveIntervalResult, toi_upper) == offsetof(p2c_interval_result, toi_upper));
static_assert(offsetof(PrimitiveIntervalResult, witness_id_b) ==
              offsetof(p2c_interval_result, witness_id_b));
static_assert(offsetof(PrimitiveIntervalResult, reason_code) == offsetof(p2c_interval_result, reason_code));
static_assert(offsetof(PrimitiveIntervalResult, next_refinement_mode) ==
              offsetof(p2c_interval_result, next_refinement_mode));

thread_local std::string g_error;

CertificateEngineConfig MakeConfig(double eps_time, double eps_space, int max_depth) {
  CertificateEngineConfig c;
  c.eps_time = eps_time;
  c.eps_space = eps_space;
  c.max_subdivision_depth = static_cast<std::uint16_t>(max_depth);
  return c;
}

template <typename Prim, typename Fn>
std::int64_t EvalRange(const Prim* prims, std::int64_t begin, std::int64_t end, double t0, double t1,
                       const CertificateEngineConfig& cfg, p2c_interval_result* out,
                       std::uint8_t* status_out, Fn fn) {
  std::int64_t bad = 0;
  for (std::int64_t i = begin; i < end; ++i) {
    Prim p;
    std::memcpy(static_cast<void*>(&p), &prims[i], sizeof(Prim));
    PrimitiveIntervalResult r;
    const p2cccd::Status s = fn(p, t0, t1, cfg, &r);
    if (!s.ok) {
      ++bad;
      std::memset(&out[i], 0, sizeof(out[i]));
      if (status_out) status_out[i] = 1;
      continue;
    }
    std::memset(&out[i], 0, sizeof(out[i]));
    std::memcpy(&out[i], &r, sizeof(r));
    // padding bytes of the reference struct are indeterminate: clear them
    std::memset(out[i].pad0, 0, sizeof(out[i].pad0));
    std::memset(out[i].pad1, 0, sizeof(out[i].pad1));
    std::memset(out[i].pad2, 0, sizeof(out[i].pad2));
    if (status_out) status_out[i] = 0;
  }
  return bad;
}

template <typename Prim, typename Fn>
std::int64_t EvalThreaded(const Prim* prims, std::int64_t n, double t0, double t1,
                          const CertificateEngineConfig& cfg, p2c_interval_result* out,
                          std::uint8_t* status_out, int threads, Fn fn) {
  if (threads <= 1 || n < 2) return EvalRange(prims, 0, n, t0, t1, cfg, out, status_out, fn);
  // Dynamic chunks so that a few deep queries do not stall one thread.
  std::atomic<std::int64_t> next{0};
  std::atomic<std::int64_t> bad{0};
  constexpr std::int64_t kChunk = 256;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&]() {
      for (;;) {
        const std::int64_t b = next.fetch_add(kChunk);
        if (b >= n) break;
        const std::int64_t e = std::min(n, b + kChunk);
        bad += EvalRange(prims, b, e, t0, t1, cfg, out, status_out, fn);
      }
    });
  }
  for (auto& th : pool) th.join();
  return bad.load();
}

auto kPt = [](const PointTriangleIntervalPrimitive& p, double t0, double t1,
              const CertificateEngineConfig& c, PrimitiveIntervalResult* r) {
  return p2cccd::EvaluatePointTriangleInterval(p, t0, t1, c, r);
};
auto kEe = [](const EdgeEdgeIntervalPrimitive& p, double t0, double t1,
              const CertificateEngineConfig& c, PrimitiveIntervalResult* r) {
  return p2cccd::EvaluateEdgeEdgeInterval(p, t0, t1, c, r);
};

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_error.c_str(); }

// EvaluatePointTriangleInterval over a batch; threads > 1 splits the batch
// across std::threads calling the unchanged function.
std::int64_t ref_eval_pt_batch(const p2c_point_triangle* prims, std::int64_t n, double t0, double t1,
                               double eps_time, double eps_space, int max_depth,
                               p2c_interval_result* out, std::uint8_t* status_out, int threads) {
  const auto cfg = MakeConfig(eps_time, eps_space, max_depth);
  return EvalThreaded(reinterpret_cast<const PointTriangleIntervalPrimitive*>(prims), n, t0, t1, cfg,
                      out, status_out, threads, kPt);
}

std::int64_t ref_eval_ee_batch(const p2c_edge_edge* prims, std::int64_t n, double t0, double t1,
                               double eps_time, double eps_space, int max_depth,
                               p2c_interval_result* out, std::uint8_t* status_out, int threads) {
  const auto cfg = MakeConfig(eps_time, eps_space, max_depth);
  return EvalThreaded(reinterpret_cast<const EdgeEdgeIntervalPrimitive*>(prims), n, t0, t1, cfg, out,
                      status_out, threads, kEe);
}

// First error message of a single evaluation (for error-behaviour parity).
int ref_eval_pt_one(const p2c_point_triangle* prim, double t0, double t1, double eps_time,
                    double eps_space, int max_depth, p2c_interval_result* out) {
  PointTriangleIntervalPrimitive p;
  std::memcpy(static_cast<void*>(&p), prim, sizeof(p));
  PrimitiveIntervalResult r;
  const auto s = p2cccd::EvaluatePointTriangleInterval(p, t0, t1, MakeConfig(eps_time, eps_space, max_depth), &r);
  if (!s.ok) {
    g_error = s.message;
    return 1;
  }
  std::memset(out, 0, sizeof(*out));
  std::memcpy(out, &r, sizeof(r));
  return 0;
}

int ref_eval_ee_one(const p2c_edge_edge* prim, double t0, double t1, double eps_time,
                    double eps_space, int max_depth, p2c_interval_result* out) {
  EdgeEdgeIntervalPrimitive p;
  std::memcpy(static_cast<void*>(&p), prim, sizeof(p));
  PrimitiveIntervalResult r;
  const auto s = p2cccd::EvaluateEdgeEdgeInterval(p, t0, t1, MakeConfig(eps_time, eps_space, max_depth), &r);
  if (!s.ok) {
    g_error = s.message;
    return 1;
  }
  std::memset(out, 0, sizeof(*out));
  std::memcpy(out, &r, sizeof(r));
  return 0;
}

// CertificateEngine::Evaluate on one work item with the given primitive lists.
int ref_evaluate_query(std::uint32_t family_mask, double t0, double t1, double eps_time,
                       double eps_space, int max_depth, const p2c_point_triangle* pts,
                       std::int64_t n_pt, const p2c_edge_edge* ees, std::int64_t n_ee,
                       p2c_query_certificate* out) {
  p2cccd::ExactCertificateQuery q;
  q.work_item.work_item_id = 1;
  q.work_item.parent_candidate_id = 1;
  q.work_item.query_id = 1;
  q.work_item.interval_t0 = t0;
  q.work_item.interval_t1 = t1;
  q.work_item.feature_family_mask = family_mask;
  q.work_item.priority_score = 1.0F;
  q.config = MakeConfig(eps_time, eps_space, max_depth);
  q.point_triangle_primitives.resize(static_cast<std::size_t>(n_pt));
  q.edge_edge_primitives.resize(static_cast<std::size_t>(n_ee));
  if (n_pt) std::memcpy(static_cast<void*>(q.point_triangle_primitives.data()), pts, sizeof(p2c_point_triangle) * n_pt);
  if (n_ee) std::memcpy(static_cast<void*>(q.edge_edge_primitives.data()), ees, sizeof(p2c_edge_edge) * n_ee);
  p2cccd::CertificateEngine engine;
  p2cccd::CertificateResult r;
  const auto s = engine.Evaluate(q, &r);
  if (!s.ok) {
    g_error = s.message;
    return 1;
  }
  std::memset(out, 0, sizeof(*out));
  out->status = static_cast<std::uint8_t>(r.status);
  out->witness_family = r.witness_family;
  out->reason_code = r.reason_code;
  out->covered_feature_mask = r.covered_feature_mask;
  out->toi_upper = r.toi_upper;
  out->safe_margin_lb = r.safe_margin_lb;
  out->witness_id_a = r.witness_id_a;
  out->witness_id_b = r.witness_id_b;
  out->witness_index = -1;
  out->next_refinement_mode = static_cast<std::uint8_t>(r.next_refinement_mode);
  return 0;
}

// BuildMeshExactCertificateQuery.  Two-call protocol: with pt_out/ee_out NULL
// only the counts are returned in *n_pt/*n_ee.  Meshes are given as vertex
// arrays (nv x 3 doubles) and triangle arrays (nf x 3 uint32).
int ref_build_mesh_query(const double* va, std::int64_t nva, const std::uint32_t* fa, std::int64_t nfa,
                         const double* ta0, const double* ta1, const double* vb, std::int64_t nvb,
                         const std::uint32_t* fb, std::int64_t nfb, const double* tb0, const double* tb1,
                         std::uint32_t family_mask, int prune, std::uint64_t max_pt, std::uint64_t max_ee,
                         p2c_point_triangle* pt_out, std::int64_t* n_pt, p2c_edge_edge* ee_out,
                         std::int64_t* n_ee) {
  p2cccd::Mesh a, b;
  a.vertices_ref.resize(static_cast<std::size_t>(nva));
  b.vertices_ref.resize(static_cast<std::size_t>(nvb));
  a.triangles.resize(static_cast<std::size_t>(nfa));
  b.triangles.resize(static_cast<std::size_t>(nfb));
  for (std::int64_t i = 0; i < nva; ++i) a.vertices_ref[i] = {va[3 * i], va[3 * i + 1], va[3 * i + 2]};
  for (std::int64_t i = 0; i < nvb; ++i) b.vertices_ref[i] = {vb[3 * i], vb[3 * i + 1], vb[3 * i + 2]};
  for (std::int64_t i = 0; i < nfa; ++i) a.triangles[i] = {fa[3 * i], fa[3 * i + 1], fa[3 * i + 2]};
  for (std::int64_t i = 0; i < nfb; ++i) b.triangles[i] = {fb[3 * i], fb[3 * i + 1], fb[3 * i + 2]};
  p2cccd::ExactWorkItem item;
  item.work_item_id = 1;
  item.parent_candidate_id = 1;
  item.query_id = 1;
  item.feature_family_mask = family_mask;
  item.priority_score = 1.0F;
  p2cccd::MeshExactBuildConfig bc;
  bc.prune_by_swept_aabb = prune != 0;
  bc.max_point_triangle_primitives = max_pt;
  bc.max_edge_edge_primitives = max_ee;
  p2cccd::MeshExactBuildResult res;
  const auto s = p2cccd::BuildMeshExactCertificateQuery(
      a, {ta0[0], ta0[1], ta0[2]}, {ta1[0], ta1[1], ta1[2]}, b, {tb0[0], tb0[1], tb0[2]},
      {tb1[0], tb1[1], tb1[2]}, item, p2cccd::CertificateEngineConfig{}, bc, &res);
  if (!s.ok) {
    g_error = s.message;
    return 1;
  }
  *n_pt = static_cast<std::int64_t>(res.query.point_triangle_primitives.size());
  *n_ee = static_cast<std::int64_t>(res.query.edge_edge_primitives.size());
  if (pt_out && *n_pt)
    std::memcpy(pt_out, res.query.point_triangle_primitives.data(), sizeof(p2c_point_triangle) * (*n_pt));
  if (ee_out && *n_ee)
    std::memcpy(ee_out, res.query.edge_edge_primitives.data(), sizeof(p2c_edge_edge) * (*n_ee));
  return 0;
}

// GenerateConservativeRefinementWorkItems (interval fields only).
int ref_refinement_children(double t0, double t1, std::uint16_t depth, std::uint8_t status,
                            std::uint8_t mode, double toi, std::uint16_t max_child_depth,
                            double min_width, double* c0, double* c1) {
  p2cccd::ExactWorkItem parent;
  parent.work_item_id = 7;
  parent.parent_candidate_id = 7;
  parent.query_id = 7;
  parent.interval_t0 = t0;
  parent.interval_t1 = t1;
  parent.depth = depth;
  parent.feature_family_mask = 1;
  parent.priority_score = 1.0F;
  p2cccd::CertificateResult cert;
  cert.work_item_id = 7;
  cert.query_id = 7;
  cert.status = static_cast<p2cccd::CertificateStatus>(status);
  cert.interval_t0 = t0;
  cert.interval_t1 = t1;
  cert.toi_upper = toi;
  cert.next_refinement_mode = static_cast<p2cccd::CertificateRefinementMode>(mode);
  if (cert.status == p2cccd::CertificateStatus::kCollision) {
    cert.witness_id_a = 1;
    cert.witness_id_b = 1;
  }
  if (cert.status == p2cccd::CertificateStatus::kSeparation) cert.covered_feature_mask = 1;
  if (cert.status == p2cccd::CertificateStatus::kUndecided) cert.reason_code = 2;
  p2cccd::ExactRefinementConfig rc;
  rc.max_child_depth = max_child_depth;
  rc.min_interval_width = min_width;
  std::vector<p2cccd::ExactWorkItem> children;
  const auto s = p2cccd::GenerateConservativeRefinementWorkItems(parent, cert, rc, &children);
  if (!s.ok) {
    g_error = s.message;
    return -1;
  }
  for (std::size_t i = 0; i < children.size(); ++i) {
    c0[i] = children[i].interval_t0;
    c1[i] = children[i].interval_t1;
  }
  return static_cast<int>(children.size());
}

// ProcessExactWorkQueueCpu on n work items (the p2c_audit_item fields; slab
// and patch ids 0, source raw) with CSR primitive lists: certificates (the
// p2c_query_certificate fields) and the audit log (*n_rows rows).
int ref_process_queue(const p2c_audit_item* items, std::int64_t n, const p2c_point_triangle* pts,
                      const std::int64_t* pt_off, const p2c_edge_edge* ees, const std::int64_t* ee_off,
                      double eps_time, double eps_space, int max_depth, std::uint64_t first_event_id,
                      std::uint64_t first_timestamp_us, int emit_dequeue, p2c_query_certificate* certs_out,
                      p2c_audit_row* rows_out, std::int64_t* n_rows) {
  std::vector<p2cccd::ExactCertificateQuery> queue(static_cast<std::size_t>(n));
  for (std::int64_t k = 0; k < n; ++k) {
    p2cccd::ExactCertificateQuery& q = queue[static_cast<std::size_t>(k)];
    const p2c_audit_item& it = items[k];
    q.work_item.work_item_id = it.work_item_id;
    q.work_item.parent_candidate_id = it.candidate_id;
    q.work_item.query_id = it.query_id;
    q.work_item.interval_t0 = it.interval_t0;
    q.work_item.interval_t1 = it.interval_t1;
    q.work_item.feature_family_mask = it.feature_family_mask;
    q.work_item.depth = it.depth;
    q.work_item.priority_score = it.priority_score;
    q.config = MakeConfig(eps_time, eps_space, max_depth);
    const std::int64_t np = pt_off[k + 1] - pt_off[k], ne = ee_off[k + 1] - ee_off[k];
    q.point_triangle_primitives.resize(static_cast<std::size_t>(np));
    q.edge_edge_primitives.resize(static_cast<std::size_t>(ne));
    if (np) std::memcpy(static_cast<void*>(q.point_triangle_primitives.data()), pts + pt_off[k], sizeof(p2c_point_triangle) * np);
    if (ne) std::memcpy(static_cast<void*>(q.edge_edge_primitives.data()), ees + ee_off[k], sizeof(p2c_edge_edge) * ne);
  }
  p2cccd::ExactWorkQueueConfig cfg;
  cfg.first_event_id = first_event_id;
  cfg.first_timestamp_us = first_timestamp_us;
  cfg.emit_dequeue_events = emit_dequeue != 0;
  p2cccd::ExactWorkQueueResult res;
  const auto st = p2cccd::ProcessExactWorkQueueCpu(queue, cfg, &res);
  if (!st.ok) {
    g_error = st.message;
    return 1;
  }
  for (std::size_t k = 0; k < res.certificates.size(); ++k) {
    const p2cccd::CertificateResult& r = res.certificates[k];
    p2c_query_certificate& o = certs_out[k];
    std::memset(&o, 0, sizeof(o));
    o.status = static_cast<std::uint8_t>(r.status);
    o.witness_family = r.witness_family;
    o.reason_code = r.reason_code;
    o.covered_feature_mask = r.covered_feature_mask;
    o.toi_upper = r.toi_upper;
    o.safe_margin_lb = r.safe_margin_lb;
    o.witness_id_a = r.witness_id_a;
    o.witness_id_b = r.witness_id_b;
    o.witness_index = -1;
    o.next_refinement_mode = static_cast<std::uint8_t>(r.next_refinement_mode);
  }
  *n_rows = static_cast<std::int64_t>(res.audit_log.size());
  for (std::size_t k = 0; k < res.audit_log.size(); ++k) {
    const p2cccd::AuditLogRow& a = res.audit_log[k];
    p2c_audit_row& o = rows_out[k];
    std::memset(&o, 0, sizeof(o));
    o.event_id = a.event_id;
    o.query_id = a.query_id;
    o.candidate_id = a.candidate_id;
    o.work_item_id = a.work_item_id;
    o.stage = static_cast<std::uint8_t>(a.stage);
    o.action = a.action;
    o.depth = a.depth;
    o.interval_t0 = a.interval_t0;
    o.interval_t1 = a.interval_t1;
    o.timestamp_us = a.timestamp_us;
    o.aux_value0 = a.aux_value0;
    o.aux_value1 = a.aux_value1;
  }
  return 0;
}

}  // extern "C"
