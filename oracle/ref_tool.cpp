// ref_tool.cpp — C ABI over the reference's scene any-hit tool, compiled
// unchanged (tools/scene_object_envelope_native_ti_walltime.cpp).
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file, which
// includes the tool's source where it lies in the reference checkout, into
// oracle/_ref/libp2c_ref_tool.so.  The tool's exact kernel (Tight-Inclusion)
// is not vendored by the reference; shim/tight_inclusion/ccd.hpp declares its
// two queries and this file defines them over the reference certifier, so the
// tool's own scene preparation (PrepareScene :497-586), sweep-and-prune
// candidates (SweepPairs / BuildVFCandidates / BuildEECandidates :603-696),
// scoring (ScoreCandidate :1102-1132) and scheduled any-hit with fallback
// replay (RunScheduledAnyHitRows :1283-1410) run as written.  Tests use it to
// pin the C restatement and the device path; the product never loads it.
#include "certificate/certificate_engine.h"

#include <tight_inclusion/ccd.hpp>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <string>
#include <unistd.h>
#include <vector>

namespace {
p2cccd::CertificateEngineConfig g_tool_config;  // certifier settings behind the shim
}  // namespace

// The tool's entry point is renamed so this library can hold the tool's
// translation unit; nothing calls it.
#define main p2c_ref_tool_main
#include "tools/scene_object_envelope_native_ti_walltime.cpp"
#undef main

namespace {

void SetTrajectory(p2cccd::LinearVertexTrajectory* t, const ticcd::Vector3& a, const ticcd::Vector3& b) {
  t->feature_id = 0;
  for (int k = 0; k < 3; ++k) {
    t->position_t0[k] = a[k];
    t->position_t1[k] = b[k];
  }
}

std::string g_tool_error;
PreparedScene g_scene;
bool g_scene_ready = false;
std::vector<Candidate> g_candidates[2];
bool g_capped[2] = {false, false};

bool WritePly(const std::string& path, const double* v, std::int64_t nv, const std::int32_t* faces, std::int64_t nf) {
  std::ofstream out(path, std::ios::binary);
  if (!out) return false;
  out << "ply\nformat binary_little_endian 1.0\n"
      << "element vertex " << nv << "\nproperty double x\nproperty double y\nproperty double z\n"
      << "element face " << nf << "\nproperty list uchar int vertex_indices\nend_header\n";
  out.write(reinterpret_cast<const char*>(v), static_cast<std::streamsize>(nv * 3 * sizeof(double)));
  for (std::int64_t f = 0; f < nf; ++f) {
    const unsigned char three = 3;
    out.write(reinterpret_cast<const char*>(&three), 1);
    out.write(reinterpret_cast<const char*>(faces + 3 * f), 3 * sizeof(std::int32_t));
  }
  return static_cast<bool>(out);
}

}  // namespace

namespace ticcd {

bool vertexFaceCCD(const Vector3& vertex_start, const Vector3& face_vertex0_start,
                   const Vector3& face_vertex1_start, const Vector3& face_vertex2_start,
                   const Vector3& vertex_end, const Vector3& face_vertex0_end,
                   const Vector3& face_vertex1_end, const Vector3& face_vertex2_end, const Array3&, Scalar,
                   Scalar&, Scalar, Scalar t_max, long, Scalar&, bool, CCDRootFindingMethod) {
  p2cccd::PointTriangleIntervalPrimitive p;
  p.point_id = 0;
  p.triangle_id = 0;
  SetTrajectory(&p.point, vertex_start, vertex_end);
  SetTrajectory(&p.triangle_v0, face_vertex0_start, face_vertex0_end);
  SetTrajectory(&p.triangle_v1, face_vertex1_start, face_vertex1_end);
  SetTrajectory(&p.triangle_v2, face_vertex2_start, face_vertex2_end);
  p2cccd::PrimitiveIntervalResult r;
  const p2cccd::Status s = p2cccd::EvaluatePointTriangleInterval(p, 0.0, t_max, g_tool_config, &r);
  return !s.ok || r.status != p2cccd::CertificateStatus::kSeparation;
}

bool edgeEdgeCCD(const Vector3& edge0_vertex0_start, const Vector3& edge0_vertex1_start,
                 const Vector3& edge1_vertex0_start, const Vector3& edge1_vertex1_start,
                 const Vector3& edge0_vertex0_end, const Vector3& edge0_vertex1_end,
                 const Vector3& edge1_vertex0_end, const Vector3& edge1_vertex1_end, const Array3&, Scalar, Scalar&,
                 Scalar, Scalar t_max, long, Scalar&, bool, CCDRootFindingMethod) {
  p2cccd::EdgeEdgeIntervalPrimitive p;
  p.edge_a_id = 0;
  p.edge_b_id = 0;
  SetTrajectory(&p.edge_a0, edge0_vertex0_start, edge0_vertex0_end);
  SetTrajectory(&p.edge_a1, edge0_vertex1_start, edge0_vertex1_end);
  SetTrajectory(&p.edge_b0, edge1_vertex0_start, edge1_vertex0_end);
  SetTrajectory(&p.edge_b1, edge1_vertex1_start, edge1_vertex1_end);
  p2cccd::PrimitiveIntervalResult r;
  const p2cccd::Status s = p2cccd::EvaluateEdgeEdgeInterval(p, 0.0, t_max, g_tool_config, &r);
  return !s.ok || r.status != p2cccd::CertificateStatus::kSeparation;
}

}  // namespace ticcd

extern "C" {

const char* ref_tool_last_error(void) { return g_tool_error.c_str(); }

// PrepareScene over the two frames (written as binary PLY to a private
// temporary directory, the tool's input format).  Returns 0 or 1 on error.
int ref_tool_prepare(const double* v_t0, const double* v_t1, std::int64_t nv, const std::int32_t* faces,
                     std::int64_t nf, double thickness, int exclude_self) {
  char dir_template[] = "/tmp/p2c_ref_tool_XXXXXX";
  const char* dir = mkdtemp(dir_template);
  if (dir == nullptr) {
    g_tool_error = "mkdtemp failed";
    return 1;
  }
  const std::string f0 = std::string(dir) + "/frame0.ply", f1 = std::string(dir) + "/frame1.ply";
  int rc = 0;
  try {
    if (!WritePly(f0, v_t0, nv, faces, nf) || !WritePly(f1, v_t1, nv, faces, nf)) {
      throw std::runtime_error("failed to write PLY frames");
    }
    g_scene = PrepareScene(f0, f1, thickness, exclude_self != 0);
    g_scene_ready = true;
    g_candidates[0].clear();
    g_candidates[1].clear();
  } catch (const std::exception& e) {
    g_tool_error = e.what();
    g_scene_ready = false;
    rc = 1;
  }
  std::remove(f0.c_str());
  std::remove(f1.c_str());
  rmdir(dir);
  return rc;
}

// Object count; per-vertex and per-face object ids of the prepared scene.
int ref_tool_objects(std::int32_t* v_obj, std::int32_t* f_obj) {
  if (!g_scene_ready) return -1;
  for (std::size_t v = 0; v < g_scene.vertex_object.size(); ++v) v_obj[v] = g_scene.vertex_object[v];
  for (std::size_t f = 0; f < g_scene.mesh0.faces.size(); ++f) f_obj[f] = g_scene.mesh0.faces[f].object_id;
  return g_scene.object_count;
}

// The tool's unique-edge list: (a, b) with a < b and the edge's object id.
std::int64_t ref_tool_edges(std::int32_t* ab, std::int32_t* obj) {
  if (!g_scene_ready) return -1;
  if (ab != nullptr) {
    for (std::size_t e = 0; e < g_scene.edges.size(); ++e) {
      ab[2 * e] = g_scene.edges[e].a;
      ab[2 * e + 1] = g_scene.edges[e].b;
      obj[e] = g_scene.edges[e].object_id;
    }
  }
  return static_cast<std::int64_t>(g_scene.edges.size());
}

// BuildVFCandidates (kind 0: vertex, face) or BuildEECandidates (kind 1:
// edge, edge) in the tool's emission order; keeps the list for the any-hit
// rows.  Writes min(count, cap) pairs; returns the count.
std::int64_t ref_tool_candidates(int kind, std::uint64_t max_candidates, std::int32_t* a, std::int32_t* b,
                                 std::int64_t cap, int* capped) {
  if (!g_scene_ready || kind < 0 || kind > 1) return -1;
  bool c = false;
  g_candidates[kind] = kind == 0 ? BuildVFCandidates(g_scene, max_candidates, &c)
                                 : BuildEECandidates(g_scene, max_candidates, &c);
  g_capped[kind] = c;
  if (capped != nullptr) *capped = c ? 1 : 0;
  const std::int64_t n = static_cast<std::int64_t>(g_candidates[kind].size());
  for (std::int64_t i = 0; i < n && i < cap; ++i) {
    a[i] = g_candidates[kind][static_cast<std::size_t>(i)].a;
    b[i] = g_candidates[kind][static_cast<std::size_t>(i)].b;
  }
  return n;
}

// ScoreCandidate under the tool's "random" policy for the kept candidates.
int ref_tool_random_scores(int kind, double* out) {
  if (!g_scene_ready || kind < 0 || kind > 1) return 1;
  const std::string k = kind == 0 ? "vf" : "ee";
  const TinyStpfWeights weights;
  for (std::size_t i = 0; i < g_candidates[kind].size(); ++i) {
    out[i] = ScoreCandidate(g_scene, k, g_candidates[kind][i], i, "random", weights);
  }
  return 0;
}

// RunAllExactRows (the group truth) then RunScheduledAnyHitRows with the
// "random" score policy and proposal_top_k = top_k over the kept candidates.
// out[0..15] = {all-exact: exact_calls, hit_count, group_count,
// positive_groups; scheduled: exact_calls, proposal_exact_calls,
// fallback_exact_calls, hit_count, group_count, positive_groups,
// fallback_groups, tp, fp, fn, tn, positive_first_hit_rank_sum}.
int ref_tool_anyhit(int kind, std::uint64_t top_k, double eps_time, double eps_space, int max_depth,
                    std::uint64_t* out) {
  if (!g_scene_ready || kind < 0 || kind > 1) return 1;
  g_tool_config.eps_time = eps_time;
  g_tool_config.eps_space = eps_space;
  g_tool_config.max_subdivision_depth = static_cast<std::uint16_t>(max_depth);
  Args args;
  args.proposal_top_k = static_cast<std::size_t>(top_k);
  const std::string k = kind == 0 ? "vf" : "ee";
  std::unordered_map<std::uint64_t, GroupTruth> truth;
  try {
    const MethodRow all = RunAllExactRows(g_scene, args, k, g_candidates[kind], g_capped[kind], 0.0, &truth);
    const TinyStpfWeights weights;
    const MethodRow row = RunScheduledAnyHitRows(g_scene, args, k, g_candidates[kind], g_capped[kind], 0.0,
                                                 "ScheduledAnyHit", "random", weights, truth);
    const std::uint64_t v[16] = {all.exact_calls,        all.hit_count,          all.group_count,
                                 all.positive_groups,    row.exact_calls,        row.proposal_exact_calls,
                                 row.fallback_exact_calls, row.hit_count,        row.group_count,
                                 row.positive_groups,    row.fallback_groups,    row.tp,
                                 row.fp,                 row.fn,                 row.tn,
                                 row.positive_first_hit_rank_sum};
    for (int i = 0; i < 16; ++i) out[i] = v[i];
  } catch (const std::exception& e) {
    g_tool_error = e.what();
    return 1;
  }
  return 0;
}

// One timed step of the tool on the prepared scene, single-threaded as the
// tool runs: candidate generation of both families, then the scheduled
// any-hit of each family ("random" scores).  The group set handed to
// RunScheduledAnyHitRows is built from the candidates without certifying
// them (the every-candidate truth rows are not part of the step).
// seconds[0..2] = {candidates, any-hit vf, any-hit ee}; calls[0..1] = exact
// calls of the vf and ee rows; cands[0..1] = candidate counts.
int ref_tool_time_step(std::uint64_t top_k, double eps_time, double eps_space, int max_depth, double* seconds,
                       std::uint64_t* calls, std::uint64_t* cands) {
  if (!g_scene_ready) return 1;
  g_tool_config.eps_time = eps_time;
  g_tool_config.eps_space = eps_space;
  g_tool_config.max_subdivision_depth = static_cast<std::uint16_t>(max_depth);
  Args args;
  args.proposal_top_k = static_cast<std::size_t>(top_k);
  try {
    const auto t0 = std::chrono::steady_clock::now();
    bool c0 = false, c1 = false;
    g_candidates[0] = BuildVFCandidates(g_scene, 0, &c0);
    g_candidates[1] = BuildEECandidates(g_scene, 0, &c1);
    const auto t1 = std::chrono::steady_clock::now();
    seconds[0] = std::chrono::duration<double>(t1 - t0).count();
    const TinyStpfWeights weights;
    for (int kind = 0; kind < 2; ++kind) {
      const std::string k = kind == 0 ? "vf" : "ee";
      std::unordered_map<std::uint64_t, GroupTruth> groups;
      for (const Candidate& c : g_candidates[kind]) groups[GroupKey(g_scene, k, c)];
      const auto a = std::chrono::steady_clock::now();
      const MethodRow row = RunScheduledAnyHitRows(g_scene, args, k, g_candidates[kind], false, 0.0,
                                                   "ScheduledAnyHit", "random", weights, groups);
      const auto b = std::chrono::steady_clock::now();
      seconds[1 + kind] = std::chrono::duration<double>(b - a).count();
      calls[kind] = row.exact_calls;
      cands[kind] = g_candidates[kind].size();
    }
  } catch (const std::exception& e) {
    g_tool_error = e.what();
    return 1;
  }
  return 0;
}

// One timed every-candidate step of the tool on the prepared scene (its
// RunAllExactRows, :1239-1281, for both families after the candidate sweep),
// single-threaded.  seconds[0..1] = {candidates, certificates}; returns the
// number of certified candidates through *calls.
int ref_tool_time_all_exact(double eps_time, double eps_space, int max_depth, double* seconds,
                            std::uint64_t* calls) {
  if (!g_scene_ready) return 1;
  g_tool_config.eps_time = eps_time;
  g_tool_config.eps_space = eps_space;
  g_tool_config.max_subdivision_depth = static_cast<std::uint16_t>(max_depth);
  Args args;
  try {
    const auto t0 = std::chrono::steady_clock::now();
    bool c0 = false, c1 = false;
    g_candidates[0] = BuildVFCandidates(g_scene, 0, &c0);
    g_candidates[1] = BuildEECandidates(g_scene, 0, &c1);
    const auto t1 = std::chrono::steady_clock::now();
    std::uint64_t n = 0;
    for (int kind = 0; kind < 2; ++kind) {
      std::unordered_map<std::uint64_t, GroupTruth> truth;
      const MethodRow row =
          RunAllExactRows(g_scene, args, kind == 0 ? "vf" : "ee", g_candidates[kind], false, 0.0, &truth);
      n += row.exact_calls;
    }
    const auto t2 = std::chrono::steady_clock::now();
    seconds[0] = std::chrono::duration<double>(t1 - t0).count();
    seconds[1] = std::chrono::duration<double>(t2 - t1).count();
    *calls = n;
  } catch (const std::exception& e) {
    g_tool_error = e.what();
    return 1;
  }
  return 0;
}

}  // extern "C"
