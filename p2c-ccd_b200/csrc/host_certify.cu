// host_certify.cu — the library's CPU certifier.
//
// The reference cross-checks its CUDA kernel against its CPU recursion
// (CrossCheckCpuCudaExact, certificate_cuda.cu:616-679); this file is the CPU
// side of that check inside this library, so a caller's cross-check compares
// the GPU engine with an independent host evaluation of the same procedure
// (EvaluateIntervalRecursive, certificate_engine.cpp:300-386): three samples
// per node (t0, mid, t1) with the first sample within eps_space giving a
// collision, then the motion lower bound, then the depth / width limit, then
// left before right.  It shares only the distance and motion-radius formulas
// with the device (certify_core.cuh, compiled here for the host: plain IEEE
// operators, no FMA contraction); the traversal is a depth-first loop of its
// own.  The GPU entry points never call it: it is not a fallback.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "certify_core.cuh"
#include "p2c_internal.cuh"

namespace p2c {
namespace {

// Geometry of one 240-byte record: [id_a, id_b, 4 x (feature_id, p0[3], p1[3])].
struct HostGeo {
  double a0[12], a1[12];
  __host__ __device__ double p0(int k) const { return a0[k]; }
  __host__ __device__ double p1(int k) const { return a1[k]; }
};

struct HostNode {
  double t0, t1, d0, d1;
  int depth;
};

void pack_result(p2c_interval_result* out, int status, unsigned mask, double t0, double t1, double toi, double margin,
                 int witness_family, long long ida, long long idb, int reason, int refine) {
  std::memset(out, 0, sizeof(*out));
  out->status = (uint8_t)status;
  out->covered_feature_mask = mask;
  out->interval_t0 = t0;
  out->interval_t1 = t1;
  out->toi_upper = toi;
  out->safe_margin_lb = margin;
  out->witness_family = (uint8_t)witness_family;
  out->witness_id_a = ida;
  out->witness_id_b = idb;
  out->reason_code = (uint16_t)reason;
  out->next_refinement_mode = (uint8_t)refine;
}

template <int kFamily>
void certify_one(const unsigned long long* rec, double T0, double T1, const p2c_cert_config& cfg,
                 p2c_interval_result* out, std::vector<HostNode>& stack) {
  HostGeo g;
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 3; ++k) {
      std::memcpy(&g.a0[3 * i + k], rec + 3 + 7 * i + k, 8);
      std::memcpy(&g.a1[3 * i + k], rec + 6 + 7 * i + k, 8);
    }
  const long long ida = (long long)rec[0], idb = (long long)rec[1];
  NoCount nc;
  double nrm[4];
  motion_norms(g, nrm, nc);
  const double eps = cfg.eps_space;
  stack.clear();
  stack.push_back({T0, T1, distance_at<kFamily>(g, T0, nc), distance_at<kFamily>(g, T1, nc), 0});
  double margin = INFINITY;
  bool undecided = false;
  while (!stack.empty()) {
    const HostNode nd = stack.back();
    stack.pop_back();
    const double mid = mul(0.5, add(nd.t0, nd.t1));
    const double dm = distance_at<kFamily>(g, mid, nc);
    if (nd.d0 <= eps || dm <= eps || nd.d1 <= eps) {  // the first sample within eps_space, in t0, mid, t1 order
      const double toi = nd.d0 <= eps ? nd.t0 : (dm <= eps ? mid : nd.t1);
      pack_result(out, P2C_STATUS_COLLISION, 0u, nd.t0, nd.t1, toi, 0.0, kFamily, ida, idb, P2C_REASON_NONE,
                  P2C_REFINE_NONE);
      return;
    }
    const double lb = sub(dm, motion_radius<kFamily>(nrm, nd.t0, nd.t1, nc));
    if (lb > eps) {
      margin = std::min(margin, max_std(0.0, sub(lb, eps)));
      continue;
    }
    if (nd.depth >= cfg.max_subdivision_depth || sub(nd.t1, nd.t0) <= cfg.eps_time) {
      undecided = true;
      continue;
    }
    stack.push_back({mid, nd.t1, dm, nd.d1, nd.depth + 1});  // right, visited after the whole left subtree
    stack.push_back({nd.t0, mid, nd.d0, dm, nd.depth + 1});
  }
  if (undecided)
    pack_result(out, P2C_STATUS_UNDECIDED, 0u, T0, T1, T1, 0.0, 0, -1, -1, P2C_REASON_MAX_SUBDIVISION_DEPTH,
                P2C_REFINE_BISECT_INTERVAL);
  else
    pack_result(out, P2C_STATUS_SEPARATION, (unsigned)kFamily, T0, T1, T1, margin, 0, -1, -1, P2C_REASON_NONE,
                P2C_REFINE_NONE);
}

// ValidatePointTrianglePrimitive / ValidateEdgeEdgePrimitive (certificate_engine.cpp:244-264).
int validate_record(const unsigned long long* rec, int family, long long index) {
  if ((long long)rec[0] < 0 || (long long)rec[1] < 0)
    return fail(P2C_ERR_INVALID, "%s primitive ids are required (primitive %lld)",
                family == 1 ? "point-triangle" : "edge-edge", index);
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 6; ++k) {
      double v;
      std::memcpy(&v, rec + 3 + 7 * i + k, 8);
      if (!std::isfinite(v))
        return fail(P2C_ERR_INVALID, "%s primitive trajectories must be finite (primitive %lld)",
                    family == 1 ? "point-triangle" : "edge-edge", index);
    }
  return P2C_OK;
}

int certify_cpu(const void* prims, long long n, int family, double t0, double t1, const p2c_cert_config* cfg,
                p2c_interval_result* out) {
  if (cfg == nullptr) return fail(P2C_ERR_INVALID, "CertificateEngineConfig pointer is null");
  if (!std::isfinite(cfg->eps_time) || cfg->eps_time <= 0.0)
    return fail(P2C_ERR_INVALID, "CertificateEngineConfig.eps_time must be finite and positive");
  if (!std::isfinite(cfg->eps_space) || cfg->eps_space <= 0.0)
    return fail(P2C_ERR_INVALID, "CertificateEngineConfig.eps_space must be finite and positive");
  if (!std::isfinite(t0) || !std::isfinite(t1))
    return fail(P2C_ERR_INVALID, "certificate interval endpoints must be finite");
  if (t0 < 0.0 || t1 > 1.0 || t0 > t1) return fail(P2C_ERR_INVALID, "certificate interval must satisfy 0 <= t0 <= t1 <= 1");
  if (n < 0) return fail(P2C_ERR_INVALID, "primitive count must be non-negative");
  if (n == 0) return P2C_OK;
  if (prims == nullptr || out == nullptr) return fail(P2C_ERR_INVALID, "primitive or result pointer is null");
  const unsigned long long* recs = static_cast<const unsigned long long*>(prims);
  for (long long i = 0; i < n; ++i) {
    const int rc = validate_record(recs + 30 * i, family, i);
    if (rc != P2C_OK) return rc;
  }
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const long long workers = std::min<long long>(hw, (n + 255) / 256);
  auto run = [&](long long w) {
    std::vector<HostNode> stack;
    for (long long i = w; i < n; i += workers) {
      if (family == 1) certify_one<1>(recs + 30 * i, t0, t1, *cfg, out + i, stack);
      else certify_one<2>(recs + 30 * i, t0, t1, *cfg, out + i, stack);
    }
  };
  std::vector<std::thread> pool;
  for (long long w = 1; w < workers; ++w) pool.emplace_back(run, w);
  run(0);
  for (auto& th : pool) th.join();
  return P2C_OK;
}

}  // namespace
}  // namespace p2c

extern "C" {

int p2c_certify_pt_batch_cpu(const p2c_point_triangle* prims_host, int64_t n, double interval_t0, double interval_t1,
                             const p2c_cert_config* config, p2c_interval_result* results_host) {
  return p2c::certify_cpu(prims_host, n, 1, interval_t0, interval_t1, config, results_host);
}

int p2c_certify_ee_batch_cpu(const p2c_edge_edge* prims_host, int64_t n, double interval_t0, double interval_t1,
                             const p2c_cert_config* config, p2c_interval_result* results_host) {
  return p2c::certify_cpu(prims_host, n, 2, interval_t0, interval_t1, config, results_host);
}

}  // extern "C"
