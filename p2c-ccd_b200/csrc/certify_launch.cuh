// certify_launch.cuh — launch shape, scratch layout and validation shared by
// every entry point that runs the warp certifier.
#pragma once

#include <cmath>
#include <cstring>

#include "certify_core.cuh"
#include "certify_engine.cuh"
#include "p2c_internal.cuh"

namespace p2c {

constexpr int kCertifyThreads = 128;  // 4 warps per block, one WarpSlots each
constexpr int kCertifyWarps = kCertifyThreads / 32;
constexpr int kCertifyMinBlocks = 4;  // 16 warps per SM: caps registers at 128 per thread

// Device scratch of one certification launch (reset by the launcher).
struct CertifyScratch {
  p2c_certify_stats stats;             // exported verbatim to the caller
  unsigned long long invalid_key[2];   // min over (index << 2 | reason), ~0 if none
  EngineState engine;                  // queues, pool cursors, hungry warps
};

// Fixed-size pools of the cross-warp sharing (independent of the batch size):
// reduction records of trees whose subtrees left their warp, and published
// subtree tasks.  Task tags must read zero before each launch.
constexpr unsigned long long kTreeAggCap = 8192;
constexpr unsigned long long kTaskCap = 16384;
#ifndef P2C_HELPERS_PER_SM
#define P2C_HELPERS_PER_SM 2
#endif
#ifndef P2C_FETCH_PCT
#define P2C_FETCH_PCT 100
#endif
constexpr unsigned long long kHelperWarps = 148ull * P2C_HELPERS_PER_SM;  // idle warps that stay for subtrees
constexpr size_t kScratchHeaderBytes = (sizeof(CertifyScratch) + 255) & ~size_t(255);
constexpr size_t kPoolBytes = kTreeAggCap * sizeof(TreeAgg) + kTaskCap * sizeof(SubtreeTask);

__host__ __device__ inline EnginePools pools_at(void* scratch) {
  EnginePools p;
  char* base = static_cast<char*>(scratch) + kScratchHeaderBytes;
  p.tasks = reinterpret_cast<SubtreeTask*>(base);
  p.aggs = reinterpret_cast<TreeAgg*>(base + kTaskCap * sizeof(SubtreeTask));
  p.task_cap = kTaskCap;
  p.agg_cap = kTreeAggCap;
  p.helper_cap = kHelperWarps;
  return p;
}

struct LaunchShape {
  int grid = 0;
  size_t smem = 0;
};

inline cudaError_t reset_scratch(CertifyScratch* sc, cudaStream_t s, bool with_pools = false) {
  cudaError_t e = cudaMemsetAsync(sc, 0, sizeof(CertifyScratch), s);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(sc->invalid_key, 0xff, sizeof(sc->invalid_key), s);
  if (e != cudaSuccess || !with_pools) return e;
  return cudaMemsetAsync(pools_at(sc).tasks, 0, kTaskCap * sizeof(SubtreeTask), s);
}

template <class K>
int certify_shape(K kernel, LaunchShape* shape) {
  DeviceInfo dev;
  int rc = current_device_info(&dev);
  if (rc != P2C_OK) return rc;
  const size_t smem = sizeof(EngineShared) * kCertifyWarps;
  if (smem > 48 * 1024) {
    P2C_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  int per_sm = 0;
  P2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kCertifyThreads, smem));
  if (per_sm < 1) per_sm = 1;
  shape->grid = dev.sm_count * per_sm;
  shape->smem = smem;
  return P2C_OK;
}

inline CertParams make_params(const p2c_cert_config& cfg, const LaunchShape& shape, long long n) {
  CertParams p;
  p.eps_time = cfg.eps_time;
  p.eps_space = cfg.eps_space;
  p.max_depth = cfg.max_subdivision_depth;
  const long long warps = (long long)shape.grid * kCertifyWarps;
  long long per_warp = warps > 0 ? (n + warps - 1) / warps : 32;
  per_warp = (per_warp * P2C_FETCH_PCT + 99) / 100;  // queries a warp takes at first, in percent of its share
  if (per_warp < 1) per_warp = 1;
  if (per_warp > 32) per_warp = 32;
  p.fetch_limit = (int)per_warp;
  p.budget_ns = device_budget_ns();
  return p;
}

// Validation of CertificateEngineConfig and the interval
// (certificate_engine.cpp:224-242) plus the GPU engine's depth range: node
// keys are 64-bit with a sentinel bit, so a tree deeper than 63 levels must be
// impossible, which holds when max_subdivision_depth <= 63 or eps_time >=
// 2^-50 (bisection of a sub-interval of [0, 1] reaches width <= 2^-50 within
// 51 levels).
inline int validate_cert_config(const p2c_cert_config& cfg, double t0, double t1) {
  if (!std::isfinite(cfg.eps_time) || cfg.eps_time <= 0.0)
    return fail(P2C_ERR_INVALID, "CertificateEngineConfig.eps_time must be finite and positive");
  if (!std::isfinite(cfg.eps_space) || cfg.eps_space <= 0.0)
    return fail(P2C_ERR_INVALID, "CertificateEngineConfig.eps_space must be finite and positive");
  if (!std::isfinite(t0) || !std::isfinite(t1))
    return fail(P2C_ERR_INVALID, "certificate interval endpoints must be finite");
  if (t0 < 0.0 || t1 > 1.0 || t0 > t1)
    return fail(P2C_ERR_INVALID, "certificate interval must satisfy 0 <= t0 <= t1 <= 1");
  if (cfg.max_subdivision_depth > kMaxTreeDepth && cfg.eps_time < std::ldexp(1.0, -50))
    return fail(P2C_ERR_INVALID,
                "CertificateEngineConfig.max_subdivision_depth > 63 needs eps_time >= 2^-50 on the GPU "
                "certifier (interval trees deeper than 63 levels are not supported)");
  return P2C_OK;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void flush_stats(const WarpStats& st, bool ok, CertifyScratch* sc) {
  const unsigned long long nodes = warp_sum(st.nodes), evals = warp_sum(st.evals),
                           don = warp_sum(st.donations), q = warp_sum(st.queries), ops = warp_sum(st.ops);
  if ((threadIdx.x & 31) == 0) {
    // iteration counters are warp-uniform: lane 0's copy is the warp's
    if (st.iters) atomicMax((unsigned long long*)&sc->stats.max_warp_iterations, st.iters);
    if (st.busy) atomicAdd((unsigned long long*)&sc->stats.busy_lane_iterations, st.busy);
    if (nodes) atomicAdd((unsigned long long*)&sc->stats.nodes_evaluated, nodes);
    if (evals) atomicAdd((unsigned long long*)&sc->stats.distance_evals, evals);
    if (don) atomicAdd((unsigned long long*)&sc->stats.donations, don);
    if (q) atomicAdd((unsigned long long*)&sc->stats.queries, q);
    if (ops) atomicAdd((unsigned long long*)&sc->stats.fp64_ops, ops);
    if (!ok) atomicOr((unsigned long long*)&sc->stats.error_word, 1ull);
  }
}

inline int export_stats(CertifyScratch* sc, p2c_certify_stats* stats_dev, cudaStream_t s) {
  if (stats_dev == nullptr) return P2C_OK;
  P2C_CUDA(cudaMemcpyAsync(stats_dev, &sc->stats, sizeof(p2c_certify_stats), cudaMemcpyDeviceToDevice, s));
  return P2C_OK;
}

// Host check after a synchronous launch: time budget and invalid primitives,
// reported with the reference's messages (certificate_engine.cpp:244-264).
inline int check_scratch_outcome(const CertifyScratch& sc, int family) {
  if (sc.stats.error_word != 0ull)
    return fail(P2C_ERR_TIMEOUT, "certification exceeded the device time budget (P2C_DEVICE_BUDGET_MS)");
  const int slot = family == 1 ? 0 : 1;
  const unsigned long long key = sc.invalid_key[slot];
  if (key != ~0ull) {
    const unsigned long long index = key >> 2;
    const int reason = (int)(key & 3ull);
    const char* what = family == 1 ? (reason == 1 ? "point-triangle primitive ids are required"
                                                  : "point-triangle primitive trajectories must be finite")
                                   : (reason == 1 ? "edge-edge primitive ids are required"
                                                  : "edge-edge primitive trajectories must be finite");
    return fail(P2C_ERR_INVALID, "%s (primitive %llu)", what, index);
  }
  return P2C_OK;
}

}  // namespace p2c
