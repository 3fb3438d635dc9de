// ref_cuda.cpp — C ABI over the reference's CUDA batch certifier compiled
// unchanged (cpp/certificate/certificate_cuda.cu) for sm_100a.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles the reference's
// certificate_cuda.cu and certificate_engine.cpp where they lie in the
// reference checkout, with this file, into oracle/_ref/libp2c_ref_cuda.so.
// It is the reference's own GPU path (EvaluatePointTriangleBatchCuda /
// EvaluateEdgeEdgeBatchCuda: host vectors in, cudaMalloc + cudaMemcpy + one
// thread per primitive with a 128-entry interval stack + cudaDeviceSynchronize
// + cudaFree per call, certificate_cuda.cu:348-552), timed as a comparison
// row.  Its answers are not parity truth: it returns undecided at the first
// undecided leaf where the CPU recursion goes on to the right half.  The
// product never loads this library.
#include "certificate/certificate_cuda.h"
#include "certificate/certificate_engine.h"

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../include/p2c_b200.h"

namespace {

static_assert(sizeof(p2cccd::PointTriangleIntervalPrimitive) == sizeof(p2c_point_triangle));
static_assert(sizeof(p2cccd::EdgeEdgeIntervalPrimitive) == sizeof(p2c_edge_edge));
static_assert(sizeof(p2cccd::PrimitiveIntervalResult) == sizeof(p2c_interval_result));

thread_local std::string g_error;

p2cccd::CertificateEngineConfig MakeConfig(double eps_time, double eps_space, int max_depth) {
  p2cccd::CertificateEngineConfig c;
  c.eps_time = eps_time;
  c.eps_space = eps_space;
  c.max_subdivision_depth = static_cast<std::uint16_t>(max_depth);
  return c;
}

template <typename Prim, typename Fn>
int Run(const void* records, std::int64_t n, double t0, double t1, double eps_time, double eps_space, int max_depth,
        p2c_interval_result* out, Fn fn) {
  std::vector<Prim> prims(static_cast<std::size_t>(n));
  if (n > 0) std::memcpy(prims.data(), records, sizeof(Prim) * static_cast<std::size_t>(n));
  std::vector<p2cccd::PrimitiveIntervalResult> res;
  const p2cccd::Status st = fn(prims, t0, t1, MakeConfig(eps_time, eps_space, max_depth), &res);
  if (!st.ok) {
    g_error = st.message;
    return 1;
  }
  if (!res.empty()) std::memcpy(out, res.data(), sizeof(p2c_interval_result) * res.size());
  return 0;
}

}  // namespace

extern "C" {

const char* ref_cuda_last_error() { return g_error.c_str(); }

int ref_cuda_is_built() { return p2cccd::IsCudaExactBuilt() ? 1 : 0; }

// family 1: point-triangle records, 2: edge-edge records (240 bytes each).
int ref_cuda_eval_batch(int family, const void* records, std::int64_t n, double t0, double t1, double eps_time,
                        double eps_space, int max_depth, p2c_interval_result* out) {
  if (family == 1)
    return Run<p2cccd::PointTriangleIntervalPrimitive>(records, n, t0, t1, eps_time, eps_space, max_depth, out,
                                                       p2cccd::EvaluatePointTriangleBatchCuda);
  return Run<p2cccd::EdgeEdgeIntervalPrimitive>(records, n, t0, t1, eps_time, eps_space, max_depth, out,
                                                p2cccd::EvaluateEdgeEdgeBatchCuda);
}

// CrossCheckCpuCudaExact (certificate_cuda.cu:616-679): 0 when the CPU and
// CUDA certificates agree under the reference's comparison rules.
int ref_cuda_cross_check(const void* pt, std::int64_t n_pt, const void* ee, std::int64_t n_ee, double t0, double t1,
                         double eps_time, double eps_space, int max_depth, double eps_cert) {
  std::vector<p2cccd::PointTriangleIntervalPrimitive> a(static_cast<std::size_t>(n_pt));
  std::vector<p2cccd::EdgeEdgeIntervalPrimitive> b(static_cast<std::size_t>(n_ee));
  if (n_pt > 0) std::memcpy(a.data(), pt, sizeof(p2c_point_triangle) * static_cast<std::size_t>(n_pt));
  if (n_ee > 0) std::memcpy(b.data(), ee, sizeof(p2c_edge_edge) * static_cast<std::size_t>(n_ee));
  const p2cccd::Status st =
      p2cccd::CrossCheckCpuCudaExact(a, b, t0, t1, MakeConfig(eps_time, eps_space, max_depth), eps_cert);
  g_error = st.message;
  return st.ok ? 0 : 1;
}

}  // extern "C"
