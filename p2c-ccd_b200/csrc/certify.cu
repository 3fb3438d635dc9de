// certify.cu — batch interval certificates over the reference's 240-byte
// primitive records: the sm_100a replacement of PointTriangleKernel /
// EdgeEdgeKernel + RunCudaBatch (cpp/certificate/certificate_cuda.cu:348-552),
// with the CPU certifier's semantics (certificate_engine.cpp:300-386, 481-551).
#include "certify_core.cuh"
#include "certify_launch.cuh"
#include "p2c_internal.cuh"

namespace p2c {

namespace {

// Word layout of a 240-byte record: [id_a, id_b, 4 x (feature_id, p0[3], p1[3])].
__device__ __forceinline__ void load_record(const unsigned long long* __restrict__ rec, Geo& g, int& bad) {
  const long long ida = (long long)__ldg(rec + 0);
  const long long idb = (long long)__ldg(rec + 1);
  bool finite = true;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double a = __longlong_as_double((long long)__ldg(rec + 3 + 7 * i + k));
      const double b = __longlong_as_double((long long)__ldg(rec + 6 + 7 * i + k));
      g.p0[3 * i + k] = a;
      g.p1[3 * i + k] = b;
      finite = finite && isfinite(a) && isfinite(b);
    }
  }
  bad = (ida < 0 || idb < 0) ? 1 : (finite ? 0 : 2);
}

// Both families of a batch of 240-byte records over one interval.
struct RecordProblem {
  const unsigned long long* recs[2];  // 30 words per record
  long long count[2];
  p2c_interval_result* out[2];
  unsigned long long* invalid_key;    // [2]: min over (index << 2 | reason)
  double T0, T1;
  __device__ __forceinline__ long long n(int f) const { return pick(count, f); }
  __device__ __forceinline__ bool skip(int, long long) const { return false; }
  __device__ __forceinline__ void load(int f, long long q, Geo& g, double& t0, double& t1, int& bad) const {
    load_record(pick(recs, f) + 30 * q, g, bad);
    t0 = T0;
    t1 = T1;
  }
  __device__ __forceinline__ void finish(int f, long long q, const Outcome& o) const {
    const unsigned long long* r = pick(recs, f) + 30 * q;
    store_interval_result(pick(out, f) + q, f, o, (long long)r[0], (long long)r[1]);
  }
  __device__ __forceinline__ void invalid(int f, long long q, int bad, double t0, double t1) const {
    Outcome o{3, t0, t1, t1, 0.0};
    store_interval_result(pick(out, f) + q, f, o, -1, -1);
    atomicMin(&invalid_key[f - 1], ((unsigned long long)q << 2) | (unsigned long long)bad);
  }
};

template <bool kShare, bool kCount>
__global__ void __launch_bounds__(kCertifyThreads, kCertifyMinBlocks)
    certify_records_kernel(const __grid_constant__ RecordProblem prob, const __grid_constant__ CertParams prm,
                           int fetch_pt, int fetch_ee, const __grid_constant__ EnginePools pools,
                           CertifyScratch* scratch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EngineShared& sh = reinterpret_cast<EngineShared*>(smem_raw)[threadIdx.x >> 5];
  WarpStats st;
  const unsigned long long t_start = global_ns();
  // odd warps take the edge-edge queue first, so that the tail of one family
  // overlaps the bulk of the other
  const bool ee_first = ((blockIdx.x * kCertifyWarps + (threadIdx.x >> 5)) & 1u) != 0u;
  const bool ok = run_engine<kShare, kShare, kCount>(prob, prm, fetch_pt, fetch_ee, ee_first, sh, st,
                                                     &scratch->engine, pools, t_start);
  flush_stats(st, ok, scratch);
}

}  // namespace

// Launch both families in one persistent launch.  Scratch must hold a
// CertifyScratch and is reset here.
int launch_certify_records(const void* pt, long long n_pt, const void* ee, long long n_ee, double T0,
                           double T1, const p2c_cert_config& cfg, p2c_interval_result* out_pt,
                           p2c_interval_result* out_ee, void* scratch, size_t scratch_bytes, bool census,
                           cudaStream_t stream) {
  if (scratch_bytes < kScratchHeaderBytes + kPoolBytes)
    return fail(P2C_ERR_INVALID, "certification workspace too small: %zu < %zu bytes", scratch_bytes,
                kScratchHeaderBytes + kPoolBytes);
  CertifyScratch* sc = reinterpret_cast<CertifyScratch*>(scratch);
  P2C_CUDA(reset_scratch(sc, stream, !census));
  if (n_pt + n_ee == 0) return P2C_OK;
  LaunchShape shape;
  int rc = census ? certify_shape(certify_records_kernel<false, true>, &shape)
                  : certify_shape(certify_records_kernel<true, false>, &shape);
  if (rc != P2C_OK) return rc;
  const CertParams ppt = make_params(cfg, shape, n_pt);
  const CertParams pee = make_params(cfg, shape, n_ee);
  RecordProblem prob;
  prob.recs[0] = reinterpret_cast<const unsigned long long*>(pt);
  prob.recs[1] = reinterpret_cast<const unsigned long long*>(ee);
  prob.count[0] = n_pt;
  prob.count[1] = n_ee;
  prob.out[0] = out_pt;
  prob.out[1] = out_ee;
  prob.invalid_key = sc->invalid_key;
  prob.T0 = T0;
  prob.T1 = T1;
  const EnginePools pools = pools_at(sc);
  if (census) {
    certify_records_kernel<false, true><<<shape.grid, kCertifyThreads, shape.smem, stream>>>(
        prob, ppt, ppt.fetch_limit, pee.fetch_limit, pools, sc);
  } else {
    certify_records_kernel<true, false><<<shape.grid, kCertifyThreads, shape.smem, stream>>>(
        prob, ppt, ppt.fetch_limit, pee.fetch_limit, pools, sc);
  }
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

}  // namespace p2c

using namespace p2c;

namespace {

int validate_batch_args(int64_t n, double t0, double t1, const p2c_cert_config* cfg, const void* prims,
                        const void* out) {
  if (cfg == nullptr) return fail(P2C_ERR_INVALID, "CertificateEngineConfig pointer is null");
  if (n < 0) return fail(P2C_ERR_INVALID, "primitive count must be non-negative");
  if (n > 0 && (prims == nullptr || out == nullptr))
    return fail(P2C_ERR_INVALID, "CUDA exact result output pointer is null");
  return validate_cert_config(*cfg, t0, t1);
}

HostApiBuffers g_host_buffers;

int certify_host(const void* prims, int64_t n, int family, double t0, double t1, const p2c_cert_config* cfg,
                 p2c_interval_result* results) {
  int rc = validate_batch_args(n, t0, t1, cfg, prims, results);
  if (rc != P2C_OK) return rc;
  if (n == 0) return P2C_OK;  // RunCudaBatch returns Ok on empty input (certificate_cuda.cu:465-468)
  std::lock_guard<std::mutex> lock(g_host_buffers.mu);
  const size_t in_bytes = (size_t)n * 240u, out_bytes = (size_t)n * sizeof(p2c_interval_result);
  const size_t ws_off = (in_bytes + out_bytes + 255u) & ~size_t(255);
  const size_t ws_bytes = kScratchHeaderBytes + kPoolBytes;
  rc = ensure_buffer(g_host_buffers, ws_off + ws_bytes);
  if (rc != P2C_OK) return rc;
  char* base = static_cast<char*>(g_host_buffers.dev);
  void* d_in = base;
  auto* d_out = reinterpret_cast<p2c_interval_result*>(base + in_bytes);
  void* d_ws = base + ws_off;
  cudaStream_t s = nullptr;
  P2C_CUDA(cudaMemcpyAsync(d_in, prims, in_bytes, cudaMemcpyHostToDevice, s));
  rc = family == 1 ? launch_certify_records(d_in, n, nullptr, 0, t0, t1, *cfg, d_out, nullptr, d_ws, ws_bytes,
                                            false, s)
                   : launch_certify_records(nullptr, 0, d_in, n, t0, t1, *cfg, nullptr, d_out, d_ws, ws_bytes,
                                            false, s);
  if (rc != P2C_OK) return rc;
  P2C_CUDA(cudaMemcpyAsync(results, d_out, out_bytes, cudaMemcpyDeviceToHost, s));
  CertifyScratch host_sc;
  P2C_CUDA(cudaMemcpyAsync(&host_sc, d_ws, sizeof(CertifyScratch), cudaMemcpyDeviceToHost, s));
  P2C_CUDA(cudaStreamSynchronize(s));
  return check_scratch_outcome(host_sc, family);
}

}  // namespace

extern "C" {

size_t p2c_certify_workspace_bytes(int64_t n) {
  (void)n;  // the scratch does not grow with the batch
  return kScratchHeaderBytes + kPoolBytes;
}

int p2c_certify_pt_batch(const p2c_point_triangle* prims_dev, int64_t n, double interval_t0, double interval_t1,
                         const p2c_cert_config* config, p2c_interval_result* results_dev, void* workspace_dev,
                         size_t workspace_bytes, p2c_certify_stats* stats_dev, void* stream) {
  int rc = validate_batch_args(n, interval_t0, interval_t1, config, prims_dev, results_dev);
  if (rc != P2C_OK) return rc;
  if (workspace_dev == nullptr) return fail(P2C_ERR_INVALID, "workspace pointer is null");
  rc = launch_certify_records(prims_dev, n, nullptr, 0, interval_t0, interval_t1, *config, results_dev, nullptr,
                              workspace_dev, workspace_bytes, false, as_stream(stream));
  if (rc != P2C_OK) return rc;
  return export_stats(reinterpret_cast<CertifyScratch*>(workspace_dev), stats_dev, as_stream(stream));
}

int p2c_certify_ee_batch(const p2c_edge_edge* prims_dev, int64_t n, double interval_t0, double interval_t1,
                         const p2c_cert_config* config, p2c_interval_result* results_dev, void* workspace_dev,
                         size_t workspace_bytes, p2c_certify_stats* stats_dev, void* stream) {
  int rc = validate_batch_args(n, interval_t0, interval_t1, config, prims_dev, results_dev);
  if (rc != P2C_OK) return rc;
  if (workspace_dev == nullptr) return fail(P2C_ERR_INVALID, "workspace pointer is null");
  rc = launch_certify_records(nullptr, 0, prims_dev, n, interval_t0, interval_t1, *config, nullptr, results_dev,
                              workspace_dev, workspace_bytes, false, as_stream(stream));
  if (rc != P2C_OK) return rc;
  return export_stats(reinterpret_cast<CertifyScratch*>(workspace_dev), stats_dev, as_stream(stream));
}

int p2c_certify_batch2(const p2c_point_triangle* pt_dev, int64_t n_pt, const p2c_edge_edge* ee_dev, int64_t n_ee,
                       double interval_t0, double interval_t1, const p2c_cert_config* config,
                       p2c_interval_result* pt_results_dev, p2c_interval_result* ee_results_dev,
                       void* workspace_dev, size_t workspace_bytes, p2c_certify_stats* stats_dev, void* stream) {
  int rc = validate_batch_args(n_pt, interval_t0, interval_t1, config, pt_dev, pt_results_dev);
  if (rc != P2C_OK) return rc;
  rc = validate_batch_args(n_ee, interval_t0, interval_t1, config, ee_dev, ee_results_dev);
  if (rc != P2C_OK) return rc;
  if (workspace_dev == nullptr) return fail(P2C_ERR_INVALID, "workspace pointer is null");
  rc = launch_certify_records(pt_dev, n_pt, ee_dev, n_ee, interval_t0, interval_t1, *config, pt_results_dev,
                              ee_results_dev, workspace_dev, workspace_bytes, false, as_stream(stream));
  if (rc != P2C_OK) return rc;
  return export_stats(reinterpret_cast<CertifyScratch*>(workspace_dev), stats_dev, as_stream(stream));
}

int p2c_certify_pt_batch_host(const p2c_point_triangle* prims_host, int64_t n, double interval_t0,
                              double interval_t1, const p2c_cert_config* config,
                              p2c_interval_result* results_host) {
  return certify_host(prims_host, n, 1, interval_t0, interval_t1, config, results_host);
}

int p2c_certify_ee_batch_host(const p2c_edge_edge* prims_host, int64_t n, double interval_t0,
                              double interval_t1, const p2c_cert_config* config,
                              p2c_interval_result* results_host) {
  return certify_host(prims_host, n, 2, interval_t0, interval_t1, config, results_host);
}

int p2c_certify_census(const p2c_point_triangle* pt_dev, int64_t n_pt, const p2c_edge_edge* ee_dev, int64_t n_ee,
                       double interval_t0, double interval_t1, const p2c_cert_config* config,
                       p2c_interval_result* pt_results_dev, p2c_interval_result* ee_results_dev,
                       void* workspace_dev, size_t workspace_bytes, p2c_certify_stats* stats_dev,
                       void* stream) {
  int rc = validate_batch_args(n_pt, interval_t0, interval_t1, config, pt_dev, pt_results_dev);
  if (rc != P2C_OK) return rc;
  rc = validate_batch_args(n_ee, interval_t0, interval_t1, config, ee_dev, ee_results_dev);
  if (rc != P2C_OK) return rc;
  if (workspace_dev == nullptr) return fail(P2C_ERR_INVALID, "workspace pointer is null");
  rc = launch_certify_records(pt_dev, n_pt, ee_dev, n_ee, interval_t0, interval_t1, *config, pt_results_dev,
                              ee_results_dev, workspace_dev, workspace_bytes, true, as_stream(stream));
  if (rc != P2C_OK) return rc;
  return export_stats(reinterpret_cast<CertifyScratch*>(workspace_dev), stats_dev, as_stream(stream));
}

}  // extern "C"

#ifdef P2C_ENGINE_PROFILE
// Measurement build only: the engine phase clock of this file's kernels (see
// certify_engine.cuh), read and cleared by the host.
extern "C" int p2c_engine_profile_certify(unsigned long long* out16, int clear) {
  if (cudaMemcpyFromSymbol(out16, p2c::g_engine_prof, 16 * sizeof(unsigned long long)) != cudaSuccess) return 2;
  if (clear) {
    static const unsigned long long zero[16] = {};
    if (cudaMemcpyToSymbol(p2c::g_engine_prof, zero, sizeof(zero)) != cudaSuccess) return 2;
  }
  return 0;
}
#endif
