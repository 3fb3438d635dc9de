// queries.cu — many work items certified in one launch: the device form of
// CertificateEngine::Evaluate (cpp/certificate/certificate_engine.cpp:729-824)
// applied to every ExactCertificateQuery of a work queue
// (ProcessExactWorkQueueCpu, :593-661).
//
// Input: the queue's point-triangle and edge-edge primitives as two flat
// record lists, each primitive tagged with its query index (non-decreasing:
// a query's primitives are contiguous and in its list order), and per query
// the work item's interval and feature_family_mask.  Each primitive is
// certified over its query's interval; a per-query reduction then reproduces
// Evaluate: the first colliding primitive in list order (VF list, then EE
// list) is the witness; a primitive that fails validation before that point
// makes the query an InvalidInput error (Evaluate returns the status, and the
// work queue turns it into an undecided InvalidInput certificate, :629-632);
// otherwise any undecided makes it undecided, else separation.
#include <mutex>

#include "certify_core.cuh"
#include "certify_launch.cuh"

namespace p2c {
namespace {

struct QueryAgg {
  unsigned long long first_key;    // min over collisions of (fam << 62 | primitive index)
  unsigned long long invalid_key;  // min over invalid primitives, same key
  unsigned long long margin_bits;
  unsigned int any_sep[2];
  unsigned int any_undecided[2];
};

__device__ __forceinline__ void load_rec(const unsigned long long* __restrict__ rec, Geo& g, int& bad) {
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

// Both families of a work queue: each primitive over its work item's interval.
struct QueryProblem {
  const unsigned long long* recs[2];
  const long long* prim_query[2];
  long long count[2];
  const double* q_t0;
  const double* q_t1;
  p2c_interval_result* out[2];
  QueryAgg* agg;
  __device__ __forceinline__ long long n(int f) const { return pick(count, f); }
  __device__ __forceinline__ unsigned long long key(int f, long long q) const {
    return ((unsigned long long)(f - 1) << 62) | (unsigned long long)q;
  }
  __device__ __forceinline__ bool skip(int, long long) const { return false; }
  __device__ __forceinline__ void load(int f, long long q, Geo& g, double& t0, double& t1, int& bad) const {
    load_rec(pick(recs, f) + 30 * q, g, bad);
    const long long qi = pick(prim_query, f)[q];
    t0 = q_t0[qi];
    t1 = q_t1[qi];
  }
  __device__ __forceinline__ void finish(int f, long long q, const Outcome& o) const {
    const unsigned long long* r = pick(recs, f) + 30 * q;
    store_interval_result(pick(out, f) + q, f, o, (long long)r[0], (long long)r[1]);
    QueryAgg& a = agg[pick(prim_query, f)[q]];
    if (o.status == P2C_STATUS_COLLISION) atomicMin(&a.first_key, key(f, q));
    else if (o.status == P2C_STATUS_SEPARATION) {
      atomicMin(&a.margin_bits, (unsigned long long)__double_as_longlong(o.margin));
      if (a.any_sep[f - 1] == 0u) atomicExch(&a.any_sep[f - 1], 1u);
    } else if (a.any_undecided[f - 1] == 0u) {
      atomicExch(&a.any_undecided[f - 1], 1u);
    }
  }
  __device__ __forceinline__ void invalid(int f, long long q, int bad, double t0, double t1) const {
    Outcome o{3, t0, t1, t1, 0.0};
    store_interval_result(pick(out, f) + q, f, o, -1, -1);
    atomicMin(&agg[pick(prim_query, f)[q]].invalid_key, key(f, q));
  }
};

__global__ void __launch_bounds__(kCertifyThreads, kCertifyMinBlocks)
    certify_queries_kernel(const __grid_constant__ QueryProblem prob, const __grid_constant__ CertParams prm,
                           int fetch_pt, int fetch_ee, CertifyScratch* sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EngineShared& sh = reinterpret_cast<EngineShared*>(smem_raw)[threadIdx.x >> 5];
  WarpStats st;
  const unsigned long long t_start = global_ns();
  const bool ee_first = ((blockIdx.x * kCertifyWarps + (threadIdx.x >> 5)) & 1u) != 0u;
  // no cross-warp pools here: the scratch stays one record per work item
  const EnginePools no_pools{};
  const bool ok = run_engine<true, false, false>(prob, prm, fetch_pt, fetch_ee, ee_first, sh, st, &sc->engine,
                                                 no_pools, t_start);
  flush_stats(st, ok, sc);
}

__global__ void init_agg_kernel(QueryAgg* agg, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  QueryAgg a;
  a.first_key = ~0ull;
  a.invalid_key = ~0ull;
  a.margin_bits = 0x7ff0000000000000ull;
  a.any_sep[0] = a.any_sep[1] = 0u;
  a.any_undecided[0] = a.any_undecided[1] = 0u;
  agg[i] = a;
}

__device__ __forceinline__ uint8_t refine_for(uint16_t r) {  // :279-291
  return r == P2C_REASON_MISSING_GEOMETRY ? P2C_REFINE_REQUEST_GEOMETRY
         : r == P2C_REASON_MAX_SUBDIVISION_DEPTH ? P2C_REFINE_BISECT_INTERVAL
         : r == P2C_REASON_INVALID_INPUT ? P2C_REFINE_REQUEST_GEOMETRY
                                         : P2C_REFINE_ESCALATE_PRECISION;
}

// One thread per query.  pt_off/ee_off are CSR offsets of each query's
// primitives in the flat lists (n_queries + 1 entries).
__global__ void finalize_queries_kernel(const QueryAgg* agg, long long n_queries, const long long* pt_off,
                                        const long long* ee_off, const unsigned* q_mask, const double* q_t1,
                                        const p2c_interval_result* out_pt, const p2c_interval_result* out_ee,
                                        p2c_query_certificate* certs) {
  const long long qi = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= n_queries) return;
  const QueryAgg a = agg[qi];
  const unsigned mask = q_mask[qi];
  p2c_query_certificate c{};
  c.witness_id_a = -1;
  c.witness_id_b = -1;
  c.witness_index = -1;
  c.toi_upper = q_t1[qi];
  // an invalid primitive evaluated before the first collision fails the query
  if (a.invalid_key != ~0ull && a.invalid_key < a.first_key) {
    c.status = P2C_STATUS_UNDECIDED;
    c.reason_code = P2C_REASON_INVALID_INPUT;
    c.next_refinement_mode = refine_for(P2C_REASON_INVALID_INPUT);
    certs[qi] = c;
    return;
  }
  if (a.first_key != ~0ull) {
    const int f = (int)(a.first_key >> 62);
    const long long idx = (long long)(a.first_key & ((1ull << 62) - 1));
    const p2c_interval_result& r = (f == 0 ? out_pt : out_ee)[idx];
    c.status = P2C_STATUS_COLLISION;
    c.witness_family = r.witness_family;
    c.toi_upper = r.toi_upper;
    c.witness_id_a = r.witness_id_a;
    c.witness_id_b = r.witness_id_b;
    c.witness_index = idx - (f == 0 ? pt_off[qi] : ee_off[qi]);
    certs[qi] = c;
    return;
  }
  bool evaluated_any = false, has_undecided = false;
  uint16_t reason = P2C_REASON_NONE;
  for (int f = 0; f < 2; ++f) {
    if ((mask & (1u << f)) == 0u) continue;
    const long long n = f == 0 ? pt_off[qi + 1] - pt_off[qi] : ee_off[qi + 1] - ee_off[qi];
    if (n == 0) {
      has_undecided = true;
      reason = P2C_REASON_MISSING_GEOMETRY;
    } else {
      evaluated_any = true;
      if (a.any_undecided[f]) {
        has_undecided = true;
        reason = P2C_REASON_MAX_SUBDIVISION_DEPTH;
      }
    }
  }
  if (!evaluated_any || has_undecided) {
    const uint16_t r = !evaluated_any ? (uint16_t)P2C_REASON_MISSING_GEOMETRY
                                      : (reason == P2C_REASON_NONE ? (uint16_t)P2C_REASON_MAX_SUBDIVISION_DEPTH
                                                                   : reason);
    c.status = P2C_STATUS_UNDECIDED;
    c.reason_code = r;
    c.next_refinement_mode = refine_for(r);
  } else {
    c.status = P2C_STATUS_SEPARATION;
    const double m = __longlong_as_double((long long)a.margin_bits);
    c.safe_margin_lb = isfinite(m) ? m : 0.0;
    c.covered_feature_mask = ((mask & 1u) && a.any_sep[0] ? 1u : 0u) | ((mask & 2u) && a.any_sep[1] ? 2u : 0u);
  }
  certs[qi] = c;
}

}  // namespace

constexpr size_t queries_workspace_bytes_for(long long n_queries) {
  return ((sizeof(CertifyScratch) + 255) & ~size_t(255)) + sizeof(QueryAgg) * (size_t)(n_queries > 0 ? n_queries : 1);
}

size_t queries_workspace_bytes(long long n_queries) { return queries_workspace_bytes_for(n_queries); }

}  // namespace p2c

extern "C" {

size_t p2c_certify_queries_workspace_bytes(int64_t n_queries) { return p2c::queries_workspace_bytes(n_queries); }

int p2c_certify_queries(const p2c_point_triangle* pt_dev, int64_t n_pt, const int64_t* pt_query_dev,
                        const p2c_edge_edge* ee_dev, int64_t n_ee, const int64_t* ee_query_dev, int64_t n_queries,
                        const int64_t* pt_offsets_dev, const int64_t* ee_offsets_dev, const double* q_t0_dev,
                        const double* q_t1_dev, const uint32_t* q_mask_dev, const p2c_cert_config* config,
                        p2c_interval_result* pt_results_dev, p2c_interval_result* ee_results_dev,
                        p2c_query_certificate* certs_dev, void* workspace_dev, size_t workspace_bytes,
                        p2c_certify_stats* stats_dev, void* stream) {
  using namespace p2c;
  if (config == nullptr) return fail(P2C_ERR_INVALID, "CertificateEngineConfig pointer is null");
  // interval validity is per work item (validated by the caller); check the config
  int rc = validate_cert_config(*config, 0.0, 1.0);
  if (rc != P2C_OK) return rc;
  if (n_pt < 0 || n_ee < 0 || n_queries < 0) return fail(P2C_ERR_INVALID, "counts must be non-negative");
  if (n_queries == 0) return P2C_OK;
  if (workspace_dev == nullptr || workspace_bytes < queries_workspace_bytes(n_queries))
    return fail(P2C_ERR_INVALID, "query workspace too small");
  if (pt_offsets_dev == nullptr || ee_offsets_dev == nullptr || q_t0_dev == nullptr || q_t1_dev == nullptr ||
      q_mask_dev == nullptr || certs_dev == nullptr)
    return fail(P2C_ERR_INVALID, "query arrays are null");
  cudaStream_t s = as_stream(stream);
  CertifyScratch* sc = reinterpret_cast<CertifyScratch*>(workspace_dev);
  QueryAgg* agg = reinterpret_cast<QueryAgg*>(static_cast<char*>(workspace_dev) +
                                              ((sizeof(CertifyScratch) + 255) & ~size_t(255)));
  P2C_CUDA(reset_scratch(sc, s));
  init_agg_kernel<<<(unsigned)((n_queries + 255) / 256), 256, 0, s>>>(agg, n_queries);
  P2C_CUDA(cudaGetLastError());
  if (n_pt + n_ee > 0) {
    LaunchShape shape;
    rc = certify_shape(certify_queries_kernel, &shape);
    if (rc != P2C_OK) return rc;
    const CertParams ppt = make_params(*config, shape, n_pt), pee = make_params(*config, shape, n_ee);
    QueryProblem prob;
    prob.recs[0] = reinterpret_cast<const unsigned long long*>(pt_dev);
    prob.recs[1] = reinterpret_cast<const unsigned long long*>(ee_dev);
    prob.prim_query[0] = reinterpret_cast<const long long*>(pt_query_dev);
    prob.prim_query[1] = reinterpret_cast<const long long*>(ee_query_dev);
    prob.count[0] = n_pt;
    prob.count[1] = n_ee;
    prob.q_t0 = q_t0_dev;
    prob.q_t1 = q_t1_dev;
    prob.out[0] = pt_results_dev;
    prob.out[1] = ee_results_dev;
    prob.agg = agg;
    certify_queries_kernel<<<shape.grid, kCertifyThreads, shape.smem, s>>>(prob, ppt, ppt.fetch_limit,
                                                                           pee.fetch_limit, sc);
    P2C_CUDA(cudaGetLastError());
  }
  finalize_queries_kernel<<<(unsigned)((n_queries + 127) / 128), 128, 0, s>>>(
      agg, n_queries, reinterpret_cast<const long long*>(pt_offsets_dev),
      reinterpret_cast<const long long*>(ee_offsets_dev), q_mask_dev, q_t1_dev, pt_results_dev, ee_results_dev,
      certs_dev);
  P2C_CUDA(cudaGetLastError());
  return export_stats(sc, stats_dev, s);
}

}  // extern "C"

// ---- work queues without allocation ----------------------------------------
// Some callers cannot call cudaMalloc: code that runs while a CUDA graph is
// being captured, physics or rendering loops that forbid allocation inside a
// frame, and host frameworks that own all device memory under a fixed budget.
// For them p2c_certify_queries_static keeps its scratch (the launch counters
// and one reduction record per work item) in the file-scope array below
// instead of a caller-provided workspace.
namespace p2c {
namespace {

constexpr size_t kStaticQueueScratchBytes = 1u << 20;  // 1 MiB per device, held until exit
static __device__ __align__(256) unsigned char g_static_queue_scratch[kStaticQueueScratchBytes];
static_assert(P2C_STATIC_QUEUE_MAX_QUERIES > 0, "capacity must be positive");
static_assert(queries_workspace_bytes_for(P2C_STATIC_QUEUE_MAX_QUERIES) <= kStaticQueueScratchBytes,
              "the stated maximum queue must fit the static scratch");

std::mutex g_static_mu;
void* g_static_ptr[64] = {};

// Device address of the array on the current device (the array's host-side
// name is only a stand-in for it).  It is resolved at the first call on a
// device and again at every later call made outside stream capture, so a
// device reset, which reloads the module and can move the array, never
// leaves a stale address behind; a call under capture uses the address of
// the last call made outside it.
int static_queue_scratch(cudaStream_t s, void** out) {
  int dev = 0;
  P2C_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(P2C_ERR_CUDA, "device ordinal %d out of range", dev);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  P2C_CUDA(cudaStreamIsCapturing(s, &cap));
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (g_static_ptr[dev] == nullptr || cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_queue_scratch);
    if (e != cudaSuccess) return fail(P2C_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_static_ptr[dev] = p;
  }
  *out = g_static_ptr[dev];
  return P2C_OK;
}

}  // namespace
}  // namespace p2c

extern "C" int p2c_certify_queries_static(const p2c_point_triangle* pt_dev, int64_t n_pt, const int64_t* pt_query_dev,
                                          const p2c_edge_edge* ee_dev, int64_t n_ee, const int64_t* ee_query_dev,
                                          int64_t n_queries, const int64_t* pt_offsets_dev,
                                          const int64_t* ee_offsets_dev, const double* q_t0_dev,
                                          const double* q_t1_dev, const uint32_t* q_mask_dev,
                                          const p2c_cert_config* config, p2c_interval_result* pt_results_dev,
                                          p2c_interval_result* ee_results_dev, p2c_query_certificate* certs_dev,
                                          p2c_certify_stats* stats_dev, void* stream) {
  if (n_queries > P2C_STATIC_QUEUE_MAX_QUERIES)
    return p2c::fail(P2C_ERR_INVALID,
                     "p2c_certify_queries_static takes at most %d work items per call (got %lld); split the queue "
                     "or use p2c_certify_queries with a workspace",
                     P2C_STATIC_QUEUE_MAX_QUERIES, (long long)n_queries);
  if (p2c::queries_workspace_bytes(n_queries) > p2c::kStaticQueueScratchBytes)
    return p2c::fail(P2C_ERR_INVALID, "static scratch too small for %lld work items", (long long)n_queries);
  void* scratch = nullptr;
  const int rc = p2c::static_queue_scratch(p2c::as_stream(stream), &scratch);
  if (rc != P2C_OK) return rc;
  // the existing entry point clears the counters and the per-item records
  // it needs at the start of every call
  return p2c_certify_queries(pt_dev, n_pt, pt_query_dev, ee_dev, n_ee, ee_query_dev, n_queries, pt_offsets_dev,
                             ee_offsets_dev, q_t0_dev, q_t1_dev, q_mask_dev, config, pt_results_dev, ee_results_dev,
                             certs_dev, scratch, p2c::kStaticQueueScratchBytes, stats_dev, stream);
}

