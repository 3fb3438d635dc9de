// scene.cu — certificates of scene candidate pairs, gathered straight from the
// vertex/face/edge arrays (no 240-byte records are built), with the
// CertificateEngine::Evaluate reduction and the on-device undecided queue.
#include "broadphase.cuh"
#include "certify_core.cuh"
#include "certify_launch.cuh"
#include "scene_agg.cuh"
#include "scene_pairs.cuh"

namespace p2c {
namespace {

// Scratch of a scene certification: the engine header and pools, then the
// scene reduction.
constexpr size_t kSceneAggOffset = kScratchHeaderBytes + kPoolBytes;
constexpr size_t kSceneScratchBytes = kSceneAggOffset + ((sizeof(SceneAgg) + 255) & ~size_t(255));

__host__ __device__ inline SceneAgg* scene_agg(void* ws) {
  return reinterpret_cast<SceneAgg*>(static_cast<char*>(ws) + kSceneAggOffset);
}

// Both families of a scene's candidate pairs over one interval; each result
// also feeds the scene reduction and, when undecided, the fallback queue.
struct PairProblem {
  ScenePairs sp[2];
  long long cap[2];
  const unsigned long long* counts;  // the broad phase's counts (device): n = min(count, cap)
  unsigned family_mask;
  p2c_interval_result* out[2];
  SceneAgg* agg;
  unsigned long long* undecided_queue;
  unsigned long long undecided_cap;
  unsigned long long* error_word;
  __device__ __forceinline__ long long n(int f) const {
    if ((family_mask & (1u << (f - 1))) == 0u) return 0;
    const long long c = (long long)counts[f - 1], k = pick(cap, f);
    return c < k ? c : k;
  }
  __device__ __forceinline__ bool skip(int, long long) const { return false; }
  __device__ __forceinline__ void load(int f, long long q, Geo& g, double& t0, double& t1, int& bad) const {
    const ScenePairs& s = pick(sp, f);
    bad = load_pair(s, f, __ldg(s.pairs + q), g) ? 0 : 2;
    t0 = s.T0;
    t1 = s.T1;
  }
  __device__ __forceinline__ void finish(int fam, long long q, const Outcome& o) const {
    const unsigned long long key = pick(sp, fam).pairs[q];
    store_interval_result(pick(out, fam) + q, fam, o, (long long)(key >> 32), (long long)(key & 0xffffffffull));
    scene_agg_record(agg, fam, key, o, undecided_queue, undecided_cap, nullptr,
                     ((unsigned long long)(fam - 1) << 63) | (unsigned long long)q);
  }
  __device__ __forceinline__ void invalid(int fam, long long q, int bad, double t0, double t1) const {
    Outcome o{3, t0, t1, t1, 0.0};
    store_interval_result(pick(out, fam) + q, fam, o, -1, -1);
    atomicOr(error_word, 4ull);
  }
};

__global__ void __launch_bounds__(kCertifyThreads, kCertifyMinBlocks)
    certify_scene_kernel(const __grid_constant__ PairProblem prob, const __grid_constant__ CertParams prm,
                         const __grid_constant__ EnginePools pools, CertifyScratch* scratch) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EngineShared& sh = reinterpret_cast<EngineShared*>(smem_raw)[threadIdx.x >> 5];
  WarpStats st;
  const unsigned long long t_start = global_ns();
  const long long n_vf = prob.n(1), n_ee = prob.n(2);
  // fetch width from the device-side sizes (the host did not see them)
  const long long warps = (long long)gridDim.x * kCertifyWarps;
  const int fetch_vf = (int)min(32ll, max(1ll, (n_vf + warps - 1) / warps));
  const int fetch_ee = (int)min(32ll, max(1ll, (n_ee + warps - 1) / warps));
  const bool ee_first = ((blockIdx.x * kCertifyWarps + (threadIdx.x >> 5)) & 1u) != 0u;
  const bool ok = run_engine<true, true, false>(prob, prm, fetch_vf, fetch_ee, ee_first, sh, st, &scratch->engine,
                                                pools, t_start);
  flush_stats(st, ok, scratch);
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    prob.agg->n_certified[0] = (unsigned long long)n_vf;
    prob.agg->n_certified[1] = (unsigned long long)n_ee;
    if ((long long)prob.counts[0] > prob.cap[0] || (long long)prob.counts[1] > prob.cap[1])
      atomicOr((unsigned long long*)&scratch->stats.error_word, 2ull);
  }
}

__global__ void init_scene_agg_kernel(SceneAgg* a) {
  pdl_trigger();  // the certification launch behind it may be scheduled now
  scene_agg_init(*a);
}

// CertificateEngine::Evaluate over (VF list, EE list) from the reduced flags;
// the collision witness is the candidate whose key won the atomicMin.
__global__ void scene_summary_kernel(const CertifyScratch* sc, const SceneAgg* agg, const unsigned long long* vf_pairs,
                                     const unsigned long long* ee_pairs, const p2c_interval_result* out_vf,
                                     const p2c_interval_result* out_ee, unsigned family_mask, double T1,
                                     p2c_scene_summary* summary) {
  pdl_wait();
  pdl_trigger();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  scene_witness(*agg, t, vf_pairs, ee_pairs, out_vf, out_ee, summary);
  if (t == 0) scene_summary_fields(*agg, family_mask, T1, sc->stats.error_word, summary);
}

__global__ void materialize_kernel(ScenePairs s, long long n, int family, unsigned long long* recs) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const unsigned long long key = s.pairs[q];
  const long long a = (long long)(key >> 32), b = (long long)(key & 0xffffffffull);
  long long v[4];
  if (family == 1) {
    v[0] = a;
    v[1] = s.faces[3 * b];
    v[2] = s.faces[3 * b + 1];
    v[3] = s.faces[3 * b + 2];
  } else {
    v[0] = s.edges[2 * a];
    v[1] = s.edges[2 * a + 1];
    v[2] = s.edges[2 * b];
    v[3] = s.edges[2 * b + 1];
  }
  unsigned long long* r = recs + 30 * q;
  r[0] = (unsigned long long)a;
  r[1] = (unsigned long long)b;
  for (int i = 0; i < 4; ++i) {
    unsigned long long* t = r + 2 + 7 * i;
    t[0] = (unsigned long long)v[i];
    for (int k = 0; k < 3; ++k) {
      t[1 + k] = (unsigned long long)__double_as_longlong(s.v_t0[3 * v[i] + k]);
      t[4 + k] = (unsigned long long)__double_as_longlong(s.v_t1[3 * v[i] + k]);
    }
  }
}

}  // namespace

int launch_scene_certify(const p2c_scene& scene, const unsigned long long* vf_pairs, long long vf_cap,
                         const unsigned long long* ee_pairs, long long ee_cap, const unsigned long long* counts,
                         double T0, double T1, const p2c_cert_config& cfg, unsigned family_mask,
                         p2c_interval_result* out_vf, p2c_interval_result* out_ee, unsigned long long* uq,
                         long long uq_cap, p2c_scene_summary* summary, void* ws, size_t ws_bytes,
                         cudaStream_t s) {
  if (ws == nullptr || ws_bytes < kSceneScratchBytes)
    return fail(P2C_ERR_INVALID, "scene certification workspace too small: %zu < %zu bytes", ws_bytes,
                kSceneScratchBytes);
  CertifyScratch* sc = reinterpret_cast<CertifyScratch*>(ws);
  P2C_CUDA(reset_scratch(sc, s, true));
  init_scene_agg_kernel<<<1, 1, 0, s>>>(scene_agg(ws));
  LaunchShape shape;
  int rc = certify_shape(certify_scene_kernel, &shape);
  if (rc != P2C_OK) return rc;
  const CertParams prm = make_params(cfg, shape, 32ll * shape.grid * kCertifyWarps);
  PairProblem prob;
  prob.sp[0] = ScenePairs{scene.v_t0, scene.v_t1, scene.faces, scene.edges, vf_pairs, T0, T1};
  prob.sp[1] = ScenePairs{scene.v_t0, scene.v_t1, scene.faces, scene.edges, ee_pairs, T0, T1};
  prob.cap[0] = vf_cap;
  prob.cap[1] = ee_cap;
  prob.counts = counts;
  prob.family_mask = family_mask;
  prob.out[0] = out_vf;
  prob.out[1] = out_ee;
  prob.agg = scene_agg(ws);
  prob.undecided_queue = uq;
  prob.undecided_cap = (unsigned long long)(uq_cap > 0 ? uq_cap : 0);
  prob.error_word = (unsigned long long*)&sc->stats.error_word;
  P2C_CUDA(launch_pdl(certify_scene_kernel, dim3(shape.grid), dim3(kCertifyThreads), shape.smem, s, prob, prm,
                      pools_at(sc), sc));
  if (summary != nullptr) {
    const long long nmax = (vf_cap > ee_cap ? vf_cap : ee_cap);
    const unsigned grid = (unsigned)((nmax + 255) / 256 > 0 ? (nmax + 255) / 256 : 1);
    P2C_CUDA(launch_pdl(scene_summary_kernel, dim3(grid), dim3(256), 0, s, sc, scene_agg(ws), vf_pairs, ee_pairs,
                        out_vf, out_ee, family_mask, T1, summary));
  }
  return P2C_OK;
}

int validate_scene(const p2c_scene* sc);

}  // namespace p2c

extern "C" {

size_t p2c_scene_certify_workspace_bytes(void) { return p2c::kSceneScratchBytes; }

int p2c_scene_certify(const p2c_scene* scene, const uint64_t* vf_pairs_dev, int64_t vf_cap,
                      const uint64_t* ee_pairs_dev, int64_t ee_cap, const uint64_t* counts_dev, double interval_t0,
                      double interval_t1, const p2c_cert_config* config, uint32_t family_mask,
                      p2c_interval_result* vf_results_dev, p2c_interval_result* ee_results_dev,
                      uint64_t* undecided_queue_dev, int64_t undecided_cap, p2c_scene_summary* summary_dev,
                      void* workspace_dev, size_t workspace_bytes, void* stream) {
  int rc = p2c::validate_scene(scene);
  if (rc != P2C_OK) return rc;
  if (config == nullptr) return p2c::fail(P2C_ERR_INVALID, "CertificateEngineConfig pointer is null");
  rc = p2c::validate_cert_config(*config, interval_t0, interval_t1);
  if (rc != P2C_OK) return rc;
  if (counts_dev == nullptr) return p2c::fail(P2C_ERR_INVALID, "counts pointer is null");
  if (family_mask == 0u || family_mask > 3u)
    return p2c::fail(P2C_ERR_INVALID, "ExactWorkItem.feature_family_mask is required");
  if ((vf_cap > 0 && (vf_pairs_dev == nullptr || vf_results_dev == nullptr)) ||
      (ee_cap > 0 && (ee_pairs_dev == nullptr || ee_results_dev == nullptr)))
    return p2c::fail(P2C_ERR_INVALID, "pair or result pointer is null");
  return p2c::launch_scene_certify(*scene, reinterpret_cast<const unsigned long long*>(vf_pairs_dev), vf_cap,
                                   reinterpret_cast<const unsigned long long*>(ee_pairs_dev), ee_cap,
                                   reinterpret_cast<const unsigned long long*>(counts_dev), interval_t0, interval_t1,
                                   *config, family_mask, vf_results_dev, ee_results_dev,
                                   reinterpret_cast<unsigned long long*>(undecided_queue_dev), undecided_cap,
                                   summary_dev, workspace_dev, workspace_bytes, p2c::as_stream(stream));
}

int p2c_scene_materialize(const p2c_scene* scene, const uint64_t* vf_pairs_dev, int64_t n_vf,
                          const uint64_t* ee_pairs_dev, int64_t n_ee, p2c_point_triangle* vf_records_dev,
                          p2c_edge_edge* ee_records_dev, void* stream) {
  int rc = p2c::validate_scene(scene);
  if (rc != P2C_OK) return rc;
  cudaStream_t s = p2c::as_stream(stream);
  if (n_vf > 0) {
    p2c::ScenePairs a{scene->v_t0, scene->v_t1, scene->faces, scene->edges,
                      reinterpret_cast<const unsigned long long*>(vf_pairs_dev), 0.0, 1.0};
    p2c::materialize_kernel<<<(unsigned)((n_vf + 255) / 256), 256, 0, s>>>(
        a, n_vf, 1, reinterpret_cast<unsigned long long*>(vf_records_dev));
  }
  if (n_ee > 0) {
    p2c::ScenePairs b{scene->v_t0, scene->v_t1, scene->faces, scene->edges,
                      reinterpret_cast<const unsigned long long*>(ee_pairs_dev), 0.0, 1.0};
    p2c::materialize_kernel<<<(unsigned)((n_ee + 255) / 256), 256, 0, s>>>(
        b, n_ee, 2, reinterpret_cast<unsigned long long*>(ee_records_dev));
  }
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

}  // extern "C"

#ifdef P2C_ENGINE_PROFILE
// Measurement build only: the engine phase clock of this file's kernels (see
// certify_engine.cuh), read and cleared by the host.
extern "C" int p2c_engine_profile_scene(unsigned long long* out16, int clear) {
  if (cudaMemcpyFromSymbol(out16, p2c::g_engine_prof, 16 * sizeof(unsigned long long)) != cudaSuccess) return 2;
  if (clear) {
    static const unsigned long long zero[16] = {};
    if (cudaMemcpyToSymbol(p2c::g_engine_prof, zero, sizeof(zero)) != cudaSuccess) return 2;
  }
  return 0;
}
#endif
