// batch.cu — many scenes of uneven size certified in one persistent launch.
//
// Each scene keeps its own candidate pairs (written by p2c_scene_candidates)
// and result buffers; a device table of p2c_batch_scene descriptors ties
// them together.  A prep kernel turns the per-scene counts into prefix
// offsets of two global queues (all scenes' VF pairs, then all their EE
// pairs); the engine's warps drain both queues as one problem, each query
// finding its scene by a binary search over the offsets, so a 1,000-triangle
// scene and a 200,000-triangle scene share the GPU with no per-scene launch.
// Certificates land in the scene's own result buffers, and each scene gets
// the CertificateEngine::Evaluate reduction (certificate_engine.cpp:729-824)
// of its own candidates, exactly as a single-scene certification writes it.
#include <cub/block/block_scan.cuh>

#include "certify_core.cuh"
#include "certify_launch.cuh"
#include "scene_agg.cuh"
#include "scene_pairs.cuh"

namespace p2c {
namespace {

static_assert(sizeof(p2c_batch_scene) == 152, "p2c_batch_scene layout");
static_assert(sizeof(p2c_batch_tuning) == 16, "p2c_batch_tuning layout");

constexpr int kPrepThreads = 1024;
constexpr int kMaxBatchScenes = 1 << 20;  // scene index fits the 24 bits above an undecided entry's position

struct BatchLayout {
  CertifyScratch* sc = nullptr;
  unsigned long long* off[2] = {nullptr, nullptr};  // n_scenes + 1 prefix offsets per family
  SceneAgg* aggs = nullptr;
  unsigned long long* uq_slots = nullptr;  // entries of the shared undecided queue (all scenes)
  size_t total = 0;
};

BatchLayout carve(void* base, long long n_scenes) {
  BatchLayout L;
  size_t off = 0;
  char* b = static_cast<char*>(base);
  auto take = [&](size_t bytes) -> void* {
    void* p = b == nullptr ? nullptr : b + off;
    off += (bytes + 255) & ~size_t(255);
    return p;
  };
  L.sc = static_cast<CertifyScratch*>(take(kScratchHeaderBytes + kPoolBytes));
  L.off[0] = static_cast<unsigned long long*>(take((size_t)(n_scenes + 1) * 8));
  L.off[1] = static_cast<unsigned long long*>(take((size_t)(n_scenes + 1) * 8));
  L.aggs = static_cast<SceneAgg*>(take((size_t)std::max(n_scenes, 1ll) * sizeof(SceneAgg)));
  L.uq_slots = static_cast<unsigned long long*>(take(sizeof(unsigned long long)));
  L.total = off;
  return L;
}

__device__ __forceinline__ long long scene_count(const p2c_batch_scene& d, int f, unsigned family_mask) {
  if ((family_mask & (1u << f)) == 0u) return 0;
  const long long c = (long long)d.counts[f];
  const long long cap = f == 0 ? d.vf_cap : d.ee_cap;
  return c < cap ? c : cap;
}

// Prefix offsets of both queues (one block, chunks of 1024 scenes) and the
// per-scene reductions' initial state.
__global__ void __launch_bounds__(kPrepThreads) batch_prep_kernel(const p2c_batch_scene* scenes, int n_scenes,
                                                                  unsigned family_mask, BatchLayout L) {
  using Scan = cub::BlockScan<unsigned long long, kPrepThreads>;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ unsigned long long carry[2];
  if (threadIdx.x < 2) carry[threadIdx.x] = 0ull;
  if (threadIdx.x == 0) *L.uq_slots = 0ull;
  __syncthreads();
  for (int base = 0; base < n_scenes; base += kPrepThreads) {
    const int s = base + (int)threadIdx.x;
    unsigned long long n[2] = {0ull, 0ull};
    if (s < n_scenes) {
      const p2c_batch_scene d = scenes[s];
      n[0] = (unsigned long long)scene_count(d, 0, family_mask);
      n[1] = (unsigned long long)scene_count(d, 1, family_mask);
      scene_agg_init(L.aggs[s]);
      L.aggs[s].n_certified[0] = n[0];
      L.aggs[s].n_certified[1] = n[1];
    }
    for (int f = 0; f < 2; ++f) {
      unsigned long long excl = 0ull, total = 0ull;
      Scan(tmp).ExclusiveSum(n[f], excl, total);
      if (s < n_scenes) L.off[f][s] = carry[f] + excl;
      __syncthreads();
      if (threadIdx.x == 0) carry[f] += total;
      __syncthreads();
    }
  }
  if (threadIdx.x < 2) L.off[threadIdx.x][n_scenes] = carry[threadIdx.x];
}

// Scene holding global queue position q of family f: the last s with
// off[s] <= q (scenes with no pairs share an offset with the next scene).
__device__ __forceinline__ int find_scene(const unsigned long long* off, int n_scenes, unsigned long long q) {
  int lo = 0, hi = n_scenes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= q) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct BatchProblem {
  const p2c_batch_scene* scenes;
  int n_scenes;
  const unsigned long long* off[2];  // prefix offsets written by the prep kernel
  SceneAgg* aggs;
  unsigned long long* uq;
  unsigned long long uq_cap;
  unsigned long long* uq_slots;  // one slot counter for every scene's entries
  unsigned long long* error_word;
  double T0, T1;
  __device__ __forceinline__ long long n(int f) const { return (long long)pick(off, f)[n_scenes]; }
  __device__ __forceinline__ bool skip(int, long long) const { return false; }
  __device__ __forceinline__ void locate(int f, long long q, int& s, long long& local) const {
    s = find_scene(pick(off, f), n_scenes, (unsigned long long)q);
    local = q - (long long)__ldg(pick(off, f) + s);
  }
  __device__ __forceinline__ void load(int f, long long q, Geo& g, double& t0, double& t1, int& bad) const {
    int s;
    long long local;
    locate(f, q, s, local);
    const p2c_batch_scene& d = scenes[s];
    const ScenePairs sp{d.v_t0, d.v_t1, d.faces, d.edges,
                        reinterpret_cast<const unsigned long long*>(f == 1 ? d.vf_pairs : d.ee_pairs), T0, T1};
    bad = load_pair(sp, f, __ldg(sp.pairs + local), g) ? 0 : 2;
    t0 = T0;
    t1 = T1;
  }
  __device__ __forceinline__ void finish(int f, long long q, const Outcome& o) const {
    int s;
    long long local;
    locate(f, q, s, local);
    const p2c_batch_scene& d = scenes[s];
    const unsigned long long key = (f == 1 ? d.vf_pairs : d.ee_pairs)[local];
    store_interval_result((f == 1 ? d.vf_results : d.ee_results) + local, f, o, (long long)(key >> 32),
                          (long long)(key & 0xffffffffull));
    scene_agg_record(aggs + s, f, key, o, uq, uq_cap, uq_slots,
                     ((unsigned long long)s << 40) | ((unsigned long long)(f - 1) << 39) | (unsigned long long)local);
  }
  __device__ __forceinline__ void invalid(int f, long long q, int, double t0, double t1) const {
    int s;
    long long local;
    locate(f, q, s, local);
    const p2c_batch_scene& d = scenes[s];
    Outcome o{3, t0, t1, t1, 0.0};
    store_interval_result((f == 1 ? d.vf_results : d.ee_results) + local, f, o, -1, -1);
    atomicOr(error_word, 4ull);
  }
};

__global__ void __launch_bounds__(kCertifyThreads, kCertifyMinBlocks)
    batch_certify_kernel(const __grid_constant__ BatchProblem prob, const __grid_constant__ CertParams prm,
                         int fixed_fetch, const __grid_constant__ EnginePools pools, CertifyScratch* sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EngineShared& sh = reinterpret_cast<EngineShared*>(smem_raw)[threadIdx.x >> 5];
  WarpStats st;
  const unsigned long long t_start = global_ns();
  const long long warps = (long long)gridDim.x * kCertifyWarps;
  int f1 = fixed_fetch, f2 = fixed_fetch;
  if (fixed_fetch <= 0) {
    f1 = (int)min(32ll, max(1ll, (prob.n(1) + warps - 1) / warps));
    f2 = (int)min(32ll, max(1ll, (prob.n(2) + warps - 1) / warps));
  }
  const bool ee_first = ((blockIdx.x * kCertifyWarps + (threadIdx.x >> 5)) & 1u) != 0u;
  const bool ok = run_engine<true, true, false>(prob, prm, f1, f2, ee_first, sh, st, &sc->engine, pools, t_start);
  flush_stats(st, ok, sc);
}

// Collision witnesses (grid-stride over both queues) and per-scene fields.
__global__ void batch_witness_kernel(const p2c_batch_scene* scenes, int n_scenes, BatchLayout L,
                                     p2c_scene_summary* summaries) {
  const unsigned long long tot0 = L.off[0][n_scenes], tot = tot0 + L.off[1][n_scenes];
  for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    const int f = t < tot0 ? 0 : 1;
    const unsigned long long q = f == 0 ? t : t - tot0;
    const int s = find_scene(L.off[f], n_scenes, q);
    const SceneAgg& a = L.aggs[s];
    if (a.coll_key == ~0ull || (int)(a.coll_key >> 63) != f) continue;
    const long long local = (long long)(q - L.off[f][s]);
    const p2c_batch_scene& d = scenes[s];
    scene_witness(a, local, reinterpret_cast<const unsigned long long*>(d.vf_pairs),
                  reinterpret_cast<const unsigned long long*>(d.ee_pairs), d.vf_results, d.ee_results, summaries + s);
  }
}

__global__ void batch_fields_kernel(int n_scenes, BatchLayout L, unsigned family_mask, double T1,
                                    p2c_scene_summary* summaries) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n_scenes) scene_summary_fields(L.aggs[s], family_mask, T1, L.sc->stats.error_word, summaries + s);
}

}  // namespace

int launch_batch_certify(const p2c_batch_scene* scenes, int n_scenes, double T0, double T1, const p2c_cert_config& cfg,
                         unsigned family_mask, p2c_scene_summary* summaries, unsigned long long* uq, long long uq_cap,
                         const p2c_batch_tuning& tune, void* ws, size_t ws_bytes, cudaStream_t s) {
  const BatchLayout need = carve(nullptr, n_scenes);
  if (ws == nullptr || ws_bytes < need.total)
    return fail(P2C_ERR_INVALID, "batch workspace too small: %zu < %zu bytes", ws_bytes, need.total);
  BatchLayout L = carve(ws, n_scenes);
  P2C_CUDA(reset_scratch(L.sc, s, true));
  batch_prep_kernel<<<1, kPrepThreads, 0, s>>>(scenes, n_scenes, family_mask, L);
  P2C_CUDA(cudaGetLastError());
  LaunchShape shape;
  int rc = certify_shape(batch_certify_kernel, &shape);
  if (rc != P2C_OK) return rc;
  if (tune.blocks_per_sm > 0) {
    DeviceInfo dev;
    rc = current_device_info(&dev);
    if (rc != P2C_OK) return rc;
    const int per_sm = shape.grid / std::max(dev.sm_count, 1);
    shape.grid = dev.sm_count * std::min(per_sm, (int)tune.blocks_per_sm);
  }
  const CertParams prm = make_params(cfg, shape, 32ll * shape.grid * kCertifyWarps);
  EnginePools pools = pools_at(L.sc);
  if (tune.helper_warps > 0) pools.helper_cap = (unsigned long long)tune.helper_warps;
  BatchProblem prob;
  prob.scenes = scenes;
  prob.n_scenes = n_scenes;
  prob.off[0] = L.off[0];
  prob.off[1] = L.off[1];
  prob.aggs = L.aggs;
  prob.uq = uq;
  prob.uq_cap = (unsigned long long)(uq_cap > 0 ? uq_cap : 0);
  prob.uq_slots = L.uq_slots;
  prob.error_word = (unsigned long long*)&L.sc->stats.error_word;
  prob.T0 = T0;
  prob.T1 = T1;
  batch_certify_kernel<<<shape.grid, kCertifyThreads, shape.smem, s>>>(prob, prm, tune.fetch_limit, pools, L.sc);
  P2C_CUDA(cudaGetLastError());
  if (summaries != nullptr) {
    batch_witness_kernel<<<shape.grid, 256, 0, s>>>(scenes, n_scenes, L, summaries);
    P2C_CUDA(cudaGetLastError());
    batch_fields_kernel<<<(n_scenes + 255) / 256, 256, 0, s>>>(n_scenes, L, family_mask, T1, summaries);
    P2C_CUDA(cudaGetLastError());
  }
  return P2C_OK;
}

}  // namespace p2c

extern "C" {

size_t p2c_batch_certify_workspace_bytes(int32_t n_scenes) {
  if (n_scenes < 1) return 0;
  return p2c::carve(nullptr, n_scenes).total;
}

int p2c_batch_certify(const p2c_batch_scene* scenes_dev, int32_t n_scenes, double interval_t0, double interval_t1,
                      const p2c_cert_config* config, uint32_t family_mask, p2c_scene_summary* summaries_dev,
                      uint64_t* undecided_queue_dev, int64_t undecided_cap, const p2c_batch_tuning* tuning,
                      void* workspace_dev, size_t workspace_bytes, void* stream) {
  if (scenes_dev == nullptr) return p2c::fail(P2C_ERR_INVALID, "scene table pointer is null");
  if (n_scenes < 1 || n_scenes > p2c::kMaxBatchScenes)
    return p2c::fail(P2C_ERR_INVALID, "batch scene count must lie in [1, %d]", p2c::kMaxBatchScenes);
  if (config == nullptr) return p2c::fail(P2C_ERR_INVALID, "CertificateEngineConfig pointer is null");
  int rc = p2c::validate_cert_config(*config, interval_t0, interval_t1);
  if (rc != P2C_OK) return rc;
  if (family_mask == 0u || family_mask > 3u)
    return p2c::fail(P2C_ERR_INVALID, "ExactWorkItem.feature_family_mask is required");
  p2c_batch_tuning tune{0, 0, 0, 0};
  if (tuning != nullptr) tune = *tuning;
  if (tune.blocks_per_sm < 0 || tune.fetch_limit < 0 || tune.fetch_limit > 32 || tune.helper_warps < 0)
    return p2c::fail(P2C_ERR_INVALID, "batch tuning out of range (fetch_limit <= 32, all non-negative)");
  return p2c::launch_batch_certify(scenes_dev, n_scenes, interval_t0, interval_t1, *config, family_mask,
                                   summaries_dev, reinterpret_cast<unsigned long long*>(undecided_queue_dev),
                                   undecided_cap, tune, workspace_dev, workspace_bytes, p2c::as_stream(stream));
}

}  // extern "C"

#ifdef P2C_ENGINE_PROFILE
// Measurement build only: the engine phase clock of this file's kernels (see
// certify_engine.cuh), read and cleared by the host.
extern "C" int p2c_engine_profile_batch(unsigned long long* out16, int clear) {
  if (cudaMemcpyFromSymbol(out16, p2c::g_engine_prof, 16 * sizeof(unsigned long long)) != cudaSuccess) return 2;
  if (clear) {
    static const unsigned long long zero[16] = {};
    if (cudaMemcpyToSymbol(p2c::g_engine_prof, zero, sizeof(zero)) != cudaSuccess) return 2;
  }
  return 0;
}
#endif
