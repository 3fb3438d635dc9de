// proxy.cu — candidates of a proxy scene (patch proxies in time slabs) on the
// device: GenerateRawCandidatesCpu + CompactRawCandidates
// (rt_candidate/candidate_buffer.cpp:144-227).
//
// The reference tests every proxy pair (O(n^2)).  Here:
//   1. two stable radix sorts order the proxies by (slab, min x);
//   2. a sweep: each proxy walks forward over its slab while the partner's
//      min x is within its max x, and emits the pairs of different objects
//      whose time intervals and inclusive AABBs overlap, as (lo << 32 | hi)
//      keys (each pair once, from the proxy earlier in sweep order);
//   3. one radix sort of the keys gives the reference's (i, j) hit order and
//      the 64-byte RawCandidateHit records are written from the keys;
//   4. three stable radix sorts of 64-bit key chunks order the hits by the
//      reference's compaction key (slab, first object, first patch, second
//      object, second patch, first type, second type), and the head of every
//      run writes one CandidateRecord (ids 1, 2, ... in key order) with the
//      run's hit count, the float maximum of its motion bounds and its flags.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>

#include "broadphase.cuh"
#include "p2c_internal.cuh"

namespace p2c {
namespace {

static_assert(sizeof(p2c_raw_candidate_hit) == 64, "RawCandidateHit layout");
static_assert(sizeof(p2c_candidate_record) == 80, "CandidateRecord layout");

constexpr int kThreads = 256;
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kHitFlags = 3u;  // kRawCandidateValid | kRawCandidateAabbOverlap

unsigned grid_for(long long n) {
  const long long b = (n + kThreads - 1) / kThreads;
  return (unsigned)(b > 0 ? b : 1);
}

int bit_length(unsigned long long x) {
  int b = 0;
  while (x) {
    ++b;
    x >>= 1;
  }
  return b;
}

struct ProxyLayout {
  unsigned long long* counter;   // [0] raw hits, [1] error word
  unsigned long long* xkey[2];   // n
  unsigned* slabkey[2];          // n
  unsigned* order[2];            // n
  double* s_minx;                // n, sorted order
  double* s_maxx;
  unsigned* s_slab;
  unsigned long long* pairs[2];  // raw_cap
  unsigned long long* ck[2];     // raw_cap: compaction key chunks
  unsigned* perm[2];             // raw_cap
  unsigned long long* gk[2];     // raw_cap: gathered key chunk and its sorted copy
  unsigned* head;                // raw_cap + 1
  unsigned* seg;                 // raw_cap + 1
  void* tmp;
  size_t tmp_bytes;
  size_t total;
};

size_t temp_bytes(long long n, long long cap) {
  const int nn = (int)std::max(n, 1ll), cc = (int)std::max(cap, 1ll);
  size_t a = 0, b = 0, c = 0, d = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, a, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (const unsigned*)nullptr, (unsigned*)nullptr, std::max(nn, cc));
  cub::DeviceRadixSort::SortPairs(nullptr, b, (const unsigned*)nullptr, (unsigned*)nullptr, (const unsigned*)nullptr,
                                  (unsigned*)nullptr, nn);
  cub::DeviceRadixSort::SortKeys(nullptr, c, (const unsigned long long*)nullptr, (unsigned long long*)nullptr, cc);
  cub::DeviceScan::ExclusiveSum(nullptr, d, (const unsigned*)nullptr, (unsigned*)nullptr, cc + 1);
  return std::max(std::max(a, b), std::max(c, d));
}

ProxyLayout carve(void* base, long long n, long long cap) {
  ProxyLayout L{};
  size_t off = 0;
  char* b = static_cast<char*>(base);
  auto take = [&](size_t bytes) -> void* {
    void* p = b == nullptr ? nullptr : b + off;
    off += (std::max<size_t>(bytes, 1) + 255) & ~size_t(255);
    return p;
  };
  const size_t N = (size_t)std::max(n, 1ll), C = (size_t)std::max(cap, 1ll);
  L.counter = static_cast<unsigned long long*>(take(16));
  for (int k = 0; k < 2; ++k) {
    L.xkey[k] = static_cast<unsigned long long*>(take(8 * N));
    L.slabkey[k] = static_cast<unsigned*>(take(4 * N));
    L.order[k] = static_cast<unsigned*>(take(4 * N));
    L.pairs[k] = static_cast<unsigned long long*>(take(8 * C));
    L.ck[k] = static_cast<unsigned long long*>(take(8 * C));
    L.perm[k] = static_cast<unsigned*>(take(4 * C));
    L.gk[k] = static_cast<unsigned long long*>(take(8 * C));
  }
  L.s_minx = static_cast<double*>(take(8 * N));
  L.s_maxx = static_cast<double*>(take(8 * N));
  L.s_slab = static_cast<unsigned*>(take(4 * N));
  L.head = static_cast<unsigned*>(take(4 * (C + 1)));
  L.seg = static_cast<unsigned*>(take(4 * (C + 1)));
  L.tmp_bytes = temp_bytes(n, cap);
  L.tmp = take(L.tmp_bytes);
  L.total = off;
  return L;
}

// ValidateProxyScene's per-proxy checks (rt_candidate/proxy_scene.cpp:143-151:
// concrete type, finite t0 < t1, finite bounds with min <= max) and the x sort
// key.  Proxy ids (the array index here) and the global slab partition
// (:58-85) are checked by the host, which holds one interval per slab.
__global__ void keys_kernel(p2c_proxy_scene sc, ProxyLayout L) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sc.n) return;
  const double* b = sc.bounds + 6 * i;
  bool ok = (sc.proxy_type[i] == 1 || sc.proxy_type[i] == 2) && isfinite(sc.t0[i]) && isfinite(sc.t1[i]) &&
            sc.t0[i] < sc.t1[i];
  for (int a = 0; a < 3; ++a) ok = ok && isfinite(b[a]) && isfinite(b[3 + a]) && !(b[a] > b[3 + a]);
  if (!ok) atomicOr(L.counter + 1, 1ull);
  L.xkey[0][i] = order_key(b[0]);
  L.order[0][i] = (unsigned)i;
}

__global__ void slab_keys_kernel(p2c_proxy_scene sc, ProxyLayout L) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < sc.n) L.slabkey[0][p] = sc.slab_id[L.order[1][p]];
}

__global__ void gather_kernel(p2c_proxy_scene sc, ProxyLayout L) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= sc.n) return;
  const unsigned i = L.order[0][p];
  L.s_minx[p] = sc.bounds[6 * (long long)i];
  L.s_maxx[p] = sc.bounds[6 * (long long)i + 3];
  L.s_slab[p] = sc.slab_id[i];
}

__global__ void fill_kernel(unsigned long long* p, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = ~0ull;
}

// Sweep over the proxies sorted by (slab, min x); the tests are
// GenerateRawCandidatesCpu's (:158-173: different objects, same slab,
// TimeOverlap, AabbOverlap).
__global__ void sweep_kernel(p2c_proxy_scene sc, ProxyLayout L, unsigned long long cap) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = sc.n;
  bool live = p < n;
  unsigned i = 0, slab = 0, obj = 0;
  double maxx = 0.0, t0 = 0.0, t1 = 0.0, b[6] = {0, 0, 0, 0, 0, 0};
  if (live) {
    i = L.order[0][p];
    slab = L.s_slab[p];
    maxx = L.s_maxx[p];
    obj = sc.object_id[i];
    t0 = sc.t0[i];
    t1 = sc.t1[i];
    for (int a = 0; a < 6; ++a) b[a] = sc.bounds[6 * (long long)i + a];
  }
  long long q = p + 1;
  for (;;) {
    if (live && (q >= n || L.s_slab[q] != slab || L.s_minx[q] > maxx)) live = false;
    if (!__any_sync(kFull, live)) break;
    bool found = false;
    unsigned long long key = 0;
    if (live) {
      const unsigned j = L.order[0][q];
      if (sc.object_id[j] != obj && t0 < sc.t1[j] && sc.t0[j] < t1) {
        const double* c = sc.bounds + 6 * (long long)j;
        bool ov = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) ov = ov && !(b[3 + a] < c[a] || c[3 + a] < b[a]);
        if (ov) {
          found = true;
          key = ((unsigned long long)min(i, j) << 32) | (unsigned long long)max(i, j);
        }
      }
      ++q;
    }
    const unsigned mask = __ballot_sync(kFull, found);
    if (mask) {
      const int lane = threadIdx.x & 31, leader = __ffs((int)mask) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(L.counter, (unsigned long long)__popc(mask));
      base = __shfl_sync(kFull, base, leader);
      if (found) {
        const unsigned long long slot = base + (unsigned long long)__popc(mask & ((1u << lane) - 1u));
        if (slot < cap) L.pairs[0][slot] = key;
      }
    }
  }
}

// static_cast<float>(std::max(lhs, rhs)) with IEEE round to nearest: a double
// beyond the float range becomes infinity.  The intrinsic keeps that defined
// (a plain cast of an out-of-range value is undefined behaviour in C++, which
// lets the optimiser assume the float stays finite).
__device__ __forceinline__ float merged_bound(const double* a, const double* b, int k) {
  return __double2float_rn(a[k] < b[k] ? b[k] : a[k]);
}

// finite and not below zero (ValidateRawHit), on the bits of the float
__device__ __forceinline__ bool bound_valid(float v) {
  return (__float_as_uint(v) & 0x7f800000u) != 0x7f800000u && !(v < 0.0f);
}

// Raw hit records in (i, j) order, and the compaction key chunks of each hit
// (MakeCandidateKey, :104-124: the first proxy is the smaller (object, patch,
// proxy) tuple).
__global__ void raw_hits_kernel(p2c_proxy_scene sc, ProxyLayout L, const unsigned long long* sorted,
                                unsigned long long cap, p2c_raw_candidate_hit* raw) {
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= (long long)cap) return;
  const unsigned long long k = sorted[h];
  L.perm[0][h] = (unsigned)h;
  if (k == ~0ull) {  // past the hits: sorts last in every pass
    L.ck[0][h] = ~0ull;
    L.ck[1][h] = ~0ull;
    L.pairs[0][h] = ~0ull;
    return;
  }
  const unsigned i = (unsigned)(k >> 32), j = (unsigned)(k & 0xffffffffull);
  const double* ma = sc.motion_bound + 4 * (long long)i;
  const double* mb = sc.motion_bound + 4 * (long long)j;
  p2c_raw_candidate_hit r{};
  r.query_id = sc.query_id;
  r.pair_key = k;
  r.proxy_a_index = i;
  r.proxy_b_index = j;
  r.slab_id = sc.slab_id[i];
  r.rt_hit_count = 1u;
  r.flags = kHitFlags;
  bool bound_ok = true;
  for (int c = 0; c < 4; ++c) {
    r.motion_bound[c] = merged_bound(ma, mb, c);
    bound_ok = bound_ok && bound_valid(r.motion_bound[c]);
  }
  // ValidateRawHit (:95-99), which CompactRawCandidates applies to every hit
  if (!bound_ok) atomicOr(L.counter + 1, 2ull);
  raw[h] = r;
  // first / second proxy by (object, patch, proxy id)
  unsigned fo = sc.object_id[i], fp = sc.patch_id[i], so = sc.object_id[j], sp = sc.patch_id[j];
  unsigned ft = sc.proxy_type[i], st = sc.proxy_type[j];
  const bool swap = fo > so || (fo == so && (fp > sp || (fp == sp && i > j)));
  if (swap) {
    unsigned t = fo;
    fo = so;
    so = t;
    t = fp;
    fp = sp;
    sp = t;
    t = ft;
    ft = st;
    st = t;
  }
  // three chunks, most significant last: (slab, fo) (fp, so) (sp, ft, st)
  L.ck[0][h] = ((unsigned long long)sp << 16) | ((unsigned long long)ft << 8) | st;
  L.ck[1][h] = ((unsigned long long)fp << 32) | so;
  L.pairs[0][h] = ((unsigned long long)r.slab_id << 32) | fo;  // third chunk (the raw keys moved to pairs[1])
}

__global__ void gather_chunk_kernel(const unsigned long long* chunk, const unsigned* perm, unsigned long long* out,
                                    long long cap) {
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (h < cap) out[h] = chunk[perm[h]];
}

// Run heads of the compaction key over the hits in key order.
__global__ void heads_kernel(ProxyLayout L, const unsigned* perm, const unsigned long long* k0,
                             const unsigned long long* k1, const unsigned long long* k2, long long cap) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p > cap) return;
  const long long n_hits = (long long)min(L.counter[0], (unsigned long long)cap);
  unsigned hd = 0u;
  if (p < n_hits && p < cap) {
    const unsigned a = perm[p];
    hd = p == 0 ? 1u : 0u;
    if (p > 0) {
      const unsigned b = perm[p - 1];
      hd = (k0[a] != k0[b] || k1[a] != k1[b] || k2[a] != k2[b]) ? 1u : 0u;
    }
  }
  L.head[p] = hd;
}

__global__ void records_kernel(p2c_proxy_scene sc, ProxyLayout L, const unsigned* perm,
                               const p2c_raw_candidate_hit* raw, const unsigned long long* k0,
                               const unsigned long long* k1, const unsigned long long* k2, long long cap,
                               p2c_candidate_record* out, unsigned long long* counts) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n_hits = (long long)min(L.counter[0], (unsigned long long)cap);
  if (p == 0) {
    counts[0] = L.counter[0];
    counts[1] = n_hits > 0 ? L.seg[n_hits] : 0ull;  // seg is unwritten when the capacity is 0
    counts[2] = L.counter[1] | (L.counter[0] > (unsigned long long)n_hits ? 4ull : 0ull);
  }
  if (p >= n_hits || !L.head[p]) return;
  const unsigned a = perm[p];
  p2c_candidate_record r{};
  r.schema_version = 1u;
  r.candidate_id = (unsigned long long)L.seg[p] + 1ull;
  r.query_id = sc.query_id;
  r.slab_id = (unsigned)(k2[a] >> 32);
  r.object_a_id = (unsigned)(k2[a] & 0xffffffffull);
  r.patch_a_id = (unsigned)(k1[a] >> 32);
  r.object_b_id = (unsigned)(k1[a] & 0xffffffffull);
  r.patch_b_id = (unsigned)(k0[a] >> 16);
  r.proxy_type_a = (uint8_t)((k0[a] >> 8) & 0xffull);
  r.proxy_type_b = (uint8_t)(k0[a] & 0xffull);
  unsigned count = 0u, flags = 0u;
  float mb[4] = {0.f, 0.f, 0.f, 0.f};
  for (long long q = p; q < n_hits && (q == p || !L.head[q]); ++q) {
    const p2c_raw_candidate_hit& h = raw[perm[q]];
    if (q == p) {
      for (int c = 0; c < 4; ++c) mb[c] = h.motion_bound[c];
    } else {
      for (int c = 0; c < 4; ++c) mb[c] = mb[c] < h.motion_bound[c] ? h.motion_bound[c] : mb[c];  // std::max
    }
    count += h.rt_hit_count;
    flags |= h.flags;
  }
  r.rt_hit_count = count;
  for (int c = 0; c < 4; ++c) r.motion_bound[c] = mb[c];
  r.proxy_features_offset = 0u;
  r.flags = flags;
  out[r.candidate_id - 1] = r;
}

}  // namespace
}  // namespace p2c

extern "C" {

size_t p2c_proxy_candidates_workspace_bytes(int64_t n_proxies, int64_t raw_cap) {
  if (n_proxies < 0 || raw_cap < 0) return 0;
  return p2c::carve(nullptr, n_proxies, raw_cap).total + 256;
}

int p2c_proxy_candidates(const p2c_proxy_scene* scene, p2c_raw_candidate_hit* raw_dev, int64_t raw_cap,
                         p2c_candidate_record* candidates_dev, uint64_t* counts_dev, void* workspace_dev,
                         size_t workspace_bytes, void* stream) {
  using namespace p2c;
  if (scene == nullptr) return fail(P2C_ERR_INVALID, "proxy scene pointer is null");
  if (scene->query_id == 0) return fail(P2C_ERR_INVALID, "ProxyScene.query_id is required");
  if (scene->n < 0 || scene->n >= (1ll << 31)) return fail(P2C_ERR_INVALID, "proxy count must lie in [0, 2^31)");
  if (raw_cap < 0 || raw_cap >= (1ll << 31)) return fail(P2C_ERR_INVALID, "raw capacity must lie in [0, 2^31)");
  if (counts_dev == nullptr) return fail(P2C_ERR_INVALID, "counts pointer is null");
  if (raw_cap > 0 && (raw_dev == nullptr || candidates_dev == nullptr))
    return fail(P2C_ERR_INVALID, "raw hit or candidate output pointer is null");
  const long long n = scene->n;
  if (n > 0 && (scene->object_id == nullptr || scene->patch_id == nullptr || scene->slab_id == nullptr ||
                scene->proxy_type == nullptr || scene->t0 == nullptr || scene->t1 == nullptr ||
                scene->bounds == nullptr || scene->motion_bound == nullptr))
    return fail(P2C_ERR_INVALID, "proxy scene arrays are null");
  const size_t need = carve(nullptr, n, raw_cap).total;
  if (workspace_dev == nullptr || workspace_bytes < need)
    return fail(P2C_ERR_INVALID, "proxy candidate workspace too small: %zu < %zu bytes", workspace_bytes, need);
  ProxyLayout L = carve(workspace_dev, n, raw_cap);
  cudaStream_t s = as_stream(stream);
  const p2c_proxy_scene sc = *scene;
  const long long cap = raw_cap;
  P2C_CUDA(cudaMemsetAsync(L.counter, 0, 16, s));
  if (n > 0) {
    keys_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L);
    size_t tb = L.tmp_bytes;
    // (slab, min x): stable sort by min x, then stable sort by slab
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.xkey[0], L.xkey[1], L.order[0], L.order[1], (int)n, 0, 64,
                                             s));
    slab_keys_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L);
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.slabkey[0], L.slabkey[1], L.order[1], L.order[0], (int)n,
                                             0, 32, s));
    gather_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L);
  }
  if (cap > 0) fill_kernel<<<grid_for(cap), kThreads, 0, s>>>(L.pairs[0], cap);
  // the sweep counts every hit, also past the capacity (writes only below it)
  if (n > 0) sweep_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L, (unsigned long long)cap);
  if (cap > 0) {
    size_t tb = L.tmp_bytes;
    const int pair_bits = 32 + std::max(1, bit_length((unsigned long long)std::max(n - 1, 1ll)));
    // the hits in (i, j) order
    P2C_CUDA(cub::DeviceRadixSort::SortKeys(L.tmp, tb, L.pairs[0], L.pairs[1], (int)cap, 0,
                                            std::min(64, pair_bits), s));
    raw_hits_kernel<<<grid_for(cap), kThreads, 0, s>>>(sc, L, L.pairs[1], (unsigned long long)cap, raw_dev);
    P2C_CUDA(cudaGetLastError());
    // compaction key order: stable sorts by the chunks, least significant first
    const unsigned long long* chunk[3] = {L.ck[0], L.ck[1], L.pairs[0]};
    unsigned* perm_in = L.perm[0];
    unsigned* perm_out = L.perm[1];
    for (int c = 0; c < 3; ++c) {
      gather_chunk_kernel<<<grid_for(cap), kThreads, 0, s>>>(chunk[c], perm_in, L.gk[0], cap);
      tb = L.tmp_bytes;
      P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.gk[0], L.gk[1], perm_in, perm_out, (int)cap, 0, 64, s));
      std::swap(perm_in, perm_out);
    }
    heads_kernel<<<grid_for(cap + 1), kThreads, 0, s>>>(L, perm_in, chunk[0], chunk[1], chunk[2], cap);
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceScan::ExclusiveSum(L.tmp, tb, L.head, L.seg, (int)(cap + 1), s));
    records_kernel<<<grid_for(cap), kThreads, 0, s>>>(sc, L, perm_in, raw_dev, chunk[0], chunk[1], chunk[2], cap,
                                                      candidates_dev, reinterpret_cast<unsigned long long*>(counts_dev));
    P2C_CUDA(cudaGetLastError());
  } else {
    records_kernel<<<1, kThreads, 0, s>>>(sc, L, L.perm[0], raw_dev, L.ck[0], L.ck[1], L.pairs[0], 0, candidates_dev,
                                          reinterpret_cast<unsigned long long*>(counts_dev));
    P2C_CUDA(cudaGetLastError());
  }
  return P2C_OK;
}

}  // extern "C"
