// broadphase.cu — swept-AABB candidate generation by sweep-and-prune.
//
// Replaces the reference's CPU candidate builders: the brute-force
// BuildMeshExactCertificateQuery pair loops (cpp/certificate/
// mesh_exact_query.cpp:211-317) and the scene tool's SweepPairs /
// BuildVFCandidates / BuildEECandidates (tools/
// scene_object_envelope_native_ti_walltime.cpp:603-699).  The pair SET is
// identical: inclusive double-precision overlap on all three axes, no vertex
// against a face that contains it and no edges sharing a vertex inside one
// object, optionally no pairs inside one object at all.
//
// Steps (all on the caller's stream, no host synchronisation):
//   1. swept boxes of vertices, edges, faces (t0 and t1 positions, +thickness)
//      with per-axis statistics;
//   2. the sweep axis is chosen on the device: smallest mean box extent
//      relative to the spread of box centres;
//   3. CUB radix sort of the box minima along that axis (64-bit
//      order-preserving keys), gather into struct-of-arrays in sorted order;
//   4. sweeps: vertex-face as two bipartite passes (each pair found once:
//      from the vertex when the face minimum is >= the vertex minimum, else
//      from the face), edge-edge as one forward scan over the sorted list;
//      overlapping pairs are compacted per warp with a ballot and appended with
//      one atomic per warp.
// The object-pair permission of the scene tool (PrepareScene, :521-545) needs
// no separate pass: a primitive box lies inside its object's box (same
// vertices, same thickness), so two overlapping primitive boxes of different
// objects imply overlapping object boxes; only the same-object rule remains.
#include <cub/device/device_radix_sort.cuh>

#include "broadphase.cuh"

namespace p2c {
namespace {

constexpr int kBoxThreads = 256;
constexpr int kSweepThreads = 256;

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }  // std::max

// Swept box of primitive i made of K vertices (K = 1 vertex, 2 edge, 3 face).
template <int K>
__global__ void __launch_bounds__(kBoxThreads) boxes_kernel(const double* __restrict__ v_t0,
                                                            const double* __restrict__ v_t1,
                                                            const int32_t* __restrict__ prim, long long n,
                                                            double thickness, double* __restrict__ box,
                                                            BroadScratch* sc) {
  __shared__ double red[9][kBoxThreads / 32];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double ext[3] = {0, 0, 0}, cen[3] = {0, 0, 0}, cen2[3] = {0, 0, 0};
  unsigned long long cnt = 0;
  if (i < n) {
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    bool finite = true;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const long long v = K == 1 ? i : (long long)__ldg(prim + K * i + k);
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        const double* p = (f == 0 ? v_t0 : v_t1) + 3 * v;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double x = __ldg(p + a);
          finite = finite && isfinite(x);
          mn[a] = dmin(mn[a], x);
          mx[a] = dmax(mx[a], x);
        }
      }
    }
    double* b = box + 6 * i;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      b[a] = __dsub_rn(mn[a], thickness);
      b[3 + a] = __dadd_rn(mx[a], thickness);
      ext[a] = b[3 + a] - b[a];
      cen[a] = 0.5 * (b[3 + a] + b[a]);
      cen2[a] = cen[a] * cen[a];
    }
    cnt = 1;
    if (!finite) atomicOr(&sc->error_word, 1ull);
  }
  // block reduction of the axis statistics
  double vals[9] = {ext[0], ext[1], ext[2], cen[0], cen[1], cen[2], cen2[0], cen2[1], cen2[2]};
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    double v = vals[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
  }
  unsigned long long c = cnt;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  __syncthreads();
  if (threadIdx.x < 9) {
    double s = 0.0;
    for (int w = 0; w < kBoxThreads / 32; ++w) s += red[threadIdx.x][w];
    double* dst = threadIdx.x < 3 ? &sc->stats.extent_sum[threadIdx.x]
                  : threadIdx.x < 6 ? &sc->stats.center_sum[threadIdx.x - 3]
                                    : &sc->stats.center_sq_sum[threadIdx.x - 6];
    atomicAdd(dst, s);
  }
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(&sc->stats.count, c);
}

// Sweep axis: the one whose mean box extent is smallest relative to the
// standard deviation of box centres (fewest boxes overlap along it).
__device__ __forceinline__ int choose_axis(const AxisStats& st) {
  const double n = st.count > 0 ? (double)st.count : 1.0;
  int best = 0;
  double best_score = INFINITY;
  for (int a = 0; a < 3; ++a) {
    const double mean = st.center_sum[a] / n;
    const double var = fmax(st.center_sq_sum[a] / n - mean * mean, 0.0);
    const double score = (st.extent_sum[a] / n) / (sqrt(var) + 1e-300);
    if (score < best_score) {
      best_score = score;
      best = a;
    }
  }
  return best;
}

// Keys for one list; valid == nullptr keeps every primitive, otherwise
// primitives with valid[i] < 0 sort to the end with key ~0 and are skipped.
__global__ void __launch_bounds__(kBoxThreads) keys_kernel(const double* __restrict__ box, long long n,
                                                           const int32_t* __restrict__ skip_if_negative,
                                                           unsigned long long* __restrict__ keys,
                                                           unsigned int* __restrict__ vals, BroadScratch* sc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int axis = choose_axis(sc->stats);
  if (i == 0 && blockIdx.x == 0) sc->stats.axis = axis;
  const bool skip = skip_if_negative != nullptr && skip_if_negative[i] < 0;
  keys[i] = skip ? ~0ull : order_key(box[6 * i + axis]);
  vals[i] = (unsigned int)i;
}

__global__ void __launch_bounds__(kBoxThreads) gather_kernel(const double* __restrict__ box, long long n,
                                                             const int32_t* __restrict__ skip_if_negative,
                                                             const unsigned int* __restrict__ order,
                                                             const int32_t* __restrict__ obj, SortedBoxes s,
                                                             const BroadScratch* sc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int axis = choose_axis(sc->stats);
  const int a1 = axis == 0 ? 1 : 0;
  const int a2 = axis == 2 ? 1 : 2;
  const unsigned int j = order[i];
  if (skip_if_negative != nullptr && skip_if_negative[j] < 0) {
    // skipped entries (vertices in no face) sorted last: keep lo monotonic
    s.lo[i] = INFINITY;
    s.hi[i] = -INFINITY;
    s.alo[i] = INFINITY;
    s.ahi[i] = -INFINITY;
    s.blo[i] = INFINITY;
    s.bhi[i] = -INFINITY;
    s.id[i] = (int32_t)j;
    s.obj[i] = -1;
    return;
  }
  const double* b = box + 6 * (long long)j;
  s.lo[i] = b[axis];
  s.hi[i] = b[3 + axis];
  s.alo[i] = b[a1];
  s.ahi[i] = b[3 + a1];
  s.blo[i] = b[a2];
  s.bhi[i] = b[3 + a2];
  s.id[i] = (int32_t)j;
  s.obj[i] = obj[j];
}

// Warp-aggregated append of the pairs found by this iteration.
__device__ __forceinline__ void append_pair(bool found, unsigned long long key, unsigned long long* out,
                                            unsigned long long cap, unsigned long long* count) {
  const unsigned mask = __ballot_sync(0xffffffffu, found);
  if (mask == 0u) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs((int)mask) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (found) {
    const unsigned long long slot = base + (unsigned long long)__popc(mask & ((1u << lane) - 1u));
    if (slot < cap) out[slot] = key;
  }
}

__device__ __forceinline__ long long lower_bound_ge(const double* a, long long n, double x) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long m = (lo + hi) >> 1;
    if (a[m] < x) lo = m + 1;
    else hi = m;
  }
  return lo;
}
__device__ __forceinline__ long long upper_bound_gt(const double* a, long long n, double x) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long m = (lo + hi) >> 1;
    if (a[m] <= x) lo = m + 1;
    else hi = m;
  }
  return lo;
}

__device__ __forceinline__ bool overlap_other_axes(const SortedBoxes& p, long long i, const SortedBoxes& q,
                                                   long long j) {
  return p.alo[i] <= q.ahi[j] && q.alo[j] <= p.ahi[i] && p.blo[i] <= q.bhi[j] && q.blo[j] <= p.bhi[i];
}

// Vertex-face: threads [0, nv) scan faces from each vertex, threads
// [nv, nv + nf) scan vertices from each face.  Keys are (vertex << 32 | face).
__global__ void __launch_bounds__(kSweepThreads) sweep_vf_kernel(SortedBoxes V, long long nv, SortedBoxes F,
                                                                 long long nf, const int32_t* __restrict__ faces,
                                                                 int exclude_self, unsigned long long* out,
                                                                 unsigned long long cap, BroadScratch* sc) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool from_vertex = t < nv;
  const long long i = from_vertex ? t : t - nv;
  bool live = from_vertex ? (t < nv) : (i < nf);
  // the caller sorted skipped vertices (object < 0) to the end
  if (live && from_vertex && V.obj[i] < 0) live = false;
  const SortedBoxes P = from_vertex ? V : F;  // this thread's box
  const SortedBoxes Q = from_vertex ? F : V;  // the list it scans
  const long long nq = from_vertex ? nf : nv;
  long long j = 0;
  double hi = 0.0;
  if (live) {
    hi = P.hi[i];
    j = from_vertex ? lower_bound_ge(Q.lo, nq, P.lo[i]) : upper_bound_gt(Q.lo, nq, P.lo[i]);
  }
  const int32_t pid = live ? P.id[i] : 0, pobj = live ? P.obj[i] : 0;
  for (;;) {
    const bool active = live && j < nq && Q.lo[j] <= hi;
    if (!__any_sync(0xffffffffu, active)) break;
    bool found = false;
    unsigned long long key = 0;
    if (active) {
      const int32_t qobj = Q.obj[j];
      if (qobj >= 0 && P.lo[i] <= Q.hi[j] && overlap_other_axes(P, i, Q, j)) {
        const int32_t vtx = from_vertex ? pid : Q.id[j];
        const int32_t fc = from_vertex ? Q.id[j] : pid;
        bool ok = true;
        if (pobj == qobj) {
          if (exclude_self) ok = false;
          else {
            const int32_t* fv = faces + 3 * (long long)fc;
            ok = !(__ldg(fv) == vtx || __ldg(fv + 1) == vtx || __ldg(fv + 2) == vtx);
          }
        }
        if (ok) {
          found = true;
          key = ((unsigned long long)(unsigned)vtx << 32) | (unsigned)fc;
        }
      }
      ++j;
    }
    append_pair(found, key, out, cap, &sc->vf_count);
  }
}

// Edge-edge: each edge scans forward over the sorted list; keys are
// (min edge << 32 | max edge).
__global__ void __launch_bounds__(kSweepThreads) sweep_ee_kernel(SortedBoxes E, long long ne,
                                                                 const int32_t* __restrict__ edges, int exclude_self,
                                                                 unsigned long long* out, unsigned long long cap,
                                                                 BroadScratch* sc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < ne;
  double hi = 0.0;
  int32_t eid = 0, eobj = 0, a0 = 0, a1 = 0;
  if (live) {
    hi = E.hi[i];
    eid = E.id[i];
    eobj = E.obj[i];
    a0 = __ldg(edges + 2 * (long long)eid);
    a1 = __ldg(edges + 2 * (long long)eid + 1);
  }
  long long j = i + 1;
  for (;;) {
    const bool active = live && j < ne && E.lo[j] <= hi;
    if (!__any_sync(0xffffffffu, active)) break;
    bool found = false;
    unsigned long long key = 0;
    if (active) {
      if (overlap_other_axes(E, i, E, j)) {
        const int32_t oid = E.id[j];
        bool ok = true;
        if (E.obj[j] == eobj) {
          if (exclude_self) ok = false;
          else {
            const int32_t b0 = __ldg(edges + 2 * (long long)oid), b1 = __ldg(edges + 2 * (long long)oid + 1);
            ok = !(a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1);
          }
        }
        if (ok) {
          found = true;
          const unsigned lo = (unsigned)min(eid, oid), hi2 = (unsigned)max(eid, oid);
          key = ((unsigned long long)lo << 32) | hi2;
        }
      }
      ++j;
    }
    append_pair(found, key, out, cap, &sc->ee_count);
  }
}

__global__ void fill_u64_kernel(unsigned long long* p, long long n, unsigned long long v) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

__global__ void export_counts_kernel(const BroadScratch* sc, unsigned long long* counts) {
  counts[0] = sc->vf_count;
  counts[1] = sc->ee_count;
  counts[2] = sc->error_word;
  counts[3] = (unsigned long long)sc->stats.axis;
}

inline unsigned grid_for(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// ---- workspace carving -----------------------------------------------------
struct Carver {
  char* base;
  size_t off = 0;
  bool dry;
  template <class T>
  T* take(long long count) {
    off = (off + 255) & ~size_t(255);
    T* p = dry ? nullptr : reinterpret_cast<T*>(base + off);
    off += sizeof(T) * (size_t)(count > 0 ? count : 1);
    return p;
  }
};

size_t sort_temp_bytes(long long n) {
  size_t bytes = 0;
  cub::DoubleBuffer<unsigned long long> k(nullptr, nullptr);
  cub::DoubleBuffer<unsigned int> v(nullptr, nullptr);
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, k, v, (int)(n > 0 ? n : 1));
  return bytes;
}

size_t sort_keys_temp_bytes(long long n) {
  size_t bytes = 0;
  cub::DoubleBuffer<unsigned long long> k(nullptr, nullptr);
  cub::DeviceRadixSort::SortKeys(nullptr, bytes, k, (int)(n > 0 ? n : 1));
  return bytes;
}

struct Layout {
  BroadScratch* sc;
  BoxList V, F, E;
  void* sort_tmp;
  size_t sort_tmp_bytes;
  unsigned long long* pair_alt;  // double buffer for sorting pairs
  size_t total;
};

void carve_list(Carver& c, BoxList& L, long long n) {
  L.n = n;
  L.box = c.take<double>(6 * n);
  L.keys[0] = c.take<unsigned long long>(n);
  L.keys[1] = c.take<unsigned long long>(n);
  L.vals[0] = c.take<unsigned int>(n);
  L.vals[1] = c.take<unsigned int>(n);
  L.s.lo = c.take<double>(n);
  L.s.hi = c.take<double>(n);
  L.s.alo = c.take<double>(n);
  L.s.ahi = c.take<double>(n);
  L.s.blo = c.take<double>(n);
  L.s.bhi = c.take<double>(n);
  L.s.id = c.take<int32_t>(n);
  L.s.obj = c.take<int32_t>(n);
}

Layout carve(void* base, long long nv, long long nf, long long ne, long long pair_cap, bool dry) {
  Carver c{static_cast<char*>(base), 0, dry};
  Layout L;
  L.sc = c.take<BroadScratch>(1);
  carve_list(c, L.V, nv);
  carve_list(c, L.F, nf);
  carve_list(c, L.E, ne);
  long long nmax = nv > nf ? nv : nf;
  nmax = nmax > ne ? nmax : ne;
  size_t tb = sort_temp_bytes(nmax);
  const size_t tk = sort_keys_temp_bytes(pair_cap);
  if (tk > tb) tb = tk;
  L.sort_tmp_bytes = tb;
  L.sort_tmp = c.take<char>((long long)tb);
  L.pair_alt = c.take<unsigned long long>(pair_cap);
  L.total = c.off + 256;
  return L;
}

int sort_list(BoxList& L, const Layout& lay, cudaStream_t s) {
  if (L.n == 0) return P2C_OK;
  cub::DoubleBuffer<unsigned long long> k(L.keys[0], L.keys[1]);
  cub::DoubleBuffer<unsigned int> v(L.vals[0], L.vals[1]);
  size_t tb = lay.sort_tmp_bytes;
  P2C_CUDA(cub::DeviceRadixSort::SortPairs(lay.sort_tmp, tb, k, v, (int)L.n, 0, 64, s));
  if (k.Current() != L.keys[0]) {
    std::swap(L.keys[0], L.keys[1]);
    std::swap(L.vals[0], L.vals[1]);
  }
  return P2C_OK;
}

int sort_pairs(unsigned long long* pairs, long long cap, const Layout& lay, cudaStream_t s) {
  if (cap <= 1) return P2C_OK;
  cub::DoubleBuffer<unsigned long long> k(pairs, lay.pair_alt);
  size_t tb = lay.sort_tmp_bytes;
  P2C_CUDA(cub::DeviceRadixSort::SortKeys(lay.sort_tmp, tb, k, (int)cap, 0, 64, s));
  if (k.Current() != pairs)
    P2C_CUDA(cudaMemcpyAsync(pairs, k.Current(), sizeof(unsigned long long) * cap, cudaMemcpyDeviceToDevice, s));
  return P2C_OK;
}

}  // namespace

int validate_scene(const p2c_scene* sc) {
  if (sc == nullptr) return fail(P2C_ERR_INVALID, "scene pointer is null");
  if (sc->nv < 0 || sc->nf < 0 || sc->ne < 0) return fail(P2C_ERR_INVALID, "scene counts must be non-negative");
  if (sc->nv >= (1ll << 31) || sc->nf >= (1ll << 31) || sc->ne >= (1ll << 31))
    return fail(P2C_ERR_INVALID, "scene counts must stay below 2^31");
  if (!(sc->thickness >= 0.0) || !std::isfinite(sc->thickness))
    return fail(P2C_ERR_INVALID, "scene thickness must be finite and non-negative");
  if (sc->nv > 0 && (sc->v_t0 == nullptr || sc->v_t1 == nullptr || sc->v_obj == nullptr))
    return fail(P2C_ERR_INVALID, "scene vertex arrays are null");
  if (sc->nf > 0 && (sc->faces == nullptr || sc->f_obj == nullptr))
    return fail(P2C_ERR_INVALID, "scene face arrays are null");
  if (sc->ne > 0 && (sc->edges == nullptr || sc->e_obj == nullptr))
    return fail(P2C_ERR_INVALID, "scene edge arrays are null");
  return P2C_OK;
}

size_t broadphase_workspace_bytes(long long nv, long long nf, long long ne, long long pair_cap) {
  return carve(nullptr, nv, nf, ne, pair_cap, true).total;
}

// Candidate generation; counts_dev receives {vf_count, ee_count, error_word, axis}.
int launch_broadphase(const p2c_scene& scene, unsigned long long* vf_out, long long vf_cap,
                      unsigned long long* ee_out, long long ee_cap, unsigned long long* counts_dev, bool sort_out,
                      void* ws, size_t ws_bytes, cudaStream_t s) {
  const long long pair_cap = vf_cap > ee_cap ? vf_cap : ee_cap;
  const size_t need = broadphase_workspace_bytes(scene.nv, scene.nf, scene.ne, pair_cap);
  if (ws == nullptr || ws_bytes < need)
    return fail(P2C_ERR_INVALID, "candidate workspace too small: %zu < %zu bytes", ws_bytes, need);
  Layout L = carve(ws, scene.nv, scene.nf, scene.ne, pair_cap, false);
  P2C_CUDA(cudaMemsetAsync(L.sc, 0, sizeof(BroadScratch), s));
  if (scene.nv > 0)
    boxes_kernel<1><<<grid_for(scene.nv, kBoxThreads), kBoxThreads, 0, s>>>(scene.v_t0, scene.v_t1, nullptr,
                                                                             scene.nv, scene.thickness, L.V.box, L.sc);
  if (scene.ne > 0)
    boxes_kernel<2><<<grid_for(scene.ne, kBoxThreads), kBoxThreads, 0, s>>>(
        scene.v_t0, scene.v_t1, scene.edges, scene.ne, scene.thickness, L.E.box, L.sc);
  if (scene.nf > 0)
    boxes_kernel<3><<<grid_for(scene.nf, kBoxThreads), kBoxThreads, 0, s>>>(
        scene.v_t0, scene.v_t1, scene.faces, scene.nf, scene.thickness, L.F.box, L.sc);
  P2C_CUDA(cudaGetLastError());
  const int32_t* objs[3] = {scene.v_obj, scene.f_obj, scene.e_obj};
  BoxList* lists[3] = {&L.V, &L.F, &L.E};
  for (int k = 0; k < 3; ++k) {
    BoxList& B = *lists[k];
    if (B.n == 0) continue;
    keys_kernel<<<grid_for(B.n, kBoxThreads), kBoxThreads, 0, s>>>(B.box, B.n, k == 0 ? scene.v_obj : nullptr,
                                                                   B.keys[0], B.vals[0], L.sc);
    P2C_CUDA(cudaGetLastError());
    int rc = sort_list(B, L, s);
    if (rc != P2C_OK) return rc;
    gather_kernel<<<grid_for(B.n, kBoxThreads), kBoxThreads, 0, s>>>(B.box, B.n, k == 0 ? scene.v_obj : nullptr,
                                                                     B.vals[0], objs[k], B.s, L.sc);
    P2C_CUDA(cudaGetLastError());
  }
  if (sort_out && vf_cap > 0)
    fill_u64_kernel<<<grid_for(vf_cap, 256), 256, 0, s>>>(vf_out, vf_cap, ~0ull);
  if (sort_out && ee_cap > 0)
    fill_u64_kernel<<<grid_for(ee_cap, 256), 256, 0, s>>>(ee_out, ee_cap, ~0ull);
  if (scene.nv + scene.nf > 0 && vf_out != nullptr)
    sweep_vf_kernel<<<grid_for(scene.nv + scene.nf, kSweepThreads), kSweepThreads, 0, s>>>(
        L.V.s, scene.nv, L.F.s, scene.nf, scene.faces, scene.exclude_self, vf_out, (unsigned long long)vf_cap, L.sc);
  if (scene.ne > 0 && ee_out != nullptr)
    sweep_ee_kernel<<<grid_for(scene.ne, kSweepThreads), kSweepThreads, 0, s>>>(
        L.E.s, scene.ne, scene.edges, scene.exclude_self, ee_out, (unsigned long long)ee_cap, L.sc);
  P2C_CUDA(cudaGetLastError());
  if (sort_out) {
    int rc = sort_pairs(vf_out, vf_cap, L, s);
    if (rc != P2C_OK) return rc;
    rc = sort_pairs(ee_out, ee_cap, L, s);
    if (rc != P2C_OK) return rc;
  }
  export_counts_kernel<<<1, 1, 0, s>>>(L.sc, counts_dev);
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

}  // namespace p2c

extern "C" {

size_t p2c_scene_candidates_workspace_bytes(int64_t nv, int64_t nf, int64_t ne, int64_t vf_cap, int64_t ee_cap) {
  return p2c::broadphase_workspace_bytes(nv, nf, ne, vf_cap > ee_cap ? vf_cap : ee_cap);
}

int p2c_scene_candidates(const p2c_scene* scene, uint64_t* vf_pairs_dev, int64_t vf_cap, uint64_t* ee_pairs_dev,
                         int64_t ee_cap, uint64_t* counts_dev, int sort_pairs, void* workspace_dev,
                         size_t workspace_bytes, void* stream) {
  int rc = p2c::validate_scene(scene);
  if (rc != P2C_OK) return rc;
  if (counts_dev == nullptr) return p2c::fail(P2C_ERR_INVALID, "counts pointer is null");
  if (vf_cap < 0 || ee_cap < 0) return p2c::fail(P2C_ERR_INVALID, "pair capacities must be non-negative");
  if ((vf_cap > 0 && vf_pairs_dev == nullptr) || (ee_cap > 0 && ee_pairs_dev == nullptr))
    return p2c::fail(P2C_ERR_INVALID, "pair output pointer is null");
  return p2c::launch_broadphase(*scene, reinterpret_cast<unsigned long long*>(vf_pairs_dev), vf_cap,
                                reinterpret_cast<unsigned long long*>(ee_pairs_dev), ee_cap,
                                reinterpret_cast<unsigned long long*>(counts_dev), sort_pairs != 0, workspace_dev,
                                workspace_bytes, p2c::as_stream(stream));
}

}  // extern "C"
