// broadphase_batch.cu — swept-AABB candidates of many scenes in one launch
// sequence.
//
// The column-subdivided sweep-and-prune of p2c_scene_candidates, segmented
// by scene so that a batch of N scenes costs about the launches of one
// scene instead of N times them (a 1,000-triangle scene alone is a chain of
// ~30 launches that each run for a few microseconds).  Primitives are
// indexed scene-major (scene s holds [P[s], P[s+1]): its vertices, faces,
// edges); every kernel finds a primitive's scene by binary search over P.
//   1. prep (one block): prefix offsets of primitives, pair capacities and
//      column tables per scene; per-scene scratch initialised;
//   2. swept boxes with per-scene axis statistics and object envelopes
//      (block-level sums when a block holds one scene, warp-level otherwise);
//   3. culling and per-scene, per-list extents;
//   4. one thread per scene: sweep axis, column grid (at most
//      max(64, n/4) cells for a scene of n primitives, 128 x 128 at most),
//      quantiser;
//   5. ONE radix sort of 64-bit keys (scene, list, column, 8-bit quantised
//      min: 24 + scene bits, 4 passes for up to 256 scenes) over all
//      primitives, a gather into one struct-of-arrays in sorted
//      order and per-scene column tables holding sorted positions;
//   6. sweeps that walk only their own scene's columns, appending pairs as
//      (scene << w | packed pair), w the widest scene's packed pair, into a buffer of the scenes' summed
//      capacities (scene s owns its capacity's slice, pre-filled with its
//      padding key);
//   7. ONE sort of all pairs and a scatter into each scene's own buffer,
//      unpacked to (a << 32 | b) and padded with ~0: every scene's list comes
//      out exactly as p2c_scene_candidates with sorted pairs writes it.
#include <cub/block/block_scan.cuh>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "broadphase.cuh"

namespace p2c {

int validate_scene(const p2c_scene* sc);

namespace {

constexpr int kThreads = 256;
constexpr int kPrepThreads = 1024;
constexpr unsigned kFull = 0xffffffffu;
constexpr long long kMaxScenePrims = 1ll << 22;  // packed pairs of one scene stay below 2^44
#ifndef P2C_BATCH_QBITS
#define P2C_BATCH_QBITS 8
#endif
constexpr int kBatchQBits = P2C_BATCH_QBITS;     // quantiser of the batched key
constexpr unsigned kBatchQMax = (1u << kBatchQBits) - 1u;
constexpr int kBatchListShift = kCellBits + kBatchQBits;  // key: scene | list | column | quantised min
constexpr int kBatchSceneShift = kBatchListShift + 2;

inline unsigned grid_for(long long n, int threads) {
  const long long g = (n + threads - 1) / threads;
  return (unsigned)(g > 0 ? g : 1);
}

int bit_length(long long x) {
  int b = 0;
  while (x > 0) {
    ++b;
    x >>= 1;
  }
  return b;
}

__device__ __forceinline__ int bit_length_dev(long long x) { return x > 0 ? 64 - __clzll(x) : 0; }

// Cells of a scene's column grid per list: enough for the scene's size,
// never more than the single-scene grid.
__host__ __device__ inline long long cell_budget(long long n_prims) {
  long long c = n_prims / 4;
  if (c < 64) c = 64;
  if (c > (long long)kMaxColumns * kMaxColumns) c = (long long)kMaxColumns * kMaxColumns;
  return c;
}

struct Offsets {
  unsigned long long* prim;    // n + 1
  unsigned long long* vf_cap;  // n + 1
  unsigned long long* ee_cap;  // n + 1
  unsigned long long* cell;    // n + 1 (cells per list; a scene's tables are 3 x its budget)
};

struct BatchBroad {
  const p2c_batch_scene* scenes;
  int n;
  Offsets off;
  BroadScratch* sc;          // n
  double* box;               // 6 x P (global primitive order)
  unsigned char* active;     // P
  unsigned long long* keys[2];
  unsigned* vals[2];
  SortedBoxes S;             // P entries in sorted order (cell tables unused here)
  unsigned* cell_begin;      // 3 x total cells
  unsigned* cell_end;
  unsigned long long* pack[2][2];  // vf / ee pair buffers and their sort alternates
  int pair_bits[2];                // packed pair bits of the widest scene, per family
};

__device__ __forceinline__ unsigned long long pair_mask(int bits) { return (1ull << bits) - 1ull; }

// Scene of global primitive g, starting from the block's first scene.
__device__ __forceinline__ int scene_from(const BatchBroad& B, int s_lo, unsigned long long g) {
  int s = s_lo;
  while (s + 1 < B.n && __ldg(B.off.prim + s + 1) <= g) ++s;
  return s;
}

__device__ __forceinline__ int find_segment(const unsigned long long* off, int n, unsigned long long x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int cull_count(const p2c_batch_scene& d) {
  return (d.exclude_self && d.n_obj >= 1 && d.n_obj <= kMaxCullObjects) ? d.n_obj : 0;
}

// ---- 1. prep -----------------------------------------------------------------
__global__ void __launch_bounds__(kPrepThreads) prep_kernel(BatchBroad B) {
  using Scan = cub::BlockScan<unsigned long long, kPrepThreads>;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ unsigned long long carry[4];
  if (threadIdx.x < 4) carry[threadIdx.x] = 0ull;
  __syncthreads();
  unsigned long long* outs[4] = {B.off.prim, B.off.vf_cap, B.off.ee_cap, B.off.cell};
  for (int base = 0; base < B.n; base += kPrepThreads) {
    const int s = base + (int)threadIdx.x;
    unsigned long long v[4] = {0ull, 0ull, 0ull, 0ull};
    if (s < B.n) {
      const p2c_batch_scene& d = B.scenes[s];
      const long long np = d.nv + d.nf + d.ne;
      v[0] = (unsigned long long)np;
      v[1] = (unsigned long long)d.vf_cap;
      v[2] = (unsigned long long)d.ee_cap;
      v[3] = (unsigned long long)cell_budget(np);
      BroadScratch& sc = B.sc[s];
      for (int q = 0; q < kMaxCullObjects; ++q)
        for (int a = 0; a < 3; ++a) {
          sc.obj_lo[q][a] = ~0ull;
          sc.obj_hi[q][a] = 0ull;
        }
      for (int l = 0; l < 3; ++l)
        for (int a = 0; a < 3; ++a) {
          sc.list[l].lo_min[a] = ~0ull;
          sc.list[l].hi_max[a] = 0ull;
        }
    }
    for (int k = 0; k < 4; ++k) {
      unsigned long long excl = 0ull, total = 0ull;
      Scan(tmp).ExclusiveSum(v[k], excl, total);
      if (s < B.n) outs[k][s] = carry[k] + excl;
      __syncthreads();
      if (threadIdx.x == 0) carry[k] += total;
      __syncthreads();
    }
  }
  if (threadIdx.x < 4) outs[threadIdx.x][B.n] = carry[threadIdx.x];
}

// ---- 2. swept boxes, statistics, envelopes -----------------------------------
__global__ void __launch_bounds__(kThreads) boxes_kernel(BatchBroad B, unsigned long long P) {
  __shared__ double red[9][kThreads / 32];
  __shared__ int scene_lo, scene_hi;
  const unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool live = g < P;
  int s = -1, l = 0, o = -1;
  double b[6] = {0, 0, 0, 0, 0, 0};
  __shared__ int block_scene;
  if (threadIdx.x == 0) block_scene = find_segment(B.off.prim, B.n, (unsigned long long)blockIdx.x * blockDim.x);
  __syncthreads();
  if (live) {
    s = scene_from(B, block_scene, g);
    const p2c_batch_scene& d = B.scenes[s];
    const long long loc = (long long)(g - B.off.prim[s]);
    l = loc < d.nv ? 0 : (loc < d.nv + d.nf ? 1 : 2);
    const long long i = l == 0 ? loc : (l == 1 ? loc - d.nv : loc - d.nv - d.nf);
    const bool finite = l == 0 ? swept_box<1>(d.v_t0, d.v_t1, nullptr, i, d.thickness, b)
                        : l == 1 ? swept_box<3>(d.v_t0, d.v_t1, d.faces, i, d.thickness, b)
                                 : swept_box<2>(d.v_t0, d.v_t1, d.edges, i, d.thickness, b);
    double* dst = B.box + 6 * g;
#pragma unroll
    for (int k = 0; k < 6; ++k) dst[k] = b[k];
    if (!finite) atomicOr(&B.sc[s].error_word, 1ull);
    if (l == 0 && cull_count(d) > 0) o = d.v_obj[i];
  }
  // object envelopes: per (scene, object) one atomic per warp
  {
    const bool mine0 = o >= 0 && s >= 0 && o < kMaxCullObjects;
    unsigned remaining = __ballot_sync(kFull, mine0);
    while (remaining) {
      const int leader = __ffs((int)remaining) - 1;
      const int ls = __shfl_sync(kFull, s, leader), lo_obj = __shfl_sync(kFull, o, leader);
      const bool mine = mine0 && s == ls && o == lo_obj;
      remaining &= ~__ballot_sync(kFull, mine);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        unsigned long long kmin = mine ? order_key(b[a]) : ~0ull;
        unsigned long long kmax = mine ? order_key(b[3 + a]) : 0ull;
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) {
          kmin = min(kmin, __shfl_xor_sync(kFull, kmin, sh));
          kmax = max(kmax, __shfl_xor_sync(kFull, kmax, sh));
        }
        if (lane == leader) {
          atomicMin(&B.sc[ls].obj_lo[lo_obj][a], kmin);
          atomicMax(&B.sc[ls].obj_hi[lo_obj][a], kmax);
        }
      }
    }
  }
  // axis statistics: sums of extents, centres and squared centres
  double vals[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (live) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double c = 0.5 * (b[3 + a] + b[a]);
      vals[a] = b[3 + a] - b[a];
      vals[3 + a] = c;
      vals[6 + a] = c * c;
    }
  }
  if (threadIdx.x == 0) {
    const unsigned long long first = (unsigned long long)blockIdx.x * blockDim.x;
    const unsigned long long last = min(first + blockDim.x, P) - 1ull;
    scene_lo = find_segment(B.off.prim, B.n, first);
    scene_hi = find_segment(B.off.prim, B.n, last);
  }
  __syncthreads();
  if (scene_lo == scene_hi) {  // one scene in the block: block sums, 10 atomics
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      double v = vals[k];
#pragma unroll
      for (int sh = 16; sh > 0; sh >>= 1) v += __shfl_down_sync(kFull, v, sh);
      if (lane == 0) red[k][threadIdx.x >> 5] = v;
    }
    const unsigned cnt = __popc(__ballot_sync(kFull, live));
    __syncthreads();
    BroadScratch& sc = B.sc[scene_lo];
    if (threadIdx.x < 9) {
      double t = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) t += red[threadIdx.x][w];
      double* dst = threadIdx.x < 3 ? &sc.extent_sum[threadIdx.x]
                    : threadIdx.x < 6 ? &sc.center_sum[threadIdx.x - 3]
                                      : &sc.center_sq_sum[threadIdx.x - 6];
      atomicAdd(dst, t);
    }
    if (lane == 0 && cnt) atomicAdd(&sc.count, (unsigned long long)cnt);
  } else {  // scene boundary inside the block: per warp and scene
    unsigned todo = __ballot_sync(kFull, live);
    while (todo) {
      const int leader = __ffs((int)todo) - 1;
      const int ls = __shfl_sync(kFull, s, leader);
      const bool mine = live && s == ls;
      todo &= ~__ballot_sync(kFull, mine);
      BroadScratch& sc = B.sc[ls];
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        double v = mine ? vals[k] : 0.0;
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) v += __shfl_xor_sync(kFull, v, sh);
        if (lane == leader) {
          double* dst = k < 3 ? &sc.extent_sum[k] : k < 6 ? &sc.center_sum[k - 3] : &sc.center_sq_sum[k - 6];
          atomicAdd(dst, v);
        }
      }
      const unsigned cnt = __popc(__ballot_sync(kFull, mine));
      if (lane == leader) atomicAdd(&sc.count, (unsigned long long)cnt);
    }
  }
}

// ---- 3. culling and per-list extents -----------------------------------------
__device__ __forceinline__ void max_if_larger(unsigned long long* p, unsigned long long v) {
  if (v > *reinterpret_cast<volatile unsigned long long*>(p)) atomicMax(p, v);
}
__device__ __forceinline__ void min_if_smaller(unsigned long long* p, unsigned long long v) {
  if (v < *reinterpret_cast<volatile unsigned long long*>(p)) atomicMin(p, v);
}

__global__ void __launch_bounds__(kThreads) classify_kernel(BatchBroad B, unsigned long long P) {
  const unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool keep = false, other = false;
  int s = -1, l = 3;
  double b[6] = {0, 0, 0, 0, 0, 0};
  __shared__ int block_scene;
  if (threadIdx.x == 0) block_scene = find_segment(B.off.prim, B.n, (unsigned long long)blockIdx.x * blockDim.x);
  __syncthreads();
  if (g < P) {
    s = scene_from(B, block_scene, g);
    const p2c_batch_scene& d = B.scenes[s];
    const long long loc = (long long)(g - B.off.prim[s]);
    l = loc < d.nv ? 0 : (loc < d.nv + d.nf ? 1 : 2);
    const long long i = l == 0 ? loc : (l == 1 ? loc - d.nv : loc - d.nv - d.nf);
    const int o = (l == 0 ? d.v_obj : (l == 1 ? d.f_obj : d.e_obj))[i];
    keep = !(l == 0 && o < 0);
#pragma unroll
    for (int k = 0; k < 6; ++k) b[k] = B.box[6 * g + k];
    const int cull = cull_count(d);
    if (keep && cull > 0) {
      const BroadScratch& sc = B.sc[s];
      bool near_other = false;
      for (int q = 0; q < cull && !near_other; ++q) {
        if (q == o || sc.obj_hi[q][0] == 0ull) continue;
        bool ov = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double olo = unorder_key(sc.obj_lo[q][a]), ohi = unorder_key(sc.obj_hi[q][a]);
          ov = ov && b[a] <= ohi && olo <= b[3 + a];
        }
        near_other = ov;
      }
      keep = near_other;
    }
    B.active[g] = keep ? 1 : 0;
    other = keep && o != 0 && o != 1 && d.exclude_self && d.n_obj == 2;
  }
  if (__any_sync(kFull, other) && other) atomicOr(&B.sc[s].obj_other, 1ull);  // only malformed two-object scenes
  // per (scene, list) extents; most warps hold one scene and one list
  unsigned todo = __ballot_sync(kFull, keep);
  while (todo) {
    const int leader = __ffs((int)todo) - 1;
    const int ls = __shfl_sync(kFull, s, leader), ll = __shfl_sync(kFull, l, leader);
    const bool mine = keep && s == ls && l == ll;
    const unsigned mask = __ballot_sync(kFull, mine);
    todo &= ~mask;
    ListStats& S = B.sc[ls].list[ll];
    if ((threadIdx.x & 31) == leader) atomicAdd(&S.active, (unsigned long long)__popc(mask));
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      unsigned long long ext = mine ? (unsigned long long)__double_as_longlong(b[3 + a] - b[a]) : 0ull;
      unsigned long long lo = mine ? order_key(b[a]) : ~0ull;
      unsigned long long hi = mine ? order_key(b[3 + a]) : 0ull;
#pragma unroll
      for (int sh = 16; sh > 0; sh >>= 1) {
        ext = max(ext, __shfl_xor_sync(kFull, ext, sh));
        lo = min(lo, __shfl_xor_sync(kFull, lo, sh));
        hi = max(hi, __shfl_xor_sync(kFull, hi, sh));
      }
      if ((threadIdx.x & 31) == leader) {
        max_if_larger(&S.ext_max[a], ext);
        min_if_smaller(&S.lo_min[a], lo);
        max_if_larger(&S.hi_max[a], hi);
      }
    }
  }
}

// ---- 4. per-scene grid (one thread per scene) ---------------------------------
__global__ void grid_kernel(BatchBroad B) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B.n) return;
  BroadScratch& sc = B.sc[s];
  const long long budget = (long long)(B.off.cell[s + 1] - B.off.cell[s]);
  int max_cols = (int)floor(sqrt((double)budget));
  if (max_cols > kMaxColumns) max_cols = kMaxColumns;
  if (max_cols < 1) max_cols = 1;
  const double n = sc.count > 0 ? (double)sc.count : 1.0;
  int axis = 0;
  double best = INFINITY;
  for (int a = 0; a < 3; ++a) {
    const double mean = sc.center_sum[a] / n;
    const double var = fmax(sc.center_sq_sum[a] / n - mean * mean, 0.0);
    const double score = (sc.extent_sum[a] / n) / (sqrt(var) + 1e-300);
    if (score < best) {
      best = score;
      axis = a;
    }
  }
  Grid g;
  g.axis = axis;
  g.a1 = axis == 0 ? 1 : 0;
  g.a2 = axis == 2 ? 1 : 2;
  g.qbits = kBatchQBits;
  const p2c_batch_scene& d = B.scenes[s];
  const bool split = d.exclude_self && d.n_obj == 2 && sc.obj_other == 0ull;
  g.split_shift = split ? kBatchQBits - 1 : -1;
  g.qmax = split ? (kBatchQMax >> 1) : kBatchQMax;
  const int ax[3] = {g.a1, g.a2, axis};
  double base[3], inv[3];
  int cols[2] = {1, 1};
  for (int k = 0; k < 3; ++k) {
    double lo = INFINITY, hi = -INFINITY, reach = 0.0;
    for (int l = 0; l < 3; ++l) {
      const ListStats& L = sc.list[l];
      const double r = L.active ? __longlong_as_double((long long)L.ext_max[ax[k]]) : 0.0;
      if (k < 2) (k == 0 ? g.reach1 : g.reach2)[l] = r;
      if (L.active == 0) continue;
      lo = fmin(lo, unorder_key(L.lo_min[ax[k]]));
      hi = fmax(hi, unorder_key(L.hi_max[ax[k]]));
      reach = fmax(reach, r);
    }
    const double range = (hi > lo) ? hi - lo : 0.0;
    base[k] = isfinite(lo) ? lo : 0.0;
    if (k < 2) {
      double width = fmax(reach, range / max_cols);
      if (!(width > 0.0) || !isfinite(width)) width = 1.0;
      int c = (int)fmin((double)max_cols, floor(range / width) + 1.0);
      cols[k] = c < 1 ? 1 : c;
      inv[k] = 1.0 / width;
    } else {
      inv[k] = (range > 0.0 && isfinite(range)) ? (double)g.qmax / range : 0.0;
    }
  }
  g.base1 = base[0];
  g.base2 = base[1];
  g.inv1 = inv[0];
  g.inv2 = inv[1];
  g.g1 = cols[0];
  g.g2 = cols[1];
  g.base0 = base[2];
  g.scale0 = inv[2];
  g.seg[0] = 0;
  g.seg[1] = sc.list[0].active;
  g.seg[2] = g.seg[1] + sc.list[1].active;
  g.seg[3] = g.seg[2] + sc.list[2].active;
  sc.grid = g;
}

// ---- 5. keys, sort, gather ---------------------------------------------------------
__global__ void __launch_bounds__(kThreads) keys_kernel(BatchBroad B, unsigned long long P) {
  const unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  __shared__ int block_scene;
  if (threadIdx.x == 0) block_scene = find_segment(B.off.prim, B.n, (unsigned long long)blockIdx.x * blockDim.x);
  __syncthreads();
  if (g >= P) return;
  unsigned long long key = ~0ull;
  if (B.active[g]) {
    const int s = scene_from(B, block_scene, g);
    const p2c_batch_scene& d = B.scenes[s];
    const long long loc = (long long)(g - B.off.prim[s]);
    const int l = loc < d.nv ? 0 : (loc < d.nv + d.nf ? 1 : 2);
    const Grid& G = B.sc[s].grid;
    const double* b = B.box + 6 * g;
    const unsigned c = (unsigned)(column(b[G.a1], G.base1, G.inv1, G.g1) * G.g2 +
                                  column(b[G.a2], G.base2, G.inv2, G.g2));
    int32_t o = 0;
    if (G.split_shift >= 0) {
      const long long j = l == 0 ? loc : (l == 1 ? loc - d.nv : loc - d.nv - d.nf);
      o = (l == 0 ? d.v_obj : (l == 1 ? d.f_obj : d.e_obj))[j];
    }
    key = ((unsigned long long)s << kBatchSceneShift) | ((unsigned long long)l << kBatchListShift) |
          ((unsigned long long)c << kBatchQBits) | split_field(G, o, quantise(b[G.axis], G));
  }
  B.keys[0][g] = key;
  B.vals[0][g] = (unsigned)g;
}

__device__ __forceinline__ unsigned* cell_table(const BatchBroad& B, unsigned* base, int s, int l) {
  const unsigned long long c0 = B.off.cell[s], budget = B.off.cell[s + 1] - c0;
  return base + 3ull * c0 + (unsigned long long)l * budget;
}

__global__ void __launch_bounds__(kThreads) gather_kernel(BatchBroad B, const unsigned long long* __restrict__ keys,
                                                          const unsigned* __restrict__ order, unsigned long long P) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const unsigned long long key = keys[i];
  if (key == ~0ull) return;  // culled entries sort last
  const int s = (int)(key >> kBatchSceneShift);
  const int l = (int)((key >> kBatchListShift) & 3ull);
  const p2c_batch_scene& d = B.scenes[s];
  const Grid& G = B.sc[s].grid;
  const unsigned long long g = order[i];
  const long long loc = (long long)(g - B.off.prim[s]);
  const long long j = l == 0 ? loc : (l == 1 ? loc - d.nv : loc - d.nv - d.nf);
  const double* b = B.box + 6 * g;
  B.S.lo[i] = b[G.axis];
  B.S.hi[i] = b[3 + G.axis];
  B.S.alo[i] = b[G.a1];
  B.S.ahi[i] = b[3 + G.a1];
  B.S.blo[i] = b[G.a2];
  B.S.bhi[i] = b[3 + G.a2];
  B.S.q[i] = (unsigned)(key & kBatchQMax);
  B.S.fb[i] = fbox_entry(b[G.a1], b[3 + G.a1], b[G.a2], b[3 + G.a2]);
  B.S.id[i] = (int32_t)j;
  B.S.obj[i] = (l == 0 ? d.v_obj : (l == 1 ? d.f_obj : d.e_obj))[j];
  const unsigned long long head = key >> kBatchQBits;  // scene, list and column
  const unsigned cell = (unsigned)(head & ((1ull << kCellBits) - 1ull));
  if (i == 0 || (keys[i - 1] >> kBatchQBits) != head) cell_table(B, B.cell_begin, s, l)[cell] = (unsigned)i;
  if (i + 1 == P || (keys[i + 1] >> kBatchQBits) != head) cell_table(B, B.cell_end, s, l)[cell] = (unsigned)(i + 1);
}

// ---- 6. sweeps -------------------------------------------------------------------
// Scene s's padding key: sorts after all of its pairs, before scene s + 1's.
__global__ void fill_pack_kernel(unsigned long long* pack, const unsigned long long* cap_off, int n,
                                 unsigned long long total, int bits) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int s = find_segment(cap_off, n, i);
  pack[i] = ((unsigned long long)s << bits) | pair_mask(bits);
}

// Warp append of found pairs, one atomic per scene present in the warp.
__device__ __forceinline__ void append_scene_pair(bool found, int s, unsigned long long key, unsigned long long* pack,
                                                  const unsigned long long* cap_off, BroadScratch* sc, bool vf,
                                                  int bits) {
  unsigned todo = __ballot_sync(kFull, found);
  const int lane = threadIdx.x & 31;
  while (todo) {
    const int leader = __ffs((int)todo) - 1;
    const int ls = __shfl_sync(kFull, s, leader);
    const bool mine = found && s == ls;
    const unsigned mask = __ballot_sync(kFull, mine);
    todo &= ~mask;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(vf ? &sc[ls].vf_count : &sc[ls].ee_count, (unsigned long long)__popc(mask));
    base = __shfl_sync(kFull, base, leader);
    if (mine) {
      const unsigned long long slot = base + (unsigned long long)__popc(mask & ((1u << lane) - 1u));
      const unsigned long long cap = cap_off[s + 1] - cap_off[s];
      if (slot < cap) pack[cap_off[s] + slot] = ((unsigned long long)s << bits) | key;
    }
  }
}

__device__ __forceinline__ SortedBoxes scene_view(const BatchBroad& B, int s, int l) {
  SortedBoxes Q = B.S;
  Q.cell_begin = cell_table(B, B.cell_begin, s, l);
  Q.cell_end = cell_table(B, B.cell_end, s, l);
  return Q;
}

// Lanes that share one scanning box's columns in the batched sweeps: 2
// (the batch fills the GPU many times over, so splitting further only adds
// work; 256 uneven scenes: 11.4 ms with 1 lane, 11.1 with 2, 12.2 with 4).
constexpr int kBatchSweepLanes = 2;

// Vertex-face pairs, ownership as in the single-scene sweep: a vertex owns
// the pairs whose face minimum is >= its minimum, a face the others.
__global__ void __launch_bounds__(kThreads) sweep_vf_kernel(BatchBroad B, const unsigned long long* __restrict__ keys,
                                                            unsigned long long P) {
  const unsigned long long tt = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long i = tt / kBatchSweepLanes;
  const int lane = (int)(tt % kBatchSweepLanes);
  bool live = false;
  int s = 0;
  bool from_vertex = false;
  if (i < P) {
    const unsigned long long key = keys[i];
    const int l = key == ~0ull ? 3 : (int)((key >> kBatchListShift) & 3ull);
    live = l <= 1;
    s = (int)(key >> kBatchSceneShift);
    from_vertex = l == 0;
  }
  if (!__any_sync(kFull, live)) return;
  StridedWalker w;
  Box6 pb{};
  FBox pf{};
  SortedBoxes Q{};
  Grid g{};
  double lo = 0.0;
  int32_t pid = 0, pobj = 0;
  int shift = 1, exclude_self = 1;
  const int32_t* faces = nullptr;
  if (live) {
    const p2c_batch_scene& d = B.scenes[s];
    g = B.sc[s].grid;
    Q = scene_view(B, s, from_vertex ? 1 : 0);
    faces = d.faces;
    exclude_self = d.exclude_self;
    shift = max(1, bit_length_dev(d.nf));
    lo = B.S.lo[i];
    pid = B.S.id[i];
    pobj = B.S.obj[i];
    pb = box_at(B.S, (long long)i);
    pf = fbox_of(pb);
    strided_walker_init(w, g, lo, pb.hi, pb.alo, pb.ahi, pb.blo, pb.bhi,
                        from_vertex ? g.reach1[1] : g.reach1[0], from_vertex ? g.reach2[1] : g.reach2[0], lane,
                        kBatchSweepLanes, split_prefix(g, pobj));
    live = w.next_cell(Q, g);
  }
  for (;;) {
    if (!__any_sync(kFull, live)) break;
    bool found = false;
    unsigned long long key = 0;
    if (live) {
      const unsigned j = w.j;
      const float4 qf = Q.fb[j];
      const double qlo = Q.lo[j];
      const bool own = from_vertex ? (qlo >= lo) : (qlo > lo);
      if (own && fmay_overlap(pf, qf) && overlap3(pb, qlo, Q, j)) {
        const int32_t qobj = Q.obj[j];
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
          key = pair_key((unsigned)vtx, (unsigned)fc, shift);
        }
      }
      ++w.j;
      if (w.j >= w.j_end || Q.q[w.j] > w.q_hi) live = w.next_cell(Q, g);
    }
    append_scene_pair(found, s, key, B.pack[0][0], B.off.vf_cap, B.sc, true, B.pair_bits[0]);
  }
}

// Edge-edge pairs: an edge owns the pairs whose partner minimum is larger
// (ties: larger edge index).
__global__ void __launch_bounds__(kThreads) sweep_ee_kernel(BatchBroad B, const unsigned long long* __restrict__ keys,
                                                            unsigned long long P) {
  const unsigned long long tt = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long i = tt / kBatchSweepLanes;
  const int lane = (int)(tt % kBatchSweepLanes);
  bool live = false;
  int s = 0;
  if (i < P) {
    const unsigned long long key = keys[i];
    live = key != ~0ull && ((key >> kBatchListShift) & 3ull) == 2ull;
    s = (int)(key >> kBatchSceneShift);
  }
  if (!__any_sync(kFull, live)) return;
  StridedWalker w;
  Box6 pb{};
  FBox pf{};
  SortedBoxes E{};
  Grid g{};
  double lo = 0.0;
  int32_t eid = 0, eobj = 0, a0 = 0, a1 = 0;
  int shift = 1, exclude_self = 1;
  const int32_t* edges = nullptr;
  if (live) {
    const p2c_batch_scene& d = B.scenes[s];
    g = B.sc[s].grid;
    E = scene_view(B, s, 2);
    edges = d.edges;
    exclude_self = d.exclude_self;
    shift = max(1, bit_length_dev(d.ne));
    lo = B.S.lo[i];
    eid = B.S.id[i];
    eobj = B.S.obj[i];
    a0 = __ldg(edges + 2 * (long long)eid);
    a1 = __ldg(edges + 2 * (long long)eid + 1);
    pb = box_at(B.S, (long long)i);
    pf = fbox_of(pb);
    strided_walker_init(w, g, lo, pb.hi, pb.alo, pb.ahi, pb.blo, pb.bhi, g.reach1[2], g.reach2[2], lane,
                        kBatchSweepLanes, split_prefix(g, eobj));
    live = w.next_cell(E, g);
  }
  for (;;) {
    if (!__any_sync(kFull, live)) break;
    bool found = false;
    unsigned long long key = 0;
    if (live) {
      const unsigned j = w.j;
      const float4 qf = E.fb[j];
      const double qlo = E.lo[j];
      const int32_t oid = E.id[j];
      const bool own = qlo > lo || (qlo == lo && oid > eid);
      if (own && fmay_overlap(pf, qf) && overlap3(pb, qlo, E, j)) {
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
          key = pair_key((unsigned)min(eid, oid), (unsigned)max(eid, oid), shift);
        }
      }
      ++w.j;
      if (w.j >= w.j_end || E.q[w.j] > w.q_hi) live = w.next_cell(E, g);
    }
    append_scene_pair(found, s, key, B.pack[1][0], B.off.ee_cap, B.sc, false, B.pair_bits[1]);
  }
}

// ---- 7. scatter sorted pairs into the scenes' buffers --------------------------------
__global__ void scatter_pairs_kernel(BatchBroad B, const unsigned long long* __restrict__ sorted, int family,
                                     unsigned long long total) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const unsigned long long k = sorted[i];
  const int bits = B.pair_bits[family];
  const int s = (int)(k >> bits);
  const unsigned long long* cap_off = family == 0 ? B.off.vf_cap : B.off.ee_cap;
  const unsigned long long local = i - cap_off[s];
  const p2c_batch_scene& d = B.scenes[s];
  unsigned long long* out = reinterpret_cast<unsigned long long*>(family == 0 ? d.vf_pairs : d.ee_pairs);
  const unsigned long long p = k & pair_mask(bits);
  if (p == pair_mask(bits)) {
    out[local] = ~0ull;
  } else {
    const int shift = max(1, bit_length_dev(family == 0 ? d.nf : d.ne));
    out[local] = ((p >> shift) << 32) | (p & ((1ull << shift) - 1ull));
  }
}

__global__ void export_counts_kernel(BatchBroad B) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B.n) return;
  const BroadScratch& sc = B.sc[s];
  unsigned long long* c = reinterpret_cast<unsigned long long*>(B.scenes[s].counts);
  c[0] = sc.vf_count;
  c[1] = sc.ee_count;
  c[2] = sc.error_word;
  c[3] = (unsigned long long)sc.grid.axis | ((unsigned long long)sc.grid.g1 << 8) |
         ((unsigned long long)sc.grid.g2 << 24) | (sc.grid.seg[3] << 40);
}

// ---- workspace ---------------------------------------------------------------------
struct Totals {
  unsigned long long P = 0, vf = 0, ee = 0, cells = 0;
  int pair_bits[2] = {2, 2};  // widest packed pair of any scene: vf, ee
};

Totals totals_of(const p2c_batch_scene* h, int n) {
  Totals t;
  for (int s = 0; s < n; ++s) {
    const long long np = h[s].nv + h[s].nf + h[s].ne;
    t.P += (unsigned long long)np;
    t.vf += (unsigned long long)h[s].vf_cap;
    t.ee += (unsigned long long)h[s].ee_cap;
    t.cells += (unsigned long long)cell_budget(np);
    t.pair_bits[0] = std::max(t.pair_bits[0], bit_length(h[s].nv) + std::max(1, bit_length(h[s].nf)));
    t.pair_bits[1] = std::max(t.pair_bits[1], bit_length(h[s].ne) + std::max(1, bit_length(h[s].ne)));
  }
  return t;
}

size_t sort_temp_bytes(const Totals& t) {
  size_t a = 0, b = 0, c = 0;
  const int np = (int)std::max<unsigned long long>(t.P, 1ull);
  cub::DeviceRadixSort::SortPairs(nullptr, a, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (const unsigned*)nullptr, (unsigned*)nullptr, np);
  cub::DeviceRadixSort::SortKeys(nullptr, b, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                 (int)std::max<unsigned long long>(t.vf, 1ull));
  cub::DeviceRadixSort::SortKeys(nullptr, c, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                 (int)std::max<unsigned long long>(t.ee, 1ull));
  return std::max(a, std::max(b, c));
}

struct Carve {
  BatchBroad B;
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  size_t total = 0;
};

Carve carve(void* base, const p2c_batch_scene* scenes_dev, int n, const Totals& t) {
  Carve C;
  size_t off = 0;
  char* b = static_cast<char*>(base);
  auto take = [&](size_t bytes) -> void* {
    void* p = b == nullptr ? nullptr : b + off;
    off += (std::max<size_t>(bytes, 1) + 255) & ~size_t(255);
    return p;
  };
  const size_t P = (size_t)std::max<unsigned long long>(t.P, 1ull);
  BatchBroad& B = C.B;
  B.scenes = scenes_dev;
  B.n = n;
  B.off.prim = static_cast<unsigned long long*>(take(8 * (size_t)(n + 1)));
  B.off.vf_cap = static_cast<unsigned long long*>(take(8 * (size_t)(n + 1)));
  B.off.ee_cap = static_cast<unsigned long long*>(take(8 * (size_t)(n + 1)));
  B.off.cell = static_cast<unsigned long long*>(take(8 * (size_t)(n + 1)));
  B.sc = static_cast<BroadScratch*>(take(sizeof(BroadScratch) * (size_t)n));
  B.box = static_cast<double*>(take(48 * P));
  B.active = static_cast<unsigned char*>(take(P));
  B.keys[0] = static_cast<unsigned long long*>(take(8 * P));
  B.keys[1] = static_cast<unsigned long long*>(take(8 * P));
  B.vals[0] = static_cast<unsigned*>(take(4 * P));
  B.vals[1] = static_cast<unsigned*>(take(4 * P));
  B.S.lo = static_cast<double*>(take(8 * P));
  B.S.hi = static_cast<double*>(take(8 * P));
  B.S.alo = static_cast<double*>(take(8 * P));
  B.S.ahi = static_cast<double*>(take(8 * P));
  B.S.blo = static_cast<double*>(take(8 * P));
  B.S.bhi = static_cast<double*>(take(8 * P));
  B.S.q = static_cast<unsigned*>(take(4 * P));
  B.S.fb = static_cast<float4*>(take(16 * P));
  B.S.id = static_cast<int32_t*>(take(4 * P));
  B.S.obj = static_cast<int32_t*>(take(4 * P));
  B.cell_begin = static_cast<unsigned*>(take(4 * 3 * (size_t)t.cells));
  B.cell_end = static_cast<unsigned*>(take(4 * 3 * (size_t)t.cells));
  for (int f = 0; f < 2; ++f) {
    const size_t cap = (size_t)std::max<unsigned long long>(f == 0 ? t.vf : t.ee, 1ull);
    B.pack[f][0] = static_cast<unsigned long long*>(take(8 * cap));
    B.pack[f][1] = static_cast<unsigned long long*>(take(8 * cap));
  }
  C.tmp_bytes = sort_temp_bytes(t);
  C.tmp = take(C.tmp_bytes);
  C.total = off;
  return C;
}

int validate_table(const p2c_batch_scene* h, int n) {
  for (int s = 0; s < n; ++s) {
    const p2c_batch_scene& d = h[s];
    p2c_scene sc{d.v_t0, d.v_t1, d.faces, d.edges, d.v_obj, d.f_obj, d.e_obj, d.nv, d.nf, d.ne, d.thickness,
                 d.exclude_self, d.n_obj};
    const int rc = validate_scene(&sc);
    if (rc != P2C_OK) return fail(rc, "scene %d: %s", s, p2c_last_error());
    if (d.nv >= kMaxScenePrims || d.nf >= kMaxScenePrims || d.ne >= kMaxScenePrims)
      return fail(P2C_ERR_INVALID, "scene %d: batched candidates need nv, nf, ne < 2^22", s);
    if (d.counts == nullptr) return fail(P2C_ERR_INVALID, "scene %d: counts pointer is null", s);
    if (d.vf_cap < 0 || d.ee_cap < 0) return fail(P2C_ERR_INVALID, "scene %d: pair capacities must be non-negative", s);
    if ((d.vf_cap > 0 && d.vf_pairs == nullptr) || (d.ee_cap > 0 && d.ee_pairs == nullptr))
      return fail(P2C_ERR_INVALID, "scene %d: pair output pointer is null", s);
  }
  return P2C_OK;
}

}  // namespace

int launch_batch_candidates(const p2c_batch_scene* h, const p2c_batch_scene* dev, int n, void* ws, size_t ws_bytes,
                            cudaStream_t s) {
  const Totals t = totals_of(h, n);
  if (t.P >= (1ull << 31) || t.vf >= (1ull << 31) || t.ee >= (1ull << 31))
    return fail(P2C_ERR_INVALID, "batch too large for one candidate launch (primitives and capacities < 2^31)");
  const Carve need = carve(nullptr, dev, n, t);
  if (ws == nullptr || ws_bytes < need.total)
    return fail(P2C_ERR_INVALID, "batch candidate workspace too small: %zu < %zu bytes", ws_bytes, need.total);
  Carve C = carve(ws, dev, n, t);
  BatchBroad& B = C.B;
  const int scene_bits = std::max(1, bit_length(n - 1));
  B.pair_bits[0] = t.pair_bits[0];
  B.pair_bits[1] = t.pair_bits[1];
  P2C_CUDA(cudaMemsetAsync(B.sc, 0, sizeof(BroadScratch) * (size_t)n, s));
  P2C_CUDA(cudaMemsetAsync(B.cell_begin, 0, 4 * 3 * (size_t)t.cells, s));
  P2C_CUDA(cudaMemsetAsync(B.cell_end, 0, 4 * 3 * (size_t)t.cells, s));
  prep_kernel<<<1, kPrepThreads, 0, s>>>(B);
  P2C_CUDA(cudaGetLastError());
  const unsigned long long P = t.P;
  if (P > 0) {
    boxes_kernel<<<grid_for((long long)P, kThreads), kThreads, 0, s>>>(B, P);
    classify_kernel<<<grid_for((long long)P, kThreads), kThreads, 0, s>>>(B, P);
  }
  grid_kernel<<<grid_for(n, 128), 128, 0, s>>>(B);
  P2C_CUDA(cudaGetLastError());
  if (P > 0) {
    keys_kernel<<<grid_for((long long)P, kThreads), kThreads, 0, s>>>(B, P);
    P2C_CUDA(cudaGetLastError());
    size_t tb = C.tmp_bytes;
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(C.tmp, tb, B.keys[0], B.keys[1], B.vals[0], B.vals[1], (int)P, 0,
                                             kBatchSceneShift + scene_bits, s));
    gather_kernel<<<grid_for((long long)P, kThreads), kThreads, 0, s>>>(B, B.keys[1], B.vals[1], P);
    P2C_CUDA(cudaGetLastError());
  }
  for (int f = 0; f < 2; ++f) {
    const unsigned long long tot = f == 0 ? t.vf : t.ee;
    if (tot > 0)
      fill_pack_kernel<<<grid_for((long long)tot, 256), 256, 0, s>>>(B.pack[f][0], f == 0 ? B.off.vf_cap : B.off.ee_cap,
                                                                       n, tot, B.pair_bits[f]);
  }
  P2C_CUDA(cudaGetLastError());
  if (P > 0) {
    const long long PL = (long long)P * kBatchSweepLanes;
    if (t.vf > 0) sweep_vf_kernel<<<grid_for(PL, kThreads), kThreads, 0, s>>>(B, B.keys[1], P);
    if (t.ee > 0) sweep_ee_kernel<<<grid_for(PL, kThreads), kThreads, 0, s>>>(B, B.keys[1], P);
    P2C_CUDA(cudaGetLastError());
  }
  for (int f = 0; f < 2; ++f) {
    const unsigned long long tot = f == 0 ? t.vf : t.ee;
    if (tot == 0) continue;
    size_t tb = C.tmp_bytes;
    P2C_CUDA(cub::DeviceRadixSort::SortKeys(C.tmp, tb, B.pack[f][0], B.pack[f][1], (int)tot, 0,
                                            B.pair_bits[f] + scene_bits, s));
    scatter_pairs_kernel<<<grid_for((long long)tot, 256), 256, 0, s>>>(B, B.pack[f][1], f, tot);
    P2C_CUDA(cudaGetLastError());
  }
  export_counts_kernel<<<grid_for(n, 128), 128, 0, s>>>(B);
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

}  // namespace p2c

extern "C" {

size_t p2c_batch_candidates_workspace_bytes(const p2c_batch_scene* scenes_host, int32_t n_scenes) {
  if (scenes_host == nullptr || n_scenes < 1) return 0;
  const p2c::Totals t = p2c::totals_of(scenes_host, n_scenes);
  return p2c::carve(nullptr, nullptr, n_scenes, t).total;
}

int p2c_batch_candidates(const p2c_batch_scene* scenes_host, const p2c_batch_scene* scenes_dev, int32_t n_scenes,
                         void* workspace_dev, size_t workspace_bytes, void* stream) {
  if (scenes_host == nullptr || scenes_dev == nullptr) return p2c::fail(P2C_ERR_INVALID, "scene table pointer is null");
  if (n_scenes < 1 || n_scenes > (1 << 20))
    return p2c::fail(P2C_ERR_INVALID, "batch scene count must lie in [1, 2^20]");
  const int rc = p2c::validate_table(scenes_host, n_scenes);
  if (rc != P2C_OK) return rc;
  return p2c::launch_batch_candidates(scenes_host, scenes_dev, n_scenes, workspace_dev, workspace_bytes,
                                      p2c::as_stream(stream));
}

}  // extern "C"
