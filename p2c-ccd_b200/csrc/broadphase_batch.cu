// broadphase_batch.cu — swept-AABB candidates of many scenes in one launch
// sequence.
//
// The column-subdivided sweep-and-prune of p2c_scene_candidates, segmented
// by scene so that a batch of N scenes costs about the launches of one
// scene instead of N times them (a 1,000-triangle scene alone is a chain of
// ~30 launches that each run for a few microseconds).  Primitives are
// indexed scene-major (scene s holds [P[s], P[s+1]): its vertices, faces,
// edges); every kernel finds a primitive's scene by binary search over P.
//   1. prep (one block): prefix offsets of primitives, vertices, pair
//      capacities and column tables per scene (minima are kept as
//      complemented keys, so the zeroed scratch starts empty);
//   2. vertex swept boxes: object envelopes and per-scene axis statistics
//      (block-level sums when a block holds one scene, warp-level otherwise);
//   3. every primitive's swept box, culled against the other objects'
//      envelopes; kept boxes appended to a compact list (often a few per cent
//      of the primitives), with per-scene, per-list extents;
//   4. one thread per scene: sweep axis, column grid (at most
//      max(64, n/4) cells for a scene of n primitives, 128 x 128 at most),
//      quantiser;
//   5. ONE radix sort, with the count read on the device, of the kept boxes'
//      keys (scene, list, column, 8-bit low field: the quantised min, with
//      the object bit of a two-body split; 24 + scene bits: 32-bit keys and 4
//      passes for up to 256 scenes, 64-bit keys beyond), a gather into one
//      struct-of-arrays in sorted order and per-scene column tables holding
//      sorted positions;
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
#include "count_sort.cuh"

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
  unsigned long long* vert;    // n + 1 (vertices)
};

struct BatchBroad {
  const p2c_batch_scene* scenes;
  int n;
  Offsets off;
  BroadScratch* sc;          // n
  double* cbox;              // 6 x kept boxes, in compaction order
  unsigned* cprim;           // global primitive index of each kept box
  unsigned long long* keys[2];
  unsigned* keys32[2];       // the same buffers as 32-bit keys, used when key32 is set
  int key32;                 // the scene, list, column and quantiser fields fit 32 bits
  int sorted_buf;            // which of keys / vals [0] or [1] holds the sorted entries
  unsigned long long* n_keyed;  // boxes kept after culling (the compact and sorted entries)
  unsigned* vals[2];
  SortedBoxes S;             // P entries in sorted order (cell tables unused here)
  unsigned* cell_begin;      // 3 x total cells
  unsigned* cell_end;
  unsigned long long* pack[2][2];  // vf / ee pair buffers and their sort alternates
  uint4* chunks[2];                // queued pieces of long windows (box, first, end), per family
  unsigned long long* chunk_count; // 2 counters
  unsigned long long chunk_cap;    // chunks each queue holds
  unsigned long long* sweep_next;  // 2 counters: next slot of the vertex-face / edge-edge sweep
  int pair_bits[2];                // packed pair bits of the widest scene, per family
};

__device__ __forceinline__ unsigned long long pair_mask(int bits) { return (1ull << bits) - 1ull; }

// Sorted key i < *n_keyed from the 32- or 64-bit buffer.
__device__ __forceinline__ unsigned long long sorted_key(const BatchBroad& B, unsigned long long i) {
  return B.key32 ? (unsigned long long)B.keys32[B.sorted_buf][i] : B.keys[B.sorted_buf][i];
}

// Segment of g in offsets off (n segments), starting from the block's first
// segment.
__device__ __forceinline__ int scene_from(const unsigned long long* off, int n, int s_lo, unsigned long long g) {
  int s = s_lo;
  while (s + 1 < n && __ldg(off + s + 1) <= g) ++s;
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
  __shared__ unsigned long long carry[5];
  if (threadIdx.x < 5) carry[threadIdx.x] = 0ull;
  __syncthreads();
  unsigned long long* outs[5] = {B.off.prim, B.off.vf_cap, B.off.ee_cap, B.off.cell, B.off.vert};
  for (int base = 0; base < B.n; base += kPrepThreads) {
    const int s = base + (int)threadIdx.x;
    unsigned long long v[5] = {0ull, 0ull, 0ull, 0ull, 0ull};
    if (s < B.n) {
      const p2c_batch_scene& d = B.scenes[s];
      const long long np = d.nv + d.nf + d.ne;
      v[0] = (unsigned long long)np;
      v[1] = (unsigned long long)d.vf_cap;
      v[2] = (unsigned long long)d.ee_cap;
      v[3] = (unsigned long long)cell_budget(np);
      v[4] = (unsigned long long)d.nv;
    }
    for (int k = 0; k < 5; ++k) {
      unsigned long long excl = 0ull, total = 0ull;
      Scan(tmp).ExclusiveSum(v[k], excl, total);
      if (s < B.n) outs[k][s] = carry[k] + excl;
      __syncthreads();
      if (threadIdx.x == 0) carry[k] += total;
      __syncthreads();
    }
  }
  if (threadIdx.x < 5) outs[threadIdx.x][B.n] = carry[threadIdx.x];
}

// ---- 2. vertex envelopes and axis statistics ----------------------------------
// One thread per vertex of the batch (scene s holds vertices [vert[s],
// vert[s + 1])): its swept box joins its object's envelope (order keys, one
// atomic per object and warp) and the scene's sums of extents, centres and
// squared centres that choose the sweep axis.  Faces and edges are boxes of
// these vertices, so the vertex pass also finds every non-finite coordinate.
__global__ void __launch_bounds__(kThreads) envelope_kernel(BatchBroad B, unsigned long long V) {
  __shared__ double red[9][kThreads / 32];
  __shared__ int scene_lo, scene_hi, block_scene;
  const unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool live = g < V;
  int s = -1, o = -1;
  double b[6] = {0, 0, 0, 0, 0, 0};
  if (threadIdx.x == 0) {
    const unsigned long long first = (unsigned long long)blockIdx.x * blockDim.x;
    block_scene = scene_lo = find_segment(B.off.vert, B.n, first);
    scene_hi = find_segment(B.off.vert, B.n, min(first + blockDim.x, V) - 1ull);
  }
  __syncthreads();
  if (live) {
    s = scene_from(B.off.vert, B.n, block_scene, g);
    const p2c_batch_scene& d = B.scenes[s];
    const long long i = (long long)(g - B.off.vert[s]);
    if (!swept_box<1>(d.v_t0, d.v_t1, nullptr, i, d.thickness, b)) atomicOr(&B.sc[s].error_word, 1ull);
    if (cull_count(d) > 0) o = d.v_obj[i];
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
          atomicMax(&B.sc[ls].obj_nlo[lo_obj][a], ~kmin);
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

// ---- 3. swept boxes, culling, compaction and per-list extents ------------------
__device__ __forceinline__ void max_if_larger(unsigned long long* p, unsigned long long v) {
  if (v > *reinterpret_cast<volatile unsigned long long*>(p)) atomicMax(p, v);
}

// One thread per primitive: its swept box; kept unless it is a vertex in no
// face or (self pairs excluded) it lies outside every other object's
// envelope.  Kept boxes are appended (one atomic per warp) to a compact list
// of (box, primitive) entries that everything after works on, and their
// extents per (scene, list) size the column grids.
__global__ void __launch_bounds__(kThreads) cull_kernel(BatchBroad B, unsigned long long P) {
  const unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool keep = false, other = false;
  int s = -1, l = 3;
  double b[6] = {0, 0, 0, 0, 0, 0};
  __shared__ int block_scene;
  if (threadIdx.x == 0) block_scene = find_segment(B.off.prim, B.n, (unsigned long long)blockIdx.x * blockDim.x);
  __syncthreads();
  if (g < P) {
    s = scene_from(B.off.prim, B.n, block_scene, g);
    const p2c_batch_scene& d = B.scenes[s];
    const long long loc = (long long)(g - B.off.prim[s]);
    l = loc < d.nv ? 0 : (loc < d.nv + d.nf ? 1 : 2);
    const long long i = l == 0 ? loc : (l == 1 ? loc - d.nv : loc - d.nv - d.nf);
    const int o = (l == 0 ? d.v_obj : (l == 1 ? d.f_obj : d.e_obj))[i];
    keep = !(l == 0 && o < 0);
    if (l == 0) swept_box<1>(d.v_t0, d.v_t1, nullptr, i, d.thickness, b);
    else if (l == 1) swept_box<3>(d.v_t0, d.v_t1, d.faces, i, d.thickness, b);
    else swept_box<2>(d.v_t0, d.v_t1, d.edges, i, d.thickness, b);
    const int cull = cull_count(d);
    if (keep && cull > 0) {
      const BroadScratch& sc = B.sc[s];
      bool near_other = false;
      for (int q = 0; q < cull && !near_other; ++q) {
        if (q == o || sc.obj_hi[q][0] == 0ull) continue;
        bool ov = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double olo = unorder_key(~sc.obj_nlo[q][a]), ohi = unorder_key(sc.obj_hi[q][a]);
          ov = ov && b[a] <= ohi && olo <= b[3 + a];
        }
        near_other = ov;
      }
      keep = near_other;
    }
    other = keep && o != 0 && o != 1 && d.exclude_self && d.n_obj == 2;
  }
  if (__any_sync(kFull, other) && other) atomicOr(&B.sc[s].obj_other, 1ull);  // only malformed two-object scenes
  // compaction of the kept boxes
  {
    const unsigned m = __ballot_sync(kFull, keep);
    if (m != 0u) {
      const int lane = threadIdx.x & 31;
      const int leader = __ffs((int)m) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(B.n_keyed, (unsigned long long)__popc(m));
      base = __shfl_sync(kFull, base, leader);
      if (keep) {
        const unsigned long long c = base + (unsigned long long)__popc(m & ((1u << lane) - 1u));
        double* dst = B.cbox + 6 * c;
#pragma unroll
        for (int k = 0; k < 6; ++k) dst[k] = b[k];
        B.cprim[c] = (unsigned)g;
      }
    }
  }
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
        max_if_larger(&S.nlo_min[a], ~lo);
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
      lo = fmin(lo, unorder_key(~L.nlo_min[ax[k]]));
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
// Sort key of every kept box (compact entry c, value c): the order of the
// compact entries does not matter, they are sorted on their full keys and
// the pairs are sorted at the end.
// With pad_to > 0 the entries [kept, pad_to) get the key ~0, after every box
// (its list field, 3, names no list), for a sort sized on the host.
__global__ void __launch_bounds__(kThreads) keys_kernel(BatchBroad B, unsigned long long pad_to) {
  const unsigned long long n = *B.n_keyed;
  for (unsigned long long c = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; c < pad_to;
       c += (unsigned long long)gridDim.x * blockDim.x)
    if (c >= n) {
      if (B.key32) B.keys32[0][c] = ~0u;
      else B.keys[0][c] = ~0ull;
      B.vals[0][c] = (unsigned)c;
    }
  for (unsigned long long c = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long g = B.cprim[c];
    const int s = find_segment(B.off.prim, B.n, g);
    const p2c_batch_scene& d = B.scenes[s];
    const long long loc = (long long)(g - B.off.prim[s]);
    const int l = loc < d.nv ? 0 : (loc < d.nv + d.nf ? 1 : 2);
    const Grid& G = B.sc[s].grid;
    const double* b = B.cbox + 6 * c;
    const unsigned cell = (unsigned)(column(b[G.a1], G.base1, G.inv1, G.g1) * G.g2 +
                                     column(b[G.a2], G.base2, G.inv2, G.g2));
    int32_t o = 0;
    if (G.split_shift >= 0) {
      const long long j = l == 0 ? loc : (l == 1 ? loc - d.nv : loc - d.nv - d.nf);
      o = (l == 0 ? d.v_obj : (l == 1 ? d.f_obj : d.e_obj))[j];
    }
    const unsigned long long key = ((unsigned long long)s << kBatchSceneShift) |
                                   ((unsigned long long)l << kBatchListShift) |
                                   ((unsigned long long)cell << kBatchQBits) |
                                   split_field(G, o, quantise(b[G.axis], G));
    if (B.key32) B.keys32[0][c] = (unsigned)key;
    else B.keys[0][c] = key;
    B.vals[0][c] = (unsigned)c;
  }
}

__device__ __forceinline__ unsigned* cell_table(const BatchBroad& B, unsigned* base, int s, int l) {
  const unsigned long long c0 = B.off.cell[s], budget = B.off.cell[s + 1] - c0;
  return base + 3ull * c0 + (unsigned long long)l * budget;
}

__device__ __forceinline__ void gather_one(const BatchBroad& B, const unsigned* __restrict__ order,
                                           unsigned long long i, unsigned long long n) {
  const unsigned long long key = sorted_key(B, i);
  const int s = (int)(key >> kBatchSceneShift);
  const int l = (int)((key >> kBatchListShift) & 3ull);
  const p2c_batch_scene& d = B.scenes[s];
  const Grid& G = B.sc[s].grid;
  const unsigned c = order[i];
  const unsigned long long g = B.cprim[c];
  const long long loc = (long long)(g - B.off.prim[s]);
  const long long j = l == 0 ? loc : (l == 1 ? loc - d.nv : loc - d.nv - d.nf);
  const double* b = B.cbox + 6 * (unsigned long long)c;
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
  if (i == 0 || (sorted_key(B, i - 1) >> kBatchQBits) != head) cell_table(B, B.cell_begin, s, l)[cell] = (unsigned)i;
  if (i + 1 == n || (sorted_key(B, i + 1) >> kBatchQBits) != head)
    cell_table(B, B.cell_end, s, l)[cell] = (unsigned)(i + 1);
}

__global__ void __launch_bounds__(kThreads) gather_kernel(BatchBroad B) {
  const unsigned long long n = *B.n_keyed;
  const unsigned* __restrict__ order = B.vals[B.sorted_buf];
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    gather_one(B, order, i, n);
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
#ifndef P2C_BATCH_SWEEP_LANES
#define P2C_BATCH_SWEEP_LANES 2
#endif
constexpr int kBatchSweepLanes = P2C_BATCH_SWEEP_LANES;
#ifndef P2C_BATCH_SWEEP_BLOCKS
#define P2C_BATCH_SWEEP_BLOCKS 4
#endif
constexpr int kBatchSweepBlocks = P2C_BATCH_SWEEP_BLOCKS;  // resident blocks the sweeps are compiled for

// Long windows: a lane that has tested kChunk entries of one column's window
// and is not through it hands the rest to the chunk queue in pieces of
// kChunk entries, which a second launch spreads over the whole GPU.  A few
// boxes long along the sweep axis (swept far during the step) have windows
// of hundreds of partners; walked by one lane they set the length of the
// whole launch.  When the queue is full the lane walks on by itself.
constexpr unsigned kChunk = 32;
// Queue capacity per family: one chunk per 8 primitives of the batch, within
// [4096, 2^20] (a small batch keeps a small workspace).
__host__ __device__ inline unsigned long long chunk_cap_for(unsigned long long prims) {
  const unsigned long long c = prims / 8;
  return c < 4096ull ? 4096ull : (c > (1ull << 20) ? (1ull << 20) : c);
}

// A scanning box of the vertex-face sweep and the partner list it walks.
struct VfScan {
  Box6 pb;
  FBox pf;
  double lo;
  int32_t pid, pobj;
  bool from_vertex;
  int exclude_self, shift;
  const int32_t* faces;
  SortedBoxes Q;
};

__device__ __forceinline__ void vf_scan_at(const BatchBroad& B, unsigned long long i, int s, bool from_vertex,
                                           VfScan& c) {
  const p2c_batch_scene& d = B.scenes[s];
  c.Q = scene_view(B, s, from_vertex ? 1 : 0);
  c.from_vertex = from_vertex;
  c.faces = d.faces;
  c.exclude_self = d.exclude_self;
  c.shift = max(1, bit_length_dev(d.nf));
  c.lo = B.S.lo[i];
  c.pid = B.S.id[i];
  c.pobj = B.S.obj[i];
  c.pb = box_at(B.S, (long long)i);
  c.pf = fbox_of(c.pb);
}

// Partner entry j: a pair this box owns, overlapping on all axes and allowed
// by the object rules (the reference's BuildVFCandidates conditions).
__device__ __forceinline__ bool vf_test(const VfScan& c, unsigned j, unsigned long long& key) {
  const float4 qf = c.Q.fb[j];
  const double qlo = c.Q.lo[j];
  const bool own = c.from_vertex ? (qlo >= c.lo) : (qlo > c.lo);
  if (!(own && fmay_overlap(c.pf, qf) && overlap3(c.pb, qlo, c.Q, j))) return false;
  const int32_t qobj = c.Q.obj[j];
  const int32_t vtx = c.from_vertex ? c.pid : c.Q.id[j];
  const int32_t fc = c.from_vertex ? c.Q.id[j] : c.pid;
  if (c.pobj == qobj) {
    if (c.exclude_self) return false;
    const int32_t* fv = c.faces + 3 * (long long)fc;
    if (__ldg(fv) == vtx || __ldg(fv + 1) == vtx || __ldg(fv + 2) == vtx) return false;
  }
  key = pair_key((unsigned)vtx, (unsigned)fc, c.shift);
  return true;
}

// A scanning edge of the edge-edge sweep.
struct EeScan {
  Box6 pb;
  FBox pf;
  double lo;
  int32_t eid, eobj, a0, a1;
  int exclude_self, shift;
  const int32_t* edges;
  SortedBoxes E;
};

__device__ __forceinline__ void ee_scan_at(const BatchBroad& B, unsigned long long i, int s, EeScan& c) {
  const p2c_batch_scene& d = B.scenes[s];
  c.E = scene_view(B, s, 2);
  c.edges = d.edges;
  c.exclude_self = d.exclude_self;
  c.shift = max(1, bit_length_dev(d.ne));
  c.lo = B.S.lo[i];
  c.eid = B.S.id[i];
  c.eobj = B.S.obj[i];
  c.a0 = __ldg(c.edges + 2 * (long long)c.eid);
  c.a1 = __ldg(c.edges + 2 * (long long)c.eid + 1);
  c.pb = box_at(B.S, (long long)i);
  c.pf = fbox_of(c.pb);
}

__device__ __forceinline__ bool ee_test(const EeScan& c, unsigned j, unsigned long long& key) {
  const float4 qf = c.E.fb[j];
  const double qlo = c.E.lo[j];
  const int32_t oid = c.E.id[j];
  const bool own = qlo > c.lo || (qlo == c.lo && oid > c.eid);
  if (!(own && fmay_overlap(c.pf, qf) && overlap3(c.pb, qlo, c.E, j))) return false;
  if (c.E.obj[j] == c.eobj) {
    if (c.exclude_self) return false;
    const int32_t b0 = __ldg(c.edges + 2 * (long long)oid), b1 = __ldg(c.edges + 2 * (long long)oid + 1);
    if (c.a0 == b0 || c.a0 == b1 || c.a1 == b0 || c.a1 == b1) return false;
  }
  key = pair_key((unsigned)min(c.eid, oid), (unsigned)max(c.eid, oid), c.shift);
  return true;
}

// Hand the rest of the current window, from w.j on, to the chunk queue.
// Returns false (the lane walks on by itself) when the queue is full.
__device__ __forceinline__ bool offload_window(StridedWalker& w, const SortedBoxes& Q, unsigned long long box,
                                               uint4* queue, unsigned long long* queue_count,
                                               unsigned long long cap) {
  unsigned b = w.j, e = w.j_end;
  while (b < e) {  // first entry past the window
    const unsigned m = (b + e) >> 1;
    if (Q.q[m] <= w.q_hi) b = m + 1;
    else e = m;
  }
  const unsigned je = b;
  const unsigned long long pieces = (je - w.j + kChunk - 1) / kChunk;
  const unsigned long long base = atomicAdd(queue_count, pieces);
  if (base + pieces > cap) {
    for (unsigned long long k = base; k < cap; ++k) queue[k] = make_uint4(0u, 0u, 0u, 0u);  // empty
    return false;
  }
  for (unsigned long long k = 0; k < pieces; ++k) {
    const unsigned jb = w.j + (unsigned)k * kChunk;
    queue[base + k] = make_uint4((unsigned)box, jb, min(jb + kChunk, je), 0u);
  }
  return true;
}

// Vertex-face pairs, ownership as in the single-scene sweep: a vertex owns
// the pairs whose face minimum is >= its minimum, a face the others.
__device__ __forceinline__ void sweep_vf_slot(const BatchBroad& B, unsigned long long tt, unsigned long long P) {
  const unsigned long long i = tt / kBatchSweepLanes;
  const int lane = (int)(tt % kBatchSweepLanes);
  bool live = false;
  int s = 0;
  bool from_vertex = false;
  if (i < P) {
    const unsigned long long key = sorted_key(B, i);
    const int l = (int)((key >> kBatchListShift) & 3ull);
    live = l <= 1;
    s = (int)(key >> kBatchSceneShift);
    from_vertex = l == 0;
  }
  if (!__any_sync(kFull, live)) return;
  StridedWalker w;
  VfScan c;
  unsigned run = 0;  // entries of the current window tested here
  if (live) {
    vf_scan_at(B, i, s, from_vertex, c);
    const Grid& g = B.sc[s].grid;
    strided_walker_init(w, g, c.lo, c.pb.hi, c.pb.alo, c.pb.ahi, c.pb.blo, c.pb.bhi,
                        from_vertex ? g.reach1[1] : g.reach1[0], from_vertex ? g.reach2[1] : g.reach2[0], lane,
                        kBatchSweepLanes, split_prefix(g, c.pobj));
    live = w.next_cell(c.Q, g);
  }
  for (;;) {
    if (!__any_sync(kFull, live)) break;
    bool found = false;
    unsigned long long key = 0;
    if (live) {
      found = vf_test(c, w.j, key);
      ++w.j;
      if (w.j >= w.j_end || c.Q.q[w.j] > w.q_hi) {
        live = w.next_cell(c.Q, B.sc[s].grid);
        run = 0;
      } else if (++run == kChunk) {
        if (offload_window(w, c.Q, i, B.chunks[0], B.chunk_count + 0, B.chunk_cap)) {
          live = w.next_cell(c.Q, B.sc[s].grid);
          run = 0;
        }
      }
    }
    append_scene_pair(found, s, key, B.pack[0][0], B.off.vf_cap, B.sc, true, B.pair_bits[0]);
  }
}

// Every (kept box, lane) slot, taken 32 at a time by whichever warp is free
// (the number of kept boxes is known only on the device).
__global__ void __launch_bounds__(kThreads, kBatchSweepBlocks) sweep_vf_kernel(BatchBroad B, int dynamic) {
  const unsigned long long n = *B.n_keyed, work = n * kBatchSweepLanes;
  if (!dynamic) {  // one slot per thread, the grid sized for every primitive
    const unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x;
    if (base < work) sweep_vf_slot(B, base + threadIdx.x, n);
    return;
  }
  for (;;) {
    const unsigned long long base = (unsigned long long)next_warp_slots(B.sweep_next + 0);
    if (base >= work) break;
    sweep_vf_slot(B, base + (threadIdx.x & 31), n);
  }
}

// Edge-edge pairs: an edge owns the pairs whose partner minimum is larger
// (ties: larger edge index).
__device__ __forceinline__ void sweep_ee_slot(const BatchBroad& B, unsigned long long tt, unsigned long long P) {
  const unsigned long long i = tt / kBatchSweepLanes;
  const int lane = (int)(tt % kBatchSweepLanes);
  bool live = false;
  int s = 0;
  if (i < P) {
    const unsigned long long key = sorted_key(B, i);
    live = ((key >> kBatchListShift) & 3ull) == 2ull;
    s = (int)(key >> kBatchSceneShift);
  }
  if (!__any_sync(kFull, live)) return;
  StridedWalker w;
  EeScan c;
  unsigned run = 0;
  if (live) {
    ee_scan_at(B, i, s, c);
    const Grid& g = B.sc[s].grid;
    strided_walker_init(w, g, c.lo, c.pb.hi, c.pb.alo, c.pb.ahi, c.pb.blo, c.pb.bhi, g.reach1[2], g.reach2[2], lane,
                        kBatchSweepLanes, split_prefix(g, c.eobj));
    live = w.next_cell(c.E, g);
  }
  for (;;) {
    if (!__any_sync(kFull, live)) break;
    bool found = false;
    unsigned long long key = 0;
    if (live) {
      found = ee_test(c, w.j, key);
      ++w.j;
      if (w.j >= w.j_end || c.E.q[w.j] > w.q_hi) {
        live = w.next_cell(c.E, B.sc[s].grid);
        run = 0;
      } else if (++run == kChunk) {
        if (offload_window(w, c.E, i, B.chunks[1], B.chunk_count + 1, B.chunk_cap)) {
          live = w.next_cell(c.E, B.sc[s].grid);
          run = 0;
        }
      }
    }
    append_scene_pair(found, s, key, B.pack[1][0], B.off.ee_cap, B.sc, false, B.pair_bits[1]);
  }
}

__global__ void __launch_bounds__(kThreads, kBatchSweepBlocks) sweep_ee_kernel(BatchBroad B, int dynamic) {
  const unsigned long long n = *B.n_keyed, work = n * kBatchSweepLanes;
  if (!dynamic) {  // one slot per thread, the grid sized for every primitive
    const unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x;
    if (base < work) sweep_ee_slot(B, base + threadIdx.x, n);
    return;
  }
  for (;;) {
    const unsigned long long base = (unsigned long long)next_warp_slots(B.sweep_next + 1);
    if (base >= work) break;
    sweep_ee_slot(B, base + (threadIdx.x & 31), n);
  }
}

// The queued pieces of long windows, one lane each (at most kChunk entries).
template <int kFamily>
__global__ void __launch_bounds__(kThreads) chunk_kernel(BatchBroad B) {
  const unsigned long long n = min(B.chunk_count[kFamily - 1], B.chunk_cap);
  for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < n;
       base += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long k = base + threadIdx.x;
    uint4 item = make_uint4(0u, 0u, 0u, 0u);
    if (k < n) item = B.chunks[kFamily - 1][k];
    const bool live = item.z > item.y;
    int s = 0;
    VfScan cv;
    EeScan ce;
    if (live) {
      const unsigned long long key = sorted_key(B, item.x);
      s = (int)(key >> kBatchSceneShift);
      if (kFamily == 1) vf_scan_at(B, item.x, s, ((key >> kBatchListShift) & 3ull) == 0ull, cv);
      else ee_scan_at(B, item.x, s, ce);
    }
    for (unsigned t = 0; t < kChunk; ++t) {
      const unsigned j = item.y + t;
      bool found = false;
      unsigned long long key = 0;
      if (live && j < item.z) found = kFamily == 1 ? vf_test(cv, j, key) : ee_test(ce, j, key);
      if (kFamily == 1) append_scene_pair(found, s, key, B.pack[0][0], B.off.vf_cap, B.sc, true, B.pair_bits[0]);
      else append_scene_pair(found, s, key, B.pack[1][0], B.off.ee_cap, B.sc, false, B.pair_bits[1]);
    }
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
  unsigned long long P = 0, V = 0, vf = 0, ee = 0, cells = 0;
  int pair_bits[2] = {2, 2};  // widest packed pair of any scene: vf, ee
};

Totals totals_of(const p2c_batch_scene* h, int n) {
  Totals t;
  for (int s = 0; s < n; ++s) {
    const long long np = h[s].nv + h[s].nf + h[s].ne;
    t.P += (unsigned long long)np;
    t.V += (unsigned long long)h[s].nv;
    t.vf += (unsigned long long)h[s].vf_cap;
    t.ee += (unsigned long long)h[s].ee_cap;
    t.cells += (unsigned long long)cell_budget(np);
    t.pair_bits[0] = std::max(t.pair_bits[0], bit_length(h[s].nv) + std::max(1, bit_length(h[s].nf)));
    t.pair_bits[1] = std::max(t.pair_bits[1], bit_length(h[s].ne) + std::max(1, bit_length(h[s].ne)));
  }
  return t;
}

size_t sort_temp_bytes(const Totals& t) {
  size_t b = 0, c = 0;
  size_t a32 = 0, a64 = 0;
  const int np = (int)std::max<unsigned long long>(t.P, 1ull);
  cub::DeviceRadixSort::SortPairs(nullptr, a32, (const unsigned*)nullptr, (unsigned*)nullptr, (const unsigned*)nullptr,
                                  (unsigned*)nullptr, np);
  cub::DeviceRadixSort::SortPairs(nullptr, a64, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (const unsigned*)nullptr, (unsigned*)nullptr, np);
  const size_t a = std::max(count_sort_scratch_bytes((long long)np), std::max(a32, a64));
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
  B.off.vert = static_cast<unsigned long long*>(take(8 * (size_t)(n + 1)));
  B.cbox = static_cast<double*>(take(48 * P));
  B.cprim = static_cast<unsigned*>(take(4 * P));
  B.keys[0] = static_cast<unsigned long long*>(take(8 * P));
  B.keys[1] = static_cast<unsigned long long*>(take(8 * P));
  B.keys32[0] = reinterpret_cast<unsigned*>(B.keys[0]);
  B.keys32[1] = reinterpret_cast<unsigned*>(B.keys[1]);
  B.key32 = 0;
  B.sorted_buf = 0;
  B.n_keyed = static_cast<unsigned long long*>(take(8));
  B.chunk_count = static_cast<unsigned long long*>(take(16));
  B.sweep_next = static_cast<unsigned long long*>(take(16));
  B.chunk_cap = chunk_cap_for(t.P);
  B.chunks[0] = static_cast<uint4*>(take(16 * B.chunk_cap));
  B.chunks[1] = static_cast<uint4*>(take(16 * B.chunk_cap));
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

// Blocks of a loop over device-counted work: exactly what the device holds at
// once (SMs x resident blocks of this kernel).  All blocks then run side by
// side and each pass of the loop covers one contiguous stretch of the sorted
// entries, so the partners they read stay in the L2 (a larger grid runs its
// blocks in waves that each walk their own far-apart stretches).
template <class K>
unsigned resident_grid(K kernel, const DeviceInfo& info) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return (unsigned)std::max(1, info.sm_count) * (unsigned)per_sm;
}

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
  const int key_bits = kBatchSceneShift + scene_bits;
  B.key32 = key_bits <= 32 ? 1 : 0;  // up to 256 scenes: 32-bit keys halve the key traffic of the sort
  B.pair_bits[0] = t.pair_bits[0];
  B.pair_bits[1] = t.pair_bits[1];
  P2C_CUDA(cudaMemsetAsync(B.sc, 0, sizeof(BroadScratch) * (size_t)n, s));
  P2C_CUDA(cudaMemsetAsync(B.cell_begin, 0, 4 * 3 * (size_t)t.cells, s));
  P2C_CUDA(cudaMemsetAsync(B.cell_end, 0, 4 * 3 * (size_t)t.cells, s));
  P2C_CUDA(cudaMemsetAsync(B.n_keyed, 0, sizeof(unsigned long long), s));
  P2C_CUDA(cudaMemsetAsync(B.chunk_count, 0, 2 * sizeof(unsigned long long), s));
  P2C_CUDA(cudaMemsetAsync(B.sweep_next, 0, 2 * sizeof(unsigned long long), s));
  prep_kernel<<<1, kPrepThreads, 0, s>>>(B);
  P2C_CUDA(cudaGetLastError());
  const unsigned long long P = t.P;
  if (t.V > 0) envelope_kernel<<<grid_for((long long)t.V, kThreads), kThreads, 0, s>>>(B, t.V);
  if (P > 0) cull_kernel<<<grid_for((long long)P, kThreads), kThreads, 0, s>>>(B, P);
  grid_kernel<<<grid_for(n, 128), 128, 0, s>>>(B);
  P2C_CUDA(cudaGetLastError());
  DeviceInfo info;
  int rc = current_device_info(&info);
  if (rc != P2C_OK) return rc;
  bool any_cull = false;
  for (int k = 0; k < n && !any_cull; ++k)
    any_cull = h[k].exclude_self && h[k].n_obj >= 1 && h[k].n_obj <= kMaxCullObjects;
  if (P > 0) {
    // No scene culls: nearly every box is kept, and the library's onesweep
    // sort over all P entries (the others padded to sort last) beats ranking
    // them with the count sort; otherwise only the kept boxes are ranked.
    keys_kernel<<<std::min(grid_for((long long)P, kThreads), resident_grid(keys_kernel, info)), kThreads, 0, s>>>(B, any_cull ? 0ull : P);
    P2C_CUDA(cudaGetLastError());
    bool second = false;
    if (!any_cull) {
      size_t tb = C.tmp_bytes;
      if (B.key32) {
        cub::DoubleBuffer<unsigned> k(B.keys32[0], B.keys32[1]);
        cub::DoubleBuffer<unsigned> v(B.vals[0], B.vals[1]);
        P2C_CUDA(cub::DeviceRadixSort::SortPairs(C.tmp, tb, k, v, (int)P, 0, key_bits, s));
        second = k.selector == 1;
      } else {
        cub::DoubleBuffer<unsigned long long> k(B.keys[0], B.keys[1]);
        cub::DoubleBuffer<unsigned> v(B.vals[0], B.vals[1]);
        P2C_CUDA(cub::DeviceRadixSort::SortPairs(C.tmp, tb, k, v, (int)P, 0, key_bits, s));
        second = k.selector == 1;
      }
    } else {
      rc = B.key32 ? count_sort_pairs(B.keys32[0], B.vals[0], B.keys32[1], B.vals[1], B.n_keyed, (long long)P,
                                      key_bits, C.tmp, C.tmp_bytes, s, &second)
                   : count_sort_pairs(B.keys[0], B.vals[0], B.keys[1], B.vals[1], B.n_keyed, (long long)P, key_bits,
                                      C.tmp, C.tmp_bytes, s, &second);
      if (rc != P2C_OK) return rc;
    }
    B.sorted_buf = second ? 1 : 0;
    gather_kernel<<<std::min(grid_for((long long)P, kThreads), resident_grid(gather_kernel, info)), kThreads, 0,
                    s>>>(B);
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
    // with culling (often a few per cent kept) warps take sweep slots from a
    // counter over a resident grid; without, one slot per thread over a grid
    // for every primitive (faster on dense sheets: no slot fetches)
#ifdef P2C_BATCH_SWEEP_DYNAMIC
    const int dynamic = P2C_BATCH_SWEEP_DYNAMIC;
#else
    const int dynamic = any_cull ? 1 : 0;
#endif
    const unsigned slots = grid_for((long long)P * kBatchSweepLanes, kThreads);
    const unsigned vf_grid = dynamic ? std::min(slots, resident_grid(sweep_vf_kernel, info)) : slots;
    const unsigned ee_grid = dynamic ? std::min(slots, resident_grid(sweep_ee_kernel, info)) : slots;
    if (t.vf > 0) sweep_vf_kernel<<<vf_grid, kThreads, 0, s>>>(B, dynamic);
    if (t.ee > 0) sweep_ee_kernel<<<ee_grid, kThreads, 0, s>>>(B, dynamic);
    if (t.vf > 0) chunk_kernel<1><<<resident_grid(chunk_kernel<1>, info), kThreads, 0, s>>>(B);
    if (t.ee > 0) chunk_kernel<2><<<resident_grid(chunk_kernel<2>, info), kThreads, 0, s>>>(B);
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
