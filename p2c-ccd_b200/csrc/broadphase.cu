// broadphase.cu — swept-AABB candidate generation by a column-subdivided
// sweep-and-prune.
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
// A one-axis sweep over a surface mesh scans windows of ~sqrt(n) boxes (a
// whole slice of surface projects onto the axis).  Here the two non-sweep
// axes are cut into columns at least as wide as the largest box, each box is
// filed under the column of its min corner, and a box scans only the columns
// its partners' min corners can lie in (at most 3 x 3).  Steps, all on the
// caller's stream without host synchronisation:
//   1. vertex swept boxes (t0 and t1 positions, +thickness): object
//      envelopes (reduced per warp before the atomics) and per-axis
//      statistics;
//   2. swept boxes of every vertex, face and edge and culling: with self
//      pairs excluded, a primitive outside every other object's envelope
//      cannot have a candidate (the scene tool's object-pair permission,
//      PrepareScene :521-545, used as a filter); kept boxes are appended to a
//      compact list, often a few per cent of the scene;
//   3. device-side choice of the sweep axis (smallest mean extent relative to
//      the spread of centres), the column grid and an 8- or 16-bit quantiser
//      of the sweep-axis minimum (by scene size);
//   4. ONE radix sort of the kept boxes, with their count read on the device,
//      on a 24- or 32-bit key (list | column | low field: the quantised
//      minimum, with the object bit of a two-body split; 3 or 4 passes) and a
//      gather into per-list struct-of-arrays;
//   5. sweeps over monotone quantised windows with exact double tests and an
//      ownership rule so that every pair is emitted once; pairs are compacted
//      per warp with a ballot and appended with one atomic per warp.
// Overlapping boxes of different objects imply overlapping object envelopes
// (each box lies inside its object's envelope), so beyond culling only the
// same-object rule remains.
#include <cub/block/block_radix_sort.cuh>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cstdlib>
#include <cmath>

#include "broadphase.cuh"
#include "count_sort.cuh"

namespace p2c {
namespace {

constexpr int kThreads = 256;
constexpr unsigned kFull = 0xffffffffu;
constexpr long long kCountSortMinPrims = 1ll << 20;  // scenes ranked by the count sort when culled

// The size from which a culled scene's kept boxes are ranked by the count
// sort: kCountSortMinPrims, or P2C_COUNT_SORT_MIN_PRIMS (tests set 0 to run
// that path on small scenes).
long long count_sort_min_prims() {
  const char* e = std::getenv("P2C_COUNT_SORT_MIN_PRIMS");
  if (e == nullptr || *e == 0) return kCountSortMinPrims;
  char* end = nullptr;
  const long long v = std::strtoll(e, &end, 10);
  return (end != e && v >= 0) ? v : kCountSortMinPrims;
}

inline unsigned grid_for(long long n, int threads) {
  const long long g = (n + threads - 1) / threads;
  return (unsigned)(g > 0 ? g : 1);
}

struct Lists {
  long long off[4];  // global index g: list l holds [off[l], off[l + 1])
  const int32_t* prim[3];
  const int32_t* obj[3];
  __device__ __forceinline__ int list_of(long long g) const { return g < off[1] ? 0 : (g < off[2] ? 1 : 2); }
};

// Block sums of the per-axis statistics that choose the sweep axis (extents,
// centres and squared centres of the boxes), ten atomics per block.
__device__ __forceinline__ void axis_stats(const double b[6], bool live, BroadScratch* sc) {
  __shared__ double red[9][kThreads / 32];
  const int lane = threadIdx.x & 31;
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
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    double v = vals[k];
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v += __shfl_down_sync(kFull, v, s);
    if (lane == 0) red[k][threadIdx.x >> 5] = v;
  }
  const unsigned cnt = __popc(__ballot_sync(kFull, live));
  __syncthreads();
  if (threadIdx.x < 9) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) s += red[threadIdx.x][w];
    double* dst = threadIdx.x < 3 ? &sc->extent_sum[threadIdx.x]
                  : threadIdx.x < 6 ? &sc->center_sum[threadIdx.x - 3]
                                    : &sc->center_sq_sum[threadIdx.x - 6];
    atomicAdd(dst, s);
  }
  if (lane == 0 && cnt) atomicAdd(&sc->count, (unsigned long long)cnt);
}

// Vertex swept boxes (Extend/Expand/SweptPointBox,
// scene_object_envelope_native_ti_walltime.cpp:256-301): each joins its
// object's envelope (the union of the object's vertex boxes; one atomic per
// object per warp) and the per-axis statistics that choose the sweep axis.
// Faces and edges are boxes of these vertices, so this pass also finds
// every non-finite coordinate.
__global__ void __launch_bounds__(kThreads) envelope_kernel(const double* __restrict__ v_t0,
                                                            const double* __restrict__ v_t1,
                                                            const int32_t* __restrict__ v_obj, long long nv,
                                                            double thickness, int cull_objects, BroadScratch* sc) {
  pdl_wait();
  pdl_trigger();
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  double b[6] = {0, 0, 0, 0, 0, 0};
  const bool live = g < nv;
  int o = -1;
  if (live) {
    if (!swept_box<1>(v_t0, v_t1, nullptr, g, thickness, b)) atomicOr(&sc->error_word, 1ull);
    o = v_obj[g];
  }
  if (cull_objects > 0) {
    const bool mine0 = live && o >= 0 && o < cull_objects;
    unsigned remaining = __ballot_sync(kFull, mine0);
    while (remaining) {
      const int leader = __ffs((int)remaining) - 1;
      const int lo_obj = __shfl_sync(kFull, o, leader);
      const bool mine = mine0 && o == lo_obj;
      remaining &= ~__ballot_sync(kFull, mine);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        unsigned long long kmin = mine ? order_key(b[a]) : ~0ull;
        unsigned long long kmax = mine ? order_key(b[3 + a]) : 0ull;
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
          kmin = min(kmin, __shfl_xor_sync(kFull, kmin, s));
          kmax = max(kmax, __shfl_xor_sync(kFull, kmax, s));
        }
        if (lane == leader) {
          atomicMax(&sc->obj_nlo[lo_obj][a], ~kmin);
          atomicMax(&sc->obj_hi[lo_obj][a], kmax);
        }
      }
    }
  }
#ifndef P2C_STATS_ALL
  axis_stats(b, live, sc);
#endif
}

// Sweep axis, column grid, sweep-axis quantiser and list segments, by one
// thread of the last block of the cull launch.  two_body: self pairs are
// excluded and the scene has two objects, so the keys split by object unless
// an id other than 0 and 1 was kept.
__device__ void compute_grid(BroadScratch* sc, int qbits, int two_body) {
  const double n = sc->count > 0 ? (double)sc->count : 1.0;
  int axis = 0;
  double best = INFINITY;
  for (int a = 0; a < 3; ++a) {
    const double mean = sc->center_sum[a] / n;
    const double var = fmax(sc->center_sq_sum[a] / n - mean * mean, 0.0);
    const double score = (sc->extent_sum[a] / n) / (sqrt(var) + 1e-300);
    if (score < best) {
      best = score;
      axis = a;
    }
  }
  Grid g;
#ifdef P2C_FORCE_AXIS
  axis = P2C_FORCE_AXIS;
#endif
  g.axis = axis;
  g.a1 = axis == 0 ? 1 : 0;
  g.a2 = axis == 2 ? 1 : 2;
  g.qbits = qbits;
  const bool split = two_body != 0 && __ldcg(&sc->obj_other) == 0ull;
  g.split_shift = split ? qbits - 1 : -1;
  g.qmax = (1u << (split ? qbits - 1 : qbits)) - 1u;
  const int ax[3] = {g.a1, g.a2, axis};
  // the kept boxes' counts and extents, summed by every block of the cull
  // launch (read past L1)
  unsigned long long active[3], ext_max[3][3], lo_min[3][3], hi_max[3][3];
  for (int l = 0; l < 3; ++l) {
    active[l] = __ldcg(&sc->list[l].active);
    for (int a = 0; a < 3; ++a) {
      ext_max[l][a] = __ldcg(&sc->list[l].ext_max[a]);
      lo_min[l][a] = ~__ldcg(&sc->list[l].nlo_min[a]);
      hi_max[l][a] = __ldcg(&sc->list[l].hi_max[a]);
    }
  }
  double base[3], inv[3];
  int cols[2] = {1, 1};
  for (int k = 0; k < 3; ++k) {
    double lo = INFINITY, hi = -INFINITY, reach = 0.0;
    for (int l = 0; l < 3; ++l) {
      const double r = active[l] ? __longlong_as_double((long long)ext_max[l][ax[k]]) : 0.0;
      if (k < 2) (k == 0 ? g.reach1 : g.reach2)[l] = r;
      if (active[l] == 0) continue;
      lo = fmin(lo, unorder_key(lo_min[l][ax[k]]));
      hi = fmax(hi, unorder_key(hi_max[l][ax[k]]));
      reach = fmax(reach, r);
    }
    const double range = (hi > lo) ? hi - lo : 0.0;
    base[k] = isfinite(lo) ? lo : 0.0;
    if (k < 2) {
      double width = fmax(reach, range / kMaxColumns);
      if (!(width > 0.0) || !isfinite(width)) width = 1.0;
      int c = (int)fmin((double)kMaxColumns, floor(range / width) + 1.0);
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
  g.seg[1] = active[0];
  g.seg[2] = g.seg[1] + active[1];
  g.seg[3] = g.seg[2] + active[2];
  sc->grid = g;
}

__global__ void grid_kernel(BroadScratch* sc, int qbits, int two_body) {
  pdl_wait();
  pdl_trigger();
  compute_grid(sc, qbits, two_body);
}

// Every primitive's swept box (Swept*Box, :256-301), kept unless it is a
// vertex in no face or (self pairs excluded) it lies outside every other
// object's envelope.  Kept boxes are appended (one atomic per warp) to a
// compact list of (box, primitive) entries that everything after works on;
// their extents per list size the column grid.
__global__ void __launch_bounds__(kThreads) cull_kernel(const double* __restrict__ v_t0,
                                                        const double* __restrict__ v_t1, Lists L, double thickness,
                                                        int cull_objects, int ordered, double* __restrict__ cbox,
                                                        unsigned* __restrict__ cprim, BroadScratch* sc, int qbits,
                                                        int two_body) {
  pdl_wait();
  pdl_trigger();
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool keep = false, other = false;
  int l = 3;
  double b[6] = {0, 0, 0, 0, 0, 0};
  if (g < L.off[3]) {
    l = L.list_of(g);
    const long long i = g - L.off[l];
    const int o = L.obj[l][i];
    keep = !(l == 0 && o < 0);
    if (l == 0) swept_box<1>(v_t0, v_t1, nullptr, i, thickness, b);
    else if (l == 1) swept_box<3>(v_t0, v_t1, L.prim[1], i, thickness, b);
    else swept_box<2>(v_t0, v_t1, L.prim[2], i, thickness, b);
    if (keep && cull_objects > 0) {
      bool near_other = false;
      for (int q = 0; q < cull_objects && !near_other; ++q) {
        if (q == o || sc->obj_hi[q][0] == 0ull) continue;
        bool ov = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double olo = unorder_key(~sc->obj_nlo[q][a]), ohi = unorder_key(sc->obj_hi[q][a]);
          ov = ov && b[a] <= ohi && olo <= b[3 + a];
        }
        near_other = ov;
      }
      keep = near_other;
    }
    other = keep && o != 0 && o != 1;
  }
  if (__any_sync(kFull, other) && (threadIdx.x & 31) == 0) atomicOr(&sc->obj_other, 1ull);
  if (ordered) {
    // nothing is culled: every entry in place, in primitive order (a vertex
    // in no face marked), so the sort ranks equal keys by primitive and the
    // order of the sorted lists does not depend on the order warps ran in
    if (g < L.off[3]) {
      double* dst = cbox + 6 * g;
#pragma unroll
      for (int k = 0; k < 6; ++k) dst[k] = b[k];
      cprim[g] = keep ? (unsigned)g : ~0u;
    }
  } else {
    const unsigned m = __ballot_sync(kFull, keep);
    if (m != 0u) {
      const int lane = threadIdx.x & 31;
      const int leader = __ffs((int)m) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(&sc->keyed, (unsigned long long)__popc(m));
      base = __shfl_sync(kFull, base, leader);
      if (keep) {
        const unsigned long long c = base + (unsigned long long)__popc(m & ((1u << lane) - 1u));
        double* dst = cbox + 6 * c;
#pragma unroll
        for (int k = 0; k < 6; ++k) dst[k] = b[k];
        cprim[c] = (unsigned)g;
      }
    }
  }
  // per-list reductions; most warps hold one list only
  const int l0 = __shfl_sync(kFull, l, 0);
  const bool uniform = __all_sync(kFull, l == l0);
  for (int ll = 0; ll < 3; ++ll) {
    if (uniform && ll != l0) continue;
    const bool mine = keep && l == ll;
    const unsigned mask = __ballot_sync(kFull, mine);
    if (mask == 0u) continue;
    ListStats& S = sc->list[ll];
    if ((threadIdx.x & 31) == 0) atomicAdd(&S.active, (unsigned long long)__popc(mask));
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      unsigned long long ext = mine ? (unsigned long long)__double_as_longlong(b[3 + a] - b[a]) : 0ull;
      unsigned long long lo = mine ? order_key(b[a]) : ~0ull;
      unsigned long long hi = mine ? order_key(b[3 + a]) : 0ull;
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) {
        ext = max(ext, __shfl_xor_sync(kFull, ext, s));
        lo = min(lo, __shfl_xor_sync(kFull, lo, s));
        hi = max(hi, __shfl_xor_sync(kFull, hi, s));
      }
      if ((threadIdx.x & 31) == 0) {
        atomicMax(&S.ext_max[a], ext);
        atomicMax(&S.nlo_min[a], ~lo);
        atomicMax(&S.hi_max[a], hi);
      }
    }
  }
#ifdef P2C_STATS_ALL
  axis_stats(b, g < L.off[3], sc);
#endif
  // the last block to finish sizes the grid from everyone's sums
  __shared__ bool last_block;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last_block = atomicAdd(&sc->blocks_done, 1u) == gridDim.x - 1u;
  }
  __syncthreads();
  if (last_block && threadIdx.x == 0) {
    __threadfence();
    compute_grid(sc, qbits, two_body);
  }
}


// Sort key of every kept box (compact entry c, value c).  The order of the
// compact entries does not matter: they are sorted on their full keys and
// the pairs are sorted at the end.
// With pad_to > 0 the entries [kept, pad_to) get the key ~0, which sorts
// after every box (its list field, 3, names no list): a sort sized on the
// host then ranks them last.
__global__ void __launch_bounds__(kThreads) keys_kernel(Lists L, const double* __restrict__ cbox,
                                                        const unsigned* __restrict__ cprim,
                                                        unsigned* __restrict__ keys, unsigned* __restrict__ vals,
                                                        const BroadScratch* sc, unsigned long long pad_to,
                                                        int ordered) {
  pdl_wait();
  pdl_trigger();
  const Grid& G = sc->grid;
  // ordered: entries [0, pad_to) in primitive order, culled ones marked ~0;
  // else the first sc->keyed entries are kept boxes and the rest, up to
  // pad_to, padding
  const unsigned long long n = ordered ? pad_to : sc->keyed;
  for (unsigned long long c = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; c < pad_to;
       c += (unsigned long long)gridDim.x * blockDim.x)
    if (c >= n) {
      keys[c] = ~0u;
      vals[c] = (unsigned)c;
    }
  for (unsigned long long c = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (unsigned long long)gridDim.x * blockDim.x) {
    if (cprim[c] == ~0u) {
      keys[c] = ~0u;
      vals[c] = (unsigned)c;
      continue;
    }
    const long long g = cprim[c];
    const int l = L.list_of(g);
    const double* b = cbox + 6 * c;
    const unsigned cell = (unsigned)(column(b[G.a1], G.base1, G.inv1, G.g1) * G.g2 +
                                     column(b[G.a2], G.base2, G.inv2, G.g2));
    const int32_t o = G.split_shift >= 0 ? L.obj[l][g - L.off[l]] : 0;
    keys[c] = ((unsigned)l << (kCellBits + G.qbits)) | (cell << G.qbits) | split_field(G, o, quantise(b[G.axis], G));
    vals[c] = (unsigned)c;
  }
}

// Sorted entries into per-list struct-of-arrays plus the column ranges.
__global__ void __launch_bounds__(kThreads) gather_kernel(Lists L, const double* __restrict__ cbox,
                                                          const unsigned* __restrict__ cprim,
                                                          const unsigned* __restrict__ keys,
                                                          const unsigned* __restrict__ order, SortedBoxes s0,
                                                          SortedBoxes s1, SortedBoxes s2, const BroadScratch* sc) {
  pdl_wait();
  pdl_trigger();
  const Grid& G = sc->grid;
  const long long n = (long long)G.seg[3];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned key = keys[i];
    const int l = (int)(key >> (kCellBits + G.qbits));
    const SortedBoxes s = l == 0 ? s0 : (l == 1 ? s1 : s2);
    const long long k = i - (long long)G.seg[l];
    const unsigned c = order[i];
    const long long j = (long long)cprim[c] - L.off[l];
    const double* b = cbox + 6 * (long long)c;
    s.lo[k] = b[G.axis];
    s.hi[k] = b[3 + G.axis];
    s.alo[k] = b[G.a1];
    s.ahi[k] = b[3 + G.a1];
    s.blo[k] = b[G.a2];
    s.bhi[k] = b[3 + G.a2];
    s.q[k] = key & ((1u << G.qbits) - 1u);  // quantised min, with the object bit when split
    s.fb[k] = fbox_entry(b[G.a1], b[3 + G.a1], b[G.a2], b[3 + G.a2]);
    s.id[k] = (int32_t)j;
    s.obj[k] = L.obj[l][j];
    const unsigned head = key >> G.qbits;  // list and column
    const unsigned cell = head & ((1u << kCellBits) - 1u);
    if (i == (long long)G.seg[l] || (keys[i - 1] >> G.qbits) != head) s.cell_begin[cell] = (unsigned)k;
    if (i + 1 == (long long)G.seg[l + 1] || (keys[i + 1] >> G.qbits) != head) s.cell_end[cell] = (unsigned)(k + 1);
  }
}

// Warp-aggregated append of the pairs found by this iteration.
__device__ __forceinline__ void append_pair(bool found, unsigned long long key, unsigned long long* out,
                                            unsigned long long cap, unsigned long long* count) {
  const unsigned mask = __ballot_sync(kFull, found);
  if (mask == 0u) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs((int)mask) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(mask));
  base = __shfl_sync(kFull, base, leader);
  if (found) {
    const unsigned long long slot = base + (unsigned long long)__popc(mask & ((1u << lane) - 1u));
    if (slot < cap) out[slot] = key;
  }
}

// Lanes that share one scanning box in the scene sweeps (its columns are
// taken in turn): a box's walk is a chain of dependent loads, and splitting
// it shortens the chain and puts more warps on the SMs.
constexpr int kSceneSweepLanes = 8;

// Resident blocks the sweeps are compiled for (registers per thread capped
// to fit): the walks are chains of dependent loads, so warps per SM set
// their speed (the cloth's edge-edge sweep at 54 registers, 4 blocks per SM,
// took twice as long as at 48, 5 blocks).
#ifndef P2C_SWEEP_VF_BLOCKS
#define P2C_SWEEP_VF_BLOCKS 4
#endif
#ifndef P2C_SWEEP_EE_BLOCKS
#define P2C_SWEEP_EE_BLOCKS 5
#endif
constexpr int kSweepVfBlocks = P2C_SWEEP_VF_BLOCKS, kSweepEeBlocks = P2C_SWEEP_EE_BLOCKS;

// Vertex-face pairs: boxes [0, nv) scan faces from a vertex and own the
// pairs whose face minimum is >= the vertex minimum; boxes [nv, nv + nf)
// scan vertices from a face and own the others.  Keys (vertex, face).
__device__ __forceinline__ void sweep_vf_slot(const SortedBoxes& V, const SortedBoxes& F,
                                              const int32_t* __restrict__ faces, int exclude_self, int pack_shift,
                                              unsigned long long* out, unsigned long long cap, BroadScratch* sc,
                                              long long tt) {
  const Grid& g = sc->grid;
  const long long nv = (long long)(g.seg[1] - g.seg[0]), nf = (long long)(g.seg[2] - g.seg[1]);
  const long long t = tt / kSceneSweepLanes;
  const int lane = (int)(tt % kSceneSweepLanes);
  const bool from_vertex = t < nv;
  const long long i = from_vertex ? t : t - nv;
  bool live = from_vertex || i < nf;
  const SortedBoxes P = from_vertex ? V : F;
  const SortedBoxes Q = from_vertex ? F : V;
  StridedWalker w;
  Box6 pb{};
  FBox pf{};
  double lo = 0.0;
  int32_t pid = 0, pobj = 0;
  if (live) {
    lo = P.lo[i];
    pid = P.id[i];
    pobj = P.obj[i];
    pb = box_at(P, i);
    pf = fbox_of(pb);
    strided_walker_init(w, g, lo, pb.hi, pb.alo, pb.ahi, pb.blo, pb.bhi, from_vertex ? g.reach1[1] : g.reach1[0],
                        from_vertex ? g.reach2[1] : g.reach2[0], lane, kSceneSweepLanes, split_prefix(g, pobj));
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
          key = pair_key((unsigned)vtx, (unsigned)fc, pack_shift);
        }
      }
      ++w.j;
      if (w.j >= w.j_end || Q.q[w.j] > w.q_hi) live = w.next_cell(Q, g);
    }
    append_pair(found, key, out, cap, &sc->vf_count);
  }
}

// Every (kept box, lane) slot, taken 32 at a time by whichever warp is free
// (the kept boxes are counted on the device): the warps walk the sorted
// entries in order and none waits on a share fixed in advance.
__global__ void __launch_bounds__(kThreads, kSweepVfBlocks) sweep_vf_kernel(SortedBoxes V, SortedBoxes F,
                                                            const int32_t* __restrict__ faces, int exclude_self,
                                                            int pack_shift, unsigned long long* out,
                                                            unsigned long long cap, BroadScratch* sc, int dynamic) {
  pdl_wait();
  pdl_trigger();
  const long long work = (long long)(sc->grid.seg[2] - sc->grid.seg[0]) * kSceneSweepLanes;
  if (!dynamic) {  // one slot per thread, the grid sized for every entry
    const long long base = (long long)blockIdx.x * blockDim.x;
    if (base < work) sweep_vf_slot(V, F, faces, exclude_self, pack_shift, out, cap, sc, base + threadIdx.x);
    return;
  }
  for (;;) {
    const long long base = next_warp_slots(&sc->sweep_next[0]);
    if (base >= work) break;
    sweep_vf_slot(V, F, faces, exclude_self, pack_shift, out, cap, sc, base + (threadIdx.x & 31));
  }
}

// Edge-edge pairs: each edge scans its own list and owns the pairs whose
// partner minimum is larger (ties: larger edge index).  Keys (lower, higher).
__device__ __forceinline__ void sweep_ee_slot(const SortedBoxes& E, const int32_t* __restrict__ edges,
                                              int exclude_self, int pack_shift, unsigned long long* out,
                                              unsigned long long cap, BroadScratch* sc, long long tt) {
  const Grid& g = sc->grid;
  const long long ne = (long long)(g.seg[3] - g.seg[2]);
  const long long i = tt / kSceneSweepLanes;
  const int lane = (int)(tt % kSceneSweepLanes);
  bool live = i < ne;
  StridedWalker w;
  Box6 pb{};
  FBox pf{};
  double lo = 0.0;
  int32_t eid = 0, eobj = 0, a0 = 0, a1 = 0;
  if (live) {
    lo = E.lo[i];
    eid = E.id[i];
    eobj = E.obj[i];
    a0 = __ldg(edges + 2 * (long long)eid);
    a1 = __ldg(edges + 2 * (long long)eid + 1);
    pb = box_at(E, i);
    pf = fbox_of(pb);
    strided_walker_init(w, g, lo, pb.hi, pb.alo, pb.ahi, pb.blo, pb.bhi, g.reach1[2], g.reach2[2], lane,
                        kSceneSweepLanes, split_prefix(g, eobj));
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
          key = pair_key((unsigned)min(eid, oid), (unsigned)max(eid, oid), pack_shift);
        }
      }
      ++w.j;
      if (w.j >= w.j_end || E.q[w.j] > w.q_hi) live = w.next_cell(E, g);
    }
    append_pair(found, key, out, cap, &sc->ee_count);
  }
}

__global__ void __launch_bounds__(kThreads, kSweepEeBlocks) sweep_ee_kernel(SortedBoxes E, const int32_t* __restrict__ edges,
                                                            int exclude_self, int pack_shift, unsigned long long* out,
                                                            unsigned long long cap, BroadScratch* sc, int dynamic) {
  pdl_wait();
  pdl_trigger();
  const long long work = (long long)(sc->grid.seg[3] - sc->grid.seg[2]) * kSceneSweepLanes;
  if (!dynamic) {  // one slot per thread, the grid sized for every entry
    const long long base = (long long)blockIdx.x * blockDim.x;
    if (base < work) sweep_ee_slot(E, edges, exclude_self, pack_shift, out, cap, sc, base + threadIdx.x);
    return;
  }
  for (;;) {
    const long long base = next_warp_slots(&sc->sweep_next[1]);
    if (base >= work) break;
    sweep_ee_slot(E, edges, exclude_self, pack_shift, out, cap, sc, base + (threadIdx.x & 31));
  }
}

__global__ void fill_u64_kernel(unsigned long long* p, long long n, unsigned long long v) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// Packed (a << shift | b) keys back to (a << 32 | b); padding stays ~0.
__global__ void unpack_pairs_kernel(unsigned long long* p, long long n, int shift) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long k = p[i];
  if (k == ~0ull) return;
  p[i] = ((k >> shift) << 32) | (k & ((1ull << shift) - 1ull));
}

// Pair lists that fit one block are sorted in ONE launch for both families
// (block 0: vertex-face, block 1: edge-edge): padding, a block radix sort of
// the packed keys and the unpack, instead of a fill, a device-wide sort and
// an unpack launch per family.
// 512 threads x 16 keys with 7-bit digits (5 passes over a 34-bit pair key,
// 130 KB of shared memory): measured against 1024 x 8 with 4-, 5- and 6-bit
// digits, the fastest on the two-sphere scene.  Each block sorts only the
// smallest power-of-two tile (512 x 2, 4, 8 or 16 keys) that holds its list's
// count, read on the device, and writes the padding beyond it directly: a
// radix pass costs in proportion to the keys it ranks.
constexpr int kSmallSortThreads = 512;
constexpr int kSmallSortItems = 16;
constexpr int kSmallSortRadixBits = 7;
constexpr long long kSmallSortCap = (long long)kSmallSortThreads * kSmallSortItems;
template <int kItems>
using SmallSortT = cub::BlockRadixSort<unsigned long long, kSmallSortThreads, kItems, cub::NullType,
                                       kSmallSortRadixBits>;
using SmallSort = SmallSortT<kSmallSortItems>;
constexpr size_t kSmallSortSmem =
    std::max(std::max(sizeof(SmallSortT<16>::TempStorage), sizeof(SmallSortT<8>::TempStorage)),
             std::max(sizeof(SmallSortT<4>::TempStorage), sizeof(SmallSortT<2>::TempStorage)));

template <int kItems>
__device__ __forceinline__ void small_sort_tile(unsigned long long* p, long long cap, long long n, int bits, int shift,
                                                unsigned char* smem) {
  typename SmallSortT<kItems>::TempStorage& tmp = *reinterpret_cast<typename SmallSortT<kItems>::TempStorage*>(smem);
  unsigned long long k[kItems];
#pragma unroll
  for (int u = 0; u < kItems; ++u) {
    const long long i = (long long)threadIdx.x * kItems + u;
    k[u] = i < n ? p[i] : ~0ull;
  }
  SmallSortT<kItems>(tmp).Sort(k, 0, bits);  // ~0 padding has every sorted bit set: it sorts last
#pragma unroll
  for (int u = 0; u < kItems; ++u) {
    const long long i = (long long)threadIdx.x * kItems + u;
    if (i < cap) p[i] = k[u] == ~0ull ? ~0ull : ((k[u] >> shift) << 32) | (k[u] & ((1ull << shift) - 1ull));
  }
  for (long long i = (long long)kSmallSortThreads * kItems + threadIdx.x; i < cap; i += kSmallSortThreads)
    p[i] = ~0ull;  // padding beyond the tile
}

__device__ __forceinline__ void export_counts(const BroadScratch* sc, unsigned long long* counts) {
  counts[0] = sc->vf_count;
  counts[1] = sc->ee_count;
  counts[2] = sc->error_word;
  counts[3] = (unsigned long long)sc->grid.axis | ((unsigned long long)sc->grid.g1 << 8) |
              ((unsigned long long)sc->grid.g2 << 24) | (sc->grid.seg[3] << 40);
}

__global__ void __launch_bounds__(kSmallSortThreads) small_sort_pairs_kernel(
    unsigned long long* vf, long long vf_cap, int vf_bits, int vf_shift, unsigned long long* ee, long long ee_cap,
    int ee_bits, int ee_shift, const BroadScratch* sc, unsigned long long* counts) {
  pdl_wait();
  pdl_trigger();
  if (blockIdx.x == 0 && threadIdx.x == 0) export_counts(sc, counts);  // final once the sweeps are done
  extern __shared__ __align__(16) unsigned char smem_sort[];
  const bool is_vf = blockIdx.x == 0;
  unsigned long long* p = is_vf ? vf : ee;
  const long long cap = is_vf ? vf_cap : ee_cap;
  if (p == nullptr || cap <= 0) return;  // uniform per block
  const int bits = is_vf ? vf_bits : ee_bits, shift = is_vf ? vf_shift : ee_shift;
  const long long count = (long long)(is_vf ? sc->vf_count : sc->ee_count);
  const long long n = count < cap ? count : cap;
  if (n <= 2 * kSmallSortThreads) small_sort_tile<2>(p, cap, n, bits, shift, smem_sort);
  else if (n <= 4 * kSmallSortThreads) small_sort_tile<4>(p, cap, n, bits, shift, smem_sort);
  else if (n <= 8 * kSmallSortThreads) small_sort_tile<8>(p, cap, n, bits, shift, smem_sort);
  else small_sort_tile<16>(p, cap, n, bits, shift, smem_sort);
}

__global__ void export_counts_kernel(const BroadScratch* sc, unsigned long long* counts) {
  pdl_wait();
  pdl_trigger();
  export_counts(sc, counts);
}

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

size_t sort_entries_temp_bytes(long long n) {
  size_t bytes = 0;
  cub::DoubleBuffer<unsigned> k(nullptr, nullptr);
  cub::DoubleBuffer<unsigned> v(nullptr, nullptr);
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, k, v, (int)(n > 0 ? n : 1));
  return bytes;
}

size_t sort_keys_temp_bytes(long long n) {
  size_t bytes = 0;
  cub::DoubleBuffer<unsigned long long> k(nullptr, nullptr);
  cub::DeviceRadixSort::SortKeys(nullptr, bytes, k, (int)(n > 0 ? n : 1));
  return bytes;
}

constexpr long long kCells = (long long)kMaxColumns * kMaxColumns;

struct Layout {
  BroadScratch* sc;
  BoxList B[3];  // vertices, faces, edges
  double* cbox;     // kept boxes, compaction order
  unsigned* cprim;  // their primitive indices
  void* cs_scratch;
  size_t cs_bytes;
  unsigned* keys[2];
  unsigned* vals[2];
  unsigned* cells;  // 3 lists x (begin, end) x kCells
  void* sort_tmp;
  size_t sort_tmp_bytes;
  unsigned long long* pair_alt;
  size_t total;
};

void carve_list(Carver& c, BoxList& L, long long n) {
  L.n = n;
  L.s.lo = c.take<double>(n);
  L.s.hi = c.take<double>(n);
  L.s.alo = c.take<double>(n);
  L.s.ahi = c.take<double>(n);
  L.s.blo = c.take<double>(n);
  L.s.bhi = c.take<double>(n);
  L.s.q = c.take<unsigned>(n);
  L.s.fb = c.take<float4>(n);
  L.s.id = c.take<int32_t>(n);
  L.s.obj = c.take<int32_t>(n);
}

Layout carve(void* base, long long nv, long long nf, long long ne, long long pair_cap, bool dry) {
  Carver c{static_cast<char*>(base), 0, dry};
  Layout L;
  const long long n = nv + nf + ne;
  L.sc = c.take<BroadScratch>(1);
  carve_list(c, L.B[0], nv);
  carve_list(c, L.B[1], nf);
  carve_list(c, L.B[2], ne);
  L.cbox = c.take<double>(6 * n);
  L.cprim = c.take<unsigned>(n);
  L.cs_bytes = count_sort_scratch_bytes(n);
  L.cs_scratch = c.take<char>((long long)L.cs_bytes);
  L.keys[0] = c.take<unsigned>(n);
  L.keys[1] = c.take<unsigned>(n);
  L.vals[0] = c.take<unsigned>(n);
  L.vals[1] = c.take<unsigned>(n);
  L.cells = c.take<unsigned>(6 * kCells);
  for (int l = 0; l < 3; ++l) {
    L.B[l].s.cell_begin = dry ? nullptr : L.cells + (2 * l) * kCells;
    L.B[l].s.cell_end = dry ? nullptr : L.cells + (2 * l + 1) * kCells;
  }
  L.sort_tmp_bytes = std::max(sort_entries_temp_bytes(n), sort_keys_temp_bytes(pair_cap));
  L.sort_tmp = c.take<char>((long long)L.sort_tmp_bytes);
  L.pair_alt = c.take<unsigned long long>(pair_cap);
  L.total = c.off + 256;
  return L;
}

int bit_length(long long x) {
  int b = 0;
  while (x > 0) {
    ++b;
    x >>= 1;
  }
  return b;
}

int sort_pairs(unsigned long long* pairs, long long cap, int key_bits, const Layout& lay, cudaStream_t s) {
  if (cap <= 1) return P2C_OK;
  cub::DoubleBuffer<unsigned long long> k(pairs, lay.pair_alt);
  size_t tb = lay.sort_tmp_bytes;
  P2C_CUDA(cub::DeviceRadixSort::SortKeys(lay.sort_tmp, tb, k, (int)cap, 0, key_bits, s));
  if (k.Current() != pairs)
    P2C_CUDA(cudaMemcpyAsync(pairs, k.Current(), sizeof(unsigned long long) * cap, cudaMemcpyDeviceToDevice, s));
  return P2C_OK;
}

}  // namespace

int validate_scene(const p2c_scene* sc) {
  if (sc == nullptr) return fail(P2C_ERR_INVALID, "scene pointer is null");
  if (sc->nv < 0 || sc->nf < 0 || sc->ne < 0) return fail(P2C_ERR_INVALID, "scene counts must be non-negative");
  if (sc->nv + sc->nf + sc->ne >= (1ll << 31)) return fail(P2C_ERR_INVALID, "scene primitive count must stay below 2^31");
  if (!(sc->thickness >= 0.0) || !std::isfinite(sc->thickness))
    return fail(P2C_ERR_INVALID, "scene thickness must be finite and non-negative");
  if (sc->n_obj < 0) return fail(P2C_ERR_INVALID, "scene n_obj must be non-negative");
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

// A second stream (per host thread and device) the vertex-face and edge-edge
// sweeps fork onto: both read the sorted boxes and append to their own pair
// lists, so they run side by side and fill each other's tail waves.  Created
// outside stream capture only; while none exists the sweeps run in order.
struct SweepFork {
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

SweepFork* sweep_fork(cudaStream_t s) {
  constexpr int kMaxDevices = 64;
  static thread_local SweepFork forks[kMaxDevices];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  SweepFork& f = forks[dev];
  if (f.stream == nullptr) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return nullptr;
    if (cudaStreamCreateWithFlags(&f.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&f.join, cudaEventDisableTiming) != cudaSuccess) {
      f.stream = nullptr;
      return nullptr;
    }
  }
  return &f;
}

// Candidate generation; counts_dev receives {vf_count, ee_count, error_word,
// axis | g1 << 8 | g2 << 24 | kept boxes << 40}.
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

int launch_broadphase(const p2c_scene& scene, unsigned long long* vf_out, long long vf_cap,
                      unsigned long long* ee_out, long long ee_cap, unsigned long long* counts_dev, bool sort_out,
                      void* ws, size_t ws_bytes, cudaStream_t s) {
  const long long pair_cap = std::max(vf_cap, ee_cap);
  const size_t need = broadphase_workspace_bytes(scene.nv, scene.nf, scene.ne, pair_cap);
  if (ws == nullptr || ws_bytes < need)
    return fail(P2C_ERR_INVALID, "candidate workspace too small: %zu < %zu bytes", ws_bytes, need);
  Layout L = carve(ws, scene.nv, scene.nf, scene.ne, pair_cap, false);
  const long long n = scene.nv + scene.nf + scene.ne;
  const int cull = (scene.exclude_self && scene.n_obj >= 1 && scene.n_obj <= kMaxCullObjects) ? scene.n_obj : 0;
  const bool ordered = cull == 0;  // nothing culled: entries stay in primitive order, no compaction
  Lists lists;
  lists.off[0] = 0;
  lists.off[1] = scene.nv;
  lists.off[2] = scene.nv + scene.nf;
  lists.off[3] = n;
  lists.prim[0] = nullptr;
  lists.prim[1] = scene.faces;
  lists.prim[2] = scene.edges;
  lists.obj[0] = scene.v_obj;
  lists.obj[1] = scene.f_obj;
  lists.obj[2] = scene.e_obj;
  DeviceInfo info;
  int rc = current_device_info(&info);
  if (rc != P2C_OK) return rc;
  P2C_CUDA(cudaMemsetAsync(L.sc, 0, sizeof(BroadScratch), s));
  P2C_CUDA(cudaMemsetAsync(L.cells, 0, sizeof(unsigned) * 6 * kCells, s));
  if (scene.nv > 0)
    P2C_CUDA(launch_pdl(envelope_kernel, dim3(grid_for(scene.nv, kThreads)), dim3(kThreads), 0, s, scene.v_t0,
                        scene.v_t1, scene.v_obj, (long long)scene.nv, scene.thickness, cull, L.sc));
  const int qbits = n <= kSmallSceneQPrims ? kQBitsSmall : kQBitsLarge;
  const int two_body = scene.exclude_self && scene.n_obj == 2 ? 1 : 0;
  if (n > 0)
    P2C_CUDA(launch_pdl(cull_kernel, dim3(grid_for(n, kThreads)), dim3(kThreads), 0, s, scene.v_t0, scene.v_t1,
                        lists, scene.thickness, cull, ordered ? 1 : 0, L.cbox, L.cprim, L.sc, qbits, two_body));
  else  // no primitive, no cull launch: the (empty) grid on its own
    P2C_CUDA(launch_pdl(grid_kernel, dim3(1), dim3(1), 0, s, L.sc, qbits, two_body));
  if (n > 0) {
    const unsigned loop_grid = std::min(grid_for(n, kThreads), resident_grid(gather_kernel, info));
    // The library's onesweep sort over all n entries (the culled ones padded
    // to sort last) unless culling applies to a scene of more than
    // kCountSortMinPrims primitives: then the kept boxes, often a few per
    // cent, are ranked alone by the count sort.  Below that size the count
    // sort's twelve launches cost more than ranking every entry (two 40,960-
    // triangle spheres: 92 us against 56 us cold for 4,464 kept of 245,764).
    const bool all_entries = ordered || n < count_sort_min_prims();
    P2C_CUDA(launch_pdl(keys_kernel, dim3(loop_grid), dim3(kThreads), 0, s, lists, (const double*)L.cbox,
                        (const unsigned*)L.cprim, L.keys[0], L.vals[0], (const BroadScratch*)L.sc,
                        (unsigned long long)(all_entries ? n : 0), ordered ? 1 : 0));
    int b = 0;
    if (all_entries) {
      cub::DoubleBuffer<unsigned> k(L.keys[0], L.keys[1]);
      cub::DoubleBuffer<unsigned> v(L.vals[0], L.vals[1]);
      size_t tb = L.sort_tmp_bytes;
      P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.sort_tmp, tb, k, v, (int)n, 0, kCellBits + qbits + 2, s));
      b = k.selector;
    } else {
      bool second = false;
      rc = count_sort_pairs(L.keys[0], L.vals[0], L.keys[1], L.vals[1], &L.sc->keyed, n, kCellBits + qbits + 2,
                            L.cs_scratch, L.cs_bytes, s, &second);
      if (rc != P2C_OK) return rc;
      b = second ? 1 : 0;
    }
    P2C_CUDA(launch_pdl(gather_kernel, dim3(loop_grid), dim3(kThreads), 0, s, lists, (const double*)L.cbox,
                        (const unsigned*)L.cprim, (const unsigned*)L.keys[b], (const unsigned*)L.vals[b], L.B[0].s,
                        L.B[1].s, L.B[2].s, (const BroadScratch*)L.sc));
  }
  // with sorting, pairs are emitted packed so that the sort touches fewer bits
  const int vf_shift = sort_out ? std::max(1, bit_length(scene.nf)) : 0;
  const int ee_shift = sort_out ? std::max(1, bit_length(scene.ne)) : 0;
  const bool small_sort = sort_out && vf_cap <= kSmallSortCap && ee_cap <= kSmallSortCap;
  if (sort_out && !small_sort && vf_cap > 0)
    fill_u64_kernel<<<grid_for(vf_cap, 256), 256, 0, s>>>(vf_out, vf_cap, ~0ull);
  if (sort_out && !small_sort && ee_cap > 0)
    fill_u64_kernel<<<grid_for(ee_cap, 256), 256, 0, s>>>(ee_out, ee_cap, ~0ull);
  const bool do_vf = scene.nv + scene.nf > 0 && vf_out != nullptr;
  const bool do_ee = scene.ne > 0 && ee_out != nullptr;
  // Sweep slots: with culling (often a few per cent of the boxes kept) warps
  // take them 32 at a time from a counter over a resident grid; without, one
  // slot per thread over a grid for every entry.
#ifdef P2C_SWEEP_DYNAMIC
  const int dynamic = P2C_SWEEP_DYNAMIC;
#else
  const int dynamic = ordered ? 0 : 1;
#endif
  auto sweep_blocks = [&](auto kernel, long long slots) -> unsigned {
    const unsigned full = grid_for(slots, kThreads);
    return dynamic ? std::min(full, resident_grid(kernel, info)) : full;
  };
  SweepFork* fk = do_vf && do_ee ? sweep_fork(s) : nullptr;
  cudaStream_t ee_stream = s;
  if (fk != nullptr) {
    P2C_CUDA(cudaEventRecord(fk->fork, s));
    P2C_CUDA(cudaStreamWaitEvent(fk->stream, fk->fork, 0));
    ee_stream = fk->stream;
  }
  if (do_ee)
    P2C_CUDA(launch_pdl(sweep_ee_kernel, dim3(sweep_blocks(sweep_ee_kernel, scene.ne * kSceneSweepLanes)),
                        dim3(kThreads), 0, ee_stream, L.B[2].s, scene.edges, scene.exclude_self, ee_shift, ee_out,
                        (unsigned long long)ee_cap, L.sc, dynamic));
  if (fk != nullptr) P2C_CUDA(cudaEventRecord(fk->join, fk->stream));
  if (do_vf)
    P2C_CUDA(launch_pdl(sweep_vf_kernel, dim3(sweep_blocks(sweep_vf_kernel, (scene.nv + scene.nf) * kSceneSweepLanes)),
                        dim3(kThreads), 0, s, L.B[0].s, L.B[1].s, scene.faces, scene.exclude_self, vf_shift, vf_out,
                        (unsigned long long)vf_cap, L.sc, dynamic));
  if (fk != nullptr) P2C_CUDA(cudaStreamWaitEvent(s, fk->join, 0));
  P2C_CUDA(cudaGetLastError());
  if (small_sort) {
    static bool attr_set = false;  // the block sort's storage is above the 48 KB static limit
    if (!attr_set) {
      P2C_CUDA(cudaFuncSetAttribute(small_sort_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kSmallSortSmem));
      attr_set = true;
    }
    P2C_CUDA(launch_pdl(small_sort_pairs_kernel, dim3(2), dim3(kSmallSortThreads), kSmallSortSmem, s,
                        vf_out, vf_cap, bit_length(scene.nv) + vf_shift, vf_shift, ee_out, ee_cap,
                        bit_length(scene.ne) + ee_shift, ee_shift, (const BroadScratch*)L.sc, counts_dev));
  } else if (sort_out) {
    int rc = sort_pairs(vf_out, vf_cap, bit_length(scene.nv) + vf_shift, L, s);
    if (rc != P2C_OK) return rc;
    rc = sort_pairs(ee_out, ee_cap, bit_length(scene.ne) + ee_shift, L, s);
    if (rc != P2C_OK) return rc;
    if (vf_cap > 0) unpack_pairs_kernel<<<grid_for(vf_cap, 256), 256, 0, s>>>(vf_out, vf_cap, vf_shift);
    if (ee_cap > 0) unpack_pairs_kernel<<<grid_for(ee_cap, 256), 256, 0, s>>>(ee_out, ee_cap, ee_shift);
  }
  if (!small_sort)  // the block sort writes the counts itself
    P2C_CUDA(launch_pdl(export_counts_kernel, dim3(1), dim3(1), 0, s, (const BroadScratch*)L.sc, counts_dev));
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
