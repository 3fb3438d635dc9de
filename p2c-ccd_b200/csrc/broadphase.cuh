// broadphase.cuh — scratch layout of the column-subdivided sweep-and-prune
// (device side of p2c_scene_candidates).
#pragma once

#include <cstdint>

#include "p2c_b200.h"
#include "p2c_internal.cuh"

namespace p2c {

constexpr int kMaxCullObjects = 64;  // object-envelope culling up to this many objects
constexpr int kMaxColumns = 128;     // columns per non-sweep axis (cell id < 2^14)
constexpr int kCellBits = 14;
// Width of the quantised sweep-axis minimum in a scene's sort key
// (list << (14 + q) | cell << q | quantised min): 8 bits keep the key at 24
// bits (3 radix passes) for scenes up to kSmallSceneQPrims primitives, 16
// bits (4 passes) give larger scenes - dense flat sheets above all - tighter
// sweep windows.  Chosen on the host from the primitive count.
constexpr int kQBitsSmall = 8, kQBitsLarge = 16;
constexpr long long kSmallSceneQPrims = 1000000;

// Order-preserving maps to unsigned integers (radix-sortable keys).
__device__ __forceinline__ unsigned long long order_key(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double unorder_key(unsigned long long k) {
  const unsigned long long b = (k & 0x8000000000000000ull) ? (k & ~0x8000000000000000ull) : ~k;
  return __longlong_as_double((long long)b);
}
__device__ __forceinline__ unsigned fkey_bits(float f) {
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
// Float keys that bracket a double: down(x) <= x <= up(x) in key order.
__device__ __forceinline__ unsigned fkey_down(double x) { return fkey_bits(__double2float_rd(x)); }
__device__ __forceinline__ unsigned fkey_up(double x) { return fkey_bits(__double2float_ru(x)); }

// One primitive list in (column, min) order, struct-of-arrays for coalesced scans.
struct SortedBoxes {
  double* lo;     // min along the sweep axis
  double* hi;     // max along the sweep axis
  double* alo;    // min / max along the first non-sweep axis
  double* ahi;
  double* blo;    // min / max along the second non-sweep axis
  double* bhi;
  unsigned* q;    // quantised min along the sweep axis (the sort key's low bits)
  float4* fb;     // the non-sweep bounds rounded outward to float: (alo down, ahi up, blo down, bhi up)
  int32_t* id;    // primitive index in the scene
  int32_t* obj;   // object id
  unsigned* cell_begin;  // [kMaxColumns^2] first entry of each column
  unsigned* cell_end;    // [kMaxColumns^2] one past its last entry
};

struct BoxList {
  long long n = 0;
  SortedBoxes s{};
};

struct ListStats {
  unsigned long long active;     // boxes kept
  unsigned long long ext_max[3]; // bit pattern of the largest extent per axis (non-negative)
  unsigned long long nlo_min[3]; // ~order_key of the smallest min per axis (raised by atomicMax: zero = empty)
  unsigned long long hi_max[3];  // order_key of the largest max per axis
};

struct Grid {
  int axis, a1, a2, g1, g2;
  unsigned qmax;                    // largest quantised value
  int qbits;                        // width of the key's low field (scene keys)
  // Two-body split: with self pairs excluded and exactly two objects (ids 0
  // and 1), the low field is (object << (qbits - 1)) | quantised min, so a
  // column's entries of each object form their own sorted run and a box
  // walks only the other object's run.  split_shift is qbits - 1 then, else
  // -1 (the low field is the quantised min alone).
  int split_shift;
  double base1, base2, inv1, inv2;  // column = floor((x - base) * inv)
  double base0, scale0;             // quantiser of the sweep axis: floor((x - base0) * scale0)
  double reach1[3], reach2[3];      // per list: the largest extent along a1 / a2
  unsigned long long seg[4];        // list l's sorted entries are [seg[l], seg[l + 1])
};

struct BroadScratch {
  double extent_sum[3], center_sum[3], center_sq_sum[3];
  unsigned long long count;
  unsigned long long obj_nlo[kMaxCullObjects][3];  // ~order keys of the objects' swept-box minima (zero = empty)
  unsigned long long obj_hi[kMaxCullObjects][3];
  ListStats list[3];  // 0 vertices, 1 faces, 2 edges
  Grid grid;
  unsigned long long vf_count;
  unsigned long long ee_count;
  unsigned long long error_word;  // bit 0: non-finite coordinate
  unsigned long long obj_other;   // non-zero: a kept primitive's object id is neither 0 nor 1
  unsigned long long keyed;       // single scene: boxes kept after culling (compact entries)
  unsigned long long sweep_next[2];  // single scene: next slot of the vertex-face / edge-edge sweep
  unsigned blocks_done;              // single scene: cull blocks finished (the last sizes the grid)
};

// The next 32 sweep slots for the calling warp (one atomic per warp).
__device__ __forceinline__ long long next_warp_slots(unsigned long long* next) {
  unsigned long long base = 0;
  if ((threadIdx.x & 31) == 0) base = atomicAdd(next, 32ull);
  return (long long)__shfl_sync(0xffffffffu, base, 0);
}

// Prefix of the partner object's run in a split low field (0 unsplit): a
// box of object o (0 or 1) walks the entries of object 1 - o.
__device__ __forceinline__ unsigned split_prefix(const Grid& g, int32_t obj) {
  return g.split_shift >= 0 ? (unsigned)(1 - obj) << g.split_shift : 0u;
}
// The low field of an entry of object obj with quantised min q.
__device__ __forceinline__ unsigned split_field(const Grid& g, int32_t obj, unsigned q) {
  return g.split_shift >= 0 ? ((unsigned)obj << g.split_shift) | q : q;
}


// ---- device helpers shared by the single-scene and batched sweeps ---------
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }  // std::max

// Swept box of a primitive with K vertices (Extend/Expand/Swept*Box,
// scene_object_envelope_native_ti_walltime.cpp:256-301): min/max over the
// t0 and t1 positions, then +-thickness.  Returns false on a non-finite
// coordinate.
template <int K>
__device__ __forceinline__ bool swept_box(const double* __restrict__ v_t0, const double* __restrict__ v_t1,
                                          const int32_t* __restrict__ prim, long long i, double thickness,
                                          double b[6]) {
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
#pragma unroll
  for (int a = 0; a < 3; ++a) {  // Expand(box, thickness), :263-270
    b[a] = __dsub_rn(mn[a], thickness);
    b[3 + a] = __dadd_rn(mx[a], thickness);
  }
  return finite;
}

__device__ __forceinline__ int column(double x, double base, double inv, int g) {
  const double c = floor((x - base) * inv);
  return c < 0.0 ? 0 : (c >= (double)g ? g - 1 : (int)c);
}

// Monotone (non-decreasing) in x: the sweep windows rely on it.
__device__ __forceinline__ unsigned quantise(double x, const Grid& g) {
  const double c = floor((x - g.base0) * g.scale0);
  return c < 0.0 ? 0u : (c >= (double)g.qmax ? g.qmax : (unsigned)c);
}

// Walk over the candidate entries of one scanning box: the columns its
// partners' min corners can lie in, and in each the quantised window
// [q(lo), q(hi)] of the partner list.
struct Walker {
  int c1, c1_end, c2_begin, c2, c2_end;
  unsigned j, j_end, q_lo, q_hi;

  __device__ __forceinline__ bool next_cell(const SortedBoxes& Q, const Grid& g) {
    for (;;) {
      if (++c2 > c2_end) {
        c2 = c2_begin;
        if (++c1 > c1_end) return false;
      }
      const int cell = c1 * g.g2 + c2;
      unsigned b = Q.cell_begin[cell], e = Q.cell_end[cell];
      const unsigned end = e;
      while (b < e) {  // first entry with q >= q_lo
        const unsigned m = (b + e) >> 1;
        if (Q.q[m] < q_lo) b = m + 1;
        else e = m;
      }
      j = b;
      j_end = end;
      if (j < j_end && Q.q[j] <= q_hi) return true;
    }
  }
};

__device__ __forceinline__ void walker_init(Walker& w, const Grid& g, double lo, double hi, double alo, double ahi,
                                            double blo, double bhi, double reach1, double reach2) {
  // widen the lower columns by a relative 2^-40 so that the rounding of
  // alo - reach can never skip the column of a partner's min corner
  const double l1 = alo - reach1 - (fabs(alo) + reach1) * 0x1p-40;
  const double l2 = blo - reach2 - (fabs(blo) + reach2) * 0x1p-40;
  w.c1 = column(l1, g.base1, g.inv1, g.g1);
  w.c1_end = column(ahi, g.base1, g.inv1, g.g1);
  w.c2_begin = column(l2, g.base2, g.inv2, g.g2);
  w.c2_end = column(bhi, g.base2, g.inv2, g.g2);
  w.c2 = w.c2_begin - 1;
  w.j = w.j_end = 0;
  w.q_lo = quantise(lo, g);
  w.q_hi = quantise(hi, g);
}

// The same walk with the columns of one box shared by several lanes: lane l
// of a group of `step` takes columns l, l + step, ... of the box's
// rectangle (row-major over [c1, c1_end] x [c2_begin, c2_end]).
struct StridedWalker {
  int c1a, c2a, n2, n_cells, k, step;
  unsigned j, j_end, q_lo, q_hi;

  __device__ __forceinline__ bool next_cell(const SortedBoxes& Q, const Grid& g) {
    for (;;) {
      k += step;
      if (k >= n_cells) return false;
      const int cell = (c1a + k / n2) * g.g2 + (c2a + k % n2);
      unsigned b = Q.cell_begin[cell], e = Q.cell_end[cell];
      const unsigned end = e;
      while (b < e) {  // first entry with q >= q_lo
        const unsigned m = (b + e) >> 1;
        if (Q.q[m] < q_lo) b = m + 1;
        else e = m;
      }
      j = b;
      j_end = end;
      if (j < j_end && Q.q[j] <= q_hi) return true;
    }
  }
};

__device__ __forceinline__ void strided_walker_init(StridedWalker& w, const Grid& g, double lo, double hi, double alo,
                                                    double ahi, double blo, double bhi, double reach1, double reach2,
                                                    int lane, int step, unsigned prefix) {
  Walker v;
  walker_init(v, g, lo, hi, alo, ahi, blo, bhi, reach1, reach2);
  w.c1a = v.c1;
  w.c2a = v.c2_begin;
  w.n2 = v.c2_end - v.c2_begin + 1;
  w.n_cells = (v.c1_end - v.c1 + 1) * w.n2;
  w.step = step;
  w.k = lane - step;
  w.j = w.j_end = 0;
  w.q_lo = v.q_lo + prefix;
  w.q_hi = v.q_hi + prefix;
}

// A scanning box held in registers for the length of its walk.
struct Box6 {
  double lo, hi, alo, ahi, blo, bhi;
};

__device__ __forceinline__ Box6 box_at(const SortedBoxes& P, long long i) {
  return Box6{P.lo[i], P.hi[i], P.alo[i], P.ahi[i], P.blo[i], P.bhi[i]};
}

// A box's non-sweep bounds rounded outward to float, for the prefilter below.
struct FBox {
  float alo, ahi, blo, bhi;
};

__device__ __forceinline__ FBox fbox_of(const Box6& b) {
  return FBox{__double2float_rd(b.alo), __double2float_ru(b.ahi), __double2float_rd(b.blo), __double2float_ru(b.bhi)};
}

__device__ __forceinline__ float4 fbox_entry(double alo, double ahi, double blo, double bhi) {
  return make_float4(__double2float_rd(alo), __double2float_ru(ahi), __double2float_rd(blo), __double2float_ru(bhi));
}

// Conservative prefilter on the two non-sweep axes from one 16-byte load:
// false only when the double boxes are disjoint there (a lower bound rounded
// down above an upper bound rounded up orders the doubles the same way), so
// every pair the exact test accepts passes it.
__device__ __forceinline__ bool fmay_overlap(const FBox& p, const float4 q) {
  return !(p.alo > q.y || q.x > p.ahi || p.blo > q.w || q.z > p.bhi);
}

// Inclusive overlap on all three axes (Overlap, :270-274); qlo is Q.lo[j],
// already loaded by the caller's ownership test.
__device__ __forceinline__ bool overlap3(const Box6& p, double qlo, const SortedBoxes& Q, long long j) {
  return p.lo <= Q.hi[j] && qlo <= p.hi && p.alo <= Q.ahi[j] && Q.alo[j] <= p.ahi && p.blo <= Q.bhi[j] &&
         Q.blo[j] <= p.bhi;
}

__device__ __forceinline__ unsigned long long pair_key(unsigned a, unsigned b, int pack_shift) {
  return pack_shift > 0 ? (((unsigned long long)a << pack_shift) | b) : (((unsigned long long)a << 32) | b);
}

}  // namespace p2c
