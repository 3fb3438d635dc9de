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
constexpr int kQBits = 16;           // quantised sweep-axis minimum
constexpr unsigned kQMax = (1u << kQBits) - 1u;

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
  int32_t* id;    // primitive index in the scene
  int32_t* obj;   // object id
  unsigned* cell_begin;  // [kMaxColumns^2] first entry of each column
  unsigned* cell_end;    // [kMaxColumns^2] one past its last entry
};

struct BoxList {
  long long n = 0;
  double* box = nullptr;  // n x 6 (primitive order)
  SortedBoxes s{};
};

struct ListStats {
  unsigned long long active;     // boxes kept
  unsigned long long ext_max[3]; // bit pattern of the largest extent per axis (non-negative)
  unsigned long long lo_min[3];  // order_key of the smallest min per axis
  unsigned long long hi_max[3];  // order_key of the largest max per axis
};

struct Grid {
  int axis, a1, a2, g1, g2, pad;
  double base1, base2, inv1, inv2;  // column = floor((x - base) * inv)
  double base0, scale0;             // quantiser of the sweep axis: floor((x - base0) * scale0)
  double reach1[3], reach2[3];      // per list: the largest extent along a1 / a2
  unsigned long long seg[4];        // list l's sorted entries are [seg[l], seg[l + 1])
};

struct BroadScratch {
  double extent_sum[3], center_sum[3], center_sq_sum[3];
  unsigned long long count;
  unsigned long long obj_lo[kMaxCullObjects][3];  // order keys of object swept boxes
  unsigned long long obj_hi[kMaxCullObjects][3];
  ListStats list[3];  // 0 vertices, 1 faces, 2 edges
  Grid grid;
  unsigned long long vf_count;
  unsigned long long ee_count;
  unsigned long long error_word;  // bit 0: non-finite coordinate
};

}  // namespace p2c
