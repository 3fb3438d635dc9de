// broadphase.cuh — scene description and scratch layout of the swept-AABB
// sweep-and-prune (device side of p2c_scene_candidates).
#pragma once

#include <cstdint>

#include "p2c_b200.h"
#include "p2c_internal.cuh"

namespace p2c {

// Order-preserving map of a finite double to uint64 (radix-sortable key).
__device__ __forceinline__ unsigned long long order_key(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

// One primitive list sorted along the sweep axis, struct-of-arrays so that a
// warp scanning consecutive sorted entries issues coalesced loads.
struct SortedBoxes {
  double* lo;   // min along the sweep axis
  double* hi;   // max along the sweep axis
  double* alo;  // min / max along the other two axes
  double* ahi;
  double* blo;
  double* bhi;
  int32_t* id;  // primitive index in the scene
  int32_t* obj; // object id
};

struct BoxList {
  long long n = 0;
  double* box = nullptr;                // n x 6 (unsorted, primitive order)
  unsigned long long* keys[2] = {nullptr, nullptr};
  unsigned int* vals[2] = {nullptr, nullptr};
  SortedBoxes s{};
};

// Per-axis statistics for the device-side choice of the sweep axis.
struct AxisStats {
  double extent_sum[3];
  double center_sum[3];
  double center_sq_sum[3];
  unsigned long long count;
  int axis;
  int pad;
};

struct BroadScratch {
  AxisStats stats;
  unsigned long long vf_count;
  unsigned long long ee_count;
  unsigned long long error_word;  // bit 0: non-finite coordinate
  unsigned long long pad[5];
};

}  // namespace p2c
