// scene_pairs.cuh — certificate geometry gathered straight from a scene's
// vertex/face/edge arrays for one candidate pair (no 240-byte record).
#pragma once

#include "certify_core.cuh"

namespace p2c {

// One family's candidate pairs of a scene over one interval.  A pair key is
// (vertex << 32 | face) for point-triangle and (edge_a << 32 | edge_b) for
// edge-edge, as the broad phase writes them.
struct ScenePairs {
  const double* v_t0;
  const double* v_t1;
  const int32_t* faces;
  const int32_t* edges;
  const unsigned long long* pairs;
  double T0, T1;
};

__device__ __forceinline__ void load_vertex(const ScenePairs& s, long long v, Geo& g, int slot, bool& finite) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double x0 = __ldg(s.v_t0 + 3 * v + a), x1 = __ldg(s.v_t1 + 3 * v + a);
    g.p0[3 * slot + a] = x0;
    g.p1[3 * slot + a] = x1;
    finite = finite && isfinite(x0) && isfinite(x1);
  }
}

// Vertex order of the reference primitives: (point, v0, v1, v2) for family 1,
// (a0, a1, b0, b1) for family 2.  Returns false on a non-finite coordinate.
__device__ __forceinline__ bool load_pair(const ScenePairs& s, int family, unsigned long long key, Geo& g) {
  const long long a = (long long)(key >> 32), b = (long long)(key & 0xffffffffull);
  bool finite = true;
  if (family == 1) {  // point = vertex a, triangle = face b
    load_vertex(s, a, g, 0, finite);
    const int32_t* fc = s.faces + 3 * b;
    load_vertex(s, __ldg(fc), g, 1, finite);
    load_vertex(s, __ldg(fc + 1), g, 2, finite);
    load_vertex(s, __ldg(fc + 2), g, 3, finite);
  } else {  // edge a then edge b
    const int32_t* ea = s.edges + 2 * a;
    const int32_t* eb = s.edges + 2 * b;
    load_vertex(s, __ldg(ea), g, 0, finite);
    load_vertex(s, __ldg(ea + 1), g, 1, finite);
    load_vertex(s, __ldg(eb), g, 2, finite);
    load_vertex(s, __ldg(eb + 1), g, 3, finite);
  }
  return finite;
}

}  // namespace p2c

namespace p2c {

// The seeded scheduler stub: a uniform score in [0, 1) from (seed, family,
// pair key), mixed by the splitmix64 finaliser (Steele, Lea and Flood,
// "Fast splittable pseudorandom number generators", OOPSLA 2014).  It depends
// only on the candidate's identity, so a candidate scores the same alone and
// in any batch, whatever its position in the candidate list.
__host__ __device__ inline double stub_score(unsigned long long seed, int family, unsigned long long key) {
  unsigned long long x = seed ^ (key * 0x9e3779b97f4a7c15ull) ^ ((unsigned long long)family << 62);
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  x ^= x >> 31;
  return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace p2c
