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
