// certify_core.cuh — FP64 interval certifier for sm_100a.
//
// Restates the reference certifier (cpp/certificate/certificate_engine.cpp) so
// that every decision, time of impact and margin is bit-identical:
//  * all arithmetic goes through explicitly rounded intrinsics (__dmul_rn,
//    __dadd_rn, __dsub_rn, __ddiv_rn, __dsqrt_rn), so no FMA contraction can
//    occur whatever the compiler flags; the association order is the one the
//    reference source writes;
//  * std::clamp/min/max are restated with the same comparisons (NaN and signed
//    zero behave as in libstdc++).
//
// Engine: one persistent loop per warp.  A lane owns one interval node at a
// time and walks its subtree depth-first, left child first, with no stack: the
// node is (path bits, depth) and its endpoints are recomputed from the root by
// replaying the bisections (the same 0.5*(a+b) roundings the reference
// recursion performs).  Every non-root node needs only its midpoint sample:
// its endpoints are midpoints or endpoints of ancestors, already known to be
// farther than eps_space (otherwise the ancestor would be a collision leaf).
// When the query queue is empty, idle lanes take the shallowest pending right
// subtree of a busy lane ("donation"), so one grazing query is bisected by up
// to 32 lanes.  Per-query reduction in shared memory reproduces the recursion's
// result exactly: the leftmost collision leaf in depth-first order (smallest
// left-aligned path key) wins; else any undecided leaf makes the query
// undecided; else separation with the minimum leaf margin.  Nodes right of a
// known collision are pruned (the serial recursion never visits them).
#pragma once

#include <cmath>
#include <cstdint>
#include <type_traits>

#include "p2c_b200.h"

namespace p2c {

constexpr double kNumEps = 1.0e-14;  // kNumericalEpsilon, certificate_engine.cpp:20

struct V3 {
  double x, y, z;
};

// Every operation is rounded once, to nearest: the explicitly rounded
// intrinsics on the device; on the host (the library's CPU certifier, built
// with -ffp-contract=off and no FMA target) the plain IEEE operators, which
// round the same way.
#define P2C_HD __host__ __device__ __forceinline__
P2C_HD double mul(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
P2C_HD double add(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
P2C_HD double sub(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
P2C_HD double dvd(double a, double b) {
#ifdef __CUDA_ARCH__
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}
P2C_HD double sqrt_rn(double a) {
#ifdef __CUDA_ARCH__
  return __dsqrt_rn(a);
#else
  return std::sqrt(a);
#endif
}

// ---- optional FP64 operation census ---------------------------------------
struct NoCount {
  static constexpr unsigned long long n = 0;
  P2C_HD void add(int) {}
};
struct OpCount {
  unsigned long long n = 0;
  P2C_HD void add(int k) { n += (unsigned long long)k; }
};


P2C_HD V3 vadd(V3 a, V3 b) { return {add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)}; }
P2C_HD V3 vsub(V3 a, V3 b) { return {sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)}; }
P2C_HD V3 vscale(V3 a, double s) { return {mul(a.x, s), mul(a.y, s), mul(a.z, s)}; }
// a.x*b.x + a.y*b.y + a.z*b.z, left to right
P2C_HD double vdot(V3 a, V3 b) {
  return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z));
}
P2C_HD V3 vcross(V3 a, V3 b) {
  return {sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)),
          sub(mul(a.x, b.y), mul(a.y, b.x))};
}
// std::clamp(v, lo, hi) as libstdc++ evaluates it
P2C_HD double clamp_std(double v, double lo, double hi) {
  return (v < lo) ? lo : ((hi < v) ? hi : v);
}
P2C_HD double max_std(double a, double b) { return (a < b) ? b : a; }
P2C_HD double min_std(double a, double b) { return (b < a) ? b : a; }

template <class C>
P2C_HD double dist_pp(V3 a, V3 b, C& c) {  // :78-80
  c.add(9);
  const V3 d = vsub(a, b);
  return sqrt_rn(vdot(d, d));
}

template <class C>
P2C_HD double dist_point_segment(V3 p, V3 a, V3 b, C& c) {  // :82-90
  const V3 ab = vsub(b, a);
  const double ab2 = vdot(ab, ab);
  c.add(8);
  if (ab2 <= kNumEps) return dist_pp(p, a, c);
  const double t = clamp_std(dvd(vdot(vsub(p, a), ab), ab2), 0.0, 1.0);
  c.add(15);
  return dist_pp(p, vadd(a, vscale(ab, t)), c);
}

// DistancePointTriangle, certificate_engine.cpp:133-184.  The Voronoi region
// is found with the reference's tests, in its order, on the quantities it
// computes; every region then ends in one of three forms: a vertex
// (|p - v|), an edge (v = num / den, |p - (base + dir * v)|) or the face
// (|dot(ap, n) / |n||).  Evaluating the tails after the region is known, one
// form at a time, lets a warp whose lanes sit in different regions issue at
// most one division and two square roots instead of one of each per region
// present; every lane still performs exactly its region's operations, in the
// reference's order, so the value is the same bit for bit.
template <class C>
P2C_HD double dist_point_triangle(V3 p, V3 a, V3 b, V3 cc, C& c) {
  const V3 ab = vsub(b, a);
  const V3 ac = vsub(cc, a);
  const V3 n = vcross(ab, ac);
  c.add(20);
  const double nn2 = vdot(n, n);
  if (nn2 <= kNumEps) {
    double m = dist_point_segment(p, a, b, c);
    const double m1 = dist_point_segment(p, b, cc, c);
    const double m2 = dist_point_segment(p, cc, a, c);
    if (m1 < m) m = m1;  // std::min({...}) keeps the first smallest
    if (m2 < m) m = m2;
    return m;
  }
  const V3 ap = vsub(p, a);
  const double d1 = vdot(ab, ap);
  const double d2 = vdot(ac, ap);
  c.add(13);
  int form;  // 0 vertex, 1 edge, 2 face
  V3 base = a, dir = ab;
  double num = 0.0, den = 1.0;
  if (d1 <= 0.0 && d2 <= 0.0) {
    form = 0;  // vertex a
  } else {
    const V3 bp = vsub(p, b);
    const double d3 = vdot(ab, bp);
    const double d4 = vdot(ac, bp);
    c.add(13);
    if (d3 >= 0.0 && d4 <= d3) {
      form = 0;  // vertex b
      base = b;
    } else {
      const double vc = sub(mul(d1, d4), mul(d3, d2));
      c.add(3);
      if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        form = 1;  // edge ab: v = d1 / (d1 - d3)
        num = d1;
        den = sub(d1, d3);
        c.add(8);
      } else {
        const V3 cp = vsub(p, cc);
        const double d5 = vdot(ab, cp);
        const double d6 = vdot(ac, cp);
        c.add(13);
        if (d6 >= 0.0 && d5 <= d6) {
          form = 0;  // vertex c
          base = cc;
        } else {
          const double vb = sub(mul(d5, d2), mul(d1, d6));
          c.add(3);
          if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
            form = 1;  // edge ac: w = d2 / (d2 - d6)
            dir = ac;
            num = d2;
            den = sub(d2, d6);
            c.add(8);
          } else {
            const double va = sub(mul(d3, d6), mul(d5, d4));
            const double d43 = sub(d4, d3);
            const double d56 = sub(d5, d6);
            c.add(5);
            if (va <= 0.0 && d43 >= 0.0 && d56 >= 0.0) {
              form = 1;  // edge bc: w = d43 / (d43 + d56), from b along c - b
              base = b;
              dir = vsub(cc, b);
              num = d43;
              den = add(d43, d56);
              c.add(11);
            } else {
              form = 2;  // face: dot(ap, n) / |n|
              c.add(12);
            }
          }
        }
      }
    }
  }
  if (form == 2) {
    num = vdot(ap, n);
    den = sqrt_rn(nn2);
  }
  double v = 0.0;
  if (form != 0) v = dvd(num, den);
  if (form == 2) return fabs(v);
  const V3 q = form == 1 ? vadd(base, vscale(dir, v)) : base;
  c.add(9);
  const V3 d = vsub(p, q);
  return sqrt_rn(vdot(d, d));
}

// DistanceSegmentSegment, certificate_engine.cpp:92-131
template <class C>
P2C_HD double dist_segment_segment(V3 p1, V3 q1, V3 p2, V3 q2, C& c) {
  const V3 d1 = vsub(q1, p1);
  const V3 d2 = vsub(q2, p2);
  const V3 r = vsub(p1, p2);
  const double a = vdot(d1, d1);
  const double e = vdot(d2, d2);
  const double f = vdot(d2, r);
  c.add(24);
  double s = 0.0, t = 0.0;
  if (a <= kNumEps && e <= kNumEps) return dist_pp(p1, p2, c);
  if (a <= kNumEps) {
    t = clamp_std(dvd(f, e), 0.0, 1.0);
    c.add(1);
  } else {
    const double cd = vdot(d1, r);
    c.add(5);
    if (e <= kNumEps) {
      s = clamp_std(dvd(-cd, a), 0.0, 1.0);
      c.add(1);
    } else {
      const double b = vdot(d1, d2);
      const double denom = sub(mul(a, e), mul(b, b));
      c.add(8);
      if (denom != 0.0) {
        s = clamp_std(dvd(sub(mul(b, f), mul(cd, e)), denom), 0.0, 1.0);
        c.add(4);
      }
      t = dvd(add(mul(b, s), f), e);
      c.add(3);
      if (t < 0.0) {
        t = 0.0;
        s = clamp_std(dvd(-cd, a), 0.0, 1.0);
        c.add(1);
      } else if (t > 1.0) {
        t = 1.0;
        s = clamp_std(dvd(sub(b, cd), a), 0.0, 1.0);
        c.add(2);
      }
    }
  }
  c.add(12);
  return dist_pp(vadd(p1, vscale(d1, s)), vadd(p2, vscale(d2, t)), c);
}

// Query geometry: 4 trajectories (VF: point, v0, v1, v2; EE: a0, a1, b0, b1).
struct Geo {
  double p0[12];
  double p1[12];
};

// Query geometry held in a warp's shared slot (struct-of-arrays [k][slot]):
// lanes read their own slot's 24 coordinates per sample instead of keeping
// them in registers, which halves the engine's register footprint.
template <class Slots>
struct SlotGeo {
  const Slots& ws;
  int slot;
  __device__ __forceinline__ double p0(int k) const { return ws.p0[k][slot]; }
  __device__ __forceinline__ double p1(int k) const { return ws.p1[k][slot]; }
};

// PositionAt (:67-69) for the 4 vertices, then the family's distance.
template <int kFamily, class G, class C>
P2C_HD double distance_at(const G& g, double t, C& c) {
  V3 x[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double u = sub(1.0, t);
    x[i] = vadd(vscale(V3{g.p0(3 * i), g.p0(3 * i + 1), g.p0(3 * i + 2)}, u),
                vscale(V3{g.p1(3 * i), g.p1(3 * i + 1), g.p1(3 * i + 2)}, t));
  }
  c.add(40);
  if (kFamily == 1) return dist_point_triangle(x[0], x[1], x[2], x[3], c);
  return dist_segment_segment(x[0], x[1], x[2], x[3], c);
}

// Norm(Sub(p1, p0)) of each trajectory: constant per query, hoisted out of
// MaxDisplacementFromMidpoint (:71-76); the same rounded value either way.
template <class G, class C>
P2C_HD void motion_norms(const G& g, double nrm[4], C& c) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const V3 d = vsub(V3{g.p1(3 * i), g.p1(3 * i + 1), g.p1(3 * i + 2)},
                      V3{g.p0(3 * i), g.p0(3 * i + 1), g.p0(3 * i + 2)});
    nrm[i] = sqrt_rn(vdot(d, d));
  }
  c.add(36);
}

// PointTriangleMotionRadius / EdgeEdgeMotionRadius (:200-222); each
// MaxDisplacementFromMidpoint is (0.5 * max(0, t1 - t0)) * norm.
template <int kFamily, class C>
P2C_HD double motion_radius(const double nrm[4], double t0, double t1, C& c) {
  const double h = mul(0.5, max_std(0.0, sub(t1, t0)));
  const double m0 = mul(h, nrm[0]), m1 = mul(h, nrm[1]), m2 = mul(h, nrm[2]), m3 = mul(h, nrm[3]);
  c.add(7);
  if (kFamily == 1) {
    double m = m1;  // std::max({...}) keeps the first largest
    if (m < m2) m = m2;
    if (m < m3) m = m3;
    return add(m0, m);
  }
  return add(max_std(m0, m1), max_std(m2, m3));
}

// ---- path arithmetic -------------------------------------------------------
// Level l (1-based) of a node's path is bit (64 - l); bit 1 = went right.
__device__ __forceinline__ unsigned long long top_bits(int k) {  // levels 1..k
  return k <= 0 ? 0ull : (k >= 64 ? ~0ull : (~0ull << (64 - k)));
}
__device__ __forceinline__ unsigned long long level_bit(int l) { return 1ull << (64 - l); }

// Pending right siblings of the current node inside the lane's subtree:
// levels in (sub_depth, depth] where the path went left and that were not
// handed to another lane.
__device__ __forceinline__ unsigned long long pending_levels(unsigned long long path,
                                                             unsigned long long donated, int depth,
                                                             int sub_depth) {
  return top_bits(depth) & ~top_bits(sub_depth) & ~path & ~donated;
}

// Endpoints of the node (path, depth) under root [T0, T1], recomputed with the
// recursion's own roundings.  Under the root [0, 1] every bisection is exact:
// the endpoints at depth d are multiples of 2^-d, so a + b needs at most d + 1
// significant bits and 0.5 * (a + b) is exact for d <= 52.  The node at depth
// d with path bits k (its first d levels read as a binary number) is then
// [k * 2^-d, (k + 1) * 2^-d], bit for bit what the recursion computes, without
// the d dependent steps.
__device__ __forceinline__ void replay(double T0, double T1, unsigned long long path, int depth,
                                       double& a, double& b) {
  if (T0 == 0.0 && T1 == 1.0 && depth <= 52) {
    if (depth <= 0) {
      a = 0.0;
      b = 1.0;
      return;
    }
    const unsigned long long k = path >> (64 - depth);
    const double u = __longlong_as_double((long long)(1023 - depth) << 52);  // 2^-depth
    a = __dmul_rn(__ull2double_rn(k), u);
    b = __dmul_rn(__ull2double_rn(k + 1ull), u);
    return;
  }
  a = T0;
  b = T1;
  for (int l = 1; l <= depth; ++l) {
    const double m = mul(0.5, add(a, b));
    if ((path >> (64 - l)) & 1ull) a = m;
    else b = m;
  }
}

// ---- result packing (p2c_interval_result, 72 B = 9 words) ---------------
struct Outcome {
  int status;
  double t0, t1, toi, margin;
};

__device__ __forceinline__ void store_interval_result(p2c_interval_result* dst, int family, const Outcome& o,
                                                      long long id_a, long long id_b) {
  unsigned long long* w = reinterpret_cast<unsigned long long*>(dst);
  unsigned long long w0, w5, w8;
  long long ia = -1, ib = -1;
  if (o.status == P2C_STATUS_COLLISION) {
    w0 = 0ull;
    w5 = (unsigned long long)family;
    ia = id_a;
    ib = id_b;
    w8 = 0ull;
  } else if (o.status == P2C_STATUS_SEPARATION) {
    w0 = 1ull | ((unsigned long long)family << 32);
    w5 = 0ull;
    w8 = 0ull;
  } else if (o.status == P2C_STATUS_UNDECIDED) {
    w0 = 2ull;
    w5 = 0ull;
    w8 = (unsigned long long)P2C_REASON_MAX_SUBDIVISION_DEPTH |
         ((unsigned long long)P2C_REFINE_BISECT_INTERVAL << 16);
  } else {  // invalid primitive: undecided with InvalidInput (never produced by a valid query)
    w0 = 2ull;
    w5 = 0ull;
    w8 = (unsigned long long)P2C_REASON_INVALID_INPUT |
         ((unsigned long long)P2C_REFINE_REQUEST_GEOMETRY << 16);
  }
  w[0] = w0;
  w[1] = __double_as_longlong(o.t0);
  w[2] = __double_as_longlong(o.t1);
  w[3] = __double_as_longlong(o.toi);
  w[4] = __double_as_longlong(o.margin);
  w[5] = w5;
  w[6] = (unsigned long long)ia;
  w[7] = (unsigned long long)ib;
  w[8] = w8;
}

struct CertParams {
  double eps_time;
  double eps_space;
  int max_depth;
  int fetch_limit;               // queries a warp keeps in flight (1..32)
  unsigned long long budget_ns;  // device time budget of one launch (0 = none)
};

// Per-warp shared state: 32 query slots, struct-of-arrays so that lanes
// reading their own slot hit distinct banks.  A slot caches one query's
// geometry for the lanes of this warp that work on it; the query's reduction
// lives in global memory (QueryAgg) so that other warps can share its tree.
struct WarpSlots {
  double p0[12][32];
  double p1[12][32];
  double T0[32], T1[32];
  unsigned long long coll_key[32];  // this warp's view of the leftmost collision (pruning)
  long long qidx[32];
  int family[32];
  double nrm[4][32];                // motion norms of the slot's primitive (MotionRadius factors)
};

struct WarpStats {
  unsigned long long nodes = 0, evals = 0, donations = 0, queries = 0, ops = 0, iters = 0, busy = 0;
};

// Position of the (r+1)-th set bit of m (r counts from 0); m has > r set bits.
// Entry f-1 of a two-entry member array, chosen by value: a run-time index
// into such an array would move the whole object to local memory.
template <class T>
__device__ __forceinline__ T pick(const T (&a)[2], int f) {
  return f == 1 ? a[0] : a[1];
}

__device__ __forceinline__ int nth_set_bit(unsigned m, int r) {
  for (int i = 0; i < r; ++i) m &= m - 1u;
  return __ffs((int)m) - 1;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

}  // namespace p2c
