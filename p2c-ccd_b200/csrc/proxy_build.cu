// proxy_build.cu — BuildProxyScene (rt_candidate/proxy_scene.cpp:156-213) with
// the per-patch work on the device.
//
// A proxy scene has one proxy per (object, motion segment, time slab, patch).
// Everything that depends only on (object, segment, slab) — the uniform slab
// grid, the interpolated rigid poses at both slab ends (a quaternion slerp
// with acos/sin/cos), the rotation angle and its half-angle sine — is a
// handful of values per slab and is computed here on the host with the C
// library's functions, exactly the calls the reference makes, so every bit
// matches.  Those slab records go to the device, where one thread per proxy
// transforms its patch centre to both slab ends and forms the motion bound
// and the swept-AABB or capsule bounds: additions, products and square roots
// only, bit-identical with --fmad=false.
#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <utility>
#include <vector>

#include "p2c_internal.cuh"

namespace p2c {
namespace {

constexpr int kThreads = 256;

// One (object, segment, slab): the poses at both slab ends, with the
// rotations normalised as TransformPoint uses them.
struct SlabRecord {
  double tr0[3], q0[4], tr1[3], q1[4];
  double translation_bound, rotation_angle, half_angle_sin;
  double t0, t1, eps;
  long long proxy_base, patch_offset;
  unsigned n_patches, object_id, slab_id, segment_id, proxy_type, pad;
};

using V3 = std::array<double, 3>;
using Q4 = std::array<double, 4>;

bool finite3(const double* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }
bool finite4(const double* v) { return finite3(v) && std::isfinite(v[3]); }

double dot4(const Q4& a, const Q4& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3]; }

double clampd(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }  // std::clamp

// NormalizeQuaternion (geometry/motion_utils.cpp:64-77)
int normalize(const double* in, Q4* out) {
  if (!finite4(in)) return fail(P2C_ERR_INVALID, "quaternion contains a non-finite value");
  const Q4 q{in[0], in[1], in[2], in[3]};
  const double norm = std::sqrt(dot4(q, q));
  if (!std::isfinite(norm) || norm <= 0.0) return fail(P2C_ERR_INVALID, "quaternion norm must be positive and finite");
  *out = {q[0] / norm, q[1] / norm, q[2] / norm, q[3] / norm};
  return P2C_OK;
}

// ValidatePose (:79-85)
int validate_pose(const double* translation, const double* rotation, const char* name) {
  if (!finite3(translation)) return fail(P2C_ERR_INVALID, "%s.translation contains a non-finite value", name);
  Q4 q;
  return normalize(rotation, &q);
}

// ValidateMotionSegment (:165-173)
int validate_segment(const p2c_motion_segment& s) {
  if (!std::isfinite(s.t0) || !std::isfinite(s.t1) || s.t0 >= s.t1)
    return fail(P2C_ERR_INVALID, "motion segment must satisfy finite t0 < t1");
  if (int rc = validate_pose(s.translation_t0, s.rotation_t0, "pose_t0")) return rc;
  return validate_pose(s.translation_t1, s.rotation_t1, "pose_t1");
}

// Slerp (:99-126) of two unit quaternions; the near-parallel branch is
// LerpAndNormalize (:87-97).
Q4 slerp(const Q4& a, Q4 b, double alpha) {
  double d = dot4(a, b);
  if (d < 0.0) {
    b = {-b[0], -b[1], -b[2], -b[3]};
    d = -d;
  }
  d = clampd(d, -1.0, 1.0);
  if (d > 0.9995) {
    const Q4 q{(1.0 - alpha) * a[0] + alpha * b[0], (1.0 - alpha) * a[1] + alpha * b[1],
               (1.0 - alpha) * a[2] + alpha * b[2], (1.0 - alpha) * a[3] + alpha * b[3]};
    const double norm = std::sqrt(dot4(q, q));
    return {q[0] / norm, q[1] / norm, q[2] / norm, q[3] / norm};
  }
  const double theta0 = std::acos(d);
  const double theta = theta0 * alpha;
  const double sin_theta = std::sin(theta);
  const double sin_theta0 = std::sin(theta0);
  const double s0 = std::cos(theta) - d * sin_theta / sin_theta0;
  const double s1 = sin_theta / sin_theta0;
  return {s0 * a[0] + s1 * b[0], s0 * a[1] + s1 * b[1], s0 * a[2] + s1 * b[2], s0 * a[3] + s1 * b[3]};
}

// InterpolateRigidMotion (:196-229) at a slab end t (inside the segment).
int interpolate(const p2c_motion_segment& s, double t, V3* tr, Q4* rot) {
  const double tol = 1.0e-12 * std::max(1.0, s.t1 - s.t0);
  if (!std::isfinite(t) || t < s.t0 - tol || t > s.t1 + tol)
    return fail(P2C_ERR_INVALID, "interpolation time must lie inside the motion segment");
  const double ct = clampd(t, s.t0, s.t1);
  const double alpha = (ct - s.t0) / (s.t1 - s.t0);
  for (int a = 0; a < 3; ++a) (*tr)[a] = (1.0 - alpha) * s.translation_t0[a] + alpha * s.translation_t1[a];
  Q4 q0, q1;
  if (int rc = normalize(s.rotation_t0, &q0)) return rc;
  if (int rc = normalize(s.rotation_t1, &q1)) return rc;
  *rot = slerp(q0, q1, alpha);
  return P2C_OK;
}

// The per-object checks of BuildProxyScene (:170-185).
int check_object(const p2c_proxy_object_input& o) {
  if (o.proxy_type != 1u && o.proxy_type != 2u)
    return fail(P2C_ERR_INVALID, "ProxyObjectBuildInput.proxy_type must be concrete");
  if (o.n_patches <= 0) return fail(P2C_ERR_INVALID, "ProxyObjectBuildInput.patches is empty");
  if (o.n_segments <= 0) return fail(P2C_ERR_INVALID, "ProxyObjectBuildInput.motion_segments is empty");
  if (o.slabs_per_motion_segment == 0u) return fail(P2C_ERR_INVALID, "slabs_per_motion_segment must be positive");
  if (!std::isfinite(o.eps_proxy) || o.eps_proxy < 0.0)
    return fail(P2C_ERR_INVALID, "eps_proxy must be finite and non-negative");
  if (o.segments == nullptr) return fail(P2C_ERR_INVALID, "motion segment array is null");
  if (o.patch_offset < 0) return fail(P2C_ERR_INVALID, "patch offset is negative");
  return P2C_OK;
}

long long count_proxies(const p2c_proxy_object_input* objects, long long n_objects, long long* n_records) {
  long long total = 0, records = 0;
  for (long long k = 0; k < n_objects; ++k) {
    const p2c_proxy_object_input& o = objects[k];
    if (check_object(o) != P2C_OK) return -1;
    const long long slabs = o.n_segments * (long long)o.slabs_per_motion_segment;
    if (slabs >= (1ll << 31) || o.n_patches >= (1ll << 31) || slabs * o.n_patches >= (1ll << 31)) {
      fail(P2C_ERR_INVALID, "proxy count must stay below 2^31");
      return -1;
    }
    records += slabs;
    total += slabs * o.n_patches;
    if (total >= (1ll << 31)) {
      fail(P2C_ERR_INVALID, "proxy count must stay below 2^31");
      return -1;
    }
  }
  if (n_records) *n_records = records;
  return total;
}

// One object's slab records (:186-204 and ComputePatchMotionBound's
// per-slab part, motion_utils.cpp:281-313).
int object_records(const p2c_proxy_object_input& o, long long* proxy_base, std::vector<SlabRecord>* out) {
  const unsigned S = o.slabs_per_motion_segment;
  for (long long seg = 0; seg < o.n_segments; ++seg) {
    const p2c_motion_segment& s = o.segments[seg];
    if (int rc = validate_segment(s)) return rc;  // GenerateTimeSlabsForMotionSegment (:187-194)
    const double dt = (s.t1 - s.t0) / static_cast<double>(S);  // GenerateUniformTimeSlabs (:175-185)
    for (unsigned k = 0; k < S; ++k) {
      const double t0 = k == 0 ? s.t0 : s.t0 + dt * k;
      const double t1 = k + 1 == S ? s.t1 : s.t0 + dt * (k + 1);
      // ValidateTimeSlab (:137-148)
      if (!std::isfinite(t0) || !std::isfinite(t1) || t0 >= t1)
        return fail(P2C_ERR_INVALID, "time slab must satisfy finite t0 < t1");
      const double tol = 1.0e-12 * std::max(1.0, s.t1 - s.t0);
      if (t0 < s.t0 - tol || t1 > s.t1 + tol)
        return fail(P2C_ERR_INVALID, "time slab must lie inside the motion segment");
      V3 tr0, tr1;
      Q4 r0, r1, q0, q1;
      if (int rc = interpolate(s, t0, &tr0, &r0)) return rc;
      if (int rc = interpolate(s, t1, &tr1, &r1)) return rc;
      // TransformPoint validates and normalises each pose (:231-249)
      if (int rc = validate_pose(tr0.data(), r0.data(), "pose")) return rc;
      if (int rc = validate_pose(tr1.data(), r1.data(), "pose")) return rc;
      if (int rc = normalize(r0.data(), &q0)) return rc;
      if (int rc = normalize(r1.data(), &q1)) return rc;
      SlabRecord r{};
      for (int a = 0; a < 3; ++a) {
        r.tr0[a] = tr0[a];
        r.tr1[a] = tr1[a];
      }
      for (int a = 0; a < 4; ++a) {
        r.q0[a] = q0[a];
        r.q1[a] = q1[a];
      }
      // ComputeRotationAngle (:251-267)
      const double d = clampd(std::abs(dot4(q0, q1)), 0.0, 1.0);
      r.rotation_angle = 2.0 * std::acos(d);
      const double dx = tr0[0] - tr1[0], dy = tr0[1] - tr1[1], dz = tr0[2] - tr1[2];
      r.translation_bound = std::sqrt(dx * dx + dy * dy + dz * dz);
      r.half_angle_sin = std::sin(0.5 * r.rotation_angle);
      r.t0 = t0;
      r.t1 = t1;
      r.eps = o.eps_proxy;
      r.proxy_base = *proxy_base;
      r.patch_offset = o.patch_offset;
      r.n_patches = (unsigned)o.n_patches;
      r.object_id = o.object_id;
      r.slab_id = (unsigned)seg * S + k;
      r.segment_id = (unsigned)seg;
      r.proxy_type = o.proxy_type;
      out->push_back(r);
      *proxy_base += o.n_patches;
    }
  }
  return P2C_OK;
}

double time_tolerance(double t0, double t1) {  // proxy_scene.cpp:37-39
  return 1.0e-12 * std::max({1.0, std::abs(t0), std::abs(t1), std::abs(t1 - t0)});
}

// ValidateGlobalSlabPartition (proxy_scene.cpp:58-85) over the slab records:
// every proxy of a record carries the record's slab id and interval.
int check_slab_partition(const std::vector<SlabRecord>& recs) {
  std::map<unsigned, std::pair<double, double>> first;
  for (const SlabRecord& r : recs) {
    auto it = first.emplace(r.slab_id, std::make_pair(r.t0, r.t1)).first;
    const double tol = time_tolerance(it->second.first, it->second.second);
    if (!(std::abs(it->second.first - r.t0) <= tol) || !(std::abs(it->second.second - r.t1) <= tol))
      return fail(P2C_ERR_INVALID, "proxy scene slab_id must map to one global time interval");
  }
  std::vector<std::pair<unsigned, std::pair<double, double>>> ordered(first.begin(), first.end());
  std::sort(ordered.begin(), ordered.end(), [](const auto& a, const auto& b) {
    return a.second.first == b.second.first ? a.first < b.first : a.second.first < b.second.first;
  });
  for (size_t i = 1; i < ordered.size(); ++i) {
    const auto& a = ordered[i - 1].second;
    const auto& b = ordered[i].second;
    const double tol = std::max(time_tolerance(a.first, a.second), time_tolerance(b.first, b.second));
    if (a.first < b.second - tol && b.first < a.second - tol)
      return fail(P2C_ERR_INVALID, "proxy scene global slab intervals must not overlap");
  }
  return P2C_OK;
}

// RotateVector (motion_utils.cpp:128-135): 2 (u.v) u + (s^2 - u.u) v + 2 s (u x v)
__device__ __forceinline__ void rotate(const double* q, const double* v, double* o) {
  const double u0 = q[0], u1 = q[1], u2 = q[2], s = q[3];
  const double k0 = 2.0 * (u0 * v[0] + u1 * v[1] + u2 * v[2]);
  const double k1 = s * s - (u0 * u0 + u1 * u1 + u2 * u2);
  const double k2 = 2.0 * s;
  const double c0 = u1 * v[2] - u2 * v[1], c1 = u2 * v[0] - u0 * v[2], c2 = u0 * v[1] - u1 * v[0];
  o[0] = (u0 * k0 + v[0] * k1) + c0 * k2;
  o[1] = (u1 * k0 + v[1] * k1) + c1 * k2;
  o[2] = (u2 * k0 + v[2] * k1) + c2 * k2;
}

__device__ __forceinline__ bool finite_d(double v) { return isfinite(v); }

// One proxy per thread: the patch's motion bound over the slab
// (ComputePatchMotionBound, :269-325) and its bounds
// (BuildEndpointSweptAabbProxy / BuildCapsuleProxy, geometry/proxy.cpp:70-131,
// CapsuleBounds and ValidateAabbBounds, proxy_scene.cpp:17-35).
__global__ void __launch_bounds__(kThreads) build_kernel(const SlabRecord* __restrict__ recs, int n_recs,
                                                         long long n, const unsigned* __restrict__ patch_id,
                                                         const double* __restrict__ center,
                                                         const double* __restrict__ radius,
                                                         p2c_proxy_build_out out, unsigned long long* err) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int lo = 0, hi = n_recs;  // last record with proxy_base <= p
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (recs[mid].proxy_base <= p) lo = mid;
    else hi = mid;
  }
  const SlabRecord& r = recs[lo];
  const long long pi = r.patch_offset + (p - r.proxy_base);
  const double lc[3] = {center[3 * pi], center[3 * pi + 1], center[3 * pi + 2]};
  const double rad = radius[pi];
  unsigned long long e = 0;
  if (!(finite_d(lc[0]) && finite_d(lc[1]) && finite_d(lc[2]))) e |= 1ull;  // ValidatePatchForMotionBound
  if (!finite_d(rad) || rad < 0.0) e |= 2ull;
  double c0[3], c1[3];
  rotate(r.q0, lc, c0);
  rotate(r.q1, lc, c1);
  for (int a = 0; a < 3; ++a) {
    c0[a] = c0[a] + r.tr0[a];
    c1[a] = c1[a] + r.tr1[a];
  }
  const double hs = r.half_angle_sin;
  const double crb = 2.0 * sqrt(lc[0] * lc[0] + lc[1] * lc[1] + lc[2] * lc[2]) * hs;
  const double srb = 2.0 * rad * hs;
  const double radial = r.translation_bound + crb + srb;
  const double cons = rad + crb;
  double mn[3], mx[3], cap_r = 0.0;
  if (r.proxy_type == 1u) {
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
      mn[a] = (c1[a] < c0[a] ? c1[a] : c0[a]) - cons;  // std::min, std::max
      mx[a] = (c0[a] < c1[a] ? c1[a] : c0[a]) + cons;
      ok = ok && finite_d(mn[a]) && finite_d(mx[a]) && !(mn[a] > mx[a]);
    }
    if (!ok) e |= 4ull;  // InflateAabb's ValidateAabb
    for (int a = 0; a < 3; ++a) {
      mn[a] = mn[a] - r.eps;
      mx[a] = mx[a] + r.eps;
    }
  } else {
    if (!finite_d(cons) || cons < 0.0) e |= 8ull;  // InflateCapsule
    cap_r = cons + r.eps;
    for (int a = 0; a < 3; ++a) {
      mn[a] = (c1[a] < c0[a] ? c1[a] : c0[a]) - cap_r;
      mx[a] = (c0[a] < c1[a] ? c1[a] : c0[a]) + cap_r;
    }
  }
  for (int a = 0; a < 3; ++a)
    if (!finite_d(mn[a]) || !finite_d(mx[a]) || mn[a] > mx[a]) e |= 16ull;
  if (e) atomicOr(err, e);
  out.object_id[p] = r.object_id;
  out.patch_id[p] = patch_id[pi];
  out.slab_id[p] = r.slab_id;
  out.motion_segment_id[p] = r.segment_id;
  out.proxy_type[p] = (uint8_t)r.proxy_type;
  out.t0[p] = r.t0;
  out.t1[p] = r.t1;
  for (int a = 0; a < 3; ++a) {
    out.bounds[6 * p + a] = mn[a];
    out.bounds[6 * p + 3 + a] = mx[a];
  }
  out.motion_bound[4 * p + 0] = r.translation_bound;
  out.motion_bound[4 * p + 1] = r.rotation_angle;
  out.motion_bound[4 * p + 2] = radial;
  out.motion_bound[4 * p + 3] = cons;
  if (out.motion_detail) {
    double* d = out.motion_detail + 8 * p;
    for (int a = 0; a < 3; ++a) {
      d[a] = c0[a];
      d[3 + a] = c1[a];
    }
    d[6] = crb;
    d[7] = srb;
  }
  if (out.capsule_radius) out.capsule_radius[p] = cap_r;
}

}  // namespace
}  // namespace p2c

extern "C" {

int64_t p2c_proxy_scene_count(const p2c_proxy_object_input* objects, int64_t n_objects) {
  using namespace p2c;
  if (n_objects <= 0 || objects == nullptr) {
    fail(P2C_ERR_INVALID, "ProxySceneBuildInput.objects is empty");
    return -1;
  }
  return count_proxies(objects, n_objects, nullptr);
}

size_t p2c_proxy_scene_build_workspace_bytes(const p2c_proxy_object_input* objects, int64_t n_objects) {
  long long records = 0;
  for (long long k = 0; objects != nullptr && k < n_objects; ++k)
    records += std::max<long long>(objects[k].n_segments, 0) * (long long)objects[k].slabs_per_motion_segment;
  return (size_t)std::max(records, 1ll) * sizeof(p2c::SlabRecord) + 256;
}

int p2c_proxy_scene_build(uint64_t query_id, const p2c_proxy_object_input* objects, int64_t n_objects,
                          const uint32_t* patch_id_dev, const double* patch_center_dev,
                          const double* patch_radius_dev, int64_t n_patch_entries, int64_t proxy_cap,
                          const p2c_proxy_build_out* out,
                          uint64_t* error_word_dev, void* workspace_dev, size_t workspace_bytes, void* stream) {
  using namespace p2c;
  if (query_id == 0) return fail(P2C_ERR_INVALID, "ProxySceneBuildInput.query_id is required");
  if (n_objects <= 0 || objects == nullptr) return fail(P2C_ERR_INVALID, "ProxySceneBuildInput.objects is empty");
  if (out == nullptr || error_word_dev == nullptr) return fail(P2C_ERR_INVALID, "output pointer is null");
  std::vector<SlabRecord> recs;
  long long base = 0;
  for (long long k = 0; k < n_objects; ++k) {
    if (int rc = check_object(objects[k])) return rc;
    if (objects[k].n_patches > n_patch_entries - objects[k].patch_offset)
      return fail(P2C_ERR_INVALID, "object %lld: patches [%lld, +%lld) exceed the %lld patch entries", k,
                  (long long)objects[k].patch_offset, (long long)objects[k].n_patches, (long long)n_patch_entries);
    const long long slabs = objects[k].n_segments * (long long)objects[k].slabs_per_motion_segment;
    if (slabs >= (1ll << 31) || base + slabs * objects[k].n_patches >= (1ll << 31))
      return fail(P2C_ERR_INVALID, "proxy count must stay below 2^31");
    if (int rc = object_records(objects[k], &base, &recs)) return rc;
  }
  if (int rc = check_slab_partition(recs)) return rc;
  const long long n = base;
  if (proxy_cap < n) return fail(P2C_ERR_INVALID, "proxy capacity %lld below the %lld proxies", (long long)proxy_cap, n);
  if (n > 0 && (patch_id_dev == nullptr || patch_center_dev == nullptr || patch_radius_dev == nullptr ||
                out->object_id == nullptr || out->patch_id == nullptr || out->slab_id == nullptr ||
                out->motion_segment_id == nullptr || out->proxy_type == nullptr || out->t0 == nullptr ||
                out->t1 == nullptr || out->bounds == nullptr || out->motion_bound == nullptr))
    return fail(P2C_ERR_INVALID, "patch or proxy output arrays are null");
  const size_t need = recs.size() * sizeof(SlabRecord);
  if (workspace_dev == nullptr || workspace_bytes < need)
    return fail(P2C_ERR_INVALID, "proxy build workspace too small: %zu < %zu bytes", workspace_bytes, need);
  cudaStream_t s = as_stream(stream);
  P2C_CUDA(cudaMemsetAsync(error_word_dev, 0, sizeof(uint64_t), s));
  if (n == 0) return P2C_OK;
  // pageable source: the call returns once the records are staged
  P2C_CUDA(cudaMemcpyAsync(workspace_dev, recs.data(), need, cudaMemcpyHostToDevice, s));
  const unsigned blocks = (unsigned)((n + kThreads - 1) / kThreads);
  build_kernel<<<blocks, kThreads, 0, s>>>(static_cast<const SlabRecord*>(workspace_dev), (int)recs.size(), n,
                                           patch_id_dev, patch_center_dev, patch_radius_dev, *out,
                                           reinterpret_cast<unsigned long long*>(error_word_dev));
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

}  // extern "C"
