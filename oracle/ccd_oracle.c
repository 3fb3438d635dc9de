/*
 * ccd_oracle.c — CPU oracle of the P2C-CCD certification hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg compare the CUDA path against.  The product
 * path never links or calls it.  Build: oracle/Makefile (-O2 -ffp-contract=off,
 * no -march, no -ffast-math), so every double operation rounds exactly as the
 * reference C++ build does (that build uses ISO C++20 with extensions off,
 * which makes GCC default to -ffp-contract=off, and no -march, so no FMA).
 *
 * Each function names the reference lines it restates (paths relative to the
 * reference project's src/ directory).  Pinned by tests/test_oracle.py against
 * the reference's known-answer tests and against oracle/_ref (the reference
 * sources compiled unchanged).
 */
#include "ccd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* kNumericalEpsilon, cpp/certificate/certificate_engine.cpp:20 */
#define ORACLE_NUM_EPS 1.0e-14

typedef struct {
  double x, y, z;
} v3;

static v3 v_add(v3 a, v3 b) { v3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static v3 v_sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static v3 v_scale(v3 a, double s) { v3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static double v_dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 v_cross(v3 a, v3 b) {
  v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  return r;
}
static double v_norm(v3 a) { return sqrt(v_dot(a, a)); }
static v3 v_load(const double* p) { v3 r = {p[0], p[1], p[2]}; return r; }

/* std::clamp(v, lo, hi) as libstdc++ evaluates it. */
static double clamp_std(double v, double lo, double hi) {
  return (v < lo) ? lo : ((hi < v) ? hi : v);
}
/* std::max(a, b) / std::min(a, b). */
static double max_std(double a, double b) { return (a < b) ? b : a; }
static double min_std(double a, double b) { return (b < a) ? b : a; }

/* certificate_engine.cpp:78-90 */
static double dist_point_point(v3 a, v3 b) { return v_norm(v_sub(a, b)); }

static double dist_point_segment(v3 p, v3 a, v3 b) {
  const v3 ab = v_sub(b, a);
  const double ab2 = v_dot(ab, ab);
  if (ab2 <= ORACLE_NUM_EPS) return dist_point_point(p, a);
  const double t = clamp_std(v_dot(v_sub(p, a), ab) / ab2, 0.0, 1.0);
  return dist_point_point(p, v_add(a, v_scale(ab, t)));
}

/* certificate_engine.cpp:92-131 */
static double dist_segment_segment(v3 p1, v3 q1, v3 p2, v3 q2) {
  const v3 d1 = v_sub(q1, p1);
  const v3 d2 = v_sub(q2, p2);
  const v3 r = v_sub(p1, p2);
  const double a = v_dot(d1, d1);
  const double e = v_dot(d2, d2);
  const double f = v_dot(d2, r);
  double s = 0.0, t = 0.0;
  if (a <= ORACLE_NUM_EPS && e <= ORACLE_NUM_EPS) return dist_point_point(p1, p2);
  if (a <= ORACLE_NUM_EPS) {
    t = clamp_std(f / e, 0.0, 1.0);
  } else {
    const double c = v_dot(d1, r);
    if (e <= ORACLE_NUM_EPS) {
      s = clamp_std(-c / a, 0.0, 1.0);
    } else {
      const double b = v_dot(d1, d2);
      const double denom = a * e - b * b;
      if (denom != 0.0) s = clamp_std((b * f - c * e) / denom, 0.0, 1.0);
      t = (b * s + f) / e;
      if (t < 0.0) {
        t = 0.0;
        s = clamp_std(-c / a, 0.0, 1.0);
      } else if (t > 1.0) {
        t = 1.0;
        s = clamp_std((b - c) / a, 0.0, 1.0);
      }
    }
  }
  return dist_point_point(v_add(p1, v_scale(d1, s)), v_add(p2, v_scale(d2, t)));
}

/* certificate_engine.cpp:133-184 */
static double dist_point_triangle(v3 p, v3 a, v3 b, v3 c) {
  const v3 ab = v_sub(b, a);
  const v3 ac = v_sub(c, a);
  const v3 n = v_cross(ab, ac);
  if (v_dot(n, n) <= ORACLE_NUM_EPS) {
    /* std::min({x, y, z}) keeps the first smallest */
    double m = dist_point_segment(p, a, b);
    const double m1 = dist_point_segment(p, b, c);
    const double m2 = dist_point_segment(p, c, a);
    if (m1 < m) m = m1;
    if (m2 < m) m = m2;
    return m;
  }
  const v3 ap = v_sub(p, a);
  const double d1 = v_dot(ab, ap);
  const double d2 = v_dot(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return dist_point_point(p, a);
  const v3 bp = v_sub(p, b);
  const double d3 = v_dot(ab, bp);
  const double d4 = v_dot(ac, bp);
  if (d3 >= 0.0 && d4 <= d3) return dist_point_point(p, b);
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
    const double v = d1 / (d1 - d3);
    return dist_point_point(p, v_add(a, v_scale(ab, v)));
  }
  const v3 cp = v_sub(p, c);
  const double d5 = v_dot(ab, cp);
  const double d6 = v_dot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return dist_point_point(p, c);
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
    const double w = d2 / (d2 - d6);
    return dist_point_point(p, v_add(a, v_scale(ac, w)));
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
    const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    return dist_point_point(p, v_add(b, v_scale(v_sub(c, b), w)));
  }
  const double sd = v_dot(ap, n) / v_norm(n);
  return fabs(sd);
}

typedef struct {
  v3 p0[4];
  v3 p1[4];
  int family; /* 1 = point-triangle, 2 = edge-edge */
  int64_t id_a, id_b;
  const p2c_cert_config* cfg;
  uint64_t nodes;
} ctx_t;

/* certificate_engine.cpp:67-69, 186-198 */
static double distance_at(const ctx_t* c, double t) {
  v3 x[4];
  for (int i = 0; i < 4; ++i) x[i] = v_add(v_scale(c->p0[i], 1.0 - t), v_scale(c->p1[i], t));
  return c->family == 1 ? dist_point_triangle(x[0], x[1], x[2], x[3])
                        : dist_segment_segment(x[0], x[1], x[2], x[3]);
}

/* certificate_engine.cpp:71-76 */
static double max_disp(const ctx_t* c, int i, double t0, double t1) {
  const double len = max_std(0.0, t1 - t0);
  return 0.5 * len * v_norm(v_sub(c->p1[i], c->p0[i]));
}

/* certificate_engine.cpp:200-222 */
static double motion_radius(const ctx_t* c, double t0, double t1) {
  if (c->family == 1) {
    const double pt = max_disp(c, 0, t0, t1);
    double m = max_disp(c, 1, t0, t1); /* std::max({...}) keeps the first largest */
    const double m1 = max_disp(c, 2, t0, t1);
    const double m2 = max_disp(c, 3, t0, t1);
    if (m < m1) m = m1;
    if (m < m2) m = m2;
    return pt + m;
  }
  const double a = max_std(max_disp(c, 0, t0, t1), max_disp(c, 1, t0, t1));
  const double b = max_std(max_disp(c, 2, t0, t1), max_disp(c, 3, t0, t1));
  return a + b;
}

static void make_result(p2c_interval_result* r, int status, uint32_t family, double t0, double t1) {
  memset(r, 0, sizeof(*r));
  r->status = (uint8_t)status;
  r->covered_feature_mask = status == P2C_STATUS_SEPARATION ? family : 0u;
  r->interval_t0 = t0;
  r->interval_t1 = t1;
  r->toi_upper = t1;
  r->safe_margin_lb = 0.0;
  r->witness_family = 0;
  r->witness_id_a = -1;
  r->witness_id_b = -1;
  r->reason_code = P2C_REASON_NONE;
  r->next_refinement_mode = P2C_REFINE_NONE;
}

static void mark_undecided_depth(p2c_interval_result* r) {
  /* MarkUndecided with kCertificateReasonMaxSubdivisionDepth, :293-298 */
  r->status = P2C_STATUS_UNDECIDED;
  r->covered_feature_mask = 0u;
  r->reason_code = P2C_REASON_MAX_SUBDIVISION_DEPTH;
  r->next_refinement_mode = P2C_REFINE_BISECT_INTERVAL;
}

/* EvaluateIntervalRecursive, certificate_engine.cpp:300-386 */
static void eval_rec(ctx_t* c, double t0, double t1, uint16_t depth, p2c_interval_result* out) {
  c->nodes += 1;
  const p2c_cert_config* cfg = c->cfg;
  const uint32_t fam = (uint32_t)c->family;
  const double mid = 0.5 * (t0 + t1);
  const double ts[3] = {t0, mid, t1};
  double ds[3];
  ds[0] = distance_at(c, t0);
  ds[1] = distance_at(c, mid);
  ds[2] = distance_at(c, t1);
  for (int k = 0; k < 3; ++k) {
    if (ds[k] <= cfg->eps_space) {
      make_result(out, P2C_STATUS_COLLISION, fam, t0, t1);
      out->toi_upper = ts[k];
      out->witness_family = (uint8_t)fam;
      out->witness_id_a = c->id_a;
      out->witness_id_b = c->id_b;
      out->safe_margin_lb = 0.0;
      return;
    }
  }
  const double lb = distance_at(c, mid) - motion_radius(c, t0, t1);
  if (lb > cfg->eps_space) {
    make_result(out, P2C_STATUS_SEPARATION, fam, t0, t1);
    out->safe_margin_lb = max_std(0.0, lb - cfg->eps_space);
    return;
  }
  if (depth >= cfg->max_subdivision_depth || t1 - t0 <= cfg->eps_time) {
    make_result(out, P2C_STATUS_UNDECIDED, fam, t0, t1);
    mark_undecided_depth(out);
    return;
  }
  p2c_interval_result left, right;
  eval_rec(c, t0, mid, (uint16_t)(depth + 1), &left);
  if (left.status == P2C_STATUS_COLLISION) {
    *out = left;
    return;
  }
  eval_rec(c, mid, t1, (uint16_t)(depth + 1), &right);
  if (right.status == P2C_STATUS_COLLISION) {
    *out = right;
    return;
  }
  if (left.status == P2C_STATUS_SEPARATION && right.status == P2C_STATUS_SEPARATION) {
    make_result(out, P2C_STATUS_SEPARATION, fam, t0, t1);
    out->safe_margin_lb = min_std(left.safe_margin_lb, right.safe_margin_lb);
    return;
  }
  make_result(out, P2C_STATUS_UNDECIDED, fam, t0, t1);
  mark_undecided_depth(out);
}

static int finite3(const double* p) { return isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]); }
static int finite_traj(const p2c_trajectory* t) {
  return finite3(t->position_t0) && finite3(t->position_t1);
}

/* ValidateConfig / ValidateInterval, certificate_engine.cpp:224-242 */
static const char* validate_common(double t0, double t1, const p2c_cert_config* cfg) {
  if (!isfinite(cfg->eps_time) || cfg->eps_time <= 0.0)
    return "CertificateEngineConfig.eps_time must be finite and positive";
  if (!isfinite(cfg->eps_space) || cfg->eps_space <= 0.0)
    return "CertificateEngineConfig.eps_space must be finite and positive";
  if (!isfinite(t0) || !isfinite(t1)) return "certificate interval endpoints must be finite";
  if (t0 < 0.0 || t1 > 1.0 || t0 > t1) return "certificate interval must satisfy 0 <= t0 <= t1 <= 1";
  return NULL;
}

static void load_traj(const p2c_trajectory* t, v3* p0, v3* p1) {
  *p0 = v_load(t->position_t0);
  *p1 = v_load(t->position_t1);
}

/* EvaluatePointTriangleInterval, certificate_engine.cpp:481-515 */
int oracle_eval_pt(const p2c_point_triangle* prim, double t0, double t1,
                   const p2c_cert_config* cfg, p2c_interval_result* out,
                   uint64_t* nodes_out, const char** err) {
  const char* msg = validate_common(t0, t1, cfg);
  if (!msg && (prim->point_id < 0 || prim->triangle_id < 0))
    msg = "point-triangle primitive ids are required";
  if (!msg && !(finite_traj(&prim->point) && finite_traj(&prim->triangle_v0) &&
                finite_traj(&prim->triangle_v1) && finite_traj(&prim->triangle_v2)))
    msg = "point-triangle primitive trajectories must be finite";
  if (msg) {
    if (err) *err = msg;
    return 1;
  }
  ctx_t c;
  memset(&c, 0, sizeof(c));
  load_traj(&prim->point, &c.p0[0], &c.p1[0]);
  load_traj(&prim->triangle_v0, &c.p0[1], &c.p1[1]);
  load_traj(&prim->triangle_v1, &c.p0[2], &c.p1[2]);
  load_traj(&prim->triangle_v2, &c.p0[3], &c.p1[3]);
  c.family = 1;
  c.id_a = prim->point_id;
  c.id_b = prim->triangle_id;
  c.cfg = cfg;
  eval_rec(&c, t0, t1, 0, out);
  if (nodes_out) *nodes_out += c.nodes;
  return 0;
}

/* EvaluateEdgeEdgeInterval, certificate_engine.cpp:517-551 */
int oracle_eval_ee(const p2c_edge_edge* prim, double t0, double t1,
                   const p2c_cert_config* cfg, p2c_interval_result* out,
                   uint64_t* nodes_out, const char** err) {
  const char* msg = validate_common(t0, t1, cfg);
  if (!msg && (prim->edge_a_id < 0 || prim->edge_b_id < 0))
    msg = "edge-edge primitive ids are required";
  if (!msg && !(finite_traj(&prim->edge_a0) && finite_traj(&prim->edge_a1) &&
                finite_traj(&prim->edge_b0) && finite_traj(&prim->edge_b1)))
    msg = "edge-edge primitive trajectories must be finite";
  if (msg) {
    if (err) *err = msg;
    return 1;
  }
  ctx_t c;
  memset(&c, 0, sizeof(c));
  load_traj(&prim->edge_a0, &c.p0[0], &c.p1[0]);
  load_traj(&prim->edge_a1, &c.p0[1], &c.p1[1]);
  load_traj(&prim->edge_b0, &c.p0[2], &c.p1[2]);
  load_traj(&prim->edge_b1, &c.p0[3], &c.p1[3]);
  c.family = 2;
  c.id_a = prim->edge_a_id;
  c.id_b = prim->edge_b_id;
  c.cfg = cfg;
  eval_rec(&c, t0, t1, 0, out);
  if (nodes_out) *nodes_out += c.nodes;
  return 0;
}

int64_t oracle_eval_pt_batch(const p2c_point_triangle* prims, int64_t n, double t0, double t1,
                             const p2c_cert_config* cfg, p2c_interval_result* out,
                             uint8_t* status_out, uint64_t* nodes_out) {
  int64_t bad = 0;
  for (int64_t i = 0; i < n; ++i) {
    uint64_t nodes = 0;
    const int s = oracle_eval_pt(&prims[i], t0, t1, cfg, &out[i], &nodes, NULL);
    if (s) {
      memset(&out[i], 0, sizeof(out[i]));
      ++bad;
    }
    if (status_out) status_out[i] = (uint8_t)s;
    if (nodes_out) nodes_out[i] = nodes;
  }
  return bad;
}

int64_t oracle_eval_ee_batch(const p2c_edge_edge* prims, int64_t n, double t0, double t1,
                             const p2c_cert_config* cfg, p2c_interval_result* out,
                             uint8_t* status_out, uint64_t* nodes_out) {
  int64_t bad = 0;
  for (int64_t i = 0; i < n; ++i) {
    uint64_t nodes = 0;
    const int s = oracle_eval_ee(&prims[i], t0, t1, cfg, &out[i], &nodes, NULL);
    if (s) {
      memset(&out[i], 0, sizeof(out[i]));
      ++bad;
    }
    if (status_out) status_out[i] = (uint8_t)s;
    if (nodes_out) nodes_out[i] = nodes;
  }
  return bad;
}

/* RefinementModeForReason, certificate_engine.cpp:279-291 */
static uint8_t refinement_for_reason(uint16_t reason) {
  switch (reason) {
    case P2C_REASON_MISSING_GEOMETRY: return P2C_REFINE_REQUEST_GEOMETRY;
    case P2C_REASON_MAX_SUBDIVISION_DEPTH: return P2C_REFINE_BISECT_INTERVAL;
    case P2C_REASON_INVALID_INPUT: return P2C_REFINE_REQUEST_GEOMETRY;
    default: return P2C_REFINE_ESCALATE_PRECISION;
  }
}

/* CertificateEngine::Evaluate aggregation, certificate_engine.cpp:729-824, with
 * ApplyPrimitiveCollision / ApplyUndecided at :404-424. */
void oracle_aggregate(uint32_t family_mask, double interval_t1,
                      const p2c_interval_result* pt, int64_t n_pt,
                      const p2c_interval_result* ee, int64_t n_ee,
                      p2c_query_certificate* out) {
  memset(out, 0, sizeof(*out));
  out->status = P2C_STATUS_UNDECIDED;
  out->witness_id_a = -1;
  out->witness_id_b = -1;
  out->witness_index = -1;
  out->toi_upper = interval_t1;
  double margin = INFINITY;
  uint32_t mask = 0u;
  int evaluated_any = 0, has_undecided = 0;
  uint16_t undecided_reason = P2C_REASON_NONE;
  for (int fam = 1; fam <= 2; ++fam) {
    if ((family_mask & (uint32_t)fam) == 0u) continue;
    const p2c_interval_result* list = fam == 1 ? pt : ee;
    const int64_t n = fam == 1 ? n_pt : n_ee;
    if (n == 0) {
      has_undecided = 1;
      undecided_reason = P2C_REASON_MISSING_GEOMETRY;
    }
    for (int64_t i = 0; i < n; ++i) {
      evaluated_any = 1;
      const p2c_interval_result* r = &list[i];
      if (r->status == P2C_STATUS_COLLISION) {
        out->status = P2C_STATUS_COLLISION;
        out->toi_upper = r->toi_upper;
        out->safe_margin_lb = 0.0;
        out->witness_family = r->witness_family;
        out->witness_id_a = r->witness_id_a;
        out->witness_id_b = r->witness_id_b;
        out->witness_index = i;
        out->covered_feature_mask = 0u;
        out->reason_code = P2C_REASON_NONE;
        out->next_refinement_mode = P2C_REFINE_NONE;
        return;
      }
      if (r->status == P2C_STATUS_SEPARATION) {
        mask |= r->covered_feature_mask;
        margin = min_std(margin, r->safe_margin_lb);
      } else {
        has_undecided = 1;
        undecided_reason = r->reason_code;
      }
    }
  }
  if (!evaluated_any || has_undecided) {
    const uint16_t reason = !evaluated_any ? (uint16_t)P2C_REASON_MISSING_GEOMETRY : undecided_reason;
    out->status = P2C_STATUS_UNDECIDED;
    out->covered_feature_mask = 0u;
    out->safe_margin_lb = 0.0;
    out->reason_code = reason == P2C_REASON_NONE ? (uint16_t)P2C_REASON_MAX_SUBDIVISION_DEPTH : reason;
    out->next_refinement_mode = refinement_for_reason(out->reason_code);
    return;
  }
  out->status = P2C_STATUS_SEPARATION;
  out->safe_margin_lb = isfinite(margin) ? margin : 0.0;
  out->covered_feature_mask = mask;
  out->reason_code = P2C_REASON_NONE;
  out->next_refinement_mode = P2C_REFINE_NONE;
}

/* ---- broad phase ------------------------------------------------------- */

/* Extend/Expand/Swept*Box, scene_object_envelope_native_ti_walltime.cpp:256-301 */
void oracle_swept_boxes(const double* v_t0, const double* v_t1,
                        const int32_t* prim_vertices, int k, int64_t n_prims,
                        double thickness, double* boxes_out) {
  for (int64_t i = 0; i < n_prims; ++i) {
    double mn[3] = {INFINITY, INFINITY, INFINITY};
    double mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int j = 0; j < k; ++j) {
      const int64_t v = prim_vertices ? prim_vertices[i * k + j] : i;
      for (int f = 0; f < 2; ++f) {
        const double* p = (f == 0 ? v_t0 : v_t1) + 3 * v;
        for (int a = 0; a < 3; ++a) {
          mn[a] = min_std(mn[a], p[a]);
          mx[a] = max_std(mx[a], p[a]);
        }
      }
    }
    double* b = boxes_out + 6 * i;
    for (int a = 0; a < 3; ++a) {
      b[a] = mn[a] - thickness;
      b[3 + a] = mx[a] + thickness;
    }
  }
}

/* Overlap, :270-274 (inclusive on every axis) */
static int box_overlap(const double* a, const double* b) {
  return a[0] <= b[3] && b[0] <= a[3] && a[1] <= b[4] && b[1] <= a[4] && a[2] <= b[5] && b[2] <= a[5];
}

static int obj_allowed(const uint8_t* allowed, int32_t n_obj, int32_t a, int32_t b) {
  if (a < 0 || b < 0 || a >= n_obj || b >= n_obj) return 0;
  return allowed[(int64_t)a * n_obj + b] != 0;
}

static int vf_accept(const int32_t* v_obj, const int32_t* f_obj, const int32_t* faces,
                     const uint8_t* allowed, int32_t n_obj, int64_t v, int64_t f) {
  const int32_t ov = v_obj[v], of = f_obj[f];
  if (!obj_allowed(allowed, n_obj, ov, of)) return 0;
  if (ov == of && (faces[3 * f] == v || faces[3 * f + 1] == v || faces[3 * f + 2] == v)) return 0;
  return 1;
}

static int ee_accept(const int32_t* e_obj, const int32_t* edges, const uint8_t* allowed,
                     int32_t n_obj, int64_t a, int64_t b) {
  if (a >= b) return 0;
  const int32_t oa = e_obj[a], ob = e_obj[b];
  if (!obj_allowed(allowed, n_obj, oa, ob)) return 0;
  if (oa == ob) {
    const int32_t a0 = edges[2 * a], a1 = edges[2 * a + 1], b0 = edges[2 * b], b1 = edges[2 * b + 1];
    if (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1) return 0;
  }
  return 1;
}

static void emit(uint64_t* out, int64_t cap, int64_t* count, int64_t a, int64_t b) {
  if (*count < cap && out) out[*count] = ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
  *count += 1;
}

int64_t oracle_vf_pairs_brute(const double* vbox, const int32_t* v_obj, const uint8_t* v_valid, int64_t nv,
                              const double* fbox, const int32_t* f_obj, const int32_t* faces, int64_t nf,
                              const uint8_t* allowed, int32_t n_obj, uint64_t* out, int64_t cap) {
  int64_t count = 0;
  for (int64_t v = 0; v < nv; ++v) {
    if (v_valid && !v_valid[v]) continue;
    for (int64_t f = 0; f < nf; ++f) {
      if (!box_overlap(vbox + 6 * v, fbox + 6 * f)) continue;
      if (!vf_accept(v_obj, f_obj, faces, allowed, n_obj, v, f)) continue;
      emit(out, cap, &count, v, f);
    }
  }
  return count;
}

int64_t oracle_ee_pairs_brute(const double* ebox, const int32_t* e_obj, const int32_t* edges, int64_t ne,
                              const uint8_t* allowed, int32_t n_obj, uint64_t* out, int64_t cap) {
  int64_t count = 0;
  for (int64_t a = 0; a < ne; ++a) {
    for (int64_t b = a + 1; b < ne; ++b) {
      if (!box_overlap(ebox + 6 * a, ebox + 6 * b)) continue;
      if (!ee_accept(e_obj, edges, allowed, n_obj, a, b)) continue;
      emit(out, cap, &count, a, b);
    }
  }
  return count;
}

/* std::stable_sort of indices by box min.x (merge sort keeps equal keys in order). */
static void stable_sort_by_minx(int64_t* idx, int64_t n, const double* boxes) {
  if (n < 2) return;
  int64_t* tmp = (int64_t*)malloc((size_t)n * sizeof(int64_t));
  for (int64_t width = 1; width < n; width *= 2) {
    for (int64_t lo = 0; lo < n; lo += 2 * width) {
      int64_t mid = lo + width < n ? lo + width : n;
      int64_t hi = lo + 2 * width < n ? lo + 2 * width : n;
      int64_t i = lo, j = mid, k = lo;
      while (i < mid && j < hi) {
        /* take from the right only if strictly smaller: stable */
        if (boxes[6 * idx[j]] < boxes[6 * idx[i]]) tmp[k++] = idx[j++];
        else tmp[k++] = idx[i++];
      }
      while (i < mid) tmp[k++] = idx[i++];
      while (j < hi) tmp[k++] = idx[j++];
    }
    memcpy(idx, tmp, (size_t)n * sizeof(int64_t));
  }
  free(tmp);
}

typedef int (*accept_fn)(const void* ctx, int64_t a, int64_t b);

/* SweepPairs, :603-649 */
static int64_t sweep(const int64_t* lhs_ids, int64_t nl, const double* lbox,
                     const int64_t* rhs_ids, int64_t nr, const double* rbox,
                     accept_fn accept, const void* ctx, uint64_t* out, int64_t cap) {
  int64_t* lo = (int64_t*)malloc((size_t)(nl > 0 ? nl : 1) * sizeof(int64_t));
  int64_t* ro = (int64_t*)malloc((size_t)(nr > 0 ? nr : 1) * sizeof(int64_t));
  int64_t* active = (int64_t*)malloc((size_t)(nr > 0 ? nr : 1) * sizeof(int64_t));
  memcpy(lo, lhs_ids, (size_t)nl * sizeof(int64_t));
  memcpy(ro, rhs_ids, (size_t)nr * sizeof(int64_t));
  stable_sort_by_minx(lo, nl, lbox);
  stable_sort_by_minx(ro, nr, rbox);
  int64_t n_active = 0, cursor = 0, count = 0;
  for (int64_t ii = 0; ii < nl; ++ii) {
    const int64_t ai = lo[ii];
    const double* ab = lbox + 6 * ai;
    while (cursor < nr && rbox[6 * ro[cursor]] <= ab[3]) active[n_active++] = ro[cursor++];
    int64_t w = 0;
    for (int64_t k = 0; k < n_active; ++k)
      if (rbox[6 * active[k] + 3] >= ab[0]) active[w++] = active[k];
    n_active = w;
    for (int64_t k = 0; k < n_active; ++k) {
      const int64_t bi = active[k];
      if (!box_overlap(ab, rbox + 6 * bi)) continue;
      if (accept(ctx, ai, bi)) emit(out, cap, &count, ai, bi);
    }
  }
  free(lo);
  free(ro);
  free(active);
  return count;
}

typedef struct {
  const int32_t *v_obj, *f_obj, *faces, *e_obj, *edges;
  const uint8_t* allowed;
  int32_t n_obj;
} sweep_ctx;

static int vf_accept_cb(const void* p, int64_t v, int64_t f) {
  const sweep_ctx* c = (const sweep_ctx*)p;
  return vf_accept(c->v_obj, c->f_obj, c->faces, c->allowed, c->n_obj, v, f);
}
static int ee_accept_cb(const void* p, int64_t a, int64_t b) {
  const sweep_ctx* c = (const sweep_ctx*)p;
  return ee_accept(c->e_obj, c->edges, c->allowed, c->n_obj, a, b);
}

int64_t oracle_vf_pairs_sweep(const double* vbox, const int32_t* v_obj, const uint8_t* v_valid, int64_t nv,
                              const double* fbox, const int32_t* f_obj, const int32_t* faces, int64_t nf,
                              const uint8_t* allowed, int32_t n_obj, uint64_t* out, int64_t cap) {
  int64_t* lids = (int64_t*)malloc((size_t)(nv > 0 ? nv : 1) * sizeof(int64_t));
  int64_t* rids = (int64_t*)malloc((size_t)(nf > 0 ? nf : 1) * sizeof(int64_t));
  int64_t nl = 0;
  for (int64_t v = 0; v < nv; ++v)
    if (!v_valid || v_valid[v]) lids[nl++] = v;
  for (int64_t f = 0; f < nf; ++f) rids[f] = f;
  sweep_ctx c = {v_obj, f_obj, faces, NULL, NULL, allowed, n_obj};
  const int64_t n = sweep(lids, nl, vbox, rids, nf, fbox, vf_accept_cb, &c, out, cap);
  free(lids);
  free(rids);
  return n;
}

int64_t oracle_ee_pairs_sweep(const double* ebox, const int32_t* e_obj, const int32_t* edges, int64_t ne,
                              const uint8_t* allowed, int32_t n_obj, uint64_t* out, int64_t cap) {
  int64_t* ids = (int64_t*)malloc((size_t)(ne > 0 ? ne : 1) * sizeof(int64_t));
  for (int64_t e = 0; e < ne; ++e) ids[e] = e;
  sweep_ctx c = {NULL, NULL, NULL, e_obj, edges, allowed, n_obj};
  const int64_t n = sweep(ids, ne, ebox, ids, ne, ebox, ee_accept_cb, &c, out, cap);
  free(ids);
  return n;
}

/* PrepareScene object envelopes and permission matrix, :521-545 */
void oracle_object_allowed(const double* v_t0, const double* v_t1, const int32_t* v_obj, int64_t nv,
                           int32_t n_obj, double thickness, int exclude_self, uint8_t* allowed) {
  double* ob = (double*)malloc((size_t)(n_obj > 0 ? n_obj : 1) * 6 * sizeof(double));
  for (int32_t o = 0; o < n_obj; ++o) {
    for (int a = 0; a < 3; ++a) {
      ob[6 * o + a] = INFINITY;
      ob[6 * o + 3 + a] = -INFINITY;
    }
  }
  for (int64_t v = 0; v < nv; ++v) {
    const int32_t o = v_obj[v];
    if (o < 0) continue;
    for (int f = 0; f < 2; ++f) {
      const double* p = (f == 0 ? v_t0 : v_t1) + 3 * v;
      for (int a = 0; a < 3; ++a) {
        ob[6 * o + a] = min_std(ob[6 * o + a], p[a]);
        ob[6 * o + 3 + a] = max_std(ob[6 * o + 3 + a], p[a]);
      }
    }
  }
  for (int32_t o = 0; o < n_obj; ++o) {
    for (int a = 0; a < 3; ++a) {
      ob[6 * o + a] -= thickness;
      ob[6 * o + 3 + a] += thickness;
    }
  }
  memset(allowed, 0, (size_t)n_obj * (size_t)n_obj);
  for (int32_t a = 0; a < n_obj; ++a) {
    for (int32_t b = a; b < n_obj; ++b) {
      if ((a == b && !exclude_self) || (a != b && box_overlap(ob + 6 * a, ob + 6 * b))) {
        allowed[(int64_t)a * n_obj + b] = 1;
        allowed[(int64_t)b * n_obj + a] = 1;
      }
    }
  }
  free(ob);
}

/* RunScheduledAnyHitRows, :1283-1410: per group the top-K in priority order is
 * certified until the first hit; groups without a hit then replay every other
 * candidate of the group in input order until a hit. */
void oracle_group_anyhit(int64_t n_cand, const int32_t* cand_group, const uint8_t* cand_hit,
                         int32_t n_groups, const int64_t* top_offsets, const int64_t* top_index,
                         uint8_t* detected, int64_t* proposal_calls, int64_t* fallback_calls,
                         uint8_t* evaluated) {
  uint8_t* visited_top = (uint8_t*)calloc((size_t)(n_cand > 0 ? n_cand : 1), 1);
  memset(evaluated, 0, (size_t)n_cand);
  for (int32_t g = 0; g < n_groups; ++g) {
    detected[g] = 0;
    proposal_calls[g] = 0;
    fallback_calls[g] = 0;
    for (int64_t k = top_offsets[g]; k < top_offsets[g + 1]; ++k) {
      const int64_t i = top_index[k];
      visited_top[i] = 1;
      evaluated[i] = 1;
      proposal_calls[g] += 1;
      if (cand_hit[i]) {
        detected[g] = 1;
        break;
      }
    }
  }
  for (int64_t i = 0; i < n_cand; ++i) {
    if (visited_top[i]) continue;
    const int32_t g = cand_group[i];
    if (detected[g]) continue;
    evaluated[i] = 1;
    fallback_calls[g] += 1;
    if (cand_hit[i]) detected[g] = 1;
  }
  free(visited_top);
}

/* GenerateConservativeRefinementWorkItems interval logic, certificate_engine.cpp:686-719 */
int oracle_refinement_children(double t0, double t1, uint16_t depth, uint8_t status,
                               uint8_t mode, double toi, uint16_t max_child_depth,
                               double min_width, double* c0, double* c1) {
  if (depth >= max_child_depth) return 0;
  if (status == P2C_STATUS_COLLISION) {
    const double ct1 = clamp_std(toi, t0, t1);
    if (ct1 - t0 > min_width) {
      c0[0] = t0;
      c1[0] = ct1;
      return 1;
    }
    return 0;
  }
  if (status == P2C_STATUS_UNDECIDED && mode == P2C_REFINE_BISECT_INTERVAL) {
    if (t1 - t0 > min_width) {
      const double mid = 0.5 * (t0 + t1);
      c0[0] = t0;
      c1[0] = mid;
      c0[1] = mid;
      c1[1] = t1;
      return 2;
    }
  }
  return 0;
}
