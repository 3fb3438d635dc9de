/*
 * ccd_oracle.h — CPU oracle of the P2C-CCD certification hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path links, loads or calls
 * this code; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg use it, as the checker.  It restates, in plain C, the reference
 * algorithms cited beside each function, and is pinned against the reference's
 * own known-answer tests and against the reference sources compiled unchanged
 * (oracle/_ref, built by oracle/Makefile).
 */
#ifndef P2C_CCD_ORACLE_H_
#define P2C_CCD_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#include "../include/p2c_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-primitive interval certificates (certificate_engine.cpp:481-551).
 * Returns 0 on success, 1 on invalid input (message in *err if non-NULL).
 * nodes_out (may be NULL) accumulates recursion nodes visited. */
int oracle_eval_pt(const p2c_point_triangle* prim, double t0, double t1,
                   const p2c_cert_config* cfg, p2c_interval_result* out,
                   uint64_t* nodes_out, const char** err);
int oracle_eval_ee(const p2c_edge_edge* prim, double t0, double t1,
                   const p2c_cert_config* cfg, p2c_interval_result* out,
                   uint64_t* nodes_out, const char** err);

/* Batch forms; status_out[i] = 0 ok / 1 invalid.  Returns number of invalid. */
int64_t oracle_eval_pt_batch(const p2c_point_triangle* prims, int64_t n, double t0, double t1,
                             const p2c_cert_config* cfg, p2c_interval_result* out,
                             uint8_t* status_out, uint64_t* nodes_out);
int64_t oracle_eval_ee_batch(const p2c_edge_edge* prims, int64_t n, double t0, double t1,
                             const p2c_cert_config* cfg, p2c_interval_result* out,
                             uint8_t* status_out, uint64_t* nodes_out);

/* CertificateEngine::Evaluate aggregation (certificate_engine.cpp:729-824) over
 * already-computed per-primitive results, in list order.  family_mask is the
 * work item's feature_family_mask; non-collision certificates keep
 * toi_upper = the work item's interval_t1 (MakeBaseCertificateResult, :388-402). */
void oracle_aggregate(uint32_t family_mask, double interval_t1,
                      const p2c_interval_result* pt_results, int64_t n_pt,
                      const p2c_interval_result* ee_results, int64_t n_ee,
                      p2c_query_certificate* out);

/* Swept boxes (scene_object_envelope_native_ti_walltime.cpp:276-301): box[6] =
 * {minx,miny,minz,maxx,maxy,maxz} over the t0 and t1 positions of k vertices,
 * expanded by thickness. */
void oracle_swept_boxes(const double* v_t0, const double* v_t1,
                        const int32_t* prim_vertices, int k, int64_t n_prims,
                        double thickness, double* boxes_out);

/* Brute-force candidate enumeration with the scene tool's filters
 * (BuildVFCandidates/BuildEECandidates, :651-699): inclusive box overlap,
 * object-pair permission, no vertex against its own face, no edges sharing a
 * vertex inside one object, EE pairs with a < b.  object_allowed is an
 * n_obj x n_obj byte matrix.  Pairs are written as (a << 32 | b) into out
 * (capacity cap); the return value is the total number of pairs. */
int64_t oracle_vf_pairs_brute(const double* vbox, const int32_t* v_obj, const uint8_t* v_valid, int64_t nv,
                              const double* fbox, const int32_t* f_obj, const int32_t* faces, int64_t nf,
                              const uint8_t* object_allowed, int32_t n_obj,
                              uint64_t* out, int64_t cap);
int64_t oracle_ee_pairs_brute(const double* ebox, const int32_t* e_obj, const int32_t* edges, int64_t ne,
                              const uint8_t* object_allowed, int32_t n_obj,
                              uint64_t* out, int64_t cap);

/* The same pair sets by the reference's sort-and-sweep (SweepPairs, :603-649):
 * stable sort by min.x, active list, inclusive overlap.  Pairs are emitted in
 * the sweep's own order. */
int64_t oracle_vf_pairs_sweep(const double* vbox, const int32_t* v_obj, const uint8_t* v_valid, int64_t nv,
                              const double* fbox, const int32_t* f_obj, const int32_t* faces, int64_t nf,
                              const uint8_t* object_allowed, int32_t n_obj,
                              uint64_t* out, int64_t cap);
int64_t oracle_ee_pairs_sweep(const double* ebox, const int32_t* e_obj, const int32_t* edges, int64_t ne,
                              const uint8_t* object_allowed, int32_t n_obj,
                              uint64_t* out, int64_t cap);

/* Object-pair permission (PrepareScene, :497-545): object boxes over all
 * referenced vertices at t0 and t1 expanded by thickness; allowed[a][b] =
 * (a == b && !exclude_self) || (a != b && boxes overlap). */
void oracle_object_allowed(const double* v_t0, const double* v_t1, const int32_t* v_obj, int64_t nv,
                           int32_t n_obj, double thickness, int exclude_self, uint8_t* allowed_out);

/* Priority-ordered any-hit with fallback replay (RunScheduledAnyHitRows,
 * :1283-1410).  Candidates are in input order with group ids in [0, n_groups),
 * a per-candidate hit flag (from certification), and per group the candidate
 * indices of its top-K in priority order (CSR: top_offsets[n_groups+1],
 * top_index).  Outputs per group: detected flag, proposal-phase exact calls,
 * fallback-phase exact calls; per candidate: evaluated flag. */
void oracle_group_anyhit(int64_t n_cand, const int32_t* cand_group, const uint8_t* cand_hit,
                         int32_t n_groups, const int64_t* top_offsets, const int64_t* top_index,
                         uint8_t* group_detected, int64_t* group_proposal_calls,
                         int64_t* group_fallback_calls, uint8_t* cand_evaluated);

/* Conservative refinement children (certificate_engine.cpp:663-720) for the
 * interval part of a work item: returns the child count (0, 1 or 2) and writes
 * child intervals.  status/next_refinement_mode/toi_upper are the parent's
 * certificate fields. */
int oracle_refinement_children(double parent_t0, double parent_t1, uint16_t parent_depth,
                               uint8_t status, uint8_t next_refinement_mode, double toi_upper,
                               uint16_t max_child_depth, double min_interval_width,
                               double* child_t0, double* child_t1);

#ifdef __cplusplus
}
#endif

#endif
