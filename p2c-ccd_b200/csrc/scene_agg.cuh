// scene_agg.cuh — the CertificateEngine::Evaluate reduction of one scene's
// candidate certificates (certificate_engine.cpp:729-824), accumulated with
// atomics as certificates finish, and the scene summary written from it.
#pragma once

#include "certify_core.cuh"

namespace p2c {

struct SceneAgg {
  unsigned long long coll_key;     // min over collisions of (family - 1) << 63 | pair key
  unsigned long long margin_bits;  // min separation margin (bit pattern of a non-negative double)
  unsigned int any_sep[2];
  unsigned int any_undecided[2];
  unsigned long long collisions, separations, undecided, queued;
  unsigned long long n_certified[2];
  unsigned int dropped;  // an undecided entry of this scene found the queue full
};

__device__ __forceinline__ void scene_agg_init(SceneAgg& a) {
  SceneAgg z{};
  z.coll_key = ~0ull;
  z.margin_bits = 0x7ff0000000000000ull;  // +inf
  a = z;
}

// One finished certificate of family fam (1: VF, 2: EE) with pair key `key`;
// an undecided one is appended to the undecided (fallback-replay) queue as
// `entry` when the queue exists.  Queue slots come from `uq_slots`, the
// counter of everything written to that queue: a queue shared by several
// scenes passes one launch-wide counter (each scene still counts its own
// entries in agg->queued); nullptr means the queue is this scene's alone and
// agg->queued is the slot counter.  An entry past uq_cap is counted but not
// written, and marks the scene (error bit 8 of its summary).
// Lanes that finish together add their counts with one atomic per (scene,
// status); a minimum is only written when it can still decrease.
__device__ __forceinline__ void scene_agg_record(SceneAgg* agg, int fam, unsigned long long key, const Outcome& o,
                                                 unsigned long long* uq, unsigned long long uq_cap,
                                                 unsigned long long* uq_slots, unsigned long long entry) {
  const int f = fam - 1;
  const unsigned act = __activemask();
  const unsigned m = __match_any_sync(act, (reinterpret_cast<unsigned long long>(agg) << 2) | o.status);
  const bool leader = (int)(threadIdx.x & 31) == __ffs((int)m) - 1;
  const unsigned long long n = (unsigned long long)__popc(m);
  // The minima only decrease, so a stale (L1-cached) copy is an upper bound
  // of the current value: skipping the atomic when the new value is not below
  // it never loses a minimum, and the read rarely leaves the SM.
  if (o.status == P2C_STATUS_COLLISION) {
    const unsigned long long k = ((unsigned long long)f << 63) | key;
    if (k < __ldca(&agg->coll_key)) atomicMin(&agg->coll_key, k);
    if (leader) atomicAdd(&agg->collisions, n);
  } else if (o.status == P2C_STATUS_SEPARATION) {
    const unsigned long long mb = (unsigned long long)__double_as_longlong(o.margin);
    if (mb < __ldca(&agg->margin_bits)) atomicMin(&agg->margin_bits, mb);
    if (agg->any_sep[f] == 0u) atomicExch(&agg->any_sep[f], 1u);
    if (leader) atomicAdd(&agg->separations, n);
  } else {
    if (agg->any_undecided[f] == 0u) atomicExch(&agg->any_undecided[f], 1u);
    if (leader) atomicAdd(&agg->undecided, n);
    if (uq != nullptr) {
      const unsigned long long slot = atomicAdd(uq_slots != nullptr ? uq_slots : &agg->queued, 1ull);
      if (uq_slots != nullptr) atomicAdd(&agg->queued, 1ull);
      if (slot < uq_cap) uq[slot] = entry;
      else atomicExch(&agg->dropped, 1u);
    }
  }
}

__device__ __forceinline__ uint8_t refinement_for_reason(uint16_t r) {  // certificate_engine.cpp:279-291
  return r == P2C_REASON_MISSING_GEOMETRY ? P2C_REFINE_REQUEST_GEOMETRY
         : r == P2C_REASON_MAX_SUBDIVISION_DEPTH ? P2C_REFINE_BISECT_INTERVAL
         : r == P2C_REASON_INVALID_INPUT ? P2C_REFINE_REQUEST_GEOMETRY
                                         : P2C_REFINE_ESCALATE_PRECISION;
}

// The collision witness: candidate t of the winning family whose pair key
// won the atomicMin writes the query certificate (keys are unique).
__device__ __forceinline__ void scene_witness(const SceneAgg& a, long long t, const unsigned long long* vf_pairs,
                                              const unsigned long long* ee_pairs, const p2c_interval_result* out_vf,
                                              const p2c_interval_result* out_ee, p2c_scene_summary* summary) {
  if (a.coll_key == ~0ull) return;
  const int f = (int)(a.coll_key >> 63);
  const unsigned long long key = a.coll_key & ~(1ull << 63);
  const long long n = (long long)a.n_certified[f];
  const unsigned long long* pairs = f == 0 ? vf_pairs : ee_pairs;
  if (t < n && pairs[t] == key) {
    const p2c_interval_result& r = (f == 0 ? out_vf : out_ee)[t];
    p2c_query_certificate q{};
    q.status = P2C_STATUS_COLLISION;
    q.witness_family = r.witness_family;
    q.toi_upper = r.toi_upper;
    q.witness_id_a = r.witness_id_a;
    q.witness_id_b = r.witness_id_b;
    q.witness_index = t;
    summary->query = q;
  }
}

// Counts, error word and (without a collision) the undecided-or-separation
// certificate with the reference's reason order.
__device__ __forceinline__ void scene_summary_fields(const SceneAgg& a, unsigned family_mask, double T1,
                                                     unsigned long long error_word, p2c_scene_summary* summary) {
  const long long n_vf = (long long)a.n_certified[0], n_ee = (long long)a.n_certified[1];
  summary->collisions = a.collisions;
  summary->separations = a.separations;
  summary->undecided = a.undecided;
  summary->vf_certified = (unsigned long long)n_vf;
  summary->ee_certified = (unsigned long long)n_ee;
  summary->undecided_queued = a.queued;
  summary->error_word = error_word | (a.dropped ? 8ull : 0ull);
  if (a.coll_key != ~0ull) return;
  p2c_query_certificate q{};
  q.witness_id_a = -1;
  q.witness_id_b = -1;
  q.witness_index = -1;
  q.toi_upper = T1;
  bool evaluated_any = false, has_undecided = false;
  uint16_t reason = P2C_REASON_NONE;
  for (int f = 0; f < 2; ++f) {
    if ((family_mask & (1u << f)) == 0u) continue;
    const long long n = f == 0 ? n_vf : n_ee;
    if (n == 0) {
      has_undecided = true;
      reason = P2C_REASON_MISSING_GEOMETRY;
    } else {
      evaluated_any = true;
      if (a.any_undecided[f]) {
        has_undecided = true;
        reason = P2C_REASON_MAX_SUBDIVISION_DEPTH;
      }
    }
  }
  if (!evaluated_any || has_undecided) {
    const uint16_t r = !evaluated_any ? (uint16_t)P2C_REASON_MISSING_GEOMETRY
                                      : (reason == P2C_REASON_NONE ? (uint16_t)P2C_REASON_MAX_SUBDIVISION_DEPTH
                                                                   : reason);
    q.status = P2C_STATUS_UNDECIDED;
    q.reason_code = r;
    q.next_refinement_mode = refinement_for_reason(r);
  } else {
    q.status = P2C_STATUS_SEPARATION;
    const double m = __longlong_as_double((long long)a.margin_bits);
    q.safe_margin_lb = isfinite(m) ? m : 0.0;
    q.covered_feature_mask = (a.any_sep[0] ? 1u : 0u) | (a.any_sep[1] ? 2u : 0u);
  }
  summary->query = q;
}

}  // namespace p2c
