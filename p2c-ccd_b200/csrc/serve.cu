// serve.cu — continuous batching of CCD steps on one GPU (p2c_serve_*).
//
// The host runtime around the batched kernels: resident meshes and their
// candidate state, one device arena allocated at creation (first-fit ranges,
// so a group is admitted when its memory fits, whatever the sizes of the
// groups in flight), page-locked staging per slot, one stream per slot.  A
// group's device work is one p2c_batch_candidates sequence plus either one
// p2c_batch_certify launch or one p2c_batch_anyhit sequence; nothing on that
// path allocates or synchronises.  Completion is observed with events.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <deque>
#include <iterator>
#include <map>
#include <vector>

#include "certify_launch.cuh"
#include "p2c_b200.h"
#include "p2c_internal.cuh"

namespace p2c {
namespace {

constexpr size_t kNoRange = ~size_t(0);

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// First-fit ranges of one device allocation; freed ranges merge with their
// neighbours.
class Arena {
 public:
  void init(size_t bytes) {
    bytes_ = bytes;
    free_.clear();
    free_[0] = bytes;
  }
  size_t alloc(size_t bytes) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      const size_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > bytes) free_[off + bytes] = len - bytes;
      in_use_ += bytes;
      peak_ = std::max(peak_, in_use_);
      return off;
    }
    return kNoRange;
  }
  void release(size_t off, size_t bytes) {
    in_use_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t bytes() const { return bytes_; }
  size_t in_use() const { return in_use_; }
  size_t peak() const { return peak_; }

 private:
  size_t bytes_ = 0, in_use_ = 0, peak_ = 0;
  std::map<size_t, size_t> free_;
};

struct Mesh {
  int64_t nv = 0, nf = 0, ne = 0;
  int32_t n_obj = 1, exclude_self = 1;
  double thickness = 0.0;
  int32_t *faces = nullptr, *edges = nullptr, *v_obj = nullptr, *f_obj = nullptr, *e_obj = nullptr;
  int64_t vf_cap = 0, ee_cap = 0;
};

struct Req {
  int64_t id = 0;
  p2c_serve_request r{};
  cudaEvent_t arrival = nullptr;
  int32_t reruns = 0;
};

// Byte layout of one group inside its arena range.
struct GroupPlan {
  size_t table = 0, counts = 0, summaries = 0, seeds = 0, groups = 0, uq = 0, ws_bb = 0, ws_nar = 0;
  size_t ws_bb_bytes = 0, ws_nar_bytes = 0, total = 0;
  std::vector<size_t> v0, v1, vfp, eep, vfr, eer;
  std::vector<int64_t> vf_cap, ee_cap;
  int64_t uq_cap = 0;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
  std::vector<Req> reqs;
  GroupPlan plan;
  size_t off = kNoRange;
  std::vector<p2c_batch_scene> table;
  // page-locked staging (max_group rows each)
  p2c_batch_scene* h_table = nullptr;
  uint64_t* h_counts = nullptr;
  p2c_scene_summary* h_summ = nullptr;
  p2c_anyhit_summary* h_ah = nullptr;
  uint64_t* h_seeds = nullptr;
};

}  // namespace

struct ServeState {
  p2c_serve_config cfg{};
  int device = -1;
  char* arena_base = nullptr;
  Arena arena;
  std::vector<Mesh> meshes;
  std::deque<Req> pending;
  std::deque<p2c_serve_result> finished;
  std::vector<Slot> slots;
  std::vector<cudaEvent_t> event_pool;
  cudaStream_t clock = nullptr;
  int64_t next_id = 0;
  int64_t uq_cap = 0;
  p2c_serve_stats st{};
};

namespace {

cudaEvent_t take_event(ServeState& S) {
  if (!S.event_pool.empty()) {
    cudaEvent_t e = S.event_pool.back();
    S.event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

bool anyhit_mode(const ServeState& S) { return S.cfg.narrow == P2C_SERVE_ANYHIT; }

// Memory plan of a group of requests (offsets within its range).
GroupPlan plan_group(const ServeState& S, const std::vector<Req>& reqs) {
  GroupPlan p;
  const int n = (int)reqs.size();
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += align256(bytes);
    return o;
  };
  p.table = take(sizeof(p2c_batch_scene) * n);
  p.counts = take(32ull * n);
  std::vector<p2c_batch_scene> sizes(n);
  size_t groups = 0;
  for (int j = 0; j < n; ++j) {
    const Mesh& m = S.meshes[reqs[j].r.mesh_id];
    p.vf_cap.push_back(std::max<int64_t>(1, m.vf_cap));
    p.ee_cap.push_back(std::max<int64_t>(1, m.ee_cap));
    p.v0.push_back(take(24ull * m.nv));
    p.v1.push_back(take(24ull * m.nv));
    p.vfp.push_back(take(8ull * p.vf_cap[j]));
    p.eep.push_back(take(8ull * p.ee_cap[j]));
    if (!anyhit_mode(S)) {
      p.vfr.push_back(take(sizeof(p2c_interval_result) * p.vf_cap[j]));
      p.eer.push_back(take(sizeof(p2c_interval_result) * p.ee_cap[j]));
    }
    p2c_batch_scene& d = sizes[j];
    std::memset(&d, 0, sizeof(d));
    d.nv = m.nv;
    d.nf = m.nf;
    d.ne = m.ne;
    d.vf_cap = p.vf_cap[j];
    d.ee_cap = p.ee_cap[j];
    d.n_obj = m.n_obj;
    d.exclude_self = m.exclude_self;
    d.thickness = m.thickness;
    groups += 2ull * (size_t)m.n_obj * (size_t)m.n_obj;
  }
  p.ws_bb_bytes = p2c_batch_candidates_workspace_bytes(sizes.data(), n);
  p.ws_bb = take(p.ws_bb_bytes);
  if (anyhit_mode(S)) {
    p.summaries = take(sizeof(p2c_anyhit_summary) * 2 * n);
    p.seeds = take(8ull * n);
    p.groups = take(std::max<size_t>(groups, 1));
    p.ws_nar_bytes = p2c_batch_anyhit_workspace_bytes(sizes.data(), n, 3u);
  } else {
    p.summaries = take(sizeof(p2c_scene_summary) * n);
    p.uq_cap = S.uq_cap;
    p.uq = take(8ull * p.uq_cap);
    p.ws_nar_bytes = p2c_batch_certify_workspace_bytes(n);
  }
  p.ws_nar = take(p.ws_nar_bytes);
  p.total = off;
  return p;
}

void fail_request(ServeState& S, const Req& q, int code) {
  p2c_serve_result r{};
  r.request_id = q.id;
  r.status = code;
  r.reruns = q.reruns;
  S.finished.push_back(r);
  if (q.arrival != nullptr) S.event_pool.push_back(q.arrival);
  S.st.failed += 1;
}

int launch_group(ServeState& S, Slot& sl) {
  const int n = (int)sl.reqs.size();
  GroupPlan& p = sl.plan;
  char* base = S.arena_base + sl.off;
  auto at = [&](size_t o) { return static_cast<void*>(base + o); };
  sl.table.assign(n, p2c_batch_scene{});
  for (int j = 0; j < n; ++j) {
    const Mesh& m = S.meshes[sl.reqs[j].r.mesh_id];
    p2c_batch_scene& d = sl.table[j];
    d.v_t0 = static_cast<const double*>(at(p.v0[j]));
    d.v_t1 = static_cast<const double*>(at(p.v1[j]));
    d.faces = m.faces;
    d.edges = m.edges;
    d.vf_pairs = static_cast<uint64_t*>(at(p.vfp[j]));
    d.ee_pairs = static_cast<uint64_t*>(at(p.eep[j]));
    d.vf_cap = p.vf_cap[j];
    d.ee_cap = p.ee_cap[j];
    d.counts = static_cast<uint64_t*>(at(p.counts)) + 4 * j;
    d.vf_results = anyhit_mode(S) ? nullptr : static_cast<p2c_interval_result*>(at(p.vfr[j]));
    d.ee_results = anyhit_mode(S) ? nullptr : static_cast<p2c_interval_result*>(at(p.eer[j]));
    d.v_obj = m.v_obj;
    d.f_obj = m.f_obj;
    d.e_obj = m.e_obj;
    d.nv = m.nv;
    d.nf = m.nf;
    d.ne = m.ne;
    d.thickness = m.thickness;
    d.exclude_self = m.exclude_self;
    d.n_obj = m.n_obj;
    sl.h_table[j] = d;
    sl.h_seeds[j] = sl.reqs[j].r.seed;
  }
  cudaStream_t s = sl.stream;
  P2C_CUDA(cudaMemcpyAsync(at(p.table), sl.h_table, sizeof(p2c_batch_scene) * n, cudaMemcpyHostToDevice, s));
  for (int j = 0; j < n; ++j) {
    const Mesh& m = S.meshes[sl.reqs[j].r.mesh_id];
    P2C_CUDA(cudaMemcpyAsync(at(p.v0[j]), sl.reqs[j].r.v_t0, 24ull * m.nv, cudaMemcpyHostToDevice, s));
    P2C_CUDA(cudaMemcpyAsync(at(p.v1[j]), sl.reqs[j].r.v_t1, 24ull * m.nv, cudaMemcpyHostToDevice, s));
  }
  const p2c_batch_scene* d_table = static_cast<const p2c_batch_scene*>(at(p.table));
  int rc = p2c_batch_candidates(sl.table.data(), d_table, n, at(p.ws_bb), p.ws_bb_bytes, s);
  if (rc != P2C_OK) return rc;
  if (anyhit_mode(S)) {
    P2C_CUDA(cudaMemcpyAsync(at(p.seeds), sl.h_seeds, 8ull * n, cudaMemcpyHostToDevice, s));
    rc = p2c_batch_anyhit(sl.table.data(), d_table, n, 3u, nullptr, static_cast<const uint64_t*>(at(p.seeds)),
                          S.cfg.top_k, S.cfg.interval_t0, S.cfg.interval_t1, &S.cfg.cert,
                          static_cast<p2c_anyhit_summary*>(at(p.summaries)), static_cast<uint8_t*>(at(p.groups)),
                          nullptr, nullptr, at(p.ws_nar), p.ws_nar_bytes, s);
    if (rc != P2C_OK) return rc;
    P2C_CUDA(cudaMemcpyAsync(sl.h_ah, at(p.summaries), sizeof(p2c_anyhit_summary) * 2 * n, cudaMemcpyDeviceToHost, s));
  } else {
    rc = p2c_batch_certify(d_table, n, S.cfg.interval_t0, S.cfg.interval_t1, &S.cfg.cert, 3u,
                           static_cast<p2c_scene_summary*>(at(p.summaries)), static_cast<uint64_t*>(at(p.uq)),
                           p.uq_cap, nullptr, at(p.ws_nar), p.ws_nar_bytes, s);
    if (rc != P2C_OK) return rc;
    P2C_CUDA(cudaMemcpyAsync(sl.h_summ, at(p.summaries), sizeof(p2c_scene_summary) * n, cudaMemcpyDeviceToHost, s));
  }
  P2C_CUDA(cudaMemcpyAsync(sl.h_counts, at(p.counts), 32ull * n, cudaMemcpyDeviceToHost, s));
  P2C_CUDA(cudaEventRecord(sl.done, s));
  return P2C_OK;
}

// Fill the optional host outputs of request j of a finished group.
int copy_outputs(ServeState& S, Slot& sl, int j, p2c_serve_result& res, const std::vector<uint64_t>& uq_all) {
  const Req& q = sl.reqs[j];
  const GroupPlan& p = sl.plan;
  char* base = S.arena_base + sl.off;
  const uint64_t n_vf = sl.h_counts[4 * j], n_ee = sl.h_counts[4 * j + 1];
  if (!anyhit_mode(S)) {
    if (q.r.vf_results != nullptr || q.r.ee_results != nullptr) {
      const int64_t cap = std::max<int64_t>(0, q.r.results_cap);
      const uint64_t a = std::min<uint64_t>(n_vf, (uint64_t)cap), b = std::min<uint64_t>(n_ee, (uint64_t)cap);
      if (a < n_vf || b < n_ee) res.truncated |= 1ull;
      if (q.r.vf_results != nullptr && a > 0)
        P2C_CUDA(cudaMemcpyAsync(q.r.vf_results, base + p.vfr[j], sizeof(p2c_interval_result) * a,
                                 cudaMemcpyDeviceToHost, sl.stream));
      if (q.r.ee_results != nullptr && b > 0)
        P2C_CUDA(cudaMemcpyAsync(q.r.ee_results, base + p.eer[j], sizeof(p2c_interval_result) * b,
                                 cudaMemcpyDeviceToHost, sl.stream));
      P2C_CUDA(cudaStreamSynchronize(sl.stream));
    }
    res.undecided_entries = sl.h_summ[j].undecided_queued;
    if (q.r.undecided != nullptr) {
      int64_t k = 0;
      for (uint64_t e : uq_all) {
        if ((int)(e >> 40) != j) continue;
        if (k < q.r.undecided_cap) q.r.undecided[k] = (((e >> 39) & 1ull) << 63) | (e & ((1ull << 39) - 1ull));
        ++k;
      }
      if (k > q.r.undecided_cap) res.truncated |= 2ull;
    }
  } else if (q.r.group_detected != nullptr) {
    const Mesh& m = S.meshes[q.r.mesh_id];
    const int64_t g = 2ll * m.n_obj * m.n_obj;
    const int64_t c = std::min<int64_t>(g, std::max<int64_t>(0, q.r.groups_cap));
    if (c < g) res.truncated |= 4ull;
    // the group space is family-major: this request's VF groups, then (after
    // every request's VF groups) its EE groups
    size_t vf_base = 0, ee_base = 0, total_vf = 0;
    for (size_t i = 0; i < sl.reqs.size(); ++i) {
      const Mesh& mi = S.meshes[sl.reqs[i].r.mesh_id];
      const size_t gi = (size_t)mi.n_obj * mi.n_obj;
      if ((int)i < j) vf_base += gi;
      total_vf += gi;
    }
    ee_base = total_vf + vf_base;
    const int64_t half = (int64_t)m.n_obj * m.n_obj;
    const int64_t a = std::min(c, half), b = std::max<int64_t>(0, c - half);
    if (a > 0)
      P2C_CUDA(cudaMemcpyAsync(q.r.group_detected, base + p.groups + vf_base, a, cudaMemcpyDeviceToHost, sl.stream));
    if (b > 0)
      P2C_CUDA(cudaMemcpyAsync(q.r.group_detected + half, base + p.groups + ee_base, b, cudaMemcpyDeviceToHost,
                               sl.stream));
    P2C_CUDA(cudaStreamSynchronize(sl.stream));
  }
  return P2C_OK;
}

int complete_group(ServeState& S, Slot& sl) {
  const int n = (int)sl.reqs.size();
  std::vector<uint64_t> uq_all;
  uint64_t uq_total = 0;
  if (!anyhit_mode(S)) {
    bool want = false;
    for (int j = 0; j < n; ++j) {
      uq_total += sl.h_summ[j].undecided_queued;
      want = want || sl.reqs[j].r.undecided != nullptr;
    }
    // entries of a request that found the queue full are flagged (bit 8) and
    // the request re-runs; every other request's entries were all written
    const uint64_t written = std::min<uint64_t>(uq_total, (uint64_t)sl.plan.uq_cap);
    if (want && written > 0) {
      uq_all.resize(written);
      P2C_CUDA(cudaMemcpyAsync(uq_all.data(), S.arena_base + sl.off + sl.plan.uq, 8ull * written,
                               cudaMemcpyDeviceToHost, sl.stream));
      P2C_CUDA(cudaStreamSynchronize(sl.stream));
    }
  }
  std::vector<Req> rerun;
  for (int j = 0; j < n; ++j) {
    Req& q = sl.reqs[j];
    Mesh& m = S.meshes[q.r.mesh_id];
    const uint64_t n_vf = sl.h_counts[4 * j], n_ee = sl.h_counts[4 * j + 1], flags = sl.h_counts[4 * j + 2];
    if (flags & 1ull) {
      fail(P2C_ERR_INVALID, "request %lld: scene trajectories must be finite", (long long)q.id);
      fail_request(S, q, P2C_ERR_INVALID);
      continue;
    }
    if ((int64_t)n_vf > sl.plan.vf_cap[j] || (int64_t)n_ee > sl.plan.ee_cap[j]) {
      m.vf_cap = std::max<int64_t>(m.vf_cap, (int64_t)(n_vf + n_vf / 4) + 1024);
      m.ee_cap = std::max<int64_t>(m.ee_cap, (int64_t)(n_ee + n_ee / 4) + 1024);
      q.reruns += 1;
      rerun.push_back(q);
      continue;
    }
    const uint64_t err = anyhit_mode(S) ? (sl.h_ah[2 * j].error_word | sl.h_ah[2 * j + 1].error_word)
                                        : sl.h_summ[j].error_word;
    if (err & 1ull) {
      fail(P2C_ERR_TIMEOUT, "certification exceeded the device time budget (P2C_DEVICE_BUDGET_MS)");
      fail_request(S, q, P2C_ERR_TIMEOUT);
      continue;
    }
    if (!anyhit_mode(S) && (err & 8ull)) {
      q.reruns += 1;
      rerun.push_back(q);
      continue;
    }
    // candidate state: the mesh's next requests get buffers fitted to this step's counts
    m.vf_cap = std::min<int64_t>(m.vf_cap, (int64_t)(n_vf + n_vf / 4) + 1024);
    m.ee_cap = std::min<int64_t>(m.ee_cap, (int64_t)(n_ee + n_ee / 4) + 1024);
    p2c_serve_result res{};
    res.request_id = q.id;
    res.status = P2C_OK;
    res.reruns = q.reruns;
    res.vf_candidates = n_vf;
    res.ee_candidates = n_ee;
    float ms = 0.0f;
    P2C_CUDA(cudaEventElapsedTime(&ms, q.arrival, sl.done));
    res.latency_ms = ms;
    if (anyhit_mode(S)) {
      res.anyhit[0] = sl.h_ah[2 * j];
      res.anyhit[1] = sl.h_ah[2 * j + 1];
      S.st.calls += res.anyhit[0].proposal_calls + res.anyhit[0].fallback_calls + res.anyhit[1].proposal_calls +
                    res.anyhit[1].fallback_calls;
    } else {
      res.certify = sl.h_summ[j];
      S.st.calls += n_vf + n_ee;
    }
    int rc = copy_outputs(S, sl, j, res, uq_all);
    if (rc != P2C_OK) return rc;
    S.st.candidates += n_vf + n_ee;
    S.st.completed += 1;
    S.finished.push_back(res);
    S.event_pool.push_back(q.arrival);
  }
  if (uq_total > (uint64_t)sl.plan.uq_cap)
    S.uq_cap = std::max<int64_t>(S.uq_cap, (int64_t)(uq_total + uq_total / 4) + 1024);
  S.st.reruns += rerun.size();
  for (auto it = rerun.rbegin(); it != rerun.rend(); ++it) S.pending.push_front(*it);
  S.arena.release(sl.off, sl.plan.total);
  sl.off = kNoRange;
  sl.busy = false;
  sl.reqs.clear();
  return P2C_OK;
}

// Triangles a group takes before it closes (a larger request still forms a
// group alone): a long step holds its whole group, so small requests are not
// batched behind it and the slots stay busy with work of similar length.
#ifndef P2C_SERVE_GROUP_TRIANGLES
#define P2C_SERVE_GROUP_TRIANGLES 600000
#endif
constexpr long long kGroupTriangles = P2C_SERVE_GROUP_TRIANGLES;

// Admit waiting requests into a free slot, in arrival order: as many as
// max_group allows while the group stays within kGroupTriangles and its
// memory fits a free range of the arena.
int admit_into(ServeState& S, Slot& sl, bool others_in_flight) {
  std::vector<Req> group;
  GroupPlan plan;
  long long tris = 0;
  while (!S.pending.empty() && (int)group.size() < S.cfg.max_group) {
    const long long nf = S.meshes[S.pending.front().r.mesh_id].nf;
    if (!group.empty() && tris + nf > kGroupTriangles) break;
    tris += nf;
    group.push_back(S.pending.front());
    GroupPlan p = plan_group(S, group);
    const size_t o = S.arena.alloc(p.total);  // does the larger group still fit a free range?
    if (o == kNoRange) {
      group.pop_back();
      if (group.empty() && !others_in_flight) {
        // alone on an idle server it does not fit: it never will
        fail(P2C_ERR_CAPACITY, "request %lld needs %zu bytes of device memory; the serving arena holds %zu",
             (long long)S.pending.front().id, p.total, S.arena.bytes());
        fail_request(S, S.pending.front(), P2C_ERR_CAPACITY);
        S.pending.pop_front();
        continue;
      }
      break;
    }
    S.arena.release(o, p.total);
    S.pending.pop_front();
    plan = std::move(p);
  }
  if (group.empty()) return P2C_OK;
  sl.off = S.arena.alloc(plan.total);  // fitted a moment ago, nothing allocated since
  sl.reqs = std::move(group);
  sl.plan = std::move(plan);
  sl.busy = true;
  S.st.groups += 1;
  const int rc = launch_group(S, sl);
  if (rc != P2C_OK) {
    for (const Req& q : sl.reqs) fail_request(S, q, rc);
    cudaStreamSynchronize(sl.stream);  // nothing of the group may still use its range
    S.arena.release(sl.off, sl.plan.total);
    sl.busy = false;
    sl.reqs.clear();
    sl.off = kNoRange;
  }
  return P2C_OK;
}

int copy_host_array(void** dst, const void* src, size_t bytes) {
  if (bytes == 0) {
    *dst = nullptr;
    return P2C_OK;
  }
  P2C_CUDA(cudaMalloc(dst, bytes));
  P2C_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
  return P2C_OK;
}

}  // namespace
}  // namespace p2c

struct p2c_serve : p2c::ServeState {};

extern "C" {

int p2c_serve_create(const p2c_serve_config* config, p2c_serve** out) {
  using namespace p2c;
  if (config == nullptr || out == nullptr) return fail(P2C_ERR_INVALID, "config and out pointers are required");
  const p2c_serve_config& c = *config;
  if (c.slots < 1 || c.slots > 64) return fail(P2C_ERR_INVALID, "slots must lie in [1, 64]");
  if (c.max_group < 1 || c.max_group > 4096) return fail(P2C_ERR_INVALID, "max_group must lie in [1, 4096]");
  if (c.narrow != P2C_SERVE_CERTIFY && c.narrow != P2C_SERVE_ANYHIT)
    return fail(P2C_ERR_INVALID, "narrow must be P2C_SERVE_CERTIFY or P2C_SERVE_ANYHIT");
  if (c.top_k < 0) return fail(P2C_ERR_INVALID, "top_k must be non-negative");
  if (c.memory_budget < 0 || c.undecided_capacity < 0)
    return fail(P2C_ERR_INVALID, "memory_budget and undecided_capacity must be non-negative");
  int rc = validate_cert_config(c.cert, c.interval_t0, c.interval_t1);
  if (rc != P2C_OK) return rc;
  p2c_serve* S = new p2c_serve();
  S->cfg = c;
  auto bail = [&](int code) {
    p2c_serve_destroy(S);
    return code;
  };
  if (cudaGetDevice(&S->device) != cudaSuccess) return bail(fail(P2C_ERR_CUDA, "no current CUDA device"));
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return bail(fail(P2C_ERR_CUDA, "cudaMemGetInfo failed"));
  size_t budget = c.memory_budget > 0 ? (size_t)c.memory_budget : free_b / 2;
  budget = align256(budget);
  if (cudaMalloc(reinterpret_cast<void**>(&S->arena_base), budget) != cudaSuccess)
    return bail(fail(P2C_ERR_CUDA, "could not allocate the %zu-byte serving arena", budget));
  S->arena.init(budget);
  S->uq_cap = c.undecided_capacity > 0 ? c.undecided_capacity : (1 << 14);
  if (cudaStreamCreateWithFlags(&S->clock, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(P2C_ERR_CUDA, "stream creation failed"));
  S->slots.resize(c.slots);
  for (Slot& sl : S->slots) {
    if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&sl.done) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&sl.h_table), sizeof(p2c_batch_scene) * c.max_group) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&sl.h_counts), 32ull * c.max_group) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&sl.h_summ), sizeof(p2c_scene_summary) * c.max_group) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&sl.h_ah), sizeof(p2c_anyhit_summary) * 2 * c.max_group) !=
            cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&sl.h_seeds), 8ull * c.max_group) != cudaSuccess)
      return bail(fail(P2C_ERR_CUDA, "slot set-up failed (stream, event or page-locked staging)"));
  }
  S->st.arena_bytes = budget;
  *out = S;
  return P2C_OK;
}

int p2c_serve_destroy(p2c_serve* S) {
  using namespace p2c;
  if (S == nullptr) return P2C_OK;
  for (Slot& sl : S->slots) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    for (Req& q : sl.reqs)
      if (q.arrival) cudaEventDestroy(q.arrival);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    if (sl.h_table) cudaFreeHost(sl.h_table);
    if (sl.h_counts) cudaFreeHost(sl.h_counts);
    if (sl.h_summ) cudaFreeHost(sl.h_summ);
    if (sl.h_ah) cudaFreeHost(sl.h_ah);
    if (sl.h_seeds) cudaFreeHost(sl.h_seeds);
  }
  for (Req& q : S->pending)
    if (q.arrival) cudaEventDestroy(q.arrival);
  for (cudaEvent_t e : S->event_pool) cudaEventDestroy(e);
  for (Mesh& m : S->meshes)
    for (int32_t* p : {m.faces, m.edges, m.v_obj, m.f_obj, m.e_obj})
      if (p) cudaFree(p);
  if (S->clock) cudaStreamDestroy(S->clock);
  if (S->arena_base) cudaFree(S->arena_base);
  delete S;
  return P2C_OK;
}

int p2c_serve_register_mesh(p2c_serve* S, const p2c_serve_mesh* mesh, int32_t* mesh_id) {
  using namespace p2c;
  if (S == nullptr || mesh == nullptr || mesh_id == nullptr) return fail(P2C_ERR_INVALID, "null argument");
  const p2c_serve_mesh& h = *mesh;
  if (h.nv < 0 || h.nf < 0 || h.ne < 0 || h.nv >= (1 << 22) || h.nf >= (1 << 22) || h.ne >= (1 << 22))
    return fail(P2C_ERR_INVALID, "mesh sizes must lie in [0, 2^22)");
  if ((h.nf > 0 && (h.faces == nullptr || h.f_obj == nullptr)) || (h.ne > 0 && (h.edges == nullptr || h.e_obj == nullptr)) ||
      (h.nv > 0 && h.v_obj == nullptr))
    return fail(P2C_ERR_INVALID, "mesh arrays are required for non-empty lists");
  if (h.n_obj < 1 || h.n_obj > 4096) return fail(P2C_ERR_INVALID, "mesh n_obj must lie in [1, 4096]");
  if (!(h.thickness >= 0.0) || h.thickness > 1e300) return fail(P2C_ERR_INVALID, "thickness must be finite and >= 0");
  for (int64_t i = 0; i < 3 * h.nf; ++i)
    if (h.faces[i] < 0 || h.faces[i] >= h.nv) return fail(P2C_ERR_INVALID, "face %lld: vertex index out of range", (long long)(i / 3));
  for (int64_t i = 0; i < 2 * h.ne; ++i)
    if (h.edges[i] < 0 || h.edges[i] >= h.nv) return fail(P2C_ERR_INVALID, "edge %lld: vertex index out of range", (long long)(i / 2));
  Mesh m;
  m.nv = h.nv;
  m.nf = h.nf;
  m.ne = h.ne;
  m.n_obj = h.n_obj;
  m.exclude_self = h.exclude_self ? 1 : 0;
  m.thickness = h.thickness;
  m.vf_cap = h.vf_capacity > 0 ? h.vf_capacity : std::max<int64_t>(1024, h.nf / 2);
  m.ee_cap = h.ee_capacity > 0 ? h.ee_capacity : std::max<int64_t>(1024, h.nf);
  int rc = P2C_OK;
  if ((rc = copy_host_array(reinterpret_cast<void**>(&m.faces), h.faces, 12ull * h.nf)) != P2C_OK ||
      (rc = copy_host_array(reinterpret_cast<void**>(&m.edges), h.edges, 8ull * h.ne)) != P2C_OK ||
      (rc = copy_host_array(reinterpret_cast<void**>(&m.v_obj), h.v_obj, 4ull * h.nv)) != P2C_OK ||
      (rc = copy_host_array(reinterpret_cast<void**>(&m.f_obj), h.f_obj, 4ull * h.nf)) != P2C_OK ||
      (rc = copy_host_array(reinterpret_cast<void**>(&m.e_obj), h.e_obj, 4ull * h.ne)) != P2C_OK) {
    for (int32_t* p : {m.faces, m.edges, m.v_obj, m.f_obj, m.e_obj})
      if (p) cudaFree(p);
    return rc;
  }
  S->meshes.push_back(m);
  *mesh_id = (int32_t)(S->meshes.size() - 1);
  return P2C_OK;
}

int p2c_serve_admit(p2c_serve* S, const p2c_serve_request* request, int64_t* request_id) {
  using namespace p2c;
  if (S == nullptr || request == nullptr) return fail(P2C_ERR_INVALID, "null argument");
  const p2c_serve_request& r = *request;
  if (r.mesh_id < 0 || r.mesh_id >= (int32_t)S->meshes.size()) return fail(P2C_ERR_INVALID, "mesh %d is not registered", r.mesh_id);
  if (S->meshes[r.mesh_id].nv > 0 && (r.v_t0 == nullptr || r.v_t1 == nullptr))
    return fail(P2C_ERR_INVALID, "request trajectories are required");
  Req q;
  q.id = S->next_id++;
  q.r = r;
  q.arrival = take_event(*S);
  if (q.arrival == nullptr) return fail(P2C_ERR_CUDA, "event creation failed");
  P2C_CUDA(cudaEventRecord(q.arrival, S->clock));
  S->pending.push_back(q);
  S->st.admitted += 1;
  if (request_id != nullptr) *request_id = q.id;
  return P2C_OK;
}

int p2c_serve_poll(p2c_serve* S, p2c_serve_result* results, int32_t max_results, int32_t* n_results) {
  using namespace p2c;
  if (S == nullptr) return fail(P2C_ERR_INVALID, "null server");
  for (Slot& sl : S->slots) {
    if (!sl.busy) continue;
    const cudaError_t e = cudaEventQuery(sl.done);
    if (e == cudaErrorNotReady) continue;
    if (e != cudaSuccess) return fail(P2C_ERR_CUDA, "group completion: %s", cudaGetErrorString(e));
    const int rc = complete_group(*S, sl);
    if (rc != P2C_OK) return rc;
  }
  for (Slot& sl : S->slots) {
    if (sl.busy || S->pending.empty()) continue;
    bool others = false;
    for (const Slot& o : S->slots) others = others || o.busy;
    const int rc = admit_into(*S, sl, others);
    if (rc != P2C_OK) return rc;
  }
  int32_t k = 0;
  while (results != nullptr && k < max_results && !S->finished.empty()) {
    results[k++] = S->finished.front();
    S->finished.pop_front();
  }
  if (n_results != nullptr) *n_results = k;
  return P2C_OK;
}

int p2c_serve_read_stats(p2c_serve* S, p2c_serve_stats* out) {
  using namespace p2c;
  if (S == nullptr || out == nullptr) return fail(P2C_ERR_INVALID, "null argument");
  p2c_serve_stats st = S->st;
  st.pending = S->pending.size();
  uint64_t fl = 0;
  for (const Slot& sl : S->slots) fl += sl.busy ? sl.reqs.size() : 0;
  st.in_flight = fl;
  st.arena_bytes = S->arena.bytes();
  st.arena_in_use = S->arena.in_use();
  st.arena_peak = S->arena.peak();
  *out = st;
  return P2C_OK;
}

}  // extern "C"
