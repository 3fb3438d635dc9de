// certify_engine.cuh — the persistent warp engine of the interval certifier.
//
// A query is one interval tree (one primitive over one interval).  A lane
// walks a subtree depth-first, left child first, with no stack: a node is
// (path bits, depth) and its endpoints are recomputed from the root by
// replaying the bisections (the same 0.5*(a+b) roundings the reference
// recursion performs, certificate_engine.cpp:311).  Every non-root node needs
// only its midpoint sample: its endpoints are midpoints or endpoints of
// ancestors, already known to be farther than eps_space (otherwise the
// ancestor would be a collision leaf and would not have been split).
//
// Work sharing, in three levels:
//   * queries: warps take queries from per-family queues (at most
//     fetch_limit in flight, so small batches leave lanes free to help);
//   * lanes: an idle lane takes the shallowest pending right subtree of a
//     busy lane of its warp (donation);
//   * warps (kExport): when some warp has nothing to do, busy warps publish
//     pending subtrees to a global pool that idle warps drain, so one deep
//     tree is bisected by many warps.
// The reduction of a tree reproduces the recursion's result exactly: the
// leftmost collision leaf in depth-first order wins (keys are left-aligned
// paths with a sentinel bit below the last level, so disjoint nodes compare
// in depth-first order and the key encodes the leaf), else any undecided leaf
// makes the tree undecided, else separation with the minimum leaf margin.  A
// tree's reduction lives in its warp's shared slot until one of its subtrees
// leaves the warp, then in a pooled global record.  Nodes right of a known
// collision are pruned: the recursion never reaches them.
//
// No wait in this engine is unbounded: every loop checks the launch's device
// time budget (CertParams::budget_ns); on expiry the engine returns false and
// the launcher reports P2C_ERR_TIMEOUT.
#pragma once

#include "certify_core.cuh"

namespace p2c {

// Global reduction record of a tree whose subtrees left its warp.
struct TreeAgg {
  unsigned long long coll_key;     // min leaf_key over collision leaves (~0: none)
  unsigned long long margin_bits;  // min separation margin (bit pattern of a non-negative double)
  unsigned int undecided;          // any undecided leaf
  unsigned int outstanding;        // live units: lanes working in it + pooled tasks
};

struct SubtreeTask {
  unsigned long long path;
  unsigned long long tag;  // 1 + (q << 24 | agg index (16 bits) << 8 | depth << 1 | family - 1); 0 = unpublished
};

// Launch-wide counters, one 128-byte line each: idle warps poll some of them
// while busy warps update others.
struct alignas(128) PaddedCounter {
  unsigned long long v;
  unsigned long long pad[15];
};

struct EngineState {
  PaddedCounter queue_head[2];  // next query of each family
  PaddedCounter finalized;      // queries finished (both families)
  PaddedCounter task_reserve;   // pool slots reserved
  PaddedCounter task_head;      // pool slots claimed
  PaddedCounter agg_next;       // TreeAgg records handed out
  PaddedCounter hungry;         // fully idle warps waiting for subtrees
  PaddedCounter helpers;        // idle warps allowed to stay and wait
};

struct EnginePools {
  TreeAgg* aggs = nullptr;        // capacity agg_cap
  SubtreeTask* tasks = nullptr;   // capacity task_cap
  unsigned long long agg_cap = 0;
  unsigned long long task_cap = 0;
  unsigned long long helper_cap = 0;  // idle warps that wait for subtrees
};

constexpr int kMaxTreeDepth = 63;  // leaf keys need one bit below the deepest level

// Work-sharing parameters of the loop below (compile-time):
//   P2C_EXPORT_LANES   subtrees one warp may publish to the pool per iteration;
//   P2C_EXPORT_FULL    1: only a warp whose lanes are all busy publishes;
//   P2C_EXPORT_SLACK   a lane publishes when its shallowest pending level is
//                      within this many levels of the warp's shallowest;
//   P2C_POOL_POLL      a warp that still has busy lanes looks at the pool
//                      every this many iterations (a fully idle warp every one);
//   P2C_HUNGRY_PERIOD  iterations between reads of the idle-warp count (a
//                      power of two).
#ifndef P2C_EXPORT_LANES
#define P2C_EXPORT_LANES 1
#endif
#ifndef P2C_EXPORT_FULL
#define P2C_EXPORT_FULL 1
#endif
#ifndef P2C_EXPORT_SLACK
#define P2C_EXPORT_SLACK 0
#endif
#ifndef P2C_POOL_POLL
#define P2C_POOL_POLL 8
#endif
#ifndef P2C_HUNGRY_PERIOD
#define P2C_HUNGRY_PERIOD 8
#endif
static_assert((P2C_HUNGRY_PERIOD & (P2C_HUNGRY_PERIOD - 1)) == 0, "P2C_HUNGRY_PERIOD must be a power of two");

// Phase clock of one warp iteration, compiled only with -DP2C_ENGINE_PROFILE
// (a measurement build; the library is built without it): lane 0 of every
// warp adds the SM clock cycles spent in each phase of the loop below to
// g_engine_prof (0 fetch, 1 donation, 2 pool take, 3 idle wait, 4 distance
// sample, 5 classify, 6 record, 7 move to the next node, 8 export,
// 9 finalise, 10 budget check, 11 iterations).
#ifdef P2C_ENGINE_PROFILE
static __device__ unsigned long long g_engine_prof[16];
#define P2C_PROF_DECL              \
  unsigned long long prof_t = 0;   \
  unsigned long long prof_acc[12]; \
  for (int _k = 0; _k < 12; ++_k) prof_acc[_k] = 0ull;
#define P2C_PROF_START() prof_t = clock64();
#define P2C_PROF_MARK(k)                               \
  {                                                    \
    __syncwarp();                                      \
    const unsigned long long _now = clock64();         \
    prof_acc[k] += _now - prof_t;                      \
    prof_t = _now;                                     \
  }
#define P2C_PROF_FLUSH()                                                               \
  if ((threadIdx.x & 31) == 0)                                                         \
    for (int _k = 0; _k < 12; ++_k) atomicAdd(&g_engine_prof[_k], prof_acc[_k]);
#define P2C_PROF_COUNT(k) prof_acc[k] += 1ull;
#else
#define P2C_PROF_DECL
#define P2C_PROF_START()
#define P2C_PROF_MARK(k)
#define P2C_PROF_FLUSH()
#define P2C_PROF_COUNT(k)
#endif

__device__ __forceinline__ unsigned long long leaf_key(unsigned long long path, int depth) {
  return path | (1ull << (63 - depth));
}

// Publication of pooled subtrees and the last decrement of a shared tree
// (P2C_ACQ_REL): a release store of the task tag and an acquire load by its
// taker, and an acquire-release decrement of the tree's outstanding units,
// instead of full fences around relaxed accesses.
#ifndef P2C_ACQ_REL
#define P2C_ACQ_REL 1
#endif
__device__ __forceinline__ void store_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long load_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned decrement_acq_rel(unsigned* p) {  // returns the value before
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(0xffffffffu) : "memory");
  return old;
}

__device__ __forceinline__ unsigned long long volatile_load(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ unsigned volatile_load(const unsigned* p) {
  return *reinterpret_cast<const volatile unsigned*>(p);
}

// Shared per-slot reduction while a tree is private to its warp.
struct SlotAgg {
  double margin[32];     // min margin (as double; non-negative)
  int undecided[32];
  int outstanding[32];   // live lanes of this warp in the tree
  int gidx[32];          // TreeAgg index once shared, else -1
};

struct EngineShared {
  WarpSlots ws;
  SlotAgg sa;
};

// The problem a launch certifies: both families' queries.  P provides
//   long long n(int family) const;
//   bool skip(int family, long long q) const;   // drop q unevaluated (a cancelled candidate)
//   void load(int family, long long q, Geo&, double& T0, double& T1, int& bad) const;
//   void finish(int family, long long q, const Outcome&) const;
//   void invalid(int family, long long q, int bad, double T0, double T1) const;
template <bool kDonate, bool kExport, bool kCount, class P>
__device__ bool run_engine(const P& prob, const CertParams& prm, int fetch1, int fetch2, bool ee_first,
                           EngineShared& sh, WarpStats& st, EngineState* es, const EnginePools& pools,
                           unsigned long long t_start) {
  using Counter = typename std::conditional<kCount, OpCount, NoCount>::type;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  WarpSlots& ws = sh.ws;
  SlotAgg& sa = sh.sa;
  const long long n1 = prob.n(1), n2 = prob.n(2);
  const unsigned long long n_total = (unsigned long long)(n1 + n2);
  const double eps_space = prm.eps_space, eps_time = prm.eps_time;
  const int max_depth = prm.max_depth;

  int slot = -1, fam = 1, phase = 0, depth = 0, sub_depth = 0;
  unsigned long long path = 0, donated = 0;
  double t0 = 0.0, t1 = 0.0, T0 = 0.0, T1 = 0.0, d1root = 0.0;
  double nrm[4];
  Counter ops;
  unsigned free_mask = FULL;
  int cur = ee_first ? 2 : 1;              // family whose queue this warp drains
  unsigned exhausted = (n1 == 0 ? 1u : 0u) | (n2 == 0 ? 2u : 0u);  // bit f-1: family f's queue is empty
  bool hungry = false;                     // this warp is counted in es->hungry
  bool helper = false;                     // this warp is counted in es->helpers
  unsigned backoff = 256;                  // ns slept per idle poll (doubles up to 512 ns)
  unsigned long long pool_hungry = 0, pool_size = 0;
  bool ok = true;

  auto queues_done = [&]() { return exhausted == 3u; };
  P2C_PROF_DECL

  // Finish a tree: one result for query (f, q).
  auto finalize = [&](int f, long long q, const Outcome& o) {
    prob.finish(f, q, o);
    atomicAdd(&es->finalized.v, 1ull);
  };
  auto outcome_from = [&](unsigned long long key, unsigned long long mbits, bool und, double RT0,
                          double RT1) {
    Outcome o;
    if (key != ~0ull) {  // a non-root collision leaf: recover it from its key
      const int d = 64 - __ffsll((long long)key);
      const unsigned long long pth = key & ~(1ull << (63 - d));
      double a, b;
      replay(RT0, RT1, pth, d, a, b);
      o.status = P2C_STATUS_COLLISION;
      o.t0 = a;
      o.t1 = b;
      o.toi = mul(0.5, add(a, b));
      o.margin = 0.0;
    } else if (und) {
      o.status = P2C_STATUS_UNDECIDED;
      o.t0 = RT0;
      o.t1 = RT1;
      o.toi = RT1;
      o.margin = 0.0;
    } else {
      o.status = P2C_STATUS_SEPARATION;
      o.t0 = RT0;
      o.t1 = RT1;
      o.toi = RT1;
      o.margin = __longlong_as_double((long long)mbits);
    }
    return o;
  };

  P2C_PROF_START()
  for (unsigned iter = 0;; ++iter) {
    if ((iter & 63u) == 0u && prm.budget_ns != 0ull) {
      int over = 0;
      if (lane == 0) over = (global_ns() - t_start) > prm.budget_ns;
      if (__shfl_sync(FULL, over, 0)) {
        ok = false;
        break;
      }
    }
    P2C_PROF_MARK(10)
    // ---- (A) new queries from the per-family queues -------------------------
    unsigned idle = __ballot_sync(FULL, slot < 0);
    if (idle != 0u && !queues_done()) {
      if (exhausted & (1u << (cur - 1))) cur = 3 - cur;
      const int fetch_limit = cur == 1 ? fetch1 : fetch2;
      const int room = fetch_limit - (32 - __popc(free_mask));
      if (room > 0) {
        const long long nc = cur == 1 ? n1 : n2;
        const int k = min(__popc(idle), room);
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&es->queue_head[cur - 1].v, (unsigned long long)k);
        base = __shfl_sync(FULL, base, 0);
        if ((long long)base + k >= nc) exhausted |= 1u << (cur - 1);
        bool fresh = false;
        const int r = __popc(idle & lt_mask);
        if (slot < 0 && r < k) {
          const long long q = (long long)base + r;
          if (q < nc) {
            const int s = nth_set_bit(free_mask, r);
            int bad = 0;
            Geo g;
            double RT0, RT1;
            const bool dropped = prob.skip(cur, q);
            if (!dropped) prob.load(cur, q, g, RT0, RT1, bad);
            if (dropped) {
              atomicAdd(&es->finalized.v, 1ull);
            } else if (bad != 0) {
              prob.invalid(cur, q, bad, RT0, RT1);
              atomicAdd(&es->finalized.v, 1ull);
            } else {
              slot = s;
              fresh = true;
              fam = cur;
#pragma unroll
              for (int i = 0; i < 12; ++i) {
                ws.p0[i][s] = g.p0[i];
                ws.p1[i][s] = g.p1[i];
              }
              ws.T0[s] = RT0;
              ws.T1[s] = RT1;
              ws.coll_key[s] = ~0ull;
              ws.qidx[s] = q;
              ws.family[s] = cur;
              sa.margin[s] = INFINITY;
              sa.undecided[s] = 0;
              sa.outstanding[s] = 1;
              sa.gidx[s] = -1;
              T0 = RT0;
              T1 = RT1;
              motion_norms(SlotGeo<WarpSlots>{ws, s}, nrm, ops);
#pragma unroll
              for (int i = 0; i < 4; ++i) ws.nrm[i][s] = nrm[i];
              phase = 0;
              path = 0ull;
              donated = 0ull;
              depth = 0;
              sub_depth = 0;
              t0 = T0;
              t1 = T1;
              st.queries += 1;
            }
          }
        }
        free_mask &= ~__reduce_or_sync(FULL, fresh ? (1u << slot) : 0u);
        __syncwarp();
      }
    }
    P2C_PROF_MARK(0)
    // ---- (B) donation inside the warp ---------------------------------------
    if (kDonate) {
      idle = __ballot_sync(FULL, slot < 0);
      if (idle != 0u) {
        const unsigned long long pend =
            (slot >= 0 && phase == 2) ? pending_levels(path, donated, depth, sub_depth) : 0ull;
        const unsigned donors = __ballot_sync(FULL, pend != 0ull);
        const int npair = min(__popc(idle), __popc(donors));
        if (npair > 0) {
          unsigned long long gpath = 0ull;
          int gdepth = 0, gslot = -1;
          if (((donors >> lane) & 1u) && __popc(donors & lt_mask) < npair) {
            const int b = 63 - __clzll((long long)pend);
            const int l = 64 - b;
            donated |= (1ull << b);
            gpath = (path & top_bits(l - 1)) | (1ull << b);
            gdepth = l;
            gslot = slot;
            atomicAdd(&sa.outstanding[slot], 1);
            const int gi = sa.gidx[slot];
            if (gi >= 0) atomicAdd(&pools.aggs[gi].outstanding, 1u);
            st.donations += 1;
          }
          const bool receiver = ((idle >> lane) & 1u) && __popc(idle & lt_mask) < npair;
          const int src_lane = receiver ? nth_set_bit(donors, __popc(idle & lt_mask)) : lane;
          const unsigned long long rpath = __shfl_sync(FULL, gpath, src_lane);
          const int rdepth = __shfl_sync(FULL, gdepth, src_lane);
          const int rslot = __shfl_sync(FULL, gslot, src_lane);
          __syncwarp();
          if (receiver) {
            slot = rslot;
            fam = ws.family[slot];
            T0 = ws.T0[slot];
            T1 = ws.T1[slot];
#pragma unroll
            for (int i = 0; i < 4; ++i) nrm[i] = ws.nrm[i][slot];  // the owner's rounded values
            path = rpath;
            depth = rdepth;
            sub_depth = rdepth;
            donated = 0ull;
            phase = 2;
            double a, b;
            replay(T0, T1, path, depth - 1, a, b);
            t0 = mul(0.5, add(a, b));
            t1 = b;
          }
          __syncwarp();
        }
      }
    }
    P2C_PROF_MARK(1)
    // ---- (C) subtrees from the global pool ------------------------------------
    if (kExport) {
      idle = __ballot_sync(FULL, slot < 0);
      if (idle != 0u && queues_done() && (idle == FULL || iter % P2C_POOL_POLL == 0u)) {
        unsigned long long h = 0;
        int take = 0;
        if (lane == 0) {
          h = volatile_load(&es->task_head.v);
          const unsigned long long r = min(volatile_load(&es->task_reserve.v), pools.task_cap);
          const unsigned long long avail = r > h ? r - h : 0ull;
          take = (int)min((unsigned long long)__popc(idle), avail);
          if (take > 0 && atomicCAS(&es->task_head.v, h, h + (unsigned long long)take) != h) take = 0;
        }
        take = __shfl_sync(FULL, take, 0);
        h = __shfl_sync(FULL, h, 0);
        const int r = __popc(idle & lt_mask);
        bool fresh = false;
        if (slot < 0 && r < take) {
          // the slot was reserved by a producer that publishes it right after;
          // wait for its tag, bounded by the time budget
          const SubtreeTask* tk = pools.tasks + h + (unsigned long long)r;
          unsigned long long tag = P2C_ACQ_REL ? load_acquire(&tk->tag) : volatile_load(&tk->tag);
          for (unsigned spin = 0; tag == 0ull; ++spin) {
            __nanosleep(64);
            tag = P2C_ACQ_REL ? load_acquire(&tk->tag) : volatile_load(&tk->tag);
            if ((spin & 255u) == 255u && prm.budget_ns != 0ull && (global_ns() - t_start) > prm.budget_ns) break;
          }
          if (tag != 0ull) {
            if (!P2C_ACQ_REL) __threadfence();
            tag -= 1ull;
            const int f = (int)(tag & 1ull) + 1;
            const int d = (int)((tag >> 1) & 127ull);
            const int gi = (int)((tag >> 8) & 0xffffull);
            const long long q = (long long)(tag >> 24);
            const unsigned long long pth = volatile_load(&tk->path);
            const int s = nth_set_bit(free_mask, r);
            Geo g;
            int bad = 0;
            double RT0, RT1;
            prob.load(f, q, g, RT0, RT1, bad);
            slot = s;
            fresh = true;
            fam = f;
#pragma unroll
            for (int i = 0; i < 12; ++i) {
              ws.p0[i][s] = g.p0[i];
              ws.p1[i][s] = g.p1[i];
            }
            ws.T0[s] = RT0;
            ws.T1[s] = RT1;
            ws.coll_key[s] = volatile_load(&pools.aggs[gi].coll_key);
            ws.qidx[s] = q;
            ws.family[s] = f;
            sa.margin[s] = INFINITY;
            sa.undecided[s] = 0;
            sa.outstanding[s] = 1;
            sa.gidx[s] = gi;
            T0 = RT0;
            T1 = RT1;
            NoCount nc;
            motion_norms(SlotGeo<WarpSlots>{ws, s}, nrm, nc);
#pragma unroll
            for (int i = 0; i < 4; ++i) ws.nrm[i][s] = nrm[i];
            path = pth;
            depth = d;
            sub_depth = d;
            donated = 0ull;
            phase = 2;
            double a, b;
            replay(T0, T1, path, depth - 1, a, b);
            t0 = mul(0.5, add(a, b));
            t1 = b;
          }
        }
        free_mask &= ~__reduce_or_sync(FULL, fresh ? (1u << slot) : 0u);
        __syncwarp();
      }
      // a warp is hungry while all its lanes are idle and nothing is left to take
      const bool want = queues_done() && __ballot_sync(FULL, slot < 0) == FULL;
      if (want != hungry) {
        if (lane == 0) {
          if (want) atomicAdd(&es->hungry.v, 1ull);
          else atomicAdd(&es->hungry.v, ~0ull);
        }
        hungry = want;
      }
    }
    P2C_PROF_MARK(2)
    const unsigned busy = __ballot_sync(FULL, slot >= 0);
    if (busy == 0u) {
      if (queues_done()) {
        if (!kExport) break;
        if (volatile_load(&es->finalized.v) >= n_total) break;
        // at most two idle warps per SM stay to take subtrees; the others leave
        if (!helper) {
          int stay = 0;
          if (lane == 0) {
            stay = atomicAdd(&es->helpers.v, 1ull) < pools.helper_cap;
            if (!stay) atomicAdd(&es->helpers.v, ~0ull);
          }
          helper = __shfl_sync(FULL, stay, 0) != 0;
          if (!helper) break;
        }
        __nanosleep(backoff);
        backoff = min(backoff * 2u, 512u);
      }
      P2C_PROF_MARK(3)
      continue;
    }
    P2C_PROF_COUNT(11)
    backoff = 256u;
    st.iters += 1;
    st.busy += (unsigned long long)__popc(busy);
    // ---- (D) prune: a node right of a known collision is never needed --------
    bool done_lane = false;
    if (slot >= 0 && phase == 2 && depth > 0 && ws.coll_key[slot] < leaf_key(path, depth)) done_lane = true;
    const bool active = slot >= 0 && !done_lane;
    // ---- (E) one distance sample per active lane -----------------------------
    double d = 0.0, mid = 0.0;
    if (active) {
      mid = mul(0.5, add(t0, t1));
      const double t = phase == 0 ? t0 : (phase == 1 ? t1 : mid);
      d = fam == 1 ? distance_at<1>(SlotGeo<WarpSlots>{ws, slot}, t, ops)
                   : distance_at<2>(SlotGeo<WarpSlots>{ws, slot}, t, ops);
      st.evals += 1;
      if (phase == 0 || (phase == 2 && depth > 0)) st.nodes += 1;
      if (kCount) ops.add(phase == 2 ? 2 : 0);
    }
    P2C_PROF_MARK(4)
    // ---- (F) classify: 0 none, 1 collision, 2 separation, 3 undecided ---------
    int leaf = 0;
    double toi = 0.0, margin = 0.0;
    if (active) {
      if (phase == 0) {
        if (d <= eps_space) {
          leaf = 1;
          toi = t0;
        } else {
          phase = 1;
        }
      } else if (phase == 1) {
        d1root = d;
        phase = 2;
      } else {
        if (d <= eps_space) {
          leaf = 1;
          toi = mid;
        } else if (depth == 0 && d1root <= eps_space) {
          leaf = 1;
          toi = t1;
        } else {
          const double lb = sub(d, fam == 1 ? motion_radius<1>(nrm, t0, t1, ops) : motion_radius<2>(nrm, t0, t1, ops));
          if (kCount) ops.add(1);
          if (lb > eps_space) {
            leaf = 2;
            margin = max_std(0.0, sub(lb, eps_space));
            if (kCount) ops.add(1);
          } else if (depth >= max_depth || sub(t1, t0) <= eps_time) {
            leaf = 3;
          } else {
            depth += 1;  // descend into the left child (its path bit stays 0)
            t1 = mid;
          }
        }
      }
    }
    P2C_PROF_MARK(5)
    // ---- (G) record leaves ------------------------------------------------------
    bool root_collision = false;
    if (leaf != 0) {
      if (leaf == 1 && depth == 0) {
        root_collision = true;  // the root is the only node: finish below
      } else {
        const int gi = sa.gidx[slot];
        if (leaf == 1) {
          const unsigned long long key = leaf_key(path, depth);
          atomicMin(&ws.coll_key[slot], key);
          if (gi >= 0) atomicMin(&pools.aggs[gi].coll_key, key);
        } else if (leaf == 2) {
          if (gi >= 0) atomicMin(&pools.aggs[gi].margin_bits, (unsigned long long)__double_as_longlong(margin));
          else atomicMin((unsigned long long*)&sa.margin[slot], (unsigned long long)__double_as_longlong(margin));
        } else {
          if (gi >= 0) atomicOr(&pools.aggs[gi].undecided, 1u);
          else sa.undecided[slot] = 1;
        }
      }
    }
    __syncwarp();
    P2C_PROF_MARK(6)
    // ---- (H) after a leaf, move to the deepest pending right sibling ---------
    if (leaf != 0 && !root_collision) {
      const unsigned long long pend = pending_levels(path, donated, depth, sub_depth);
      if (pend == 0ull) {
        done_lane = true;
      } else {
        const int b = __ffsll((long long)pend) - 1;
        const int l = 64 - b;
        path = (path & top_bits(l - 1)) | (1ull << b);
        donated &= top_bits(l - 1);
        double a, bb;
        replay(T0, T1, path, l - 1, a, bb);
        t0 = mul(0.5, add(a, bb));
        t1 = bb;
        depth = l;
        phase = 2;
      }
    }
    P2C_PROF_MARK(7)
    // ---- (I) export pending subtrees to hungry warps ---------------------------
    if (kExport) {
      if ((iter & (P2C_HUNGRY_PERIOD - 1u)) == 0u) {
        if (lane == 0) {
          pool_hungry = (unsigned long long)volatile_load(&es->hungry.v);
          const unsigned long long rsv = volatile_load(&es->task_reserve.v), hd = volatile_load(&es->task_head.v);
          pool_size = rsv > hd ? rsv - hd : 0ull;
          pool_size = rsv >= pools.task_cap ? ~0ull : pool_size;  // pool full: stop exporting
        }
        pool_hungry = __shfl_sync(FULL, pool_hungry, 0);
        pool_size = __shfl_sync(FULL, pool_size, 0);
      }
      // a warp whose lanes are all busy (nothing left to donate inside it)
      // gives work away: up to P2C_EXPORT_LANES subtrees per iteration, the
      // shallowest ones
      if ((!P2C_EXPORT_FULL || busy == FULL) && pool_hungry > 0ull && pool_size < pool_hungry * 4ull) {
        const unsigned long long pend =
            (slot >= 0 && !done_lane && phase == 2) ? pending_levels(path, donated, depth, sub_depth) : 0ull;
        const int lvl = pend != 0ull ? __clzll((long long)pend) : 64;  // 64 - shallowest level's bit
        const int best = __reduce_min_sync(FULL, (unsigned)lvl);
        const unsigned exporters = __ballot_sync(FULL, pend != 0ull && lvl <= best + P2C_EXPORT_SLACK);
        const bool me = ((exporters >> lane) & 1u) != 0u && __popc(exporters & lt_mask) < P2C_EXPORT_LANES;
        if (me) {
          int gi = sa.gidx[slot];
          // a tree's first export moves its reduction from the slot to a pooled
          // record; one lane of the warp claims the move (others skip this iteration)
          if (gi == -1 && atomicCAS(&sa.gidx[slot], -1, -2) == -1) {
            const unsigned long long idx = atomicAdd(&es->agg_next.v, 1ull);
            if (idx < pools.agg_cap) {
              TreeAgg& A = pools.aggs[idx];
              A.coll_key = ws.coll_key[slot];
              A.margin_bits = (unsigned long long)__double_as_longlong(sa.margin[slot]);
              A.undecided = (unsigned)sa.undecided[slot];
              A.outstanding = (unsigned)sa.outstanding[slot];
              __threadfence();
              atomicExch(&sa.gidx[slot], (int)idx);
              gi = (int)idx;
            } else {
              atomicExch(&sa.gidx[slot], -1);  // pool exhausted: the tree stays in the warp
            }
          }
          if (gi >= 0) {
            const int b = 63 - __clzll((long long)pend);
            const int l = 64 - b;
            const unsigned long long task = atomicAdd(&es->task_reserve.v, 1ull);
            if (task < pools.task_cap) {  // claims never pass task_cap, so no one waits past it
              donated |= (1ull << b);
              atomicAdd(&pools.aggs[gi].outstanding, 1u);
              SubtreeTask* tk = pools.tasks + task;
              tk->path = (path & top_bits(l - 1)) | (1ull << b);
              const unsigned long long q = (unsigned long long)ws.qidx[slot];
              const unsigned long long tag = ((q << 24) | ((unsigned long long)gi << 8) |
                                              ((unsigned long long)l << 1) | (unsigned long long)(fam - 1)) + 1ull;
              if (P2C_ACQ_REL) {
                store_release(&tk->tag, tag);
              } else {
                __threadfence();
                atomicExch(&tk->tag, tag);
              }
              st.donations += 1;
            }
          }
        }
        __syncwarp();
      }
    }
    P2C_PROF_MARK(8)
    // ---- (J) a finished lane leaves its tree; the last unit finalises it ------
    unsigned freed = 0u;
    if (root_collision) {
      Outcome o{P2C_STATUS_COLLISION, T0, T1, toi, 0.0};
      finalize(fam, ws.qidx[slot], o);
      freed = 1u << slot;
      slot = -1;
    } else if (done_lane) {
      const int s = slot;
      const long long q = ws.qidx[s];
      const int f = fam;
      const int gi = sa.gidx[s];
      const bool last_here = atomicSub(&sa.outstanding[s], 1) == 1;
      if (gi >= 0) {
        bool last = false;
        if (P2C_ACQ_REL) {
          last = decrement_acq_rel(&pools.aggs[gi].outstanding) == 1u;
        } else {
          __threadfence();
          last = atomicSub(&pools.aggs[gi].outstanding, 1u) == 1u;
          if (last) __threadfence();
        }
        if (last) {
          const TreeAgg& A = pools.aggs[gi];
          const Outcome o = outcome_from(volatile_load(&A.coll_key), volatile_load(&A.margin_bits),
                                         volatile_load(&A.undecided) != 0u, T0, T1);
          finalize(f, q, o);
        }
      } else if (last_here) {
        const unsigned long long mb = (unsigned long long)__double_as_longlong(sa.margin[s]);
        const Outcome o = outcome_from(ws.coll_key[s], mb, sa.undecided[s] != 0, T0, T1);
        finalize(f, q, o);
      }
      if (last_here) freed = 1u << s;
      slot = -1;
    }
    free_mask |= __reduce_or_sync(FULL, freed);
    __syncwarp();
    P2C_PROF_MARK(9)
  }
  P2C_PROF_FLUSH()
  if (kExport && hungry && lane == 0) atomicAdd(&es->hungry.v, ~0ull);
  if (kCount) st.ops += ops.n;
  return ok;
}

}  // namespace p2c
