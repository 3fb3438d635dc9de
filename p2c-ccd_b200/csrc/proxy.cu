// proxy.cu — candidates of a proxy scene (patch proxies in time slabs) on the
// device: GenerateRawCandidatesCpu + CompactRawCandidates
// (rt_candidate/candidate_buffer.cpp:144-227).
//
// The reference tests every proxy pair (O(n^2)).  Here:
//   1. one radix sort orders the proxies by (slab, column of the min corner
//      over the two narrower axes, quantised min along the widest axis), and
//      they are gathered into that order as struct-of-arrays;
//   2. a column-subdivided sweep: each proxy scans the columns and the
//      sweep-axis window its partners' min corners can lie in, and emits the
//      pairs of different objects whose time intervals and inclusive AABBs
//      overlap, as (lo << 32 | hi) keys, each pair once;
//   3. one radix sort of the keys gives the reference's (i, j) hit order and
//      the 64-byte RawCandidateHit records are written from the keys;
//   4. dense ranks of the slab ids and of the (object, patch) pairs keep the
//      order of the reference's compaction key (slab, first object, first
//      patch, second object, second patch, first type, second type), so two
//      stable radix sorts of exact bit widths order the hits by it; the
//      head of every run writes one CandidateRecord (ids 1, 2, ... in key
//      order) with the run's hit count, the float maximum of its motion
//      bounds and its flags.
#include <cooperative_groups.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>

#include "broadphase.cuh"
#include "p2c_internal.cuh"

namespace p2c {
namespace {

namespace cg = cooperative_groups;

static_assert(sizeof(p2c_raw_candidate_hit) == 64, "RawCandidateHit layout");
static_assert(sizeof(p2c_candidate_record) == 80, "CandidateRecord layout");

constexpr int kThreads = 256;
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kHitFlags = 3u;  // kRawCandidateValid | kRawCandidateAabbOverlap
constexpr unsigned long long kErrHitCountOverflow = 16ull;  // a candidate's summed rt_hit_count exceeds 32 bits

unsigned grid_for(long long n) {
  const long long b = (n + kThreads - 1) / kThreads;
  return (unsigned)(b > 0 ? b : 1);
}

int bit_length(unsigned long long x) {
  int b = 0;
  while (x) {
    ++b;
    x >>= 1;
  }
  return b;
}

struct ProxyStats {
  unsigned long long lo_min[3], lo_max[3];  // order keys of the smallest / largest min corner per axis
  unsigned long long ext_max[3];            // bit patterns of the largest extent per axis (>= 0)
  double ext_sum[3];                        // sum of extents per axis (grid heuristic only)
};

// Columns over the two non-sweep axes (each box stored in the column of its
// min corner) and a 16-bit quantiser of the sweep-axis min.
struct ProxyGrid {
  int axis, a1, a2, g1, g2;
  double base0, scale0, base1, inv1, base2, inv2, reach1, reach2;
};

struct ProxyLayout {
  unsigned long long* counter;   // [0] raw hits, [1] error word, [2] first invalid given hit (hit << 4 | check)
  ProxyStats* stats;
  ProxyGrid* grid;
  unsigned long long* key[2];    // n: (slab << 30 | column << 16 | q), sorted copy
  unsigned* order[2];            // n: proxy index, sorted copy
  double* s_box;                 // 6 x n, sorted order, struct of arrays: lo, hi, alo, ahi, blo, bhi
  double* s_t0;                  // n
  double* s_t1;
  unsigned* s_obj;
  float4* s_f;                   // n: column-axis bounds rounded outward (a float prefilter)
  unsigned long long* okey[2];   // n: (object << 32 | patch), sorted copy
  unsigned* oidx;                // n: proxy index in (object, patch) order
  unsigned* flag;                // n: run heads of a sorted key
  unsigned* scan;                // n: their inclusive sum
  unsigned* rank_op;             // n: dense rank of the proxy's (object, patch)
  unsigned* rank_slab;           // n: dense rank of the proxy's slab
  // direct (slab, column) table, when the slab ids are known to be narrow:
  // per run {first entry, one past the last, float keys of the largest max
  // corner along the two column axes}
  int table_bits;                // slab id bits of the table (0: no table, binary search)
  uint4* cells;                  // [2^(table_bits + 14)]
  size_t table_bytes;
  unsigned long long* pairs[2];  // raw_cap
  unsigned long long* ck[2];     // raw_cap: compaction key chunks
  unsigned* perm[2];             // raw_cap
  unsigned long long* gk[2];     // raw_cap: gathered key chunk and its sorted copy
  unsigned* head;                // raw_cap + 1
  unsigned* seg;                 // raw_cap + 1
  void* tmp;
  size_t tmp_bytes;
  size_t total;
};

size_t temp_bytes(long long n, long long cap) {
  const int nn = (int)std::max(n, 1ll), cc = (int)std::max(cap, 1ll);
  size_t a = 0, c = 0, d = 0, e = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, a, (const unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                  (const unsigned*)nullptr, (unsigned*)nullptr, std::max(nn, cc));
  cub::DeviceRadixSort::SortKeys(nullptr, c, (const unsigned long long*)nullptr, (unsigned long long*)nullptr, cc);
  cub::DeviceScan::ExclusiveSum(nullptr, d, (const unsigned*)nullptr, (unsigned*)nullptr, cc + 1);
  cub::DeviceScan::InclusiveSum(nullptr, e, (const unsigned*)nullptr, (unsigned*)nullptr, nn);
  return std::max(std::max(a, e), std::max(c, d));
}

// The direct (slab, column) table is used for slab ids of at most this many
// bits (2^(6 + 14) runs of 16 bytes, 16 MB).
constexpr int kTableSlabBits = 6;

int table_bits_for(uint32_t slab_bits) {
  return slab_bits > 0 && slab_bits <= (uint32_t)kTableSlabBits ? (int)slab_bits : 0;
}

ProxyLayout carve(void* base, long long n, long long cap, int table_bits) {
  ProxyLayout L{};
  size_t off = 0;
  char* b = static_cast<char*>(base);
  auto take = [&](size_t bytes) -> void* {
    void* p = b == nullptr ? nullptr : b + off;
    off += (std::max<size_t>(bytes, 1) + 255) & ~size_t(255);
    return p;
  };
  const size_t N = (size_t)std::max(n, 1ll), C = (size_t)std::max(cap, 1ll);
  L.counter = static_cast<unsigned long long*>(take(24));
  L.stats = static_cast<ProxyStats*>(take(sizeof(ProxyStats)));
  L.grid = static_cast<ProxyGrid*>(take(sizeof(ProxyGrid)));
  for (int k = 0; k < 2; ++k) {
    L.key[k] = static_cast<unsigned long long*>(take(8 * N));
    L.order[k] = static_cast<unsigned*>(take(4 * N));
    L.pairs[k] = static_cast<unsigned long long*>(take(8 * C));
    L.ck[k] = static_cast<unsigned long long*>(take(8 * C));
    L.perm[k] = static_cast<unsigned*>(take(4 * C));
    L.gk[k] = static_cast<unsigned long long*>(take(8 * C));
  }
  L.s_box = static_cast<double*>(take(6 * 8 * N));
  L.s_t0 = static_cast<double*>(take(8 * N));
  L.s_t1 = static_cast<double*>(take(8 * N));
  L.s_obj = static_cast<unsigned*>(take(4 * N));
  for (int k = 0; k < 2; ++k) L.okey[k] = static_cast<unsigned long long*>(take(8 * N));
  L.oidx = static_cast<unsigned*>(take(4 * N));
  L.flag = static_cast<unsigned*>(take(4 * N));
  L.scan = static_cast<unsigned*>(take(4 * N));
  L.rank_op = static_cast<unsigned*>(take(4 * N));
  L.rank_slab = static_cast<unsigned*>(take(4 * N));
  L.s_f = static_cast<float4*>(take(sizeof(float4) * N));
  L.table_bits = table_bits;
  const size_t T = table_bits > 0 ? (size_t)1 << (table_bits + kCellBits) : 0;
  L.table_bytes = sizeof(uint4) * T;
  L.cells = static_cast<uint4*>(take(L.table_bytes));
  L.head = static_cast<unsigned*>(take(4 * (C + 1)));
  L.seg = static_cast<unsigned*>(take(4 * (C + 1)));
  L.tmp_bytes = temp_bytes(n, cap);
  L.tmp = take(L.tmp_bytes);
  L.total = off;
  return L;
}

__global__ void stats_init_kernel(ProxyLayout L) {
  if (threadIdx.x != 0) return;
  ProxyStats& S = *L.stats;
  for (int a = 0; a < 3; ++a) {
    S.lo_min[a] = ~0ull;
    S.lo_max[a] = 0ull;
    S.ext_max[a] = 0ull;
    S.ext_sum[a] = 0.0;
  }
}

// ValidateProxyScene's per-proxy checks (rt_candidate/proxy_scene.cpp:143-151:
// concrete type, finite t0 < t1, finite bounds with min <= max) and the
// statistics of the grid.  Proxy ids (the array index here) and the global
// slab partition (:58-85) are checked by the host, which holds one interval
// per slab.
__global__ void keys_kernel(p2c_proxy_scene sc, ProxyLayout L) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < sc.n;
  double lo[3] = {0, 0, 0}, ext[3] = {0, 0, 0};
  bool ok = true;
  if (live) {
    const double* b = sc.bounds + 6 * i;
    ok = (sc.proxy_type[i] == 1 || sc.proxy_type[i] == 2) && isfinite(sc.t0[i]) && isfinite(sc.t1[i]) &&
         sc.t0[i] < sc.t1[i];
    for (int a = 0; a < 3; ++a) {
      ok = ok && isfinite(b[a]) && isfinite(b[3 + a]) && !(b[a] > b[3 + a]);
      lo[a] = b[a];
      ext[a] = b[3 + a] - b[a];
    }
    if (!ok) atomicOr(L.counter + 1, 1ull);
    if ((sc.slab_bits && sc.slab_bits < 32 && (sc.slab_id[i] >> sc.slab_bits)) ||
        (sc.object_bits && sc.object_bits < 32 && (sc.object_id[i] >> sc.object_bits)) ||
        (sc.patch_bits && sc.patch_bits < 32 && (sc.patch_id[i] >> sc.patch_bits)))
      atomicOr(L.counter + 1, 8ull);
  }
  // block-reduced statistics of the valid boxes (an invalid scene fails as a whole)
  const bool use = live && ok;
  __shared__ unsigned long long s_kmin[kThreads / 32][3], s_kmax[kThreads / 32][3], s_emax[kThreads / 32][3];
  __shared__ double s_esum[kThreads / 32][3];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    unsigned long long kmin = use ? order_key(lo[a]) : ~0ull, kmax = use ? order_key(lo[a]) : 0ull;
    unsigned long long emax = use ? (unsigned long long)__double_as_longlong(ext[a]) : 0ull;
    double esum = use ? ext[a] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      kmin = min(kmin, __shfl_xor_sync(kFull, kmin, o));
      kmax = max(kmax, __shfl_xor_sync(kFull, kmax, o));
      emax = max(emax, __shfl_xor_sync(kFull, emax, o));
      esum += __shfl_xor_sync(kFull, esum, o);
    }
    if (lane == 0) {
      s_kmin[warp][a] = kmin;
      s_kmax[warp][a] = kmax;
      s_emax[warp][a] = emax;
      s_esum[warp][a] = esum;
    }
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int a = threadIdx.x;
    unsigned long long kmin = ~0ull, kmax = 0ull, emax = 0ull;
    double esum = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) {
      kmin = min(kmin, s_kmin[w][a]);
      kmax = max(kmax, s_kmax[w][a]);
      emax = max(emax, s_emax[w][a]);
      esum += s_esum[w][a];
    }
    ProxyStats& S = *L.stats;
    if (kmin != ~0ull) atomicMin(&S.lo_min[a], kmin);
    if (kmax != 0ull) atomicMax(&S.lo_max[a], kmax);
    if (emax != 0ull) atomicMax(&S.ext_max[a], emax);
    if (esum != 0.0) atomicAdd(&S.ext_sum[a], esum);
  }
}

// Clamp to [0, hi], NaN to 0.
__device__ __forceinline__ int clamp_index(double c, int hi) {
  return !(c >= 0.0) ? 0 : (c >= (double)hi ? hi : (int)c);
}

// Sweep axis = the widest spread of min corners; columns over the other two
// axes one (direct table: a column costs one 16-byte load) or two (binary
// search) mean extents wide, at most kMaxColumns each.
__global__ void grid_kernel(ProxyLayout L, long long n) {
  const double width_mult = L.table_bits > 0 ? 1.0 : 2.0;
  if (threadIdx.x != 0) return;
  const ProxyStats& S = *L.stats;
  double base[3], range[3], mean[3], reach[3];
  for (int a = 0; a < 3; ++a) {
    const bool any = S.lo_min[a] != ~0ull;
    base[a] = any ? unorder_key(S.lo_min[a]) : 0.0;
    range[a] = any ? unorder_key(S.lo_max[a]) - base[a] : 0.0;
    if (!(range[a] >= 0.0) || !isfinite(range[a])) range[a] = 0.0;
    mean[a] = n > 0 ? S.ext_sum[a] / (double)n : 0.0;
    reach[a] = __longlong_as_double((long long)S.ext_max[a]);
    if (!isfinite(reach[a])) reach[a] = 0.0;
  }
  ProxyGrid g{};
  g.axis = 0;
  for (int a = 1; a < 3; ++a)
    if (range[a] > range[g.axis]) g.axis = a;
  g.a1 = g.axis == 0 ? 1 : 0;
  g.a2 = g.axis == 2 ? 1 : 2;
  const int ax[2] = {g.a1, g.a2};
  int gg[2];
  double inv[2];
  for (int k = 0; k < 2; ++k) {
    const int a = ax[k];
    const double w = fmax(width_mult * mean[a], range[a] / kMaxColumns);
    gg[k] = w > 0.0 ? clamp_index(floor(range[a] / w), kMaxColumns) : 1;
    if (gg[k] < 1) gg[k] = 1;
    inv[k] = range[a] > 0.0 ? (double)gg[k] / range[a] : 0.0;
  }
  g.g1 = gg[0];
  g.g2 = gg[1];
  g.base1 = base[g.a1];
  g.inv1 = inv[0];
  g.base2 = base[g.a2];
  g.inv2 = inv[1];
  g.reach1 = reach[g.a1];
  g.reach2 = reach[g.a2];
  g.base0 = base[g.axis];
  g.scale0 = range[g.axis] > 0.0 ? 65535.0 / range[g.axis] : 0.0;
  *L.grid = g;
}

__device__ __forceinline__ int proxy_column(double x, double base, double inv, int g) {
  return clamp_index(floor((x - base) * inv), g - 1);
}

// Monotone (non-decreasing) in x.
__device__ __forceinline__ unsigned proxy_quantise(double x, const ProxyGrid& g) {
  return (unsigned)clamp_index(floor((x - g.base0) * g.scale0), 65535);
}

__global__ void cell_keys_kernel(p2c_proxy_scene sc, ProxyLayout L) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sc.n) return;
  const ProxyGrid g = *L.grid;
  const double* b = sc.bounds + 6 * i;
  const int c1 = proxy_column(b[g.a1], g.base1, g.inv1, g.g1);
  const int c2 = proxy_column(b[g.a2], g.base2, g.inv2, g.g2);
  const unsigned q = proxy_quantise(b[g.axis], g);
  L.key[0][i] = ((unsigned long long)sc.slab_id[i] << 30) | ((unsigned long long)(c1 * g.g2 + c2) << 16) | q;
  L.order[0][i] = (unsigned)i;
}

// Proxies in (slab, column, q) order as struct-of-arrays.
__global__ void gather_kernel(p2c_proxy_scene sc, ProxyLayout L) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= sc.n) return;
  const ProxyGrid g = *L.grid;
  const long long n = sc.n;
  const unsigned i = L.order[1][p];
  const double* b = sc.bounds + 6 * (long long)i;
  L.s_box[p] = b[g.axis];
  L.s_box[n + p] = b[3 + g.axis];
  L.s_box[2 * n + p] = b[g.a1];
  L.s_box[3 * n + p] = b[3 + g.a1];
  L.s_box[4 * n + p] = b[g.a2];
  L.s_box[5 * n + p] = b[3 + g.a2];
  L.s_t0[p] = sc.t0[i];
  L.s_t1[p] = sc.t1[i];
  L.s_obj[p] = sc.object_id[i];
  L.s_f[p] = make_float4(__double2float_rd(b[g.a1]), __double2float_ru(b[3 + g.a1]), __double2float_rd(b[g.a2]),
                         __double2float_ru(b[3 + g.a2]));
}

// Begin / end of every (slab, column) run of the sorted keys and the float
// keys (rounded up) of the largest max corner of its boxes on the two column
// axes.
__global__ void table_kernel(ProxyLayout L, long long n) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const unsigned long long* K = L.key[1];
  const unsigned long long run = K[p] >> 16;  // slab << 14 | column
  if ((K[p] >> 30) >> L.table_bits) return;   // a slab id past its width hint (error word bit 8)
  uint4* c = L.cells + run;
  if (p == 0 || (K[p - 1] >> 16) != run) c->x = (unsigned)p;
  if (p == n - 1 || (K[p + 1] >> 16) != run) c->y = (unsigned)(p + 1);
  atomicMax(&c->z, fkey_up(L.s_box[3 * n + p]));
  atomicMax(&c->w, fkey_up(L.s_box[5 * n + p]));
}

__global__ void fill_kernel(unsigned long long* p, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = ~0ull;
}

// First position in [0, n) whose key is >= k.
__device__ __forceinline__ long long lower_bound(const unsigned long long* __restrict__ keys, long long n,
                                                 unsigned long long k) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long m = (lo + hi) >> 1;
    if (keys[m] < k) lo = m + 1;
    else hi = m;
  }
  return lo;
}

// Column-subdivided sweep over the sorted proxies.  A box is stored in the
// column of its min corner, so a partner overlapping box p on the two
// column axes has its min corner in columns [col(min - reach), col(max)];
// in each, the partners whose sweep-axis min lies in [p.min, p.max] are the
// key window [q(p.min), q(p.max)] of p's slab.  A pair is emitted by the box
// with the smaller (sweep min, index), so exactly once.  The tests are
// GenerateRawCandidatesCpu's (candidate_buffer.cpp:158-173: different
// objects, same slab, TimeOverlap, inclusive AabbOverlap).
//
// kSweepLanes lanes share one box and take its columns in turn: the work of
// a box is a chain of dependent loads (a column lookup, a search for the
// window's start, then the window's walk), and splitting it shortens the
// chain and fills the SMs.  With narrow slab ids a direct (slab, column)
// table gives each column's run and lets columns whose boxes cannot reach
// the scanning box be skipped; otherwise a binary search over all keys
// finds each window.
constexpr int kSweepLanes = 8;

// 6 blocks of 256 threads per SM (40 registers, a few spilled values): more
// warps to hide the walk's load latency than the 4 blocks the unbounded
// 54-register build allows (1.64 M proxies: 7.6 -> 7.1 ms per step).
__global__ void __launch_bounds__(kThreads, 6) sweep_kernel(ProxyLayout L, long long n, unsigned long long cap,
                                                         int rank_bits) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long p = t / kSweepLanes;
  const int lane = (int)(t % kSweepLanes);
  if (p >= n) return;
  const ProxyGrid g = *L.grid;
  const double* __restrict__ B = L.s_box;
  const unsigned long long* __restrict__ K = L.key[1];
  const double lo = B[p], hi = B[n + p], alo = B[2 * n + p], ahi = B[3 * n + p], blo = B[4 * n + p],
               bhi = B[5 * n + p];
  const unsigned obj = L.s_obj[p], id = L.order[1][p];
  const double t0 = L.s_t0[p], t1 = L.s_t1[p];
  const unsigned long long slab = K[p] >> 30;
  // widen the lower columns by a relative 2^-40 so that the rounding of
  // min - reach never skips the column of a partner's min corner
  const int c1a = proxy_column(alo - g.reach1 - (fabs(alo) + g.reach1) * 0x1p-40, g.base1, g.inv1, g.g1);
  const int c1b = proxy_column(ahi, g.base1, g.inv1, g.g1);
  const int c2a = proxy_column(blo - g.reach2 - (fabs(blo) + g.reach2) * 0x1p-40, g.base2, g.inv2, g.g2);
  const int c2b = proxy_column(bhi, g.base2, g.inv2, g.g2);
  const int n2 = c2b - c2a + 1, n_cells = (c1b - c1a + 1) * n2;
  const unsigned q_lo = proxy_quantise(lo, g), q_hi = proxy_quantise(hi, g);
  // column-axis bounds rounded outward: a pair that overlaps in doubles
  // overlaps in these floats, so they reject most entries with one load
  const float f_alo = __double2float_rd(alo), f_ahi = __double2float_ru(ahi), f_blo = __double2float_rd(blo),
              f_bhi = __double2float_ru(bhi);
  // one partner entry j: prefilter, ownership, exact overlap, object and time tests, then append
  auto visit = [&](long long j) {
    const float4 f = L.s_f[j];
    if (f.y < f_alo || f_ahi < f.x || f.w < f_blo || f_bhi < f.z) return;
    const double lj = B[j];
    const unsigned idj = L.order[1][j];
    if (lj < lo || (lj == lo && idj <= id) || lj > hi) return;  // owned by the other box / no overlap
    if (B[3 * n + j] < alo || ahi < B[2 * n + j] || B[5 * n + j] < blo || bhi < B[4 * n + j]) return;
    if (L.s_obj[j] == obj || !(t0 < L.s_t1[j] && L.s_t0[j] < t1)) return;
    const cg::coalesced_group grp = cg::coalesced_threads();
    unsigned long long base = 0;
    if (grp.thread_rank() == 0) base = atomicAdd(L.counter, (unsigned long long)grp.size());
    base = grp.shfl(base, 0);
    const unsigned long long slot = base + grp.thread_rank();
    if (slot < cap)
      L.pairs[0][slot] = ((unsigned long long)min(id, idj) << rank_bits) | (unsigned long long)max(id, idj);
  };
  if (L.table_bits > 0) {
    if (slab >> L.table_bits) return;  // past the slab width hint (error word bit 8)
    const unsigned k_alo = fkey_down(alo), k_blo = fkey_down(blo);
    for (int k = lane; k < n_cells; k += kSweepLanes) {
      const int c1 = c1a + k / n2, c2 = c2a + k % n2;
      const uint4 c = L.cells[(slab << kCellBits) | (unsigned long long)(c1 * g.g2 + c2)];
      // empty, or no box of this column reaches the scanning box on a column axis
      if (c.x >= c.y || c.z < k_alo || c.w < k_blo) continue;
      unsigned b = c.x, r = c.y;
      while (b < r) {  // first entry of the column with q >= q_lo
        const unsigned m = (b + r) >> 1;
        if ((unsigned)(K[m] & 0xffffull) < q_lo) b = m + 1;
        else r = m;
      }
      for (unsigned j = b; j < c.y && (unsigned)(K[j] & 0xffffull) <= q_hi; ++j) visit(j);
    }
    return;
  }
  for (int k = lane; k < n_cells; k += kSweepLanes) {
    const int c1 = c1a + k / n2, c2 = c2a + k % n2;
    const unsigned long long cell = (slab << 30) | ((unsigned long long)(c1 * g.g2 + c2) << 16);
    const unsigned long long k_end = cell | q_hi;
    for (long long j = lower_bound(K, n, cell | q_lo); j < n && K[j] <= k_end; ++j) visit(j);
  }
}

// Dense ranks that preserve the compaction key's order
// (MakeCandidateKey, candidate_buffer.cpp:104-124, compared field by field):
// the slab id's rank among the scene's slabs and the (object, patch) pair's
// rank among the scene's pairs.  Equal ranks <=> equal fields, so the key
// (slab, first (object, patch), second (object, patch), types) sorts as
// (slab rank, first rank, second rank, types) in few radix passes.
__global__ void slab_flags_kernel(ProxyLayout L, long long n) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) L.flag[p] = (p == 0 || (L.key[1][p] >> 30) != (L.key[1][p - 1] >> 30)) ? 1u : 0u;
}

__global__ void slab_rank_kernel(ProxyLayout L, long long n) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) L.rank_slab[L.order[1][p]] = L.scan[p] - 1u;
}

__global__ void op_keys_kernel(p2c_proxy_scene sc, ProxyLayout L, int patch_bits) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sc.n) return;
  L.okey[0][i] = ((unsigned long long)sc.object_id[i] << patch_bits) | sc.patch_id[i];
  L.order[0][i] = (unsigned)i;
}

__global__ void op_flags_kernel(ProxyLayout L, long long n) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) L.flag[p] = (p == 0 || L.okey[1][p] != L.okey[1][p - 1]) ? 1u : 0u;
}

__global__ void op_rank_kernel(ProxyLayout L, long long n) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) L.rank_op[L.oidx[p]] = L.scan[p] - 1u;
}

// The first / second proxy of a hit: the smaller (object, patch, proxy id)
// tuple first (MakeCandidateKey).
__device__ __forceinline__ bool hit_swapped(const p2c_proxy_scene& sc, unsigned i, unsigned j) {
  const unsigned fo = sc.object_id[i], so = sc.object_id[j], fp = sc.patch_id[i], sp = sc.patch_id[j];
  return fo > so || (fo == so && (fp > sp || (fp == sp && i > j)));
}

// static_cast<float>(std::max(lhs, rhs)) with IEEE round to nearest: a double
// beyond the float range becomes infinity.  The intrinsic keeps that defined
// (a plain cast of an out-of-range value is undefined behaviour in C++, which
// lets the optimiser assume the float stays finite).
__device__ __forceinline__ float merged_bound(const double* a, const double* b, int k) {
  return __double2float_rn(a[k] < b[k] ? b[k] : a[k]);
}

// finite and not below zero (ValidateRawHit), on the bits of the float
__device__ __forceinline__ bool bound_valid(float v) {
  return (__float_as_uint(v) & 0x7f800000u) != 0x7f800000u && !(v < 0.0f);
}

// Raw hit records in (i, j) order, and the compaction key of each hit from
// the dense ranks (slab rank D, first and second (object, patch) ranks, the
// two proxy types 1 / 2 as one bit each): one key (D, first, second, types)
// when it fits 64 bits, else two chunks (second, types) and (D, first).
struct CompactionKey {
  int rank_bits;  // bits of a proxy index and of an (object, patch) rank
  int d_bits;     // bits of a slab rank
  bool single;    // the whole key fits one 64-bit chunk
};

__global__ void raw_hits_kernel(p2c_proxy_scene sc, ProxyLayout L, const unsigned long long* sorted,
                                unsigned long long cap, CompactionKey ck, p2c_raw_candidate_hit* raw) {
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= (long long)cap) return;
  const unsigned long long k = sorted[h];
  L.perm[0][h] = (unsigned)h;
  if (k == ~0ull) {  // past the hits: sorts last in every pass
    L.ck[0][h] = ~0ull;
    L.ck[1][h] = ~0ull;
    return;
  }
  const unsigned i = (unsigned)(k >> ck.rank_bits), j = (unsigned)(k & ((1ull << ck.rank_bits) - 1ull));
  const double* ma = sc.motion_bound + 4 * (long long)i;
  const double* mb = sc.motion_bound + 4 * (long long)j;
  p2c_raw_candidate_hit r{};
  r.query_id = sc.query_id;
  r.pair_key = ((unsigned long long)i << 32) | j;  // PairKey
  r.proxy_a_index = i;
  r.proxy_b_index = j;
  r.slab_id = sc.slab_id[i];
  r.rt_hit_count = 1u;
  r.flags = kHitFlags;
  bool bound_ok = true;
  for (int c = 0; c < 4; ++c) {
    r.motion_bound[c] = merged_bound(ma, mb, c);
    bound_ok = bound_ok && bound_valid(r.motion_bound[c]);
  }
  // ValidateRawHit (:95-99), which CompactRawCandidates applies to every hit
  if (!bound_ok) atomicOr(L.counter + 1, 2ull);
  raw[h] = r;
  const bool sw = hit_swapped(sc, i, j);
  const unsigned f = sw ? j : i, t = sw ? i : j;
  const unsigned long long types = ((unsigned long long)((sc.proxy_type[f] - 1u) & 1u) << 1) |
                                   ((sc.proxy_type[t] - 1u) & 1u);
  const unsigned long long lo = ((unsigned long long)L.rank_op[t] << 2) | types;  // rank_bits + 2 bits
  const unsigned long long hi = ((unsigned long long)L.rank_slab[i] << ck.rank_bits) | L.rank_op[f];
  if (ck.single) {
    L.ck[0][h] = (hi << (ck.rank_bits + 2)) | lo;
  } else {
    L.ck[0][h] = lo;
    L.ck[1][h] = hi;
  }
}

__global__ void gather_chunk_kernel(const unsigned long long* chunk, const unsigned* perm, unsigned long long* out,
                                    long long cap) {
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (h < cap) out[h] = chunk[perm[h]];
}

// Run heads of the compaction key over the hits in key order.
__global__ void heads_kernel(ProxyLayout L, const unsigned* perm, const unsigned long long* k0,
                             const unsigned long long* k1, long long cap) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p > cap) return;
  const long long n_hits = (long long)min(L.counter[0], (unsigned long long)cap);
  unsigned hd = 0u;
  if (p < n_hits && p < cap) {
    const unsigned a = perm[p];
    hd = p == 0 ? 1u : 0u;
    if (p > 0) {
      const unsigned b = perm[p - 1];
      hd = (k0[a] != k0[b] || k1[a] != k1[b]) ? 1u : 0u;
    }
  }
  L.head[p] = hd;
}

// Given raw hits: ValidateRawHit (candidate_buffer.cpp:71-101) on each, the
// first failing hit's first failing check kept as (hit << 4 | check) in
// counter[2]; then the compaction key chunks as raw_hits_kernel forms them,
// from the hit's own proxy indices.
__global__ void external_hits_kernel(p2c_proxy_scene sc, ProxyLayout L, const p2c_raw_candidate_hit* raw,
                                     long long n_raw, CompactionKey ck) {
  const long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= n_raw) return;
  L.perm[0][h] = (unsigned)h;
  const p2c_raw_candidate_hit r = raw[h];
  const unsigned long long n = (unsigned long long)sc.n;
  unsigned check = 0u;
  if ((r.flags & 1u) == 0u) check = 1;
  else if (r.query_id == 0ull) check = 2;
  else if (r.query_id != sc.query_id) check = 3;
  else if (r.proxy_a_index >= n || r.proxy_b_index >= n) check = 4;
  else if (r.proxy_a_index == r.proxy_b_index) check = 5;
  else {
    const unsigned a = r.proxy_a_index, b = r.proxy_b_index;
    const unsigned long long pk = ((unsigned long long)(a < b ? a : b) << 32) | (a < b ? b : a);
    bool bound_ok = true;
    for (int c = 0; c < 4; ++c) bound_ok = bound_ok && bound_valid(r.motion_bound[c]);
    if (r.pair_key != pk) check = 6;
    else if (sc.object_id[a] == sc.object_id[b]) check = 7;
    else if (sc.slab_id[a] != sc.slab_id[b] || r.slab_id != sc.slab_id[a]) check = 8;
    else if (!bound_ok) check = 9;
  }
  if (check != 0u) {
    atomicMin(L.counter + 2, ((unsigned long long)h << 4) | check);
    L.ck[0][h] = ~0ull;
    L.ck[1][h] = ~0ull;
    return;
  }
  const unsigned i = r.proxy_a_index, j = r.proxy_b_index;
  const bool sw = hit_swapped(sc, i, j);
  const unsigned f = sw ? j : i, t = sw ? i : j;
  const unsigned long long types = ((unsigned long long)((sc.proxy_type[f] - 1u) & 1u) << 1) |
                                   ((sc.proxy_type[t] - 1u) & 1u);
  const unsigned long long lo = ((unsigned long long)L.rank_op[t] << 2) | types;
  const unsigned long long hi = ((unsigned long long)L.rank_slab[i] << ck.rank_bits) | L.rank_op[f];
  if (ck.single) {
    L.ck[0][h] = (hi << (ck.rank_bits + 2)) | lo;
  } else {
    L.ck[0][h] = lo;
    L.ck[1][h] = hi;
  }
}

// After the records: the error bits they set (a count overflow) and the
// first invalid given hit.
__global__ void first_invalid_kernel(ProxyLayout L, uint64_t* counts) {
  if (threadIdx.x == 0) {
    counts[2] |= L.counter[1];
    counts[3] = L.counter[2];
  }
}

__global__ void set_hits_kernel(ProxyLayout L, long long n_raw) {
  if (threadIdx.x == 0) {
    L.counter[0] = (unsigned long long)n_raw;
    L.counter[2] = ~0ull;
  }
}

__global__ void records_kernel(p2c_proxy_scene sc, ProxyLayout L, const unsigned* perm,
                               const p2c_raw_candidate_hit* raw, long long cap, p2c_candidate_record* out,
                               unsigned long long* counts) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n_hits = (long long)min(L.counter[0], (unsigned long long)cap);
  if (p == 0) {
    counts[0] = L.counter[0];
    counts[1] = n_hits > 0 ? L.seg[n_hits] : 0ull;  // seg is unwritten when the capacity is 0
    counts[2] = L.counter[1] | (L.counter[0] > (unsigned long long)n_hits ? 4ull : 0ull);
  }
  if (p >= n_hits || !L.head[p]) return;
  const unsigned a = perm[p];
  p2c_candidate_record r{};
  r.schema_version = 1u;
  r.candidate_id = (unsigned long long)L.seg[p] + 1ull;
  r.query_id = sc.query_id;
  const unsigned i = raw[a].proxy_a_index, j = raw[a].proxy_b_index;
  if ((long long)i >= sc.n || (long long)j >= sc.n) return;  // an invalid given hit (reported, not compacted)
  const bool sw = hit_swapped(sc, i, j);
  const unsigned f = sw ? j : i, t = sw ? i : j;
  r.slab_id = raw[a].slab_id;
  r.object_a_id = sc.object_id[f];
  r.patch_a_id = sc.patch_id[f];
  r.object_b_id = sc.object_id[t];
  r.patch_b_id = sc.patch_id[t];
  r.proxy_type_a = sc.proxy_type[f];
  r.proxy_type_b = sc.proxy_type[t];
  unsigned long long count = 0ull;
  unsigned flags = 0u;
  float mb[4] = {0.f, 0.f, 0.f, 0.f};
  for (long long q = p; q < n_hits && (q == p || !L.head[q]); ++q) {
    const p2c_raw_candidate_hit& h = raw[perm[q]];
    if (q == p) {
      for (int c = 0; c < 4; ++c) mb[c] = h.motion_bound[c];
    } else {
      for (int c = 0; c < 4; ++c) mb[c] = mb[c] < h.motion_bound[c] ? h.motion_bound[c] : mb[c];  // std::max
    }
    count += h.rt_hit_count;
    flags |= h.flags;
  }
  if (count > 0xffffffffull) atomicOr(L.counter + 1, kErrHitCountOverflow);  // the reference's u32 sum overflows
  r.rt_hit_count = (unsigned)count;
  for (int c = 0; c < 4; ++c) r.motion_bound[c] = mb[c];
  r.proxy_features_offset = 0u;
  r.flags = flags;
  out[r.candidate_id - 1] = r;
}

}  // namespace
}  // namespace p2c

extern "C" {

size_t p2c_proxy_candidates_workspace_bytes(int64_t n_proxies, int64_t raw_cap, uint32_t slab_bits) {
  if (n_proxies < 0 || raw_cap < 0) return 0;
  return p2c::carve(nullptr, n_proxies, raw_cap, p2c::table_bits_for(slab_bits)).total + 256;
}

}  // extern "C"

namespace p2c {
namespace {

struct ProxyRun {
  p2c_proxy_scene sc;
  ProxyLayout L;
  long long n = 0;
  int rank_bits = 1, slab_bits = 32, object_bits = 32, patch_bits = 32;
};

int proxy_checks(const p2c_proxy_scene* scene) {
  if (scene == nullptr) return fail(P2C_ERR_INVALID, "proxy scene pointer is null");
  if (scene->query_id == 0) return fail(P2C_ERR_INVALID, "ProxyScene.query_id is required");
  if (scene->n < 0 || scene->n >= (1ll << 31)) return fail(P2C_ERR_INVALID, "proxy count must lie in [0, 2^31)");
  if (scene->n > 0 && (scene->object_id == nullptr || scene->patch_id == nullptr || scene->slab_id == nullptr ||
                       scene->proxy_type == nullptr || scene->t0 == nullptr || scene->t1 == nullptr ||
                       scene->bounds == nullptr || scene->motion_bound == nullptr))
    return fail(P2C_ERR_INVALID, "proxy scene arrays are null");
  return P2C_OK;
}

// Validation, the sorted proxy layout of the sweep and the dense slab and
// (object, patch) ranks the compaction keys are built from.
int prepare(ProxyRun& R, cudaStream_t s) {
  const p2c_proxy_scene& sc = R.sc;
  ProxyLayout& L = R.L;
  const long long n = R.n;
  P2C_CUDA(cudaMemsetAsync(L.counter, 0, 24, s));
  if (n > 0) {
    stats_init_kernel<<<1, 32, 0, s>>>(L);
    keys_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L);
    grid_kernel<<<1, 32, 0, s>>>(L, n);
    cell_keys_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L);
    size_t tb = L.tmp_bytes;
    // (slab, column, quantised min) order, ties in proxy order
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.key[0], L.key[1], L.order[0], L.order[1], (int)n, 0,
                                             30 + R.slab_bits, s));
    gather_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L);
    if (L.table_bits > 0) {
      P2C_CUDA(cudaMemsetAsync(L.cells, 0, L.table_bytes, s));
      table_kernel<<<grid_for(n), kThreads, 0, s>>>(L, n);
    }
    // dense slab ranks from the sorted keys; dense (object, patch) ranks from one more sort
    slab_flags_kernel<<<grid_for(n), kThreads, 0, s>>>(L, n);
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceScan::InclusiveSum(L.tmp, tb, L.flag, L.scan, (int)n, s));
    slab_rank_kernel<<<grid_for(n), kThreads, 0, s>>>(L, n);
    op_keys_kernel<<<grid_for(n), kThreads, 0, s>>>(sc, L, R.patch_bits);
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.okey[0], L.okey[1], L.order[0], L.oidx, (int)n, 0,
                                             R.object_bits + R.patch_bits, s));
    op_flags_kernel<<<grid_for(n), kThreads, 0, s>>>(L, n);
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceScan::InclusiveSum(L.tmp, tb, L.flag, L.scan, (int)n, s));
    op_rank_kernel<<<grid_for(n), kThreads, 0, s>>>(L, n);
  }
  return P2C_OK;
}

// Compaction of the hits [0, cap) whose key chunks and identity permutation
// are written: stable sorts by the chunks, run heads, candidate ids, records.
int compact(ProxyRun& R, const CompactionKey& ckey, const p2c_raw_candidate_hit* raw, long long cap,
            p2c_candidate_record* candidates_dev, uint64_t* counts_dev, cudaStream_t s) {
  ProxyLayout& L = R.L;
  const int rank_bits = ckey.rank_bits;
  const int n_chunks = ckey.single ? 1 : 2;
  const unsigned long long* chunk[2] = {L.ck[0], L.ck[1]};
  const int chunk_bits[2] = {ckey.single ? ckey.d_bits + 2 * rank_bits + 2 : rank_bits + 2, ckey.d_bits + rank_bits};
  unsigned* perm_in = L.perm[0];
  unsigned* perm_out = L.perm[1];
  size_t tb;
  for (int c = 0; c < n_chunks; ++c) {
    gather_chunk_kernel<<<grid_for(cap), kThreads, 0, s>>>(chunk[c], perm_in, L.gk[0], cap);
    tb = L.tmp_bytes;
    P2C_CUDA(cub::DeviceRadixSort::SortPairs(L.tmp, tb, L.gk[0], L.gk[1], perm_in, perm_out, (int)cap, 0,
                                             chunk_bits[c], s));
    std::swap(perm_in, perm_out);
  }
  heads_kernel<<<grid_for(cap + 1), kThreads, 0, s>>>(L, perm_in, chunk[0], ckey.single ? chunk[0] : chunk[1], cap);
  tb = L.tmp_bytes;
  P2C_CUDA(cub::DeviceScan::ExclusiveSum(L.tmp, tb, L.head, L.seg, (int)(cap + 1), s));
  records_kernel<<<grid_for(cap), kThreads, 0, s>>>(R.sc, L, perm_in, raw, cap, candidates_dev,
                                                    reinterpret_cast<unsigned long long*>(counts_dev));
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

CompactionKey compaction_key(const ProxyRun& R) {
  CompactionKey ckey;
  ckey.rank_bits = R.rank_bits;
  ckey.d_bits = std::min(R.rank_bits, R.slab_bits);  // slab ranks < min(n, 2^slab_bits)
  ckey.single = ckey.d_bits + 2 * R.rank_bits + 2 <= 64;
  return ckey;
}

int setup(const p2c_proxy_scene* scene, long long raw_cap, void* workspace_dev, size_t workspace_bytes,
          ProxyRun& R) {
  R.sc = *scene;
  R.n = scene->n;
  const int table_bits = table_bits_for(scene->slab_bits);
  const size_t need = carve(nullptr, R.n, raw_cap, table_bits).total;
  if (workspace_dev == nullptr || workspace_bytes < need)
    return fail(P2C_ERR_INVALID, "proxy candidate workspace too small: %zu < %zu bytes", workspace_bytes, need);
  R.L = carve(workspace_dev, R.n, raw_cap, table_bits);
  R.rank_bits = std::max(1, bit_length((unsigned long long)std::max(R.n - 1, 1ll)));  // indices, ranks < n
  R.slab_bits = R.sc.slab_bits > 0 && R.sc.slab_bits < 32 ? (int)R.sc.slab_bits : 32;
  R.object_bits = R.sc.object_bits > 0 && R.sc.object_bits < 32 ? (int)R.sc.object_bits : 32;
  R.patch_bits = R.sc.patch_bits > 0 && R.sc.patch_bits < 32 ? (int)R.sc.patch_bits : 32;
  return P2C_OK;
}

}  // namespace
}  // namespace p2c

extern "C" {

int p2c_proxy_candidates(const p2c_proxy_scene* scene, p2c_raw_candidate_hit* raw_dev, int64_t raw_cap,
                         p2c_candidate_record* candidates_dev, uint64_t* counts_dev, void* workspace_dev,
                         size_t workspace_bytes, void* stream) {
  using namespace p2c;
  if (int rc = proxy_checks(scene)) return rc;
  if (raw_cap < 0 || raw_cap >= (1ll << 31)) return fail(P2C_ERR_INVALID, "raw capacity must lie in [0, 2^31)");
  if (counts_dev == nullptr) return fail(P2C_ERR_INVALID, "counts pointer is null");
  if (raw_cap > 0 && (raw_dev == nullptr || candidates_dev == nullptr))
    return fail(P2C_ERR_INVALID, "raw hit or candidate output pointer is null");
  ProxyRun R;
  if (int rc = setup(scene, raw_cap, workspace_dev, workspace_bytes, R)) return rc;
  cudaStream_t s = as_stream(stream);
  if (int rc = prepare(R, s)) return rc;
  ProxyLayout& L = R.L;
  const long long n = R.n, cap = raw_cap;
  if (cap > 0) fill_kernel<<<grid_for(cap), kThreads, 0, s>>>(L.pairs[0], cap);
  // the sweep counts every hit, also past the capacity (writes only below it)
  if (n > 0) sweep_kernel<<<grid_for(n * kSweepLanes), kThreads, 0, s>>>(L, n, (unsigned long long)cap, R.rank_bits);
  if (cap > 0) {
    size_t tb = L.tmp_bytes;
    const CompactionKey ckey = compaction_key(R);
    // the hits in (i, j) order
    P2C_CUDA(cub::DeviceRadixSort::SortKeys(L.tmp, tb, L.pairs[0], L.pairs[1], (int)cap, 0, 2 * R.rank_bits, s));
    raw_hits_kernel<<<grid_for(cap), kThreads, 0, s>>>(R.sc, L, L.pairs[1], (unsigned long long)cap, ckey, raw_dev);
    P2C_CUDA(cudaGetLastError());
    return compact(R, ckey, raw_dev, cap, candidates_dev, counts_dev, s);
  }
  records_kernel<<<1, kThreads, 0, s>>>(R.sc, L, L.perm[0], raw_dev, 0, candidates_dev,
                                        reinterpret_cast<unsigned long long*>(counts_dev));
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

size_t p2c_compact_raw_candidates_workspace_bytes(int64_t n_proxies, int64_t n_raw, uint32_t slab_bits) {
  return p2c_proxy_candidates_workspace_bytes(n_proxies, n_raw, slab_bits);
}

int p2c_compact_raw_candidates(const p2c_proxy_scene* scene, const p2c_raw_candidate_hit* raw_dev, int64_t n_raw,
                               p2c_candidate_record* candidates_dev, uint64_t* counts_dev, void* workspace_dev,
                               size_t workspace_bytes, void* stream) {
  using namespace p2c;
  if (int rc = proxy_checks(scene)) return rc;
  if (n_raw < 0 || n_raw >= (1ll << 31)) return fail(P2C_ERR_INVALID, "raw hit count must lie in [0, 2^31)");
  if (counts_dev == nullptr) return fail(P2C_ERR_INVALID, "counts pointer is null");
  if (n_raw > 0 && (raw_dev == nullptr || candidates_dev == nullptr))
    return fail(P2C_ERR_INVALID, "raw hit or candidate pointer is null");
  ProxyRun R;
  if (int rc = setup(scene, n_raw, workspace_dev, workspace_bytes, R)) return rc;
  cudaStream_t s = as_stream(stream);
  if (int rc = prepare(R, s)) return rc;
  set_hits_kernel<<<1, 32, 0, s>>>(R.L, n_raw);
  if (n_raw == 0) {
    records_kernel<<<1, kThreads, 0, s>>>(R.sc, R.L, R.L.perm[0], raw_dev, 0, candidates_dev,
                                          reinterpret_cast<unsigned long long*>(counts_dev));
  } else {
    const CompactionKey ckey = compaction_key(R);
    external_hits_kernel<<<grid_for(n_raw), kThreads, 0, s>>>(R.sc, R.L, raw_dev, n_raw, ckey);
    if (int rc = compact(R, ckey, raw_dev, n_raw, candidates_dev, counts_dev, s)) return rc;
  }
  first_invalid_kernel<<<1, 32, 0, s>>>(R.L, counts_dev);
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

}  // extern "C"
