// count_sort.cuh — LSD radix sort of (key, value) pairs whose count is read
// on the device.
//
// The broad phases sort only the boxes that survive culling (often a few per
// cent of a scene), and their number is known only on the device: a library
// sort sized on the host would rank every culled entry as well.  Each 8-bit
// pass is three launches over tiles of kCsTile items:
//   upsweep    per-tile digit histograms, stored digit-major;
//   scan       exclusive sum over all (digit, tile) counts: the first output
//              position of each tile's run of each digit;
//   downsweep  a stable block radix sort of the tile on the digit, then each
//              item goes to its run's position plus its rank in the run.
// Tiles at or beyond the count exit at once, so a pass costs in proportion
// to the live items; the grid is sized for the host-known capacity.  Passes
// alternate between the two buffer pairs; after an odd number of passes the
// result is in the second pair.
#pragma once

#include <cub/block/block_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "p2c_internal.cuh"

namespace p2c {

constexpr int kCsThreads = 256;
constexpr int kCsItems = 8;
constexpr int kCsTile = kCsThreads * kCsItems;
constexpr int kCsBins = 256;  // 8-bit digits

inline unsigned cs_tiles(long long cap) { return (unsigned)std::max<long long>(1, (cap + kCsTile - 1) / kCsTile); }

template <class K>
__global__ void __launch_bounds__(kCsThreads) cs_upsweep_kernel(const K* __restrict__ keys,
                                                                const unsigned long long* __restrict__ count,
                                                                int shift, unsigned* __restrict__ hist, unsigned tiles) {
  __shared__ unsigned h[kCsBins];
  for (int b = threadIdx.x; b < kCsBins; b += kCsThreads) h[b] = 0u;
  __syncthreads();
  const unsigned long long n = *count;
  const unsigned long long base = (unsigned long long)blockIdx.x * kCsTile;
  if (base < n) {
#pragma unroll
    for (int k = 0; k < kCsItems; ++k) {
      const unsigned long long i = base + (unsigned long long)(k * kCsThreads + threadIdx.x);
      if (i < n) atomicAdd(&h[(unsigned)(keys[i] >> shift) & (kCsBins - 1)], 1u);
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kCsBins; b += kCsThreads) hist[(size_t)b * tiles + blockIdx.x] = h[b];
}

template <class K, class V>
struct CsDown {
  using Sort = cub::BlockRadixSort<K, kCsThreads, kCsItems, V, 4>;
  union Storage {
    typename Sort::TempStorage sort;
    struct {
      unsigned start[kCsBins];  // first tile position of each digit's run
      unsigned long long out[kCsBins];
    } runs;
  };
};

template <class K, class V>
__global__ void __launch_bounds__(kCsThreads) cs_downsweep_kernel(const K* __restrict__ keys_in,
                                                                  const V* __restrict__ vals_in,
                                                                  K* __restrict__ keys_out, V* __restrict__ vals_out,
                                                                  const unsigned long long* __restrict__ count,
                                                                  int shift, const unsigned* __restrict__ offsets,
                                                                  unsigned tiles) {
  using D = CsDown<K, V>;
  __shared__ typename D::Storage sm;
  __shared__ unsigned hist[kCsBins];
  const unsigned long long n = *count;
  const unsigned long long base = (unsigned long long)blockIdx.x * kCsTile;
  if (base >= n) return;  // uniform per block
  const unsigned live = (unsigned)min((unsigned long long)kCsTile, n - base);
  // blocked arrangement: thread t holds items t * kCsItems + k of the tile
  K k[kCsItems];
  V v[kCsItems];
#pragma unroll
  for (int j = 0; j < kCsItems; ++j) {
    const unsigned p = threadIdx.x * kCsItems + j;
    if (p < live) {
      k[j] = keys_in[base + p];
      v[j] = vals_in[base + p];
    } else {
      k[j] = ~K(0);  // digit 0xff, after every live item of that digit (the sort is stable)
      v[j] = V(0);
    }
  }
  for (int b = threadIdx.x; b < kCsBins; b += kCsThreads) hist[b] = 0u;
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kCsItems; ++j)
    if (threadIdx.x * kCsItems + j < live) atomicAdd(&hist[(unsigned)(k[j] >> shift) & (kCsBins - 1)], 1u);
  __syncthreads();
  typename D::Sort(sm.sort).Sort(k, v, shift, shift + 8);
  __syncthreads();  // the union's sort storage is reused below
  if (threadIdx.x == 0) {
    unsigned run = 0;
    for (int b = 0; b < kCsBins; ++b) {
      sm.runs.start[b] = run;
      run += hist[b];
    }
  }
  for (int b = threadIdx.x; b < kCsBins; b += kCsThreads)
    sm.runs.out[b] = (unsigned long long)offsets[(size_t)b * tiles + blockIdx.x];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kCsItems; ++j) {
    const unsigned p = threadIdx.x * kCsItems + j;  // position in the sorted tile
    const unsigned d = (unsigned)(k[j] >> shift) & (kCsBins - 1);
    const unsigned r = p - sm.runs.start[d];
    if (r < hist[d]) {  // padding items rank past their digit's live count
      const unsigned long long o = sm.runs.out[d] + r;
      keys_out[o] = k[j];
      vals_out[o] = v[j];
    }
  }
}

// Scratch of count_sort_pairs for up to cap items.
inline size_t count_sort_scratch_bytes(long long cap) {
  const size_t entries = (size_t)kCsBins * cs_tiles(cap);
  size_t scan = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan, (const unsigned*)nullptr, (unsigned*)nullptr, (int)entries);
  return 2 * ((entries * sizeof(unsigned) + 255) & ~size_t(255)) + ((scan + 255) & ~size_t(255));
}

// Sort the first *count_dev pairs of (k0, v0) on bits [0, end_bit) into
// (k0, v0) or (k1, v1): *in_second is set when the result is in (k1, v1).
template <class K, class V>
int count_sort_pairs(K* k0, V* v0, K* k1, V* v1, const unsigned long long* count_dev, long long cap, int end_bit,
                     void* scratch, size_t scratch_bytes, cudaStream_t s, bool* in_second) {
  const unsigned tiles = cs_tiles(cap);
  const size_t entries = (size_t)kCsBins * tiles;
  const size_t hb = (entries * sizeof(unsigned) + 255) & ~size_t(255);
  if (scratch_bytes < count_sort_scratch_bytes(cap)) return fail(P2C_ERR_INVALID, "count sort scratch too small");
  unsigned* hist = static_cast<unsigned*>(scratch);
  unsigned* offs = reinterpret_cast<unsigned*>(static_cast<char*>(scratch) + hb);
  void* tmp = static_cast<char*>(scratch) + 2 * hb;
  size_t tmp_bytes = scratch_bytes - 2 * hb;
  K* ka[2] = {k0, k1};
  V* va[2] = {v0, v1};
  int cur = 0;
  for (int shift = 0; shift < end_bit; shift += 8) {
    cs_upsweep_kernel<K><<<tiles, kCsThreads, 0, s>>>(ka[cur], count_dev, shift, hist, tiles);
    P2C_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, hist, offs, (int)entries, s));
    cs_downsweep_kernel<K, V><<<tiles, kCsThreads, 0, s>>>(ka[cur], va[cur], ka[1 - cur], va[1 - cur], count_dev,
                                                           shift, offs, tiles);
    P2C_CUDA(cudaGetLastError());
    cur = 1 - cur;
  }
  *in_second = cur == 1;
  return P2C_OK;
}

}  // namespace p2c
