// refine.cu — conservative refinement children of certified work items on
// the device: GenerateConservativeRefinementWorkItems
// (cpp/certificate/certificate_engine.cpp:663-720) for a whole queue at once.
//
// Per parent: a collision gives one child [t0, clamp(toi_upper, t0, t1)] when
// it is wider than min_interval_width; an undecided certificate that asks for
// bisection gives the two halves around 0.5 * (t0 + t1) when the parent is
// wider than min_interval_width; nothing at max_child_depth.  Children are
// written compacted in parent order (a count pass, a CUB exclusive scan, a
// write pass), so child k carries work_item_id first_child_work_item_id + k:
// the ids the reference assigns when it is called once per parent in queue
// order with the next free id.
#include <cub/device/device_scan.cuh>

#include "certify_core.cuh"
#include "p2c_internal.cuh"

namespace p2c {
namespace {

struct RefineArgs {
  long long n;
  const double* t0;
  const double* t1;
  const uint16_t* depth;
  const p2c_query_certificate* certs;
  uint16_t max_child_depth;
  double min_width;
  unsigned long long first_id;
  long long* child_parent;
  double* child_t0;
  double* child_t1;
  uint16_t* child_depth;
  unsigned long long* child_id;
  unsigned long long* child_count;
  unsigned* counts;   // n + 1
  unsigned* offsets;  // n + 1
  unsigned long long* error_word;
};

// Children of parent i: their number and intervals (as certificate_engine.cpp:686-719).
__device__ __forceinline__ int children_of(const RefineArgs& a, long long i, double c0[2], double c1[2]) {
  const double t0 = a.t0[i], t1 = a.t1[i];
  if (!(isfinite(t0) && isfinite(t1)) || t0 < 0.0 || t1 > 1.0 || t0 > t1) {
    atomicOr(a.error_word, 1ull);  // not a valid work-item interval: no children
    return 0;
  }
  if (a.depth[i] >= a.max_child_depth) return 0;
  const p2c_query_certificate& c = a.certs[i];
  if (c.status == P2C_STATUS_COLLISION) {
    const double ct1 = clamp_std(c.toi_upper, t0, t1);
    if (sub(ct1, t0) > a.min_width) {
      c0[0] = t0;
      c1[0] = ct1;
      return 1;
    }
    return 0;
  }
  if (c.status == P2C_STATUS_UNDECIDED && c.next_refinement_mode == P2C_REFINE_BISECT_INTERVAL &&
      sub(t1, t0) > a.min_width) {
    const double mid = mul(0.5, add(t0, t1));
    c0[0] = t0;
    c1[0] = mid;
    c0[1] = mid;
    c1[1] = t1;
    return 2;
  }
  return 0;
}

__global__ void count_kernel(RefineArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > a.n) return;
  if (i == a.n) {
    a.counts[i] = 0u;
    return;
  }
  double c0[2], c1[2];
  a.counts[i] = (unsigned)children_of(a, i, c0, c1);
}

__global__ void write_kernel(RefineArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *a.child_count = a.offsets[a.n];
  if (i >= a.n) return;
  double c0[2], c1[2];
  const int k = a.counts[i];
  if (k == 0) return;
  children_of(a, i, c0, c1);
  const unsigned base = a.offsets[i];
  for (int j = 0; j < k; ++j) {
    const unsigned long long slot = (unsigned long long)base + (unsigned)j;
    a.child_parent[slot] = i;
    a.child_t0[slot] = c0[j];
    a.child_t1[slot] = c1[j];
    a.child_depth[slot] = (uint16_t)(a.depth[i] + 1);
    a.child_id[slot] = a.first_id + slot;
  }
}

size_t scan_temp_bytes(long long n) {
  size_t b = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const unsigned*)nullptr, (unsigned*)nullptr, (int)(n + 1));
  return b;
}

struct RefineLayout {
  unsigned* counts;
  unsigned* offsets;
  unsigned long long* error_word;
  void* tmp;
  size_t tmp_bytes;
  size_t total;
};

RefineLayout carve(void* base, long long n) {
  RefineLayout L{};
  size_t off = 0;
  char* b = static_cast<char*>(base);
  auto take = [&](size_t bytes) -> void* {
    void* p = b == nullptr ? nullptr : b + off;
    off += (bytes + 255) & ~size_t(255);
    return p;
  };
  L.counts = static_cast<unsigned*>(take(4 * (size_t)(n + 1)));
  L.offsets = static_cast<unsigned*>(take(4 * (size_t)(n + 1)));
  L.error_word = static_cast<unsigned long long*>(take(8));
  L.tmp_bytes = scan_temp_bytes(n);
  L.tmp = take(L.tmp_bytes);
  L.total = off;
  return L;
}

}  // namespace
}  // namespace p2c

extern "C" {

size_t p2c_refinement_children_workspace_bytes(int64_t n_parents) {
  if (n_parents < 0 || n_parents >= (1ll << 30)) return 0;
  return p2c::carve(nullptr, n_parents).total;
}

int p2c_refinement_children(int64_t n_parents, const double* parent_t0_dev, const double* parent_t1_dev,
                            const uint16_t* parent_depth_dev, const p2c_query_certificate* certs_dev,
                            uint16_t max_child_depth, double min_interval_width, uint64_t first_child_work_item_id,
                            int64_t* child_parent_dev, double* child_t0_dev, double* child_t1_dev,
                            uint16_t* child_depth_dev, uint64_t* child_work_item_id_dev, uint64_t* child_count_dev,
                            uint64_t* error_word_dev, void* workspace_dev, size_t workspace_bytes, void* stream) {
  using namespace p2c;
  if (n_parents < 0 || n_parents >= (1ll << 30)) return fail(P2C_ERR_INVALID, "parent count must lie in [0, 2^30)");
  if (first_child_work_item_id == 0)
    return fail(P2C_ERR_INVALID, "ExactRefinementConfig.first_child_work_item_id must be non-zero");
  if (!std::isfinite(min_interval_width) || min_interval_width <= 0.0)
    return fail(P2C_ERR_INVALID, "ExactRefinementConfig.min_interval_width must be finite and positive");
  if (child_count_dev == nullptr) return fail(P2C_ERR_INVALID, "child count pointer is null");
  if (n_parents > 0 && (parent_t0_dev == nullptr || parent_t1_dev == nullptr || parent_depth_dev == nullptr ||
                        certs_dev == nullptr || child_parent_dev == nullptr || child_t0_dev == nullptr ||
                        child_t1_dev == nullptr || child_depth_dev == nullptr || child_work_item_id_dev == nullptr))
    return fail(P2C_ERR_INVALID, "parent or child array pointer is null");
  const RefineLayout need = carve(nullptr, n_parents);
  if (workspace_dev == nullptr || workspace_bytes < need.total)
    return fail(P2C_ERR_INVALID, "refinement workspace too small: %zu < %zu bytes", workspace_bytes, need.total);
  RefineLayout L = carve(workspace_dev, n_parents);
  cudaStream_t s = as_stream(stream);
  RefineArgs a{n_parents, parent_t0_dev, parent_t1_dev, parent_depth_dev, certs_dev, max_child_depth,
               min_interval_width, (unsigned long long)first_child_work_item_id,
               reinterpret_cast<long long*>(child_parent_dev), child_t0_dev, child_t1_dev, child_depth_dev,
               reinterpret_cast<unsigned long long*>(child_work_item_id_dev),
               reinterpret_cast<unsigned long long*>(child_count_dev), L.counts, L.offsets,
               error_word_dev != nullptr ? reinterpret_cast<unsigned long long*>(error_word_dev) : L.error_word};
  if (error_word_dev != nullptr) P2C_CUDA(cudaMemsetAsync(error_word_dev, 0, sizeof(uint64_t), s));
  const unsigned grid = (unsigned)((n_parents + 1 + 255) / 256);
  count_kernel<<<grid, 256, 0, s>>>(a);
  P2C_CUDA(cudaGetLastError());
  size_t tb = L.tmp_bytes;
  P2C_CUDA(cub::DeviceScan::ExclusiveSum(L.tmp, tb, L.counts, L.offsets, (int)(n_parents + 1), s));
  write_kernel<<<grid, 256, 0, s>>>(a);
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}

}  // extern "C"
