// p2c_internal.cuh — host-side plumbing shared by the library's translation
// units: last-error string, CUDA status checks, device properties, a
// per-device scratch cache for the host-buffer entry points.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <mutex>
#include <string>

#include "p2c_b200.h"

namespace p2c {

void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

inline int cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return P2C_OK;
  return fail(P2C_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define P2C_CUDA(call)                                   \
  do {                                                   \
    const int p2c_rc_ = ::p2c::cuda_check((call), #call); \
    if (p2c_rc_ != P2C_OK) return p2c_rc_;               \
  } while (0)

struct DeviceInfo {
  int device = -1;
  int sm_count = 0;
  int max_smem_optin = 0;
  int cc_major = 0, cc_minor = 0;
};
int current_device_info(DeviceInfo* info);

// Grow-only device buffer owned by the library, one per (device, purpose);
// used only by the host-buffer (reference-ownership) entry points.
struct HostApiBuffers {
  std::mutex mu;
  void* dev = nullptr;
  size_t bytes = 0;
  int device = -1;
};
int ensure_buffer(HostApiBuffers& b, size_t bytes);

// Device time budget for one launch, from P2C_DEVICE_BUDGET_MS (default 30 s).
unsigned long long device_budget_ns();

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Programmatic dependent launch: the kernel may be scheduled while its
// predecessor on the stream (or in the graph) finishes its last wave.  Every
// kernel launched this way starts with pdl_wait() (the predecessor has
// completed and its writes are visible) before it reads anything, then
// pdl_trigger() lets its own successor be scheduled.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

#ifdef __CUDACC__
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
#endif

}  // namespace p2c
