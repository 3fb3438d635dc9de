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

}  // namespace p2c
