// p2c_runtime.cu — library-wide host plumbing: last-error string, device
// properties, scratch for the host-buffer entry points, ABI version.
#include "p2c_internal.cuh"

#include <cstdlib>

namespace p2c {

namespace {
thread_local std::string g_last_error;
}

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int current_device_info(DeviceInfo* info) {
  static std::mutex mu;
  static DeviceInfo cache[64];
  int dev = 0;
  P2C_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(P2C_ERR_CUDA, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(mu);
  if (cache[dev].device != dev) {
    DeviceInfo d;
    d.device = dev;
    P2C_CUDA(cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev));
    P2C_CUDA(cudaDeviceGetAttribute(&d.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    P2C_CUDA(cudaDeviceGetAttribute(&d.cc_major, cudaDevAttrComputeCapabilityMajor, dev));
    P2C_CUDA(cudaDeviceGetAttribute(&d.cc_minor, cudaDevAttrComputeCapabilityMinor, dev));
    cache[dev] = d;
  }
  *info = cache[dev];
  return P2C_OK;
}

int ensure_buffer(HostApiBuffers& b, size_t bytes) {
  int dev = 0;
  P2C_CUDA(cudaGetDevice(&dev));
  if (b.dev != nullptr && b.device == dev && b.bytes >= bytes) return P2C_OK;
  if (b.dev != nullptr && b.device == dev) {
    P2C_CUDA(cudaFree(b.dev));
    b.dev = nullptr;
    b.bytes = 0;
  }
  size_t want = bytes < 4096 ? 4096 : bytes + bytes / 4;
  P2C_CUDA(cudaMalloc(&b.dev, want));
  b.bytes = want;
  b.device = dev;
  return P2C_OK;
}

unsigned long long device_budget_ns() {
  static unsigned long long v = [] {
    const char* e = std::getenv("P2C_DEVICE_BUDGET_MS");
    unsigned long long ms = 30000ull;
    if (e != nullptr && *e != '\0') ms = std::strtoull(e, nullptr, 10);
    if (ms == 0ull || ms > 600000ull) ms = 30000ull;  // never unbounded, never above 10 minutes
    return ms * 1000000ull;
  }();
  return v;
}

}  // namespace p2c

extern "C" {

const char* p2c_last_error(void) { return p2c::g_last_error.c_str(); }

int p2c_abi_version(void) { return 1; }

int p2c_is_cuda_exact_built(void) { return 1; }

int p2c_device_info(int* sm_count, int* max_smem_per_block, int* cc_major, int* cc_minor) {
  p2c::DeviceInfo d;
  const int rc = p2c::current_device_info(&d);
  if (rc != P2C_OK) return rc;
  if (sm_count) *sm_count = d.sm_count;
  if (max_smem_per_block) *max_smem_per_block = d.max_smem_optin;
  if (cc_major) *cc_major = d.cc_major;
  if (cc_minor) *cc_minor = d.cc_minor;
  return P2C_OK;
}

}  // extern "C"
