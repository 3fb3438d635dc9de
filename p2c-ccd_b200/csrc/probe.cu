// probe.cu — FP64 throughput probe: the measured denominator of the
// certifier's roofline.  Eight independent chains per thread of separately
// rounded multiply and add (DMUL + DADD, the instruction mix of the
// --fmad=false certifier; no DFMA), over a full-occupancy grid.
#include "p2c_internal.cuh"

namespace p2c {
namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeChains = 8;

__global__ void __launch_bounds__(kProbeThreads) fp64_probe_kernel(double* out, int iters) {
  const double seed = 1.0 + 1e-9 * (double)(blockIdx.x * blockDim.x + threadIdx.x);
  double a[kProbeChains];
#pragma unroll
  for (int k = 0; k < kProbeChains; ++k) a[k] = seed + 0.125 * k;
  const double m = 0.999999999, c = 1e-9;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kProbeChains; ++k) a[k] = __dadd_rn(__dmul_rn(a[k], m), c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kProbeChains; ++k) s += a[k];
  if (s == 12345.678) out[0] = s;  // keeps the chains live; practically never taken
}

}  // namespace
}  // namespace p2c

extern "C" int p2c_probe_fp64(void* out_dev, int iters, long long* fp64_ops_out, void* stream) {
  p2c::DeviceInfo dev;
  int rc = p2c::current_device_info(&dev);
  if (rc != P2C_OK) return rc;
  if (out_dev == nullptr || iters <= 0) return p2c::fail(P2C_ERR_INVALID, "probe needs an output and iters > 0");
  int per_sm = 0;
  P2C_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, p2c::fp64_probe_kernel, p2c::kProbeThreads, 0));
  if (per_sm < 1) per_sm = 1;
  const int grid = dev.sm_count * per_sm;
  p2c::fp64_probe_kernel<<<grid, p2c::kProbeThreads, 0, p2c::as_stream(stream)>>>(static_cast<double*>(out_dev),
                                                                                 iters);
  P2C_CUDA(cudaGetLastError());
  if (fp64_ops_out)
    *fp64_ops_out = (long long)grid * p2c::kProbeThreads * (long long)iters * p2c::kProbeChains * 2;
  return P2C_OK;
}
