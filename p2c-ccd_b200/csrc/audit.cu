// audit.cu — the audit log of an exact work queue, written on the device
// from the certificates (ProcessExactWorkQueueCpu's rows,
// certificate/certificate_engine.cpp:593-661, MakeAuditRow :456-477,
// AuditActionForCertificate :443-454).  Event ids and timestamps are the
// reference's counters (first value + row position), so the rows are
// deterministic and identical to the reference's.
#include "p2c_internal.cuh"

namespace p2c {
namespace {

constexpr int kThreads = 256;
constexpr uint8_t kStageExact = 2, kStageCertify = 4;
constexpr uint16_t kDequeued = 1, kCollision = 2, kSeparation = 3, kUndecided = 4, kInvalidInput = 5;
constexpr uint16_t kReasonInvalidInput = 3;

// ValidateAuditLogRow (common/validators.cpp:295-315); event ids are non-zero
// by construction (checked on the host).
__device__ __forceinline__ bool row_valid(const p2c_audit_row& r) {
  return r.query_id != 0 && isfinite(r.interval_t0) && isfinite(r.interval_t1) && !(r.interval_t0 < 0.0) &&
         !(r.interval_t1 > 1.0) && !(r.interval_t0 > r.interval_t1) && r.timestamp_us != 0 &&
         isfinite(r.aux_value0) && isfinite(r.aux_value1);
}

__device__ __forceinline__ p2c_audit_row make_row(const p2c_audit_item& it, unsigned long long event,
                                                  unsigned long long ts, uint8_t stage, uint16_t action, double aux0,
                                                  double aux1) {
  p2c_audit_row r{};
  r.event_id = event;
  r.query_id = it.query_id;
  r.candidate_id = it.candidate_id;
  r.work_item_id = it.work_item_id;
  r.stage = stage;
  r.action = action;
  r.depth = it.depth;
  r.interval_t0 = it.interval_t0;
  r.interval_t1 = it.interval_t1;
  r.timestamp_us = ts;
  r.aux_value0 = aux0;
  r.aux_value1 = aux1;
  return r;
}

__global__ void audit_kernel(const p2c_audit_item* __restrict__ items, const p2c_query_certificate* __restrict__ certs,
                             long long n, unsigned long long first_event, unsigned long long first_ts, int emit,
                             p2c_audit_row* rows, unsigned long long* err) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const p2c_audit_item it = items[k];
  const p2c_query_certificate c = certs[k];
  const long long per = emit ? 2 : 1, base = k * per;
  bool ok = true;
  if (emit) {
    const p2c_audit_row d = make_row(it, first_event + base, first_ts + base, kStageExact, kDequeued,
                                     (double)it.priority_score, (double)it.feature_family_mask);
    ok = ok && row_valid(d);
    rows[base] = d;
  }
  const uint16_t action = c.status == 0 ? kCollision
                          : c.status == 1 ? kSeparation
                                          : (c.reason_code == kReasonInvalidInput ? kInvalidInput : kUndecided);
  const p2c_audit_row r = make_row(it, first_event + base + per - 1, first_ts + base + per - 1, kStageCertify,
                                   action, c.status == 1 ? c.safe_margin_lb : c.toi_upper,
                                   (double)c.next_refinement_mode);
  ok = ok && row_valid(r);
  rows[base + per - 1] = r;
  if (!ok) {
    atomicOr(err, 1ull);
    atomicMin(err + 1, (unsigned long long)base);
  }
}

__global__ void audit_init_kernel(unsigned long long* err) {
  if (threadIdx.x == 0) {
    err[0] = 0ull;
    err[1] = ~0ull;
  }
}

}  // namespace
}  // namespace p2c

extern "C" int p2c_audit_rows(const p2c_audit_item* items_dev, const p2c_query_certificate* certs_dev, int64_t n,
                              uint64_t first_event_id, uint64_t first_timestamp_us, int emit_dequeue_events,
                              p2c_audit_row* rows_dev, uint64_t* error_dev, void* stream) {
  using namespace p2c;
  if (first_event_id == 0) return fail(P2C_ERR_INVALID, "ExactWorkQueueConfig.first_event_id must be non-zero");
  if (first_timestamp_us == 0)
    return fail(P2C_ERR_INVALID, "ExactWorkQueueConfig.first_timestamp_us must be non-zero");
  if (n < 0) return fail(P2C_ERR_INVALID, "work item count is negative");
  if (error_dev == nullptr || (n > 0 && (items_dev == nullptr || certs_dev == nullptr || rows_dev == nullptr)))
    return fail(P2C_ERR_INVALID, "item, certificate, row or error pointer is null");
  cudaStream_t s = as_stream(stream);
  unsigned long long* err = reinterpret_cast<unsigned long long*>(error_dev);
  audit_init_kernel<<<1, 32, 0, s>>>(err);
  if (n > 0)
    audit_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(
        items_dev, certs_dev, n, first_event_id, first_timestamp_us, emit_dequeue_events ? 1 : 0, rows_dev, err);
  P2C_CUDA(cudaGetLastError());
  return P2C_OK;
}
