// Host-side plumbing shared by the kernels' C-ABI wrappers: status codes,
// the per-thread error latch of the drop-in symbols, argument checks and a
// per-device cache of staging buffers for host-pointer calls.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <mutex>

#include "../../include/multifloats_cuda.h"

namespace mfcuda {

// Status of the calling thread's last drop-in call.
void set_last_error(int code);
int last_error();

#define MF_TRY_CUDA(expr)                          \
  do {                                             \
    cudaError_t mf_err_ = (expr);                  \
    if (mf_err_ != cudaSuccess) {                  \
      (void)cudaGetLastError();                    \
      return mf_err_ == cudaErrorMemoryAllocation  \
                 ? MFCUDA_ERR_ALLOC                \
                 : MFCUDA_ERR_CUDA;                \
    }                                              \
  } while (0)

#define MF_TRY(expr)               \
  do {                             \
    int mf_rc_ = (expr);           \
    if (mf_rc_ != MFCUDA_OK)       \
      return mf_rc_;               \
  } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// n elements of `elem` bytes: false on negative sizes or byte-count overflow.
inline bool size_ok(int64_t n, size_t elem) {
  if (n < 0) return false;
  return (uint64_t)n <= (UINT64_MAX / 2) / elem;
}
inline bool mul_ok(int64_t a, int64_t b) {
  if (a < 0 || b < 0) return false;
  if (a == 0 || b == 0) return true;
  return a <= INT64_MAX / b;
}

// Checks that a compute-capability-10.x device is current.
int require_device();

// Number of SMs of the current device (cached per device).
int sm_count();

// Grow-only device staging buffers used by the drop-in (host-pointer) calls.
// Each drop-in call holds the cache lock for its whole duration, so one
// process-wide set of buffers per device is enough.
constexpr int kStagingEvents = 8;
struct Staging {
  std::unique_lock<std::mutex> lock;
  cudaStream_t stream = nullptr;
  cudaStream_t copy = nullptr;            // second stream for copies that overlap the compute stream
  cudaEvent_t ev[kStagingEvents] = {};    // ordering events between the two (no timing)
  void *buf[4] = {nullptr, nullptr, nullptr, nullptr};
};
// Acquire staging buffers of the given byte sizes on the current device.
int staging_acquire(Staging &st, const size_t bytes[4]);

// Test hook: when the environment variable MFCUDA_FAIL_ALLOC is set to a
// positive integer N, the N-th staging/workspace allocation of the process
// reports MFCUDA_ERR_ALLOC without calling the CUDA allocator.
bool injected_alloc_failure();

// Limit (ns) of the bounded waits in the tensor-core kernels launched from
// now on (mfcuda_set_wait_limit_ns; 2 s unless set).
uint64_t wait_limit_ns();

// Stream-ordered workspace allocation for device-pointer calls given no workspace.
int ws_alloc(void **p, size_t bytes, cudaStream_t s);
void ws_free(void *p, cudaStream_t s);

}  // namespace mfcuda
