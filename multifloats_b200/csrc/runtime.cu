// Host runtime of libmultifloats_cuda: error latch, device checks, staging
// buffers for the drop-in (host-pointer) symbols, workspace allocation.
#include <atomic>
#include <cstdlib>
#include <cstring>

#include "common.cuh"

namespace mfcuda {

static thread_local int t_last_error = MFCUDA_OK;
void set_last_error(int code) { t_last_error = code; }
int last_error() { return t_last_error; }

static constexpr int kMaxDevices = 64;

int require_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return MFCUDA_ERR_NO_DEVICE;
  }
  if (dev < 0 || dev >= kMaxDevices) return MFCUDA_ERR_NO_DEVICE;
  static std::atomic<int> major_cache[kMaxDevices];
  int major = major_cache[dev].load(std::memory_order_relaxed);
  if (major == 0) {
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
      (void)cudaGetLastError();
      return MFCUDA_ERR_NO_DEVICE;
    }
    major_cache[dev].store(major, std::memory_order_relaxed);
  }
  // The kernels are built for sm_100a only.
  return major == 10 ? MFCUDA_OK : MFCUDA_ERR_NO_DEVICE;
}

int sm_count() {
  int dev = 0;
  cudaGetDevice(&dev);
  static std::atomic<int> cache[kMaxDevices];
  int v = (dev >= 0 && dev < kMaxDevices) ? cache[dev].load() : 0;
  if (v == 0) {
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    if (v <= 0) v = 148;
    if (dev >= 0 && dev < kMaxDevices) cache[dev].store(v);
  }
  return v;
}

bool injected_alloc_failure() {
  static std::atomic<long> counter{0};
  static long target = [] {
    const char *s = std::getenv("MFCUDA_FAIL_ALLOC");
    return s ? std::atol(s) : 0L;
  }();
  if (target <= 0) return false;
  return counter.fetch_add(1) + 1 == target;
}

static std::atomic<uint64_t> g_wait_limit_ns{0};  // 0: the default
static constexpr uint64_t kDefaultWaitNs = 2000000000ull;
uint64_t wait_limit_ns() {
  const uint64_t v = g_wait_limit_ns.load(std::memory_order_relaxed);
  return v ? v : kDefaultWaitNs;
}

namespace {
struct DeviceStaging {
  std::mutex mu;
  cudaStream_t stream = nullptr, copy = nullptr;
  cudaEvent_t ev[kStagingEvents] = {};
  bool have_ev = false;
  void *buf[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t cap[4] = {0, 0, 0, 0};
};
DeviceStaging g_staging[kMaxDevices];
}  // namespace

int staging_acquire(Staging &st, const size_t bytes[4]) {
  int dev = 0;
  MF_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return MFCUDA_ERR_NO_DEVICE;
  DeviceStaging &ds = g_staging[dev];
  st.lock = std::unique_lock<std::mutex>(ds.mu);
  if (!ds.stream) MF_TRY_CUDA(cudaStreamCreateWithFlags(&ds.stream, cudaStreamNonBlocking));
  if (!ds.copy) MF_TRY_CUDA(cudaStreamCreateWithFlags(&ds.copy, cudaStreamNonBlocking));
  if (!ds.have_ev) {
    for (int i = 0; i < kStagingEvents; ++i)
      MF_TRY_CUDA(cudaEventCreateWithFlags(&ds.ev[i], cudaEventDisableTiming));
    ds.have_ev = true;
  }
  st.stream = ds.stream;
  st.copy = ds.copy;
  for (int i = 0; i < kStagingEvents; ++i) st.ev[i] = ds.ev[i];
  for (int i = 0; i < 4; ++i) {
    if (bytes[i] > ds.cap[i]) {
      if (ds.buf[i]) {
        MF_TRY_CUDA(cudaStreamSynchronize(ds.stream));
        MF_TRY_CUDA(cudaFree(ds.buf[i]));
        ds.buf[i] = nullptr;
        ds.cap[i] = 0;
      }
      if (injected_alloc_failure()) return MFCUDA_ERR_ALLOC;
      size_t want = bytes[i] < 256 ? 256 : bytes[i];
      MF_TRY_CUDA(cudaMalloc(&ds.buf[i], want));
      ds.cap[i] = want;
    }
    st.buf[i] = ds.buf[i];
  }
  return MFCUDA_OK;
}

int ws_alloc(void **p, size_t bytes, cudaStream_t s) {
  *p = nullptr;
  if (bytes == 0) return MFCUDA_OK;
  if (injected_alloc_failure()) return MFCUDA_ERR_ALLOC;
  MF_TRY_CUDA(cudaMallocAsync(p, bytes, s));
  return MFCUDA_OK;
}
void ws_free(void *p, cudaStream_t s) {
  if (p) (void)cudaFreeAsync(p, s);
}

}  // namespace mfcuda

extern "C" {

MULTIFLOATS_CUDA_API int mfcuda_last_error(void) { return mfcuda::last_error(); }

MULTIFLOATS_CUDA_API const char *mfcuda_error_string(int code) {
  switch (code) {
    case MFCUDA_OK: return "success";
    case MFCUDA_ERR_INVALID_ARG: return "invalid argument";
    case MFCUDA_ERR_CUDA: return "CUDA runtime error";
    case MFCUDA_ERR_ALLOC: return "allocation failed";
    case MFCUDA_ERR_NO_DEVICE: return "no sm_100 device";
    case MFCUDA_ERR_TIMEOUT: return "device-side wait timed out";
    case MFCUDA_ERR_WORKSPACE: return "workspace too small";
    case MFCUDA_ERR_UNSUPPORTED: return "unsupported shape or parameter";
    default: return "unknown error";
  }
}

MULTIFLOATS_CUDA_API const char *mfcuda_version(void) { return "0.1.0"; }

MULTIFLOATS_CUDA_API uint64_t mfcuda_set_wait_limit_ns(uint64_t ns) {
  return mfcuda::g_wait_limit_ns.exchange(ns);
}

}  // extern "C"
