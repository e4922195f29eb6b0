// Peak-throughput probes used as roofline denominators by bench.py (not part of
// the library's C ABI): FP64 pipe instruction rate.  Each thread runs
// independent FMA chains on registers only; the grid fills every SM.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) fp64_fma_probe(double *out, int64_t iters, double a,
                                                      double b) {
  double x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3 + c;
  for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = __fma_rn(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == 1.2345) out[0] = s;  // keeps the chains alive
}

}  // namespace

extern "C" __attribute__((visibility("default"))) int mfpeak_fp64(int64_t iters, void *stream_,
                                                                   double *ms_out,
                                                                   double *instr_out) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 2;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double *out = nullptr;
  if (cudaMallocAsync(&out, 8, stream) != cudaSuccess) return 3;
  int blocks = sms * 8;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fp64_fma_probe<<<blocks, 256, 0, stream>>>(out, iters / 8, 0.999999, 1e-7);  // warm-up
  cudaEventRecord(e0, stream);
  fp64_fma_probe<<<blocks, 256, 0, stream>>>(out, iters, 0.999999, 1e-7);
  cudaEventRecord(e1, stream);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(out, stream);
  *ms_out = ms;
  *instr_out = (double)blocks * 256.0 * (double)iters * kChains;
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// ---- INT8 tensor pipe: tcgen05.mma kind::i8, M=128 N=256 K=32 from shared memory ----
#include "tcgen05.cuh"

namespace {
constexpr int kProbeN = 256;
__global__ void __launch_bounds__(128, 1) int8_mma_probe(int iters, int *status) {
  extern __shared__ uint8_t dyn[];
  uint8_t *tileA = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(dyn) + 1023) & ~uintptr_t(1023));
  uint8_t *tileB = tileA + 128 * 128;
  __shared__ __align__(8) uint64_t done;
  __shared__ uint32_t tslot;
  for (int i = threadIdx.x; i < 128 * 128; i += blockDim.x) tileA[i] = (uint8_t)(i * 7);
  for (int i = threadIdx.x; i < 256 * 128; i += blockDim.x) tileB[i] = (uint8_t)(i * 13);
  const int warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    mftc::mbar_init(&done, 1);
    mftc::fence_mbar_init();
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    mftc::tmem_alloc(&tslot, 2 * kProbeN);
    mftc::tmem_relinquish();
  }
  mftc::tc_fence_before();
  __syncthreads();
  mftc::tc_fence_after();
  const uint32_t tbase = tslot;
  if (threadIdx.x == 0) {
    const uint32_t idesc = mftc::idesc_i8(128, kProbeN);
    const uint32_t a0 = mftc::smem_u32(tileA), b0 = mftc::smem_u32(tileB);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        mftc::umma_i8(tbase + (uint32_t)((it & 1) * kProbeN), mftc::smem_desc_k_sw128(a0 + kk * 32),
                      mftc::smem_desc_k_sw128(b0 + kk * 32), idesc, (it > 1 || kk > 0) ? 1u : 0u);
    }
    mftc::umma_commit(&done);
    uint64_t t0, t1;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t0));
    while (!mftc::mbar_try_wait(&done, 0)) {
      asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t1));
      if (t1 - t0 > 2000000000ull) {
        atomicOr(status, 1);
        break;
      }
    }
  }
  mftc::tc_fence_before();
  __syncthreads();
  mftc::tc_fence_after();
  if (warp == 0) mftc::tmem_dealloc(tbase, 2 * kProbeN);
}
}  // namespace

// INT8 tensor ops per second of back-to-back M=128 N=256 K=32 MMAs on every SM.
extern "C" __attribute__((visibility("default"))) int mfpeak_int8(int iters, void *stream_,
                                                                  double *ms_out, double *ops_out) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 2;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int *status = nullptr;
  if (cudaMallocAsync(&status, 4, stream) != cudaSuccess) return 3;
  cudaMemsetAsync(status, 0, 4, stream);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int smem = 120 * 1024;  // tiles need 49 KiB; the rest keeps one CTA per SM
  cudaFuncSetAttribute(int8_mma_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  int8_mma_probe<<<sms, 128, smem, stream>>>(iters / 8 > 0 ? iters / 8 : 1, status);  // warm-up
  cudaEventRecord(e0, stream);
  int8_mma_probe<<<sms, 128, smem, stream>>>(iters, status);
  cudaEventRecord(e1, stream);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  int st = 0;
  cudaMemcpy(&st, status, 4, cudaMemcpyDeviceToHost);
  cudaFreeAsync(status, stream);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms_out = ms;
  *ops_out = (double)sms * iters * 4.0 * 2.0 * 128.0 * kProbeN * 32.0;
  if (st) return 5;
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
