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
