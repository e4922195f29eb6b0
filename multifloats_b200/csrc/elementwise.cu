// Elementwise DD kernels: y[i] = f(x[i]) for f in exp, log, sin, cos, sqrt.
//
// Semantics: the Fortran elemental map (fsrc/multifloats.fypp:792-798,
// :1407-1412) calling expdd / logdd / sindd / cosdd / sqrtdd per element
// (src/float64x2/abi.inc:30-68).  Each element is independent: one thread per
// element in a grid-stride loop, one 16-byte vector load and one 16-byte
// vector store per element.  The bound is the FP64 pipe (a few hundred FP64
// instructions per element against 32 bytes of HBM traffic); sqrt is the
// exception and is HBM-bound.
#include "common.cuh"
#include "dd_device.cuh"

namespace mfcuda {

template <int OP>
__device__ __forceinline__ mfdev::dd apply(mfdev::dd x) {
  if constexpr (OP == MFCUDA_EXP) return mfdev::dd_exp(x);
  if constexpr (OP == MFCUDA_LOG) return mfdev::dd_log(x);
  if constexpr (OP == MFCUDA_SIN) return mfdev::dd_sin(x);
  if constexpr (OP == MFCUDA_COS) return mfdev::dd_cos(x);
  return mfdev::dd_sqrt(x);
}

// ALIGNED: x and y are 16-byte aligned, so limbs move as one double2.
template <int OP, bool ALIGNED>
__global__ void __launch_bounds__(256) unary_kernel(const double *__restrict__ x,
                                                    double *__restrict__ y, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    mfdev::dd v;
    if constexpr (ALIGNED) {
      double2 t = __ldcs(reinterpret_cast<const double2 *>(x) + i);
      v.hi = t.x;
      v.lo = t.y;
    } else {
      v.hi = x[2 * i];
      v.lo = x[2 * i + 1];
    }
    mfdev::dd r = apply<OP>(v);
    if constexpr (ALIGNED) {
      __stcs(reinterpret_cast<double2 *>(y) + i, make_double2(r.hi, r.lo));
    } else {
      y[2 * i] = r.hi;
      y[2 * i + 1] = r.lo;
    }
  }
}

template <int OP>
static int launch_unary(const double *x, double *y, int64_t n, cudaStream_t s) {
  if (n == 0) return MFCUDA_OK;
  const int threads = 256;
  // Grid: enough blocks to fill every SM several times; the grid-stride loop
  // covers the rest.
  int64_t want = (n + threads - 1) / threads;
  int64_t cap = (int64_t)sm_count() * 16;
  int blocks = (int)(want < cap ? want : cap);
  bool aligned = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
  if (aligned)
    unary_kernel<OP, true><<<blocks, threads, 0, s>>>(x, y, n);
  else
    unary_kernel<OP, false><<<blocks, threads, 0, s>>>(x, y, n);
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

int unary_dev(int op, const float64x2 *x, float64x2 *y, int64_t n, cudaStream_t s) {
  if (!size_ok(n, sizeof(float64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (n > 0 && (!x || !y)) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  const double *xd = reinterpret_cast<const double *>(x);
  double *yd = reinterpret_cast<double *>(y);
  switch (op) {
    case MFCUDA_EXP: return launch_unary<MFCUDA_EXP>(xd, yd, n, s);
    case MFCUDA_LOG: return launch_unary<MFCUDA_LOG>(xd, yd, n, s);
    case MFCUDA_SIN: return launch_unary<MFCUDA_SIN>(xd, yd, n, s);
    case MFCUDA_COS: return launch_unary<MFCUDA_COS>(xd, yd, n, s);
    case MFCUDA_SQRT: return launch_unary<MFCUDA_SQRT>(xd, yd, n, s);
    default: return MFCUDA_ERR_INVALID_ARG;
  }
}

// Host-pointer form: stage through the device, synchronous.
static int unary_host(int op, const float64x2 *x, float64x2 *y, int64_t n) {
  if (!size_ok(n, sizeof(float64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (n == 0) return MFCUDA_OK;
  if (!x || !y) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  size_t bytes = (size_t)n * sizeof(float64x2);
  size_t sz[4] = {bytes, 0, 0, 0};
  Staging st;
  MF_TRY(staging_acquire(st, sz));
  float64x2 *d = static_cast<float64x2 *>(st.buf[0]);
  MF_TRY_CUDA(cudaMemcpyAsync(d, x, bytes, cudaMemcpyHostToDevice, st.stream));
  MF_TRY(unary_dev(op, d, d, n, st.stream));
  MF_TRY_CUDA(cudaMemcpyAsync(y, d, bytes, cudaMemcpyDeviceToHost, st.stream));
  MF_TRY_CUDA(cudaStreamSynchronize(st.stream));
  return MFCUDA_OK;
}

}  // namespace mfcuda

extern "C" {

MULTIFLOATS_CUDA_API int mfcuda_unary_dd(int op, const float64x2 *x, float64x2 *y, int64_t n,
                                         void *stream) {
  return mfcuda::unary_dev(op, x, y, n, mfcuda::as_stream(stream));
}

#define MF_UNARY_DROPIN(NAME, OP)                                               \
  MULTIFLOATS_CUDA_API void NAME(const float64x2 *x, float64x2 *y, int64_t n) { \
    mfcuda::set_last_error(mfcuda::unary_host(OP, x, y, n));                     \
  }
MF_UNARY_DROPIN(expdd_array, MFCUDA_EXP)
MF_UNARY_DROPIN(logdd_array, MFCUDA_LOG)
MF_UNARY_DROPIN(sindd_array, MFCUDA_SIN)
MF_UNARY_DROPIN(cosdd_array, MFCUDA_COS)
MF_UNARY_DROPIN(sqrtdd_array, MFCUDA_SQRT)
#undef MF_UNARY_DROPIN

}  // extern "C"
