// Elementwise DD kernels: y[i] = f(x[i]) for f in exp, log, sin, cos, sqrt,
// exp2, log2, log10, plus the fused sincos and the complex exp / cexpi maps.
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
  if constexpr (OP == MFCUDA_EXP2) return mfdev::dd_exp2(x);
  if constexpr (OP == MFCUDA_LOG2) return mfdev::dd_log2(x);
  if constexpr (OP == MFCUDA_LOG10) return mfdev::dd_log10(x);
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
    case MFCUDA_EXP2: return launch_unary<MFCUDA_EXP2>(xd, yd, n, s);
    case MFCUDA_LOG2: return launch_unary<MFCUDA_LOG2>(xd, yd, n, s);
    case MFCUDA_LOG10: return launch_unary<MFCUDA_LOG10>(xd, yd, n, s);
    default: return MFCUDA_ERR_INVALID_ARG;
  }
}

// ---- two-output and complex maps -------------------------------------------
// KIND 0: sincos   x (DD) -> s, c (DD arrays)           sincosdd, abi.inc:123-125
// KIND 1: cexpi    x (DD) -> z = cos x + i sin x        cexpidd, abi.inc:226-229
// KIND 2: cexp     z (complex DD) -> exp(z)             cexpdd, complex64x2/abi.inc:189
// Loads and stores are 16-byte vectors when every pointer is 16-byte aligned.
template <int KIND, bool ALIGNED>
__global__ void __launch_bounds__(256) pair_kernel(const double *__restrict__ x, double *__restrict__ y0,
                                                   double *__restrict__ y1, int64_t n) {
  auto ld = [](const double *p) -> mfdev::dd {
    if constexpr (ALIGNED) {
      double2 t = __ldcs(reinterpret_cast<const double2 *>(p));
      return mfdev::make(t.x, t.y);
    }
    return mfdev::make(p[0], p[1]);
  };
  auto st = [](double *p, mfdev::dd v) {
    if constexpr (ALIGNED) {
      __stcs(reinterpret_cast<double2 *>(p), make_double2(v.hi, v.lo));
    } else {
      p[0] = v.hi;
      p[1] = v.lo;
    }
  };
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    mfdev::dd a, b;
    if constexpr (KIND == 2) {
      mfdev::dd re = ld(x + 4 * i), im = ld(x + 4 * i + 2);
      mfdev::dd_cexp(re, im, a, b);
      st(y0 + 4 * i, a);
      st(y0 + 4 * i + 2, b);
    } else {
      mfdev::dd_sincos(ld(x + 2 * i), a, b);  // a = sin, b = cos
      if constexpr (KIND == 0) {
        st(y0 + 2 * i, a);
        st(y1 + 2 * i, b);
      } else {
        st(y0 + 4 * i, b);
        st(y0 + 4 * i + 2, a);
      }
    }
  }
}

template <int KIND>
static int launch_pair(const double *x, double *y0, double *y1, int64_t n, cudaStream_t s) {
  if (n == 0) return MFCUDA_OK;
  const int threads = 256;
  int64_t want = (n + threads - 1) / threads, cap = (int64_t)sm_count() * 16;
  int blocks = (int)(want < cap ? want : cap);
  bool aligned = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y0) |
                   reinterpret_cast<uintptr_t>(y1)) & 15) == 0;
  if (aligned)
    pair_kernel<KIND, true><<<blocks, threads, 0, s>>>(x, y0, y1, n);
  else
    pair_kernel<KIND, false><<<blocks, threads, 0, s>>>(x, y0, y1, n);
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

int pair_dev(int kind, const void *x, void *y0, void *y1, int64_t n, cudaStream_t s) {
  const size_t in_elem = kind == 2 ? sizeof(complex64x2) : sizeof(float64x2);
  if (!size_ok(n, in_elem) || !size_ok(n, sizeof(complex64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (n > 0 && (!x || !y0 || (kind == 0 && !y1))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  const double *xd = static_cast<const double *>(x);
  double *a = static_cast<double *>(y0), *b = static_cast<double *>(kind == 0 ? y1 : y0);
  switch (kind) {
    case 0: return launch_pair<0>(xd, a, b, n, s);
    case 1: return launch_pair<1>(xd, a, b, n, s);
    case 2: return launch_pair<2>(xd, a, b, n, s);
    default: return MFCUDA_ERR_INVALID_ARG;
  }
}

static int pair_host(int kind, const void *x, void *y0, void *y1, int64_t n) {
  const size_t in_elem = kind == 2 ? sizeof(complex64x2) : sizeof(float64x2);
  if (!size_ok(n, sizeof(complex64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (n == 0) return MFCUDA_OK;
  if (!x || !y0 || (kind == 0 && !y1)) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  const size_t bin = (size_t)n * in_elem;
  const size_t b0 = (size_t)n * (kind == 0 ? sizeof(float64x2) : sizeof(complex64x2));
  const size_t b1 = kind == 0 ? (size_t)n * sizeof(float64x2) : 0;
  size_t sz[4] = {bin, b0, b1, 0};
  Staging st;
  MF_TRY(staging_acquire(st, sz));
  MF_TRY_CUDA(cudaMemcpyAsync(st.buf[0], x, bin, cudaMemcpyHostToDevice, st.stream));
  MF_TRY(pair_dev(kind, st.buf[0], st.buf[1], st.buf[2], n, st.stream));
  MF_TRY_CUDA(cudaMemcpyAsync(y0, st.buf[1], b0, cudaMemcpyDeviceToHost, st.stream));
  if (b1) MF_TRY_CUDA(cudaMemcpyAsync(y1, st.buf[2], b1, cudaMemcpyDeviceToHost, st.stream));
  MF_TRY_CUDA(cudaStreamSynchronize(st.stream));
  return MFCUDA_OK;
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
MF_UNARY_DROPIN(exp2dd_array, MFCUDA_EXP2)
MF_UNARY_DROPIN(log2dd_array, MFCUDA_LOG2)
MF_UNARY_DROPIN(log10dd_array, MFCUDA_LOG10)
#undef MF_UNARY_DROPIN

MULTIFLOATS_CUDA_API int mfcuda_sincos_dd(const float64x2 *x, float64x2 *s, float64x2 *c, int64_t n,
                                          void *stream) {
  return mfcuda::pair_dev(0, x, s, c, n, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_cexpi_dd(const float64x2 *x, complex64x2 *z, int64_t n, void *stream) {
  return mfcuda::pair_dev(1, x, z, nullptr, n, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_cexp_dd(const complex64x2 *z, complex64x2 *w, int64_t n, void *stream) {
  return mfcuda::pair_dev(2, z, w, nullptr, n, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API void sincosdd_array(const float64x2 *x, float64x2 *s, float64x2 *c, int64_t n) {
  mfcuda::set_last_error(mfcuda::pair_host(0, x, s, c, n));
}
MULTIFLOATS_CUDA_API void cexpidd_array(const float64x2 *x, complex64x2 *z, int64_t n) {
  mfcuda::set_last_error(mfcuda::pair_host(1, x, z, nullptr, n));
}
MULTIFLOATS_CUDA_API void cexpdd_array(const complex64x2 *z, complex64x2 *w, int64_t n) {
  mfcuda::set_last_error(mfcuda::pair_host(2, z, w, nullptr, n));
}

}  // extern "C"
