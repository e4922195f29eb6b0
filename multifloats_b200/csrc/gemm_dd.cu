// Plain compensated DD matmul on the FP64 pipe (real and complex), plus the
// matrix-vector forms.
//
// Semantics (src/float64x2/matmul.inc:6-239): C(m,n) = A(m,k) * B(k,n),
// column-major, leading dimension = first extent, C overwritten.  For every
// output the reference runs mac_inl(A[i,p], B[p,j]) for p = 0..k-1 in order,
// renormalises after each full chunk of `renorm_interval` steps when more
// steps remain, and renormalises once at the end.  The kernels below keep the
// k-loop of each output sequential and reproduce that cadence, so results are
// bit-identical to matmuldd_mm / _mv / _vm.  The complex kernel reproduces the
// Fortran cdd_matmul_mm (fsrc/multifloats.fypp:2609-2621): four real products
// rr, ii, ri, ir accumulated side by side, then re = rr - ii, im = ri + ir with
// the DD operators.
//
// Tiling: a 256-thread CTA owns a BM x BN output tile; each thread owns a
// TM x TN register tile of (s_hi, s_lo) accumulators.  A and B k-slices of
// depth BK are staged in shared memory with cp.async (16-byte copies,
// zero-filled past the matrix edge) in a two-stage ring.  Bound: FP64 pipe,
// 13 FP64 instructions per MAC plus 6 per renormalisation.
#include "common.cuh"
#include "dd_device.cuh"
#include "gemm_tile.cuh"

namespace mfcuda {

using gtile::load_dd;
using gtile::cp_async_commit;
using gtile::cp_async_wait_all;

// ---------------------------------------------------------------------------
// Real GEMM: one 64 x 64 tile per CTA (4 x 4 outputs per thread).
// ---------------------------------------------------------------------------
constexpr int kThreads = gtile::kThreads;
constexpr int kTM = 4, kTN = 4;
constexpr int kBM = 16 * kTM, kBN = 16 * kTN;

template <bool ALIGNED>
__global__ void __launch_bounds__(kThreads, 2)
    gemm_dd_kernel(const double *__restrict__ A, const double *__restrict__ B,
                   double *__restrict__ C, int64_t M, int64_t K, int64_t N, int64_t ri) {
  __shared__ gtile::Smem sm;
  gtile::gemm_tile<kTM, kTN, ALIGNED>(A, B, C, M, K, N, ri, (int64_t)blockIdx.x * kBM,
                                      (int64_t)blockIdx.y * kBN, sm);
}

// ---------------------------------------------------------------------------
// Complex GEMM: one 32 x 32 tile per CTA (gtile::cgemm_tile).
// ---------------------------------------------------------------------------
constexpr int kCBM = gtile::kCBM, kCBN = gtile::kCBN;

template <bool ALIGNED>
__global__ void __launch_bounds__(kThreads, 2)
    cgemm_dd_kernel(const double *__restrict__ A, const double *__restrict__ B,
                    double *__restrict__ C, int64_t M, int64_t K, int64_t N, int64_t ri) {
  __shared__ gtile::CSmem sm;
  gtile::cgemm_tile<ALIGNED>(A, B, C, M, K, N, ri, (int64_t)blockIdx.x * kCBM, (int64_t)blockIdx.y * kCBN, sm);
}

// ---------------------------------------------------------------------------
// y(m) = A(m,k) x(k): one thread per row, k sequential (gaxpy_mv_panel,
// matmul.inc:47-88, A is the MAC's first operand).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) gemv_dd_kernel(const double *__restrict__ A,
                                                      const double *__restrict__ x,
                                                      double *__restrict__ y, int64_t M,
                                                      int64_t K, int64_t ri) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  double sh = 0.0, sl = 0.0;
  int64_t cnt = 0;
  for (int64_t p = 0; p < K; ++p) {
    double ah = A[2 * (p * M + i)], al = A[2 * (p * M + i) + 1];
    double xh = __ldg(x + 2 * p), xl = __ldg(x + 2 * p + 1);
    mfdev::mac(ah, al, xh, xl, sh, sl);
    if (ri > 0 && ++cnt == ri) {
      cnt = 0;
      if (p + 1 < K) mfdev::renorm(sh, sl);
    }
  }
  mfdev::renorm(sh, sl);
  y[2 * i] = sh;
  y[2 * i + 1] = sl;
}

// y(n) = x(k) B(k,n): one thread per column, k sequential, x is the MAC's
// first operand (vm_impl, matmul.inc:213-239).  B k-slices are staged in
// shared memory so the column reads coalesce.
constexpr int kVmP = 8;
__global__ void __launch_bounds__(256) gevm_dd_kernel(const double *__restrict__ x,
                                                      const double *__restrict__ B,
                                                      double *__restrict__ y, int64_t K,
                                                      int64_t N, int64_t ri) {
  __shared__ double2 Bs[256][kVmP + 1];
  const int t = threadIdx.x;
  const int64_t j0 = (int64_t)blockIdx.x * 256;
  const int64_t j = j0 + t;
  double sh = 0.0, sl = 0.0;
  int64_t cnt = 0;
  for (int64_t p0 = 0; p0 < K; p0 += kVmP) {
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kVmP; ++r) {
      int idx = t + r * 256;
      int col = idx / kVmP, pp = idx % kVmP;
      int64_t gj = j0 + col, gp = p0 + pp;
      double2 v = make_double2(0.0, 0.0);
      if (gj < N && gp < K) {
        const double *src = B + 2 * (gj * K + gp);
        v = make_double2(src[0], src[1]);
      }
      Bs[col][pp] = v;
    }
    __syncthreads();
    int pmax = (K - p0) < kVmP ? (int)(K - p0) : kVmP;
    for (int pp = 0; pp < pmax; ++pp) {
      int64_t p = p0 + pp;
      double xh = __ldg(x + 2 * p), xl = __ldg(x + 2 * p + 1);
      double2 b = Bs[t][pp];
      mfdev::mac(xh, xl, b.x, b.y, sh, sl);
      if (ri > 0 && ++cnt == ri) {
        cnt = 0;
        if (p + 1 < K) mfdev::renorm(sh, sl);
      }
    }
  }
  if (j < N) {
    mfdev::renorm(sh, sl);
    y[2 * j] = sh;
    y[2 * j + 1] = sl;
  }
}

static bool aligned16(const void *a, const void *b, const void *c) {
  return ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) |
           reinterpret_cast<uintptr_t>(c)) & 15) == 0;
}

static bool shape_ok(int64_t m, int64_t k, int64_t n, size_t elem) {
  return size_ok(m, elem) && size_ok(k, elem) && size_ok(n, elem) && mul_ok(m, k) &&
         mul_ok(k, n) && mul_ok(m, n) && size_ok(m * k, elem) && size_ok(k * n, elem) &&
         size_ok(m * n, elem);
}

// Output with k == 0: the reference finalises zero accumulators -> +0.
__global__ void zero_fill_kernel(double *p, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) p[i] = 0.0;
}
static int zero_fill(double *p, int64_t ndoubles, cudaStream_t s) {
  if (ndoubles == 0) return MFCUDA_OK;
  int64_t blocks = (ndoubles + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  zero_fill_kernel<<<(int)blocks, 256, 0, s>>>(p, ndoubles);
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

int gemm_dev(const float64x2 *a, const float64x2 *b, float64x2 *c, int64_t m, int64_t k,
             int64_t n, int64_t ri, cudaStream_t s) {
  if (!shape_ok(m, k, n, sizeof(float64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return MFCUDA_OK;
  if (!c || (k > 0 && (!a || !b))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  double *C = reinterpret_cast<double *>(c);
  if (k == 0) return zero_fill(C, 2 * m * n, s);
  const double *A = reinterpret_cast<const double *>(a);
  const double *B = reinterpret_cast<const double *>(b);
  int64_t gx = (m + kBM - 1) / kBM, gy = (n + kBN - 1) / kBN;
  if (gy > 65535) return MFCUDA_ERR_UNSUPPORTED;
  dim3 grid((unsigned)gx, (unsigned)gy);
  if (aligned16(a, b, c))
    gemm_dd_kernel<true><<<grid, kThreads, 0, s>>>(A, B, C, m, k, n, ri);
  else
    gemm_dd_kernel<false><<<grid, kThreads, 0, s>>>(A, B, C, m, k, n, ri);
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

int cgemm_dev(const complex64x2 *a, const complex64x2 *b, complex64x2 *c, int64_t m, int64_t k,
              int64_t n, int64_t ri, cudaStream_t s) {
  if (!shape_ok(m, k, n, sizeof(complex64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return MFCUDA_OK;
  if (!c || (k > 0 && (!a || !b))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  double *C = reinterpret_cast<double *>(c);
  if (k == 0) return zero_fill(C, 4 * m * n, s);
  const double *A = reinterpret_cast<const double *>(a);
  const double *B = reinterpret_cast<const double *>(b);
  int64_t gx = (m + kCBM - 1) / kCBM, gy = (n + kCBN - 1) / kCBN;
  if (gy > 65535) return MFCUDA_ERR_UNSUPPORTED;
  dim3 grid((unsigned)gx, (unsigned)gy);
  if (aligned16(a, b, c))
    cgemm_dd_kernel<true><<<grid, kThreads, 0, s>>>(A, B, C, m, k, n, ri);
  else
    cgemm_dd_kernel<false><<<grid, kThreads, 0, s>>>(A, B, C, m, k, n, ri);
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

int gemv_dev(const float64x2 *a, const float64x2 *x, float64x2 *y, int64_t m, int64_t k,
             int64_t ri, cudaStream_t s) {
  if (!shape_ok(m, k, 1, sizeof(float64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (m == 0) return MFCUDA_OK;
  if (!y || (k > 0 && (!a || !x))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  int64_t blocks = (m + 255) / 256;
  if (blocks > INT32_MAX) return MFCUDA_ERR_UNSUPPORTED;
  gemv_dd_kernel<<<(unsigned)blocks, 256, 0, s>>>(reinterpret_cast<const double *>(a),
                                                   reinterpret_cast<const double *>(x),
                                                   reinterpret_cast<double *>(y), m, k, ri);
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

int gevm_dev(const float64x2 *x, const float64x2 *b, float64x2 *y, int64_t k, int64_t n,
             int64_t ri, cudaStream_t s) {
  if (!shape_ok(1, k, n, sizeof(float64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (n == 0) return MFCUDA_OK;
  if (!y || (k > 0 && (!b || !x))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  int64_t blocks = (n + 255) / 256;
  if (blocks > INT32_MAX) return MFCUDA_ERR_UNSUPPORTED;
  gevm_dd_kernel<<<(unsigned)blocks, 256, 0, s>>>(reinterpret_cast<const double *>(x),
                                                   reinterpret_cast<const double *>(b),
                                                   reinterpret_cast<double *>(y), k, n, ri);
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

// ---- host-pointer (drop-in) forms -----------------------------------------
static int gemm_host(const float64x2 *a, const float64x2 *b, float64x2 *c, int64_t m, int64_t k,
                     int64_t n, int64_t ri) {
  if (!shape_ok(m, k, n, sizeof(float64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return MFCUDA_OK;
  if (!c || (k > 0 && (!a || !b))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  size_t ba = (size_t)(m * k) * sizeof(float64x2), bb = (size_t)(k * n) * sizeof(float64x2),
         bc = (size_t)(m * n) * sizeof(float64x2);
  size_t sz[4] = {ba, bb, bc, 0};
  Staging st;
  MF_TRY(staging_acquire(st, sz));
  auto *da = static_cast<float64x2 *>(st.buf[0]);
  auto *db = static_cast<float64x2 *>(st.buf[1]);
  auto *dc = static_cast<float64x2 *>(st.buf[2]);
  if (ba) MF_TRY_CUDA(cudaMemcpyAsync(da, a, ba, cudaMemcpyHostToDevice, st.stream));
  if (bb) MF_TRY_CUDA(cudaMemcpyAsync(db, b, bb, cudaMemcpyHostToDevice, st.stream));
  MF_TRY(gemm_dev(da, db, dc, m, k, n, ri, st.stream));
  MF_TRY_CUDA(cudaMemcpyAsync(c, dc, bc, cudaMemcpyDeviceToHost, st.stream));
  MF_TRY_CUDA(cudaStreamSynchronize(st.stream));
  return MFCUDA_OK;
}

static int cgemm_host(const complex64x2 *a, const complex64x2 *b, complex64x2 *c, int64_t m,
                      int64_t k, int64_t n, int64_t ri) {
  if (!shape_ok(m, k, n, sizeof(complex64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return MFCUDA_OK;
  if (!c || (k > 0 && (!a || !b))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  size_t ba = (size_t)(m * k) * sizeof(complex64x2), bb = (size_t)(k * n) * sizeof(complex64x2),
         bc = (size_t)(m * n) * sizeof(complex64x2);
  size_t sz[4] = {ba, bb, bc, 0};
  Staging st;
  MF_TRY(staging_acquire(st, sz));
  auto *da = static_cast<complex64x2 *>(st.buf[0]);
  auto *db = static_cast<complex64x2 *>(st.buf[1]);
  auto *dc = static_cast<complex64x2 *>(st.buf[2]);
  if (ba) MF_TRY_CUDA(cudaMemcpyAsync(da, a, ba, cudaMemcpyHostToDevice, st.stream));
  if (bb) MF_TRY_CUDA(cudaMemcpyAsync(db, b, bb, cudaMemcpyHostToDevice, st.stream));
  MF_TRY(cgemm_dev(da, db, dc, m, k, n, ri, st.stream));
  MF_TRY_CUDA(cudaMemcpyAsync(c, dc, bc, cudaMemcpyDeviceToHost, st.stream));
  MF_TRY_CUDA(cudaStreamSynchronize(st.stream));
  return MFCUDA_OK;
}

static int gemv_host(const float64x2 *a, const float64x2 *x, float64x2 *y, int64_t m, int64_t k,
                     int64_t ri) {
  if (!shape_ok(m, k, 1, sizeof(float64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (m == 0) return MFCUDA_OK;
  if (!y || (k > 0 && (!a || !x))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  size_t ba = (size_t)(m * k) * sizeof(float64x2), bx = (size_t)k * sizeof(float64x2),
         by = (size_t)m * sizeof(float64x2);
  size_t sz[4] = {ba, bx, by, 0};
  Staging st;
  MF_TRY(staging_acquire(st, sz));
  auto *da = static_cast<float64x2 *>(st.buf[0]);
  auto *dx = static_cast<float64x2 *>(st.buf[1]);
  auto *dy = static_cast<float64x2 *>(st.buf[2]);
  if (ba) MF_TRY_CUDA(cudaMemcpyAsync(da, a, ba, cudaMemcpyHostToDevice, st.stream));
  if (bx) MF_TRY_CUDA(cudaMemcpyAsync(dx, x, bx, cudaMemcpyHostToDevice, st.stream));
  MF_TRY(gemv_dev(da, dx, dy, m, k, ri, st.stream));
  MF_TRY_CUDA(cudaMemcpyAsync(y, dy, by, cudaMemcpyDeviceToHost, st.stream));
  MF_TRY_CUDA(cudaStreamSynchronize(st.stream));
  return MFCUDA_OK;
}

static int gevm_host(const float64x2 *x, const float64x2 *b, float64x2 *y, int64_t k, int64_t n,
                     int64_t ri) {
  if (!shape_ok(1, k, n, sizeof(float64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (n == 0) return MFCUDA_OK;
  if (!y || (k > 0 && (!b || !x))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  size_t bx = (size_t)k * sizeof(float64x2), bb = (size_t)(k * n) * sizeof(float64x2),
         by = (size_t)n * sizeof(float64x2);
  size_t sz[4] = {bx, bb, by, 0};
  Staging st;
  MF_TRY(staging_acquire(st, sz));
  auto *dx = static_cast<float64x2 *>(st.buf[0]);
  auto *db = static_cast<float64x2 *>(st.buf[1]);
  auto *dy = static_cast<float64x2 *>(st.buf[2]);
  if (bx) MF_TRY_CUDA(cudaMemcpyAsync(dx, x, bx, cudaMemcpyHostToDevice, st.stream));
  if (bb) MF_TRY_CUDA(cudaMemcpyAsync(db, b, bb, cudaMemcpyHostToDevice, st.stream));
  MF_TRY(gevm_dev(dx, db, dy, k, n, ri, st.stream));
  MF_TRY_CUDA(cudaMemcpyAsync(y, dy, by, cudaMemcpyDeviceToHost, st.stream));
  MF_TRY_CUDA(cudaStreamSynchronize(st.stream));
  return MFCUDA_OK;
}

}  // namespace mfcuda

extern "C" {

MULTIFLOATS_CUDA_API int mfcuda_matmuldd_mm(const float64x2 *a, const float64x2 *b, float64x2 *c,
                                            int64_t m, int64_t k, int64_t n, int64_t ri,
                                            void *stream) {
  return mfcuda::gemm_dev(a, b, c, m, k, n, ri, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_matmuldd_mv(const float64x2 *a, const float64x2 *x, float64x2 *y,
                                            int64_t m, int64_t k, int64_t ri, void *stream) {
  return mfcuda::gemv_dev(a, x, y, m, k, ri, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_matmuldd_vm(const float64x2 *x, const float64x2 *b, float64x2 *y,
                                            int64_t k, int64_t n, int64_t ri, void *stream) {
  return mfcuda::gevm_dev(x, b, y, k, n, ri, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_cmatmuldd_mm(const complex64x2 *a, const complex64x2 *b,
                                             complex64x2 *c, int64_t m, int64_t k, int64_t n,
                                             int64_t ri, void *stream) {
  return mfcuda::cgemm_dev(a, b, c, m, k, n, ri, mfcuda::as_stream(stream));
}

MULTIFLOATS_CUDA_API void matmuldd_mm(const float64x2 *a, const float64x2 *b, float64x2 *c,
                                      int64_t m, int64_t k, int64_t n, int64_t ri) {
  mfcuda::set_last_error(mfcuda::gemm_host(a, b, c, m, k, n, ri));
}
MULTIFLOATS_CUDA_API void matmuldd_mv(const float64x2 *a, const float64x2 *x, float64x2 *y,
                                      int64_t m, int64_t k, int64_t ri) {
  mfcuda::set_last_error(mfcuda::gemv_host(a, x, y, m, k, ri));
}
MULTIFLOATS_CUDA_API void matmuldd_vm(const float64x2 *x, const float64x2 *b, float64x2 *y,
                                      int64_t k, int64_t n, int64_t ri) {
  mfcuda::set_last_error(mfcuda::gevm_host(x, b, y, k, n, ri));
}
MULTIFLOATS_CUDA_API void matmulf64x2_mm(const float64x2 *a, const float64x2 *b, float64x2 *c,
                                         int64_t m, int64_t k, int64_t n, int64_t ri) {
  matmuldd_mm(a, b, c, m, k, n, ri);
}
MULTIFLOATS_CUDA_API void matmulf64x2_mv(const float64x2 *a, const float64x2 *x, float64x2 *y,
                                         int64_t m, int64_t k, int64_t ri) {
  matmuldd_mv(a, x, y, m, k, ri);
}
MULTIFLOATS_CUDA_API void matmulf64x2_vm(const float64x2 *x, const float64x2 *b, float64x2 *y,
                                         int64_t k, int64_t n, int64_t ri) {
  matmuldd_vm(x, b, y, k, n, ri);
}
MULTIFLOATS_CUDA_API void cmatmuldd_mm(const complex64x2 *a, const complex64x2 *b,
                                       complex64x2 *c, int64_t m, int64_t k, int64_t n,
                                       int64_t ri) {
  mfcuda::set_last_error(mfcuda::cgemm_host(a, b, c, m, k, n, ri));
}

}  // extern "C"
