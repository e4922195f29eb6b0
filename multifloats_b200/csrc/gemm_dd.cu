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
#include <mutex>

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
// Matrix-vector forms.  Every output keeps the reference's sequential MAC over
// p = 0..k-1, so there is one dependency chain per output and only a few
// thousand of them; a CTA owns 32 outputs and splits each MAC
// (matmul.inc:6-19) in two:
//   * three producer warps stream the matrix through a 4-stage cp.async ring
//     (32 outputs x 32 k per stage) and compute the accumulator-independent
//     part of every MAC, p = ah*bh and q = fma(ah,bh,-p) + fma(ah,bl,al*bh),
//     into a double-buffered shared array;
//   * one warp runs the accumulator chain (two_sum of s_hi with p, then
//     s_lo += q + (aerr + berr)) and the renorm cadence, lane = output.
// The operations and their order per output are the reference's, so results
// are bit-identical; the producers and the chain hand over through
// __syncthreads once per stage.
// ---------------------------------------------------------------------------
constexpr int kGvN = 32, kGvK = 32, kGvStages = 4, kGvPitch = 33, kGvProd = 3;
constexpr int kGvThreads = 32 * (1 + kGvProd);
constexpr size_t kGvRingBytes = sizeof(double2) * kGvStages * kGvN * kGvPitch;
constexpr size_t kGvSmem = kGvRingBytes + sizeof(double2) * 2 * kGvK * kGvPitch;

template <int N>
__device__ __forceinline__ void cp_async_wait_n() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// The accumulator half of mac_inl for one output: p and q from the producers.
__device__ __forceinline__ void mac_chain(double p, double q, double &s_hi, double &s_lo) {
  double t = mfdev::add(s_hi, p);
  double bp = mfdev::sub(t, s_hi);
  double ap = mfdev::sub(t, bp);
  double aerr = mfdev::sub(s_hi, ap);
  double berr = mfdev::sub(p, bp);
  s_lo = mfdev::add(s_lo, mfdev::add(q, mfdev::add(aerr, berr)));
  s_hi = t;
}
// The accumulator-independent half: p = ah bh, q = e + cross (same operations as mac).
__device__ __forceinline__ double2 mac_terms(double ah, double al, double bh, double bl) {
  double p = mfdev::mul(ah, bh);
  double e = mfdev::fma_(ah, bh, -p);
  double cross = mfdev::fma_(ah, bl, mfdev::mul(al, bh));
  return make_double2(p, mfdev::add(e, cross));
}

// Runs the chain over stage st's terms (lane = output), renorm cadence as in
// the reference: after each full chunk of ri steps when more remain.  The
// MACs between two renorm points run as one branch-free loop, so the
// compiler can start a MAC's t = s_hi + p while the previous MAC's error
// terms are still in flight (same operations, same order).
__device__ __forceinline__ void chain_stage(const double2 *__restrict__ pq, int cmax, int64_t p0, int64_t K,
                                            int64_t ri, int lane, double &sh, double &sl, int64_t &cnt) {
  int c = 0;
  while (c < cmax) {
    const int run = ri > 0 ? (int)min((int64_t)(cmax - c), ri - cnt) : cmax - c;
    const double2 *v = pq + (size_t)c * kGvPitch + lane;
#pragma unroll 8
    for (int r = 0; r < run; ++r) mac_chain(v[r * kGvPitch].x, v[r * kGvPitch].y, sh, sl);
    c += run;
    if (ri > 0) {
      cnt += run;
      if (cnt == ri) {
        cnt = 0;
        if (p0 + c < K) mfdev::renorm(sh, sl);
      }
    }
  }
}

// y(m) = A(m,k) x(k) (gaxpy_mv_panel, matmul.inc:47-88; A is the MAC's first
// operand).  Producer warp w copies and evaluates the stage columns c with
// c % 3 == w - 1, lane l = row i0 + l (each copy instruction moves one
// 512-byte segment of column-major A; a thread reads only what it copied).
template <bool ALIGNED>
__global__ void __launch_bounds__(kGvThreads) gemv_dd_kernel(const double *__restrict__ A,
                                                             const double *__restrict__ x,
                                                             double *__restrict__ y, int64_t M,
                                                             int64_t K, int64_t ri) {
  extern __shared__ double2 smem_gv[];
  double2 *ring = smem_gv;                                   // [stage][k][row pitch]
  double2 *pq = smem_gv + (size_t)kGvStages * kGvK * kGvPitch;  // [2][k][row pitch]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t i = (int64_t)blockIdx.x * kGvN + lane;
  const bool row_ok = i < M;
  const int64_t nst = (K + kGvK - 1) / kGvK;
  const int w = warp - 1;  // producer index
  auto issue = [&](int64_t st) {
    if (st < nst) {
      double2 *dst = ring + (size_t)(st % kGvStages) * kGvK * kGvPitch;
      const int64_t p0 = st * kGvK;
      const double *src = A + 2 * ((p0 + w) * M + i);
#pragma unroll
      for (int c = w; c < kGvK; c += kGvProd, src += 2 * kGvProd * M)
        load_dd<ALIGNED>(&dst[c * kGvPitch + lane], src, row_ok && p0 + c < K, A);
    }
    cp_async_commit();
  };
  auto load_x = [&](int64_t st) {  // lane l: x[st * 32 + l] (zero past k), one stage ahead of use
    double2 v = make_double2(0.0, 0.0);
    const int64_t p = st * kGvK + lane;
    if (st < nst && p < K) {
      const double *xp = x + 2 * p;
      v = ALIGNED ? *reinterpret_cast<const double2 *>(xp) : make_double2(xp[0], xp[1]);
    }
    return v;
  };
  auto produce = [&](int64_t st, double2 xv) {  // terms of stage st into pq[st % 2]
    if (st >= nst) return;
    const int64_t p0 = st * kGvK;
    const int cmax = (K - p0) < kGvK ? (int)(K - p0) : kGvK;
    const double2 *src = ring + (size_t)(st % kGvStages) * kGvK * kGvPitch;
    double2 *out = pq + (size_t)(st & 1) * kGvK * kGvPitch;
#pragma unroll
    for (int c0 = 0; c0 < kGvK; c0 += kGvProd) {
      const int c = c0 + w;
      const double xh = __shfl_sync(0xffffffffu, xv.x, c & 31), xl = __shfl_sync(0xffffffffu, xv.y, c & 31);
      if (c < cmax) {
        const double2 av = src[c * kGvPitch + lane];
        out[c * kGvPitch + lane] = mac_terms(av.x, av.y, xh, xl);
      }
    }
  };
  double2 xnext = make_double2(0.0, 0.0);
  if (warp > 0) {
    for (int s0 = 0; s0 < kGvStages - 1; ++s0) issue(s0);
    const double2 x0 = load_x(0);
    xnext = load_x(1);
    cp_async_wait_n<kGvStages - 2>();  // stage 0 landed
    produce(0, x0);
  }
  __syncthreads();
  double sh = 0.0, sl = 0.0;
  int64_t cnt = 0;
  for (int64_t st = 0; st < nst; ++st) {
    if (warp == 0) {
      const int64_t p0 = st * kGvK;
      const int cmax = (K - p0) < kGvK ? (int)(K - p0) : kGvK;
      chain_stage(pq + (size_t)(st & 1) * kGvK * kGvPitch, cmax, p0, K, ri, lane, sh, sl, cnt);
    } else {
      issue(st + kGvStages - 1);        // into the slot of stage st - 1, consumed already
      const double2 xcur = xnext;
      xnext = load_x(st + 2);
      cp_async_wait_n<kGvStages - 2>();  // stage st + 1 landed
      produce(st + 1, xcur);
    }
    __syncthreads();
  }
  if (warp > 0) cp_async_wait_n<0>();
  if (warp == 0 && row_ok) {
    mfdev::renorm(sh, sl);
    y[2 * i] = sh;
    y[2 * i + 1] = sl;
  }
}

// y(n) = x(k) B(k,n) (vm_impl, matmul.inc:213-239; x is the MAC's first
// operand).  Producer warp w copies the stage's columns jj with
// jj % 3 == w - 1, lane l taking k = p0 + l (one 512-byte segment of
// column-major B per copy instruction), and evaluates exactly the entries it
// copied; the chain warp's lane j owns column j0 + j.
template <bool ALIGNED>
__global__ void __launch_bounds__(kGvThreads) gevm_dd_kernel(const double *__restrict__ x,
                                                             const double *__restrict__ B,
                                                             double *__restrict__ y, int64_t K,
                                                             int64_t N, int64_t ri) {
  extern __shared__ double2 smem_gv[];
  double2 *ring = smem_gv;                                   // [stage][column][k pitch]
  double2 *pq = smem_gv + (size_t)kGvStages * kGvN * kGvPitch;  // [2][k][column pitch]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t j0 = (int64_t)blockIdx.x * kGvN;
  const int64_t nst = (K + kGvK - 1) / kGvK;
  const int w = warp - 1;
  auto issue = [&](int64_t st) {
    if (st < nst) {
      double2 *dst = ring + (size_t)(st % kGvStages) * kGvN * kGvPitch;
      const int64_t p = st * kGvK + lane;
      const double *src = B + 2 * ((j0 + w) * K + p);
#pragma unroll
      for (int jj = w; jj < kGvN; jj += kGvProd, src += 2 * kGvProd * K)
        load_dd<ALIGNED>(&dst[jj * kGvPitch + lane], src, j0 + jj < N && p < K, B);
    }
    cp_async_commit();
  };
  auto load_x = [&](int64_t st) {  // lane l: x[st * 32 + l] (zero past k), one stage ahead of use
    double2 v = make_double2(0.0, 0.0);
    const int64_t p = st * kGvK + lane;
    if (st < nst && p < K) {
      const double *xp = x + 2 * p;
      v = ALIGNED ? *reinterpret_cast<const double2 *>(xp) : make_double2(xp[0], xp[1]);
    }
    return v;
  };
  auto produce = [&](int64_t st, double2 xv) {
    if (st >= nst) return;
    const int64_t p0 = st * kGvK;
    const int cmax = (K - p0) < kGvK ? (int)(K - p0) : kGvK;
    if (lane >= cmax) return;  // k = p0 + lane past the end: never read
    const double2 *src = ring + (size_t)(st % kGvStages) * kGvN * kGvPitch;
    double2 *out = pq + (size_t)(st & 1) * kGvK * kGvPitch;
#pragma unroll
    for (int jj = w; jj < kGvN; jj += kGvProd) {
      const double2 bv = src[jj * kGvPitch + lane];
      out[lane * kGvPitch + jj] = mac_terms(xv.x, xv.y, bv.x, bv.y);  // pitch 33: conflict-free
    }
  };
  double2 xnext = make_double2(0.0, 0.0);
  if (warp > 0) {
    for (int s0 = 0; s0 < kGvStages - 1; ++s0) issue(s0);
    const double2 x0 = load_x(0);
    xnext = load_x(1);
    cp_async_wait_n<kGvStages - 2>();
    produce(0, x0);
  }
  __syncthreads();
  double sh = 0.0, sl = 0.0;
  int64_t cnt = 0;
  for (int64_t st = 0; st < nst; ++st) {
    if (warp == 0) {
      const int64_t p0 = st * kGvK;
      const int cmax = (K - p0) < kGvK ? (int)(K - p0) : kGvK;
      chain_stage(pq + (size_t)(st & 1) * kGvK * kGvPitch, cmax, p0, K, ri, lane, sh, sl, cnt);
    } else {
      issue(st + kGvStages - 1);
      const double2 xcur = xnext;
      xnext = load_x(st + 2);
      cp_async_wait_n<kGvStages - 2>();
      produce(st + 1, xcur);
    }
    __syncthreads();
  }
  if (warp > 0) cp_async_wait_n<0>();
  const int64_t j = j0 + lane;
  if (warp == 0 && j < N) {
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

// dynamic shared memory above the 48 KB default, set once per process
static void gv_attrs() {
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute(gemv_dd_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGvSmem);
    cudaFuncSetAttribute(gemv_dd_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGvSmem);
    cudaFuncSetAttribute(gevm_dd_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGvSmem);
    cudaFuncSetAttribute(gevm_dd_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGvSmem);
  });
}

int gemv_dev(const float64x2 *a, const float64x2 *x, float64x2 *y, int64_t m, int64_t k,
             int64_t ri, cudaStream_t s) {
  if (!shape_ok(m, k, 1, sizeof(float64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (m == 0) return MFCUDA_OK;
  if (!y || (k > 0 && (!a || !x))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  int64_t blocks = (m + kGvN - 1) / kGvN;
  if (blocks > INT32_MAX) return MFCUDA_ERR_UNSUPPORTED;
  gv_attrs();
  const double *A = reinterpret_cast<const double *>(a), *X = reinterpret_cast<const double *>(x);
  double *Y = reinterpret_cast<double *>(y);
  if (aligned16(a, x, y))
    gemv_dd_kernel<true><<<(unsigned)blocks, kGvThreads, kGvSmem, s>>>(A, X, Y, m, k, ri);
  else
    gemv_dd_kernel<false><<<(unsigned)blocks, kGvThreads, kGvSmem, s>>>(A, X, Y, m, k, ri);
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

int gevm_dev(const float64x2 *x, const float64x2 *b, float64x2 *y, int64_t k, int64_t n,
             int64_t ri, cudaStream_t s) {
  if (!shape_ok(1, k, n, sizeof(float64x2))) return MFCUDA_ERR_INVALID_ARG;
  if (n == 0) return MFCUDA_OK;
  if (!y || (k > 0 && (!b || !x))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  int64_t blocks = (n + kGvN - 1) / kGvN;
  if (blocks > INT32_MAX) return MFCUDA_ERR_UNSUPPORTED;
  gv_attrs();
  const double *X = reinterpret_cast<const double *>(x), *Bm = reinterpret_cast<const double *>(b);
  double *Y = reinterpret_cast<double *>(y);
  if (aligned16(x, b, y))
    gevm_dd_kernel<true><<<(unsigned)blocks, kGvThreads, kGvSmem, s>>>(X, Bm, Y, k, n, ri);
  else
    gevm_dd_kernel<false><<<(unsigned)blocks, kGvThreads, kGvSmem, s>>>(X, Bm, Y, k, n, ri);
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
