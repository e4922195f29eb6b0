// One output tile of the plain compensated DD matmul (src/float64x2/matmul.inc:6-39
// semantics: per output, the MAC over p = 0..k-1 in order, renormalised after
// each full chunk of `ri` steps when more remain and once at the end), shared
// by the single-problem kernel and the grouped (batched) kernel.
//
// A 256-thread CTA owns a (16 TM) x (16 TN) tile; thread t owns rows
// tx + 16 i (i < TM) and columns ty + 16 j (j < TN), tx = t % 16, ty = t / 16.
// A and B k-slices of depth 8 go through a two-stage cp.async ring in shared
// memory (zero-filled past the edges).
#pragma once
#include "dd_device.cuh"

namespace mfcuda {
namespace gtile {

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// 16-byte async copy; src_bytes = 0 zero-fills the destination.
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes));
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// Copy one DD (16 bytes) or zero-fill it.  `safe` is an in-bounds address
// (the matrix base) handed to the copy when nothing is read.
template <bool ALIGNED>
__device__ __forceinline__ void load_dd(double2 *dst, const double *src, bool valid,
                                        const double *safe) {
  if constexpr (ALIGNED) {
    cp_async16(dst, valid ? src : safe, valid ? 16 : 0);
  } else {
    double *d = reinterpret_cast<double *>(dst);
    cp_async8(d, valid ? src : safe, valid ? 8 : 0);
    cp_async8(d + 1, valid ? src + 1 : safe, valid ? 8 : 0);
  }
}


constexpr int kThreads = 256;
constexpr int kBK = 8;
constexpr int kBMax = 64;  // largest tile edge (TM, TN <= 4)

// Shared staging of the largest tile; smaller tiles use the first rows.
struct Smem {
  double2 A[2][kBK][kBMax];
  double2 B[2][kBK][kBMax];
};

template <int TM, int TN, bool ALIGNED>
__device__ __forceinline__ void gemm_tile(const double *__restrict__ A, const double *__restrict__ B,
                                          double *__restrict__ C, int64_t M, int64_t K, int64_t N,
                                          int64_t ri, int64_t m0, int64_t n0, Smem &sm) {
  constexpr int BM = 16 * TM, BN = 16 * TN;
  const int t = threadIdx.x;
  const int tx = t % 16, ty = t / 16;

  double s_hi[TM][TN], s_lo[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) s_hi[i][j] = s_lo[i][j] = 0.0;

  auto issue = [&](int stage, int64_t k0) {
#pragma unroll
    for (int idx = t; idx < kBK * BM; idx += kThreads) {
      int row = idx % BM, kk = idx / BM;
      int64_t gi = m0 + row, gk = k0 + kk;
      bool v = gi < M && gk < K;
      load_dd<ALIGNED>(&sm.A[stage][kk][row], A + 2 * (gk * M + gi), v, A);
    }
#pragma unroll
    for (int idx = t; idx < kBK * BN; idx += kThreads) {
      int kk = idx % kBK, col = idx / kBK;
      int64_t gj = n0 + col, gk = k0 + kk;
      bool v = gj < N && gk < K;
      load_dd<ALIGNED>(&sm.B[stage][kk][col], B + 2 * (gj * K + gk), v, B);
    }
    cp_async_commit();
  };

  const int64_t ntiles = (K + kBK - 1) / kBK;
  int64_t cnt = 0;
  if (ntiles > 0) issue(0, 0);
  for (int64_t kt = 0; kt < ntiles; ++kt) {
    const int stage = (int)(kt & 1);
    cp_async_wait_all();
    __syncthreads();
    if (kt + 1 < ntiles) issue(stage ^ 1, (kt + 1) * kBK);
    const int64_t k0 = kt * kBK;
    const int kmax = (K - k0) < kBK ? (int)(K - k0) : kBK;
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      if (kk < kmax) {
        double ah[TM], al[TM], bh[TN], bl[TN];
#pragma unroll
        for (int i = 0; i < TM; ++i) {
          double2 v = sm.A[stage][kk][tx + 16 * i];
          ah[i] = v.x;
          al[i] = v.y;
        }
#pragma unroll
        for (int j = 0; j < TN; ++j) {
          double2 v = sm.B[stage][kk][ty + 16 * j];
          bh[j] = v.x;
          bl[j] = v.y;
        }
#pragma unroll
        for (int j = 0; j < TN; ++j)
#pragma unroll
          for (int i = 0; i < TM; ++i) mfdev::mac(ah[i], al[i], bh[j], bl[j], s_hi[i][j], s_lo[i][j]);
        if (ri > 0) {
          if (++cnt == ri) {
            cnt = 0;
            if (k0 + kk + 1 < K) {
#pragma unroll
              for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) mfdev::renorm(s_hi[i][j], s_lo[i][j]);
            }
          }
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < TN; ++j) {
    int64_t gj = n0 + ty + 16 * j;
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      int64_t gi = m0 + tx + 16 * i;
      double h = s_hi[i][j], l = s_lo[i][j];
      mfdev::renorm(h, l);
      if (gi < M && gj < N) {
        double *dst = C + 2 * (gj * M + gi);
        if constexpr (ALIGNED) {
          *reinterpret_cast<double2 *>(dst) = make_double2(h, l);
        } else {
          dst[0] = h;
          dst[1] = l;
        }
      }
    }
  }
}


// ---------------------------------------------------------------------------
// One 32 x 32 output tile of the complex product (the Fortran cdd_matmul_mm
// composition, fsrc/multifloats.fypp:2609-2621): each thread owns a 2 x 2
// complex tile with four real accumulators per output (rr, ii, ri, ir), each
// run with the real MAC and renorm cadence, then re = rr - ii, im = ri + ir
// with the DD operators.
// ---------------------------------------------------------------------------
constexpr int kCTM = 2, kCTN = 2;
constexpr int kCBM = 16 * kCTM, kCBN = 16 * kCTN, kCBK = kBK;

struct CSmem {
  double2 A[2][kCBK][kCBM][2];
  double2 B[2][kCBK][kCBN][2];
};

template <bool ALIGNED>
__device__ __forceinline__ void cgemm_tile(const double *__restrict__ A, const double *__restrict__ B,
                                           double *__restrict__ C, int64_t M, int64_t K, int64_t N,
                                           int64_t ri, int64_t m0, int64_t n0, CSmem &sm) {
  // complex element = 4 doubles = two double2 (re, im)
  auto &As = sm.A;
  auto &Bs = sm.B;
  const int t = threadIdx.x;
  const int tx = t % 16, ty = t / 16;

  double s_hi[kCTM][kCTN][4], s_lo[kCTM][kCTN][4];
#pragma unroll
  for (int i = 0; i < kCTM; ++i)
#pragma unroll
    for (int j = 0; j < kCTN; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) s_hi[i][j][q] = s_lo[i][j][q] = 0.0;

  auto issue = [&](int stage, int64_t k0) {
    // A: kCBK x kCBM complex = 256 complex = 512 DD; each thread copies 2 DD.
#pragma unroll
    for (int r = 0; r < (kCBK * kCBM * 2) / kThreads; ++r) {
      int idx = t + r * kThreads;
      int part = idx & 1, e = idx >> 1;
      int row = e % kCBM, kk = e / kCBM;
      int64_t gi = m0 + row, gk = k0 + kk;
      bool v = gi < M && gk < K;
      load_dd<ALIGNED>(&As[stage][kk][row][part], A + 4 * (gk * M + gi) + 2 * part, v, A);
    }
#pragma unroll
    for (int r = 0; r < (kCBK * kCBN * 2) / kThreads; ++r) {
      int idx = t + r * kThreads;
      int part = idx & 1, e = idx >> 1;
      int kk = e % kCBK, col = e / kCBK;
      int64_t gj = n0 + col, gk = k0 + kk;
      bool v = gj < N && gk < K;
      load_dd<ALIGNED>(&Bs[stage][kk][col][part], B + 4 * (gj * K + gk) + 2 * part, v, B);
    }
    cp_async_commit();
  };

  const int64_t ntiles = (K + kCBK - 1) / kCBK;
  int64_t cnt = 0;
  if (ntiles > 0) issue(0, 0);
  for (int64_t kt = 0; kt < ntiles; ++kt) {
    const int stage = (int)(kt & 1);
    cp_async_wait_all();
    __syncthreads();
    if (kt + 1 < ntiles) issue(stage ^ 1, (kt + 1) * kCBK);
    const int64_t k0 = kt * kCBK;
    const int kmax = (K - k0) < kCBK ? (int)(K - k0) : kCBK;
#pragma unroll
    for (int kk = 0; kk < kCBK; ++kk) {
      if (kk < kmax) {
        double2 ar[kCTM], ai[kCTM], br[kCTN], bi[kCTN];
#pragma unroll
        for (int i = 0; i < kCTM; ++i) {
          ar[i] = As[stage][kk][tx + 16 * i][0];
          ai[i] = As[stage][kk][tx + 16 * i][1];
        }
#pragma unroll
        for (int j = 0; j < kCTN; ++j) {
          br[j] = Bs[stage][kk][ty + 16 * j][0];
          bi[j] = Bs[stage][kk][ty + 16 * j][1];
        }
#pragma unroll
        for (int j = 0; j < kCTN; ++j)
#pragma unroll
          for (int i = 0; i < kCTM; ++i) {
            mfdev::mac(ar[i].x, ar[i].y, br[j].x, br[j].y, s_hi[i][j][0], s_lo[i][j][0]);
            mfdev::mac(ai[i].x, ai[i].y, bi[j].x, bi[j].y, s_hi[i][j][1], s_lo[i][j][1]);
            mfdev::mac(ar[i].x, ar[i].y, bi[j].x, bi[j].y, s_hi[i][j][2], s_lo[i][j][2]);
            mfdev::mac(ai[i].x, ai[i].y, br[j].x, br[j].y, s_hi[i][j][3], s_lo[i][j][3]);
          }
        if (ri > 0) {
          if (++cnt == ri) {
            cnt = 0;
            if (k0 + kk + 1 < K) {
#pragma unroll
              for (int i = 0; i < kCTM; ++i)
#pragma unroll
                for (int j = 0; j < kCTN; ++j)
#pragma unroll
                  for (int q = 0; q < 4; ++q) mfdev::renorm(s_hi[i][j][q], s_lo[i][j][q]);
            }
          }
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < kCTN; ++j) {
    int64_t gj = n0 + ty + 16 * j;
#pragma unroll
    for (int i = 0; i < kCTM; ++i) {
      int64_t gi = m0 + tx + 16 * i;
      mfdev::dd p[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double h = s_hi[i][j][q], l = s_lo[i][j][q];
        mfdev::renorm(h, l);
        p[q] = mfdev::make(h, l);
      }
      mfdev::dd re = mfdev::dd_sub(p[0], p[1]);
      mfdev::dd im = mfdev::dd_add(p[2], p[3]);
      if (gi < M && gj < N) {
        double *dst = C + 4 * (gj * M + gi);
        if constexpr (ALIGNED) {
          reinterpret_cast<double2 *>(dst)[0] = make_double2(re.hi, re.lo);
          reinterpret_cast<double2 *>(dst)[1] = make_double2(im.hi, im.lo);
        } else {
          dst[0] = re.hi;
          dst[1] = re.lo;
          dst[2] = im.hi;
          dst[3] = im.lo;
        }
      }
    }
  }
}

}  // namespace gtile
}  // namespace mfcuda
