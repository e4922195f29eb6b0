// BLAS-style shims over double-double matrices: DGEMM and DTRSM argument
// semantics (transposition, alpha / beta, leading dimensions, unit diagonal)
// as in test/integration/blas/wgemm.f90 and wtrsm.f90, with results
// bit-identical to those Fortran loops run with the DD operators
// (include/multifloats/float64x2.h:203-311; the Fortran operators are the same,
// test/integration/crosscheck.cc).
//
// wgemm: every output is one sequential chain over l = 1..k in the Fortran's
// order, so the kernel is a 64 x 64 output tile per CTA (4 x 4 per thread)
// over a two-stage cp.async ring of k-slices, like the plain matmul, with the
// wgemm MAC instead of mac_inl:
//   A not transposed (wgemm.f90:68-84, 106-122): c := beta c (or 0, or c when
//     beta is one), then c := c + (alpha b_lj) a_il; alpha b_lj is formed once
//     per staged element of B in shared memory;
//   A transposed (wgemm.f90:86-99, 124-137): t := sum_l a_li b_lj from zero,
//     then c := alpha t (beta zero) or alpha t + beta c.
//
// wtrsm: each column of B (left side) or row of B (right side) is an
// independent triangular recurrence.  In six of the eight (side, uplo, trans)
// cases every element receives its updates in the order its pivots are
// finalised, which a blocked right-looking solve reproduces exactly: a CTA
// owns 16 vectors, walks the pivots in blocks of 32 (diagonal block solved
// pivot by pivot in shared memory, then the block applied to the remaining
// elements chunk by chunk) and applies the same per-element operations in the
// same order, including the zero tests that skip an update.  In the other two
// (left with A^T lower, right with A lower) each element's updates run in the
// opposite order, so those run as one sequential chain per vector.
#include <cstring>

#include "common.cuh"
#include "dd_device.cuh"
#include "gemm_tile.cuh"

// xerbla from the caller's LAPACK / BLAS, when one is linked (the reference
// shims call it on an invalid argument).
extern "C" void xerbla_(const char *srname, const int *info, size_t len)
    __attribute__((weak, visibility("default")));

namespace mfcuda {
namespace {

using mfdev::dd;
using mfdev::dd_add;
using mfdev::dd_div;
using mfdev::dd_mul;
using mfdev::dd_sub;

// ---- argument logic (host) ---------------------------------------------------
inline char up(char c) { return (c >= 'a' && c <= 'z') ? static_cast<char>(c - 32) : c; }
inline bool lsame(char a, char b) { return up(a) == up(b); }
inline int64_t max1(int64_t x) { return x > 1 ? x : 1; }
// DD == (h, 0) compares both limbs (fsrc/multifloats.fypp:2920-2928).
inline bool dd_is(const float64x2 *v, double h) {
  const double *p = reinterpret_cast<const double *>(v);
  return p[0] == h && p[1] == 0.0;
}
inline dd to_dd(const float64x2 *v) {
  const double *p = reinterpret_cast<const double *>(v);
  dd r;
  r.hi = p[0];
  r.lo = p[1];
  return r;
}

// wgemm.f90:16-48: the info code handed to xerbla, 0 when the arguments are valid.
int wgemm_info(char ta, char tb, int64_t m, int64_t n, int64_t k, int64_t lda, int64_t ldb,
               int64_t ldc) {
  const bool nota = lsame(ta, 'N'), notb = lsame(tb, 'N');
  const int64_t nrowa = nota ? m : k, nrowb = notb ? k : n;
  if (!nota && !lsame(ta, 'C') && !lsame(ta, 'T')) return 1;
  if (!notb && !lsame(tb, 'C') && !lsame(tb, 'T')) return 2;
  if (m < 0) return 3;
  if (n < 0) return 4;
  if (k < 0) return 5;
  if (lda < max1(nrowa)) return 8;
  if (ldb < max1(nrowb)) return 10;
  if (ldc < max1(m)) return 13;
  return 0;
}

// wtrsm.f90:16-44.
int wtrsm_info(char side, char uplo, char ta, char diag, int64_t m, int64_t n, int64_t lda,
               int64_t ldb) {
  const bool lside = lsame(side, 'L'), upper = lsame(uplo, 'U');
  const int64_t nrowa = lside ? m : n;
  if (!lside && !lsame(side, 'R')) return 1;
  if (!upper && !lsame(uplo, 'L')) return 2;
  if (!lsame(ta, 'N') && !lsame(ta, 'T') && !lsame(ta, 'C')) return 3;
  if (!lsame(diag, 'U') && !lsame(diag, 'N')) return 4;
  if (m < 0) return 5;
  if (n < 0) return 6;
  if (lda < max1(nrowa)) return 9;
  if (ldb < max1(m)) return 11;
  return 0;
}

// A rows x cols column-major operand with leading dimension ld addressable in
// 64-bit element and byte counts.
bool span_ok(int64_t ld, int64_t cols) {
  return mul_ok(ld, cols) && size_ok(ld * cols, sizeof(float64x2));
}

// ---- device helpers -----------------------------------------------------------
__device__ __forceinline__ dd ld_dd(const double *p) {
  dd r;
  r.hi = p[0];
  r.lo = p[1];
  return r;
}
template <bool ALIGNED>
__device__ __forceinline__ dd ld_dd_a(const double *p) {
  if constexpr (ALIGNED) {
    double2 v = *reinterpret_cast<const double2 *>(p);
    dd r;
    r.hi = v.x;
    r.lo = v.y;
    return r;
  } else {
    return ld_dd(p);
  }
}
template <bool ALIGNED>
__device__ __forceinline__ void st_dd(double *p, dd v) {
  if constexpr (ALIGNED) {
    *reinterpret_cast<double2 *>(p) = make_double2(v.hi, v.lo);
  } else {
    p[0] = v.hi;
    p[1] = v.lo;
  }
}
__device__ __forceinline__ bool is_zero(dd v) { return v.hi == 0.0 && v.lo == 0.0; }
__device__ __forceinline__ dd dd0() { return mfdev::make(0.0, 0.0); }

// ---- scaling pass: C := beta C, or C := 0 (wgemm.f90:50-65, wtrsm.f90:46-53) --
__global__ void scale_kernel(double *__restrict__ C, int64_t ldc, int64_t M, int64_t N, dd beta,
                             int zero) {
  const int64_t total = M * N;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % M, j = e / M;
    double *p = C + 2 * (i + j * ldc);
    dd v = zero ? dd0() : dd_mul(beta, ld_dd(p));
    p[0] = v.hi;
    p[1] = v.lo;
  }
}

int launch_scale(double *C, int64_t ldc, int64_t M, int64_t N, dd beta, int zero, cudaStream_t s) {
  const int64_t total = M * N;
  if (total == 0) return MFCUDA_OK;
  int64_t blocks = (total + 255) / 256;
  const int64_t cap = 8LL * sm_count();
  if (blocks > cap) blocks = cap;
  scale_kernel<<<(unsigned)blocks, 256, 0, s>>>(C, ldc, M, N, beta, zero);
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

// ---- wgemm tile kernel ---------------------------------------------------------
constexpr int kWThreads = 256;
constexpr int kWTile = 64;  // 16 x 4 outputs per tile edge
constexpr int kWK = gtile::kBK;
enum { BETA_ZERO = 0, BETA_ONE = 1, BETA_OTHER = 2 };

// The 16 accumulator chains of a thread use the branch-free operator forms so
// that the compiler interleaves them.  Registers: the dot form keeps one CTA
// per SM with the full register file; the C-update form runs two CTAs per SM at
// <= 128 registers (measured on B200 at 2048^3 and 4096^3).
template <bool TA, bool TB, bool ALIGNED>
__global__ void __launch_bounds__(kWThreads, TA ? 1 : 2)
    wgemm_kernel(const double *__restrict__ A, int64_t lda, const double *__restrict__ B,
                 int64_t ldb, double *__restrict__ C, int64_t ldc, int64_t M, int64_t N, int64_t K,
                 dd alpha, dd beta, int beta_mode) {
  __shared__ __align__(16) gtile::Smem sm;
  const int t = threadIdx.x, tx = t % 16, ty = t / 16;
  const int64_t m0 = (int64_t)blockIdx.x * kWTile, n0 = (int64_t)blockIdx.y * kWTile;

  dd acc[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      acc[i][j] = dd0();
      if constexpr (!TA) {  // C := beta C before the k loop
        const int64_t gi = m0 + tx + 16 * i, gj = n0 + ty + 16 * j;
        if (beta_mode != BETA_ZERO && gi < M && gj < N) {
          dd c = ld_dd_a<ALIGNED>(C + 2 * (gi + gj * ldc));
          acc[i][j] = beta_mode == BETA_ONE ? c : dd_mul(beta, c);
        }
      }
    }

  auto issue = [&](int stage, int64_t k0) {
#pragma unroll
    for (int idx = t; idx < kWK * kWTile; idx += kWThreads) {
      // logical A(i, l): element (i, l) of op(A); lanes run along the contiguous index
      const int row = TA ? idx / kWK : idx % kWTile, kk = TA ? idx % kWK : idx / kWTile;
      const int64_t gi = m0 + row, gk = k0 + kk;
      const bool v = gi < M && gk < K;
      const double *src = TA ? A + 2 * (gk + gi * lda) : A + 2 * (gi + gk * lda);
      gtile::load_dd<ALIGNED>(&sm.A[stage][kk][row], src, v, A);
    }
#pragma unroll
    for (int idx = t; idx < kWK * kWTile; idx += kWThreads) {
      const int col = TB ? idx % kWTile : idx / kWK, kk = TB ? idx / kWTile : idx % kWK;
      const int64_t gj = n0 + col, gk = k0 + kk;
      const bool v = gj < N && gk < K;
      const double *src = TB ? B + 2 * (gj + gk * ldb) : B + 2 * (gk + gj * ldb);
      gtile::load_dd<ALIGNED>(&sm.B[stage][kk][col], src, v, B);
    }
    gtile::cp_async_commit();
  };

  const int64_t ntiles = (K + kWK - 1) / kWK;
  if (ntiles > 0) issue(0, 0);
  for (int64_t kt = 0; kt < ntiles; ++kt) {
    const int stage = (int)(kt & 1);
    gtile::cp_async_wait_all();
    __syncthreads();
    if (kt + 1 < ntiles) issue(stage ^ 1, (kt + 1) * kWK);
    if constexpr (!TA) {  // temp = alpha * b(l, j), once per staged element
#pragma unroll
      for (int idx = t; idx < kWK * kWTile; idx += kWThreads) {
        double2 &e = sm.B[stage][idx % kWK][idx / kWK];
        dd v = dd_mul(alpha, mfdev::make(e.x, e.y));
        e = make_double2(v.hi, v.lo);
      }
      __syncthreads();
    }
    const int64_t k0 = kt * kWK;
    const int kmax = (K - k0) < kWK ? (int)(K - k0) : kWK;
#pragma unroll
    for (int kk = 0; kk < kWK; ++kk) {
      if (kk < kmax) {
        dd a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          double2 v = sm.A[stage][kk][tx + 16 * i];
          a[i] = mfdev::make(v.x, v.y);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          double2 v = sm.B[stage][kk][ty + 16 * j];
          b[j] = mfdev::make(v.x, v.y);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int i = 0; i < 4; ++i)
            acc[i][j] = TA ? mfdev::dd_add_bf(acc[i][j], mfdev::dd_mul_bf(a[i], b[j]))   // temp + a(l,i) * b
                           : mfdev::dd_add_bf(acc[i][j], mfdev::dd_mul_bf(b[j], a[i]));  // c + temp * a(i,l)
      }
    }
    __syncthreads();
  }

#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t gj = n0 + ty + 16 * j;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int64_t gi = m0 + tx + 16 * i;
      if (gi < M && gj < N) {
        double *dst = C + 2 * (gi + gj * ldc);
        dd r = acc[i][j];
        if constexpr (TA) {
          r = dd_mul(alpha, r);
          if (beta_mode != BETA_ZERO) r = dd_add(r, dd_mul(beta, ld_dd_a<ALIGNED>(dst)));
        }
        st_dd<ALIGNED>(dst, r);
      }
    }
  }
}

template <bool TA, bool TB>
void launch_wgemm_t(bool aligned, dim3 grid, cudaStream_t s, const double *A, int64_t lda,
                    const double *B, int64_t ldb, double *C, int64_t ldc, int64_t m, int64_t n,
                    int64_t k, dd alpha, dd beta, int bm) {
  if (aligned)
    wgemm_kernel<TA, TB, true><<<grid, kWThreads, 0, s>>>(A, lda, B, ldb, C, ldc, m, n, k, alpha, beta, bm);
  else
    wgemm_kernel<TA, TB, false><<<grid, kWThreads, 0, s>>>(A, lda, B, ldb, C, ldc, m, n, k, alpha, beta, bm);
}

// ---- wtrsm blocked solve ------------------------------------------------------
// Kinds: left side with A or A^T, right side with A or A^T.
enum { T_LN = 0, T_LT = 1, T_RN = 2, T_RT = 3 };
constexpr int kTThreads = 256;
constexpr int kTV = 16;   // vectors per CTA
constexpr int kTNB = 32;  // pivots per diagonal block
constexpr int kTCH = 64;  // positions per chunk of the update of the remaining elements

struct TrsmSmem {
  double2 xs[kTNB][kTV];  // the block's elements (pivots once final)
  union {
    double2 cb[kTNB][kTNB + 1];  // diagonal block: [element][pivot]
    double2 ct[kTNB][kTCH];      // chunk of the remaining elements: [pivot][position]
  } u;
  unsigned char act[kTNB][kTV];  // left, A not transposed: pivot was non-zero (update applies)
};

// Pivot order: DESC walks the element index from L-1 down to 0.
//   LN upper / LT lower / RN lower / RT upper: descending.
// Coefficient of pivot k in the update of element e:
//   LN: A(e, k)   LT: A(k, e)   RN: A(k, e)   RT: A(e, k).
// Zero tests that skip an update: LN on the pivot value before its division
// (wtrsm.f90:65, 85), RN / RT on the coefficient (wtrsm.f90:181, 231, 285, 329);
// LT never skips.  Product operand order as in the Fortran:
//   LN: b(k,j) * a(i,k)   others: a * b.
template <int KIND, bool UPPER>
__global__ void __launch_bounds__(kTThreads)
    wtrsm_kernel(const double *__restrict__ A, int64_t lda, double *__restrict__ B, int64_t ldb,
                 int64_t L, int64_t NV, dd alpha, int alpha_not_one, int nounit) {
  constexpr bool LEFT = KIND == T_LN || KIND == T_LT;
  constexpr bool DESC = (KIND == T_LN && UPPER) || (KIND == T_LT && !UPPER) ||
                        (KIND == T_RN && !UPPER) || (KIND == T_RT && UPPER);
  constexpr bool COLK = KIND == T_LN || KIND == T_RT;
  __shared__ __align__(16) TrsmSmem sm;
  const int t = threadIdx.x;
  const int64_t v0 = (int64_t)blockIdx.x * kTV;

  auto eidx = [&](int64_t q) -> int64_t { return DESC ? L - 1 - q : q; };
  auto xptr = [&](int64_t e, int64_t v) -> double * {
    return LEFT ? B + 2 * (e + v * ldb) : B + 2 * (v + e * ldb);
  };
  auto cptr = [&](int64_t e, int64_t k) -> const double * {
    return COLK ? A + 2 * (e + k * lda) : A + 2 * (k + e * lda);
  };
  // x - coef * x_p with the Fortran's operand order (LN: b(k,j) * a(i,k))
  auto update = [&](dd x, dd coef, dd xp) -> dd {
    return KIND == T_LN ? mfdev::fmadd_dd<true>(x, xp, coef) : mfdev::fmadd_dd<true>(x, coef, xp);
  };

  // alpha before any update: LN / RN when alpha /= one (wtrsm.f90:58-62,
  // 137-141), LT always (temp = alpha * b(i,j), wtrsm.f90:106).
  if (KIND == T_LT || ((KIND == T_LN || KIND == T_RN) && alpha_not_one)) {
    for (int64_t id = t; id < L * kTV; id += kTThreads) {
      const int64_t e = LEFT ? id % L : id / kTV, v = v0 + (LEFT ? id / L : id % kTV);
      if (v < NV) {
        double *p = xptr(e, v);
        dd x = dd_mul(alpha, ld_dd(p));
        p[0] = x.hi;
        p[1] = x.lo;
      }
    }
    __syncthreads();
  }

  for (int64_t q0 = 0; q0 < L; q0 += kTNB) {
    const int nb = (L - q0) < kTNB ? (int)(L - q0) : kTNB;
    // the block's elements and its coefficients
    for (int id = t; id < kTNB * kTV; id += kTThreads) {
      const int a = LEFT ? id % kTNB : id / kTV, v = LEFT ? id / kTNB : id % kTV;
      dd x = dd0();
      if (a < nb && v0 + v < NV) x = ld_dd(xptr(eidx(q0 + a), v0 + v));
      sm.xs[a][v] = make_double2(x.hi, x.lo);
    }
    for (int id = t; id < kTNB * kTNB; id += kTThreads) {
      const int a = COLK ? id % kTNB : id / kTNB, p = COLK ? id / kTNB : id % kTNB;
      dd c = dd0();
      if (a < nb && p < nb) c = ld_dd(cptr(eidx(q0 + a), eidx(q0 + p)));
      sm.u.cb[a][p] = make_double2(c.hi, c.lo);
    }
    __syncthreads();

    // diagonal block, pivot by pivot
    for (int p = 0; p < nb; ++p) {
      if (t < kTV) {
        double2 xv = sm.xs[p][t], dv = sm.u.cb[p][p];
        dd x = mfdev::make(xv.x, xv.y), d = mfdev::make(dv.x, dv.y);
        unsigned char act = 1;
        if (KIND == T_LN) {
          act = !is_zero(x);
          if (act && nounit) x = dd_div(x, d);
        } else if (KIND == T_LT) {
          if (nounit) x = dd_div(x, d);
        } else if (nounit) {  // temp = one / a(j,j); b = temp * b
          x = dd_mul(dd_div(mfdev::make(1.0, 0.0), d), x);
        }
        sm.xs[p][t] = make_double2(x.hi, x.lo);
        sm.act[p][t] = act;
      }
      __syncthreads();
      const int rem = (nb - p - 1) * kTV;
      for (int id = t; id < rem; id += kTThreads) {
        const int a = p + 1 + id / kTV, v = id % kTV;
        double2 cv = sm.u.cb[a][p], pv = sm.xs[p][v], av = sm.xs[a][v];
        const dd c = mfdev::make(cv.x, cv.y);
        const bool skip = KIND == T_LN ? !sm.act[p][v] : (KIND == T_LT ? false : is_zero(c));
        if (!skip) {
          dd x = update(mfdev::make(av.x, av.y), c, mfdev::make(pv.x, pv.y));
          sm.xs[a][v] = make_double2(x.hi, x.lo);
        }
      }
      __syncthreads();
    }

    // the block is final: store it (right side with A^T: alpha after the pivot's
    // last use, wtrsm.f90:297-301, 341-345)
    for (int id = t; id < kTNB * kTV; id += kTThreads) {
      const int a = LEFT ? id % kTNB : id / kTV, v = LEFT ? id / kTNB : id % kTV;
      if (a < nb && v0 + v < NV) {
        double2 xv = sm.xs[a][v];
        dd x = mfdev::make(xv.x, xv.y);
        if (KIND == T_RT && alpha_not_one) x = dd_mul(alpha, x);
        double *p = xptr(eidx(q0 + a), v0 + v);
        p[0] = x.hi;
        p[1] = x.lo;
      }
    }

    // the block's pivots applied to the remaining elements, chunk by chunk
    for (int64_t c0 = q0 + nb; c0 < L; c0 += kTCH) {
      const int cn = (L - c0) < kTCH ? (int)(L - c0) : kTCH;
      __syncthreads();  // the previous chunk's coefficients are no longer read
      for (int id = t; id < kTNB * kTCH; id += kTThreads) {
        const int qq = COLK ? id % kTCH : id / kTNB, p = COLK ? id / kTCH : id % kTNB;
        dd c = dd0();
        if (qq < cn && p < nb) c = ld_dd(cptr(eidx(c0 + qq), eidx(q0 + p)));
        sm.u.ct[p][qq] = make_double2(c.hi, c.lo);
      }
      __syncthreads();
      // four (position, vector) pairs per thread; lanes along the contiguous index of B
      int qq[4], vv[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        qq[r] = LEFT ? t % kTCH : t / kTV + 16 * r;
        vv[r] = LEFT ? t / kTCH + 4 * r : t % kTV;
      }
      dd x[4];
      bool live[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        live[r] = qq[r] < cn && v0 + vv[r] < NV;
        x[r] = live[r] ? ld_dd(xptr(eidx(c0 + qq[r]), v0 + vv[r])) : dd0();
      }
      for (int p = 0; p < nb; ++p) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          double2 cv = sm.u.ct[p][qq[r]], pv = sm.xs[p][vv[r]];
          const dd c = mfdev::make(cv.x, cv.y);
          const bool skip = KIND == T_LN ? !sm.act[p][vv[r]] : (KIND == T_LT ? false : is_zero(c));
          const dd u = update(x[r], c, mfdev::make(pv.x, pv.y));
          x[r].hi = skip ? x[r].hi : u.hi;  // a skipped update leaves the element as it is
          x[r].lo = skip ? x[r].lo : u.lo;
        }
      }
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (live[r]) {
          double *p = xptr(eidx(c0 + qq[r]), v0 + vv[r]);
          p[0] = x[r].hi;
          p[1] = x[r].lo;
        }
    }
    __syncthreads();  // before the next block reuses shared memory
  }
}

// Left side with A^T lower (wtrsm.f90:118-131) and right side with A lower
// (wtrsm.f90:154-176): the pivots are finalised from the last index down, but
// each element accumulates its updates over k = i+1 .. L-1 in ascending order,
// i.e. starting from the pivot finalised last.  Every element's chain therefore
// waits for the previous element's whole chain, and no blocking can reorder
// it without changing the bits: one thread runs one vector's recurrence
// in the Fortran's order, vectors in parallel.  Coefficients A(k, e) run down
// column e (one address per warp, broadcast).
//   LT: t = alpha b_i; t -= A(k,i) b_k (k ascending); t /= A(i,i) if non-unit.
//   RN: x = alpha x if alpha /= one; x -= A(k,j) x_k unless A(k,j) = 0;
//       x = (one / A(j,j)) x if non-unit.
constexpr int kChainThreads = 32;
constexpr int kChainBatch = 16;  // (coefficient, pivot) pairs loaded one batch ahead

template <int KIND, bool ALIGNED>
__global__ void __launch_bounds__(kChainThreads)
    wtrsm_chain_kernel(const double *__restrict__ A, int64_t lda, double *__restrict__ B,
                       int64_t ldb, int64_t L, int64_t NV, dd alpha, int alpha_not_one, int nounit) {
  const int64_t v = (int64_t)blockIdx.x * kChainThreads + threadIdx.x;
  if (v >= NV) return;
  // element e of this vector at xv + e * xs (doubles)
  const int64_t xs = KIND == T_LT ? 2 : 2 * ldb;
  double *const xv = KIND == T_LT ? B + 2 * v * ldb : B + 2 * v;
  for (int64_t e = L - 1; e >= 0; --e) {
    dd x = ld_dd_a<ALIGNED>(xv + e * xs);
    if (KIND == T_LT || alpha_not_one) x = dd_mul(alpha, x);
    // the chain x -= A(k,e) x_k over k = e+1 .. L-1 in batches: the loads and
    // products of a batch do not depend on the chain and go ahead of it
    const double *cp = A + 2 * (e * lda + e + 1);
    const double *xp = xv + (e + 1) * xs;
    int64_t rem = L - 1 - e;
    dd cn[kChainBatch], xn[kChainBatch];
    auto fetch = [&]() {
#pragma unroll
      for (int u = 0; u < kChainBatch; ++u) {
        cn[u] = ld_dd_a<ALIGNED>(cp + 2 * u);
        xn[u] = ld_dd_a<ALIGNED>(xp + u * xs);
      }
    };
    // the product's general path with only its high limb selected: when the
    // product short-circuits (non-finite), so does the subtraction, and its low
    // limb is never read
    auto product = [&](dd c, dd xk, double &ph, double &pl) {
      double p00, e00;
      mfdev::two_prod(c.hi, xk.hi, p00, e00);
      double p01 = __dmul_rn(c.hi, xk.lo);
      const double p10 = __dmul_rn(c.lo, xk.hi);
      p01 = __dadd_rn(p01, p10);
      e00 = __dadd_rn(e00, p01);
      mfdev::fast_two_sum(p00, e00, ph, pl);
      ph = mfdev::finite_bits(p00) ? ph : p00;
    };
    auto step = [&](dd c, double ph, double pl) {
      const dd r = mfdev::dd_sub_bf(x, mfdev::make(ph, pl));
      const bool skip = KIND == T_RN && mfdev::both_zero_bits(c.hi, c.lo);
      x.hi = skip ? x.hi : r.hi;
      x.lo = skip ? x.lo : r.lo;
    };
    if (rem >= kChainBatch) fetch();
    while (rem >= kChainBatch) {
      dd c[kChainBatch], xk[kChainBatch];
#pragma unroll
      for (int u = 0; u < kChainBatch; ++u) {
        c[u] = cn[u];
        xk[u] = xn[u];
      }
      cp += 2 * kChainBatch;
      xp += kChainBatch * xs;
      rem -= kChainBatch;
      if (rem >= kChainBatch) fetch();
      double ph[kChainBatch], pl[kChainBatch];
#pragma unroll
      for (int u = 0; u < kChainBatch; ++u) product(c[u], xk[u], ph[u], pl[u]);
#pragma unroll
      for (int u = 0; u < kChainBatch; ++u) step(c[u], ph[u], pl[u]);
    }
    for (; rem > 0; --rem, cp += 2, xp += xs) {
      const dd c = ld_dd_a<ALIGNED>(cp);
      double ph, pl;
      product(c, ld_dd_a<ALIGNED>(xp), ph, pl);
      step(c, ph, pl);
    }
    const dd d = ld_dd_a<ALIGNED>(A + 2 * (e * lda + e));
    if (nounit) x = KIND == T_LT ? dd_div(x, d) : dd_mul(dd_div(mfdev::make(1.0, 0.0), d), x);
    double *p = xv + e * xs;
    st_dd<ALIGNED>(p, x);
  }
}

template <int KIND>
void launch_wtrsm_k(bool upper, unsigned grid, cudaStream_t s, const double *A, int64_t lda,
                    double *B, int64_t ldb, int64_t L, int64_t NV, dd alpha, int ano, int nounit) {
  if (upper)
    wtrsm_kernel<KIND, true><<<grid, kTThreads, 0, s>>>(A, lda, B, ldb, L, NV, alpha, ano, nounit);
  else
    wtrsm_kernel<KIND, false><<<grid, kTThreads, 0, s>>>(A, lda, B, ldb, L, NV, alpha, ano, nounit);
}

}  // namespace

// ---- device-pointer entry points ------------------------------------------------
int wgemm_dev(char ta, char tb, int64_t m, int64_t n, int64_t k, const float64x2 *alpha,
              const float64x2 *a, int64_t lda, const float64x2 *b, int64_t ldb,
              const float64x2 *beta, float64x2 *c, int64_t ldc, int *info_out, cudaStream_t s) {
  const int info = wgemm_info(ta, tb, m, n, k, lda, ldb, ldc);
  if (info_out) *info_out = info;
  if (info) return MFCUDA_ERR_INVALID_ARG;
  if (!alpha || !beta) return MFCUDA_ERR_INVALID_ARG;
  const bool nota = lsame(ta, 'N'), notb = lsame(tb, 'N');
  if (!span_ok(lda, nota ? k : m) || !span_ok(ldb, notb ? n : k) || !span_ok(ldc, n))
    return MFCUDA_ERR_INVALID_ARG;
  const bool alpha0 = dd_is(alpha, 0.0), beta1 = dd_is(beta, 1.0), beta0 = dd_is(beta, 0.0);
  if (m == 0 || n == 0 || ((alpha0 || k == 0) && beta1)) return MFCUDA_OK;  // wgemm.f90:49
  if (!c) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  double *C = reinterpret_cast<double *>(c);
  if (alpha0) return launch_scale(C, ldc, m, n, to_dd(beta), beta0, s);
  if (k > 0 && (!a || !b)) return MFCUDA_ERR_INVALID_ARG;
  const int64_t gx = (m + kWTile - 1) / kWTile, gy = (n + kWTile - 1) / kWTile;
  if (gy > 65535 || gx > INT32_MAX) return MFCUDA_ERR_UNSUPPORTED;
  const dim3 grid((unsigned)gx, (unsigned)gy);
  const double *A = reinterpret_cast<const double *>(a), *Bm = reinterpret_cast<const double *>(b);
  const bool al = ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) |
                    reinterpret_cast<uintptr_t>(c)) & 15) == 0;
  const int bm = beta0 ? BETA_ZERO : (beta1 ? BETA_ONE : BETA_OTHER);
  const dd av = to_dd(alpha), bv = to_dd(beta);
  if (nota && notb) launch_wgemm_t<false, false>(al, grid, s, A, lda, Bm, ldb, C, ldc, m, n, k, av, bv, bm);
  else if (nota) launch_wgemm_t<false, true>(al, grid, s, A, lda, Bm, ldb, C, ldc, m, n, k, av, bv, bm);
  else if (notb) launch_wgemm_t<true, false>(al, grid, s, A, lda, Bm, ldb, C, ldc, m, n, k, av, bv, bm);
  else launch_wgemm_t<true, true>(al, grid, s, A, lda, Bm, ldb, C, ldc, m, n, k, av, bv, bm);
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

int wtrsm_dev(char side, char uplo, char ta, char diag, int64_t m, int64_t n,
              const float64x2 *alpha, const float64x2 *a, int64_t lda, float64x2 *b, int64_t ldb,
              int *info_out, cudaStream_t s) {
  const int info = wtrsm_info(side, uplo, ta, diag, m, n, lda, ldb);
  if (info_out) *info_out = info;
  if (info) return MFCUDA_ERR_INVALID_ARG;
  if (!alpha) return MFCUDA_ERR_INVALID_ARG;
  const bool lside = lsame(side, 'L');
  const int64_t na = lside ? m : n;
  if (!span_ok(lda, na) || !span_ok(ldb, n)) return MFCUDA_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return MFCUDA_OK;
  if (!b) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  double *Bm = reinterpret_cast<double *>(b);
  if (dd_is(alpha, 0.0)) return launch_scale(Bm, ldb, m, n, to_dd(alpha), 1, s);
  if (!a) return MFCUDA_ERR_INVALID_ARG;
  const int64_t L = na, NV = lside ? n : m;
  const int64_t blocks = (NV + kTV - 1) / kTV;
  if (blocks > INT32_MAX) return MFCUDA_ERR_UNSUPPORTED;
  const double *A = reinterpret_cast<const double *>(a);
  const bool upper = lsame(uplo, 'U'), notr = lsame(ta, 'N');
  const int ano = !dd_is(alpha, 1.0), nounit = lsame(diag, 'N');
  const dd av = to_dd(alpha);
  const unsigned g = (unsigned)blocks;
  if (!upper && lside != notr) {  // LT lower / RN lower: the sequential chain form
    const int64_t cb = (NV + kChainThreads - 1) / kChainThreads;
    const bool al = ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15) == 0;
    if (lside && al)
      wtrsm_chain_kernel<T_LT, true><<<(unsigned)cb, kChainThreads, 0, s>>>(A, lda, Bm, ldb, L, NV, av, ano, nounit);
    else if (lside)
      wtrsm_chain_kernel<T_LT, false><<<(unsigned)cb, kChainThreads, 0, s>>>(A, lda, Bm, ldb, L, NV, av, ano, nounit);
    else if (al)
      wtrsm_chain_kernel<T_RN, true><<<(unsigned)cb, kChainThreads, 0, s>>>(A, lda, Bm, ldb, L, NV, av, ano, nounit);
    else
      wtrsm_chain_kernel<T_RN, false><<<(unsigned)cb, kChainThreads, 0, s>>>(A, lda, Bm, ldb, L, NV, av, ano, nounit);
    MF_TRY_CUDA(cudaGetLastError());
    return MFCUDA_OK;
  }
  if (lside && notr) launch_wtrsm_k<T_LN>(upper, g, s, A, lda, Bm, ldb, L, NV, av, ano, nounit);
  else if (lside) launch_wtrsm_k<T_LT>(upper, g, s, A, lda, Bm, ldb, L, NV, av, ano, nounit);
  else if (notr) launch_wtrsm_k<T_RN>(upper, g, s, A, lda, Bm, ldb, L, NV, av, ano, nounit);
  else launch_wtrsm_k<T_RT>(upper, g, s, A, lda, Bm, ldb, L, NV, av, ano, nounit);
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

// ---- host-pointer (Fortran-callable) forms ----------------------------------------
namespace {

// rows x cols block of a column-major host matrix (leading dimension ld) to or
// from a packed device buffer.
cudaError_t copy_in(void *dst, const void *src, int64_t ld, int64_t rows, int64_t cols, cudaStream_t s) {
  if (rows == 0 || cols == 0) return cudaSuccess;
  return cudaMemcpy2DAsync(dst, (size_t)rows * 16, src, (size_t)ld * 16, (size_t)rows * 16,
                           (size_t)cols, cudaMemcpyHostToDevice, s);
}
cudaError_t copy_out(void *dst, const void *src, int64_t ld, int64_t rows, int64_t cols, cudaStream_t s) {
  if (rows == 0 || cols == 0) return cudaSuccess;
  return cudaMemcpy2DAsync(dst, (size_t)ld * 16, src, (size_t)rows * 16, (size_t)rows * 16,
                           (size_t)cols, cudaMemcpyDeviceToHost, s);
}

void report(const char *name, int info) {
  if (xerbla_) xerbla_(name, &info, 6);
}

int wgemm_host(char ta, char tb, int64_t m, int64_t n, int64_t k, const float64x2 *alpha,
               const float64x2 *a, int64_t lda, const float64x2 *b, int64_t ldb,
               const float64x2 *beta, float64x2 *c, int64_t ldc) {
  const int info = wgemm_info(ta, tb, m, n, k, lda, ldb, ldc);
  if (info) {
    report("DGEMM ", info);
    return MFCUDA_ERR_INVALID_ARG;
  }
  if (!alpha || !beta) return MFCUDA_ERR_INVALID_ARG;
  const bool alpha0 = dd_is(alpha, 0.0), beta1 = dd_is(beta, 1.0), beta0 = dd_is(beta, 0.0);
  if (m == 0 || n == 0 || ((alpha0 || k == 0) && beta1)) return MFCUDA_OK;
  const bool nota = lsame(ta, 'N'), notb = lsame(tb, 'N');
  const int64_t ra = alpha0 ? 0 : (nota ? m : k), ca = alpha0 ? 0 : (nota ? k : m);
  const int64_t rb = alpha0 ? 0 : (notb ? k : n), cb = alpha0 ? 0 : (notb ? n : k);
  if (!span_ok(lda, ca) || !span_ok(ldb, cb) || !span_ok(ldc, n) || !span_ok(ra, ca) ||
      !span_ok(rb, cb) || !span_ok(m, n))
    return MFCUDA_ERR_INVALID_ARG;
  if (!c || (ra * ca > 0 && !a) || (rb * cb > 0 && !b)) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  size_t sz[4] = {(size_t)(ra * ca) * 16, (size_t)(rb * cb) * 16, (size_t)(m * n) * 16, 0};
  Staging st;
  MF_TRY(staging_acquire(st, sz));
  auto *da = static_cast<float64x2 *>(st.buf[0]);
  auto *db = static_cast<float64x2 *>(st.buf[1]);
  auto *dc = static_cast<float64x2 *>(st.buf[2]);
  MF_TRY_CUDA(copy_in(da, a, lda, ra, ca, st.stream));
  MF_TRY_CUDA(copy_in(db, b, ldb, rb, cb, st.stream));
  if (!beta0) MF_TRY_CUDA(copy_in(dc, c, ldc, m, n, st.stream));  // beta = 0: C is not read
  MF_TRY(wgemm_dev(ta, tb, m, n, k, alpha, da, max1(nota ? m : k), db, max1(notb ? k : n), beta,
                   dc, m, nullptr, st.stream));
  MF_TRY_CUDA(copy_out(c, dc, ldc, m, n, st.stream));
  MF_TRY_CUDA(cudaStreamSynchronize(st.stream));
  return MFCUDA_OK;
}

int wtrsm_host(char side, char uplo, char ta, char diag, int64_t m, int64_t n,
               const float64x2 *alpha, const float64x2 *a, int64_t lda, float64x2 *b,
               int64_t ldb) {
  const int info = wtrsm_info(side, uplo, ta, diag, m, n, lda, ldb);
  if (info) {
    report("DTRSM ", info);
    return MFCUDA_ERR_INVALID_ARG;
  }
  if (!alpha) return MFCUDA_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return MFCUDA_OK;
  const bool alpha0 = dd_is(alpha, 0.0);
  const int64_t nrowa = lsame(side, 'L') ? m : n, na = alpha0 ? 0 : nrowa;  // alpha = 0: A is not read
  if (!span_ok(lda, na) || !span_ok(ldb, n) || !span_ok(na, na) || !span_ok(m, n))
    return MFCUDA_ERR_INVALID_ARG;
  if (!b || (na > 0 && !a)) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  size_t sz[4] = {(size_t)(na * na) * 16, (size_t)(m * n) * 16, 0, 0};
  Staging st;
  MF_TRY(staging_acquire(st, sz));
  auto *da = static_cast<float64x2 *>(st.buf[0]);
  auto *db = static_cast<float64x2 *>(st.buf[1]);
  MF_TRY_CUDA(copy_in(da, a, lda, na, na, st.stream));
  if (!alpha0) MF_TRY_CUDA(copy_in(db, b, ldb, m, n, st.stream));  // alpha = 0: B is not read
  MF_TRY(wtrsm_dev(side, uplo, ta, diag, m, n, alpha, da, max1(nrowa), db, m, nullptr, st.stream));
  MF_TRY_CUDA(copy_out(b, db, ldb, m, n, st.stream));
  MF_TRY_CUDA(cudaStreamSynchronize(st.stream));
  return MFCUDA_OK;
}

}  // namespace
}  // namespace mfcuda

extern "C" {

MULTIFLOATS_CUDA_API int mfcuda_wgemm_dd(char transa, char transb, int64_t m, int64_t n, int64_t k,
                                         const float64x2 *alpha, const float64x2 *a, int64_t lda,
                                         const float64x2 *b, int64_t ldb, const float64x2 *beta,
                                         float64x2 *c, int64_t ldc, int *info, void *stream) {
  return mfcuda::wgemm_dev(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, info,
                           mfcuda::as_stream(stream));
}

MULTIFLOATS_CUDA_API int mfcuda_wtrsm_dd(char side, char uplo, char transa, char diag, int64_t m,
                                         int64_t n, const float64x2 *alpha, const float64x2 *a,
                                         int64_t lda, float64x2 *b, int64_t ldb, int *info,
                                         void *stream) {
  return mfcuda::wtrsm_dev(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, info,
                           mfcuda::as_stream(stream));
}

MULTIFLOATS_CUDA_API void wgemm_(const char *transa, const char *transb, const int *m, const int *n,
                                 const int *k, const float64x2 *alpha, const float64x2 *a,
                                 const int *lda, const float64x2 *b, const int *ldb,
                                 const float64x2 *beta, float64x2 *c, const int *ldc,
                                 size_t transa_len, size_t transb_len) {
  (void)transa_len;
  (void)transb_len;
  if (!transa || !transb || !m || !n || !k || !lda || !ldb || !ldc) {
    mfcuda::set_last_error(MFCUDA_ERR_INVALID_ARG);
    return;
  }
  mfcuda::set_last_error(mfcuda::wgemm_host(*transa, *transb, *m, *n, *k, alpha, a, *lda, b, *ldb,
                                            beta, c, *ldc));
}

MULTIFLOATS_CUDA_API void wtrsm_(const char *side, const char *uplo, const char *transa,
                                 const char *diag, const int *m, const int *n,
                                 const float64x2 *alpha, const float64x2 *a, const int *lda,
                                 float64x2 *b, const int *ldb, size_t side_len, size_t uplo_len,
                                 size_t transa_len, size_t diag_len) {
  (void)side_len;
  (void)uplo_len;
  (void)transa_len;
  (void)diag_len;
  if (!side || !uplo || !transa || !diag || !m || !n || !lda || !ldb) {
    mfcuda::set_last_error(MFCUDA_ERR_INVALID_ARG);
    return;
  }
  mfcuda::set_last_error(
      mfcuda::wtrsm_host(*side, *uplo, *transa, *diag, *m, *n, alpha, a, *lda, b, *ldb));
}

}  // extern "C"
