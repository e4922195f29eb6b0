// ORACLE -- test infrastructure only.  Array loops and a multi-threaded
// driver around the reference library's own C ABI, compiled together with the
// reference sources into oracle/_ref/libmfref.so by oracle/Makefile.  Used to
// pin the C restatement, to generate golden vectors, and as the timed CPU
// baseline (bench.py --impl reference).  Every value comes from the
// reference's exported functions (expdd, logdd, ..., matmuldd_mm); this file
// only loops over them.
#include <multifloats/float64x2.h>

#include <cstdint>
#include <thread>
#include <vector>

using multifloats::float64x2;
using namespace multifloats;

extern "C" {

void ref_unary_array(int op, const float64x2 *x, float64x2 *y, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    switch (op) {
      case 0: y[i] = expdd(x[i]); break;
      case 1: y[i] = logdd(x[i]); break;
      case 2: y[i] = sindd(x[i]); break;
      case 3: y[i] = cosdd(x[i]); break;
      case 5: y[i] = exp2dd(x[i]); break;
      case 6: y[i] = log2dd(x[i]); break;
      case 7: y[i] = log10dd(x[i]); break;
      default: y[i] = sqrtdd(x[i]); break;
    }
  }
}

// kind 0: sincosdd into s, c; 1: cexpidd into complex z; 2: cexpdd over complex z.
void ref_pair_array(int kind, const void *x, void *y0, void *y1, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    if (kind == 0) {
      sincosdd(static_cast<const float64x2 *>(x)[i], static_cast<float64x2 *>(y0) + i,
               static_cast<float64x2 *>(y1) + i);
    } else if (kind == 1) {
      static_cast<complex64x2 *>(y0)[i] = cexpidd(static_cast<const float64x2 *>(x)[i]);
    } else {
      static_cast<complex64x2 *>(y0)[i] = cexpdd(static_cast<const complex64x2 *>(x)[i]);
    }
  }
}

void ref_binary_array(int op, const float64x2 *a, const float64x2 *b, float64x2 *y, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    switch (op) {
      case 0: y[i] = adddd(a[i], b[i]); break;
      case 1: y[i] = subdd(a[i], b[i]); break;
      case 2: y[i] = muldd(a[i], b[i]); break;
      default: y[i] = divdd(a[i], b[i]); break;
    }
  }
}

// Unary map over n elements with `threads` threads (contiguous ranges).
void ref_unary_array_mt(int op, const float64x2 *x, float64x2 *y, int64_t n, int threads) {
  if (threads <= 1 || n < 1024) {
    ref_unary_array(op, x, y, n);
    return;
  }
  std::vector<std::thread> pool;
  int64_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    int64_t lo = t * chunk, hi = lo + chunk < n ? lo + chunk : n;
    if (lo >= hi) break;
    pool.emplace_back([=] { ref_unary_array(op, x + lo, y + lo, hi - lo); });
  }
  for (auto &th : pool) th.join();
}

// matmuldd_mm with the columns of B and C sharded over `threads` threads.
// Each output column is computed by exactly the code path a single call
// takes, so the result is bit-identical to matmuldd_mm(a, b, c, m, k, n, ri).
void ref_matmul_mm_mt(const float64x2 *a, const float64x2 *b, float64x2 *c, int64_t m, int64_t k,
                      int64_t n, int64_t ri, int threads) {
  if (threads <= 1 || n < 4) {
    matmuldd_mm(a, b, c, m, k, n, ri);
    return;
  }
  // even column counts keep the reference's NR=2 panel pairing identical
  int64_t chunk = (n + threads - 1) / threads;
  chunk += chunk & 1;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    int64_t j0 = t * chunk, j1 = j0 + chunk < n ? j0 + chunk : n;
    if (j0 >= j1) break;
    pool.emplace_back([=] { matmuldd_mm(a, b + j0 * k, c + j0 * m, m, k, j1 - j0, ri); });
  }
  for (auto &th : pool) th.join();
}

// BLAS-style shims test/integration/blas/wgemm.f90 and wtrsm.f90 (Fortran, not
// buildable here: no Fortran compiler) written out on the reference's own
// float64x2 operators, which are bit-identical to the Fortran ones
// (test/integration/crosscheck.cc).  Column-major with leading dimensions,
// transposition and diagonal flags as upper-case letters; the argument checks
// are left to the caller.  Same loop order as the Fortran.
void ref_wgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, const float64x2 *alpha_,
               const float64x2 *a, int64_t lda, const float64x2 *b, int64_t ldb,
               const float64x2 *beta_, float64x2 *c, int64_t ldc) {
  const float64x2 one(1.0), zero(0.0), alpha = *alpha_, beta = *beta_;
  auto A = [&](int64_t i, int64_t j) { return a[i + j * lda]; };
  auto B = [&](int64_t i, int64_t j) { return b[i + j * ldb]; };
  auto C = [&](int64_t i, int64_t j) -> float64x2 & { return c[i + j * ldc]; };
  const bool nota = ta == 'N', notb = tb == 'N';
  if (m == 0 || n == 0 || ((alpha == zero || k == 0) && beta == one)) return;
  if (alpha == zero) {
    for (int64_t j = 0; j < n; ++j)
      for (int64_t i = 0; i < m; ++i) C(i, j) = beta == zero ? zero : beta * C(i, j);
    return;
  }
  for (int64_t j = 0; j < n; ++j) {
    if (nota) {
      if (beta == zero) {
        for (int64_t i = 0; i < m; ++i) C(i, j) = zero;
      } else if (beta != one) {
        for (int64_t i = 0; i < m; ++i) C(i, j) = beta * C(i, j);
      }
      for (int64_t l = 0; l < k; ++l) {
        float64x2 temp = alpha * (notb ? B(l, j) : B(j, l));
        for (int64_t i = 0; i < m; ++i) C(i, j) = C(i, j) + temp * A(i, l);
      }
    } else {
      for (int64_t i = 0; i < m; ++i) {
        float64x2 temp = zero;
        for (int64_t l = 0; l < k; ++l) temp = temp + A(l, i) * (notb ? B(l, j) : B(j, l));
        C(i, j) = beta == zero ? alpha * temp : alpha * temp + beta * C(i, j);
      }
    }
  }
}

void ref_wtrsm(char side, char uplo, char ta, char diag, int64_t m, int64_t n,
               const float64x2 *alpha_, const float64x2 *a, int64_t lda, float64x2 *b,
               int64_t ldb) {
  const float64x2 one(1.0), zero(0.0), alpha = *alpha_;
  auto A = [&](int64_t i, int64_t j) { return a[i + j * lda]; };
  auto B = [&](int64_t i, int64_t j) -> float64x2 & { return b[i + j * ldb]; };
  const bool lside = side == 'L', upper = uplo == 'U', nounit = diag == 'N', notr = ta == 'N';
  if (m == 0 || n == 0) return;
  if (alpha == zero) {
    for (int64_t j = 0; j < n; ++j)
      for (int64_t i = 0; i < m; ++i) B(i, j) = zero;
    return;
  }
  float64x2 temp;
  if (lside && notr) {
    for (int64_t j = 0; j < n; ++j) {
      if (alpha != one)
        for (int64_t i = 0; i < m; ++i) B(i, j) = alpha * B(i, j);
      for (int64_t s = 0; s < m; ++s) {
        const int64_t k = upper ? m - 1 - s : s;
        if (B(k, j) != zero) {
          if (nounit) B(k, j) = B(k, j) / A(k, k);
          for (int64_t i = upper ? 0 : k + 1; i < (upper ? k : m); ++i)
            B(i, j) = B(i, j) - B(k, j) * A(i, k);
        }
      }
    }
  } else if (lside) {
    for (int64_t j = 0; j < n; ++j)
      for (int64_t s = 0; s < m; ++s) {
        const int64_t i = upper ? s : m - 1 - s;
        temp = alpha * B(i, j);
        for (int64_t k = upper ? 0 : i + 1; k < (upper ? i : m); ++k) temp = temp - A(k, i) * B(k, j);
        if (nounit) temp = temp / A(i, i);
        B(i, j) = temp;
      }
  } else if (notr) {
    for (int64_t s = 0; s < n; ++s) {
      const int64_t j = upper ? s : n - 1 - s;
      if (alpha != one)
        for (int64_t i = 0; i < m; ++i) B(i, j) = alpha * B(i, j);
      for (int64_t k = upper ? 0 : j + 1; k < (upper ? j : n); ++k)
        if (A(k, j) != zero)
          for (int64_t i = 0; i < m; ++i) B(i, j) = B(i, j) - A(k, j) * B(i, k);
      if (nounit) {
        temp = one / A(j, j);
        for (int64_t i = 0; i < m; ++i) B(i, j) = temp * B(i, j);
      }
    }
  } else {
    for (int64_t s = 0; s < n; ++s) {
      const int64_t k = upper ? n - 1 - s : s;
      if (nounit) {
        temp = one / A(k, k);
        for (int64_t i = 0; i < m; ++i) B(i, k) = temp * B(i, k);
      }
      for (int64_t j = upper ? 0 : k + 1; j < (upper ? k : n); ++j)
        if (A(j, k) != zero) {
          temp = A(j, k);
          for (int64_t i = 0; i < m; ++i) B(i, j) = B(i, j) - temp * B(i, k);
        }
      if (alpha != one)
        for (int64_t i = 0; i < m; ++i) B(i, k) = alpha * B(i, k);
    }
  }
}

// Column-sharded (wgemm; wtrsm on the left) or row-sharded (wtrsm on the
// right) drivers over `threads` threads: the shims' outputs are independent
// per column of C / per vector of B, so each shard runs exactly the loops of a
// single call and the result is bit-identical to it.
void ref_wgemm_mt(char ta, char tb, int64_t m, int64_t n, int64_t k, const float64x2 *alpha,
                  const float64x2 *a, int64_t lda, const float64x2 *b, int64_t ldb,
                  const float64x2 *beta, float64x2 *c, int64_t ldc, int threads) {
  if (threads < 1) threads = 1;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    const int64_t j0 = n * t / threads, j1 = n * (t + 1) / threads;
    if (j1 <= j0) continue;
    const float64x2 *bs = tb == 'N' ? b + j0 * ldb : b + j0;
    pool.emplace_back(ref_wgemm, ta, tb, m, j1 - j0, k, alpha, a, lda, bs, ldb, beta, c + j0 * ldc, ldc);
  }
  for (auto &th : pool) th.join();
}

void ref_wtrsm_mt(char side, char uplo, char ta, char diag, int64_t m, int64_t n,
                  const float64x2 *alpha, const float64x2 *a, int64_t lda, float64x2 *b,
                  int64_t ldb, int threads) {
  if (threads < 1) threads = 1;
  const bool lside = side == 'L';
  const int64_t nv = lside ? n : m;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    const int64_t v0 = nv * t / threads, v1 = nv * (t + 1) / threads;
    if (v1 <= v0) continue;
    if (lside)
      pool.emplace_back(ref_wtrsm, side, uplo, ta, diag, m, v1 - v0, alpha, a, lda, b + v0 * ldb, ldb);
    else
      pool.emplace_back(ref_wtrsm, side, uplo, ta, diag, v1 - v0, n, alpha, a, lda, b + v0, ldb);
  }
  for (auto &th : pool) th.join();
}

}  // extern "C"

extern "C" {

// Fortran cdd_matmul_mm (fsrc/multifloats.fypp:2609-2621) composed from the
// reference's own matmuldd_mm and DD operators: split into re/im temporaries,
// four real products, then p_re = rr - ii, p_im = ri + ir.
void ref_cmatmul_mm(const float64x2 *a, const float64x2 *b, float64x2 *c, int64_t m, int64_t k,
                    int64_t n, int64_t ri) {
  std::vector<float64x2> ar(m * k), ai(m * k), br(k * n), bi(k * n);
  for (int64_t i = 0; i < m * k; ++i) { ar[i] = a[2 * i]; ai[i] = a[2 * i + 1]; }
  for (int64_t i = 0; i < k * n; ++i) { br[i] = b[2 * i]; bi[i] = b[2 * i + 1]; }
  std::vector<float64x2> rr(m * n), ii(m * n), rim(m * n), irm(m * n);
  matmuldd_mm(ar.data(), br.data(), rr.data(), m, k, n, ri);
  matmuldd_mm(ai.data(), bi.data(), ii.data(), m, k, n, ri);
  matmuldd_mm(ar.data(), bi.data(), rim.data(), m, k, n, ri);
  matmuldd_mm(ai.data(), br.data(), irm.data(), m, k, n, ri);
  for (int64_t i = 0; i < m * n; ++i) {
    c[2 * i] = rr[i] - ii[i];
    c[2 * i + 1] = rim[i] + irm[i];
  }
}

// Fortran dd_norm2_1d (fypp:2338-2352) with the reference's DD operators
// (bit-identical to the Fortran ones, test/integration/crosscheck.cc) and sqrtdd.
float64x2 ref_norm2_serial(const float64x2 *x, int64_t n) {
  float64x2 s(0.0);
  for (int64_t i = 0; i < n; ++i) s = s + x[i] * x[i];
  return sqrtdd(s);
}

}  // extern "C"
