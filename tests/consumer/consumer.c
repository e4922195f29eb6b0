/* A compiled C (or C++) caller of the drop-in boundary, built by
 * oracle/Makefile (target `consumers`) in three ways:
 *
 *   consumer_c_own     C, include/multifloats_cuda.h alone, linked with
 *                      libmultifloats_cuda only;
 *   consumer_c_ref     C, the reference's multifloats/float64x2.h included
 *                      FIRST (it defines MULTIFLOATS_ABI_VERSION, so the
 *                      library header reuses the reference's structs instead
 *                      of defining its own), linked -lmultifloats_cuda ahead
 *                      of the reference library;
 *   consumer_cxx_ref   the same compiled as C++ (the reference's class
 *                      float64x2 with its member operators).
 *
 * It calls matmuldd_mm, expdd_array and dotdd_array with host pointers on
 * seeded inputs and writes inputs and outputs to the file named by argv[1]
 * for the test to compare with the oracle.  With the reference linked it
 * also compares expdd_array element by element with the reference's own
 * scalar expdd (which stays with the reference library: the GPU library has
 * no scalar symbol) and prints, through dladdr, the shared object each
 * symbol was bound to.  Exit status: 0 ok, 2 a library call latched an
 * error, 3 a scalar mismatch, 1 usage or I/O. */
#ifndef _GNU_SOURCE
#define _GNU_SOURCE
#endif
#ifdef WITH_REFERENCE
#include <multifloats/float64x2.h>
#ifdef __cplusplus
using multifloats::expdd;  /* the reference's C ABI lives in namespace multifloats under C++ */
#endif
#endif
#include "multifloats_cuda.h"

#include <dlfcn.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef WITH_REFERENCE
#if !defined(MULTIFLOATS_ABI_VERSION) || MULTIFLOATS_ABI_VERSION != 2
#error "expected the reference header's ABI version 2"
#endif
#endif

#ifdef __cplusplus
static_assert(sizeof(float64x2) == 16 && sizeof(complex64x2) == 32, "layout");
#else
_Static_assert(sizeof(float64x2) == 16 && sizeof(complex64x2) == 32, "layout");
#endif

static uint64_t g_state = 0x9E3779B97F4A7C15ull;
static double uniform(void) { /* [-1, 1) */
  g_state = g_state * 6364136223846793005ull + 1442695040888963407ull;
  return (double)(g_state >> 11) * 0x1p-52 - 1.0;
}
static void fill(float64x2 *v, int64_t n, double scale) {
  for (int64_t i = 0; i < n; ++i) {
    double hi = uniform() * scale, lo = hi * 0x1p-53 * uniform();
    double s = hi + lo, bb = s - hi;
    v[i].limbs[0] = s;
    v[i].limbs[1] = (hi - (s - bb)) + (lo - bb);
  }
}
static const char *where(void *sym) {
  Dl_info info;
  if (sym && dladdr(sym, &info) && info.dli_fname) {
    const char *s = strrchr(info.dli_fname, '/');
    return s ? s + 1 : info.dli_fname;
  }
  return "?";
}

int main(int argc, char **argv) {
  if (argc < 2) return 1;
  const int64_t m = 64, k = 48, n = 40, nx = 4096;
  float64x2 *a = (float64x2 *)malloc(sizeof(float64x2) * m * k);
  float64x2 *b = (float64x2 *)malloc(sizeof(float64x2) * k * n);
  float64x2 *c = (float64x2 *)malloc(sizeof(float64x2) * m * n);
  float64x2 *x = (float64x2 *)malloc(sizeof(float64x2) * nx);
  float64x2 *y = (float64x2 *)malloc(sizeof(float64x2) * nx);
  float64x2 *w = (float64x2 *)malloc(sizeof(float64x2) * nx);
  fill(a, m * k, 1.0);
  fill(b, k * n, 1.0);
  fill(x, nx, 700.0);
  fill(w, nx, 1.0);
  matmuldd_mm(a, b, c, m, k, n, 8);
  if (mfcuda_last_error()) return 2;
  expdd_array(x, y, nx);
  if (mfcuda_last_error()) return 2;
  float64x2 d = dotdd_array(x, w, nx, 8);
  if (mfcuda_last_error()) return 2;
  printf("matmuldd_mm from %s\n", where((void *)&matmuldd_mm));
  printf("expdd_array from %s\n", where((void *)&expdd_array));
#ifdef WITH_REFERENCE
  printf("expdd from %s\n", where((void *)&expdd));
  int64_t same = 0;
  for (int64_t i = 0; i < nx; ++i) {
    float64x2 r = expdd(x[i]);
    same += memcmp(&r, &y[i], sizeof r) == 0;
  }
  printf("scalar expdd matches expdd_array: %lld / %lld\n", (long long)same, (long long)nx);
  if (same != nx) return 3;
#endif
  FILE *f = fopen(argv[1], "wb");
  if (!f) return 1;
  int64_t hdr[4] = {m, k, n, nx};
  fwrite(hdr, sizeof hdr, 1, f);
  fwrite(a, sizeof(float64x2), (size_t)(m * k), f);
  fwrite(b, sizeof(float64x2), (size_t)(k * n), f);
  fwrite(c, sizeof(float64x2), (size_t)(m * n), f);
  fwrite(x, sizeof(float64x2), (size_t)nx, f);
  fwrite(y, sizeof(float64x2), (size_t)nx, f);
  fwrite(w, sizeof(float64x2), (size_t)nx, f);
  fwrite(&d, sizeof d, 1, f);
  fclose(f);
  free(a); free(b); free(c); free(x); free(y); free(w);
  return 0;
}
