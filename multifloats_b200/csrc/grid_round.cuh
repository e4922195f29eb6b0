// Rounding of a double-double entry to the W-bit fixed-point grid of its row
// (A) or column (B): the first step of both split-INT8 forms (digit slices
// and CRT residues).  Host- and device-compilable, so the host can check it.
//
// With t = W - sigma (every |entry| of the row / column is below 2^sigma)
// and IEEE double operations rounding to nearest even:
//   H = hi 2^t, L = lo 2^t                  (exact; L rounded once if it underflows)
//   P = rint(H),  Q = rint((H - P) + L),    X = P + Q  (an exact integer sum)
// then X is clamped to |X| <= 2^W - 1.  Before the clamp
// |X - (hi + lo) 2^t| <= 1/2 + 2^-52 (when |H| >= 2^53, H - P = 0 and the
// error is at most 1/2); the clamp only acts when |(hi + lo) 2^t| is within 1
// of 2^W, so afterwards |X - (hi + lo) 2^t| <= 1 always: one unit of the
// grid, the rounding term of the split forms' error bound.
//
// Only double operations and 64-bit integer arithmetic are used: P (up to
// 2^110) is split exactly as P = P1 2^56 + P0 (P1 = rint(P 2^-56), P0 = P -
// P1 2^56 by one fma, |P0| <= 2^55), every piece converts exactly to a 64-bit
// integer, and X is assembled as T 2^56 + R with 0 <= R < 2^56.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

namespace mfcuda {
namespace split {

// Exact power of two 2^e for -1022 <= e <= 1023.
__host__ __device__ __forceinline__ double grid_pow2(int e) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)(e + 1023) << 52);
#else
  const uint64_t b = (uint64_t)(e + 1023) << 52;
  double d;
  memcpy(&d, &b, sizeof d);
  return d;
#endif
}
// x 2^e rounded like ldexp: one multiplication by an exact power of two when
// 2^e is a normal double, ldexp otherwise.
__host__ __device__ __forceinline__ double grid_scale(double x, int e) {
  return (e >= -1022 && e <= 1023) ? x * grid_pow2(e) : ldexp(x, e);
}

// The clamp limits of a W-bit grid in (T, R) form (X = T 2^56 + R,
// 0 <= R < 2^56): X >= 2^W  <=>  (T, R) >= (up_t, up_r);  X <= -2^W  <=>
// (T, R) <= (dn_t, dn_r); the clamped values are (upc_t, upc_r) = 2^W - 1
// and (dnc_t, dnc_r) = -(2^W - 1).  W in [1, 118].
struct GridLimits {
  int64_t up_t, dn_t, upc_t, dnc_t;
  uint64_t up_r, dn_r, upc_r, dnc_r;
};
constexpr uint64_t kGridM56 = (1ull << 56) - 1;
__host__ __device__ __forceinline__ GridLimits grid_limits(int W) {
  GridLimits g;
  if (W >= 56) {
    const int64_t wt = (int64_t)1 << (W - 56);
    g.up_t = wt;
    g.up_r = 0;
    g.upc_t = wt - 1;
    g.upc_r = kGridM56;
    g.dn_t = -wt;
    g.dn_r = 0;
    g.dnc_t = -wt;
    g.dnc_r = 1;
  } else {
    const uint64_t wr = 1ull << W;
    g.up_t = 0;
    g.up_r = wr;
    g.upc_t = 0;
    g.upc_r = wr - 1;
    g.dn_t = -1;
    g.dn_r = (1ull << 56) - wr;
    g.dnc_t = -1;
    g.dnc_r = (1ull << 56) - wr + 1;
  }
  return g;
}

// X (as above) of the entry (hi, lo) as T 2^56 + R.
__host__ __device__ __forceinline__ void grid_round(double hi, double lo, int sigma, const GridLimits &g,
                                                    int W, int64_t &T, uint64_t &R) {
  const int t = W - sigma;
  const double H = grid_scale(hi, t), L = grid_scale(lo, t);
  const double P = rint(H);
  const double Q = rint((H - P) + L);
  const double P1 = rint(P * 0x1p-56);
  const double P0 = fma(-P1, 0x1p56, P);
  const int64_t r = (int64_t)P0 + (int64_t)Q;  // |r| < 2^59
  T = (int64_t)P1 + (r >> 56);                 // arithmetic shift: floor
  R = (uint64_t)r & kGridM56;
  if (T > g.up_t || (T == g.up_t && R >= g.up_r)) {
    T = g.upc_t;
    R = g.upc_r;
  } else if (T < g.dn_t || (T == g.dn_t && R <= g.dn_r)) {
    T = g.dnc_t;
    R = g.dnc_r;
  }
}

// Y = X + sum_{q<14} 128 * 256^q as four little-endian 32-bit words.  The
// balanced base-256 representation X = sum_q d_q 256^q with d_q in
// [-128, 127] is unique, and 0 <= Y < 256^14, so byte q of Y is exactly
// d_q + 128 (digit q as a signed byte: byte q of Y xor 0x80, no carry chain).
__host__ __device__ __forceinline__ void grid_biased_words(int64_t T, uint64_t R, uint32_t (&y)[4]) {
  const uint64_t xlo = R | ((uint64_t)T << 56);
  const uint64_t xhi = (uint64_t)(T >> 8);  // arithmetic shift: the sign extends
  const uint64_t ylo = xlo + 0x8080808080808080ull;
  const uint64_t yhi = xhi + 0x0000808080808080ull + (ylo < xlo ? 1u : 0u);
  y[0] = (uint32_t)ylo;
  y[1] = (uint32_t)(ylo >> 32);
  y[2] = (uint32_t)yhi;
  y[3] = (uint32_t)(yhi >> 32);
}

}  // namespace split
}  // namespace mfcuda
