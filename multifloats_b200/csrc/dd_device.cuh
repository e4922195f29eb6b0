// Device double-double (DD) core for sm_100a.
//
// A DD value is two IEEE binary64 limbs (hi, lo) with |lo| <= ulp(hi)/2,
// stored back to back (16 bytes) exactly like the reference's `float64x2`
// (include/multifloats/float64x2.h:125-186).  Every operation below restates
// the reference's arithmetic step for step with explicitly rounded device
// intrinsics (__dadd_rn, __dmul_rn, __fma_rn, __ddiv_rn, __dsqrt_rn), so that
// nvcc can neither contract a multiply-add into an FMA nor reassociate; the
// library is additionally compiled with --fmad=false.  Results are therefore
// bit-identical to the reference CPU build compiled with -ffp-contract=off.
#pragma once
#include <cstdint>
#include <math_constants.h>

#define MF_TABLE static __constant__
#define MF_GTABLE static __device__ const
#include "dd_tables.h"

namespace mfdev {

struct dd {
  double hi, lo;
};

__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double div_(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ double gload(const double* p) { return __ldg(p); }

// ---- error-free transformations (float64x2.h:84-107) ----------------------
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  double ss = add(a, b);
  double ap = sub(ss, b);
  double bp = sub(ss, ap);
  e = add(sub(a, ap), sub(b, bp));
  s = ss;
}
__device__ __forceinline__ void fast_two_sum(double a, double b, double& s, double& e) {
  double ss = add(a, b);
  double bp = sub(ss, a);
  e = sub(b, bp);
  s = ss;
}
__device__ __forceinline__ void two_prod(double a, double b, double& p, double& e) {
  double pp = mul(a, b);
  e = fma_(a, b, -pp);
  p = pp;
}

__device__ __forceinline__ dd make(double h, double l) { dd r; r.hi = h; r.lo = l; return r; }
// The quiet NaN of std::numeric_limits<double>::quiet_NaN() (sign bit clear),
// which the reference returns; its sign is visible through copysign (complex exp).
__device__ __forceinline__ double qnan() { return __longlong_as_double(0x7ff8000000000000ll); }
__device__ __forceinline__ dd neg(dd a) { return make(-a.hi, -a.lo); }

// ---- DD operators (float64x2.h:203-311) -----------------------------------
__device__ __forceinline__ dd dd_add(dd x, dd y) {
  double s = add(x.hi, y.hi);
  if (!isfinite(s)) return make(s, 0.0);
  if (x.hi == 0.0 && y.hi == 0.0) return make(s, add(x.lo, y.lo));
  double a, b, c, d;
  two_sum(x.hi, y.hi, a, b);
  two_sum(x.lo, y.lo, c, d);
  fast_two_sum(a, c, a, c);
  b = add(b, d);
  b = add(b, c);
  dd r;
  fast_two_sum(a, b, r.hi, r.lo);
  return r;
}
__device__ __forceinline__ dd dd_sub(dd x, dd y) {
  double s = sub(x.hi, y.hi);
  if (!isfinite(s)) return make(s, 0.0);
  if (x.hi == 0.0 && y.hi == 0.0) return make(s, sub(x.lo, y.lo));
  double a, b, c, d;
  two_sum(x.hi, -y.hi, a, b);
  two_sum(x.lo, -y.lo, c, d);
  fast_two_sum(a, c, a, c);
  b = add(b, d);
  b = add(b, c);
  dd r;
  fast_two_sum(a, b, r.hi, r.lo);
  return r;
}
__device__ __forceinline__ dd dd_mul(dd x, dd y) {
  double p00, e00;
  two_prod(x.hi, y.hi, p00, e00);
  if (!isfinite(p00)) return make(p00, 0.0);
  double p01 = mul(x.hi, y.lo);
  double p10 = mul(x.lo, y.hi);
  p01 = add(p01, p10);
  e00 = add(e00, p01);
  dd r;
  fast_two_sum(p00, e00, r.hi, r.lo);
  return r;
}
__device__ __forceinline__ dd dd_div(dd x, dd y) {
  double q1 = div_(x.hi, y.hi);
  if (!isfinite(q1)) return make(q1, q1);
  if (!isfinite(y.hi)) return make(q1, 0.0);
  double p00, e00;
  two_prod(q1, y.hi, p00, e00);
  double p01 = mul(q1, y.lo);
  double qhi = p00;
  double qlo = add(e00, p01);
  double r0, r0e;
  two_sum(x.hi, -qhi, r0, r0e);
  double r1 = add(sub(x.lo, qlo), r0e);
  double rh, rl;
  fast_two_sum(r0, r1, rh, rl);
  double q2 = div_(rh, y.hi);
  dd r;
  fast_two_sum(q1, q2, r.hi, r.lo);
  return r;
}

// ---- multiply-add forms for the long loops ----------------------------------
// Integer tests on the bit patterns (no FP64 compares): not inf / NaN, and two
// values both +-0.
//
// fmadd_dd: acc + x * y (or acc - x * y) with the DD operators, bit-identical
// to dd_add(acc, dd_mul(x, y)) (dd_sub) for every input.  The general paths of
// both operators are evaluated unconditionally; every short-circuit case of
// the two operators (non-finite product -- its general-path high limb is then
// NaN --, non-finite sum, both high limbs of the addition zero) shows as a
// non-finite leading sum or two zero high limbs, and only then is the step
// redone with the operators themselves.
__device__ __forceinline__ bool finite_bits(double v) {
  return (__double2hiint(v) & 0x7ff00000) != 0x7ff00000;
}
__device__ __forceinline__ bool both_zero_bits(double a, double b) {
  return ((((unsigned)__double2hiint(a) | (unsigned)__double2hiint(b)) & 0x7fffffffu) |
          (unsigned)__double2loint(a) | (unsigned)__double2loint(b)) == 0u;
}
// Branch-free forms of +, -, *: bit-identical to dd_add / dd_sub / dd_mul for
// every input; the short-circuit results are selected instead of branched to,
// so the compiler can interleave many independent chains (a tile of
// accumulators) or hoist independent products ahead of a dependent chain.
__device__ __forceinline__ dd add_parts_bf(double xh, double xl, double yh, double yl) {
  double s, b, c, d, a2, c2, rh, rl;
  two_sum(xh, yh, s, b);
  two_sum(xl, yl, c, d);  // c = xl + yl, the short-circuit low limb
  fast_two_sum(s, c, a2, c2);
  b = add(b, d);
  b = add(b, c2);
  fast_two_sum(a2, b, rh, rl);
  const bool fin = finite_bits(s), zz = both_zero_bits(xh, yh);
  dd r;
  r.hi = (fin && !zz) ? rh : s;
  r.lo = fin ? (zz ? c : rl) : 0.0;
  return r;
}
__device__ __forceinline__ dd dd_add_bf(dd x, dd y) { return add_parts_bf(x.hi, x.lo, y.hi, y.lo); }
__device__ __forceinline__ dd dd_sub_bf(dd x, dd y) { return add_parts_bf(x.hi, x.lo, -y.hi, -y.lo); }
__device__ __forceinline__ dd dd_mul_bf(dd x, dd y) {
  double p00, e00, rh, rl;
  two_prod(x.hi, y.hi, p00, e00);
  double p01 = mul(x.hi, y.lo);
  const double p10 = mul(x.lo, y.hi);
  p01 = add(p01, p10);
  e00 = add(e00, p01);
  fast_two_sum(p00, e00, rh, rl);
  const bool fin = finite_bits(p00);
  dd r;
  r.hi = fin ? rh : p00;
  r.lo = fin ? rl : 0.0;
  return r;
}

// Guarded form: the general path and a branch (not taken on ordinary data) to
// the operators.  Fewer instructions than the select form, but each step ends a
// basic block, so it suits loops with few chains per thread and many warps.
template <bool SUB>
__device__ __forceinline__ dd fmadd_dd(dd acc, dd x, dd y) {
  double p00, e00;
  two_prod(x.hi, y.hi, p00, e00);
  double p01 = mul(x.hi, y.lo);
  const double p10 = mul(x.lo, y.hi);
  p01 = add(p01, p10);
  e00 = add(e00, p01);
  double ph, pl;
  fast_two_sum(p00, e00, ph, pl);
  if (SUB) {
    ph = -ph;
    pl = -pl;
  }
  double s, b, c, d, a2, c2;
  two_sum(acc.hi, ph, s, b);
  two_sum(acc.lo, pl, c, d);
  fast_two_sum(s, c, a2, c2);
  b = add(b, d);
  b = add(b, c2);
  dd r;
  fast_two_sum(a2, b, r.hi, r.lo);
  if (__builtin_expect(!finite_bits(s) || both_zero_bits(acc.hi, ph), 0))
    r = SUB ? dd_sub(acc, dd_mul(x, y)) : dd_add(acc, dd_mul(x, y));
  return r;
}

// ---- sqrt (float64x2.h:2190-2212), Karp/Markstein --------------------------
__device__ __forceinline__ dd dd_sqrt(dd x) {
  double c = __dsqrt_rn(x.hi);
  if (!(x.hi > 0.0) || !isfinite(c)) return make(c, 0.0);
  double u, uu;
  two_prod(c, c, u, uu);
  double cc = div_(add(sub(sub(x.hi, u), uu), x.lo), mul(2.0, c));
  dd r;
  r.hi = add(c, cc);
  r.lo = add(sub(c, r.hi), cc);
  return r;
}

// ---- polynomial evaluators (src/float64x2/poly.inc) ------------------------
// horner: n = coefficient count (poly.inc:9-16).
__device__ __forceinline__ dd horner(dd y, const double* hi, const double* lo, int n) {
  dd p = make(hi[n - 1], lo[n - 1]);
  for (int i = n - 2; i >= 0; --i) p = dd_add(dd_mul(p, y), make(hi[i], lo[i]));
  return p;
}
// neval (Estrin), degree 10 and 12 cases (poly.inc:33-102).  C++ `a + b * c`
// is a + (b*c); chains of `+` associate left.
__device__ __forceinline__ dd neval10(dd x, const double* hi, const double* lo) {
#define MF_C(i) make(hi[i], lo[i])
  dd x2 = dd_mul(x, x);
  dd x4 = dd_mul(x2, x2);
  dd x8 = dd_mul(x4, x4);
  dd p01 = dd_add(MF_C(0), dd_mul(MF_C(1), x));
  dd p23 = dd_add(MF_C(2), dd_mul(MF_C(3), x));
  dd p45 = dd_add(MF_C(4), dd_mul(MF_C(5), x));
  dd p67 = dd_add(MF_C(6), dd_mul(MF_C(7), x));
  dd p89 = dd_add(MF_C(8), dd_mul(MF_C(9), x));
  dd p03 = dd_add(p01, dd_mul(p23, x2));
  dd p47 = dd_add(p45, dd_mul(p67, x2));
  dd p810 = dd_add(p89, dd_mul(MF_C(10), x2));
  return dd_add(dd_add(p03, dd_mul(p47, x4)), dd_mul(p810, x8));
}
__device__ __forceinline__ dd neval12(dd x, const double* hi, const double* lo) {
  dd x2 = dd_mul(x, x);
  dd x4 = dd_mul(x2, x2);
  dd x8 = dd_mul(x4, x4);
  dd p01 = dd_add(MF_C(0), dd_mul(MF_C(1), x));
  dd p23 = dd_add(MF_C(2), dd_mul(MF_C(3), x));
  dd p45 = dd_add(MF_C(4), dd_mul(MF_C(5), x));
  dd p67 = dd_add(MF_C(6), dd_mul(MF_C(7), x));
  dd p89 = dd_add(MF_C(8), dd_mul(MF_C(9), x));
  dd p1011 = dd_add(MF_C(10), dd_mul(MF_C(11), x));
  dd p03 = dd_add(p01, dd_mul(p23, x2));
  dd p47 = dd_add(p45, dd_mul(p67, x2));
  dd p811 = dd_add(p89, dd_mul(p1011, x2));
  return dd_add(dd_add(p03, dd_mul(p47, x4)), dd_mul(dd_add(p811, dd_mul(MF_C(12), x4)), x8));
#undef MF_C
}

// ---- exp (src/float64x2/exp_log.inc:26-72, :237-277) -----------------------
__device__ __forceinline__ dd exp2_from_reduced(double n_d, double rh, double rl) {
  if (n_d > 1100.0) return make(CUDART_INF, 0.0);
  if (n_d < -1100.0) return make(0.0, 0.0);
  double k_d = rint(mul(rh, 256.0));
  int k = (int)k_d;
  if (k > 128) k = 128;
  if (k < -128) k = -128;
  double sh = sub(rh, div_((double)k, 256.0));
  double sl = rl;
  fast_two_sum(sh, sl, sh, sl);
  dd s = make(sh, sl);
  dd q = make(mf_exp2_coefs_hi[9], mf_exp2_coefs_lo[9]);
#pragma unroll
  for (int j = 8; j >= 1; --j) {
    q = dd_mul(q, s);
    q = dd_add(q, make(mf_exp2_coefs_hi[j], mf_exp2_coefs_lo[j]));
  }
  dd pow2s = dd_add(make(1.0, 0.0), dd_mul(s, q));
  dd T = make(gload(&mf_exp2_table_hi[k + 128]), gload(&mf_exp2_table_lo[k + 128]));
  dd m = dd_mul(T, pow2s);
  int n = (int)n_d;
  return make(ldexp(m.hi, n), ldexp(m.lo, n));
}

__device__ __forceinline__ dd dd_exp(dd x) {
  double h = x.hi;
  if (!isfinite(h)) {
    if (h > 0.0) return make(h, 0.0);
    if (h < 0.0) return make(0.0, 0.0);
    return make(h, 0.0);
  }
  if (h > mf_exp_max[0]) return make(CUDART_INF, 0.0);
  if (h < mf_exp_min[0]) return make(0.0, 0.0);
  double n_d = rint(mul(h, mf_log2_e_hi[0]));
  double rh, rl, t;
  two_sum(h, -mul(n_d, mf_ln2_cw[0]), rh, t);
  rl = add(t, x.lo);
  fast_two_sum(rh, rl, rh, rl);
  double p_hi = mul(n_d, mf_ln2_cw[1]);
  double p_lo = fma_(n_d, mf_ln2_cw[1], -p_hi);
  two_sum(rh, -p_hi, rh, t);
  rl = add(rl, sub(t, p_lo));
  fast_two_sum(rh, rl, rh, rl);
  two_sum(rh, -mul(n_d, mf_ln2_cw[2]), rh, t);
  rl = add(rl, t);
  dd rr;
  fast_two_sum(rh, rl, rr.hi, rr.lo);
  dd y = dd_mul(rr, make(mf_log2_e_hi[0], mf_log2_e_lo[0]));
  return exp2_from_reduced(n_d, y.hi, y.lo);
}

// ---- log (exp_log.inc:280-341) ---------------------------------------------
__device__ __forceinline__ dd log2_kernel(dd x) {
  double hi = x.hi;
  if (hi > 15.0 / 16.0 && hi < 17.0 / 16.0) {
    dd num = dd_sub(x, make(1.0, 0.0));
    dd den = dd_add(x, make(1.0, 0.0));
    dd t = dd_div(num, den);
    dd t2 = dd_mul(t, t);
    dd p = neval10(t2, mf_log2_wide_hi, mf_log2_wide_lo);
    return dd_mul(t, p);
  }
  int e = ilogb(hi);
  dd m = make(ldexp(x.hi, -e), ldexp(x.lo, -e));
  int idx = (int)mul(sub(m.hi, 1.0), 32.0);
  if (idx < 0) idx = 0;
  if (idx > 31) idx = 31;
  dd c = make(gload(&mf_log2_centers[idx]), 0.0);
  dd v = make(gload(&mf_log2_values_hi[idx]), gload(&mf_log2_values_lo[idx]));
  dd num = dd_sub(m, c);
  dd den = dd_add(m, c);
  dd t = dd_div(num, den);
  dd t2 = dd_mul(t, t);
  dd p = horner(t2, mf_log2_narrow_hi, mf_log2_narrow_lo, 7);
  return dd_add(dd_add(make((double)e, 0.0), v), dd_mul(t, p));
}
__device__ __forceinline__ dd dd_log2(dd x) {
  if (isnan(x.hi) || x.hi < 0.0) return make(qnan(), 0.0);
  if (x.hi == 0.0) return make(-CUDART_INF, 0.0);
  if (!isfinite(x.hi)) return make(CUDART_INF, 0.0);
  return log2_kernel(x);
}
__device__ __forceinline__ dd dd_log(dd x) {
  if (!isfinite(x.hi)) return make(log(x.hi), 0.0);
  dd l2 = dd_log2(x);
  if (!isfinite(l2.hi)) return l2;
  return dd_mul(l2, make(mf_ln_2_hi[0], mf_ln_2_lo[0]));
}

// ---- sin / cos (src/float64x2/trig.inc:114-266) ----------------------------
__device__ __forceinline__ void dd_sub_step(double& rh, double& rl, double ph, double pl) {
  double sh, sl, tl, tll;
  two_sum(rh, -ph, sh, sl);
  two_sum(rl, -pl, tl, tll);
  sl = add(sl, tl);
  fast_two_sum(sh, sl, rh, rl);
  rl = add(rl, tll);
  fast_two_sum(rh, rl, rh, rl);
}
__device__ __forceinline__ dd reduce_pi_half(dd x, int& n_mod4) {
  double n_float = rint(mul(x.hi, 0.6366197723675814));
  double rh = x.hi, rl = x.lo, ph, pl;
  ph = mul(n_float, mf_pi_half_cw[0]);
  pl = fma_(n_float, mf_pi_half_cw[0], -ph);
  dd_sub_step(rh, rl, ph, pl);
  ph = mul(n_float, mf_pi_half_cw[1]);
  pl = fma_(n_float, mf_pi_half_cw[1], -ph);
  dd_sub_step(rh, rl, ph, pl);
  ph = mul(n_float, mf_pi_half_cw[2]);
  dd_sub_step(rh, rl, ph, 0.0);
  long long nn = (long long)fabs(n_float) & 3LL;
  if (n_float < 0.0) nn = (4 - nn) & 3;
  n_mod4 = (int)nn;
  return make(rh, rl);
}
__device__ __forceinline__ dd sin_kernel(dd x) {
  dd x2 = dd_mul(x, x);
  return dd_mul(neval12(x2, mf_sin_taylor_hi, mf_sin_taylor_lo), x);
}
__device__ __forceinline__ dd cos_kernel(dd x) {
  dd x2 = dd_mul(x, x);
  return neval12(x2, mf_cos_taylor_hi, mf_cos_taylor_lo);
}
// Estrin degree-12 evaluation (poly.inc:91-102) given the powers y2 = y*y,
// y4 = y2*y2, y8 = y4*y4 of its argument y, so the sin and cos polynomials of
// the same argument can share them.
__device__ __forceinline__ dd neval12_pow(dd y, dd y2, dd y4, dd y8, const double* hi,
                                          const double* lo) {
#define MF_C(i) make(hi[i], lo[i])
  dd p01 = dd_add(MF_C(0), dd_mul(MF_C(1), y));
  dd p23 = dd_add(MF_C(2), dd_mul(MF_C(3), y));
  dd p45 = dd_add(MF_C(4), dd_mul(MF_C(5), y));
  dd p67 = dd_add(MF_C(6), dd_mul(MF_C(7), y));
  dd p89 = dd_add(MF_C(8), dd_mul(MF_C(9), y));
  dd p1011 = dd_add(MF_C(10), dd_mul(MF_C(11), y));
  dd p03 = dd_add(p01, dd_mul(p23, y2));
  dd p47 = dd_add(p45, dd_mul(p67, y2));
  dd p811 = dd_add(p89, dd_mul(p1011, y2));
  return dd_add(dd_add(p03, dd_mul(p47, y4)), dd_mul(dd_add(p811, dd_mul(MF_C(12), y4)), y8));
#undef MF_C
}

// sin_eval / cos_eval of trig.inc:165-187 without warp divergence.  The
// reference evaluates sin_kernel(r) or cos_kernel(r) when |r| <= pi/8, and
// both kernels at r -/+ pi/4 otherwise.  Here every thread evaluates both
// kernels at its own argument (r, or r -/+ pi/4) with the powers of x*x
// shared, then selects; each value is produced by exactly the reference's
// sequence of operations, so results are bit-identical.
__device__ __forceinline__ dd sincos_eval_one(dd r, bool want_sin) {
  const double pi8 = 0.392699081698724;
  const bool small = fabs(r.hi) <= pi8;
  const bool pos = r.hi > 0.0;
  dd pi4 = make(mf_pi_quarter_hi[0], mf_pi_quarter_lo[0]);
  dd arg = small ? r : (pos ? dd_sub(r, pi4) : dd_add(r, pi4));
  dd x2 = dd_mul(arg, arg);
  dd y2 = dd_mul(x2, x2);
  dd y4 = dd_mul(y2, y2);
  dd y8 = dd_mul(y4, y4);
  dd sk = dd_mul(neval12_pow(x2, y2, y4, y8, mf_sin_taylor_hi, mf_sin_taylor_lo), arg);
  dd ck = neval12_pow(x2, y2, y4, y8, mf_cos_taylor_hi, mf_cos_taylor_lo);
  if (small) return want_sin ? sk : ck;
  dd is2 = make(mf_inv_sqrt2_hi[0], mf_inv_sqrt2_lo[0]);
  dd u, v;
  if (want_sin) {
    u = sk;
    v = ck;  // pos: (sk + ck), neg: (sk - ck)
  } else {
    u = ck;
    v = neg(sk);  // pos: (ck - sk), neg: (ck + sk)
  }
  return pos ? dd_mul(dd_add(u, v), is2) : dd_mul(dd_sub(u, v), is2);
}
__device__ __forceinline__ bool trig_arg_too_large(double a) { return !(fabs(a) < 0x1p55); }

__device__ __forceinline__ dd dd_sin(dd x) {
  if (x.hi == 0.0 && x.lo == 0.0) return x;
  if (!isfinite(x.hi) || trig_arg_too_large(x.hi)) return make(qnan(), 0.0);
  int q;
  dd r = reduce_pi_half(x, q);
  // q=0: sin, q=1: cos, q=2: -sin, q=3: -cos
  dd v = sincos_eval_one(r, (q & 1) == 0);
  return (q & 2) ? neg(v) : v;
}
__device__ __forceinline__ dd dd_cos(dd x) {
  if (!isfinite(x.hi) || trig_arg_too_large(x.hi)) return make(qnan(), 0.0);
  int q;
  dd r = reduce_pi_half(x, q);
  // q=0: cos, q=1: -sin, q=2: -cos, q=3: sin
  dd v = sincos_eval_one(r, (q & 1) == 1);
  return (q == 1 || q == 2) ? neg(v) : v;
}

// ---- fused sin / cos (trig.inc:189-236): one reduction, both evaluations ----
// sincos_eval: the same two Taylor kernels and pi/4 shift as sin_eval and
// cos_eval, so each output equals the separate call bit for bit.
__device__ __forceinline__ void sincos_eval_both(dd r, dd &s, dd &c) {
  const double pi8 = 0.392699081698724;
  const bool small = fabs(r.hi) <= pi8;
  const bool pos = r.hi > 0.0;
  dd pi4 = make(mf_pi_quarter_hi[0], mf_pi_quarter_lo[0]);
  dd arg = small ? r : (pos ? dd_sub(r, pi4) : dd_add(r, pi4));
  dd x2 = dd_mul(arg, arg);
  dd y2 = dd_mul(x2, x2);
  dd y4 = dd_mul(y2, y2);
  dd y8 = dd_mul(y4, y4);
  dd sk = dd_mul(neval12_pow(x2, y2, y4, y8, mf_sin_taylor_hi, mf_sin_taylor_lo), arg);
  dd ck = neval12_pow(x2, y2, y4, y8, mf_cos_taylor_hi, mf_cos_taylor_lo);
  if (small) {
    s = sk;
    c = ck;
    return;
  }
  dd is2 = make(mf_inv_sqrt2_hi[0], mf_inv_sqrt2_lo[0]);
  s = pos ? dd_mul(dd_add(sk, ck), is2) : dd_mul(dd_sub(sk, ck), is2);
  c = pos ? dd_mul(dd_sub(ck, sk), is2) : dd_mul(dd_add(ck, sk), is2);
}
// sincos(x, s, c) (trig.inc:216-236)
__device__ __forceinline__ void dd_sincos(dd x, dd &s, dd &c) {
  if (!isfinite(x.hi) || trig_arg_too_large(x.hi)) {
    s = c = make(qnan(), 0.0);
    return;
  }
  if (x.hi == 0.0 && x.lo == 0.0) {  // sin(+-0) = +-0, cos(+-0) = 1
    s = x;
    c = make(1.0, 0.0);
    return;
  }
  int q;
  dd r = reduce_pi_half(x, q);
  dd ss, cc;
  sincos_eval_both(r, ss, cc);
  switch (q) {
    case 0: s = ss; c = cc; break;
    case 1: s = cc; c = neg(ss); break;
    case 2: s = neg(ss); c = neg(cc); break;
    default: s = neg(cc); c = ss; break;
  }
}

// ---- exp2 (exp_log.inc:109-128) ------------------------------------------
__device__ __forceinline__ dd dd_exp2(dd x) {
  const double h = x.hi;
  if (!isfinite(h)) return make(h < 0.0 ? 0.0 : h, 0.0);  // +inf, -inf -> 0, NaN
  if (h < mf_exp2_min[0]) return make(0.0, 0.0);
  if (h > mf_exp2_max[0]) return make(CUDART_INF, 0.0);
  double n_d = rint(h);
  double rh, rl, t;
  two_sum(h, -n_d, rh, t);
  rl = add(t, x.lo);
  fast_two_sum(rh, rl, rh, rl);
  return exp2_from_reduced(n_d, rh, rl);
}

// ---- log10 (exp_log.inc:344-353) -------------------------------------------
__device__ __forceinline__ dd dd_log10(dd x) {
  if (!isfinite(x.hi)) return make(log10(x.hi), 0.0);
  dd l2 = dd_log2(x);
  if (!isfinite(l2.hi)) return l2;
  return dd_mul(l2, make(mf_log10_2_hi[0], mf_log10_2_lo[0]));
}

// ---- complex exp (src/complex64x2/std.inc:20-74) ------------------------------
// exp(a + bi) = e^a (cos b + i sin b), with the C99 Annex G.6.3.1 special
// values handled first, as the reference does.
__device__ __forceinline__ void dd_cexp(dd a, dd b, dd &re, dd &im) {
  const double a_hi = a.hi, b_hi = b.hi;
  const bool b_zero = b_hi == 0.0 && b.lo == 0.0;
  if (!isfinite(a_hi) || !isfinite(b_hi)) {
    const dd nan2 = make(qnan(), 0.0), zero = make(0.0, 0.0), pinf = make(CUDART_INF, 0.0);
    if (isnan(a_hi)) {
      re = nan2;
      im = b_zero ? b : nan2;
      return;
    }
    if (isinf(b_hi)) {
      if (isinf(a_hi)) {
        if (a_hi > 0.0) {
          re = pinf;
          im = nan2;
        } else {
          re = zero;
          im = zero;
        }
        return;
      }
      re = im = nan2;
      return;
    }
    if (isnan(b_hi)) {
      if (a_hi > 0.0) {
        re = pinf;
        im = nan2;
      } else {
        re = zero;
        im = zero;
      }
      return;
    }
    // a = +-inf, b finite
    if (b_zero) {
      re = a_hi > 0.0 ? pinf : zero;
      im = b;
      return;
    }
    dd s, c;
    dd_sincos(b, s, c);
    const double mag = a_hi > 0.0 ? CUDART_INF : 0.0;
    re = make(copysign(mag, c.hi), 0.0);
    im = make(copysign(mag, s.hi), 0.0);
    return;
  }
  dd ea = dd_exp(a);
  dd s, c;
  dd_sincos(b, s, c);
  re = dd_mul(ea, c);
  im = dd_mul(ea, s);
}

// ---- compensated matmul MAC (src/float64x2/matmul.inc:6-39) ----------------
__device__ __forceinline__ void mac(double ah, double al, double bh, double bl, double& s_hi,
                                    double& s_lo) {
  double p = mul(ah, bh);
  double e = fma_(ah, bh, -p);
  double cross = fma_(ah, bl, mul(al, bh));
  double t = add(s_hi, p);
  double bp = sub(t, s_hi);
  double ap = sub(t, bp);
  double aerr = sub(s_hi, ap);
  double berr = sub(p, bp);
  s_lo = add(s_lo, add(add(e, cross), add(aerr, berr)));
  s_hi = t;
}
__device__ __forceinline__ void renorm(double& s_hi, double& s_lo) {
  double t = add(s_hi, s_lo);
  double bp = sub(t, s_hi);
  double ap = sub(t, bp);
  double aerr = sub(s_hi, ap);
  double berr = sub(s_lo, bp);
  s_lo = add(aerr, berr);
  s_hi = t;
}

}  // namespace mfdev
