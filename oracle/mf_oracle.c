/* ORACLE -- test infrastructure only.  Nothing in the product links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, as the checker.
 *
 * A plain-C (C99 + __int128) restatement of the multifloats 0.10.3 algorithms
 * on the array hot path, compiled with -ffp-contract=off so that every
 * operation rounds exactly as written (the reference pins the same flag,
 * src/CMakeLists.txt:105-118).  Each function cites the reference file:line it
 * follows.  Pinning: tests/test_oracle_pin.py compares these functions with
 * the reference library itself (built from the reference sources into
 * oracle/_ref/ by oracle/Makefile when the sources are present) and with the
 * golden vectors under tests/golden/ that the reference produced.
 *
 * Also here: the fixed blocked order of the device reductions, restated so the
 * GPU results can be checked bit for bit, and an exact superaccumulator used to
 * measure GEMM / dot errors in DD ulps (1 DD ulp = 2^-104).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MF_TABLE static const
#define MF_GTABLE static const
#include "../multifloats_b200/csrc/dd_tables.h"

typedef struct {
  double hi, lo;
} dd;

static dd mk(double h, double l) {
  dd r;
  r.hi = h;
  r.lo = l;
  return r;
}

/* ---- EFTs: include/multifloats/float64x2.h:84-107 ---------------------- */
static void two_sum(double a, double b, double *s, double *e) {
  double ss = a + b;
  double ap = ss - b;
  double bp = ss - ap;
  *e = (a - ap) + (b - bp);
  *s = ss;
}
static void fast_two_sum(double a, double b, double *s, double *e) {
  double ss = a + b;
  double bp = ss - a;
  *e = b - bp;
  *s = ss;
}
static void two_prod(double a, double b, double *p, double *e) {
  double pp = a * b;
  *e = fma(a, b, -pp);
  *p = pp;
}

/* ---- DD operators: float64x2.h:203-311 ---------------------------------- */
static dd dd_add(dd x, dd y) {
  double s = x.hi + y.hi;
  if (!isfinite(s)) return mk(s, 0.0);
  if (x.hi == 0.0 && y.hi == 0.0) return mk(s, x.lo + y.lo);
  double a, b, c, d;
  two_sum(x.hi, y.hi, &a, &b);
  two_sum(x.lo, y.lo, &c, &d);
  fast_two_sum(a, c, &a, &c);
  b += d;
  b += c;
  dd r;
  fast_two_sum(a, b, &r.hi, &r.lo);
  return r;
}
static dd dd_sub(dd x, dd y) {
  double s = x.hi - y.hi;
  if (!isfinite(s)) return mk(s, 0.0);
  if (x.hi == 0.0 && y.hi == 0.0) return mk(s, x.lo - y.lo);
  double a, b, c, d;
  two_sum(x.hi, -y.hi, &a, &b);
  two_sum(x.lo, -y.lo, &c, &d);
  fast_two_sum(a, c, &a, &c);
  b += d;
  b += c;
  dd r;
  fast_two_sum(a, b, &r.hi, &r.lo);
  return r;
}
static dd dd_mul(dd x, dd y) {
  double p00, e00;
  two_prod(x.hi, y.hi, &p00, &e00);
  if (!isfinite(p00)) return mk(p00, 0.0);
  double p01 = x.hi * y.lo;
  double p10 = x.lo * y.hi;
  p01 += p10;
  e00 += p01;
  dd r;
  fast_two_sum(p00, e00, &r.hi, &r.lo);
  return r;
}
static dd dd_div(dd x, dd y) {
  double q1 = x.hi / y.hi;
  if (!isfinite(q1)) return mk(q1, q1);
  if (!isfinite(y.hi)) return mk(q1, 0.0);
  double p00, e00;
  two_prod(q1, y.hi, &p00, &e00);
  double p01 = q1 * y.lo;
  double qhi = p00, qlo = e00 + p01;
  double r0, r0e;
  two_sum(x.hi, -qhi, &r0, &r0e);
  double r1 = (x.lo - qlo) + r0e;
  double rh, rl;
  fast_two_sum(r0, r1, &rh, &rl);
  double q2 = rh / y.hi;
  dd r;
  fast_two_sum(q1, q2, &r.hi, &r.lo);
  return r;
}
static dd dd_neg(dd a) { return mk(-a.hi, -a.lo); }

/* ---- sqrt: float64x2.h:2190-2212 ---------------------------------------- */
static dd dd_sqrt(dd x) {
  double c = sqrt(x.hi);
  if (!(x.hi > 0.0) || !isfinite(c)) return mk(c, 0.0);
  double u, uu;
  two_prod(c, c, &u, &uu);
  double cc = ((x.hi - u) - uu + x.lo) / (2.0 * c);
  dd r;
  r.hi = c + cc;
  r.lo = (c - r.hi) + cc;
  return r;
}

/* ---- polynomial evaluators: src/float64x2/poly.inc:9-102 ------------------ */
static dd horner(dd y, const double *hi, const double *lo, int n) {
  dd p = mk(hi[n - 1], lo[n - 1]);
  for (int i = n - 2; i >= 0; --i) p = dd_add(dd_mul(p, y), mk(hi[i], lo[i]));
  return p;
}
#define C_(i) mk(hi[i], lo[i])
static dd neval10(dd x, const double *hi, const double *lo) {
  dd x2 = dd_mul(x, x), x4 = dd_mul(x2, x2), x8 = dd_mul(x4, x4);
  dd p01 = dd_add(C_(0), dd_mul(C_(1), x));
  dd p23 = dd_add(C_(2), dd_mul(C_(3), x));
  dd p45 = dd_add(C_(4), dd_mul(C_(5), x));
  dd p67 = dd_add(C_(6), dd_mul(C_(7), x));
  dd p89 = dd_add(C_(8), dd_mul(C_(9), x));
  dd p03 = dd_add(p01, dd_mul(p23, x2));
  dd p47 = dd_add(p45, dd_mul(p67, x2));
  dd p810 = dd_add(p89, dd_mul(C_(10), x2));
  return dd_add(dd_add(p03, dd_mul(p47, x4)), dd_mul(p810, x8));
}
static dd neval12(dd x, const double *hi, const double *lo) {
  dd x2 = dd_mul(x, x), x4 = dd_mul(x2, x2), x8 = dd_mul(x4, x4);
  dd p01 = dd_add(C_(0), dd_mul(C_(1), x));
  dd p23 = dd_add(C_(2), dd_mul(C_(3), x));
  dd p45 = dd_add(C_(4), dd_mul(C_(5), x));
  dd p67 = dd_add(C_(6), dd_mul(C_(7), x));
  dd p89 = dd_add(C_(8), dd_mul(C_(9), x));
  dd p1011 = dd_add(C_(10), dd_mul(C_(11), x));
  dd p03 = dd_add(p01, dd_mul(p23, x2));
  dd p47 = dd_add(p45, dd_mul(p67, x2));
  dd p811 = dd_add(p89, dd_mul(p1011, x2));
  return dd_add(dd_add(p03, dd_mul(p47, x4)), dd_mul(dd_add(p811, dd_mul(C_(12), x4)), x8));
}
#undef C_

/* ---- exp: src/float64x2/exp_log.inc:26-72, :237-277 ---------------------- */
static dd exp2_from_reduced(double n_d, double rh, double rl) {
  if (n_d > 1100.0) return mk(INFINITY, 0.0);
  if (n_d < -1100.0) return mk(0.0, 0.0);
  double k_d = nearbyint(rh * 256.0);
  int k = (int)k_d;
  if (k > 128) k = 128;
  if (k < -128) k = -128;
  double sh = rh - (double)k / 256.0;
  double sl = rl;
  fast_two_sum(sh, sl, &sh, &sl);
  dd s = mk(sh, sl);
  dd q = mk(mf_exp2_coefs_hi[9], mf_exp2_coefs_lo[9]);
  for (int j = 8; j >= 1; --j) {
    q = dd_mul(q, s);
    q = dd_add(q, mk(mf_exp2_coefs_hi[j], mf_exp2_coefs_lo[j]));
  }
  dd pow2s = dd_add(mk(1.0, 0.0), dd_mul(s, q));
  dd T = mk(mf_exp2_table_hi[k + 128], mf_exp2_table_lo[k + 128]);
  dd m = dd_mul(T, pow2s);
  int n = (int)n_d;
  return mk(ldexp(m.hi, n), ldexp(m.lo, n));
}
static dd orc_exp1(dd x) {
  double h = x.hi;
  if (!isfinite(h)) {
    if (h > 0.0) return mk(h, 0.0);
    if (h < 0.0) return mk(0.0, 0.0);
    return mk(h, 0.0);
  }
  if (h > mf_exp_max[0]) return mk(INFINITY, 0.0);
  if (h < mf_exp_min[0]) return mk(0.0, 0.0);
  double n_d = nearbyint(h * mf_log2_e_hi[0]);
  double rh, rl, t;
  two_sum(h, -(n_d * mf_ln2_cw[0]), &rh, &t);
  rl = t + x.lo;
  fast_two_sum(rh, rl, &rh, &rl);
  double p_hi = n_d * mf_ln2_cw[1];
  double p_lo = fma(n_d, mf_ln2_cw[1], -p_hi);
  two_sum(rh, -p_hi, &rh, &t);
  rl += t - p_lo;
  fast_two_sum(rh, rl, &rh, &rl);
  two_sum(rh, -(n_d * mf_ln2_cw[2]), &rh, &t);
  rl += t;
  dd rr;
  fast_two_sum(rh, rl, &rr.hi, &rr.lo);
  dd y = dd_mul(rr, mk(mf_log2_e_hi[0], mf_log2_e_lo[0]));
  return exp2_from_reduced(n_d, y.hi, y.lo);
}

/* ---- log: exp_log.inc:280-341 -------------------------------------------- */
static dd log2_kernel(dd x) {
  double hi = x.hi;
  if (hi > 15.0 / 16.0 && hi < 17.0 / 16.0) {
    dd num = dd_sub(x, mk(1.0, 0.0));
    dd den = dd_add(x, mk(1.0, 0.0));
    dd t = dd_div(num, den);
    dd t2 = dd_mul(t, t);
    return dd_mul(t, neval10(t2, mf_log2_wide_hi, mf_log2_wide_lo));
  }
  int e = ilogb(hi);
  dd m = mk(ldexp(x.hi, -e), ldexp(x.lo, -e));
  int idx = (int)((m.hi - 1.0) * 32.0);
  if (idx < 0) idx = 0;
  if (idx > 31) idx = 31;
  dd c = mk(mf_log2_centers[idx], 0.0);
  dd v = mk(mf_log2_values_hi[idx], mf_log2_values_lo[idx]);
  dd t = dd_div(dd_sub(m, c), dd_add(m, c));
  dd t2 = dd_mul(t, t);
  dd p = horner(t2, mf_log2_narrow_hi, mf_log2_narrow_lo, 7);
  return dd_add(dd_add(mk((double)e, 0.0), v), dd_mul(t, p));
}
static dd orc_log2(dd x) {
  if (isnan(x.hi) || x.hi < 0.0) return mk(NAN, 0.0);
  if (x.hi == 0.0) return mk(-INFINITY, 0.0);
  if (!isfinite(x.hi)) return mk(INFINITY, 0.0);
  return log2_kernel(x);
}
static dd orc_log1(dd x) {
  if (!isfinite(x.hi)) return mk(log(x.hi), 0.0);
  dd l2 = orc_log2(x);
  if (!isfinite(l2.hi)) return l2;
  return dd_mul(l2, mk(mf_ln_2_hi[0], mf_ln_2_lo[0]));
}

/* ---- sin / cos: src/float64x2/trig.inc:114-266 ---------------------------- */
static void dd_sub_step(double *rh, double *rl, double ph, double pl) {
  double sh, sl, tl, tll;
  two_sum(*rh, -ph, &sh, &sl);
  two_sum(*rl, -pl, &tl, &tll);
  sl += tl;
  fast_two_sum(sh, sl, rh, rl);
  *rl += tll;
  fast_two_sum(*rh, *rl, rh, rl);
}
static dd reduce_pi_half(dd x, int *n_mod4) {
  double n_float = nearbyint(x.hi * 0.6366197723675814);
  double rh = x.hi, rl = x.lo, ph, pl;
  ph = n_float * mf_pi_half_cw[0];
  pl = fma(n_float, mf_pi_half_cw[0], -ph);
  dd_sub_step(&rh, &rl, ph, pl);
  ph = n_float * mf_pi_half_cw[1];
  pl = fma(n_float, mf_pi_half_cw[1], -ph);
  dd_sub_step(&rh, &rl, ph, pl);
  ph = n_float * mf_pi_half_cw[2];
  dd_sub_step(&rh, &rl, ph, 0.0);
  long long nn = (long long)fabs(n_float) & 3LL;
  if (n_float < 0.0) nn = (4 - nn) & 3;
  *n_mod4 = (int)nn;
  return mk(rh, rl);
}
static dd sin_kernel(dd x) {
  dd x2 = dd_mul(x, x);
  return dd_mul(neval12(x2, mf_sin_taylor_hi, mf_sin_taylor_lo), x);
}
static dd cos_kernel(dd x) {
  dd x2 = dd_mul(x, x);
  return neval12(x2, mf_cos_taylor_hi, mf_cos_taylor_lo);
}
static dd sin_eval(dd r) {
  const double pi8 = 0.392699081698724;
  if (fabs(r.hi) <= pi8) return sin_kernel(r);
  dd pi4 = mk(mf_pi_quarter_hi[0], mf_pi_quarter_lo[0]);
  dd is2 = mk(mf_inv_sqrt2_hi[0], mf_inv_sqrt2_lo[0]);
  int pos = r.hi > 0.0;
  dd rp = pos ? dd_sub(r, pi4) : dd_add(r, pi4);
  dd sk = sin_kernel(rp), ck = cos_kernel(rp);
  return pos ? dd_mul(dd_add(sk, ck), is2) : dd_mul(dd_sub(sk, ck), is2);
}
static dd cos_eval(dd r) {
  const double pi8 = 0.392699081698724;
  if (fabs(r.hi) <= pi8) return cos_kernel(r);
  dd pi4 = mk(mf_pi_quarter_hi[0], mf_pi_quarter_lo[0]);
  dd is2 = mk(mf_inv_sqrt2_hi[0], mf_inv_sqrt2_lo[0]);
  int pos = r.hi > 0.0;
  dd rp = pos ? dd_sub(r, pi4) : dd_add(r, pi4);
  dd sk = sin_kernel(rp), ck = cos_kernel(rp);
  return pos ? dd_mul(dd_sub(ck, sk), is2) : dd_mul(dd_add(ck, sk), is2);
}
static int trig_too_large(double a) { return !(fabs(a) < 0x1p55); }
static dd orc_sin1(dd x) {
  if (x.hi == 0.0 && x.lo == 0.0) return x;
  if (!isfinite(x.hi) || trig_too_large(x.hi)) return mk(NAN, 0.0);
  int q;
  dd r = reduce_pi_half(x, &q);
  switch (q) {
    case 0: return sin_eval(r);
    case 1: return cos_eval(r);
    case 2: return dd_neg(sin_eval(r));
    default: return dd_neg(cos_eval(r));
  }
}
static dd orc_cos1(dd x) {
  if (!isfinite(x.hi) || trig_too_large(x.hi)) return mk(NAN, 0.0);
  int q;
  dd r = reduce_pi_half(x, &q);
  switch (q) {
    case 0: return cos_eval(r);
    case 1: return dd_neg(sin_eval(r));
    case 2: return dd_neg(cos_eval(r));
    default: return sin_eval(r);
  }
}

/* ---- exp2 (exp_log.inc:109-128), log10 (exp_log.inc:344-353) ----------- */
static dd orc_exp2_1(dd x) {
  double h = x.hi;
  if (!isfinite(h)) return mk(h > 0.0 ? h : (h < 0.0 ? 0.0 : h), 0.0);
  if (h < mf_exp2_min[0]) return mk(0.0, 0.0);
  if (h > mf_exp2_max[0]) return mk(INFINITY, 0.0);
  double n_d = nearbyint(h);
  double rh, rl, t;
  two_sum(h, -n_d, &rh, &t);
  rl = t + x.lo;
  fast_two_sum(rh, rl, &rh, &rl);
  return exp2_from_reduced(n_d, rh, rl);
}
static dd orc_log10_1(dd x) {
  if (!isfinite(x.hi)) return mk(log10(x.hi), 0.0);
  dd l2 = orc_log2(x);
  if (!isfinite(l2.hi)) return l2;
  return dd_mul(l2, mk(mf_log10_2_hi[0], mf_log10_2_lo[0]));
}

/* ---- sincos (trig.inc:189-236): sincos_eval shares the kernels of the
 * pi/4-shifted argument between both outputs ----------------------------- */
static void sincos_eval(dd r, dd *s, dd *c) {
  const double pi8 = 0.392699081698724;
  if (fabs(r.hi) <= pi8) {
    *s = sin_kernel(r);
    *c = cos_kernel(r);
    return;
  }
  dd pi4 = mk(mf_pi_quarter_hi[0], mf_pi_quarter_lo[0]);
  dd is2 = mk(mf_inv_sqrt2_hi[0], mf_inv_sqrt2_lo[0]);
  int pos = r.hi > 0.0;
  dd rp = pos ? dd_sub(r, pi4) : dd_add(r, pi4);
  dd sk = sin_kernel(rp), ck = cos_kernel(rp);
  if (pos) {
    *s = dd_mul(dd_add(sk, ck), is2);
    *c = dd_mul(dd_sub(ck, sk), is2);
  } else {
    *s = dd_mul(dd_sub(sk, ck), is2);
    *c = dd_mul(dd_add(ck, sk), is2);
  }
}
static void orc_sincos1(dd x, dd *s, dd *c) {
  if (!isfinite(x.hi) || trig_too_large(x.hi)) {
    *s = *c = mk(NAN, 0.0);
    return;
  }
  if (x.hi == 0.0 && x.lo == 0.0) {
    *s = x;
    *c = mk(1.0, 0.0);
    return;
  }
  int q;
  dd r = reduce_pi_half(x, &q), ss, cc;
  sincos_eval(r, &ss, &cc);
  switch (q) {
    case 0: *s = ss; *c = cc; break;
    case 1: *s = cc; *c = dd_neg(ss); break;
    case 2: *s = dd_neg(ss); *c = dd_neg(cc); break;
    default: *s = dd_neg(cc); *c = ss; break;
  }
}

/* ---- complex exp (src/complex64x2/std.inc:20-74) ------------------------ */
static void orc_cexp1(dd a, dd b, dd *re, dd *im) {
  int b_zero = b.hi == 0.0 && b.lo == 0.0;
  if (!isfinite(a.hi) || !isfinite(b.hi)) {
    dd nan2 = mk(NAN, 0.0), zero = mk(0.0, 0.0), pinf = mk(INFINITY, 0.0);
    if (isnan(a.hi)) {
      *re = nan2;
      *im = b_zero ? b : nan2;
      return;
    }
    if (isinf(b.hi)) {
      if (isinf(a.hi)) {
        *re = a.hi > 0.0 ? pinf : zero;
        *im = a.hi > 0.0 ? nan2 : zero;
      } else {
        *re = *im = nan2;
      }
      return;
    }
    if (isnan(b.hi)) {
      *re = a.hi > 0.0 ? pinf : zero;
      *im = a.hi > 0.0 ? nan2 : zero;
      return;
    }
    if (b_zero) {
      *re = a.hi > 0.0 ? pinf : zero;
      *im = b;
      return;
    }
    dd sn, cs;
    orc_sincos1(b, &sn, &cs);
    double mag = a.hi > 0.0 ? INFINITY : 0.0;
    *re = mk(copysign(mag, cs.hi), 0.0);
    *im = mk(copysign(mag, sn.hi), 0.0);
    return;
  }
  dd ea = orc_exp1(a), sn, cs;
  orc_sincos1(b, &sn, &cs);
  *re = dd_mul(ea, cs);
  *im = dd_mul(ea, sn);
}

/* kind 0: sincos (s, c arrays); 1: cexpi (complex z = c + i s); 2: cexp */
void orc_pair(int kind, const double *x, double *y0, double *y1, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    dd a, b;
    if (kind == 2) {
      orc_cexp1(mk(x[4 * i], x[4 * i + 1]), mk(x[4 * i + 2], x[4 * i + 3]), &a, &b);
      y0[4 * i] = a.hi; y0[4 * i + 1] = a.lo; y0[4 * i + 2] = b.hi; y0[4 * i + 3] = b.lo;
    } else {
      orc_sincos1(mk(x[2 * i], x[2 * i + 1]), &a, &b);
      if (kind == 0) {
        y0[2 * i] = a.hi; y0[2 * i + 1] = a.lo; y1[2 * i] = b.hi; y1[2 * i + 1] = b.lo;
      } else {
        y0[4 * i] = b.hi; y0[4 * i + 1] = b.lo; y0[4 * i + 2] = a.hi; y0[4 * i + 3] = a.lo;
      }
    }
  }
}

/* ---- elementwise array maps (Fortran elemental, fypp:792-798) ---------- */
void orc_unary(int op, const double *x, double *y, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    dd v = mk(x[2 * i], x[2 * i + 1]), r;
    switch (op) {
      case 0: r = orc_exp1(v); break;
      case 1: r = orc_log1(v); break;
      case 2: r = orc_sin1(v); break;
      case 3: r = orc_cos1(v); break;
      case 5: r = orc_exp2_1(v); break;
      case 6: r = orc_log2(v); break;
      case 7: r = orc_log10_1(v); break;
      default: r = dd_sqrt(v); break;
    }
    y[2 * i] = r.hi;
    y[2 * i + 1] = r.lo;
  }
}

/* DD binary operators on arrays, for pinning the operators themselves. */
void orc_binary(int op, const double *a, const double *b, double *y, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    dd x = mk(a[2 * i], a[2 * i + 1]), z = mk(b[2 * i], b[2 * i + 1]), r;
    switch (op) {
      case 0: r = dd_add(x, z); break;
      case 1: r = dd_sub(x, z); break;
      case 2: r = dd_mul(x, z); break;
      default: r = dd_div(x, z); break;
    }
    y[2 * i] = r.hi;
    y[2 * i + 1] = r.lo;
  }
}

/* ---- matmul: src/float64x2/matmul.inc:6-39, :182-239 --------------------- */
static void mac(double ah, double al, double bh, double bl, double *s_hi, double *s_lo) {
  double p = ah * bh;
  double e = fma(ah, bh, -p);
  double cross = fma(ah, bl, al * bh);
  double t = *s_hi + p;
  double bp = t - *s_hi;
  double ap = t - bp;
  double aerr = *s_hi - ap;
  double berr = p - bp;
  *s_lo += (e + cross) + (aerr + berr);
  *s_hi = t;
}
static void renorm(double *s_hi, double *s_lo) {
  double t = *s_hi + *s_lo;
  double bp = t - *s_hi;
  double ap = t - bp;
  double aerr = *s_hi - ap;
  double berr = *s_lo - bp;
  *s_lo = aerr + berr;
  *s_hi = t;
}
/* One output: sum_p mac(x[p*sx], y[p*sy]) with the chunked renorm cadence. */
static dd mac_chain(const double *x, int64_t sx, const double *y, int64_t sy, int64_t k,
                    int64_t ri) {
  double sh = 0.0, sl = 0.0;
  int64_t cnt = 0;
  for (int64_t p = 0; p < k; ++p) {
    mac(x[2 * p * sx], x[2 * p * sx + 1], y[2 * p * sy], y[2 * p * sy + 1], &sh, &sl);
    if (ri > 0 && ++cnt == ri) {
      cnt = 0;
      if (p + 1 < k) renorm(&sh, &sl);
    }
  }
  renorm(&sh, &sl);
  return mk(sh, sl);
}
/* C(m,n) = A(m,k) B(k,n), column-major; rows [i0,i1) x cols [j0,j1) only. */
void orc_matmul_mm_block(const double *a, const double *b, double *c, int64_t m, int64_t k,
                         int64_t n, int64_t ri, int64_t i0, int64_t i1, int64_t j0, int64_t j1) {
  (void)n;
  for (int64_t j = j0; j < j1; ++j)
    for (int64_t i = i0; i < i1; ++i) {
      dd r = mac_chain(a + 2 * i, m, b + 2 * j * k, 1, k, ri);
      c[2 * (j * m + i)] = r.hi;
      c[2 * (j * m + i) + 1] = r.lo;
    }
}
void orc_matmul_mm(const double *a, const double *b, double *c, int64_t m, int64_t k, int64_t n,
                   int64_t ri) {
  orc_matmul_mm_block(a, b, c, m, k, n, ri, 0, m, 0, n);
}
void orc_matmul_mv(const double *a, const double *x, double *y, int64_t m, int64_t k, int64_t ri) {
  for (int64_t i = 0; i < m; ++i) {
    dd r = mac_chain(a + 2 * i, m, x, 1, k, ri);
    y[2 * i] = r.hi;
    y[2 * i + 1] = r.lo;
  }
}
void orc_matmul_vm(const double *x, const double *b, double *y, int64_t k, int64_t n, int64_t ri) {
  for (int64_t j = 0; j < n; ++j) {
    dd r = mac_chain(x, 1, b + 2 * j * k, 1, k, ri);
    y[2 * j] = r.hi;
    y[2 * j + 1] = r.lo;
  }
}
/* Fortran cdd_matmul_mm (fypp:2609-2621): 4 real products on the split
 * parts, re = mm(ar,br) - mm(ai,bi), im = mm(ar,bi) + mm(ai,br). */
void orc_cmatmul_mm(const double *a, const double *b, double *c, int64_t m, int64_t k, int64_t n,
                    int64_t ri) {
  for (int64_t j = 0; j < n; ++j)
    for (int64_t i = 0; i < m; ++i) {
      const double *ar = a + 4 * i, *ai = a + 4 * i + 2;
      const double *br = b + 4 * j * k, *bi = b + 4 * j * k + 2;
      dd rr = mac_chain(ar, 2 * m, br, 2, k, ri);
      dd ii = mac_chain(ai, 2 * m, bi, 2, k, ri);
      dd rim = mac_chain(ar, 2 * m, bi, 2, k, ri);
      dd irm = mac_chain(ai, 2 * m, br, 2, k, ri);
      dd re = dd_sub(rr, ii), im = dd_add(rim, irm);
      double *o = c + 4 * (j * m + i);
      o[0] = re.hi;
      o[1] = re.lo;
      o[2] = im.hi;
      o[3] = im.lo;
    }
}

/* ---- Fortran reductions, serial (fsrc/multifloats.fypp) ----------------- */
typedef struct {
  double hi, lo;
} acc2;
/* dd_sum_1d per-element update (fypp:1994-1999) */
static void sum_step(acc2 *s, double xh, double xl) {
  double t = s->hi + xh;
  double bp = t - s->hi;
  double ap = t - bp;
  double aerr = s->hi - ap;
  double berr = xh - bp;
  s->lo = s->lo + ((xl + aerr) + berr);
  s->hi = t;
}
static dd sum_finish_fast(acc2 s) { /* fypp:2004-2006 */
  double t = s.hi + s.lo;
  double bp = t - s.hi;
  return mk(t, s.lo - bp);
}
static dd sum_finish_full(acc2 s) { /* fypp:2143-2152 */
  double t = s.hi + s.lo;
  double bp = t - s.hi;
  double ap = t - bp;
  double aerr = s.hi - ap;
  double berr = s.lo - bp;
  return mk(t, aerr + berr);
}
/* dd_dot_product per-element update (fypp:2288-2298) */
static void dot_step(acc2 *s, double ah, double al, double bh, double bl) {
  double p = ah * bh;
  double e = fma(ah, bh, -p);
  double cross = ah * bl + al * bh;
  double t = s->hi + p;
  double bp = t - s->hi;
  double ap = t - bp;
  double aerr = s->hi - ap;
  double berr = p - bp;
  s->lo = s->lo + (((e + cross) + aerr) + berr);
  s->hi = t;
}
static void dot_block_renorm(acc2 *s) { /* fypp:2301-2302 */
  double t = s->hi + s->lo;
  double bp = t - s->hi;
  s->hi = t;
  s->lo = s->lo - bp;
}
static dd dot_finish(acc2 s) { /* fypp:2304-2307 */
  double t = s.hi + s.lo;
  double bp = t - s.hi;
  return mk(t, s.lo - bp);
}

/* Serial dot over elements x[i*sx], y[i*sy] (stride in DD units). */
static dd dot_serial_strided(const double *x, int64_t sx, const double *y, int64_t sy, int64_t n,
                             int64_t ri) {
  acc2 s = {0.0, 0.0};
  if (ri <= 0) {
    for (int64_t i = 0; i < n; ++i)
      dot_step(&s, x[2 * i * sx], x[2 * i * sx + 1], y[2 * i * sy], y[2 * i * sy + 1]);
  } else {
    for (int64_t kk = 0; kk < n; kk += ri) {
      int64_t ke = kk + ri < n ? kk + ri : n;
      for (int64_t i = kk; i < ke; ++i)
        dot_step(&s, x[2 * i * sx], x[2 * i * sx + 1], y[2 * i * sy], y[2 * i * sy + 1]);
      dot_block_renorm(&s);
    }
  }
  return dot_finish(s);
}

void orc_sum_serial(const double *x, int64_t n, double *out) {
  acc2 s = {0.0, 0.0};
  for (int64_t i = 0; i < n; ++i) sum_step(&s, x[2 * i], x[2 * i + 1]);
  dd r = sum_finish_fast(s);
  out[0] = r.hi;
  out[1] = r.lo;
}
void orc_csum_serial(const double *x, int64_t n, double *out) {
  acc2 re = {0.0, 0.0}, im = {0.0, 0.0};
  for (int64_t i = 0; i < n; ++i) {
    sum_step(&re, x[4 * i], x[4 * i + 1]);
    sum_step(&im, x[4 * i + 2], x[4 * i + 3]);
  }
  dd r = sum_finish_full(re), q = sum_finish_full(im);
  out[0] = r.hi;
  out[1] = r.lo;
  out[2] = q.hi;
  out[3] = q.lo;
}
void orc_dot_serial(const double *a, const double *b, int64_t n, int64_t ri, double *out) {
  dd r = dot_serial_strided(a, 1, b, 1, n, ri);
  out[0] = r.hi;
  out[1] = r.lo;
}
/* cdd_dot_product (fypp:2321-2331): conj(a).b */
void orc_cdot_serial(const double *a, const double *b, int64_t n, int64_t ri, double *out) {
  dd rr = dot_serial_strided(a, 2, b, 2, n, ri);
  dd ii = dot_serial_strided(a + 2, 2, b + 2, 2, n, ri);
  dd rim = dot_serial_strided(a, 2, b + 2, 2, n, ri);
  dd irm = dot_serial_strided(a + 2, 2, b, 2, n, ri);
  dd re = dd_add(rr, ii), im = dd_sub(rim, irm);
  out[0] = re.hi;
  out[1] = re.lo;
  out[2] = im.hi;
  out[3] = im.lo;
}
/* dd_norm2_1d (fypp:2338-2352) */
void orc_norm2_serial(const double *x, int64_t n, double *out) {
  dd s = mk(0.0, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    dd a = mk(x[2 * i], x[2 * i + 1]);
    s = dd_add(s, dd_mul(a, a));
  }
  dd r = dd_sqrt(s);
  out[0] = r.hi;
  out[1] = r.lo;
}
/* complex norm2 = norm2 of the 2n real parts in storage order */
void orc_cnorm2_serial(const double *x, int64_t n, double *out) { orc_norm2_serial(x, 2 * n, out); }

/* ---- the device's fixed blocked order, restated -------------------------- */
#define R_THREADS 256
#define R_MAX_BLOCKS 2048
#define R_PER_THREAD_MIN 16
void orc_reduce_geometry(int64_t n, int64_t *blocks, int64_t *threads) {
  int64_t per_block = (int64_t)R_THREADS * R_PER_THREAD_MIN;
  int64_t b = (n + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > R_MAX_BLOCKS) b = R_MAX_BLOCKS;
  *blocks = b;
  *threads = R_THREADS;
}
/* warp shuffle-down tree over v[0..31] per warp, then warps 0..7 -> v[0] */
static void block_tree(dd *v, int nv) {
  dd wp[R_THREADS / 32][4];
  for (int w = 0; w < R_THREADS / 32; ++w) {
    dd *lane = v + (int64_t)w * 32 * nv;
    for (int off = 16; off >= 1; off >>= 1)
      for (int l = 0; l < off; ++l)
        for (int q = 0; q < nv; ++q) lane[l * nv + q] = dd_add(lane[l * nv + q], lane[(l + off) * nv + q]);
    for (int q = 0; q < nv; ++q) wp[w][q] = lane[q];
  }
  for (int off = (R_THREADS / 32) / 2; off >= 1; off >>= 1)
    for (int l = 0; l < off; ++l)
      for (int q = 0; q < nv; ++q) wp[l][q] = dd_add(wp[l][q], wp[l + off][q]);
  for (int q = 0; q < nv; ++q) v[q] = wp[0][q];
}
/* kind: 0 sum, 1 dot, 2 norm2, 3 csum, 4 cdot, 5 cnorm2 (same as the device) */
/* The final step of each kind on the fully combined values (reduce_dd.cu
 * finish_kind). */
static void reduce_finish(int kind, const dd *v, double *out) {
  dd r0 = v[0], r1 = mk(0.0, 0.0);
  if (kind == 2 || kind == 5) r0 = dd_sqrt(v[0]);
  if (kind == 3) r1 = v[1];
  if (kind == 4) {
    r0 = dd_add(v[0], v[1]);
    r1 = dd_sub(v[2], v[3]);
  }
  out[0] = r0.hi;
  out[1] = r0.lo;
  if (kind == 3 || kind == 4) {
    out[2] = r1.hi;
    out[3] = r1.lo;
  }
}

static void reduce_blocked_impl(int kind, const double *x, const double *y, int64_t n, int64_t ri,
                                double *out, int final);

void orc_reduce_blocked(int kind, const double *x, const double *y, int64_t n, int64_t ri,
                        double *out) {
  reduce_blocked_impl(kind, x, y, n, ri, out, 1);
}

/* The device's partial for a cross-device combine (mfcuda_reduce_partial):
 * the NV combined values before the final step, as hi/lo pairs. */
void orc_reduce_blocked_partial(int kind, const double *x, const double *y, int64_t n, int64_t ri,
                                double *out) {
  reduce_blocked_impl(kind, x, y, n, ri, out, 0);
}

/* mfcuda_reduce_combine: partials of `count` devices (NV hi/lo pairs each, in
 * rank order) folded left to right with DD add, then the final step. */
void orc_reduce_combine(int kind, const double *parts, int64_t count, double *out) {
  static const int NV[6] = {1, 1, 1, 2, 4, 1};
  int nv = NV[kind];
  dd v[4];
  for (int q = 0; q < nv; ++q) v[q] = mk(parts[2 * q], parts[2 * q + 1]);
  for (int64_t r = 1; r < count; ++r)
    for (int q = 0; q < nv; ++q)
      v[q] = dd_add(v[q], mk(parts[2 * (r * nv + q)], parts[2 * (r * nv + q) + 1]));
  reduce_finish(kind, v, out);
}

static void reduce_blocked_impl(int kind, const double *x, const double *y, int64_t n, int64_t ri,
                                double *out, int final) {
  static const int NV[6] = {1, 1, 1, 2, 4, 1};
  static const int E[6] = {2, 2, 2, 4, 4, 4};
  int nv = NV[kind], e = E[kind];
  int64_t B, TPB;
  orc_reduce_geometry(n, &B, &TPB);
  int64_t T = B * TPB;
  dd *part = (dd *)malloc(sizeof(dd) * (size_t)B * nv);
  dd *v = (dd *)malloc(sizeof(dd) * R_THREADS * nv);
  for (int64_t b = 0; b < B; ++b) {
    for (int t = 0; t < R_THREADS; ++t) {
      int64_t g = b * R_THREADS + t;
      dd *o = v + (int64_t)t * nv;
      if (kind == 0 || kind == 3) {
        acc2 s[2] = {{0.0, 0.0}, {0.0, 0.0}};
        for (int64_t i = g; i < n; i += T)
          for (int q = 0; q < nv; ++q) sum_step(&s[q], x[e * i + 2 * q], x[e * i + 2 * q + 1]);
        for (int q = 0; q < nv; ++q) o[q] = kind == 0 ? sum_finish_fast(s[q]) : sum_finish_full(s[q]);
      } else if (kind == 1 || kind == 4) {
        acc2 d[4] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
        int64_t cnt = 0;
        for (int64_t i = g; i < n; i += T) {
          if (kind == 1) {
            dot_step(&d[0], x[2 * i], x[2 * i + 1], y[2 * i], y[2 * i + 1]);
          } else {
            const double *a = x + 4 * i, *bb = y + 4 * i;
            dot_step(&d[0], a[0], a[1], bb[0], bb[1]);
            dot_step(&d[1], a[2], a[3], bb[2], bb[3]);
            dot_step(&d[2], a[0], a[1], bb[2], bb[3]);
            dot_step(&d[3], a[2], a[3], bb[0], bb[1]);
          }
          if (ri > 0 && ++cnt == ri) {
            cnt = 0;
            for (int q = 0; q < nv; ++q) dot_block_renorm(&d[q]);
          }
        }
        if (ri > 0 && cnt > 0)
          for (int q = 0; q < nv; ++q) dot_block_renorm(&d[q]);
        for (int q = 0; q < nv; ++q) o[q] = dot_finish(d[q]);
      } else {
        dd s = mk(0.0, 0.0);
        for (int64_t i = g; i < n; i += T) {
          dd a = mk(x[e * i], x[e * i + 1]);
          s = dd_add(s, dd_mul(a, a));
          if (kind == 5) {
            dd bq = mk(x[e * i + 2], x[e * i + 3]);
            s = dd_add(s, dd_mul(bq, bq));
          }
        }
        o[0] = s;
      }
    }
    block_tree(v, nv);
    for (int q = 0; q < nv; ++q) part[b * nv + q] = v[q];
  }
  for (int t = 0; t < R_THREADS; ++t)
    for (int q = 0; q < nv; ++q) v[(int64_t)t * nv + q] = mk(0.0, 0.0);
  for (int t = 0; t < R_THREADS; ++t)
    for (int64_t b = t; b < B; b += R_THREADS)
      for (int q = 0; q < nv; ++q) {
        dd p = part[b * nv + q];
        v[(int64_t)t * nv + q] = (b == t) ? p : dd_add(v[(int64_t)t * nv + q], p);
      }
  block_tree(v, nv);
  if (final) {
    reduce_finish(kind, v, out);
  } else {
    for (int q = 0; q < nv; ++q) {
      out[2 * q] = v[q].hi;
      out[2 * q + 1] = v[q].lo;
    }
  }
  free(part);
  free(v);
}

/* ---- exact superaccumulator ------------------------------------------------
 * Fixed-point accumulator over bit positions 2^SA_EMIN .. 2^(SA_EMIN+32*SA_LIMBS);
 * limbs are 32-bit digits held in int64 so that up to 2^30 additions need no
 * carry propagation.  A product of two doubles is added exactly as the 106-bit
 * integer product of their significands. */
#define SA_EMIN (-2400)
#define SA_LIMBS 144
typedef struct {
  int64_t d[SA_LIMBS];
} superacc;

static void sa_add_int128(superacc *s, __int128 v, int e) {
  /* adds v * 2^e */
  if (v == 0) return;
  int neg = v < 0;
  unsigned __int128 u = neg ? (unsigned __int128)(-v) : (unsigned __int128)v;
  int pos = e - SA_EMIN;
  if (pos < 0) return; /* below 2^-2400: far under any DD error of interest */
  int limb = pos >> 5, sh = pos & 31;
  /* u << sh spans up to 128+31 bits: emit 32-bit pieces */
  unsigned __int128 lo = u << sh;
  unsigned __int128 hi = sh ? (u >> (128 - sh)) : 0;
  for (int i = 0; i < 5; ++i) {
    int64_t piece;
    if (i < 4)
      piece = (int64_t)((lo >> (32 * i)) & 0xffffffffu);
    else
      piece = (int64_t)(hi & 0xffffffffu);
    if (piece && limb + i < SA_LIMBS) s->d[limb + i] += neg ? -piece : piece;
  }
}
static void sa_add_double(superacc *s, double x) {
  if (x == 0.0 || !isfinite(x)) return;
  int ex;
  double f = frexp(x, &ex); /* x = f * 2^ex, 0.5 <= |f| < 1 */
  int64_t mant = (int64_t)ldexp(f, 53);
  sa_add_int128(s, (__int128)mant, ex - 53);
}
static void sa_add_prod(superacc *s, double a, double b) {
  if (a == 0.0 || b == 0.0 || !isfinite(a) || !isfinite(b)) return;
  int ea, eb;
  double fa = frexp(a, &ea), fb = frexp(b, &eb);
  int64_t ma = (int64_t)ldexp(fa, 53), mb = (int64_t)ldexp(fb, 53);
  sa_add_int128(s, (__int128)ma * (__int128)mb, ea + eb - 106);
}
static void sa_carry(superacc *s) {
  for (int i = 0; i < SA_LIMBS - 1; ++i) {
    int64_t c = s->d[i] >> 32; /* arithmetic shift: floor division */
    s->d[i] -= c * ((int64_t)1 << 32);
    s->d[i + 1] += c;
  }
}
static double sa_value(superacc *s) {
  /* canonical digits in [0, 2^32) below a signed top limb */
  sa_carry(s);
  int top = SA_LIMBS - 1;
  while (top > 0 && s->d[top] == 0) --top;
  double sign = 1.0;
  if (s->d[top] < 0) { /* negate to sign-magnitude */
    for (int i = 0; i < SA_LIMBS; ++i) s->d[i] = -s->d[i];
    sa_carry(s);
    sign = -1.0;
    top = SA_LIMBS - 1;
    while (top > 0 && s->d[top] == 0) --top;
  }
  double v = 0.0;
  for (int i = top; i >= 0 && i >= top - 3; --i) v += ldexp((double)s->d[i], 32 * i + SA_EMIN);
  return sign * v;
}

/* For selected outputs (i, j) of C = A B (column-major, DD), the exact error
 * err = C_ij - (A B)_ij rounded to double, and absab = (|A||B|)_ij in double.
 * complex_parts: 0 for real matrices. */
void orc_gemm_errors(const double *a, const double *b, const double *c, int64_t m, int64_t k,
                     int64_t n, const int64_t *ii, const int64_t *jj, int64_t count, double *err,
                     double *absab) {
  (void)n;
  for (int64_t q = 0; q < count; ++q) {
    int64_t i = ii[q], j = jj[q];
    superacc s;
    memset(&s, 0, sizeof(s));
    double ab = 0.0;
    for (int64_t p = 0; p < k; ++p) {
      double ah = a[2 * (p * m + i)], al = a[2 * (p * m + i) + 1];
      double bh = b[2 * (j * k + p)], bl = b[2 * (j * k + p) + 1];
      sa_add_prod(&s, ah, bh);
      sa_add_prod(&s, ah, bl);
      sa_add_prod(&s, al, bh);
      sa_add_prod(&s, al, bl);
      ab += fabs(ah + al) * fabs(bh + bl);
    }
    sa_add_double(&s, -c[2 * (j * m + i)]);
    sa_add_double(&s, -c[2 * (j * m + i) + 1]);
    err[q] = -sa_value(&s);
    absab[q] = ab;
  }
}

/* Exact error of a DD reduction result: kind 0 sum, 1 dot (real only).
 * err = result - exact, abs = sum |x| or sum |a||b|. */
void orc_reduce_error(int kind, const double *x, const double *y, int64_t n, const double *res,
                      double *err, double *absv) {
  superacc s;
  memset(&s, 0, sizeof(s));
  double ab = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    if (kind == 0) {
      sa_add_double(&s, x[2 * i]);
      sa_add_double(&s, x[2 * i + 1]);
      ab += fabs(x[2 * i] + x[2 * i + 1]);
    } else {
      double ah = x[2 * i], al = x[2 * i + 1], bh = y[2 * i], bl = y[2 * i + 1];
      sa_add_prod(&s, ah, bh);
      sa_add_prod(&s, ah, bl);
      sa_add_prod(&s, al, bh);
      sa_add_prod(&s, al, bl);
      ab += fabs(ah + al) * fabs(bh + bl);
    }
  }
  sa_add_double(&s, -res[0]);
  sa_add_double(&s, -res[1]);
  *err = -sa_value(&s);
  *absv = ab;
}

/* ---- split-INT8 GEMM, restated on the CPU ------------------------------------
 * The same algorithm as the device kernels in split_gemm.cu (scan, plan,
 * exact rounding to (8S-2)-bit integers, balanced signed 8-bit digits, exact
 * integer anti-diagonal sums D_g per K chunk, DD combine chunk by chunk, each
 * from the smallest diagonal up, exact scaling).  The integer stage is exact and the combine
 * order is fixed, so the device result must match this bit for bit. */
#define SPLIT_SMAX 14
#define SPLIT_KC (73 * 128) /* K elements per chunk, as KC_BLOCKS * BK on the device */
/* The rounding of an entry to the W-bit grid of its row / column
 * (t = W - sigma), IEEE double operations rounding to nearest even:
 *   H = ldexp(hi, t), L = ldexp(lo, t), P = rint(H), X = P + rint((H - P) + L),
 * clamped to |X| <= 2^W - 1.  |X - (hi + lo) 2^t| <= 1. */
static __int128 split_round(double hi, double lo, int sigma, int W) {
  int t = W - sigma;
  double H = ldexp(hi, t), L = ldexp(lo, t);
  double P = rint(H);
  double Q = rint((H - P) + L);
  __int128 X = (__int128)P + (__int128)Q;
  __int128 lim = ((__int128)1 << W) - 1;
  if (X > lim) X = lim;
  if (X < -lim) X = -lim;
  return X;
}
/* X of split_round as two 64-bit words (low, high; two's complement). */
void orc_grid_round(double hi, double lo, int sigma, int W, int64_t *out) {
  __int128 X = split_round(hi, lo, sigma, W);
  out[0] = (int64_t)(uint64_t)X;
  out[1] = (int64_t)(X >> 64);
}
static void split_digits(double hi, double lo, int sigma, int S, int W, int8_t *d) {
  __int128 X = split_round(hi, lo, sigma, W);
  for (int s = S - 1; s >= 1; --s) {
    int v = (int)(X & 0xFF);
    v = (v ^ 0x80) - 0x80;
    d[s] = (int8_t)v;
    X = (X - v) >> 8;
  }
  d[0] = (int8_t)X;
}
/* exponent statistics of one row/column: elements x[idx*stride] */
static void split_stats(const double *x, int64_t count, int64_t stride, int *sig, int *mu, int *bad) {
  int hi_e = -100000, lo_e = 100000, b = 0;
  for (int64_t p = 0; p < count; ++p) {
    double h = x[2 * p * stride], l = x[2 * p * stride + 1];
    if (!isfinite(h) || !isfinite(l)) {
      b = 1;
      continue;
    }
    double a = fabs(h) + fabs(l);
    if (a != 0.0) {
      int e = ilogb(a);
      if (e + 1 > hi_e) hi_e = e + 1;
      if (e < lo_e) lo_e = e;
    }
  }
  *sig = hi_e;
  *mu = lo_e;
  *bad = b;
}
int orc_split_plan(int S_req, double target, int rho_a, int rho_b) {
  if (S_req > 0) return S_req;
  for (int s = 2; s <= SPLIT_SMAX; ++s)
    if ((s + 1) * ldexp(1.0, 106 - 8 * s + rho_a + rho_b) <= target) return s;
  return SPLIT_SMAX;
}
/* info[0..2] = S, rho_a, rho_b; kc = K chunk length in elements (<= SPLIT_KC) */
void orc_split_gemm_kc(const double *a, const double *b, double *c, int64_t m, int64_t k, int64_t n,
                       int S_req, double target, int *info, int64_t kc_len);
void orc_split_gemm(const double *a, const double *b, double *c, int64_t m, int64_t k, int64_t n,
                    int S_req, double target, int *info) {
  orc_split_gemm_kc(a, b, c, m, k, n, S_req, target, info, SPLIT_KC);
}
void orc_split_gemm_kc(const double *a, const double *b, double *c, int64_t m, int64_t k, int64_t n,
                       int S_req, double target, int *info, int64_t kc_len) {
  int *sa = malloc(sizeof(int) * m), *ma = malloc(sizeof(int) * m), *fa = malloc(sizeof(int) * m);
  int *sb = malloc(sizeof(int) * n), *mb = malloc(sizeof(int) * n), *fb = malloc(sizeof(int) * n);
  int ra = 0, rb = 0;
  for (int64_t i = 0; i < m; ++i) {
    split_stats(a + 2 * i, k, m, &sa[i], &ma[i], &fa[i]);
    if (sa[i] != -100000 && sa[i] - ma[i] > ra) ra = sa[i] - ma[i];
  }
  for (int64_t j = 0; j < n; ++j) {
    split_stats(b + 2 * j * k, k, 1, &sb[j], &mb[j], &fb[j]);
    if (sb[j] != -100000 && sb[j] - mb[j] > rb) rb = sb[j] - mb[j];
  }
  for (int64_t i = 0; i < m; ++i)
    if (sa[i] == -100000) sa[i] = 0;
  for (int64_t j = 0; j < n; ++j)
    if (sb[j] == -100000) sb[j] = 0;
  int S = orc_split_plan(S_req, target, ra, rb), G = S - 1, W = 8 * S - 2;
  if (info) {
    info[0] = S;
    info[1] = ra;
    info[2] = rb;
  }
  int8_t *da = calloc((size_t)S * m * k, 1), *db = calloc((size_t)S * n * k, 1);
  for (int64_t i = 0; i < m; ++i)
    for (int64_t p = 0; p < k; ++p) {
      int8_t d[SPLIT_SMAX];
      if (fa[i]) continue;
      split_digits(a[2 * (p * m + i)], a[2 * (p * m + i) + 1], sa[i], S, W, d);
      for (int s = 0; s < S; ++s) da[((size_t)s * m + i) * k + p] = d[s];
    }
  for (int64_t j = 0; j < n; ++j)
    for (int64_t p = 0; p < k; ++p) {
      int8_t d[SPLIT_SMAX];
      if (fb[j]) continue;
      split_digits(b[2 * (j * k + p)], b[2 * (j * k + p) + 1], sb[j], S, W, d);
      for (int s = 0; s < S; ++s) db[((size_t)s * n + j) * k + p] = d[s];
    }
  int64_t nkc = (k + kc_len - 1) / kc_len;
  if (nkc < 1) nkc = 1;
  for (int64_t j = 0; j < n; ++j)
    for (int64_t i = 0; i < m; ++i) {
      double hi = 0.0, lo = 0.0;
      for (int64_t kc = 0; kc < nkc; ++kc) {
        for (int g = G; g >= 0; --g) {
          double scale = ldexp(1.0, -8 * g);
          int64_t p0 = kc * kc_len, p1 = p0 + kc_len < k ? p0 + kc_len : k;
          int64_t D = 0;
          for (int s = 0; s <= g; ++s) {
            const int8_t *ra_ = da + ((size_t)s * m + i) * k;
            const int8_t *rb_ = db + ((size_t)(g - s) * n + j) * k;
            for (int64_t p = p0; p < p1; ++p) D += (int64_t)ra_[p] * rb_[p];
          }
          double tv = (double)(int32_t)D * scale;
          double s_, e_;
          two_sum(hi, tv, &s_, &e_);
          hi = s_;
          lo = lo + e_;
        }
      }
      double h2, l2;
      two_sum(hi, lo, &h2, &l2);
      double *o = c + 2 * (j * m + i);
      if (fa[i] | fb[j]) {
        o[0] = NAN;
        o[1] = 0.0;
      } else {
        int ex = sa[i] + sb[j] - 12;
        o[0] = ldexp(h2, ex);
        o[1] = ldexp(l2, ex);
      }
    }
  free(sa); free(ma); free(fa); free(sb); free(mb); free(fb); free(da); free(db);
}

/* Complex split GEMM: re = Ar Br - Ai Bi, im = Ar Bi + Ai Br, each real
 * product by orc_split_gemm with one slice count S chosen from the exponent
 * spreads of all four operands (A side: Ar, Ai rows; B side: Br, Bi columns). */
void orc_split_cgemm_kc(const double *a, const double *b, double *c, int64_t m, int64_t k, int64_t n,
                        int S_req, double target, int *info, int64_t kc);
void orc_split_cgemm(const double *a, const double *b, double *c, int64_t m, int64_t k, int64_t n,
                     int S_req, double target, int *info) {
  orc_split_cgemm_kc(a, b, c, m, k, n, S_req, target, info, SPLIT_KC);
}
/* Complex split product with K chunks of kc elements in each real product
 * (the batched form may use shorter chunks than the single call). */
void orc_split_cgemm_kc(const double *a, const double *b, double *c, int64_t m, int64_t k, int64_t n,
                        int S_req, double target, int *info, int64_t kc) {
  double *ar = malloc(sizeof(double) * 2 * m * k), *ai = malloc(sizeof(double) * 2 * m * k);
  double *br = malloc(sizeof(double) * 2 * k * n), *bi = malloc(sizeof(double) * 2 * k * n);
  for (int64_t e = 0; e < m * k; ++e) {
    ar[2 * e] = a[4 * e]; ar[2 * e + 1] = a[4 * e + 1];
    ai[2 * e] = a[4 * e + 2]; ai[2 * e + 1] = a[4 * e + 3];
  }
  for (int64_t e = 0; e < k * n; ++e) {
    br[2 * e] = b[4 * e]; br[2 * e + 1] = b[4 * e + 1];
    bi[2 * e] = b[4 * e + 2]; bi[2 * e + 1] = b[4 * e + 3];
  }
  int ra = 0, rb = 0;
  for (int part = 0; part < 2; ++part) {
    const double *x = part ? ai : ar, *y = part ? bi : br;
    for (int64_t i = 0; i < m; ++i) {
      int sg, mu, bad;
      split_stats(x + 2 * i, k, m, &sg, &mu, &bad);
      if (sg != -100000 && sg - mu > ra) ra = sg - mu;
    }
    for (int64_t j = 0; j < n; ++j) {
      int sg, mu, bad;
      split_stats(y + 2 * j * k, k, 1, &sg, &mu, &bad);
      if (sg != -100000 && sg - mu > rb) rb = sg - mu;
    }
  }
  int S = orc_split_plan(S_req, target, ra, rb);
  if (info) {
    info[0] = S;
    info[1] = ra;
    info[2] = rb;
  }
  double *rr = malloc(sizeof(double) * 2 * m * n), *ii = malloc(sizeof(double) * 2 * m * n);
  double *ri = malloc(sizeof(double) * 2 * m * n), *ir = malloc(sizeof(double) * 2 * m * n);
  orc_split_gemm_kc(ar, br, rr, m, k, n, S, target, NULL, kc);
  orc_split_gemm_kc(ai, bi, ii, m, k, n, S, target, NULL, kc);
  orc_split_gemm_kc(ar, bi, ri, m, k, n, S, target, NULL, kc);
  orc_split_gemm_kc(ai, br, ir, m, k, n, S, target, NULL, kc);
  for (int64_t e = 0; e < m * n; ++e) {
    dd re = dd_sub(mk(rr[2 * e], rr[2 * e + 1]), mk(ii[2 * e], ii[2 * e + 1]));
    dd im = dd_add(mk(ri[2 * e], ri[2 * e + 1]), mk(ir[2 * e], ir[2 * e + 1]));
    c[4 * e] = re.hi; c[4 * e + 1] = re.lo; c[4 * e + 2] = im.hi; c[4 * e + 3] = im.lo;
  }
  free(ar); free(ai); free(br); free(bi); free(rr); free(ii); free(ri); free(ir);
}

/* ---- BLAS-style shims: test/integration/blas/wgemm.f90, wtrsm.f90 --------
 * DGEMM / DTRSM over DD values, column-major with leading dimensions, in the
 * exact loop order of the Fortran (its DD operators are bit-identical to the
 * C++ ones restated above, test/integration/crosscheck.cc).  Argument checks
 * return the BLAS info code the reference hands to xerbla, 0 when valid;
 * nothing is written when it is non-zero.  alpha and beta point at one DD. */
static int lsame1(char a, char b) {
  if (a >= 'a' && a <= 'z') a = (char)(a - 32);
  if (b >= 'a' && b <= 'z') b = (char)(b - 32);
  return a == b;
}
/* DD == / /=: both limbs compared (fsrc/multifloats.fypp:2920-2928). */
static int dd_eq(dd x, dd y) { return x.hi == y.hi && x.lo == y.lo; }
#define ODD(p, i, j, ld) mk((p)[2 * ((i) + (j) * (ld))], (p)[2 * ((i) + (j) * (ld)) + 1])
#define OSET(p, i, j, ld, v)                   \
  do {                                         \
    dd v_ = (v);                               \
    (p)[2 * ((i) + (j) * (ld))] = v_.hi;       \
    (p)[2 * ((i) + (j) * (ld)) + 1] = v_.lo;   \
  } while (0)
static int64_t max1(int64_t x) { return x > 1 ? x : 1; }

int orc_wgemm_info(char transa, char transb, int64_t m, int64_t n, int64_t k, int64_t lda,
                   int64_t ldb, int64_t ldc) { /* wgemm.f90:16-48 */
  int nota = lsame1(transa, 'N'), notb = lsame1(transb, 'N');
  int64_t nrowa = nota ? m : k, nrowb = notb ? k : n;
  if (!nota && !lsame1(transa, 'C') && !lsame1(transa, 'T')) return 1;
  if (!notb && !lsame1(transb, 'C') && !lsame1(transb, 'T')) return 2;
  if (m < 0) return 3;
  if (n < 0) return 4;
  if (k < 0) return 5;
  if (lda < max1(nrowa)) return 8;
  if (ldb < max1(nrowb)) return 10;
  if (ldc < max1(m)) return 13;
  return 0;
}

int orc_wgemm(char transa, char transb, int64_t m, int64_t n, int64_t k, const double *alpha_,
              const double *a, int64_t lda, const double *b, int64_t ldb, const double *beta_,
              double *c, int64_t ldc) {
  int info = orc_wgemm_info(transa, transb, m, n, k, lda, ldb, ldc);
  if (info) return info;
  const dd one = mk(1.0, 0.0), zero = mk(0.0, 0.0);
  dd alpha = mk(alpha_[0], alpha_[1]), beta = mk(beta_[0], beta_[1]);
  int nota = lsame1(transa, 'N'), notb = lsame1(transb, 'N');
  if (m == 0 || n == 0 || ((dd_eq(alpha, zero) || k == 0) && dd_eq(beta, one))) return 0; /* :49 */
  if (dd_eq(alpha, zero)) { /* :50-65 */
    for (int64_t j = 0; j < n; ++j)
      for (int64_t i = 0; i < m; ++i)
        OSET(c, i, j, ldc, dd_eq(beta, zero) ? zero : dd_mul(beta, ODD(c, i, j, ldc)));
    return 0;
  }
  if (nota) { /* :68-84 and :106-122: C := beta C, then C += (alpha b_lj) A(:,l) */
    for (int64_t j = 0; j < n; ++j) {
      if (dd_eq(beta, zero)) {
        for (int64_t i = 0; i < m; ++i) OSET(c, i, j, ldc, zero);
      } else if (!dd_eq(beta, one)) {
        for (int64_t i = 0; i < m; ++i) OSET(c, i, j, ldc, dd_mul(beta, ODD(c, i, j, ldc)));
      }
      for (int64_t l = 0; l < k; ++l) {
        dd temp = dd_mul(alpha, notb ? ODD(b, l, j, ldb) : ODD(b, j, l, ldb));
        for (int64_t i = 0; i < m; ++i)
          OSET(c, i, j, ldc, dd_add(ODD(c, i, j, ldc), dd_mul(temp, ODD(a, i, l, lda))));
      }
    }
  } else { /* :86-99 and :124-137: dot products down the columns of A */
    for (int64_t j = 0; j < n; ++j)
      for (int64_t i = 0; i < m; ++i) {
        dd temp = zero;
        for (int64_t l = 0; l < k; ++l)
          temp = dd_add(temp, dd_mul(ODD(a, l, i, lda), notb ? ODD(b, l, j, ldb) : ODD(b, j, l, ldb)));
        if (dd_eq(beta, zero))
          OSET(c, i, j, ldc, dd_mul(alpha, temp));
        else
          OSET(c, i, j, ldc, dd_add(dd_mul(alpha, temp), dd_mul(beta, ODD(c, i, j, ldc))));
      }
  }
  return 0;
}

int orc_wtrsm_info(char side, char uplo, char transa, char diag, int64_t m, int64_t n,
                   int64_t lda, int64_t ldb) { /* wtrsm.f90:16-44 */
  int lside = lsame1(side, 'L');
  int64_t nrowa = lside ? m : n;
  int upper = lsame1(uplo, 'U');
  if (!lside && !lsame1(side, 'R')) return 1;
  if (!upper && !lsame1(uplo, 'L')) return 2;
  if (!lsame1(transa, 'N') && !lsame1(transa, 'T') && !lsame1(transa, 'C')) return 3;
  if (!lsame1(diag, 'U') && !lsame1(diag, 'N')) return 4;
  if (m < 0) return 5;
  if (n < 0) return 6;
  if (lda < max1(nrowa)) return 9;
  if (ldb < max1(m)) return 11;
  return 0;
}

int orc_wtrsm(char side, char uplo, char transa, char diag, int64_t m, int64_t n,
              const double *alpha_, const double *a, int64_t lda, double *b, int64_t ldb) {
  int info = orc_wtrsm_info(side, uplo, transa, diag, m, n, lda, ldb);
  if (info) return info;
  const dd one = mk(1.0, 0.0), zero = mk(0.0, 0.0);
  dd alpha = mk(alpha_[0], alpha_[1]), temp;
  int lside = lsame1(side, 'L'), nounit = lsame1(diag, 'N'), upper = lsame1(uplo, 'U');
  int notr = lsame1(transa, 'N');
  if (m == 0 || n == 0) return 0;
  if (dd_eq(alpha, zero)) { /* :46-53 */
    for (int64_t j = 0; j < n; ++j)
      for (int64_t i = 0; i < m; ++i) OSET(b, i, j, ldb, zero);
    return 0;
  }
  if (lside && notr) { /* :55-102: B := alpha inv(A) B, column by column */
    for (int64_t j = 0; j < n; ++j) {
      if (!dd_eq(alpha, one))
        for (int64_t i = 0; i < m; ++i) OSET(b, i, j, ldb, dd_mul(alpha, ODD(b, i, j, ldb)));
      for (int64_t q = 0; q < m; ++q) {
        int64_t kk = upper ? m - 1 - q : q;
        if (!dd_eq(ODD(b, kk, j, ldb), zero)) {
          if (nounit) OSET(b, kk, j, ldb, dd_div(ODD(b, kk, j, ldb), ODD(a, kk, kk, lda)));
          int64_t i0 = upper ? 0 : kk + 1, i1 = upper ? kk : m;
          for (int64_t i = i0; i < i1; ++i)
            OSET(b, i, j, ldb, dd_sub(ODD(b, i, j, ldb), dd_mul(ODD(b, kk, j, ldb), ODD(a, i, kk, lda))));
        }
      }
    }
  } else if (lside) { /* :103-132: B := alpha inv(A^T) B */
    for (int64_t j = 0; j < n; ++j)
      for (int64_t q = 0; q < m; ++q) {
        int64_t i = upper ? q : m - 1 - q;
        temp = dd_mul(alpha, ODD(b, i, j, ldb));
        int64_t k0 = upper ? 0 : i + 1, k1 = upper ? i : m;
        for (int64_t kk = k0; kk < k1; ++kk)
          temp = dd_sub(temp, dd_mul(ODD(a, kk, i, lda), ODD(b, kk, j, ldb)));
        if (nounit) temp = dd_div(temp, ODD(a, i, i, lda));
        OSET(b, i, j, ldb, temp);
      }
  } else if (notr) { /* :135-177: B := alpha B inv(A) */
    for (int64_t q = 0; q < n; ++q) {
      int64_t j = upper ? q : n - 1 - q;
      if (!dd_eq(alpha, one))
        for (int64_t i = 0; i < m; ++i) OSET(b, i, j, ldb, dd_mul(alpha, ODD(b, i, j, ldb)));
      int64_t k0 = upper ? 0 : j + 1, k1 = upper ? j : n;
      for (int64_t kk = k0; kk < k1; ++kk)
        if (!dd_eq(ODD(a, kk, j, lda), zero))
          for (int64_t i = 0; i < m; ++i)
            OSET(b, i, j, ldb, dd_sub(ODD(b, i, j, ldb), dd_mul(ODD(a, kk, j, lda), ODD(b, i, kk, ldb))));
      if (nounit) {
        temp = dd_div(one, ODD(a, j, j, lda));
        for (int64_t i = 0; i < m; ++i) OSET(b, i, j, ldb, dd_mul(temp, ODD(b, i, j, ldb)));
      }
    }
  } else { /* :178-207: B := alpha B inv(A^T) */
    for (int64_t q = 0; q < n; ++q) {
      int64_t kk = upper ? n - 1 - q : q;
      if (nounit) {
        temp = dd_div(one, ODD(a, kk, kk, lda));
        for (int64_t i = 0; i < m; ++i) OSET(b, i, kk, ldb, dd_mul(temp, ODD(b, i, kk, ldb)));
      }
      int64_t j0 = upper ? 0 : kk + 1, j1 = upper ? kk : n;
      for (int64_t j = j0; j < j1; ++j)
        if (!dd_eq(ODD(a, j, kk, lda), zero)) {
          temp = ODD(a, j, kk, lda);
          for (int64_t i = 0; i < m; ++i)
            OSET(b, i, j, ldb, dd_sub(ODD(b, i, j, ldb), dd_mul(temp, ODD(b, i, kk, ldb))));
        }
      if (!dd_eq(alpha, one))
        for (int64_t i = 0; i < m; ++i) OSET(b, i, kk, ldb, dd_mul(alpha, ODD(b, i, kk, ldb)));
    }
  }
  return 0;
}
#undef ODD
#undef OSET

/* ---- CRT (modular) split form, restated on the CPU -------------------------
 * The device (split_gemm.cu, crt_device.cuh) recovers the exact integer
 * product C' = X Y^T of the rounded operands from its residues modulo N
 * moduli by the Chinese remainder theorem.  This restatement computes C'
 * directly with a 256-bit accumulator -- no moduli -- so it checks the modular
 * reconstruction too.  Same scan and exponent spreads as the digit-sliced
 * form, same plan (the smallest W whose a-priori bound meets the target), same
 * rounding X = round(a 2^(W - sigma)), same conversion to DD (crt_to_dd_c) and
 * the same exact scaling by 2^(sigma_i + tau_j - 2W). */
#include "../multifloats_b200/csrc/crt_tables.h"
#define CRT_WMAX 110
static int crt_ceil_log2(int64_t k) {
  int b = 0;
  while (b < 63 && ((int64_t)1 << b) < k) ++b;
  return b;
}
double orc_crt_bound(int W, int ra, int rb, int64_t k) {
  return (ldexp(1.0, 104 + ra - W) + ldexp(1.0, 104 + rb - W) + ldexp(1.0, 104 + ra + rb - 2 * W) + 0.5) /
         (double)k;
}
int orc_crt_plan(int bits, double target, int ra, int rb, int64_t k, int *nmod) {
  int W = bits;
  if (W <= 0) {
    W = CRT_WMAX;
    for (int w = 8; w <= CRT_WMAX; ++w)
      if (orc_crt_bound(w, ra, rb, k) <= target) {
        W = w;
        break;
      }
  }
  const int need = 2 * W + crt_ceil_log2(k) + 2;
  int n = 1;
  while (n < CRT_NMAX && crt_lg[n] < need) ++n;
  if (nmod) *nmod = n;
  return W;
}
/* the split form's rounding to the W-bit grid */
static __int128 crt_round(double hi, double lo, int sigma, int W) { return split_round(hi, lo, sigma, W); }
/* acc (256-bit two's complement, 4 little-endian words) += x * y */
static void acc_add_prod(uint64_t acc[4], __int128 x, __int128 y) {
  int neg = (x < 0) != (y < 0);
  unsigned __int128 ux = x < 0 ? (unsigned __int128)(-x) : (unsigned __int128)x;
  unsigned __int128 uy = y < 0 ? (unsigned __int128)(-y) : (unsigned __int128)y;
  uint64_t x0 = (uint64_t)ux, x1 = (uint64_t)(ux >> 64), y0 = (uint64_t)uy, y1 = (uint64_t)(uy >> 64);
  unsigned __int128 p00 = (unsigned __int128)x0 * y0, p01 = (unsigned __int128)x0 * y1;
  unsigned __int128 p10 = (unsigned __int128)x1 * y0, p11 = (unsigned __int128)x1 * y1;
  uint64_t p[4] = {0, 0, 0, 0};
  unsigned __int128 t = (unsigned __int128)(uint64_t)p00;
  p[0] = (uint64_t)t;
  t = (p00 >> 64) + (uint64_t)p01 + (uint64_t)p10;
  p[1] = (uint64_t)t;
  t = (t >> 64) + (p01 >> 64) + (p10 >> 64) + (uint64_t)p11;
  p[2] = (uint64_t)t;
  t = (t >> 64) + (p11 >> 64);
  p[3] = (uint64_t)t;
  if (neg) { /* two's complement of p */
    unsigned __int128 c = 1;
    for (int w = 0; w < 4; ++w) {
      c += (uint64_t)~p[w];
      p[w] = (uint64_t)c;
      c >>= 64;
    }
  }
  unsigned __int128 c = 0;
  for (int w = 0; w < 4; ++w) {
    c += (unsigned __int128)acc[w] + p[w];
    acc[w] = (uint64_t)c;
    c >>= 64;
  }
}
/* C' (256-bit two's complement) -> (h + l) 2^e: the magnitude's leading one
 * at bit 159 of a 160-bit window (bits below it dropped), hi = the window
 * rounded to 53 bits (nearest, ties to even), lo = the remainder
 * D 2^96 + n2 2^64 + n1 2^32 + n0 summed in doubles in that order, then
 * fast_two_sum(hi, lo 2^-107); e = weight of window bit 107. */
static void crt_to_dd_c(const uint64_t acc[4], double *h, double *l, int *e) {
  int neg = (int)(acc[3] >> 63);
  uint64_t mag[4];
  unsigned __int128 c = neg ? 1 : 0;
  for (int w = 0; w < 4; ++w) {
    uint64_t x = neg ? ~acc[w] : acc[w];
    c += x;
    mag[w] = (uint64_t)c;
    c >>= 64;
  }
  int lead = -1;
  for (int b = 255; b >= 0; --b)
    if ((mag[b / 64] >> (b % 64)) & 1) {
      lead = b;
      break;
    }
  if (lead < 0) {
    *h = *l = 0.0;
    *e = 0;
    return;
  }
  int E = lead - 159;
  uint32_t nw[5];
  for (int q = 0; q < 5; ++q) {
    uint32_t v = 0;
    for (int b = 0; b < 32; ++b) {
      int src = E + 32 * q + b;
      if (src >= 0 && ((mag[src / 64] >> (src % 64)) & 1)) v |= 1u << b;
    }
    nw[q] = v;
  }
  uint64_t T64 = ((uint64_t)nw[4] << 32) | nw[3];
  uint64_t keep = T64 >> 11;
  uint32_t r11 = (uint32_t)(T64 & 0x7FF);
  int lowz = (nw[2] | nw[1] | nw[0]) == 0;
  int up = r11 > 0x400 || (r11 == 0x400 && (!lowz || (keep & 1)));
  keep += (uint64_t)up;
  int D = (int)r11 - (up ? 2048 : 0);
  double lo = (double)D * 0x1p96;
  lo = lo + (double)nw[2] * 0x1p64;
  lo = lo + (double)nw[1] * 0x1p32;
  lo = lo + (double)nw[0];
  double hi = (double)keep;
  lo = lo * 0x1p-107;
  double hs, ls;
  fast_two_sum(hi, lo, &hs, &ls);
  if (neg) {
    hs = -hs;
    ls = -ls;
  }
  *h = hs;
  *l = ls;
  *e = E + 107;
}
/* info[0..3] = {N moduli, rho_a, rho_b, W}; rows i0 .. i1-1 of the product
 * only (c holds (i1 - i0) x n outputs, leading dimension i1 - i0). */
void orc_crt_gemm_rows(const double *a, const double *b, double *c, int64_t m, int64_t k, int64_t n,
                       int bits, double target, int *info, int64_t i0, int64_t i1) {
  int *sa = malloc(sizeof(int) * m), *ma = malloc(sizeof(int) * m), *fa = malloc(sizeof(int) * m);
  int *sb = malloc(sizeof(int) * n), *mb = malloc(sizeof(int) * n), *fb = malloc(sizeof(int) * n);
  int ra = 0, rb = 0;
  for (int64_t i = 0; i < m; ++i) {
    split_stats(a + 2 * i, k, m, &sa[i], &ma[i], &fa[i]);
    if (sa[i] != -100000 && sa[i] - ma[i] > ra) ra = sa[i] - ma[i];
  }
  for (int64_t j = 0; j < n; ++j) {
    split_stats(b + 2 * j * k, k, 1, &sb[j], &mb[j], &fb[j]);
    if (sb[j] != -100000 && sb[j] - mb[j] > rb) rb = sb[j] - mb[j];
  }
  for (int64_t i = 0; i < m; ++i)
    if (sa[i] == -100000) sa[i] = 0;
  for (int64_t j = 0; j < n; ++j)
    if (sb[j] == -100000) sb[j] = 0;
  int nmod = 0;
  int W = orc_crt_plan(bits, target, ra, rb, k, &nmod);
  if (info) {
    info[0] = nmod;
    info[1] = ra;
    info[2] = rb;
    info[3] = W;
  }
  int64_t mr = i1 - i0;
  __int128 *X = malloc(sizeof(__int128) * (size_t)(mr * k + 1)), *Y = malloc(sizeof(__int128) * (size_t)(n * k + 1));
  for (int64_t i = i0; i < i1; ++i)
    for (int64_t p = 0; p < k; ++p)
      X[(i - i0) * k + p] = fa[i] ? 0 : crt_round(a[2 * (p * m + i)], a[2 * (p * m + i) + 1], sa[i], W);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t p = 0; p < k; ++p)
      Y[j * k + p] = fb[j] ? 0 : crt_round(b[2 * (j * k + p)], b[2 * (j * k + p) + 1], sb[j], W);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t i = i0; i < i1; ++i) {
      uint64_t acc[4] = {0, 0, 0, 0};
      for (int64_t p = 0; p < k; ++p) acc_add_prod(acc, X[(i - i0) * k + p], Y[j * k + p]);
      double *o = c + 2 * (j * mr + (i - i0));
      if (fa[i] | fb[j]) {
        o[0] = NAN;
        o[1] = 0.0;
      } else {
        double hi, lo;
        int e;
        crt_to_dd_c(acc, &hi, &lo, &e);
        int ex = e + sa[i] + sb[j] - 2 * W;
        o[0] = ldexp(hi, ex);
        o[1] = ldexp(lo, ex);
      }
    }
  free(sa); free(ma); free(fa); free(sb); free(mb); free(fb); free(X); free(Y);
}
void orc_crt_gemm(const double *a, const double *b, double *c, int64_t m, int64_t k, int64_t n, int bits,
                  double target, int *info) {
  orc_crt_gemm_rows(a, b, c, m, k, n, bits, target, info, 0, m);
}

/* Complex CRT form: the four real products with one W (planned from the
 * exponent spreads of all four parts: A side Ar, Ai rows; B side Br, Bi
 * columns), re = Ar Br - Ai Bi, im = Ar Bi + Ai Br with the DD operators in
 * the device's order (store, subtract, store, add).  info = {N, rho_a, rho_b, W}. */
void orc_crt_cgemm(const double *a, const double *b, double *c, int64_t m, int64_t k, int64_t n, int bits,
                   double target, int *info) {
  double *ar = malloc(sizeof(double) * 2 * m * k), *ai = malloc(sizeof(double) * 2 * m * k);
  double *br = malloc(sizeof(double) * 2 * k * n), *bi = malloc(sizeof(double) * 2 * k * n);
  for (int64_t e = 0; e < m * k; ++e) {
    ar[2 * e] = a[4 * e]; ar[2 * e + 1] = a[4 * e + 1];
    ai[2 * e] = a[4 * e + 2]; ai[2 * e + 1] = a[4 * e + 3];
  }
  for (int64_t e = 0; e < k * n; ++e) {
    br[2 * e] = b[4 * e]; br[2 * e + 1] = b[4 * e + 1];
    bi[2 * e] = b[4 * e + 2]; bi[2 * e + 1] = b[4 * e + 3];
  }
  int ra = 0, rb = 0;
  for (int part = 0; part < 2; ++part) {
    const double *x = part ? ai : ar, *y = part ? bi : br;
    for (int64_t i = 0; i < m; ++i) {
      int sg, mu, bad;
      split_stats(x + 2 * i, k, m, &sg, &mu, &bad);
      if (sg != -100000 && sg - mu > ra) ra = sg - mu;
    }
    for (int64_t j = 0; j < n; ++j) {
      int sg, mu, bad;
      split_stats(y + 2 * j * k, k, 1, &sg, &mu, &bad);
      if (sg != -100000 && sg - mu > rb) rb = sg - mu;
    }
  }
  int nmod = 0;
  int W = orc_crt_plan(bits, target, ra, rb, k, &nmod);
  if (info) {
    info[0] = nmod;
    info[1] = ra;
    info[2] = rb;
    info[3] = W;
  }
  double *rr = malloc(sizeof(double) * 2 * m * n), *ii = malloc(sizeof(double) * 2 * m * n);
  double *ri = malloc(sizeof(double) * 2 * m * n), *ir = malloc(sizeof(double) * 2 * m * n);
  orc_crt_gemm(ar, br, rr, m, k, n, W, target, NULL);
  orc_crt_gemm(ai, bi, ii, m, k, n, W, target, NULL);
  orc_crt_gemm(ar, bi, ri, m, k, n, W, target, NULL);
  orc_crt_gemm(ai, br, ir, m, k, n, W, target, NULL);
  for (int64_t e = 0; e < m * n; ++e) {
    dd re = dd_sub(mk(rr[2 * e], rr[2 * e + 1]), mk(ii[2 * e], ii[2 * e + 1]));
    dd im = dd_add(mk(ri[2 * e], ri[2 * e + 1]), mk(ir[2 * e], ir[2 * e + 1]));
    c[4 * e] = re.hi; c[4 * e + 1] = re.lo; c[4 * e + 2] = im.hi; c[4 * e + 3] = im.lo;
  }
  free(ar); free(ai); free(br); free(bi); free(rr); free(ii); free(ri); free(ir);
}
