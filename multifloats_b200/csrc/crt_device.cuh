// CRT (modular) form of the split-INT8 DD GEMM: device pieces.
//
// The operands are rounded to the fixed-point grid of their row (A) / column
// (B) exactly as in the digit-sliced form -- X = round(a 2^(W - sigma_i)),
// |X| < 2^W -- and the exact integer product C' = X Y^T is recovered from its
// residues modulo N pairwise-coprime moduli m_t <= 256 (crt_tables.h): each
// residue product (X mod m_t)(Y mod m_t)^T (residues in [0, m_t), unsigned
// bytes) is one u8 x u8 -> s32 GEMM on the tensor cores, exact for K chunks of
// up to 73 * 128 (73 * 128 * 255^2 < 2^30), and C' follows from the Chinese
// remainder theorem,
//   C' = sum_t r_t e_t - q M,   e_t = (M / m_t) ((M / m_t)^-1 mod m_t),
//   r_t = (X Y^T mod m_t) in [0, m_t),  q = round(sum_t r_t e_t / M),
// which is exact because the moduli are chosen with M >= 4 k 2^(2W) > 4 |C'|.
// The sums over t are themselves a small u8 x u8 matrix product (residues
// times the bytes of e_t and of c_t = e_t / M in fixed point), so the
// reconstruction runs on the tensor cores too (crt_combine_tc_body), with the
// carries, q M and the sign in 32-bit integer limbs.
// C' is then converted to a double-double (crt_to_dd: hi = C' rounded to 53
// bits, lo the rest summed in doubles, renormalised) and scaled by
// 2^(sigma_i + tau_j - 2W).  Compared with the digit-sliced form (S(S+1)/2 slice products for S
// slices) the tensor work is N products: 26 instead of 105 at 4096^3.
//
// Error (a priori, per output; delta = rounding of an operand to its grid,
// |delta a_ip| <= 2^(sigma_i - W), zero for zero entries):
//   |C - AB|_ij <= (2^(rho_A - W) + 2^(rho_B - W) + 2^(rho_A + rho_B - 2W)) (|A||B|)_ij
//                + 2^-105 |C_ij|                                   (final DD rounding)
// with |a_ip| >= 2^(sigma_i - rho_A) for nonzero entries.  In units of
// k 2^-104 (|A||B|)_ij that is at most
//   (2^(104 + rho_A - W) + 2^(104 + rho_B - W) + 2^(104 + rho_A + rho_B - 2W) + 1/2) / k,
// and the plan takes the smallest W meeting the requested target.
#pragma once
#include <cstdint>

#include "split_device.cuh"  // first: dd_device.cuh defines MF_TABLE as device constant memory
#include "crt_tables.h"
#include "tcgen05.cuh"

namespace mfcuda {
namespace split {

constexpr int CRT_NL = 8;  // most 32-bit limbs of a reconstruction (256 bits)
constexpr int CRT_WMAX = 110;

// Reconstruction constants of the plan's N moduli (from the per-count tables
// of crt_tables.h, generated offline): M = prod m_t modulo 2^256 in 32-bit
// limbs, and the E matrix of the tensor-core reconstruction
// (crt_combine_tc_body) ready to copy: row b (an MMA column), byte t (a
// modulus) holds the bytes of round(c_t 2^24) in rows 0-2 (c_t = e_t / M), a
// zero row 3, and the bytes of e_t = (M / m_t)((M / m_t)^-1 mod m_t) mod
// 2^256 in rows 4-35; zero for t >= N and in rows 36-47.  Rows beyond
// 4 + nbe feed only limbs the reconstruction discards.
constexpr int CRT_EB_ROWS = 48, CRT_EB_BYTES = 64;
struct CrtConst {
  uint32_t Mw[CRT_NL];
  alignas(16) uint8_t eb[CRT_EB_ROWS][CRT_EB_BYTES];
};

// ceil(log2 k) for k >= 1.
__host__ __device__ inline int ceil_log2(int64_t k) {
  int b = 0;
  while (b < 63 && ((int64_t)1 << b) < k) ++b;
  return b;
}

// Bound of the CRT form in units of k 2^-104 (|A||B|)_ij.
__host__ __device__ inline double crt_bound(int W, int ra, int rb, int64_t k) {
  return (ldexp(1.0, 104 + ra - W) + ldexp(1.0, 104 + rb - W) + ldexp(1.0, 104 + ra + rb - 2 * W) + 0.5) /
         (double)k;
}
// Moduli needed for W-bit operands and inner dimension k: M >= 4 k 2^(2W) > 4 |C'|,
// so |C'| / M < 1/4 and the rounded quotient estimate has a margin of 1/4.
__host__ __device__ inline int crt_moduli(int W, int64_t k, const int *lg) {
  const int need = 2 * W + ceil_log2(k) + 2;
  int n = 1;
  while (n < CRT_NMAX && lg[n] < need) ++n;
  return n;
}
// Most moduli the CRT form can need for inner dimension k (W <= bits, or
// W <= CRT_WMAX when bits is 0): workspace sizing on the host.
inline int crt_slices_max(int64_t k, int bits) {
  const int need = 2 * (bits > 0 ? bits : CRT_WMAX) + ceil_log2(k < 1 ? 1 : k) + 2;
  int n = 1;
  while (n < CRT_NMAX && crt_lg_host[n] < need) ++n;
  return n;
}
// Bytes of the reconstruction (a multiple of 4): C' is computed modulo
// 2^(8 nbe) with nbe = 4 ceil(need / 32), need = 2W + ceil(log2 k) + 2 the
// bound the moduli are chosen for, so |C'| < 2^(8 nbe - 2) and bit 8 nbe - 1
// is the sign.
__host__ __device__ inline int crt_tc_bytes(int W, int64_t k) {
  return 4 * ((2 * W + ceil_log2(k) + 2 + 31) / 32);
}
// MMA columns of the reconstruction: the three bytes of round(c_t 2^24), a
// zero column, then nbe bytes of e_t, rounded up to 16 (32 or 48).
__host__ __device__ inline int crt_tc_cols(int nbe) { return (nbe + 4 + 15) / 16 * 16; }

// One block: exponent spreads (as the digit-sliced plan), then W, the moduli
// count N and the reconstruction constants.  bits > 0 forces W.
__device__ __forceinline__ void crt_plan_body(const StatSet &st, int bits, double target, int64_t k,
                                              Plan *plan, CrtConst *cc) {
  __shared__ int red[2][32];
  __shared__ int sh_n;
  int r[2] = {0, 0};
  for (int o = 0; o < st.n; ++o)
    for (int64_t i = threadIdx.x; i < st.count[o]; i += blockDim.x)
      if (st.sig[o][i] != SENT_LO) r[st.side[o]] = max(r[st.side[o]], st.sig[o][i] - st.mu[o][i]);
  int ra = r[0], rb = r[1];
  for (int off = 16; off >= 1; off >>= 1) {
    ra = max(ra, __shfl_xor_sync(0xffffffffu, ra, off));
    rb = max(rb, __shfl_xor_sync(0xffffffffu, rb, off));
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = ra;
    red[1][threadIdx.x >> 5] = rb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      ra = max(ra, red[0][w]);
      rb = max(rb, red[1][w]);
    }
    int W = bits;
    if (W <= 0) {
      // the smallest w in [8, CRT_WMAX] with crt_bound <= target (CRT_WMAX if
      // none); the bound falls strictly with w, so bisection finds it
      int lo = 8, hi = CRT_WMAX;
      if (crt_bound(hi, ra, rb, k) <= target) {
        while (lo < hi) {
          const int mid = (lo + hi) / 2;
          if (crt_bound(mid, ra, rb, k) <= target)
            hi = mid;
          else
            lo = mid + 1;
        }
      }
      W = hi;
    }
    const int n = crt_moduli(W, k, crt_lg);
    plan->S = n;
    plan->G = n - 1;
    plan->W = W;
    plan->rho_a = ra;
    plan->rho_b = rb;
    plan->crt = 1;
    plan->nl = crt_tc_bytes(W, k) / 4;
    sh_n = n;
  }
  __syncthreads();
  const int n = sh_n;
  // the constants of the n-moduli set, from the tables: column t of E
  if (threadIdx.x < (unsigned)CRT_EB_BYTES) {
    const int t = threadIdx.x;
    // the table words first (independent loads), then the 48 bytes of column t
    uint32_t cf = 0u, ev[CRT_NL];
#pragma unroll
    for (int l = 0; l < CRT_NL; ++l) ev[l] = 0u;
    if (t < n) {
      cf = crt_c_n[n - 1][t];
#pragma unroll
      for (int l = 0; l < CRT_NL; ++l) ev[l] = crt_e_n[n - 1][t][l];
    }
#pragma unroll
    for (int b = 0; b < CRT_EB_ROWS; ++b) {
      uint32_t v = 0;
      if (b < 3)
        v = (cf >> (8 * b)) & 0xFFu;
      else if (b >= 4 && b < 4 + 4 * CRT_NL)
        v = (ev[(b - 4) >> 2] >> (8 * ((b - 4) & 3))) & 0xFFu;
      cc->eb[b][t] = (uint8_t)v;
    }
  } else if (threadIdx.x < (unsigned)(CRT_EB_BYTES + CRT_NL)) {
    cc->Mw[threadIdx.x - CRT_EB_BYTES] = crt_M_n[n - 1][threadIdx.x - CRT_EB_BYTES];
  }
  __syncthreads();
  for (int o = 0; o < st.n; ++o)
    for (int64_t i = threadIdx.x; i < st.count[o]; i += blockDim.x)
      if (st.sig[o][i] == SENT_LO) st.sig[o][i] = 0;
}

// ---- residue slicing ----------------------------------------------------------
// Non-negative residue of u < 2^30 modulo m_t (Barrett: the estimate is exact
// or one too large).
__device__ __forceinline__ uint32_t crt_mod_small(uint32_t u, int t) {
  const uint32_t m = crt_mod[t];
  const uint32_t q = __umulhi(u, crt_mu[t]);
  const int r = (int)(u - q * m);
  return (uint32_t)(r < 0 ? r + (int)m : r);
}
// The residue in [0, m_t) of X = sum_q d_q 256^q (balanced digits, read from
// the biased words y of biased_bytes: digit q = byte q of y xor 0x80): dp4a
// against the digit weights give rr = sum_q d_q c_q with |rr| < 14 * 128 * 128
// < 2^18, made non-negative by the offset (a multiple of m_t of at least
// 2^18, the first dp4a's addend: u < 2^19 + 256) and reduced exactly.  For
// u < 2^20 the Barrett quotient umulhi(u, ceil(2^32 / m)) is floor(u / m)
// itself (its error u (mu m - 2^32) / (m 2^32) < u / 2^32 < 1 / m), so no
// correction step follows.  The per-modulus constants are passed in (hoisted
// by the caller).  NW = digit words in use: 3 when W <= 94 (digits 12 and 13
// are zero).
struct ModConst {
  int c0, c1, c2, c3;  // digit weights, signed bytes packed
  uint32_t m, mu, off;
};
__device__ __forceinline__ ModConst mod_const(int t) {
  ModConst k;
  k.c0 = (int)crt_digw[t][0];
  k.c1 = (int)crt_digw[t][1];
  k.c2 = (int)crt_digw[t][2];
  k.c3 = (int)crt_digw[t][3];
  k.m = crt_mod[t];
  k.mu = crt_mu[t];
  k.off = crt_off18[t];
  return k;
}
template <int NW>
__device__ __forceinline__ uint32_t crt_residue(const uint32_t (&dw)[4], const ModConst &k) {
  int rr = NW == 4 ? __dp4a((int)dw[3], k.c3, (int)k.off) : (int)k.off;
  rr = __dp4a((int)dw[2], k.c2, rr);
  rr = __dp4a((int)dw[1], k.c1, rr);
  rr = __dp4a((int)dw[0], k.c0, rr);
  const uint32_t u = (uint32_t)rr;  // in [0, 2^19 + 256)
  return u - __umulhi(u, k.mu) * k.m;
}
// Signed digit words of the biased words of one entry.
__device__ __forceinline__ void digit_words(const uint32_t (&y)[4], uint32_t (&dw)[4]) {
#pragma unroll
  for (int w = 0; w < 4; ++w) dw[w] = y[w] ^ bias_word(w);
}
// Calls f(t, word) with the residues modulo m_t of 8 entries packed in entry
// order (byte e = entry e), for t0 <= t < t1.
template <int NW, class F>
__device__ __forceinline__ void residue_words_nw(const uint32_t (&dw)[8][4], int t0, int t1, F f) {
  for (int t = t0; t < t1; ++t) {
    const ModConst k = mod_const(t);
    uint32_t r[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) r[e] = crt_residue<NW>(dw[e], k);
    // low bytes of r[0..3] and r[4..7] packed in order (byte permutes)
    const uint32_t lo = __byte_perm(__byte_perm(r[0], r[1], 0x0040), __byte_perm(r[2], r[3], 0x0040), 0x5410);
    const uint32_t hi = __byte_perm(__byte_perm(r[4], r[5], 0x0040), __byte_perm(r[6], r[7], 0x0040), 0x5410);
    f(t, (uint64_t)lo | ((uint64_t)hi << 32));
  }
}
template <class F>
__device__ __forceinline__ void for_each_residue_word(const uint32_t (&dw)[8][4], int t0, int t1, int W, F f) {
  if (W <= 94)
    residue_words_nw<3>(dw, t0, t1, f);
  else
    residue_words_nw<4>(dw, t0, t1, f);
}
// Moduli whose residues the A slicer's transposing tile holds at once (the
// tile is reused for the rest): a smaller tile lets more CTAs share an SM.
constexpr int CRT_SA_MODULI = 18;

// A (m x k column-major view) -> As[t][i][p], as slice_a_body with residues
// for digits; the transposing tile lives in dynamic shared memory
// (min(n, CRT_SA_MODULI) * SA_ROWS * SA_STRIDE bytes) and takes the moduli in
// groups of CRT_SA_MODULI.
__device__ __forceinline__ void crt_slice_a_body(const double *__restrict__ A, int64_t M, int64_t K,
                                                 int64_t stride, int64_t M_pad, int64_t K_pad, const int *sig,
                                                 const int *flag, const Plan *plan, int8_t *__restrict__ As,
                                                 uint8_t *tile, int64_t bx, int64_t by) {
  const int n = plan->S, W = plan->W;
  const int64_t i0 = bx * SA_ROWS, p0 = by * SA_COLS;
  const int t = threadIdx.x;
  const int ii = t % SA_ROWS, grp = t / SA_ROWS;
  const int64_t i = i0 + ii;
  const bool row_ok = i < M && !flag[i < M ? i : 0];
  const int sigma = i < M ? sig[i] : 0;
  uint32_t y[8][4];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    int64_t p = p0 + grp * 8 + e;
    if (row_ok && p < K) {
      double2 v = __ldg(reinterpret_cast<const double2 *>(A) + (p * M + i) * stride);
      biased_bytes(v.x, v.y, sigma, W, y[e]);
    } else {
#pragma unroll
      for (int w = 0; w < 4; ++w) y[e][w] = bias_word(w);  // X = 0: every residue zero
    }
  }
  uint32_t dw[8][4];
#pragma unroll
  for (int e = 0; e < 8; ++e) digit_words(y[e], dw[e]);
  const bool any = row_ok && p0 + grp * 8 < K;  // else padding only: every residue zero
  const int row = t / 8, seg = (t % 8) * 8;
  for (int t0 = 0; t0 < n; t0 += CRT_SA_MODULI) {  // moduli t0 .. t1 - 1 in tile slots 0 ..
    const int t1 = min(n, t0 + CRT_SA_MODULI);
    auto put = [&](int sl, uint64_t word) {
      *reinterpret_cast<uint64_t *>(&tile[((sl - t0) * SA_ROWS + ii) * SA_STRIDE + grp * 8]) = word;
    };
    if (t0 > 0) __syncthreads();  // the previous moduli's rows have been copied out
    if (any)
      for_each_residue_word(dw, t0, t1, W, put);
    else
      for (int sl = t0; sl < t1; ++sl) put(sl, 0);
    __syncthreads();
    for (int s = t0; s < t1; ++s) {
      uint64_t v = *reinterpret_cast<const uint64_t *>(&tile[((s - t0) * SA_ROWS + row) * SA_STRIDE + seg]);
      *reinterpret_cast<uint64_t *>(As + ((s * M_pad + i0 + row) * K_pad + p0 + seg)) = v;
    }
  }
}

// B (k x n column-major view) -> Bs[t][j][p]: entries p8 .. p8+7 of column j.
__device__ __forceinline__ void crt_slice_b_one(const double *__restrict__ B, int64_t K, int64_t N,
                                                int64_t stride, int64_t N_pad, int64_t K_pad, const int *sig,
                                                const int *flag, const Plan *plan, int8_t *__restrict__ Bs,
                                                int64_t j, int64_t p8) {
  const int n = plan->S, W = plan->W;
  const bool col_ok = j < N && !flag[j < N ? j : 0];
  const int tau = j < N ? sig[j] : 0;
  uint32_t y[8][4];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    int64_t p = p8 + e;
    if (col_ok && p < K) {
      double2 v = __ldg(reinterpret_cast<const double2 *>(B) + (j * K + p) * stride);
      biased_bytes(v.x, v.y, tau, W, y[e]);
    } else {
#pragma unroll
      for (int w = 0; w < 4; ++w) y[e][w] = bias_word(w);
    }
  }
  auto put = [&](int sl, uint64_t word) {
    *reinterpret_cast<uint64_t *>(Bs + (((int64_t)sl * N_pad + j) * K_pad + p8)) = word;
  };
  if (col_ok && p8 < K) {
    uint32_t dw[8][4];
#pragma unroll
    for (int e = 0; e < 8; ++e) digit_words(y[e], dw[e]);
    for_each_residue_word(dw, 0, n, W, put);
  } else {  // padding only: every residue zero
    for (int sl = 0; sl < n; ++sl) put(sl, 0);
  }
}

// ---- reconstruction ---------------------------------------------------------------
// The signed integer held in nl little-endian 32-bit limbs (two's complement,
// nl <= 8) as a double-double scaled by 2^e:
//   the magnitude is normalised (whole-limb shifts, then a funnel shift) so
//   that its leading one is bit 159 of a 160-bit window n4..n0 (bit 0 of
//   weight 2^E; bits below the window dropped);
//   hi = the window rounded to 53 bits (nearest, ties to even, the bits below
//   bit 107 of the window deciding), exact as a double: keep 2^(E + 107);
//   lo = the rest D 2^96 + n2 2^64 + n1 2^32 + n0 (D = the low 11 bits of the
//   top 64 minus 2048 when rounded up) summed in doubles in that order,
//   times 2^E; then fast_two_sum(hi, lo) in units of 2^(E + 107).
// Returns (h, l) with value (h + l) 2^e, e = E + 107.
__device__ __forceinline__ void crt_to_dd(const uint32_t *limb, int nl, double &h, double &l, int &e) {
  const bool neg = (limb[nl - 1] >> 31) != 0;
  uint32_t m[CRT_NL];
  uint32_t carry = 1;
#pragma unroll
  for (int q = 0; q < CRT_NL; ++q) {
    uint32_t x = q < nl ? limb[q] : (neg ? 0xFFFFFFFFu : 0u);
    if (neg) {  // magnitude: two's complement negation
      x = ~x;
      const uint32_t sm = x + carry;
      carry = sm < x ? 1u : 0u;
      x = sm;
    }
    m[q] = x;
  }
  // whole-limb normalisation: the leading nonzero limb into m[7]
  int E = 32 * (CRT_NL - 5);  // weight of window bit 0 before any shift
#pragma unroll
  for (int step = 4; step >= 1; step >>= 1) {
    bool zero = true;
#pragma unroll
    for (int q = CRT_NL - step; q < CRT_NL; ++q) zero = zero && m[q] == 0;
    if (zero) {
#pragma unroll
      for (int q = CRT_NL - 1; q >= 0; --q) m[q] = q >= step ? m[q - step] : 0u;
      E -= 32 * step;
    }
  }
  if (m[CRT_NL - 1] == 0) {  // the value is zero
    h = l = 0.0;
    e = 0;
    return;
  }
  const int s = __clz((int)m[CRT_NL - 1]);
  uint32_t n[5];
#pragma unroll
  for (int w = 0; w < 5; ++w) n[w] = __funnelshift_l(m[CRT_NL - 6 + w], m[CRT_NL - 5 + w], s);
  E -= s;
  const uint64_t T64 = ((uint64_t)n[4] << 32) | n[3];
  uint64_t keep = T64 >> 11;
  const uint32_t r11 = (uint32_t)(T64 & 0x7FF);
  const bool lowz = (n[2] | n[1] | n[0]) == 0;
  const bool up = r11 > 0x400 || (r11 == 0x400 && (!lowz || (keep & 1)));
  keep += up;
  const int D = (int)r11 - (up ? 2048 : 0);
  double lo = mfdev::mul((double)D, pow2(96));
  lo = mfdev::add(lo, mfdev::mul((double)n[2], pow2(64)));
  lo = mfdev::add(lo, mfdev::mul((double)n[1], pow2(32)));
  lo = mfdev::add(lo, (double)n[0]);
  double hi = (double)keep;
  lo = mfdev::mul(lo, pow2(-107));  // into units of 2^(E + 107): exact
  mfdev::fast_two_sum(hi, lo, h, l);
  if (neg) {
    h = -h;
    l = -l;
  }
  e = E + 107;
}

// Writes the two's complement integer C' held in CRT_NL limbs, times
// 2^shift, as a DD to dst (NaN when `nan`); mode 0 stores it, 1 subtracts it
// from the DD at dst, 2 adds it.
__device__ __forceinline__ void crt_emit(const uint32_t (&limb)[CRT_NL], bool nan, int shift,
                                         double *__restrict__ dst, int mode) {
  double2 out;
  if (nan) {
    out = make_double2(CUDART_NAN, 0.0);
  } else {
    double hi, lo;
    int e;
    crt_to_dd(limb, CRT_NL, hi, lo, e);
    out = make_double2(scale2(hi, e + shift), scale2(lo, e + shift));
  }
  double2 *d2 = reinterpret_cast<double2 *>(dst);
  if (mode != 0) {
    const double2 prev = *d2;
    const mfdev::dd p = mfdev::make(out.x, out.y), pv = mfdev::make(prev.x, prev.y);
    const mfdev::dd res = mode == 1 ? mfdev::dd_sub(pv, p) : mfdev::dd_add(pv, p);
    out = make_double2(res.hi, res.lo);
  }
  __stcs(d2, out);
}

// Residue layout of one product (modulus t, K chunk kc): N_pad x M_pad bytes,
// four consecutive columns interleaved per row -- byte (j, i) at
// ((j / 4) M_pad + i) 4 + j % 4 -- so a thread holding one row writes one
// 32-bit word per four columns.  Word index of the element at byte offset
// off = (plane) + j M_pad + i with j % 4 == 0:
__device__ __forceinline__ int64_t crt_word_index(int64_t off, int64_t M_pad) {
  const int64_t plane = off / (4 * M_pad) * (4 * M_pad);  // (t, kc) plane plus whole column quads
  const int64_t rest = off - plane;                        // j % 4 == 0 within the quad: rest = i
  return plane / 4 + rest;
}
// The residues of four INT32 sums packed in column order.
__device__ __forceinline__ uint32_t crt_pack4(uint32_t v0, uint32_t v1, uint32_t v2, uint32_t v3, int t);

// The residue of one product reduced in the tensor-core kernel's epilogue:
// v = the INT32 sum of one K chunk of unsigned residue products
// (0 <= v < 73 * 128 * 255^2 < 2^30), stored as v mod m_t in [0, m_t).
__device__ __forceinline__ uint8_t crt_residue_of_sum(int32_t v, int t) {
  return (uint8_t)crt_mod_small((uint32_t)v, t);
}
__device__ __forceinline__ uint32_t crt_pack4(uint32_t v0, uint32_t v1, uint32_t v2, uint32_t v3, int t) {
  return __byte_perm(__byte_perm(crt_mod_small(v0, t), crt_mod_small(v1, t), 0x0040),
                     __byte_perm(crt_mod_small(v2, t), crt_mod_small(v3, t), 0x0040), 0x5410);
}

// ---- reconstruction on the tensor cores ---------------------------------------
// The sums over moduli are an integer matrix product: for an output with
// residues r_t, the column sums
//   S_b = sum_t r_t E[t][b]   (E[t][b] = byte b of round(c_t 2^24) for b < 3,
//                              0 for b = 3, byte b - 4 of e_t mod 2^(8 nbe)
//                              for 4 <= b < 4 + nbe)
// are exact in INT32 (< 36 * 255^2), so
//   V = sum_{b < nbe} S_{4+b} 2^(8b) = sum_t r_t e_t  (mod 2^(8 nbe)),
//   q = round((S_0 + S_1 2^8 + S_2 2^16) / 2^24)  (error < 36 * 255 * 2^-25 < 1/4),
//   C' = V - q M  (mod 2^(8 nbe)),
// and |C'| < 2^(8 nbe - 2) makes bit 8 nbe - 1 the sign.  One tcgen05 u8 x u8
// MMA per output column of a 128-row tile gives the S_b of 128 outputs.
// nbe = crt_tc_bytes(W, k).
constexpr int CTC_THREADS = 128;                   // one output row per thread and TMEM lane
constexpr int CTC_QUADS = 8;                       // column quads per CTA
constexpr int CTC_B_BYTES = 48 * 128;              // E tile: up to 48 rows of 128 bytes (swizzled)
constexpr int CTC_A_OFF = 8192;                    // residue tiles (1024-aligned), 16 KiB per 32 moduli
__host__ __device__ constexpr int crt_tc_smem(int ktmax) { return CTC_A_OFF + ktmax * 16384 + 1024; }

// 16 bytes at logical chunk `chunk` (0..7) of row `row` of a K-major tile with
// 128-byte rows and the 128-byte swizzle (8-row atoms of 1024 bytes).
__device__ __forceinline__ void sw128_store16(uint8_t *tile, int row, int chunk, uint4 v) {
  *reinterpret_cast<uint4 *>(tile + (row >> 3) * 1024 + (row & 7) * 128 + ((chunk ^ (row & 7)) << 4)) = v;
}
// Bytes c of the four words a, b, c, d (one residue word per modulus holds
// four columns) regrouped per column: out[c] = {a_c, b_c, c_c, d_c}.
__device__ __forceinline__ void crt_transpose4(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t (&o)[4]) {
  const uint32_t ab0 = __byte_perm(a, b, 0x5140), ab1 = __byte_perm(a, b, 0x7362);
  const uint32_t cd0 = __byte_perm(c, d, 0x5140), cd1 = __byte_perm(c, d, 0x7362);
  o[0] = __byte_perm(ab0, cd0, 0x5410);
  o[1] = __byte_perm(ab0, cd0, 0x7632);
  o[2] = __byte_perm(ab1, cd1, 0x5410);
  o[3] = __byte_perm(ab1, cd1, 0x7632);
}

// The residue word of one modulus when the K dimension came in nkc chunks:
// per column the chunks' residues summed and reduced again.  Kept out of line
// so that the reconstruction's main path stays small in the instruction cache.
static __device__ __noinline__ uint32_t crt_chunk_residue_word(const uint32_t *src, int nkc, int64_t kstride, int t) {
  uint32_t sum[4] = {0, 0, 0, 0};
  for (int kc = 0; kc < nkc; ++kc) {
    const uint32_t v = __ldcs(src + kc * kstride);
#pragma unroll
    for (int r = 0; r < 4; ++r) sum[r] += (v >> (8 * r)) & 0xFFu;
  }
  uint32_t w = 0;
#pragma unroll
  for (int r = 0; r < 4; ++r) w |= crt_mod_small(sum[r], t) << (8 * r);
  return w;
}

// CTA of CTC_THREADS threads: rows i0 .. i0+127 of column quads qd0 ..
// qd0+CTC_QUADS-1 (thread T: row i0+T, columns 4 qd .. 4 qd + 3).  `smem`
// is 1024-aligned, crt_tc_smem(ceil(n / 32)) bytes.  `status` receives
// bit 2 if the wait for the MMAs (limit wait_ns) expires.
__device__ __forceinline__ void crt_combine_tc_body(const uint8_t *__restrict__ D8, const Plan *plan,
                                                    const CrtConst *cc, const int *sigA, const int *flagA,
                                                    const int *sigB, const int *flagB, int64_t M, int64_t N,
                                                    int64_t M_pad, int64_t N_pad, int nkc, int64_t k,
                                                    double *__restrict__ C, int64_t cstride, int mode,
                                                    int64_t i0, int64_t qd0, uint8_t *smem, int *status,
                                                    uint64_t wait_ns) {
  const int T = threadIdx.x, warp = T >> 5;
  const int n = plan->S, W = plan->W;
  const int ktn = (n + 31) / 32;
  const int nbe = crt_tc_bytes(W, k), nb = crt_tc_cols(nbe);
  const uint32_t ncols = 4 * nb <= 128 ? 128u : 256u;
  uint8_t *sB = smem;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + CTC_B_BYTES);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
  uint8_t *sA = smem + CTC_A_OFF;
  if (T == 0) {
    mftc::mbar_init(bar, 1);
    mftc::fence_mbar_init();
  }
  if (warp == 0) {
    mftc::tmem_alloc(tslot, ncols);
    mftc::tmem_relinquish();
  }
  // the E tile: row b = T holds E[t][b] at byte t (moduli 32 kt .. in bytes 32 kt ..)
  if (T < CRT_EB_ROWS)
    for (int kt = 0; kt < ktn; ++kt)
      for (int h = 0; h < 2; ++h)
        sw128_store16(sB, T, 2 * kt + h, *reinterpret_cast<const uint4 *>(&cc->eb[T][32 * kt + 16 * h]));
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mftc::tc_fence_before();
  __syncthreads();
  mftc::tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = mftc::idesc_u8(128, nb);
  const int64_t i = i0 + T;
  const bool row_ok = i < M;
  const int sa = row_ok ? sigA[i] : 0, fa = row_ok ? flagA[i] : 1;
  const int64_t nq = (N + 3) / 4;
  const int64_t kstride = N_pad * M_pad / 4, gstride = (int64_t)nkc * kstride;  // in 32-bit words
  uint32_t Mw[CRT_NL];
#pragma unroll
  for (int w = 0; w < CRT_NL; ++w) Mw[w] = cc->Mw[w];
  uint32_t phase = 0;
  // the residue words of column quad qd (modulus t: four columns in a word)
  auto load_words = [&](int64_t qd, uint32_t (&wv)[CRT_NMAX]) {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(D8) + qd * M_pad + (row_ok ? i : 0);
    if (nkc == 1) {  // the common case, kept compact: one load per modulus
#pragma unroll
      for (int t = 0; t < CRT_NMAX; ++t) wv[t] = (row_ok && t < n) ? __ldcs(src + t * gstride) : 0u;
    } else {
#pragma unroll
      for (int t = 0; t < CRT_NMAX; ++t)
        wv[t] = (row_ok && t < n) ? crt_chunk_residue_word(src + t * gstride, nkc, kstride, t) : 0u;
    }
  };
  uint32_t wv[CRT_NMAX];
  const int64_t qend = min(qd0 + CTC_QUADS, nq);
  if (qd0 < qend) load_words(qd0, wv);
  for (int64_t qd = qd0; qd < qend; ++qd) {
    // residues of the four outputs into the A tiles: row T, column c at bytes
    // [32 c, 32 c + 32) of tile kt (moduli 32 kt ..)
#pragma unroll
    for (int kt = 0; kt < (CRT_NMAX + 31) / 32; ++kt) {
      if (kt >= ktn) break;
      uint32_t x[4][8];
#pragma unroll
      for (int g = 0; g < 8; ++g) {
        uint32_t o[4];
        const int t = 32 * kt + 4 * g;
        crt_transpose4(t < CRT_NMAX ? wv[t] : 0u, t + 1 < CRT_NMAX ? wv[t + 1] : 0u,
                       t + 2 < CRT_NMAX ? wv[t + 2] : 0u, t + 3 < CRT_NMAX ? wv[t + 3] : 0u, o);
#pragma unroll
        for (int c = 0; c < 4; ++c) x[c][g] = o[c];
      }
      uint8_t *tile = sA + kt * 16384;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        sw128_store16(tile, T, 2 * c, make_uint4(x[c][0], x[c][1], x[c][2], x[c][3]));
        sw128_store16(tile, T, 2 * c + 1, make_uint4(x[c][4], x[c][5], x[c][6], x[c][7]));
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mftc::tc_fence_before();
    __syncthreads();
    if (T == 0) {
      mftc::tc_fence_after();
      for (int c = 0; c < 4; ++c)
        for (int kt = 0; kt < ktn; ++kt)
          mftc::umma_i8(tmem + (uint32_t)(c * nb), mftc::smem_desc_k_sw128(mftc::smem_u32(sA + kt * 16384 + 32 * c)),
                        mftc::smem_desc_k_sw128(mftc::smem_u32(sB + 32 * kt)), idesc, kt > 0 ? 1u : 0u);
      mftc::umma_commit(bar);
    }
    if (qd + 1 < qend) load_words(qd + 1, wv);  // in flight during the MMAs and this quad's outputs
    const bool ok = wait_bar_ns(bar, phase, wait_ns);
    if (__syncthreads_or(!ok)) {  // uniform: every thread leaves together
      if (T == 0) record_abort(status, 2);  // a bounded wait expired
      // this round's MMAs may still be writing tensor memory: give them the
      // default limit to finish before the CTA frees it
      (void)wait_bar_ns(bar, phase, WAIT_NS);
      break;
    }
    phase ^= 1;
    mftc::tc_fence_after();
    const int4 sb4 = *reinterpret_cast<const int4 *>(sigB + 4 * qd);
    const int4 fb4 = *reinterpret_cast<const int4 *>(flagB + 4 * qd);
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
      uint32_t S[48];
#pragma unroll
      for (int b = 32; b < 48; ++b) S[b] = 0;
      mftc::tmem_ld_32x32b_x32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * nb), *reinterpret_cast<uint32_t(*)[32]>(S));
      if (nb > 32)
        mftc::tmem_ld_32x32b_x16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * nb + 32),
                                 *reinterpret_cast<uint32_t(*)[16]>(S + 32));
      mftc::tmem_wait_ld();
      const int64_t j = 4 * qd + c;
      if (!row_ok || j >= N) continue;
      // q from the three fixed-point columns
      const uint64_t Q = (uint64_t)(S[0] + (S[1] << 8)) + ((uint64_t)S[2] << 16);
      const uint32_t q = (uint32_t)((Q + (1u << 23)) >> 24);
      uint32_t limb[CRT_NL];
      int64_t carry = 0;
#pragma unroll
      for (int w = 0; w < CRT_NL; ++w) {
        const uint32_t lo = S[4 + 4 * w] + (S[5 + 4 * w] << 8);  // < 2^30
        const uint32_t hi = S[6 + 4 * w] + (S[7 + 4 * w] << 8);  // < 2^30
        const int64_t v = (int64_t)lo + ((int64_t)hi << 16) - (int64_t)((uint64_t)q * Mw[w]) + carry;
        limb[w] = (uint32_t)v;
        carry = v >> 32;  // arithmetic shift
      }
      // C' mod 2^(8 nbe): the top bit of limb nbe / 4 - 1 is the sign, copied above
      uint32_t top = 0;
#pragma unroll
      for (int w = 0; w < CRT_NL; ++w) top = 4 * (w + 1) == nbe ? limb[w] : top;
      const uint32_t fill = (top >> 31) ? 0xFFFFFFFFu : 0u;
#pragma unroll
      for (int w = 0; w < CRT_NL; ++w) limb[w] = 4 * w < nbe ? limb[w] : fill;
      const int sbc = c == 0 ? sb4.x : c == 1 ? sb4.y : c == 2 ? sb4.z : sb4.w;
      const int fbc = c == 0 ? fb4.x : c == 1 ? fb4.y : c == 2 ? fb4.z : fb4.w;
      crt_emit(limb, (fa | fbc) != 0, sa + sbc - 2 * W, C + 2 * (j * M + i) * cstride, mode);
    }
    mftc::tc_fence_before();  // this round's TMEM reads before the next round's MMAs
  }
  __syncthreads();
  mftc::tc_fence_after();
  if (warp == 0) mftc::tmem_dealloc(tmem, ncols);
}

}  // namespace split
}  // namespace mfcuda
