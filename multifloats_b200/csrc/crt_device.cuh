// CRT (modular) form of the split-INT8 DD GEMM: device pieces.
//
// The operands are rounded to the fixed-point grid of their row (A) / column
// (B) exactly as in the digit-sliced form -- X = round(a 2^(W - sigma_i)),
// |X| < 2^W -- and the exact integer product C' = X Y^T is recovered from its
// residues modulo N pairwise-coprime moduli m_t <= 256 (crt_tables.h): each
// residue product (X mod m_t)(Y mod m_t)^T is one INT8 GEMM on the tensor
// cores, and C' follows from the Chinese remainder theorem,
//   C' = sum_t r_t e_t - q M,   e_t = (M / m_t) ((M / m_t)^-1 mod m_t),
//   r_t = (X Y^T mod m_t) in [0, m_t),  q = round(sum_t r_t e_t / M),
// which is exact because the moduli are chosen with M > 8 k 2^(2W) > 8 |C'|.
// C' is then rounded to a double-double (hi = RN(C''), lo = RN(C'' - hi), C''
// being C' truncated to its 160 leading bits) and scaled by 2^(sigma_i + tau_j
// - 2W).  Compared with the digit-sliced form (S(S+1)/2 slice products for S
// slices) the tensor work is N products: 27 instead of 105 at 4096^3.
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

namespace mfcuda {
namespace split {

constexpr int CRT_NL = 8;  // most 32-bit limbs of a reconstruction (256 bits)
constexpr int CRT_WMAX = 110;

// Reconstruction constants of the plan's N moduli, computed on the device.
struct CrtConst {
  uint32_t e[CRT_NMAX][CRT_NL];  // e_t mod 2^256
  uint32_t M[CRT_NL];            // M mod 2^256
  double c[CRT_NMAX];            // ((M / m_t)^-1 mod m_t) / m_t, rounded
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
// Moduli needed for W-bit operands and inner dimension k: M > 8 k 2^(2W).
__host__ __device__ inline int crt_moduli(int W, int64_t k, const int *lg) {
  const int need = 2 * W + ceil_log2(k) + 3;
  int n = 1;
  while (n < CRT_NMAX && lg[n] < need) ++n;
  return n;
}
// 32-bit limbs holding |C'| < k 2^(2W) with its sign (two's complement).
__host__ __device__ inline int crt_limbs(int W, int64_t k) { return (2 * W + ceil_log2(k) + 1 + 31) / 32; }

// Inverse of a modulo m (gcd(a, m) = 1, m <= 256), extended Euclid.
__device__ __forceinline__ uint32_t inv_mod_small(uint32_t a, uint32_t m) {
  int t = 0, nt = 1, r = (int)m, nr = (int)(a % m);
  while (nr != 0) {
    const int q = r / nr;
    int tmp = t - q * nt;
    t = nt;
    nt = tmp;
    tmp = r - q * nr;
    r = nr;
    nr = tmp;
  }
  return (uint32_t)(t < 0 ? t + (int)m : t);
}

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
      W = CRT_WMAX;
      for (int w = 8; w <= CRT_WMAX; ++w)
        if (crt_bound(w, ra, rb, k) <= target) {
          W = w;
          break;
        }
    }
    const int n = crt_moduli(W, k, crt_lg);
    plan->S = n;
    plan->G = n - 1;
    plan->W = W;
    plan->rho_a = ra;
    plan->rho_b = rb;
    plan->crt = 1;
    plan->nl = crt_limbs(W, k);
    sh_n = n;
  }
  __syncthreads();
  const int n = sh_n;
  // M = prod m_t (9 limbs: M < 2^267), e_t = (M / m_t) inv_t mod 2^256
  if (threadIdx.x < (unsigned)n) {
    const int t = threadIdx.x;
    const uint32_t mt = crt_mod[t];
    uint32_t q[CRT_NL + 1];  // M / m_t = prod_{s != t} m_s
    for (int l = 0; l <= CRT_NL; ++l) q[l] = 0;
    q[0] = 1;
    uint32_t rem = 1;  // (M / m_t) mod m_t
    for (int s = 0; s < n; ++s) {
      if (s == t) continue;
      const uint32_t ms = crt_mod[s];
      uint64_t carry = 0;
      for (int l = 0; l <= CRT_NL; ++l) {
        const uint64_t v = (uint64_t)q[l] * ms + carry;
        q[l] = (uint32_t)v;
        carry = v >> 32;
      }
      rem = (rem * (ms % mt)) % mt;
    }
    const uint32_t inv = inv_mod_small(rem, mt);
    uint64_t carry = 0;
    for (int l = 0; l < CRT_NL; ++l) {
      const uint64_t v = (uint64_t)q[l] * inv + carry;
      cc->e[t][l] = (uint32_t)v;
      carry = v >> 32;
    }
    cc->c[t] = (double)inv / (double)mt;
    if (t == 0) {  // M = (M / m_0) m_0
      uint64_t cy = 0;
      for (int l = 0; l < CRT_NL; ++l) {
        const uint64_t v = (uint64_t)q[l] * mt + cy;
        cc->M[l] = (uint32_t)v;
        cy = v >> 32;
      }
    }
  }
  __syncthreads();
  for (int o = 0; o < st.n; ++o)
    for (int64_t i = threadIdx.x; i < st.count[o]; i += blockDim.x)
      if (st.sig[o][i] == SENT_LO) st.sig[o][i] = 0;
}

// ---- residue slicing ----------------------------------------------------------
// The signed residue of X = sum_q d_q 256^q (balanced digits, read from the
// biased words y of biased_bytes: digit q = byte q of y xor 0x80) modulo m_t,
// in [crt_rlo, crt_rhi]: four dp4a against the digit weights give
// rr = sum_q d_q c_q with |rr| < 14 * 128 * 128 < 2^18, then one rounded
// float quotient and two range corrections.
__device__ __forceinline__ int crt_residue(const uint32_t (&dw)[4], int t) {
  int rr = __dp4a((int)dw[3], (int)crt_digw[t][3], 0);
  rr = __dp4a((int)dw[2], (int)crt_digw[t][2], rr);
  rr = __dp4a((int)dw[1], (int)crt_digw[t][1], rr);
  rr = __dp4a((int)dw[0], (int)crt_digw[t][0], rr);
  const int m = (int)crt_mod[t];
  const int q = __float2int_rn(__int2float_rn(rr) * __uint_as_float(crt_inv_bits[t]));
  int r = rr - q * m;
  r = r > crt_rhi[t] ? r - m : r;
  r = r < crt_rlo[t] ? r + m : r;
  return r;
}
// Signed digit words of the biased words of one entry.
__device__ __forceinline__ void digit_words(const uint32_t (&y)[4], uint32_t (&dw)[4]) {
#pragma unroll
  for (int w = 0; w < 4; ++w) dw[w] = y[w] ^ bias_word(w);
}
// Calls f(t, word) with the residues modulo m_t of 8 entries packed in entry
// order (byte e = entry e), for t < n.
template <class F>
__device__ __forceinline__ void for_each_residue_word(const uint32_t (&y)[8][4], int n, F f) {
  uint32_t dw[8][4];
#pragma unroll
  for (int e = 0; e < 8; ++e) digit_words(y[e], dw[e]);
  for (int t = 0; t < n; ++t) {
    uint32_t lo = 0, hi = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) lo |= ((uint32_t)crt_residue(dw[e], t) & 0xFFu) << (8 * e);
#pragma unroll
    for (int e = 0; e < 4; ++e) hi |= ((uint32_t)crt_residue(dw[e + 4], t) & 0xFFu) << (8 * e);
    f(t, (uint64_t)lo | ((uint64_t)hi << 32));
  }
}

// A (m x k column-major view) -> As[t][i][p], as slice_a_body with residues
// for digits; the transposing tile lives in dynamic shared memory
// (n * SA_ROWS * SA_STRIDE bytes).
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
  for_each_residue_word(y, n, [&](int sl, uint64_t word) {
    *reinterpret_cast<uint64_t *>(&tile[(sl * SA_ROWS + ii) * SA_STRIDE + grp * 8]) = word;
  });
  __syncthreads();
  const int row = t / 8, seg = (t % 8) * 8;
  for (int s = 0; s < n; ++s) {
    uint64_t v = *reinterpret_cast<const uint64_t *>(&tile[(s * SA_ROWS + row) * SA_STRIDE + seg]);
    *reinterpret_cast<uint64_t *>(As + ((s * M_pad + i0 + row) * K_pad + p0 + seg)) = v;
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
  for_each_residue_word(y, n, [&](int sl, uint64_t word) {
    *reinterpret_cast<uint64_t *>(Bs + (((int64_t)sl * N_pad + j) * K_pad + p8)) = word;
  });
}

// ---- reconstruction ---------------------------------------------------------------
// RN to 53 bits of the unsigned integer u < 2^127, as (integer mantissa, shift):
// value = mant 2^sh, mant <= 2^53.
__device__ __forceinline__ void rn53(unsigned __int128 u, uint64_t &mant, int &sh) {
  const uint64_t hi = (uint64_t)(u >> 64), lo = (uint64_t)u;
  const int lead = hi ? 127 - __clzll((long long)hi) : (lo ? 63 - __clzll((long long)lo) : -1);
  if (lead <= 52) {
    mant = lo;
    sh = 0;
    return;
  }
  sh = lead - 52;
  const unsigned __int128 keep = u >> sh;
  const unsigned __int128 rem = u - (keep << sh), half = (unsigned __int128)1 << (sh - 1);
  uint64_t k = (uint64_t)keep;
  if (rem > half || (rem == half && (k & 1))) ++k;
  mant = k;
}

// The signed integer held in nl little-endian 32-bit limbs (two's complement)
// as a double-double (hi, lo) with exponents: value ~ hi 2^eh + lo 2^el, hi
// and lo integers of at most 53 bits (exact as doubles).  C'' = |C'| truncated
// to its 160 leading bits; hi = RN(C''), lo = RN(C'' - hi).
__device__ __forceinline__ void crt_to_dd(const uint32_t *limb, int nl, double &hi, int &eh, double &lo,
                                          int &el) {
  uint32_t v[CRT_NL + 5];
  const bool neg = (limb[nl - 1] >> 31) != 0;
  uint32_t carry = 1;
#pragma unroll
  for (int l = 0; l < CRT_NL; ++l) {
    uint32_t x = l < nl ? limb[l] : (neg ? 0xFFFFFFFFu : 0u);
    if (neg) {  // magnitude: two's complement negation
      x = ~x;
      const uint32_t s = x + carry;
      carry = (s < x) ? 1u : 0u;
      x = s;
    }
    v[l + 5] = x;
  }
#pragma unroll
  for (int l = 0; l < 5; ++l) v[l] = 0;
  // top nonzero limb (index into v)
  int tl = -1;
#pragma unroll
  for (int l = CRT_NL + 4; l >= 5; --l)
    if (tl < 0 && v[l] != 0) tl = l;
  if (tl < 0) {
    hi = lo = 0.0;
    eh = el = 0;
    return;
  }
  const int s = __clz((int)v[tl]);
  // 160-bit window n4..n0, leading one at bit 159; bit 0 has weight 2^E
  uint32_t n[5];
#pragma unroll
  for (int w = 0; w < 5; ++w) {
    const uint32_t a = v[tl - w], b = v[tl - w - 1];
    n[4 - w] = s ? (a << s) | (b >> (32 - s)) : a;
  }
  const int E = 32 * (tl - 5 - 4) - s;
  const uint64_t T64 = ((uint64_t)n[4] << 32) | n[3];
  uint64_t keep = T64 >> 11;
  const uint32_t r11 = (uint32_t)(T64 & 0x7FF);
  const bool lowz = (n[2] | n[1] | n[0]) == 0;
  const bool up = r11 > 0x400 || (r11 == 0x400 && (!lowz || (keep & 1)));
  keep += up;
  hi = (double)keep;
  eh = E + 107;
  const __int128 R = ((__int128)((int64_t)r11 - (up ? 2048 : 0)) << 96) + ((__int128)n[2] << 64) +
                     ((__int128)n[1] << 32) + (__int128)n[0];
  const unsigned __int128 u = R < 0 ? (unsigned __int128)(-R) : (unsigned __int128)R;
  uint64_t mant;
  int sh;
  rn53(u, mant, sh);
  lo = R < 0 ? -(double)mant : (double)mant;
  el = E + sh;
  if (neg) {
    hi = -hi;
    lo = -lo;
  }
}

// One output: residues of its N products (summed over the K chunks) -> C' ->
// DD, scaled by 2^ex.  Constants from shared memory.
struct CrtShared {
  uint32_t e[CRT_NMAX][CRT_NL];
  uint32_t M[CRT_NL];
  double c[CRT_NMAX];
  double minv[CRT_NMAX];  // 1 / m_t rounded (quotient estimate, corrected below)
};
// Block prologue: the plan's constants into shared memory.
__device__ __forceinline__ void crt_load_shared(const CrtConst *cc, int n, CrtShared &cs) {
  for (int x = threadIdx.x; x < n * CRT_NL; x += blockDim.x) cs.e[x / CRT_NL][x % CRT_NL] = cc->e[x / CRT_NL][x % CRT_NL];
  for (int x = threadIdx.x; x < CRT_NL; x += blockDim.x) cs.M[x] = cc->M[x];
  for (int x = threadIdx.x; x < n; x += blockDim.x) {
    cs.c[x] = cc->c[x];
    cs.minv[x] = 1.0 / (double)crt_mod[x];
  }
  __syncthreads();
}
__device__ __forceinline__ double2 crt_output(const int32_t *__restrict__ D, int64_t gstride, int64_t kstride,
                                              int nkc, int n, int nl, const CrtShared &cs, int ex) {
  uint32_t r[CRT_NMAX];
  double f = 0.0;
  for (int t = 0; t < n; ++t) {
    int64_t v = 0;
    for (int kc = 0; kc < nkc; ++kc) v += __ldcs(D + t * gstride + kc * kstride);
    // v mod m_t in [0, m_t): |v| < 2^53, quotient from the rounded reciprocal,
    // off by at most one, then corrected
    const int64_t m = crt_mod[t];
    const int64_t qq = (int64_t)floor((double)v * cs.minv[t]);
    int64_t rt = v - qq * m;
    rt = rt < 0 ? rt + m : (rt >= m ? rt - m : rt);
    r[t] = (uint32_t)rt;
    f = __fma_rn((double)rt, cs.c[t], f);
  }
  const int64_t q = (int64_t)rint(f);
  int64_t acc[CRT_NL];
#pragma unroll
  for (int l = 0; l < CRT_NL; ++l) acc[l] = -(int64_t)q * (int64_t)cs.M[l];
  for (int t = 0; t < n; ++t) {
    const uint64_t rt = r[t];
#pragma unroll
    for (int l = 0; l < CRT_NL; ++l) acc[l] += (int64_t)(rt * cs.e[t][l]);
  }
  uint32_t limb[CRT_NL];
  int64_t carry = 0;
#pragma unroll
  for (int l = 0; l < CRT_NL; ++l) {
    const int64_t x = acc[l] + carry;
    limb[l] = (uint32_t)x;
    carry = x >> 32;  // arithmetic shift
  }
  double hi, lo;
  int eh, el;
  crt_to_dd(limb, nl, hi, eh, lo, el);
  return make_double2(scale2(hi, eh + ex), scale2(lo, el + ex));
}

}  // namespace split
}  // namespace mfcuda
