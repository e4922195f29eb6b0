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

namespace mfcuda {
namespace split {

constexpr int CRT_NL = 8;  // most 32-bit limbs of a reconstruction (256 bits)
constexpr int CRT_BATCH = 9;  // moduli whose residues a reconstruction thread loads at once
constexpr int CRT_WMAX = 110;

// Reconstruction constants of the plan's N moduli, computed on the device.
// The reconstruction sums r_t e_t in 39-bit limbs held in doubles: a residue
// (< 2^8) times a limb (< 2^39) is exact, and so are sums of up to 36 such
// products (< 2^53), so the FP64 pipe does the multiply-adds exactly.
constexpr int CRT_LB = 39;   // bits per reconstruction limb
constexpr int CRT_NL39 = 7;  // limbs: 273 bits >= 2W + log2(k) + 1 for W <= 110, k < 2^31
struct CrtConst {
  double e[CRT_NMAX][CRT_NL39];  // e_t mod 2^273, 39-bit limbs
  double M[CRT_NL39];            // M mod 2^273, 39-bit limbs
  double c[CRT_NMAX];            // ((M / m_t)^-1 mod m_t) / m_t, rounded: q = round(sum_t r_t c_t)
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
// 39-bit limbs holding |C'| < k 2^(2W) with its sign (two's complement).
__host__ __device__ inline int crt_limbs(int W, int64_t k) {
  return (2 * W + ceil_log2(k) + 1 + CRT_LB - 1) / CRT_LB;
}
// Bits [39 l, 39 l + 39) of the little-endian 32-bit limbs v (>= 11 limbs), as a double.
__device__ __forceinline__ double limb39(const uint32_t *v, int l) {
  const int b = CRT_LB * l, w = b / 32, o = b % 32;
  uint64_t x = ((uint64_t)v[w + 1] << 32) | v[w];
  x >>= o;
  if (o + CRT_LB > 64) x |= (uint64_t)v[w + 2] << (64 - o);
  return (double)(x & ((1ull << CRT_LB) - 1));
}

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
    uint32_t ev[CRT_NL + 3];  // e_t mod 2^288 (9 limbs) and two zero limbs for limb39
    uint64_t carry = 0;
    for (int l = 0; l <= CRT_NL; ++l) {
      const uint64_t v = (uint64_t)q[l] * inv + carry;
      ev[l] = (uint32_t)v;
      carry = v >> 32;
    }
    ev[CRT_NL + 1] = ev[CRT_NL + 2] = 0;
    for (int l = 0; l < CRT_NL39; ++l) cc->e[t][l] = limb39(ev, l);
    cc->c[t] = (double)inv / (double)mt;
    if (t == 0) {  // M = (M / m_0) m_0
      uint32_t mv[CRT_NL + 3];
      uint64_t cy = 0;
      for (int l = 0; l <= CRT_NL; ++l) {
        const uint64_t v = (uint64_t)q[l] * mt + cy;
        mv[l] = (uint32_t)v;
        cy = v >> 32;
      }
      mv[CRT_NL + 1] = mv[CRT_NL + 2] = 0;
      for (int l = 0; l < CRT_NL39; ++l) cc->M[l] = limb39(mv, l);
    }
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
// < 2^18, made non-negative and reduced exactly.  The per-modulus constants
// are passed in (hoisted by the caller).  NW = digit words in use: 3 when
// W <= 94 (digits 12 and 13 are zero).
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
  int rr = NW == 4 ? __dp4a((int)dw[3], k.c3, 0) : 0;
  rr = __dp4a((int)dw[2], k.c2, rr);
  rr = __dp4a((int)dw[1], k.c1, rr);
  rr = __dp4a((int)dw[0], k.c0, rr);
  const uint32_t u = (uint32_t)rr + k.off;  // in [0, 2^19 + 256)
  const int r = (int)(u - __umulhi(u, k.mu) * k.m);
  return (uint32_t)(r < 0 ? r + (int)k.m : r);
}
// Signed digit words of the biased words of one entry.
__device__ __forceinline__ void digit_words(const uint32_t (&y)[4], uint32_t (&dw)[4]) {
#pragma unroll
  for (int w = 0; w < 4; ++w) dw[w] = y[w] ^ bias_word(w);
}
// Calls f(t, word) with the residues modulo m_t of 8 entries packed in entry
// order (byte e = entry e), for t < n.
template <int NW, class F>
__device__ __forceinline__ void residue_words_nw(const uint32_t (&dw)[8][4], int n, F f) {
  for (int t = 0; t < n; ++t) {
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
__device__ __forceinline__ void for_each_residue_word(const uint32_t (&y)[8][4], int n, int W, F f) {
  uint32_t dw[8][4];
#pragma unroll
  for (int e = 0; e < 8; ++e) digit_words(y[e], dw[e]);
  if (W <= 94)
    residue_words_nw<3>(dw, n, f);
  else
    residue_words_nw<4>(dw, n, f);
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
  for_each_residue_word(y, n, W, [&](int sl, uint64_t word) {
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
  for_each_residue_word(y, n, W, [&](int sl, uint64_t word) {
    *reinterpret_cast<uint64_t *>(Bs + (((int64_t)sl * N_pad + j) * K_pad + p8)) = word;
  });
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

// Reconstruction constants in shared memory.
struct CrtShared {
  double e[CRT_NMAX][CRT_NL39];
  double M[CRT_NL39];
  double c[CRT_NMAX];
};
// Block prologue: the plan's constants into shared memory.
__device__ __forceinline__ void crt_load_shared(const CrtConst *cc, int n, CrtShared &cs) {
  for (int x = threadIdx.x; x < n * CRT_NL39; x += blockDim.x)
    cs.e[x / CRT_NL39][x % CRT_NL39] = cc->e[x / CRT_NL39][x % CRT_NL39];
  for (int x = threadIdx.x; x < CRT_NL39; x += blockDim.x) cs.M[x] = cc->M[x];
  for (int x = threadIdx.x; x < n; x += blockDim.x) cs.c[x] = cc->c[x];
  __syncthreads();
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

// Row i of columns j0 .. j0+3 (j0 % 4 == 0): the residues r_t (one 32-bit load
// per modulus and K chunk from the column-quad layout of crt_word_index), then
//   q = round(sum_t r_t c_t),  C' = sum_t r_t e_t - q M  in 39-bit limbs,
// every limb an exact FP64 multiply-add (see CRT_LB), carried in int64 and
// repacked into 32-bit limbs; the DD conversion and exact scaling; `mode` as
// the digit-sliced combine.
__device__ __forceinline__ void crt_combine4_body(const uint8_t *__restrict__ D8, const Plan *plan,
                                                  const CrtShared &cs, const int *sigA, const int *flagA,
                                                  const int *sigB, const int *flagB, int64_t M, int64_t N,
                                                  int64_t M_pad, int64_t N_pad, int nkc, double *__restrict__ C,
                                                  int64_t cstride, int mode, int64_t i, int64_t j0) {
  const int n = plan->S, nl = plan->nl, W = plan->W;
  if (i >= M || j0 >= N) return;
  const int64_t kstride = N_pad * M_pad / 4, gstride = (int64_t)nkc * kstride;  // in 32-bit words
  const uint32_t *src = reinterpret_cast<const uint32_t *>(D8) + (j0 / 4) * M_pad + i;
  double acc[4][CRT_NL39], f[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    f[r] = 0.0;
#pragma unroll
    for (int l = 0; l < CRT_NL39; ++l) acc[r][l] = 0.0;
  }
  // moduli in batches of CRT_BATCH: the batch's loads are all in flight before
  // its arithmetic
  for (int t0 = 0; t0 < n; t0 += CRT_BATCH) {
    uint32_t wv[CRT_BATCH];
#pragma unroll
    for (int u = 0; u < CRT_BATCH; ++u) {
      const int t = t0 + u;
      if (t >= n) {
        wv[u] = 0;
      } else if (nkc == 1) {
        wv[u] = __ldcs(src + t * gstride);
      } else {  // per-row sums of the chunks' residues, reduced again
        uint32_t sum[4] = {0, 0, 0, 0};
        for (int kc = 0; kc < nkc; ++kc) {
          const uint32_t w = __ldcs(src + t * gstride + kc * kstride);
#pragma unroll
          for (int r = 0; r < 4; ++r) sum[r] += (w >> (8 * r)) & 0xFFu;
        }
        uint32_t packed = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) packed |= crt_mod_small(sum[r], t) << (8 * r);
        wv[u] = packed;
      }
    }
#pragma unroll
    for (int u = 0; u < CRT_BATCH; ++u) {
      const int t = t0 + u;
      if (t < n) {
        const double ct = cs.c[t];
        double rd[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          // the residue byte as a double: 2^52 + r_t exactly, minus 2^52
          rd[r] = mfdev::sub(__hiloint2double(0x43300000, (int)((wv[u] >> (8 * r)) & 0xFFu)), 0x1p52);
          f[r] = mfdev::fma_(rd[r], ct, f[r]);
        }
        // each limb constant loaded once for the thread's four rows
#pragma unroll
        for (int l = 0; l < CRT_NL39; ++l)
          if (l < nl) {
            const double el = cs.e[t][l];
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[r][l] = mfdev::fma_(rd[r], el, acc[r][l]);
          }
      }
    }
  }
  const int4 sb4 = *reinterpret_cast<const int4 *>(sigB + j0);
  const int4 fb4 = *reinterpret_cast<const int4 *>(flagB + j0);
  const int sbv[4] = {sb4.x, sb4.y, sb4.z, sb4.w}, fbv[4] = {fb4.x, fb4.y, fb4.z, fb4.w};
  const int sa = sigA[i], fa = flagA[i];
#pragma unroll
  for (int r = 0; r < 4; ++r) {  // r: column j0 + r
    const int64_t j = j0 + r;
    if (j >= N) break;
    // |sum_t r_t e_t / M - C'/M - q| < 1/4 + rounding, so rint gives q exactly
    const double q = rint(f[r]);
    uint64_t L[CRT_NL39];
    int64_t carry = 0;
#pragma unroll
    for (int l = 0; l < CRT_NL39; ++l) {
      // acc - q M: both exact integers below 2^53, so the FMA is exact
      const int64_t x = (l < nl ? __double2ll_rn(mfdev::fma_(-q, cs.M[l], acc[r][l])) : 0) + carry;
      L[l] = (uint64_t)x & ((1ull << CRT_LB) - 1);
      carry = x >> CRT_LB;  // arithmetic shift
    }
    (void)carry;
    // C' mod 2^(39 nl) is exact (e and M are truncated there, so the carry out
    // of the top limb is not the sign); |C'| < 2^(39 nl - 1), so the top bit of
    // limb nl - 1 is the sign, copied into the limbs above
    uint64_t top = 0;
#pragma unroll
    for (int l = 0; l < CRT_NL39; ++l) top = l == nl - 1 ? L[l] : top;
    const uint64_t fill = (top >> (CRT_LB - 1)) & 1 ? (1ull << CRT_LB) - 1 : 0;
#pragma unroll
    for (int l = 0; l < CRT_NL39; ++l) L[l] = l < nl ? L[l] : fill;
    // repack the two's complement value into 8 32-bit limbs
    uint32_t limb[CRT_NL];
#pragma unroll
    for (int o = 0; o < CRT_NL; ++o) {
      const int b = 32 * o, l1 = b / CRT_LB, off = b % CRT_LB;
      uint64_t x = L[l1] >> off;
      if (off + 32 > CRT_LB) x |= (l1 + 1 < CRT_NL39 ? L[l1 + 1] : fill) << (CRT_LB - off);
      limb[o] = (uint32_t)x;
    }
    double2 out;
    if (fa | fbv[r]) {
      out = make_double2(CUDART_NAN, 0.0);
    } else {
      double hi, lo;
      int e;
      crt_to_dd(limb, CRT_NL, hi, lo, e);
      const int ex = e + sa + sbv[r] - 2 * W;
      out = make_double2(scale2(hi, ex), scale2(lo, ex));
    }
    double2 *dst = reinterpret_cast<double2 *>(C) + (j * M + i) * cstride;
    if (mode != 0) {
      const double2 prev = *dst;
      const mfdev::dd p = mfdev::make(out.x, out.y), pv = mfdev::make(prev.x, prev.y);
      const mfdev::dd res = mode == 1 ? mfdev::dd_sub(pv, p) : mfdev::dd_add(pv, p);
      out = make_double2(res.hi, res.lo);
    }
    __stcs(dst, out);
  }
}

}  // namespace split
}  // namespace mfcuda
