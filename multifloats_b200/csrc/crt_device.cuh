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
// C' is then converted to a double-double (crt_to_dd_nl: hi = C' rounded to 53
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
  // unrolled over the whole table (leaving at t1): each modulus' constants
  // are then constant-bank operands at fixed offsets instead of loads
#pragma unroll
  for (int t = 0; t < CRT_NMAX; ++t) {
    if (t >= t1) break;
    if (t < t0) continue;
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
// A (m x k column-major view) -> As[t][p][i]: the MN-major residue planes
// of the tensor-core kernels (the rows of one K index
// contiguous, so a thread's eight residues of consecutive rows are one
// 64-bit store and a warp's stores are contiguous; no transposition).
// Entries i8 .. i8+7 of column p.
__device__ __forceinline__ void crt_slice_a_mn_one(const double *__restrict__ A, int64_t M, int64_t K,
                                                   int64_t stride, int64_t M_pad, int64_t K_pad, const int *sig,
                                                   const int *flag, const Plan *plan, int8_t *__restrict__ As,
                                                   int64_t i8, int64_t p) {
  const int n = plan->S, W = plan->W;
  uint32_t y[8][4];
  bool any = false;
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int64_t i = i8 + e;
    if (p < K && i < M && !flag[i]) {
      const double2 v = __ldg(reinterpret_cast<const double2 *>(A) + (p * M + i) * stride);
      biased_bytes(v.x, v.y, sig[i], W, y[e]);
      any = true;
    } else {
#pragma unroll
      for (int w = 0; w < 4; ++w) y[e][w] = bias_word(w);  // X = 0: every residue zero
    }
  }
  auto put = [&](int sl, uint64_t word) {
    *reinterpret_cast<uint64_t *>(As + (((int64_t)sl * K_pad + p) * M_pad + i8)) = word;
  };
  if (any) {
    uint32_t dw[8][4];
#pragma unroll
    for (int e = 0; e < 8; ++e) digit_words(y[e], dw[e]);
    for_each_residue_word(dw, 0, n, W, put);
  } else {  // padding or flagged rows only: every residue zero
    for (int sl = 0; sl < n; ++sl) put(sl, 0);
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
// The residues of four INT32 sums of one K chunk of unsigned residue products
// (0 <= v < 73 * 128 * 255^2 < 2^30), each v mod m_t in [0, m_t), packed in
// column order (the tensor-core kernel's epilogue).
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

// One output from its column sums S with NL-limb arithmetic (defined below,
// after the limb-count specialisations); Mn8 = -M mod 2^256.
template <int NL>
__device__ __forceinline__ void crt_out_nl(const uint32_t (&S)[48], const uint32_t (&Mn8)[CRT_NL], int nbe,
                                           bool nan, int shift, double *__restrict__ dst, int mode);

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
  uint32_t Mn8[CRT_NL];  // -M mod 2^256: its low NL limbs are -M mod 2^(32 NL)
  {
    uint64_t carry = 1;
#pragma unroll
    for (int w = 0; w < CRT_NL; ++w) {
      const uint64_t v = (uint64_t)(~cc->Mw[w]) + carry;
      Mn8[w] = (uint32_t)v;
      carry = v >> 32;
    }
  }
  const int nl = nbe / 4;
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

      const int sbc = c == 0 ? sb4.x : c == 1 ? sb4.y : c == 2 ? sb4.z : sb4.w;
      const int fbc = c == 0 ? fb4.x : c == 1 ? fb4.y : c == 2 ? fb4.z : fb4.w;
      const bool nan = (fa | fbc) != 0;
      const int shift = sa + sbc - 2 * W;
      double *dst = C + 2 * (j * M + i) * cstride;
      if (nl <= 5)
        crt_out_nl<5>(S, Mn8, nbe, nan, shift, dst, mode);
      else if (nl == 6)
        crt_out_nl<6>(S, Mn8, nbe, nan, shift, dst, mode);
      else if (nl == 7)
        crt_out_nl<7>(S, Mn8, nbe, nan, shift, dst, mode);
      else
        crt_out_nl<8>(S, Mn8, nbe, nan, shift, dst, mode);
    }
    mftc::tc_fence_before();  // this round's TMEM reads before the next round's MMAs
  }
  __syncthreads();
  mftc::tc_fence_after();
  if (warp == 0) mftc::tmem_dealloc(tmem, ncols);
}

// ---- per-output arithmetic specialised on the limb count ------------------------
// NL = max(5, nbe / 4) 32-bit limbs (the reconstruction's width, uniform in a
// launch, so the callers dispatch on it once), with the multi-word additions
// as PTX carry chains:
//   crt_limb_chain: r = lo + H + q Mn  (mod 2^(32 NL)),
//   crt_inc_chain:  m = x + c          (mod 2^(32 NL)).
template <int NL>
__device__ __forceinline__ void crt_limb_chain(const uint32_t (&lo)[NL], const uint32_t (&H)[NL], uint32_t q,
                                               const uint32_t (&Mn)[NL], uint32_t (&r)[NL]);
template <int NL>
__device__ __forceinline__ void crt_inc_chain(const uint32_t (&x)[NL], uint32_t c, uint32_t (&m)[NL]);
template <>
__device__ __forceinline__ void crt_limb_chain<5>(const uint32_t (&lo)[5], const uint32_t (&H)[5], uint32_t q,
                                                   const uint32_t (&Mn)[5], uint32_t (&r)[5]) {
  asm("{\n\t"
      "add.cc.u32 %0, %5, %10;\n\t"
      "addc.cc.u32 %1, %6, %11;\n\t"
      "addc.cc.u32 %2, %7, %12;\n\t"
      "addc.cc.u32 %3, %8, %13;\n\t"
      "addc.u32 %4, %9, %14;\n\t"
      "mad.lo.cc.u32 %0, %15, %16, %0;\n\t"
      "madc.lo.cc.u32 %1, %15, %17, %1;\n\t"
      "madc.lo.cc.u32 %2, %15, %18, %2;\n\t"
      "madc.lo.cc.u32 %3, %15, %19, %3;\n\t"
      "madc.lo.u32 %4, %15, %20, %4;\n\t"
      "mad.hi.cc.u32 %1, %15, %16, %1;\n\t"
      "madc.hi.cc.u32 %2, %15, %17, %2;\n\t"
      "madc.hi.cc.u32 %3, %15, %18, %3;\n\t"
      "madc.hi.u32 %4, %15, %19, %4;\n\t"
      "}"
      : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3]), "=&r"(r[4])
      : "r"(lo[0]), "r"(lo[1]), "r"(lo[2]), "r"(lo[3]), "r"(lo[4]), "r"(H[0]), "r"(H[1]), "r"(H[2]), "r"(H[3]), "r"(H[4]), "r"(q), "r"(Mn[0]), "r"(Mn[1]), "r"(Mn[2]), "r"(Mn[3]), "r"(Mn[4]));
}
template <>
__device__ __forceinline__ void crt_limb_chain<6>(const uint32_t (&lo)[6], const uint32_t (&H)[6], uint32_t q,
                                                   const uint32_t (&Mn)[6], uint32_t (&r)[6]) {
  asm("{\n\t"
      "add.cc.u32 %0, %6, %12;\n\t"
      "addc.cc.u32 %1, %7, %13;\n\t"
      "addc.cc.u32 %2, %8, %14;\n\t"
      "addc.cc.u32 %3, %9, %15;\n\t"
      "addc.cc.u32 %4, %10, %16;\n\t"
      "addc.u32 %5, %11, %17;\n\t"
      "mad.lo.cc.u32 %0, %18, %19, %0;\n\t"
      "madc.lo.cc.u32 %1, %18, %20, %1;\n\t"
      "madc.lo.cc.u32 %2, %18, %21, %2;\n\t"
      "madc.lo.cc.u32 %3, %18, %22, %3;\n\t"
      "madc.lo.cc.u32 %4, %18, %23, %4;\n\t"
      "madc.lo.u32 %5, %18, %24, %5;\n\t"
      "mad.hi.cc.u32 %1, %18, %19, %1;\n\t"
      "madc.hi.cc.u32 %2, %18, %20, %2;\n\t"
      "madc.hi.cc.u32 %3, %18, %21, %3;\n\t"
      "madc.hi.cc.u32 %4, %18, %22, %4;\n\t"
      "madc.hi.u32 %5, %18, %23, %5;\n\t"
      "}"
      : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3]), "=&r"(r[4]), "=&r"(r[5])
      : "r"(lo[0]), "r"(lo[1]), "r"(lo[2]), "r"(lo[3]), "r"(lo[4]), "r"(lo[5]), "r"(H[0]), "r"(H[1]), "r"(H[2]), "r"(H[3]), "r"(H[4]), "r"(H[5]), "r"(q), "r"(Mn[0]), "r"(Mn[1]), "r"(Mn[2]), "r"(Mn[3]), "r"(Mn[4]), "r"(Mn[5]));
}
template <>
__device__ __forceinline__ void crt_limb_chain<7>(const uint32_t (&lo)[7], const uint32_t (&H)[7], uint32_t q,
                                                   const uint32_t (&Mn)[7], uint32_t (&r)[7]) {
  asm("{\n\t"
      "add.cc.u32 %0, %7, %14;\n\t"
      "addc.cc.u32 %1, %8, %15;\n\t"
      "addc.cc.u32 %2, %9, %16;\n\t"
      "addc.cc.u32 %3, %10, %17;\n\t"
      "addc.cc.u32 %4, %11, %18;\n\t"
      "addc.cc.u32 %5, %12, %19;\n\t"
      "addc.u32 %6, %13, %20;\n\t"
      "mad.lo.cc.u32 %0, %21, %22, %0;\n\t"
      "madc.lo.cc.u32 %1, %21, %23, %1;\n\t"
      "madc.lo.cc.u32 %2, %21, %24, %2;\n\t"
      "madc.lo.cc.u32 %3, %21, %25, %3;\n\t"
      "madc.lo.cc.u32 %4, %21, %26, %4;\n\t"
      "madc.lo.cc.u32 %5, %21, %27, %5;\n\t"
      "madc.lo.u32 %6, %21, %28, %6;\n\t"
      "mad.hi.cc.u32 %1, %21, %22, %1;\n\t"
      "madc.hi.cc.u32 %2, %21, %23, %2;\n\t"
      "madc.hi.cc.u32 %3, %21, %24, %3;\n\t"
      "madc.hi.cc.u32 %4, %21, %25, %4;\n\t"
      "madc.hi.cc.u32 %5, %21, %26, %5;\n\t"
      "madc.hi.u32 %6, %21, %27, %6;\n\t"
      "}"
      : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3]), "=&r"(r[4]), "=&r"(r[5]), "=&r"(r[6])
      : "r"(lo[0]), "r"(lo[1]), "r"(lo[2]), "r"(lo[3]), "r"(lo[4]), "r"(lo[5]), "r"(lo[6]), "r"(H[0]), "r"(H[1]), "r"(H[2]), "r"(H[3]), "r"(H[4]), "r"(H[5]), "r"(H[6]), "r"(q), "r"(Mn[0]), "r"(Mn[1]), "r"(Mn[2]), "r"(Mn[3]), "r"(Mn[4]), "r"(Mn[5]), "r"(Mn[6]));
}
template <>
__device__ __forceinline__ void crt_limb_chain<8>(const uint32_t (&lo)[8], const uint32_t (&H)[8], uint32_t q,
                                                   const uint32_t (&Mn)[8], uint32_t (&r)[8]) {
  asm("{\n\t"
      "add.cc.u32 %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32 %7, %15, %23;\n\t"
      "mad.lo.cc.u32 %0, %24, %25, %0;\n\t"
      "madc.lo.cc.u32 %1, %24, %26, %1;\n\t"
      "madc.lo.cc.u32 %2, %24, %27, %2;\n\t"
      "madc.lo.cc.u32 %3, %24, %28, %3;\n\t"
      "madc.lo.cc.u32 %4, %24, %29, %4;\n\t"
      "madc.lo.cc.u32 %5, %24, %30, %5;\n\t"
      "madc.lo.cc.u32 %6, %24, %31, %6;\n\t"
      "madc.lo.u32 %7, %24, %32, %7;\n\t"
      "mad.hi.cc.u32 %1, %24, %25, %1;\n\t"
      "madc.hi.cc.u32 %2, %24, %26, %2;\n\t"
      "madc.hi.cc.u32 %3, %24, %27, %3;\n\t"
      "madc.hi.cc.u32 %4, %24, %28, %4;\n\t"
      "madc.hi.cc.u32 %5, %24, %29, %5;\n\t"
      "madc.hi.cc.u32 %6, %24, %30, %6;\n\t"
      "madc.hi.u32 %7, %24, %31, %7;\n\t"
      "}"
      : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3]), "=&r"(r[4]), "=&r"(r[5]), "=&r"(r[6]), "=&r"(r[7])
      : "r"(lo[0]), "r"(lo[1]), "r"(lo[2]), "r"(lo[3]), "r"(lo[4]), "r"(lo[5]), "r"(lo[6]), "r"(lo[7]), "r"(H[0]), "r"(H[1]), "r"(H[2]), "r"(H[3]), "r"(H[4]), "r"(H[5]), "r"(H[6]), "r"(H[7]), "r"(q), "r"(Mn[0]), "r"(Mn[1]), "r"(Mn[2]), "r"(Mn[3]), "r"(Mn[4]), "r"(Mn[5]), "r"(Mn[6]), "r"(Mn[7]));
}
template <>
__device__ __forceinline__ void crt_inc_chain<5>(const uint32_t (&x)[5], uint32_t c, uint32_t (&m)[5]) {
  asm("{\n\t"
      "add.cc.u32 %0, %5, %10;\n\t"
      "addc.cc.u32 %1, %6, 0;\n\t"
      "addc.cc.u32 %2, %7, 0;\n\t"
      "addc.cc.u32 %3, %8, 0;\n\t"
      "addc.u32 %4, %9, 0;\n\t"
      "}"
      : "=&r"(m[0]), "=&r"(m[1]), "=&r"(m[2]), "=&r"(m[3]), "=&r"(m[4])
      : "r"(x[0]), "r"(x[1]), "r"(x[2]), "r"(x[3]), "r"(x[4]), "r"(c));
}
template <>
__device__ __forceinline__ void crt_inc_chain<6>(const uint32_t (&x)[6], uint32_t c, uint32_t (&m)[6]) {
  asm("{\n\t"
      "add.cc.u32 %0, %6, %12;\n\t"
      "addc.cc.u32 %1, %7, 0;\n\t"
      "addc.cc.u32 %2, %8, 0;\n\t"
      "addc.cc.u32 %3, %9, 0;\n\t"
      "addc.cc.u32 %4, %10, 0;\n\t"
      "addc.u32 %5, %11, 0;\n\t"
      "}"
      : "=&r"(m[0]), "=&r"(m[1]), "=&r"(m[2]), "=&r"(m[3]), "=&r"(m[4]), "=&r"(m[5])
      : "r"(x[0]), "r"(x[1]), "r"(x[2]), "r"(x[3]), "r"(x[4]), "r"(x[5]), "r"(c));
}
template <>
__device__ __forceinline__ void crt_inc_chain<7>(const uint32_t (&x)[7], uint32_t c, uint32_t (&m)[7]) {
  asm("{\n\t"
      "add.cc.u32 %0, %7, %14;\n\t"
      "addc.cc.u32 %1, %8, 0;\n\t"
      "addc.cc.u32 %2, %9, 0;\n\t"
      "addc.cc.u32 %3, %10, 0;\n\t"
      "addc.cc.u32 %4, %11, 0;\n\t"
      "addc.cc.u32 %5, %12, 0;\n\t"
      "addc.u32 %6, %13, 0;\n\t"
      "}"
      : "=&r"(m[0]), "=&r"(m[1]), "=&r"(m[2]), "=&r"(m[3]), "=&r"(m[4]), "=&r"(m[5]), "=&r"(m[6])
      : "r"(x[0]), "r"(x[1]), "r"(x[2]), "r"(x[3]), "r"(x[4]), "r"(x[5]), "r"(x[6]), "r"(c));
}
template <>
__device__ __forceinline__ void crt_inc_chain<8>(const uint32_t (&x)[8], uint32_t c, uint32_t (&m)[8]) {
  asm("{\n\t"
      "add.cc.u32 %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, 0;\n\t"
      "addc.cc.u32 %2, %10, 0;\n\t"
      "addc.cc.u32 %3, %11, 0;\n\t"
      "addc.cc.u32 %4, %12, 0;\n\t"
      "addc.cc.u32 %5, %13, 0;\n\t"
      "addc.cc.u32 %6, %14, 0;\n\t"
      "addc.u32 %7, %15, 0;\n\t"
      "}"
      : "=&r"(m[0]), "=&r"(m[1]), "=&r"(m[2]), "=&r"(m[3]), "=&r"(m[4]), "=&r"(m[5]), "=&r"(m[6]), "=&r"(m[7])
      : "r"(x[0]), "r"(x[1]), "r"(x[2]), "r"(x[3]), "r"(x[4]), "r"(x[5]), "r"(x[6]), "r"(x[7]), "r"(c));
}

// C' = V - q M modulo 2^(32 NL) from the column sums S of the reconstruction
// product: q = round((S_0 + S_1 2^8 + S_2 2^16) / 2^24) in 32-bit steps (dividing by
// 2^8 first changes no floor; S_b < 2^22), V = sum_w lo_w 2^(32 w) + sum_w
// hi_w 2^(32 w + 16) with the second sum re-cut at limb boundaries (H_w =
// hi_w 2^16 mod 2^32 + floor(hi_(w-1) / 2^16): disjoint bits), and -q M added
// as q Mn, Mn = -M mod 2^(32 NL).  nbe < 4 NL only when NL = 5: the limbs
// above nbe bytes are then filled with the sign (bit 8 nbe - 1).
template <int NL>
__device__ __forceinline__ void crt_limbs_nl(const uint32_t (&S)[48], const uint32_t (&Mn)[NL], int nbe,
                                             uint32_t (&r)[NL]) {
  const uint32_t q = ((((S[0] + (1u << 23)) >> 8) + S[1] + (S[2] << 8)) >> 16);
  uint32_t lo[NL], hi[NL], H[NL];
#pragma unroll
  for (int w = 0; w < NL; ++w) {
    lo[w] = S[4 + 4 * w] + (S[5 + 4 * w] << 8);  // < 2^30
    hi[w] = S[6 + 4 * w] + (S[7 + 4 * w] << 8);  // < 2^30
  }
  H[0] = hi[0] << 16;
#pragma unroll
  for (int w = 1; w < NL; ++w) H[w] = __funnelshift_l(hi[w - 1], hi[w], 16);
  crt_limb_chain<NL>(lo, H, q, Mn, r);
  if (NL == 5 && nbe < 20) {
    uint32_t top = 0;
#pragma unroll
    for (int w = 0; w < NL; ++w) top = 4 * (w + 1) == nbe ? r[w] : top;
    const uint32_t fill = (uint32_t)((int32_t)top >> 31);
#pragma unroll
    for (int w = 0; w < NL; ++w) r[w] = 4 * w < nbe ? r[w] : fill;
  }
}
// The signed NL-limb integer (two's complement) as a double-double scaled by
// 2^e:
//   the magnitude is normalised (whole-limb shifts, then a funnel shift) so
//   that its leading one is bit 159 of a 160-bit window n4..n0 (bit 0 of
//   weight 2^E; bits below the window dropped);
//   hi = the window rounded to 53 bits (nearest, ties to even, the bits below
//   bit 107 of the window deciding), exact as a double: keep 2^(E + 107);
//   lo = the rest D 2^96 + n2 2^64 + n1 2^32 + n0 (D = the low 11 bits of the
//   top 64 minus 2048 when rounded up) summed in doubles in that order,
//   times 2^E; then fast_two_sum(hi, lo) in units of 2^(E + 107).
// Returns (h, l) with value (h + l) 2^e, e = E + 107.
template <int NL>
__device__ __forceinline__ void crt_to_dd_nl(const uint32_t (&limb)[NL], double &h, double &l, int &e) {
  const uint32_t mask = (uint32_t)((int32_t)limb[NL - 1] >> 31);
  uint32_t x[NL], m[NL];
#pragma unroll
  for (int q = 0; q < NL; ++q) x[q] = limb[q] ^ mask;
  crt_inc_chain<NL>(x, mask & 1u, m);  // the magnitude: two's complement negation when negative
  int E = 32 * (NL - 5);                // weight of window bit 0 before any shift
#pragma unroll
  for (int step = 4; step >= 1; step >>= 1) {
    bool zero = true;
#pragma unroll
    for (int q = NL - step; q < NL; ++q) zero = zero && m[q] == 0;
    if (zero) {
#pragma unroll
      for (int q = NL - 1; q >= 0; --q) m[q] = q >= step ? m[q - step] : 0u;
      E -= 32 * step;
    }
  }
  if (m[NL - 1] == 0) {
    h = l = 0.0;
    e = 0;
    return;
  }
  const int s = __clz((int)m[NL - 1]);
  uint32_t n[5];
#pragma unroll
  for (int w = 0; w < 5; ++w) n[w] = __funnelshift_l(NL - 6 + w >= 0 ? m[NL - 6 + w] : 0u, m[NL - 5 + w], s);
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
  if (mask) {
    h = -h;
    l = -l;
  }
  e = E + 107;
}
// Writes the two's complement integer C' held in NL limbs, times 2^shift, as
// a DD to dst (NaN when `nan`); mode 0 stores it, 1 subtracts it from the DD
// at dst, 2 adds it.
template <int NL>
__device__ __forceinline__ void crt_emit_nl(const uint32_t (&limb)[NL], bool nan, int shift,
                                            double *__restrict__ dst, int mode) {
  double2 out;
  if (nan) {
    out = make_double2(CUDART_NAN, 0.0);
  } else {
    double hi, lo;
    int e;
    crt_to_dd_nl<NL>(limb, hi, lo, e);
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

template <int NL>
__device__ __forceinline__ void crt_out_nl(const uint32_t (&S)[48], const uint32_t (&Mn8)[CRT_NL], int nbe,
                                           bool nan, int shift, double *__restrict__ dst, int mode) {
  uint32_t limb[NL];
  crt_limbs_nl<NL>(S, *reinterpret_cast<const uint32_t(*)[NL]>(&Mn8[0]), nbe, limb);
  crt_emit_nl<NL>(limb, nan, shift, dst, mode);
}

// ---- reconstruction fed by TMA ---------------------------------------------------
// Work unit: 32 rows x one column quad = 128 outputs, the M dimension of one
// reconstruction MMA, M index 4 r + c <-> row i0 + r, column 4 qd + c.  In
// the residue scratch the 128 bytes of (modulus t, unit) are contiguous (rows
// i0 .. i0 + 31, four columns per row), so one TMA box of 128 bytes x 32 ktn
// moduli lands in shared memory as an MN-major operand with the 128-byte
// swizzle -- 8 moduli x 128 bytes per 1024-byte atom, atoms consecutive along
// K -- and no thread touches the residues.  The TMEM lane of an output is its
// M index, so a thread's output is row i0 + 8 (lane quadrant) + lane / 4,
// column 4 qd + lane % 4.
//
// Persistent CTA per SM: warp 0 loads (a ring of CR_RING_BYTES of boxes, one
// stage per group of CR_SETS consecutive units of the CTA), warp 1 issues one
// MMA per 32 moduli per unit into the TMEM slots (nb columns each) of one
// slot group, with one commit per group, and CR_EPI_WARPS / 4 sets of four
// epilogue warps (one per lane quadrant) take the units in turn -- set e
// unit e of every group: each copies its slot to registers, hands the group
// back (every epilogue warp arrives), and forms and stores the 128 outputs.  Planes of moduli
// t >= N (up to the allocated count, and zero-filled beyond it) meet zero
// rows of E.  K chunks (nkc > 1) are folded into chunk 0 beforehand
// (crt_fold_kernel).  All waits are bounded.
// Walks units u0, u0 + step, ... as (row block rb, quad offset qd), u = qd
// nrb + rb, without a division in the loop.
struct UnitCursor {
  int64_t u, rb, qd, step, drb, dqd, nrb;
  __device__ __forceinline__ UnitCursor(int64_t u0, int64_t step_, int64_t nrb_)
      : u(u0), rb(u0 % nrb_), qd(u0 / nrb_), step(step_), drb(step_ % nrb_), dqd(step_ / nrb_), nrb(nrb_) {}
  __device__ __forceinline__ void advance() {
    u += step;
    rb += drb;
    qd += dqd;
    if (rb >= nrb) {
      rb -= nrb;
      ++qd;
    }
  }
};
constexpr int CR_EPI_WARPS = 16;
constexpr int CR_SETS = CR_EPI_WARPS / 4;
constexpr int CR_THREADS = 64 + 32 * CR_EPI_WARPS;
constexpr int CR_RING_BYTES = 128 * 1024;
constexpr int CR_STAGES_MAX = 32;  // CR_RING_BYTES / CR_BOX_BYTES
constexpr int CR_TMEM_COLS = 512;
constexpr int CR_BOX_BYTES = 4096;  // 128 bytes x 32 moduli
__host__ __device__ constexpr int cr_slot_cols(int nb) { return nb <= 32 ? 32 : 64; }
__host__ __device__ constexpr int cr_smem(int ktn) {
  return CR_RING_BYTES + CTC_B_BYTES + 1024 + 1024;  // ring, E, barriers, alignment
}

// The epilogue warps of crt_recon_body: set e (four warps, one per TMEM
// lane quadrant) takes units e, e + CR_SETS, ... of the CTA; per unit it
// copies its slot to registers, hands the slot back, and forms and stores its
// 128 outputs with NL-limb arithmetic.
struct RecEpi {
  const CrtConst *cc;
  const int *sigA, *flagA, *sigB, *flagB;
  int64_t M, N, qbase, nrb, units;
  double *C;
  int64_t cstride;
  int mode, W, nbe, nb, slot_cols, nslots;
  uint32_t tmem;
  uint64_t *tfull, *tempty;
  volatile int *abort_flag;
  int *status;
  uint64_t wait_ns;
};
template <int NL>
__device__ __forceinline__ void crt_recon_epilogue(const RecEpi &p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = warp & 3, set = (warp - 2) >> 2;
  const int mrow = quad * 32 + lane;  // M index = TMEM lane
  uint32_t Mn[NL];                    // -M mod 2^(32 NL)
  {
    uint64_t carry = 1;
#pragma unroll
    for (int w = 0; w < NL; ++w) {
      const uint64_t v = (uint64_t)(~p.cc->Mw[w]) + carry;
      Mn[w] = (uint32_t)v;
      carry = v >> 32;
    }
  }
  int slot = set;  // nslots is a multiple of CR_SETS
  uint32_t tph = 0;
  for (UnitCursor c(blockIdx.x + (int64_t)set * gridDim.x, (int64_t)CR_SETS * gridDim.x, p.nrb); c.u < p.units;
       c.advance()) {
    const int64_t i = c.rb * 32 + (mrow >> 2), j = 4 * (p.qbase + c.qd) + (mrow & 3);
    const bool live = i < p.M && j < p.N;
    int shift = 0, bad = 0;
    if (live) {  // loaded before the wait, in flight meanwhile
      shift = p.sigA[i] + p.sigB[j] - 2 * p.W;
      bad = p.flagA[i] | p.flagB[j];
    }
    const bool got = wait_bar(&p.tfull[slot / CR_SETS], tph, p.abort_flag, p.wait_ns);
    if (!__all_sync(0xffffffffu, got)) {
      if (lane == 0) {
        *p.abort_flag = 1;
        record_abort(p.status, 2);
      }
      break;
    }
    mftc::tc_fence_after();
    uint32_t S[48];
#pragma unroll
    for (int b = 32; b < 48; ++b) S[b] = 0;
    const uint32_t taddr = p.tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(slot * p.slot_cols);
    mftc::tmem_ld_32x32b_x32(taddr, *reinterpret_cast<uint32_t(*)[32]>(S));
    if (NL == 8) mftc::tmem_ld_32x32b_x16(taddr + 32u, *reinterpret_cast<uint32_t(*)[16]>(S + 32));
    mftc::tmem_wait_ld();
    mftc::tc_fence_before();
    __syncwarp();
    if (lane == 0) mftc::mbar_arrive(&p.tempty[slot / CR_SETS]);  // the slot is in registers: hand it back
    slot += CR_SETS;
    if (slot >= p.nslots) {
      slot -= p.nslots;
      tph ^= 1;
    }
    if (live) {
      uint32_t limb[NL];
      crt_limbs_nl<NL>(S, Mn, p.nbe, limb);
      crt_emit_nl<NL>(limb, bad != 0, shift, p.C + 2 * (j * p.M + i) * p.cstride, p.mode);
    }
  }
}

__device__ __forceinline__ void crt_recon_body(const CUtensorMap *tmD, const Plan *plan, const CrtConst *cc,
                                               const int *sigA, const int *flagA, const int *sigB,
                                               const int *flagB, int64_t M, int64_t N, int64_t qbase,
                                               int64_t nrb, int64_t units, int64_t k, double *__restrict__ C,
                                               int64_t cstride, int mode, uint8_t *smem, int *status,
                                               uint64_t wait_ns) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = plan->S, W = plan->W;
  const int ktn = (n + 31) / 32;
  const int nbe = crt_tc_bytes(W, k), nb = crt_tc_cols(nbe);
  const int slot_cols = cr_slot_cols(nb), nslots = CR_TMEM_COLS / slot_cols;
  const int box_bytes = CR_BOX_BYTES * ktn;
  // one stage and one TMEM slot group per CR_SETS consecutive units of the
  // CTA (one unit per epilogue set): a barrier round trip and a commit serve
  // CR_SETS units
  const int stage_bytes = CR_SETS * box_bytes;
  const int nsg = nslots / CR_SETS;  // slot groups
  uint8_t *ring = smem;
  const int nst = CR_RING_BYTES / stage_bytes;  // stages of the ring
  uint8_t *sB = smem + CR_RING_BYTES;
  uint64_t *full = reinterpret_cast<uint64_t *>(sB + CTC_B_BYTES);
  uint64_t *empty = full + CR_STAGES_MAX;
  uint64_t *tfull = empty + CR_STAGES_MAX;  // per slot group (4 at most)
  uint64_t *tempty = tfull + 16;
  uint64_t *drain = tempty + 16;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tslot + 1);

  if (threadIdx.x == 0) {
    for (int s = 0; s < nst; ++s) {
      mftc::mbar_init(&full[s], 1);
      mftc::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 16; ++a) {
      mftc::mbar_init(&tfull[a], 1);
      mftc::mbar_init(&tempty[a], 4 * CR_SETS);  // every epilogue warp
    }
    mftc::mbar_init(drain, 1);
    *abort_flag = 0;
    mftc::fence_mbar_init();
  }
  if (warp == 0 && lane == 0) mftc::prefetch_tmap(tmD);
  if (warp == 1) {
    mftc::tmem_alloc(tslot, CR_TMEM_COLS);
    mftc::tmem_relinquish();
  }
  // the E tile (the B operand, K-major): row b holds E[t][b] at byte t
  {
    const int T = (int)threadIdx.x - 64;
    if (T >= 0 && T < CRT_EB_ROWS)
      for (int kt = 0; kt < ktn; ++kt)
        for (int h = 0; h < 2; ++h)
          sw128_store16(sB, T, 2 * kt + h, *reinterpret_cast<const uint4 *>(&cc->eb[T][32 * kt + 16 * h]));
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mftc::tc_fence_before();
  __syncthreads();
  mftc::tc_fence_after();
  const uint32_t tmem = *tslot;
  auto fail = [&](int code) {
    *abort_flag = 1;
    record_abort(status, code);
  };
  ArmedStages<CR_STAGES_MAX> arm;
  arm.clear();

  if (warp == 0) {
    if (lane == 0) {  // ---- TMA producer: a stage per group of CR_SETS units ----
      int stage = 0;
      uint32_t ph = 0;
      for (UnitCursor c(blockIdx.x, gridDim.x, nrb); c.u < units;) {
        if (!wait_bar(&empty[stage], ph ^ 1, abort_flag, wait_ns)) {
          fail(2);
          break;
        }
        const int64_t rem = (units - c.u + gridDim.x - 1) / gridDim.x;  // units of this CTA left
        const int ne = rem < CR_SETS ? (int)rem : CR_SETS;
        mftc::mbar_arrive_expect_tx(&full[stage], (uint32_t)(ne * box_bytes));
        for (int e = 0; e < ne; ++e, c.advance())
          for (int kt = 0; kt < ktn; ++kt)  // boxes of 32 moduli
            mftc::tma_load_3d(ring + stage * stage_bytes + e * box_bytes + kt * CR_BOX_BYTES, tmD, &full[stage],
                              (int32_t)(c.rb * 128), (int32_t)(qbase + c.qd), 32 * kt);
        arm.arm(stage, ph);
        if (++stage == nst) {
          stage = 0;
          ph ^= 1;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---- MMA issuer: CR_SETS units per stage, one commit each ----
      const uint32_t idesc = mftc::idesc_u8(128, nb) | mftc::IDESC_A_MN;  // A (residues) MN-major
      const uint64_t bdesc = mftc::smem_desc_k_sw128(mftc::smem_u32(sB));
      int stage = 0, sg = 0;
      uint32_t ph = 0, tph = 0;
      for (int64_t o = blockIdx.x; o < units; o += (int64_t)CR_SETS * gridDim.x) {
        const int64_t rem = (units - o + gridDim.x - 1) / gridDim.x;
        const int ne = rem < CR_SETS ? (int)rem : CR_SETS;
        if (!wait_bar(&full[stage], ph, abort_flag, wait_ns) ||
            !wait_bar(&tempty[sg], tph ^ 1, abort_flag, wait_ns)) {
          fail(2);
          break;
        }
        mftc::tc_fence_after();
        for (int e = 0; e < ne; ++e) {
          const uint64_t adesc = mftc::smem_desc_k_sw128(mftc::smem_u32(ring + stage * stage_bytes + e * box_bytes));
          const uint32_t dst = tmem + (uint32_t)((sg * CR_SETS + e) * slot_cols);
          for (int kt = 0; kt < ktn; ++kt)  // start-address steps: 4096 and 32 bytes per 32 moduli
            mftc::umma_i8(dst, adesc + (uint64_t)(kt * (CR_BOX_BYTES / 16)), bdesc + (uint64_t)(kt * 2), idesc,
                          kt > 0 ? 1u : 0u);
        }
        mftc::umma_commit(&empty[stage]);
        mftc::umma_commit(&tfull[sg]);
        if (++stage == nst) {
          stage = 0;
          ph ^= 1;
        }
        if (++sg == nsg) {
          sg = 0;
          tph ^= 1;
        }
      }
      // every MMA issued by this thread has finished once `drain` flips
      mftc::umma_commit(drain);
      (void)wait_bar_ns(drain, 0, WAIT_NS);
    }
  } else {  // ---- epilogue ----
    const int nl = nbe / 4;
    const RecEpi ep{cc, sigA, flagA, sigB, flagB, M, N, qbase, nrb, units, C, cstride, mode, W, nbe, nb, slot_cols,
                    nslots, tmem, tfull, tempty, abort_flag, status, wait_ns};
    if (nl <= 5)
      crt_recon_epilogue<5>(ep);
    else if (nl == 6)
      crt_recon_epilogue<6>(ep);
    else if (nl == 7)
      crt_recon_epilogue<7>(ep);
    else
      crt_recon_epilogue<8>(ep);
  }

  mftc::tc_fence_before();
  __syncthreads();
  mftc::tc_fence_after();
  if (*abort_flag) {  // read after the barrier: the same value in every thread
    // copies in flight that no MMA consumed land before shared memory is released
    if (warp == 0 && lane == 0) arm.drain(full, nst);
    __syncthreads();
  }
  if (warp == 1) mftc::tmem_dealloc(tmem, CR_TMEM_COLS);
}

// Folds the K chunks of the residue products into chunk 0: per modulus t <
// N and word, the chunks' residues summed and reduced modulo m_t.
__device__ __forceinline__ void crt_fold_body(uint32_t *D, const Plan *plan, int nkc, int64_t plane_words,
                                              int t, int64_t w) {
  if (t >= plan->S || w >= plane_words) return;
  uint32_t *src = D + (int64_t)t * nkc * plane_words + w;
  *src = crt_chunk_residue_word(src, nkc, plane_words, t);
}

}  // namespace split
}  // namespace mfcuda
