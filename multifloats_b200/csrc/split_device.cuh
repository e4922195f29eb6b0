// Device pieces shared by the single-problem and grouped split-INT8 GEMM
// kernels: tile constants, the per-call plan, bounded mbarrier waits, and the
// exact rounding of a DD entry to balanced signed 8-bit digits.
#pragma once
#include <cstdint>

#include "tcgen05.cuh"

namespace mfcuda {
namespace split {

constexpr int SMAX = 14;           // most slices per operand
constexpr int BM = 128, BN = 256;  // output tile (UMMA M x N)
constexpr int BK = 128;            // int8 K bytes per pipeline stage (4 UMMAs of K=32)
constexpr int UMMA_K = 32;
constexpr int NSTAGE = 4;
constexpr int A_STAGE = BM * BK;  // 16 KiB
constexpr int B_STAGE = BN * BK;  // 32 KiB
constexpr int STAGE = A_STAGE + B_STAGE;
constexpr int TMEM_COLS = 2 * BN;  // two accumulators
constexpr int MMA_THREADS = 192;   // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int MMA_SMEM = NSTAGE * STAGE + 1024 /*align*/ + 256 /*barriers*/;
// K chunk: (SMAX pairs) * K_chunk * 2^14 < 2^31  ->  73 blocks of 128
constexpr int KC_BLOCKS = (int)(2147483647LL / ((long long)SMAX * 16384LL * BK));
constexpr uint64_t WAIT_NS = 2000000000ull;  // bounded waits: 2 s

struct Plan {
  int S, G, W;
  int rho_a, rho_b;
  int pad[3];
};

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait that also gives up as soon as another role of the CTA aborted.
__device__ __forceinline__ bool wait_bar(uint64_t *bar, uint32_t parity, volatile int *abort_flag) {
  if (mftc::mbar_try_wait(bar, parity)) return true;
  uint64_t t0 = globaltimer();
  while (true) {
    if (mftc::mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
    if (globaltimer() - t0 > WAIT_NS) return false;
  }
}

constexpr int SENT_LO = -100000, SENT_HI = 100000;

static __global__ void init_stats_kernel(int *sig, int *mu, int *flag, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    sig[i] = SENT_LO;
    mu[i] = SENT_HI;
    flag[i] = 0;
  }
}

// binade of |hi| + |lo|: v < 2^e (frexp convention); 0 for v == 0 (unused)
__device__ __forceinline__ int binade_above(double v) { return ilogb(v) + 1; }
__device__ __forceinline__ int binade_below(double v) { return ilogb(v); }

// x * 2^t for the double x = m 2^e as a fixed-point integer with F fractional
// bits (floor for the bits below).
constexpr int FRAC = 16;
__device__ __forceinline__ __int128 scaled_fixed(double x, int t) {
  if (x == 0.0) return 0;
  int e = ilogb(x);
  long long m = (long long)ldexp(x, 52 - e);  // exact: |m| < 2^53
  int sh = e - 52 + t + FRAC;
  if (sh >= 0) return (__int128)m << sh;
  if (sh <= -64) return m < 0 ? (__int128)-1 : (__int128)0;
  return (__int128)(m >> (-sh));
}

// Balanced digits of round((hi + lo) 2^(W - sigma)) in SMAX positions, most
// significant first (fully unrolled, so the digits stay in registers).  Since
// |X| < 2^(8S-2), the top SMAX-S digits are zero and slice s of the S-slice
// representation is d[SMAX - S + s]; the digit left in position SMAX-S lies in
// [-64, 64].
__device__ __forceinline__ void dd_digits(double hi, double lo, int sigma, int W, int8_t (&d)[SMAX]) {
  int t = W - sigma;
  __int128 xf = scaled_fixed(hi, t) + scaled_fixed(lo, t);
  __int128 X = (xf + ((__int128)1 << (FRAC - 1))) >> FRAC;
  const __int128 lim = ((__int128)1 << W) - 1;
  if (X > lim) X = lim;
  if (X < -lim) X = -lim;
  // X = xh 2^56 + xl with 0 <= xl < 2^56: the low seven digits come from xl,
  // the carry (0 or 1) moves into xh, the high seven digits come from xh.
  long long xl = (long long)((unsigned long long)X & ((1ull << 56) - 1));
  long long xh = (long long)(X >> 56);
#pragma unroll
  for (int q = SMAX - 1; q >= SMAX - 7; --q) {
    int v = (int)(xl & 0xFF);
    v = (v ^ 0x80) - 0x80;
    d[q] = (int8_t)v;
    xl = (xl - v) >> 8;
  }
  xh += xl;
#pragma unroll
  for (int q = SMAX - 8; q >= 0; --q) {
    int v = (int)(xh & 0xFF);
    v = (v ^ 0x80) - 0x80;
    d[q] = (int8_t)v;
    xh = (xh - v) >> 8;
  }
}

}  // namespace split
}  // namespace mfcuda
