// Device pieces shared by the single-problem and grouped split-INT8 GEMM
// kernels: tile constants, the per-call plan, bounded mbarrier waits, and the
// exact rounding of a DD entry to balanced signed 8-bit digits.
#pragma once
#include <cstdint>

#include "dd_device.cuh"
#include "grid_round.cuh"
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
// Bounded waits.  WAIT_NS (2 s) is the default limit of every wait in the
// tensor-core kernels; a smaller limit can be set from the host
// (mfcuda_set_wait_limit_ns) and reaches the kernels as an argument.  The
// waits of an abort path (copies in flight landing, issued MMAs draining) keep
// WAIT_NS whatever that setting, so a kernel that gave up still lets its own
// asynchronous work finish before it frees tensor memory and exits.
constexpr uint64_t WAIT_NS = 2000000000ull;

// S: slices per operand (CRT form: moduli), G = S - 1, W: bits of the fixed-point
// operands; crt = 1 selects the CRT form (one product per item, slice t of A
// with slice t of B); nl: 32-bit limbs of its reconstruction.
struct Plan {
  int S, G, W;
  int rho_a, rho_b;
  int crt, nl, pad;
};

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait (limit_ns) that also gives up as soon as another role of the
// CTA aborted.
__device__ __forceinline__ bool wait_bar(uint64_t *bar, uint32_t parity, volatile int *abort_flag,
                                         uint64_t limit_ns) {
  if (mftc::mbar_try_wait(bar, parity)) return true;
  uint64_t t0 = globaltimer();
  while (true) {
    if (mftc::mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
    if (globaltimer() - t0 > limit_ns) return false;
  }
}
// Bounded wait without an abort flag, backing off after the first polls.
__device__ __forceinline__ bool wait_bar_ns(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
  if (mftc::mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer();
  for (int i = 0;; ++i) {
    if (mftc::mbar_try_wait(bar, parity)) return true;
    if (globaltimer() - t0 > limit_ns) return false;
    if (i > 64) __nanosleep(64);
  }
}
// The TMA producer's record of the stages it armed (the parity of each
// stage's last arming).  After an abort, copies may be in flight that no MMA
// consumed; drain() waits (default limit) for each armed stage's last phase,
// so they land before the CTA frees its shared memory.
template <int NS>
struct ArmedStages {
  bool armed[NS];
  uint32_t parity[NS];
  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int s = 0; s < NS; ++s) armed[s] = false;
  }
  __device__ __forceinline__ void arm(int s, uint32_t p) {
    armed[s] = true;
    parity[s] = p;
  }
  __device__ __forceinline__ void drain(uint64_t *full, int nst) {
    for (int s = 0; s < nst && s < NS; ++s)
      if (armed[s]) (void)wait_bar_ns(&full[s], parity[s], WAIT_NS);
  }
};
// Spins for ns nanoseconds (abort paths only).
__device__ __forceinline__ void settle_ns(uint64_t ns) {
  const uint64_t t0 = globaltimer();
  while (globaltimer() - t0 < ns) __nanosleep(256);
}

// Per-device record of given-up waits, for callers that did not ask a call
// for its status: every kernel that gives up a wait ORs its code here as well
// as into the call's status word; mfcuda_timeout_status reads and clears it.
// (One copy per translation unit; the host reads every copy.)
static __device__ int g_wait_sticky;
__device__ __forceinline__ void record_abort(int *status, int code) {
  atomicOr(status, code);
  atomicOr(&g_wait_sticky, code);
}
// This translation unit's record on the current device (-1 if the query
// fails), zeroed afterwards when `clear` (synchronous copies).
static inline int take_wait_sticky(bool clear) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_wait_sticky, sizeof(int)) != cudaSuccess) {
    (void)cudaGetLastError();
    return -1;
  }
  if (clear && v) {
    const int z = 0;
    if (cudaMemcpyToSymbol(g_wait_sticky, &z, sizeof(int)) != cudaSuccess) {
      (void)cudaGetLastError();
      return -1;
    }
  }
  return v;
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

// floor(log2 v) for a finite v > 0, read from the IEEE-754 fields (subnormals
// from the position of the leading fraction bit).
__device__ __forceinline__ int floor_log2(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  const int E = (int)((b >> 52) & 0x7FF);
  if (E) return E - 1023;
  return (63 - __clzll((long long)(b & ((1ull << 52) - 1)))) - 1074;
}
// binade of |hi| + |lo|: v < 2^e (frexp convention); 0 for v == 0 (unused)
__device__ __forceinline__ int binade_above(double v) { return floor_log2(v) + 1; }
__device__ __forceinline__ int binade_below(double v) { return floor_log2(v); }

// Exact power of two 2^e for -1022 <= e <= 1023.
__device__ __forceinline__ double pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }
// x 2^e, correctly rounded like ldexp: a multiplication by an exact power of
// two when 2^e is a normal double, ldexp otherwise.
__device__ __forceinline__ double scale2(double x, int e) {
  return (e >= -1022 && e <= 1023) ? x * pow2(e) : ldexp(x, e);
}

// The entry rounded to the fixed-point grid of its row / column
// (grid_round.cuh: X = rint(H) + rint((H - rint(H)) + L), H = hi 2^(W - sigma),
// L = lo 2^(W - sigma), clamped to |X| <= 2^W - 1; W <= 110), returned as the
// four 32-bit words of Y = X + sum_{q<14} 128 * 256^q: byte q of Y is
// balanced digit q of X plus 128.  Slice s of the S-slice representation
// (most significant first) is digit q = S-1-s; digits q >= S are zero.
// Word w of the bias (X = 0 gives all digits zero).
__host__ __device__ constexpr uint32_t bias_word(int w) { return w < 3 ? 0x80808080u : 0x00008080u; }
__device__ __forceinline__ void biased_bytes(double hi, double lo, int sigma, int W, uint32_t (&y)[4]) {
  const GridLimits g = grid_limits(W);
  int64_t T;
  uint64_t R;
  grid_round(hi, lo, sigma, g, W, T, R);
  grid_biased_words(T, R, y);
}
// Byte k of each of a, b, c, d packed as bytes 0..3.
__device__ __forceinline__ uint32_t gather_byte(uint32_t a, uint32_t b, uint32_t c, uint32_t d, int k) {
  const uint32_t sel = (uint32_t)k | ((uint32_t)(k + 4) << 4);
  return __byte_perm(__byte_perm(a, b, sel), __byte_perm(c, d, sel), 0x5410);
}
// Digit q (signed bytes) of 8 entries packed in entry order into one word.
template <int Q>
__device__ __forceinline__ uint64_t digit_word(const uint32_t (&y)[8][4]) {
  constexpr int w = Q >> 2, k = Q & 3;
  const uint32_t lo = gather_byte(y[0][w], y[1][w], y[2][w], y[3][w], k) ^ 0x80808080u;
  const uint32_t hi = gather_byte(y[4][w], y[5][w], y[6][w], y[7][w], k) ^ 0x80808080u;
  return (uint64_t)lo | ((uint64_t)hi << 32);
}
// Calls f(slice index, word) for the S slices of 8 entries.
template <class F>
__device__ __forceinline__ void for_each_slice_word(const uint32_t (&y)[8][4], int S, F f) {
#define MF_SLICE_Q(Q) \
  if (Q < S) f(S - 1 - Q, digit_word<Q>(y));
  MF_SLICE_Q(0) MF_SLICE_Q(1) MF_SLICE_Q(2) MF_SLICE_Q(3) MF_SLICE_Q(4) MF_SLICE_Q(5) MF_SLICE_Q(6)
  MF_SLICE_Q(7) MF_SLICE_Q(8) MF_SLICE_Q(9) MF_SLICE_Q(10) MF_SLICE_Q(11) MF_SLICE_Q(12) MF_SLICE_Q(13)
#undef MF_SLICE_Q
}
static_assert(SMAX == 14, "for_each_slice_word unrolls 14 digit positions");

// Operands are read through strided views: DD element e of a view lives at
// double2 index e * stride from its base (stride 1 for a real matrix, 2 for the
// real or imaginary part of a complex one).
//
// A column-major m x k: thread per row, a chunk of columns per blockIdx.y.
__device__ __forceinline__ void scan_a_body(const double *__restrict__ A, int64_t M,
                                                     int64_t K, int64_t stride, int kchunk, int *sig,
                                                     int *mu, int *flag, int64_t bx, int64_t by) {
  int64_t i = bx * blockDim.x + threadIdx.x;
  if (i >= M) return;
  int64_t p0 = by * kchunk, p1 = p0 + kchunk < K ? p0 + kchunk : K;
  int hi_e = SENT_LO, lo_e = SENT_HI, bad = 0;
  for (int64_t p = p0; p < p1; ++p) {
    double2 v = __ldg(reinterpret_cast<const double2 *>(A) + (p * M + i) * stride);
    if (!isfinite(v.x) || !isfinite(v.y)) {
      bad = 1;
      continue;
    }
    double a = fabs(v.x) + fabs(v.y);
    if (a != 0.0) {
      hi_e = max(hi_e, binade_above(a));
      lo_e = min(lo_e, binade_below(a));
    }
  }
  if (hi_e != SENT_LO) atomicMax(&sig[i], hi_e);
  if (lo_e != SENT_HI) atomicMin(&mu[i], lo_e);
  if (bad) atomicOr(&flag[i], 1);
}

// B column-major k x n: a block per (column j, chunk of 2048 rows).
__device__ __forceinline__ void scan_b_body(const double *__restrict__ B, int64_t K,
                                                     int64_t N, int64_t stride, int *sig, int *mu,
                                                     int *flag, int64_t bx, int64_t by) {
  int64_t j = by;
  int64_t p0 = bx * 2048;
  int hi_e = SENT_LO, lo_e = SENT_HI, bad = 0;
  for (int r = 0; r < 8; ++r) {
    int64_t p = p0 + threadIdx.x + 256 * r;
    if (p >= K) break;
    double2 v = __ldg(reinterpret_cast<const double2 *>(B) + (j * K + p) * stride);
    if (!isfinite(v.x) || !isfinite(v.y)) {
      bad = 1;
      continue;
    }
    double a = fabs(v.x) + fabs(v.y);
    if (a != 0.0) {
      hi_e = max(hi_e, binade_above(a));
      lo_e = min(lo_e, binade_below(a));
    }
  }
  for (int off = 16; off >= 1; off >>= 1) {
    hi_e = max(hi_e, __shfl_xor_sync(0xffffffffu, hi_e, off));
    lo_e = min(lo_e, __shfl_xor_sync(0xffffffffu, lo_e, off));
    bad |= __shfl_xor_sync(0xffffffffu, bad, off);
  }
  if ((threadIdx.x & 31) == 0) {
    if (hi_e != SENT_LO) atomicMax(&sig[j], hi_e);
    if (lo_e != SENT_HI) atomicMin(&mu[j], lo_e);
    if (bad) atomicOr(&flag[j], 1);
  }
}

// Exponent statistics of the operands of one call: A-side operands (rows of
// an m x k matrix) and B-side operands (columns of a k x n matrix).
struct StatSet {
  int *sig[4];
  const int *mu[4];
  int64_t count[4];
  int side[4];  // 0: A side, 1: B side
  int n;
};

__device__ __forceinline__ void plan_body(const StatSet &st, int slices, double target, Plan *plan) {
  __shared__ int red[2][32];
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
    int S = slices;
    if (S <= 0) {
      // smallest S with (S+1) 2^(106 - 8S + rho_a + rho_b) <= target
      S = SMAX;
      for (int q = 2; q <= SMAX; ++q) {
        double ratio = (q + 1) * ldexp(1.0, 106 - 8 * q + ra + rb);
        if (ratio <= target) {
          S = q;
          break;
        }
      }
    }
    plan->S = S;
    plan->G = S - 1;
    plan->W = 8 * S - 2;
    plan->rho_a = ra;
    plan->rho_b = rb;
    plan->crt = 0;
    plan->nl = 0;
  }
  // zero rows / columns: any sigma works, the digits are all zero
  __syncthreads();
  for (int o = 0; o < st.n; ++o)
    for (int64_t i = threadIdx.x; i < st.count[o]; i += blockDim.x)
      if (st.sig[o][i] == SENT_LO) st.sig[o][i] = 0;
}

// A (m x k column-major) -> As[s][i][p]: a block covers 32 rows x 64
// columns; thread (i = t % 32, group = t / 32) rounds and slices the 8
// consecutive entries A[i, p0 + 8 group .. + 7] (coalesced across i), packs
// the 8 digits of each slice into one 64-bit word, and the tile is transposed
// through shared memory (row stride padded to 72 bytes: conflict-free) so
// that every slice row is written as contiguous 8-byte words.
constexpr int SA_ROWS = 32, SA_COLS = 64, SA_STRIDE = 72;
__device__ __forceinline__ void slice_a_body(const double *__restrict__ A, int64_t M,
                                                      int64_t K, int64_t stride, int64_t M_pad,
                                                      int64_t K_pad, const int *sig, const int *flag,
                                                      const Plan *plan, int8_t *__restrict__ As, int64_t bx, int64_t by) {
  __shared__ __align__(16) uint8_t tile[SMAX][SA_ROWS * SA_STRIDE];
  const int S = plan->S, W = plan->W;
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
      for (int w = 0; w < 4; ++w) y[e][w] = bias_word(w);  // X = 0: all digits zero
    }
  }
  for_each_slice_word(y, S, [&](int sl, uint64_t word) {
    *reinterpret_cast<uint64_t *>(&tile[sl][ii * SA_STRIDE + grp * 8]) = word;
  });
  __syncthreads();
  const int row = t / 8, seg = (t % 8) * 8;
  for (int s = 0; s < S; ++s) {
    uint64_t v = *reinterpret_cast<const uint64_t *>(&tile[s][row * SA_STRIDE + seg]);
    *reinterpret_cast<uint64_t *>(As + ((s * M_pad + i0 + row) * K_pad + p0 + seg)) = v;
  }
}

// B (k x n column-major) -> Bs[s][j][p]: each thread rounds and slices 8
// consecutive entries of one column (128 contiguous bytes in, one 8-byte word
// per slice out).
// Entries p8 .. p8+7 of column j (0 <= j < N_pad, p8 a multiple of 8 below K_pad).
__device__ __forceinline__ void slice_b_one(const double *__restrict__ B, int64_t K, int64_t N,
                                            int64_t stride, int64_t N_pad, int64_t K_pad, const int *sig,
                                            const int *flag, const Plan *plan, int8_t *__restrict__ Bs,
                                            int64_t j, int64_t p8) {
  const int S = plan->S, W = plan->W;
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
  for_each_slice_word(y, S, [&](int sl, uint64_t word) {
    *reinterpret_cast<uint64_t *>(Bs + (((int64_t)sl * N_pad + j) * K_pad + p8)) = word;
  });
}
// A block per (column by, range of K): thread t of block bx takes entries
// (bx * blockDim.x + t) * 8 .. + 7.
__device__ __forceinline__ void slice_b_body(const double *__restrict__ B, int64_t K,
                                             int64_t N, int64_t stride, int64_t N_pad,
                                             int64_t K_pad, const int *sig, const int *flag,
                                             const Plan *plan, int8_t *__restrict__ Bs, int64_t bx, int64_t by) {
  const int64_t p8 = (bx * blockDim.x + threadIdx.x) * 8;
  if (p8 >= K_pad) return;
  slice_b_one(B, K, N, stride, N_pad, K_pad, sig, flag, plan, Bs, by, p8);
}

// Column j of B (k x n column-major view) scanned by one warp: lane l reads
// entries l, l+32, ...; the warp's max / min / or is written by lane 0 (no
// other warp touches column j).
__device__ __forceinline__ void scan_b_warp(const double *__restrict__ B, int64_t K, int64_t stride, int *sig,
                                            int *mu, int *flag, int64_t j) {
  const int lane = threadIdx.x & 31;
  int hi_e = SENT_LO, lo_e = SENT_HI, bad = 0;
  for (int64_t p = lane; p < K; p += 32) {
    double2 v = __ldg(reinterpret_cast<const double2 *>(B) + (j * K + p) * stride);
    if (!isfinite(v.x) || !isfinite(v.y)) {
      bad = 1;
      continue;
    }
    double a = fabs(v.x) + fabs(v.y);
    if (a != 0.0) {
      hi_e = max(hi_e, binade_above(a));
      lo_e = min(lo_e, binade_below(a));
    }
  }
  for (int off = 16; off >= 1; off >>= 1) {
    hi_e = max(hi_e, __shfl_xor_sync(0xffffffffu, hi_e, off));
    lo_e = min(lo_e, __shfl_xor_sync(0xffffffffu, lo_e, off));
    bad |= __shfl_xor_sync(0xffffffffu, bad, off);
  }
  if (lane == 0) {
    sig[j] = hi_e;
    mu[j] = lo_e;
    flag[j] = bad;
  }
}

// Thread per row i (consecutive threads -> consecutive rows: every load and
// store is coalesced); the grid's y dimension strides over the columns.  The
// output is a strided view (C element (i,j) at double2 index (jM + i) cstride)
// and `mode` stores the product P (0), or replaces C by the DD difference
// C - P (1) or sum C + P (2), which assembles complex products.
__device__ __forceinline__ void combine_body(const int32_t *__restrict__ D, const Plan *plan,
                                                      const int *sigA, const int *flagA,
                                                      const int *sigB, const int *flagB, int64_t M,
                                                      int64_t N, int64_t M_pad, int64_t N_pad,
                                                      int nkc, double *__restrict__ C, int64_t cstride,
                                                      int mode, int64_t bx, int64_t by, int64_t ny) {
  const int G = plan->G;
  const int64_t i = bx * blockDim.x + threadIdx.x;
  if (i >= M) return;
  const int64_t gstride = (int64_t)nkc * N_pad * M_pad;  // distance between diagonals
  const int sa = sigA[i], fa = flagA[i];
  // two columns per pass: 2 x (G+1) independent loads in flight per thread
  for (int64_t j0 = by; j0 < N; j0 += 2 * ny) {
    const int64_t jj[2] = {j0, j0 + ny};
    double hi[2] = {0.0, 0.0}, lo[2] = {0.0, 0.0};
    for (int kc = 0; kc < nkc; ++kc) {
      int32_t v[2][SMAX];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int32_t *src = D + ((int64_t)kc * N_pad + (jj[c] < N ? jj[c] : j0)) * M_pad + i;
#pragma unroll
        for (int g = 0; g < SMAX; ++g) v[c][g] = g <= G ? __ldcs(src + g * gstride) : 0;
      }
#pragma unroll
      for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int g = SMAX - 1; g >= 0; --g) {
          if (g <= G) {
            double tv = mfdev::mul((double)v[c][g], pow2(-8 * g));  // exact
            double s_, err;
            mfdev::two_sum(hi[c], tv, s_, err);
            hi[c] = s_;
            lo[c] = mfdev::add(lo[c], err);
          }
        }
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int64_t j = jj[c];
      if (j >= N) break;
      double h, l;
      mfdev::two_sum(hi[c], lo[c], h, l);
      double2 out;
      if (fa | flagB[j]) {
        out = make_double2(CUDART_NAN, 0.0);
      } else {
        int ex = sa + sigB[j] - 12;
        out = make_double2(scale2(h, ex), scale2(l, ex));
      }
      double2 *dst = reinterpret_cast<double2 *>(C) + (j * M + i) * cstride;
      if (mode != 0) {
        double2 prev = *dst;
        mfdev::dd p = mfdev::make(out.x, out.y), q = mfdev::make(prev.x, prev.y);
        mfdev::dd r = mode == 1 ? mfdev::dd_sub(q, p) : mfdev::dd_add(q, p);
        out = make_double2(r.hi, r.lo);
      }
      __stcs(dst, out);
    }
  }
}

// Same result as combine_body, element for element (same operations in the
// same order), with a thread per 4 consecutive rows of one column: each
// diagonal is one 16-byte load per thread (512 contiguous bytes per warp), all
// G+1 of them in flight before the DD accumulation.  Requires M_pad % 4 == 0
// and a 16-byte aligned D.  Thread (q = blockIdx.x * blockDim.x + t) owns rows
// 4q..4q+3 of column j = column index given by the caller.
__device__ __forceinline__ void combine4_body(const int32_t *__restrict__ D, const Plan *plan,
                                              const int *sigA, const int *flagA, const int *sigB,
                                              const int *flagB, int64_t M, int64_t N, int64_t M_pad,
                                              int64_t N_pad, int nkc, double *__restrict__ C, int64_t cstride,
                                              int mode, int64_t quad, int64_t j) {
  const int G = plan->G;
  const int64_t i0 = quad * 4;
  if (i0 >= M || j >= N) return;
  const int64_t gstride = (int64_t)nkc * N_pad * M_pad;  // int32 elements between diagonals
  double hi[4] = {0.0, 0.0, 0.0, 0.0}, lo[4] = {0.0, 0.0, 0.0, 0.0};
  for (int kc = 0; kc < nkc; ++kc) {
    const int4 *src = reinterpret_cast<const int4 *>(D + ((int64_t)kc * N_pad + j) * M_pad + i0);
    const int64_t gs4 = gstride / 4;
    int4 v[SMAX];
#pragma unroll
    for (int g = 0; g < SMAX; ++g) v[g] = g <= G ? __ldcs(src + g * gs4) : make_int4(0, 0, 0, 0);
#pragma unroll
    for (int g = SMAX - 1; g >= 0; --g) {
      if (g <= G) {
        const double sc = pow2(-8 * g);
        const int d[4] = {v[g].x, v[g].y, v[g].z, v[g].w};
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          double tv = mfdev::mul((double)d[r], sc);  // exact
          double s_, err;
          mfdev::two_sum(hi[r], tv, s_, err);
          hi[r] = s_;
          lo[r] = mfdev::add(lo[r], err);
        }
      }
    }
  }
  const int4 sa = *reinterpret_cast<const int4 *>(sigA + i0);
  const int4 fa = *reinterpret_cast<const int4 *>(flagA + i0);
  const int sav[4] = {sa.x, sa.y, sa.z, sa.w}, fav[4] = {fa.x, fa.y, fa.z, fa.w};
  const int sb = sigB[j], fb = flagB[j];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int64_t i = i0 + r;
    if (i >= M) break;
    double h, l;
    mfdev::two_sum(hi[r], lo[r], h, l);
    double2 out;
    if (fav[r] | fb) {
      out = make_double2(CUDART_NAN, 0.0);
    } else {
      int ex = sav[r] + sb - 12;
      out = make_double2(scale2(h, ex), scale2(l, ex));
    }
    double2 *dst = reinterpret_cast<double2 *>(C) + (j * M + i) * cstride;
    if (mode != 0) {
      double2 prev = *dst;
      mfdev::dd p = mfdev::make(out.x, out.y), q = mfdev::make(prev.x, prev.y);
      mfdev::dd res = mode == 1 ? mfdev::dd_sub(q, p) : mfdev::dd_add(q, p);
      out = make_double2(res.hi, res.lo);
    }
    __stcs(dst, out);
  }
}

}  // namespace split
}  // namespace mfcuda
