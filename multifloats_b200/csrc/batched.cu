// Batched ragged work in grouped launches, captured once in a CUDA graph.
//
// A batch plan binds a list of independent problems (device pointers) and
// captures their execution as a CUDA graph that mfcuda_batch_run replays:
//
//  * plain DD GEMMs: ONE persistent grouped kernel.  Its work list holds every
//    output tile of every problem, longest K first; CTAs take items from an
//    atomic counter.  Each item runs the same tile code as the single-problem
//    kernel (gemm_tile.cuh) with the tile shape the autotuner picked for that
//    problem's shape bucket (64x64, 32x32 or 16x16), so every output is
//    bit-identical to matmuldd_mm.
//  * split-INT8 DD GEMMs: each phase of the split pipeline (exponent scan,
//    plan, slicing, tcgen05 MMA, recombination) is one grouped launch over all
//    problems; the tensor-core phase is one persistent kernel whose work list
//    holds every (diagonal, K chunk, tile) item of every problem.  Per problem:
//    slice count from its plan, tile width N (256/128/64) and K chunk from the
//    autotuner.  Results are bit-identical to mfcuda_matmuldd_mm_split.
//  * ragged elementwise arrays: one grid-stride launch over the concatenated
//    index space.
//
// The autotuner times the candidate configurations of each shape bucket on
// synthetic problems of that bucket the first time the bucket is seen and keeps
// the winners in a small text cache (MFCUDA_AUTOTUNE_CACHE, default
// $HOME/.cache/multifloats_b200/autotune.txt).
#include <cudaTypedefs.h>
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "dd_device.cuh"
#include "gemm_tile.cuh"
#include "crt_device.cuh"
#include "split_device.cuh"
#include "tcgen05.cuh"

struct mfcuda_batch;

namespace mfcuda {
int unary_dev(int op, const float64x2 *x, float64x2 *y, int64_t n, cudaStream_t s);

namespace batch {

// ===========================================================================
// plain grouped GEMM
// ===========================================================================
struct PProb {
  const double *A;
  const double *B;
  double *C;
  int64_t m, k, n;
};
struct PItem {
  int prob, cfg, tm, tn;
};
constexpr int kPlainCfgs = 3;  // 0: 64x64 (4x4 per thread), 1: 32x32 (2x2), 2: 16x16 (1x1)
static int cfg_edge(int cfg) { return cfg == 0 ? 64 : cfg == 1 ? 32 : 16; }

template <bool ALIGNED>
__global__ void __launch_bounds__(256, 2)
    plain_grouped_kernel(const PProb *__restrict__ probs, const PItem *__restrict__ items, int nitems,
                         int64_t ri, int *counter) {
  __shared__ gtile::Smem sm;
  __shared__ int next;
  for (;;) {
    if (threadIdx.x == 0) next = atomicAdd(counter, 1);
    __syncthreads();
    const int w = next;
    __syncthreads();  // everyone has read `next` before thread 0 overwrites it
    if (w >= nitems) break;
    const PItem it = items[w];
    const PProb p = probs[it.prob];
    switch (it.cfg) {
      case 0:
        gtile::gemm_tile<4, 4, ALIGNED>(p.A, p.B, p.C, p.m, p.k, p.n, ri, (int64_t)it.tm * 64,
                                        (int64_t)it.tn * 64, sm);
        break;
      case 1:
        gtile::gemm_tile<2, 2, ALIGNED>(p.A, p.B, p.C, p.m, p.k, p.n, ri, (int64_t)it.tm * 32,
                                        (int64_t)it.tn * 32, sm);
        break;
      default:
        gtile::gemm_tile<1, 1, ALIGNED>(p.A, p.B, p.C, p.m, p.k, p.n, ri, (int64_t)it.tm * 16,
                                        (int64_t)it.tn * 16, sm);
        break;
    }
  }
}

// Complex problems (complex64x2): every 32 x 32 output tile runs the
// single-problem complex tile code (gtile::cgemm_tile).
template <bool ALIGNED>
__global__ void __launch_bounds__(256, 2)
    cplain_grouped_kernel(const PProb *__restrict__ probs, const PItem *__restrict__ items, int nitems,
                          int64_t ri, int *counter) {
  __shared__ gtile::CSmem sm;
  __shared__ int next;
  for (;;) {
    if (threadIdx.x == 0) next = atomicAdd(counter, 1);
    __syncthreads();
    const int w = next;
    __syncthreads();
    if (w >= nitems) break;
    const PItem it = items[w];
    const PProb p = probs[it.prob];
    gtile::cgemm_tile<ALIGNED>(p.A, p.B, p.C, p.m, p.k, p.n, ri, (int64_t)it.tm * gtile::kCBM,
                               (int64_t)it.tn * gtile::kCBN, sm);
  }
}

// ===========================================================================
// ragged elementwise
// ===========================================================================
struct RArr {
  const double *x;
  double *y;
  int64_t off;  // first index of this array in the concatenated space
};

template <int OP>
__device__ __forceinline__ mfdev::dd apply(mfdev::dd x) {
  if constexpr (OP == MFCUDA_EXP) return mfdev::dd_exp(x);
  if constexpr (OP == MFCUDA_LOG) return mfdev::dd_log(x);
  if constexpr (OP == MFCUDA_SIN) return mfdev::dd_sin(x);
  if constexpr (OP == MFCUDA_COS) return mfdev::dd_cos(x);
  return mfdev::dd_sqrt(x);
}

// last array whose start is <= e (offsets ascending, arrays may be empty)
__device__ __forceinline__ int find_array(const RArr *arrs, int narr, int64_t e) {
  int lo = 0, hi = narr - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (arrs[mid].off <= e)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

template <int OP>
__global__ void __launch_bounds__(256) ragged_unary_kernel(const RArr *__restrict__ arrs, int narr,
                                                           int64_t total) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
    const RArr a = arrs[find_array(arrs, narr, e)];
    const int64_t i = e - a.off;
    mfdev::dd v = mfdev::make(a.x[2 * i], a.x[2 * i + 1]);
    mfdev::dd r = apply<OP>(v);
    a.y[2 * i] = r.hi;
    a.y[2 * i + 1] = r.lo;
  }
}

// ===========================================================================
// split grouped pipeline
// ===========================================================================
using namespace split;

// One real product of the grouped split pipeline: a real problem, or one of
// the four real products of a complex problem (re = ArBr - AiBi,
// im = ArBi + AiBr).  Operands and the output are strided views (DD element e
// at double2 index e * stride); a product may reuse the statistics and slices
// of another product's A or B operand and share its plan (the four products
// of a complex problem use one slice count, planned from all four operands).
struct SProb {
  const double *A, *B;
  double *C;
  int64_t astride, bstride, cstride;
  int mode;  // recombination: 0 store, 1 C - P, 2 C + P
  int own_a, own_b, own_plan;
  int64_t m, k, n, M_pad, N_pad, K_pad;
  int bn, kcb, nkc, kblocks, ntm, ntn;
  int *sigA, *muA, *flagA, *sigB, *muB, *flagB;
  int *sigA2, *muA2, *sigB2, *muB2;  // the plan's second A and B operands (complex), or null
  int8_t *As, *Bs;
  int32_t *D;
  Plan *plan;
  int crt;       // CRT form (crt_device.cuh): slices are residues, items single products
  int nsl;       // slice slots per operand: SMAX digits, or the most moduli the CRT plan can use
  CrtConst *cc;  // the plan's reconstruction constants (CRT form)
};
// phases with a per-problem block count (prefix sums in a table); the
// recombination runs in two launches: stores first, then the - / + updates
enum { PH_SCAN_A, PH_SCAN_B, PH_SLICE_A, PH_SLICE_B, PH_COMBINE, PH_COMBINE2, PH_ITEMS, PH_COUNT };

__device__ __forceinline__ int find_prob(const int64_t *prefix, int nprob, int64_t b) {
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(256) g_scan_a(const SProb *probs, const int64_t *prefix, int nprob) {
  const int p = find_prob(prefix, nprob, blockIdx.x);
  const SProb &P = probs[p];
  const int64_t l = blockIdx.x - prefix[p];
  const int64_t nbx = (P.m + 255) / 256;
  scan_a_body(P.A, P.m, P.k, P.astride, 64, P.sigA, P.muA, P.flagA, l % nbx, l / nbx);
}
// a warp per column, 8 columns per block
__global__ void __launch_bounds__(256) g_scan_b(const SProb *probs, const int64_t *prefix, int nprob) {
  const int p = find_prob(prefix, nprob, blockIdx.x);
  const SProb &P = probs[p];
  const int64_t j = (int64_t)(blockIdx.x - prefix[p]) * 8 + (threadIdx.x >> 5);
  if (j < P.n) scan_b_warp(P.B, P.k, P.bstride, P.sigB, P.muB, P.flagB, j);
}
__global__ void __launch_bounds__(256) g_plan(const SProb *probs, int slices, double target) {
  const SProb &P = probs[blockIdx.x];
  if (!P.own_plan) return;
  StatSet st;
  st.n = 0;
  auto add = [&](int *sig, const int *mu, int64_t count, int side) {
    st.sig[st.n] = sig;
    st.mu[st.n] = mu;
    st.count[st.n] = count;
    st.side[st.n] = side;
    ++st.n;
  };
  add(P.sigA, P.muA, P.m, 0);
  if (P.sigA2) add(P.sigA2, P.muA2, P.m, 0);
  add(P.sigB, P.muB, P.n, 1);
  if (P.sigB2) add(P.sigB2, P.muB2, P.n, 1);
  if (P.crt)
    crt_plan_body(st, slices, target, P.k, P.plan, P.cc);  // slices: the operand bits W (0 = from target)
  else
    plan_body(st, slices, target, P.plan);
}
__global__ void __launch_bounds__(256) g_slice_a(const SProb *probs, const int64_t *prefix, int nprob) {
  const int p = find_prob(prefix, nprob, blockIdx.x);
  const SProb &P = probs[p];
  const int64_t l = blockIdx.x - prefix[p];
  const int64_t nbx = P.M_pad / 32;
  slice_a_body(P.A, P.m, P.k, P.astride, P.M_pad, P.K_pad, P.sigA, P.flagA, P.plan, P.As, l % nbx, l / nbx);
}
// CRT form: residues instead of digits, in MN-major planes As[t][p][i] (the
// rows of one K index contiguous); flat: thread t of the problem takes K
// index t / (M_pad / 8), rows 8 (t % (M_pad / 8)) .. + 7
__global__ void __launch_bounds__(256) g_crt_slice_a(const SProb *probs, const int64_t *prefix, int nprob) {
  const int p = find_prob(prefix, nprob, blockIdx.x);
  const SProb &P = probs[p];
  const int64_t t = (int64_t)(blockIdx.x - prefix[p]) * 256 + threadIdx.x;
  const int64_t per_k = P.M_pad / 8;
  const int64_t kp = t / per_k;
  if (kp < P.K_pad)
    crt_slice_a_mn_one(P.A, P.m, P.k, P.astride, P.M_pad, P.K_pad, P.sigA, P.flagA, P.plan, P.As,
                       (t % per_k) * 8, kp);
}
__global__ void __launch_bounds__(256) g_crt_slice_b(const SProb *probs, const int64_t *prefix, int nprob) {
  const int p = find_prob(prefix, nprob, blockIdx.x);
  const SProb &P = probs[p];
  const int64_t t = (int64_t)(blockIdx.x - prefix[p]) * 256 + threadIdx.x;
  const int64_t per_col = P.K_pad / 8;
  const int64_t j = t / per_col;
  if (j < P.N_pad)
    crt_slice_b_one(P.B, P.k, P.n, P.bstride, P.N_pad, P.K_pad, P.sigB, P.flagB, P.plan, P.Bs, j, (t % per_col) * 8);
}
// flat: thread t of the problem takes column t / (K_pad / 8), entries 8 (t % (K_pad / 8)) .. + 7
__global__ void __launch_bounds__(256) g_slice_b(const SProb *probs, const int64_t *prefix, int nprob) {
  const int p = find_prob(prefix, nprob, blockIdx.x);
  const SProb &P = probs[p];
  const int64_t t = (int64_t)(blockIdx.x - prefix[p]) * 256 + threadIdx.x;
  const int64_t per_col = P.K_pad / 8;
  const int64_t j = t / per_col;
  if (j < P.N_pad)
    slice_b_one(P.B, P.k, P.n, P.bstride, P.N_pad, P.K_pad, P.sigB, P.flagB, P.plan, P.Bs, j, (t % per_col) * 8);
}
// flat: thread t of the problem owns rows 4 (t % q) .. + 3 of column t / q,
// q = ceil(m / 4) (combine4_body)
constexpr int kCombineThreads = 128;
static int64_t combine_blocks(int64_t m, int64_t n) {
  return (((m + 3) / 4) * n + kCombineThreads - 1) / kCombineThreads;
}
__global__ void __launch_bounds__(kCombineThreads) g_combine(const SProb *probs, const int64_t *prefix, int nprob) {
  const int p = find_prob(prefix, nprob, blockIdx.x);
  const SProb &P = probs[p];
  const int64_t t = (int64_t)(blockIdx.x - prefix[p]) * kCombineThreads + threadIdx.x;
  const int64_t q = (P.m + 3) / 4;
  combine4_body(P.D, P.plan, P.sigA, P.flagA, P.sigB, P.flagB, P.m, P.n, P.M_pad, P.N_pad, P.nkc, P.C,
                P.cstride, P.mode, t % q, t / q);
}

// CRT form: the tensor-core reconstruction (crt_combine_tc_body), a block
// per 128 rows and CTC_QUADS column quads of a problem.
static int64_t crt_combine_blocks(int64_t m, int64_t n) {
  return ((m + CTC_THREADS - 1) / CTC_THREADS) * (((n + 3) / 4 + CTC_QUADS - 1) / CTC_QUADS);
}
__global__ void __launch_bounds__(CTC_THREADS, 4) g_crt_combine(const SProb *probs, const int64_t *prefix, int nprob,
                                                             int *status, uint64_t wait_ns) {
  extern __shared__ uint8_t ctc_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(ctc_raw) + 1023) & ~uintptr_t(1023));
  const int p = find_prob(prefix, nprob, blockIdx.x);
  const SProb &P = probs[p];
  const int64_t l = blockIdx.x - prefix[p], nbx = (P.m + CTC_THREADS - 1) / CTC_THREADS;
  crt_combine_tc_body(reinterpret_cast<const uint8_t *>(P.D), P.plan, P.cc, P.sigA, P.flagA, P.sigB, P.flagB, P.m,
                      P.n, P.M_pad, P.N_pad, P.nkc, P.k, P.C, P.cstride, P.mode, (l % nbx) * CTC_THREADS,
                      (l / nbx) * CTC_QUADS, smem, status, wait_ns);
}

struct GItem {
  int g, kc, tm, tn;
};
__device__ __forceinline__ GItem decode_item(const SProb &P, int64_t local) {
  GItem it;
  const int ntiles = P.ntm * P.ntn;
  const int64_t per_g = (int64_t)P.nkc * ntiles;
  it.g = P.nsl - 1 - (int)(local / per_g);
  const int64_t r = local % per_g;
  it.kc = (int)(r / ntiles);
  const int tile = (int)(r % ntiles);
  it.tm = tile % P.ntm;
  it.tn = tile / P.ntm;
  return it;
}

// Persistent tensor-core kernel over every problem's items (static
// round-robin).  The warp roles and barriers of split_mma_kernel, with eight
// epilogue warps (two per TMEM lane quadrant, each draining half of the
// accumulator's columns); per item it looks up the problem, skips diagonals
// beyond the problem's plan, and uses the problem's tensor maps (global
// memory) and tile width.
constexpr int G_EPI_WARPS = 8;
constexpr int G_THREADS = 64 + 32 * G_EPI_WARPS;  // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue
__global__ void __launch_bounds__(G_THREADS, 1)
    g_mma(const SProb *__restrict__ probs, const CUtensorMap *__restrict__ maps,
          const int64_t *__restrict__ prefix, int nprob, int64_t items, int *status, uint64_t wait_ns) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t *sA = smem;
  uint8_t *sB = smem + NSTAGE * A_STAGE;
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + NSTAGE * STAGE);
  uint64_t *empty = full + NSTAGE;
  uint64_t *tfull = empty + NSTAGE;
  uint64_t *tempty = tfull + 2;
  uint64_t *drain = tempty + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mftc::mbar_init(&full[s], 1);
      mftc::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mftc::mbar_init(&tfull[a], 1);
      mftc::mbar_init(&tempty[a], G_EPI_WARPS);
    }
    mftc::mbar_init(drain, 1);
    *abort_flag = 0;
    mftc::fence_mbar_init();
  }
  if (warp == 1) {
    mftc::tmem_alloc(tmem_slot, TMEM_COLS);
    mftc::tmem_relinquish();
  }
  mftc::tc_fence_before();
  __syncthreads();
  mftc::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  auto fail = [&](int code) {
    *abort_flag = 1;
    record_abort(status, code);
  };
  ArmedStages<NSTAGE> arm;  // the producer's armed stages
  arm.clear();
  // item -> (problem, decoded item, active?)
  auto lookup = [&](int64_t w, int &p, GItem &it) -> bool {
    p = find_prob(prefix, nprob, w);
    const SProb &P = probs[p];
    it = decode_item(P, w - prefix[p]);
    return it.g <= P.plan->G;
  };

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int64_t w = blockIdx.x; w < items && ok; w += gridDim.x) {
        int p;
        GItem it;
        if (!lookup(w, p, it)) continue;
        const SProb &P = probs[p];
        const int kb0 = it.kc * P.kcb, kb1 = min(P.kblocks, kb0 + P.kcb);
        const uint32_t bytes = (uint32_t)(A_STAGE + P.bn * BK);
        for (int s = P.crt ? it.g : 0; s <= it.g && ok; ++s) {  // CRT: the single product A_g B_g
          for (int kb = kb0; kb < kb1; ++kb) {
            if (!wait_bar(&empty[stage], phase ^ 1, abort_flag, wait_ns)) {
              fail(1);
              ok = false;
              break;
            }
            mftc::mbar_arrive_expect_tx(&full[stage], bytes);
            if (P.crt)  // MN-major residue planes: (row, K index, modulus)
              mftc::tma_load_3d(sA + stage * A_STAGE, &maps[2 * p], &full[stage], it.tm * BM, kb * BK, s);
            else
              mftc::tma_load_3d(sA + stage * A_STAGE, &maps[2 * p], &full[stage], kb * BK, it.tm * BM, s);
            mftc::tma_load_3d(sB + stage * B_STAGE, &maps[2 * p + 1], &full[stage], kb * BK, it.tn * P.bn,
                              P.crt ? s : it.g - s);
            arm.arm(stage, phase);
            if (++stage == NSTAGE) {
              stage = 0;
              phase ^= 1;
            }
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      for (int64_t w = blockIdx.x; w < items && ok; w += gridDim.x) {
        int p;
        GItem it;
        if (!lookup(w, p, it)) continue;
        const SProb &P = probs[p];
        const int kb0 = it.kc * P.kcb, kb1 = min(P.kblocks, kb0 + P.kcb);
        // CRT residues are unsigned, and A's planes MN-major (a K step of 32 rows is 4096 bytes)
        const uint32_t idesc = P.crt ? mftc::idesc_u8(BM, P.bn) | mftc::IDESC_A_MN : mftc::idesc_i8(BM, P.bn);
        const uint32_t a_kstep = P.crt ? 32 * 128 : UMMA_K;
        if (!wait_bar(&tempty[acc], acc_phase ^ 1, abort_flag, wait_ns)) {
          fail(2);
          break;
        }
        mftc::tc_fence_after();
        const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
        uint32_t accumulate = 0;
        for (int s = P.crt ? it.g : 0; s <= it.g && ok; ++s) {
          for (int kb = kb0; kb < kb1; ++kb) {
            if (!wait_bar(&full[stage], phase, abort_flag, wait_ns)) {
              fail(4);
              ok = false;
              break;
            }
            mftc::tc_fence_after();
            const uint32_t a0 = mftc::smem_u32(sA + stage * A_STAGE);
            const uint32_t b0 = mftc::smem_u32(sB + stage * B_STAGE);
#pragma unroll
            for (int kk = 0; kk < BK / UMMA_K; ++kk) {
              mftc::umma_i8(d_tmem, mftc::smem_desc_k_sw128(a0 + kk * a_kstep),
                            mftc::smem_desc_k_sw128(b0 + kk * UMMA_K), idesc, accumulate);
              accumulate = 1;
            }
            mftc::umma_commit(&empty[stage]);
            if (++stage == NSTAGE) {
              stage = 0;
              phase ^= 1;
            }
          }
        }
        if (!ok) break;
        mftc::umma_commit(&tfull[acc]);
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1;
        }
      }
      mftc::umma_commit(drain);
      uint64_t t0 = globaltimer();
      while (!mftc::mbar_try_wait(drain, 0) && globaltimer() - t0 < WAIT_NS) {
      }
    }
  } else {
    const int quad = warp & 3;           // TMEM lanes this warp may read
    const int half = (warp - 2) / 4;     // which half of the accumulator's columns
    const int row = quad * 32 + lane;
    int acc = 0;
    uint32_t acc_phase = 0;
    for (int64_t w = blockIdx.x; w < items; w += gridDim.x) {
      int p;
      GItem it;
      if (!lookup(w, p, it)) continue;
      const SProb &P = probs[p];
      bool got = wait_bar(&tfull[acc], acc_phase, abort_flag, wait_ns);
      if (!__all_sync(0xffffffffu, got)) {
        if (lane == 0) fail(8);
        break;
      }
      mftc::tc_fence_after();
      const int64_t off = ((int64_t)(it.g * P.nkc + it.kc) * P.N_pad + (int64_t)it.tn * P.bn) * P.M_pad +
                          (int64_t)it.tm * BM + row;
      const int nch = P.bn / 64, ch0 = half * nch;  // this warp's 32-column chunks
      if (P.crt) {  // residues modulo m_g, four columns per 32-bit word (crt_device.cuh)
        uint32_t *dst = reinterpret_cast<uint32_t *>(P.D) + crt_word_index(off, P.M_pad) + (int64_t)ch0 * 8 * P.M_pad;
        for (int chunk = ch0; chunk < ch0 + nch; ++chunk) {
          uint32_t r[32];
          mftc::tmem_ld_32x32b_x32(tmem_base + ((uint32_t)(quad * 32) << 16) + (uint32_t)(acc * BN + chunk * 32), r);
          mftc::tmem_wait_ld();
#pragma unroll
          for (int g = 0; g < 8; ++g) {
            __stcs(dst, crt_pack4(r[4 * g], r[4 * g + 1], r[4 * g + 2], r[4 * g + 3], it.g));
            dst += P.M_pad;
          }
        }
      } else {
        int32_t *dst_base = P.D + off;
        for (int chunk = ch0; chunk < ch0 + nch; ++chunk) {
          uint32_t r[32];
          mftc::tmem_ld_32x32b_x32(tmem_base + ((uint32_t)(quad * 32) << 16) + (uint32_t)(acc * BN + chunk * 32), r);
          mftc::tmem_wait_ld();
          int32_t *dst = dst_base + (int64_t)chunk * 32 * P.M_pad;
#pragma unroll
          for (int q = 0; q < 32; ++q) __stcs(dst + (int64_t)q * P.M_pad, (int32_t)r[q]);  // evict-first: keep L2 for the slices
        }
      }
      mftc::tc_fence_before();
      __syncwarp();
      if (lane == 0) mftc::mbar_arrive(&tempty[acc]);
      if (++acc == 2) {
        acc = 0;
        acc_phase ^= 1;
      }
    }
  }
  mftc::tc_fence_before();
  __syncthreads();
  mftc::tc_fence_after();
  if (*abort_flag) {  // read after the barrier: the same value in every thread
    // copies in flight that no MMA consumed land before shared memory is released
    if (warp == 0 && lane == 0) arm.drain(full, NSTAGE);
    __syncthreads();
  }
  if (warp == 1) {
    __syncwarp();
    mftc::tmem_dealloc(tmem_base, TMEM_COLS);
  }
}

__global__ void fill_kernel(int *p, int64_t n, int v) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// ===========================================================================
// autotuner cache
// ===========================================================================
static std::mutex g_tune_mu;
static std::map<std::string, int> g_tune;
static bool g_tune_loaded = false;

static std::string cache_path() {
  const char *p = std::getenv("MFCUDA_AUTOTUNE_CACHE");
  if (p && *p) return p;
  const char *home = std::getenv("HOME");
  return std::string(home ? home : "/tmp") + "/.cache/multifloats_b200/autotune.txt";
}
static void tune_load() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  FILE *f = std::fopen(cache_path().c_str(), "r");
  if (!f) return;
  char key[256];
  int v;
  while (std::fscanf(f, "%255s %d", key, &v) == 2) g_tune[key] = v;
  std::fclose(f);
}
static void tune_save() {
  std::string path = cache_path();
  std::string dir = path.substr(0, path.find_last_of('/'));
  for (size_t i = 1; i <= dir.size(); ++i)  // create the directory chain
    if (i == dir.size() || dir[i] == '/') (void)::mkdir(dir.substr(0, i).c_str(), 0755);
  FILE *f = std::fopen(path.c_str(), "w");
  if (!f) return;
  for (auto &kv : g_tune) std::fprintf(f, "%s %d\n", kv.first.c_str(), kv.second);
  std::fclose(f);
}


// ===========================================================================
// host side
// ===========================================================================
static int clog2(int64_t v) {
  int b = 0;
  while (((int64_t)1 << b) < v) ++b;
  return b;
}
static int64_t ru(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

static bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

static int plain_heuristic(int64_t m, int64_t n) {
  int64_t e = std::min(m, n);
  return e >= 48 ? 0 : e >= 24 ? 1 : 2;
}

// Plan memory: one device allocation holding the tables and the workspace.
struct Arena {
  size_t off = 0;
  size_t take(size_t bytes, size_t align = 256) {
    off = (off + align - 1) / align * align;
    size_t o = off;
    off += bytes;
    return o;
  }
};

}  // namespace batch
}  // namespace mfcuda

struct mfcuda_batch {
  int kind = 0;  // 0 plain GEMM, 1 split GEMM, 2 ragged unary
  int kchunk = 0;  // split: K chunk in elements
  int device = 0;
  void *mem = nullptr;
  size_t mem_bytes = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t count = 0, work = 0;
  int *status = nullptr;
  std::vector<int> cfg;
};

namespace mfcuda {
namespace batch {

static void destroy(mfcuda_batch *b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->mem) cudaFree(b->mem);
  delete b;
}

// Captures `enqueue` (a sequence of launches on the given stream) into the
// plan's graph.
template <class F>
static int capture(mfcuda_batch *b, F enqueue) {
  cudaStream_t cs;
  MF_TRY_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  int rc = MFCUDA_OK;
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    rc = MFCUDA_ERR_CUDA;
  } else {
    enqueue(cs);
    cudaError_t e1 = cudaGetLastError();
    cudaError_t e2 = cudaStreamEndCapture(cs, &b->graph);
    if (e1 != cudaSuccess || e2 != cudaSuccess)
      rc = MFCUDA_ERR_CUDA;
    else if (cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess)
      rc = MFCUDA_ERR_CUDA;
  }
  (void)cudaGetLastError();
  cudaStreamDestroy(cs);
  return rc;
}

// ---- plain ------------------------------------------------------------------
// complex = true: complex64x2 problems, 32 x 32 tiles (cfg ignored).
static int create_plain(const mfcuda_gemm_desc *d, int64_t count, int64_t ri, const std::vector<int> &cfg,
                        mfcuda_batch **out, bool complex = false) {
  std::vector<int64_t> order;
  bool aligned = true;
  for (int64_t p = 0; p < count; ++p) {
    if (d[p].m > 0 && d[p].n > 0) order.push_back(p);
    aligned = aligned && aligned16(d[p].a) && aligned16(d[p].b) && aligned16(d[p].c);
  }
  std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return d[x].k > d[y].k; });
  std::vector<PProb> probs(count);
  std::vector<PItem> items;
  for (int64_t p = 0; p < count; ++p)
    probs[p] = {static_cast<const double *>(d[p].a), static_cast<const double *>(d[p].b),
                static_cast<double *>(d[p].c), d[p].m, d[p].k, d[p].n};
  for (int64_t p : order) {
    const int e = complex ? gtile::kCBM : cfg_edge(cfg[p]);
    for (int64_t tn = 0; tn < (d[p].n + e - 1) / e; ++tn)
      for (int64_t tm = 0; tm < (d[p].m + e - 1) / e; ++tm)
        items.push_back({(int)p, complex ? 1 : cfg[p], (int)tm, (int)tn});
  }
  if (items.size() > (size_t)INT32_MAX) return MFCUDA_ERR_UNSUPPORTED;
  auto *b = new mfcuda_batch;
  b->kind = 0;
  b->count = count;
  b->work = (int64_t)items.size();
  b->cfg = cfg;
  cudaGetDevice(&b->device);
  Arena ar;
  size_t o_probs = ar.take(sizeof(PProb) * std::max<int64_t>(count, 1));
  size_t o_items = ar.take(sizeof(PItem) * std::max<size_t>(items.size(), 1));
  size_t o_ctr = ar.take(sizeof(int));
  b->mem_bytes = ar.off;
  if (injected_alloc_failure() || cudaMalloc(&b->mem, b->mem_bytes) != cudaSuccess) {
    (void)cudaGetLastError();
    destroy(b);
    return MFCUDA_ERR_ALLOC;
  }
  uint8_t *base = static_cast<uint8_t *>(b->mem);
  PProb *dp = reinterpret_cast<PProb *>(base + o_probs);
  PItem *di = reinterpret_cast<PItem *>(base + o_items);
  int *ctr = reinterpret_cast<int *>(base + o_ctr);
  if (cudaMemcpy(dp, probs.data(), sizeof(PProb) * count, cudaMemcpyHostToDevice) != cudaSuccess ||
      (!items.empty() &&
       cudaMemcpy(di, items.data(), sizeof(PItem) * items.size(), cudaMemcpyHostToDevice) != cudaSuccess)) {
    destroy(b);
    return MFCUDA_ERR_CUDA;
  }
  const int nitems = (int)items.size();
  int grid = sm_count() * 2;
  if (grid > nitems) grid = nitems > 0 ? nitems : 1;
  int rc = capture(b, [&](cudaStream_t cs) {
    cudaMemsetAsync(ctr, 0, sizeof(int), cs);
    if (complex) {
      if (aligned)
        cplain_grouped_kernel<true><<<grid, 256, 0, cs>>>(dp, di, nitems, ri, ctr);
      else
        cplain_grouped_kernel<false><<<grid, 256, 0, cs>>>(dp, di, nitems, ri, ctr);
    } else if (aligned) {
      plain_grouped_kernel<true><<<grid, 256, 0, cs>>>(dp, di, nitems, ri, ctr);
    } else {
      plain_grouped_kernel<false><<<grid, 256, 0, cs>>>(dp, di, nitems, ri, ctr);
    }
  });
  if (rc != MFCUDA_OK) {
    destroy(b);
    return rc;
  }
  *out = b;
  return MFCUDA_OK;
}

// ---- split ------------------------------------------------------------------
static std::once_flag g_gmma_attr;

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}
static bool make_map(CUtensorMap *map, void *base, int64_t rows, int64_t K_pad, uint32_t box_rows, int nsl) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)K_pad, (cuuint64_t)rows, (cuuint64_t)nsl};
  cuuint64_t strides[2] = {(cuuint64_t)K_pad, (cuuint64_t)(rows * K_pad)};
  cuuint32_t box[3] = {(cuuint32_t)BK, box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// MN-major residue planes (row, K index, modulus) of the CRT form's A side:
// boxes of 128 rows x BK K indices, 128-byte swizzle.
static bool make_map_mn(CUtensorMap *map, void *base, int64_t M_pad, int64_t K_pad, int nsl) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)M_pad, (cuuint64_t)K_pad, (cuuint64_t)nsl};
  cuuint64_t strides[2] = {(cuuint64_t)M_pad, (cuuint64_t)(M_pad * K_pad)};
  cuuint32_t box[3] = {128, (cuuint32_t)BK, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// One real product to plan (host side of SProb): operand / output views, its
// tile width, and where its A operand, B operand and plan come from (-1: its
// own; else the index of the product that provides them).  A plan owner lists
// in plan_a2 / plan_b2 the products whose A / B statistics also enter its plan.
struct Spec {
  const double *A, *B;
  double *C;
  int64_t astride, bstride, cstride;
  int mode;
  int64_t m, k, n;
  int bn;
  int a_src, b_src, plan_src, plan_a2, plan_b2;
};

// kcb: K chunk in blocks of 128 (shared by all products).  crt: the CRT form,
// `slices` then being the operand bits W (0: chosen for `target`).
static int create_split_specs(std::vector<Spec> specs, int64_t count, int slices, double target,
                              const std::vector<int> &cfg, int kcb_all, mfcuda_batch **out, bool crt) {
  // longest K first (stable: the products of one complex problem stay together)
  const int np = (int)specs.size();
  std::vector<int> order(np), pos(np);
  for (int q = 0; q < np; ++q) order[q] = q;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return specs[x].k > specs[y].k; });
  for (int q = 0; q < np; ++q) pos[order[q]] = q;
  std::vector<Spec> sp(np);
  for (int q = 0; q < np; ++q) {
    sp[q] = specs[order[q]];
    for (int *r : {&sp[q].a_src, &sp[q].b_src, &sp[q].plan_src, &sp[q].plan_a2, &sp[q].plan_b2})
      if (*r >= 0) *r = pos[*r];
  }
  std::vector<SProb> probs(np);
  Arena ar;
  size_t o_probs = ar.take(sizeof(SProb) * std::max(np, 1));
  size_t o_prefix = ar.take(sizeof(int64_t) * PH_COUNT * std::max(np, 1));
  size_t o_maps = ar.take(sizeof(CUtensorMap) * 2 * std::max(np, 1), 128);
  size_t o_status = ar.take(sizeof(int));
  std::vector<size_t> o_plan(np, 0), o_cc(np, 0), o_as(np, 0), o_bs(np, 0), o_d(np);
  std::vector<int64_t> rowA(np, -1), rowB(np, -1);  // statistics rows of owned operands
  int64_t rows_total = 0;
  std::vector<int64_t> prefix(PH_COUNT * (size_t)std::max(np, 1), 0);
  int64_t total[PH_COUNT] = {0, 0, 0, 0, 0, 0, 0};
  for (int q = 0; q < np; ++q) {
    const Spec &g = sp[q];
    SProb &P = probs[q];
    P.A = g.A;
    P.B = g.B;
    P.C = g.C;
    P.astride = g.astride;
    P.bstride = g.bstride;
    P.cstride = g.cstride;
    P.mode = g.mode;
    P.own_a = g.a_src < 0;
    P.own_b = g.b_src < 0;
    P.own_plan = g.plan_src < 0;
    P.m = g.m;
    P.k = g.k;
    P.n = g.n;
    P.bn = g.bn;
    P.M_pad = ru(g.m, BM);
    P.N_pad = ru(g.n, P.bn);
    P.K_pad = ru(g.k < 1 ? 1 : g.k, BK);
    P.kblocks = (int)(P.K_pad / BK);
    P.kcb = std::min(kcb_all, KC_BLOCKS);
    P.nkc = (P.kblocks + P.kcb - 1) / P.kcb;
    P.ntm = (int)(P.M_pad / BM);
    P.ntn = (int)(P.N_pad / P.bn);
    P.crt = crt ? 1 : 0;
    P.nsl = crt ? crt_slices_max(g.k < 1 ? 1 : g.k, slices) : SMAX;
    P.cc = nullptr;
    if (P.own_plan) {
      o_plan[q] = ar.take(sizeof(Plan));
      if (crt) o_cc[q] = ar.take(sizeof(CrtConst));
    }
    if (P.own_a) {
      rowA[q] = rows_total;
      rows_total += P.M_pad;
      o_as[q] = ar.take((size_t)P.nsl * P.M_pad * P.K_pad, 1024);
    }
    if (P.own_b) {
      rowB[q] = rows_total;
      rows_total += P.N_pad;
      o_bs[q] = ar.take((size_t)P.nsl * P.N_pad * P.K_pad, 1024);
    }
    // INT32 diagonal sums, or (CRT) byte residues four columns to a word
    o_d[q] = ar.take((size_t)P.nsl * P.nkc * P.N_pad * P.M_pad * (crt ? 1 : sizeof(int32_t)));
    const int64_t comb = crt ? crt_combine_blocks(P.m, P.n) : combine_blocks(P.m, P.n);
    const int64_t blocks[PH_COUNT] = {
        P.own_a ? ((P.m + 255) / 256) * ((P.k + 63) / 64) : 0,
        P.own_b && P.k > 0 ? (P.n + 7) / 8 : 0,
        P.own_a ? (crt ? (P.K_pad * (P.M_pad / 8) + 255) / 256 : (P.M_pad / 32) * (P.K_pad / 64)) : 0,
        P.own_b ? (P.N_pad * (P.K_pad / 8) + 255) / 256 : 0,
        P.mode == 0 ? comb : 0,
        P.mode != 0 ? comb : 0,
        (int64_t)P.nsl * P.nkc * P.ntm * P.ntn};
    for (int ph = 0; ph < PH_COUNT; ++ph) {
      prefix[(size_t)ph * np + q] = total[ph];
      total[ph] += blocks[ph];
    }
  }
  for (int ph = 0; ph < PH_COUNT; ++ph)
    if (total[ph] > INT32_MAX) return MFCUDA_ERR_UNSUPPORTED;
  // exponent statistics of all owned operands in three contiguous arrays
  const size_t o_sig = ar.take(sizeof(int) * std::max<int64_t>(rows_total, 1));
  const size_t o_mu = ar.take(sizeof(int) * std::max<int64_t>(rows_total, 1));
  const size_t o_flag = ar.take(sizeof(int) * std::max<int64_t>(rows_total, 1));
  auto *b = new mfcuda_batch;
  b->kind = 1;
  b->kchunk = std::min(kcb_all, KC_BLOCKS) * BK;
  b->count = count;
  b->work = total[PH_ITEMS];
  b->cfg = cfg;
  cudaGetDevice(&b->device);
  b->mem_bytes = ar.off;
  if (injected_alloc_failure() || cudaMalloc(&b->mem, b->mem_bytes) != cudaSuccess) {
    (void)cudaGetLastError();
    destroy(b);
    return MFCUDA_ERR_ALLOC;
  }
  uint8_t *base = static_cast<uint8_t *>(b->mem);
  int *sig0 = reinterpret_cast<int *>(base + o_sig), *mu0 = reinterpret_cast<int *>(base + o_mu),
      *flag0 = reinterpret_cast<int *>(base + o_flag);
  // owned storage first, then the borrowed pointers
  for (int q = 0; q < np; ++q) {
    SProb &P = probs[q];
    if (P.own_plan) {
      P.plan = reinterpret_cast<Plan *>(base + o_plan[q]);
      if (crt) P.cc = reinterpret_cast<CrtConst *>(base + o_cc[q]);
    }
    if (P.own_a) {
      P.sigA = sig0 + rowA[q];
      P.muA = mu0 + rowA[q];
      P.flagA = flag0 + rowA[q];
      P.As = reinterpret_cast<int8_t *>(base + o_as[q]);
    }
    if (P.own_b) {
      P.sigB = sig0 + rowB[q];
      P.muB = mu0 + rowB[q];
      P.flagB = flag0 + rowB[q];
      P.Bs = reinterpret_cast<int8_t *>(base + o_bs[q]);
    }
    P.D = reinterpret_cast<int32_t *>(base + o_d[q]);
  }
  std::vector<CUtensorMap> maps(2 * (size_t)std::max(np, 1));
  for (int q = 0; q < np; ++q) {
    SProb &P = probs[q];
    const Spec &g = sp[q];
    if (!P.own_plan) {
      P.plan = probs[g.plan_src].plan;
      P.cc = probs[g.plan_src].cc;
    }
    if (!P.own_a) {
      const SProb &S = probs[g.a_src];
      P.sigA = S.sigA;
      P.muA = S.muA;
      P.flagA = S.flagA;
      P.As = S.As;
    }
    if (!P.own_b) {
      const SProb &S = probs[g.b_src];
      P.sigB = S.sigB;
      P.muB = S.muB;
      P.flagB = S.flagB;
      P.Bs = S.Bs;
    }
    P.sigA2 = g.plan_a2 >= 0 ? probs[g.plan_a2].sigA : nullptr;
    P.muA2 = g.plan_a2 >= 0 ? probs[g.plan_a2].muA : nullptr;
    P.sigB2 = g.plan_b2 >= 0 ? probs[g.plan_b2].sigB : nullptr;
    P.muB2 = g.plan_b2 >= 0 ? probs[g.plan_b2].muB : nullptr;
    if (!(crt ? make_map_mn(&maps[2 * q], P.As, P.M_pad, P.K_pad, P.nsl)
              : make_map(&maps[2 * q], P.As, P.M_pad, P.K_pad, BM, P.nsl)) ||
        !make_map(&maps[2 * q + 1], P.Bs, P.N_pad, P.K_pad, (uint32_t)P.bn, P.nsl)) {
      destroy(b);
      return MFCUDA_ERR_CUDA;
    }
  }
  SProb *dp = reinterpret_cast<SProb *>(base + o_probs);
  int64_t *dprefix = reinterpret_cast<int64_t *>(base + o_prefix);
  CUtensorMap *dmaps = reinterpret_cast<CUtensorMap *>(base + o_maps);
  b->status = reinterpret_cast<int *>(base + o_status);
  if (np > 0 && (cudaMemcpy(dp, probs.data(), sizeof(SProb) * np, cudaMemcpyHostToDevice) != cudaSuccess ||
                 cudaMemcpy(dprefix, prefix.data(), sizeof(int64_t) * PH_COUNT * np, cudaMemcpyHostToDevice) !=
                     cudaSuccess ||
                 cudaMemcpy(dmaps, maps.data(), sizeof(CUtensorMap) * 2 * np, cudaMemcpyHostToDevice) !=
                     cudaSuccess)) {
    destroy(b);
    return MFCUDA_ERR_CUDA;
  }
  std::call_once(g_gmma_attr, [] {
    cudaFuncSetAttribute(g_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, MMA_SMEM);
    cudaFuncSetAttribute(g_crt_combine, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         crt_tc_smem((CRT_NMAX + 31) / 32));
  });
  // the reconstruction's shared tiles hold the most moduli of any product
  int nsl_max = 1;
  for (int q = 0; q < np; ++q) nsl_max = std::max(nsl_max, probs[q].nsl);
  int mma_grid = sm_count();
  if (mma_grid > total[PH_ITEMS]) mma_grid = (int)std::max<int64_t>(total[PH_ITEMS], 1);
  const uint64_t wait_ns = wait_limit_ns();  // captured into the graph with the plan
  int rc = capture(b, [&](cudaStream_t cs) {
    cudaMemsetAsync(b->status, 0, sizeof(int), cs);
    if (np == 0) return;
    const unsigned fb = (unsigned)((rows_total + 255) / 256);
    fill_kernel<<<fb, 256, 0, cs>>>(sig0, rows_total, SENT_LO);
    fill_kernel<<<fb, 256, 0, cs>>>(mu0, rows_total, SENT_HI);
    fill_kernel<<<fb, 256, 0, cs>>>(flag0, rows_total, 0);
    if (total[PH_SCAN_A]) g_scan_a<<<(unsigned)total[PH_SCAN_A], 256, 0, cs>>>(dp, dprefix + PH_SCAN_A * np, np);
    if (total[PH_SCAN_B]) g_scan_b<<<(unsigned)total[PH_SCAN_B], 256, 0, cs>>>(dp, dprefix + PH_SCAN_B * np, np);
    g_plan<<<np, 256, 0, cs>>>(dp, slices, target);
    if (total[PH_SLICE_A] && crt)
      g_crt_slice_a<<<(unsigned)total[PH_SLICE_A], 256, 0, cs>>>(dp, dprefix + PH_SLICE_A * np, np);
    else if (total[PH_SLICE_A])
      g_slice_a<<<(unsigned)total[PH_SLICE_A], 256, 0, cs>>>(dp, dprefix + PH_SLICE_A * np, np);
    if (total[PH_SLICE_B] && crt)
      g_crt_slice_b<<<(unsigned)total[PH_SLICE_B], 256, 0, cs>>>(dp, dprefix + PH_SLICE_B * np, np);
    else if (total[PH_SLICE_B])
      g_slice_b<<<(unsigned)total[PH_SLICE_B], 256, 0, cs>>>(dp, dprefix + PH_SLICE_B * np, np);
    g_mma<<<mma_grid, G_THREADS, MMA_SMEM, cs>>>(dp, dmaps, dprefix + PH_ITEMS * np, np, total[PH_ITEMS],
                                                   b->status, wait_ns);
    for (int ph : {PH_COMBINE, PH_COMBINE2}) {
      if (!total[ph]) continue;
      if (crt)
        g_crt_combine<<<(unsigned)total[ph], CTC_THREADS, crt_tc_smem((nsl_max + 31) / 32), cs>>>(
            dp, dprefix + ph * np, np, b->status, wait_ns);
      else
        g_combine<<<(unsigned)total[ph], kCombineThreads, 0, cs>>>(dp, dprefix + ph * np, np);
    }
  });
  if (rc != MFCUDA_OK) {
    destroy(b);
    return rc;
  }
  *out = b;
  return MFCUDA_OK;
}

// Given-up waits of the grouped tensor-core kernels (this file's record).
int wait_sticky_batched(bool clear) { return take_wait_sticky(clear); }

static bool split_args_ok(const mfcuda_gemm_desc &g) {
  return aligned16(g.a) && aligned16(g.b) && aligned16(g.c) && g.n <= 65535;
}

// Real problems: one product each.  cfg[p] = tile width N (256, 128 or 64).
static int create_split(const mfcuda_gemm_desc *d, int64_t count, int slices, double target,
                        const std::vector<int> &cfg, int kcb_all, mfcuda_batch **out, bool crt) {
  std::vector<Spec> specs;
  for (int64_t p = 0; p < count; ++p) {
    if (!split_args_ok(d[p])) return MFCUDA_ERR_UNSUPPORTED;
    if (d[p].m <= 0 || d[p].n <= 0) continue;
    specs.push_back({static_cast<const double *>(d[p].a), static_cast<const double *>(d[p].b),
                     static_cast<double *>(d[p].c), 1, 1, 1, 0, d[p].m, d[p].k, d[p].n, cfg[p], -1, -1, -1, -1,
                     -1});
  }
  return create_split_specs(std::move(specs), count, slices, target, cfg, kcb_all, out, crt);
}

// Complex problems (complex64x2 operands): four real products each, in the
// order and with the combination of mfcuda_cmatmuldd_mm_split (re = ArBr, then
// re - AiBi; im = ArBi, then im + AiBr), one plan from all four operands, each
// operand sliced once.
static int create_csplit(const mfcuda_gemm_desc *d, int64_t count, int slices, double target,
                         const std::vector<int> &cfg, int kcb_all, mfcuda_batch **out, bool crt) {
  std::vector<Spec> specs;
  for (int64_t p = 0; p < count; ++p) {
    if (!split_args_ok(d[p])) return MFCUDA_ERR_UNSUPPORTED;
    if (d[p].m <= 0 || d[p].n <= 0) continue;
    const double *A = static_cast<const double *>(d[p].a), *B = static_cast<const double *>(d[p].b);
    double *Cm = static_cast<double *>(d[p].c);
    const int64_t m = d[p].m, k = d[p].k, n = d[p].n;
    const int q = (int)specs.size();
    //           A      B      C       strides  mode  shape    bn      a_src  b_src  plan_src plan_a2 plan_b2
    specs.push_back({A, B, Cm, 2, 2, 2, 0, m, k, n, cfg[p], -1, -1, -1, q + 1, q + 1});          // re  = Ar Br
    specs.push_back({A + 2, B + 2, Cm, 2, 2, 2, 1, m, k, n, cfg[p], -1, -1, q, -1, -1});          // re -= Ai Bi
    specs.push_back({A, B + 2, Cm + 2, 2, 2, 2, 0, m, k, n, cfg[p], q, q + 1, q, -1, -1});        // im  = Ar Bi
    specs.push_back({A + 2, B, Cm + 2, 2, 2, 2, 2, m, k, n, cfg[p], q + 1, q, q, -1, -1});        // im += Ai Br
  }
  return create_split_specs(std::move(specs), count, slices, target, cfg, kcb_all, out, crt);
}

// ---- ragged elementwise -------------------------------------------------------
static int ragged_table(const float64x2 *const *xs, float64x2 *const *ys, const int64_t *ns, int64_t count,
                        std::vector<RArr> &tab, int64_t &total) {
  total = 0;
  tab.resize(count);
  for (int64_t a = 0; a < count; ++a) {
    if (ns[a] < 0 || !size_ok(ns[a], sizeof(float64x2))) return MFCUDA_ERR_INVALID_ARG;
    if (ns[a] > 0 && (!xs[a] || !ys[a])) return MFCUDA_ERR_INVALID_ARG;
    tab[a] = {reinterpret_cast<const double *>(xs[a]), reinterpret_cast<double *>(ys[a]), total};
    total += ns[a];
  }
  return MFCUDA_OK;
}
static void launch_ragged(int op, const RArr *tab, int narr, int64_t total, cudaStream_t s) {
  int64_t want = (total + 255) / 256, cap = (int64_t)sm_count() * 16;
  unsigned grid = (unsigned)std::max<int64_t>(1, std::min(want, cap));
  switch (op) {
    case MFCUDA_EXP: ragged_unary_kernel<MFCUDA_EXP><<<grid, 256, 0, s>>>(tab, narr, total); break;
    case MFCUDA_LOG: ragged_unary_kernel<MFCUDA_LOG><<<grid, 256, 0, s>>>(tab, narr, total); break;
    case MFCUDA_SIN: ragged_unary_kernel<MFCUDA_SIN><<<grid, 256, 0, s>>>(tab, narr, total); break;
    case MFCUDA_COS: ragged_unary_kernel<MFCUDA_COS><<<grid, 256, 0, s>>>(tab, narr, total); break;
    default: ragged_unary_kernel<MFCUDA_SQRT><<<grid, 256, 0, s>>>(tab, narr, total); break;
  }
}
static int create_unary(int op, const float64x2 *const *xs, float64x2 *const *ys, const int64_t *ns,
                        int64_t count, mfcuda_batch **out) {
  std::vector<RArr> tab;
  int64_t total;
  MF_TRY(ragged_table(xs, ys, ns, count, tab, total));
  auto *b = new mfcuda_batch;
  b->kind = 2;
  b->count = count;
  b->work = total;
  cudaGetDevice(&b->device);
  b->mem_bytes = sizeof(RArr) * std::max<int64_t>(count, 1);
  if (injected_alloc_failure() || cudaMalloc(&b->mem, b->mem_bytes) != cudaSuccess) {
    (void)cudaGetLastError();
    destroy(b);
    return MFCUDA_ERR_ALLOC;
  }
  RArr *dt = static_cast<RArr *>(b->mem);
  if (count > 0 && cudaMemcpy(dt, tab.data(), sizeof(RArr) * count, cudaMemcpyHostToDevice) != cudaSuccess) {
    destroy(b);
    return MFCUDA_ERR_CUDA;
  }
  int rc = capture(b, [&](cudaStream_t cs) {
    if (total > 0) launch_ragged(op, dt, (int)count, total, cs);
  });
  if (rc != MFCUDA_OK) {
    destroy(b);
    return rc;
  }
  *out = b;
  return MFCUDA_OK;
}

// ---- autotuner ------------------------------------------------------------------
// Candidates are timed on synthetic problems of the bucket's representative
// shape, in a batch as large as the bucket's population (at least enough
// tiles to fill the GPU), once per bucket; winners are cached on disk.
__global__ void synth_fill_kernel(double *p, int64_t n_dd, uint64_t seed) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_dd) return;
  uint64_t z = seed + (uint64_t)i * 0x9E3779B97F4A7C15ull;  // splitmix64
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  double u = (double)(z >> 11) * 0x1p-53 * 2.0 - 1.0;
  p[2 * i] = u;
  p[2 * i + 1] = u * 0x1p-60;
}

static double time_plan(mfcuda_batch *b, int reps) {
  cudaStream_t s;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaGraphLaunch(b->exec, s);  // warm-up
  cudaEventRecord(e0, s);
  for (int r = 0; r < reps; ++r) cudaGraphLaunch(b->exec, s);
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  return cudaGetLastError() == cudaSuccess ? ms / reps : 1e30;
}

struct Bucket {
  int bm, bn, bk;
  int64_t population;
};

// form 0: candidate = plain tile config; form 1: candidate = split tile width N.
static int tune_bucket(int form, const Bucket &bk, int64_t ri) {
  const int64_t m = (int64_t)1 << bk.bm, n = (int64_t)1 << bk.bn, k = (int64_t)1 << bk.bk;
  std::vector<int> cands = form == 0 ? std::vector<int>{0, 1, 2} : std::vector<int>{256, 128, 64};
  const int64_t tiles16 = ((m + 15) / 16) * ((n + 15) / 16);
  int64_t copies = std::max<int64_t>(bk.population, 1);
  if (form == 0) {
    copies = std::max<int64_t>(copies, (int64_t)sm_count() * 4 * 16 / std::max<int64_t>(tiles16, 1));
    copies = std::min<int64_t>(copies, 256);
  } else {
    copies = std::min<int64_t>(copies, 16);
  }
  void *buf = nullptr;
  const int64_t per = 2 * (m * k + k * n + m * n);
  if (cudaMalloc(&buf, sizeof(double) * per * copies) != cudaSuccess) {
    (void)cudaGetLastError();
    return form == 0 ? plain_heuristic(m, n) : 256;
  }
  double *p = static_cast<double *>(buf);
  synth_fill_kernel<<<(unsigned)((per * copies / 2 + 255) / 256), 256>>>(p, per * copies / 2, 12345);
  std::vector<mfcuda_gemm_desc> descs(copies);
  for (int64_t c = 0; c < copies; ++c) {
    double *base = p + c * per;
    descs[c] = {base, base + 2 * m * k, base + 2 * (m * k + k * n), m, k, n};
  }
  int best = cands[0];
  double best_ms = 1e30;
  for (int cand : cands) {
    if (form != 0 && cand > 64 && cand >= 2 * n) continue;  // wider than twice the problem: pure padding
    mfcuda_batch *b = nullptr;
    std::vector<int> cfg(copies, cand);
    int rc = form == 0 ? create_plain(descs.data(), copies, ri, cfg, &b)
                       : create_split(descs.data(), copies, 0, 8.0, cfg, KC_BLOCKS, &b, form == 2);
    if (rc != MFCUDA_OK) continue;
    double ms = time_plan(b, 2);
    destroy(b);
    if (ms < best_ms) {
      best_ms = ms;
      best = cand;
    }
  }
  cudaDeviceSynchronize();
  cudaFree(buf);
  return best;
}

static std::string bucket_key(int form, const Bucket &b) {
  char dev[256] = "gpu";
  cudaDeviceProp prop;
  int d = 0;
  if (cudaGetDevice(&d) == cudaSuccess && cudaGetDeviceProperties(&prop, d) == cudaSuccess)
    std::snprintf(dev, sizeof dev, "%s", prop.name);
  for (char *c = dev; *c; ++c)
    if (*c == ' ') *c = '_';
  char key[512];
  std::snprintf(key, sizeof key, "%s:%s:%d:%d:%d", dev, form == 0 ? "plain" : form == 1 ? "split" : "crt", b.bm,
                b.bn, b.bk);
  return key;
}

// Chooses per-problem configurations: the cached or freshly tuned winner of
// each shape bucket when tune != 0, else the built-in heuristic.
static std::vector<int> choose(int form, const mfcuda_gemm_desc *d, int64_t count, int tune, int64_t ri) {
  std::vector<int> cfg(count);
  std::map<std::tuple<int, int, int>, Bucket> buckets;
  // plain: the tile edge depends on m and n; split: the tile width N on n and
  // a coarse K class (m only changes the number of 128-row tiles)
  auto bucket_of = [&](const mfcuda_gemm_desc &g) {
    int bn = std::min(std::max(clog2(g.n), 4), 10);
    if (form == 0) return std::make_tuple(std::min(std::max(clog2(g.m), 4), 10), bn, 8);
    return std::make_tuple(bn, bn, std::min(std::max(clog2(g.k), 7), 10));
  };
  for (int64_t p = 0; p < count; ++p) {
    auto t = bucket_of(d[p]);
    auto &b = buckets[t];
    b.bm = std::get<0>(t);
    b.bn = std::get<1>(t);
    b.bk = std::get<2>(t);
    b.population++;
  }
  std::map<std::tuple<int, int, int>, int> win;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load();
    bool dirty = false;
    for (auto &kv : buckets) {
      const std::string key = bucket_key(form, kv.second);
      auto it = g_tune.find(key);
      if (it != g_tune.end()) {
        win[kv.first] = it->second;
      } else if (tune) {
        int best = tune_bucket(form, kv.second, ri);
        g_tune[key] = best;
        win[kv.first] = best;
        dirty = true;
      }
    }
    if (dirty) tune_save();
  }
  for (int64_t p = 0; p < count; ++p) {
    auto it = win.find(bucket_of(d[p]));
    if (it != win.end()) {
      cfg[p] = it->second;
    } else if (form == 0) {
      cfg[p] = plain_heuristic(d[p].m, d[p].n);
    } else {
      cfg[p] = d[p].n <= 64 ? 64 : d[p].n <= 128 ? 128 : 256;
    }
  }
  return cfg;
}

// Split-K rule: K chunks of at most KC_BLOCKS blocks (the INT32 bound); when
// the whole batch has fewer items than four per SM, shorter chunks raise the
// item count (the chunks' INT32 partials are summed exactly in the combine).
// nsl(k): slice slots (and so items per tile) of a product with inner size k.
template <class SlotFn>
static int choose_kcb(const mfcuda_gemm_desc *d, int64_t count, const std::vector<int> &cfg, int prods, SlotFn nsl) {
  int64_t items = 0, kmax = 1;
  for (int64_t p = 0; p < count; ++p) {
    if (d[p].m <= 0 || d[p].n <= 0) continue;
    int64_t kb = (ru(std::max<int64_t>(d[p].k, 1), BK)) / BK;
    kmax = std::max(kmax, kb);
    items += (int64_t)prods * nsl(d[p].k) * ((kb + KC_BLOCKS - 1) / KC_BLOCKS) * (ru(d[p].m, BM) / BM) *
             (ru(d[p].n, cfg[p]) / cfg[p]);
  }
  const int64_t want = (int64_t)sm_count() * 4;
  if (items >= want || items == 0) return KC_BLOCKS;
  int64_t split = (want + items - 1) / items;
  int64_t kcb = (std::min<int64_t>(kmax, KC_BLOCKS) + split - 1) / split;
  return (int)std::max<int64_t>(4, std::min<int64_t>(kcb, KC_BLOCKS));
}

}  // namespace batch
}  // namespace mfcuda

extern "C" {

static int batch_create(const mfcuda_gemm_desc *descs, int64_t count, int form, int64_t renorm_interval,
                        int slices, double target, int tune, mfcuda_batch **plan, bool complex) {
  using namespace mfcuda;
  if (!plan || count < 0 || (count > 0 && !descs)) return MFCUDA_ERR_INVALID_ARG;
  *plan = nullptr;
  if (form != MFCUDA_FORM_PLAIN && form != MFCUDA_FORM_SPLIT && form != MFCUDA_FORM_CRT)
    return MFCUDA_ERR_INVALID_ARG;
  if (form == MFCUDA_FORM_SPLIT && (slices < 0 || slices > split::SMAX || slices == 1 || !(target > 0.0)))
    return MFCUDA_ERR_INVALID_ARG;
  if (form == MFCUDA_FORM_CRT &&
      (slices < 0 || (slices > 0 && slices < 8) || slices > split::CRT_WMAX || !(target > 0.0)))
    return MFCUDA_ERR_INVALID_ARG;
  for (int64_t p = 0; p < count; ++p) {
    const mfcuda_gemm_desc &g = descs[p];
    if (g.m < 0 || g.k < 0 || g.n < 0 || !mul_ok(g.m, g.k) || !mul_ok(g.k, g.n) || !mul_ok(g.m, g.n))
      return MFCUDA_ERR_INVALID_ARG;
    if (g.m > 0 && g.n > 0 && (!g.c || (g.k > 0 && (!g.a || !g.b)))) return MFCUDA_ERR_INVALID_ARG;
  }
  MF_TRY(require_device());
  if (complex && form == MFCUDA_FORM_PLAIN)
    return batch::create_plain(descs, count, renorm_interval, std::vector<int>(count, 1), plan, true);
  std::vector<int> cfg = batch::choose(form, descs, count, tune, renorm_interval);
  if (form == MFCUDA_FORM_PLAIN) return batch::create_plain(descs, count, renorm_interval, cfg, plan);
  const bool crt = form == MFCUDA_FORM_CRT;
  int kcb = batch::choose_kcb(descs, count, cfg, complex ? 4 : 1, [&](int64_t k) {
    return crt ? split::crt_slices_max(k < 1 ? 1 : k, slices) : split::SMAX;
  });
  if (complex) return batch::create_csplit(descs, count, slices, target, cfg, kcb, plan, crt);
  return batch::create_split(descs, count, slices, target, cfg, kcb, plan, crt);
}

MULTIFLOATS_CUDA_API int mfcuda_batch_create_gemm(const mfcuda_gemm_desc *descs, int64_t count, int form,
                                                  int64_t renorm_interval, int slices, double target, int tune,
                                                  mfcuda_batch **plan) {
  return batch_create(descs, count, form, renorm_interval, slices, target, tune, plan, false);
}

MULTIFLOATS_CUDA_API int mfcuda_batch_create_cgemm(const mfcuda_gemm_desc *descs, int64_t count, int form,
                                                   int64_t renorm_interval, int slices, double target, int tune,
                                                   mfcuda_batch **plan) {
  return batch_create(descs, count, form, renorm_interval, slices, target, tune, plan, true);
}

MULTIFLOATS_CUDA_API int mfcuda_batch_create_unary(int op, const float64x2 *const *xs,
                                                   float64x2 *const *ys, const int64_t *ns, int64_t count,
                                                   mfcuda_batch **plan) {
  using namespace mfcuda;
  if (!plan || count < 0 || (count > 0 && (!xs || !ys || !ns))) return MFCUDA_ERR_INVALID_ARG;
  *plan = nullptr;
  if (op < MFCUDA_EXP || op > MFCUDA_SQRT || count > INT32_MAX) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  return batch::create_unary(op, xs, ys, ns, count, plan);
}

MULTIFLOATS_CUDA_API int mfcuda_batch_run(mfcuda_batch *plan, void *stream) {
  if (!plan || !plan->exec) return MFCUDA_ERR_INVALID_ARG;
  if (cudaGraphLaunch(plan->exec, mfcuda::as_stream(stream)) != cudaSuccess) {
    (void)cudaGetLastError();
    return MFCUDA_ERR_CUDA;
  }
  return MFCUDA_OK;
}

MULTIFLOATS_CUDA_API int mfcuda_batch_status(mfcuda_batch *plan) {
  if (!plan) return MFCUDA_ERR_INVALID_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) {
    (void)cudaGetLastError();
    return MFCUDA_ERR_CUDA;
  }
  if (plan->status) {
    int st = 0;
    if (cudaMemcpy(&st, plan->status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      return MFCUDA_ERR_CUDA;
    if (st) return MFCUDA_ERR_TIMEOUT;
  }
  return MFCUDA_OK;
}

MULTIFLOATS_CUDA_API int64_t mfcuda_batch_config(const mfcuda_batch *plan, int64_t i) {
  if (!plan || i < 0 || i >= (int64_t)plan->cfg.size()) return -1;
  if (plan->kind == 0) return mfcuda::batch::cfg_edge(plan->cfg[i]);
  return plan->cfg[i];
}

MULTIFLOATS_CUDA_API int64_t mfcuda_batch_work_items(const mfcuda_batch *plan) {
  return plan ? plan->work : -1;
}

MULTIFLOATS_CUDA_API int64_t mfcuda_batch_kchunk(const mfcuda_batch *plan) {
  return plan && plan->kind == 1 ? plan->kchunk : -1;
}

MULTIFLOATS_CUDA_API void mfcuda_batch_destroy(mfcuda_batch *plan) {
  if (plan) {
    cudaDeviceSynchronize();
    mfcuda::batch::destroy(plan);
  }
}

MULTIFLOATS_CUDA_API int mfcuda_unary_dd_ragged(int op, const float64x2 *const *xs, float64x2 *const *ys,
                                                const int64_t *ns, int64_t count, void *stream) {
  using namespace mfcuda;
  if (count < 0 || (count > 0 && (!xs || !ys || !ns))) return MFCUDA_ERR_INVALID_ARG;
  if (op < MFCUDA_EXP || op > MFCUDA_SQRT || count > INT32_MAX) return MFCUDA_ERR_INVALID_ARG;
  if (count == 0) return MFCUDA_OK;
  MF_TRY(require_device());
  std::vector<batch::RArr> tab;
  int64_t total;
  MF_TRY(batch::ragged_table(xs, ys, ns, count, tab, total));
  if (total == 0) return MFCUDA_OK;
  cudaStream_t s = as_stream(stream);
  void *dt = nullptr;
  MF_TRY(ws_alloc(&dt, sizeof(batch::RArr) * count, s));
  MF_TRY_CUDA(cudaMemcpyAsync(dt, tab.data(), sizeof(batch::RArr) * count, cudaMemcpyHostToDevice, s));
  // the host table must outlive the asynchronous copy
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) {
    batch::launch_ragged(op, static_cast<batch::RArr *>(dt), (int)count, total, s);
    e = cudaGetLastError();
  }
  ws_free(dt, s);
  return e == cudaSuccess ? MFCUDA_OK : MFCUDA_ERR_CUDA;
}

}  // extern "C"
