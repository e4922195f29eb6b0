// Split-INT8 double-double GEMM on tcgen05 tensor cores (no reference
// counterpart; it computes the same product as matmuldd_mm,
// src/float64x2/matmul.inc, to a stated error bound instead of bit for bit).
//
//   1. scan   : per row i of A and column j of B, the binade bound sigma_i /
//               tau_j (every |x| < 2^sigma) and the smallest binade mu of a
//               nonzero entry; non-finite entries are flagged.
//   2. plan   : slice count S (given, or the smallest S meeting the requested
//               bound for the measured exponent spreads), W = 8S-2 bits.
//   3. slice  : every DD entry is rounded to the grid of its row / column
//               (grid_round.cuh: |X - a 2^(W - sigma_i)| <= 1, |X| < 2^W) and cut into S
//               balanced signed 8-bit digits, most significant first:
//               X = sum_s d_s 256^(S-1-s), d_s in [-128, 127].  Slices are
//               stored K-major ([S][rows][K_pad] int8), zero-padded.
//   4. mma    : persistent tcgen05 kernel.  Work item = one anti-diagonal
//               g = s + t (0 <= g <= S-1) of one 128 x 256 output tile and one
//               K chunk: D_g = sum_{s+t=g} A_s B_t^T accumulated in INT32 in
//               tensor memory over K' = (g+1) K.  |d| <= 128 gives products
//               <= 2^14 and the K chunk keeps (g+1) K_chunk 2^14 < 2^31, so
//               the integer stage is exact.  Warp 0 issues TMA loads, one thread
//               of warp 1 issues the MMAs, warps 2-5 drain the accumulator to an
//               INT32 scratch ([g][kc][N_pad][M_pad]).  4-stage shared-memory
//               ring (48 KB per stage), two 256-column TMEM accumulators so the
//               drain of one item overlaps the MMAs of the next.  No multicast.
//   5. combine: C_ij = 2^(sigma_i + tau_j - 12) sum_kc sum_g D_g,kc 2^(-8g),
//               summed in DD chunk by chunk, each from the smallest diagonal
//               up, then scaled exactly.
//
// Error (a priori, per output):
//   |C - AB|_ij <= 2^-W (2^sigma_i sum_p |b_pj| + 2^tau_j sum_p |a_ip|)      (rounding of the operands,
//                                                                         at most one grid unit each)
//                + k S 2^(sigma_i + tau_j + 2 - 8S)                          (diagonals g >= S dropped)
//                + 2^-105 |C_ij|                                           (final DD rounding)
// (sums over the p whose other factor is nonzero; the products of two rounding
// errors add at most 2^(104 - 2W + rho_A + rho_B) / k in the units below).  With |a_ip| >= 2^(sigma_i - rho_A) and
// |b_pj| >= 2^(tau_j - rho_B) for nonzero entries and rho >= 1 this is at most
// (S+1) 2^(106 - 8S + rho_A + rho_B) times k 2^-104 (|A||B|)_ij, which is how
// the plan picks S for a target (S = 14 gives 15/16 for rho_A = rho_B = 1).
//
// The CRT form (crt_device.cuh) shares steps 1 and 3's rounding and the
// tensor-core kernels: residues modulo N moduli instead of digits, one product
// per modulus (u8 x u8), the epilogue reducing each INT32 sum to a residue
// byte, and a tensor-core reconstruction fed by TMA (crt_recon_kernel).  Large
// outputs run on CTA pairs (split_mma_pair_kernel, 256 x 512 tiles, eight
// epilogue warps); host-pointer CRT calls compute the output in column panels
// and copy each back while the next is computed (PanelSink).
#include <cudaTypedefs.h>

#include <mutex>
#include <vector>

#include "common.cuh"
#include "crt_device.cuh"
#include "dd_device.cuh"
#include "split_device.cuh"
#include "tcgen05.cuh"

namespace mfcuda {
namespace split {

// ---------------------------------------------------------------------------
// 1. scan
// ---------------------------------------------------------------------------
// ---- kernels of the single-problem pipeline (bodies in split_device.cuh) ----
__global__ void __launch_bounds__(256) scan_a_kernel(const double *__restrict__ A, int64_t M, int64_t K,
                                                     int64_t stride, int kchunk, int *sig, int *mu,
                                                     int *flag) {
  scan_a_body(A, M, K, stride, kchunk, sig, mu, flag, blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(256) scan_b_kernel(const double *__restrict__ B, int64_t K, int64_t N,
                                                     int64_t stride, int *sig, int *mu, int *flag) {
  scan_b_body(B, K, N, stride, sig, mu, flag, blockIdx.x, blockIdx.y);
}
// slices_dev (may be NULL): read the slice count there instead (ranks that
// agreed on one through a collective).
__global__ void plan_kernel(StatSet st, int slices, double target, Plan *plan, const int *slices_dev) {
  plan_body(st, slices_dev ? *slices_dev : slices, target, plan);
}
__global__ void __launch_bounds__(256) slice_a_kernel(const double *__restrict__ A, int64_t M, int64_t K,
                                                      int64_t stride, int64_t M_pad, int64_t K_pad,
                                                      const int *sig, const int *flag, const Plan *plan,
                                                      int8_t *__restrict__ As) {
  slice_a_body(A, M, K, stride, M_pad, K_pad, sig, flag, plan, As, blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(256) slice_b_kernel(const double *__restrict__ B, int64_t K, int64_t N,
                                                      int64_t stride, int64_t N_pad, int64_t K_pad,
                                                      const int *sig, const int *flag, const Plan *plan,
                                                      int8_t *__restrict__ Bs) {
  slice_b_body(B, K, N, stride, N_pad, K_pad, sig, flag, plan, Bs, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// 2. plan (one block)
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// 3. slice
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// 4. tcgen05 INT8 MMA, persistent
// ---------------------------------------------------------------------------
struct Item {
  int g, kc, tm, tn;
};
__device__ __forceinline__ Item decode(int w, int G, int nkc, int ntm, int ntiles) {
  Item it;
  int per_g = nkc * ntiles;
  it.g = G - w / per_g;  // heaviest diagonal first
  int r = w % per_g;
  it.kc = r / ntiles;
  int tile = r % ntiles;
  it.tm = tile % ntm;
  it.tn = tile / ntm;
  return it;
}

__global__ void __launch_bounds__(MMA_THREADS, 1)
    split_mma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     const Plan *plan, int32_t *__restrict__ D, int M_pad, int N_pad, int nkc,
                     int kblocks, int *status, uint64_t wait_ns) {
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
  const int S = plan->S, G = S - 1;
  const bool crt = plan->crt != 0;  // CRT form: item g is the single product A_g B_g
  const int ntm = M_pad / BM, ntn = N_pad / BN, ntiles = ntm * ntn;
  const int items = (G + 1) * nkc * ntiles;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mftc::mbar_init(&full[s], 1);
      mftc::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mftc::mbar_init(&tfull[a], 1);
      mftc::mbar_init(&tempty[a], 4);
    }
    mftc::mbar_init(drain, 1);
    *abort_flag = 0;
    mftc::fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    mftc::prefetch_tmap(&tmA);
    mftc::prefetch_tmap(&tmB);
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

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer ----
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int w = blockIdx.x; w < items && ok; w += gridDim.x) {
        Item it = decode(w, G, nkc, ntm, ntiles);
        int kb0 = it.kc * KC_BLOCKS, kb1 = min(kblocks, kb0 + KC_BLOCKS);
        for (int s = crt ? it.g : 0; s <= it.g && ok; ++s) {
          int t = crt ? s : it.g - s;
          for (int kb = kb0; kb < kb1; ++kb) {
            if (!wait_bar(&empty[stage], phase ^ 1, abort_flag, wait_ns)) {
              fail(1);
              ok = false;
              break;
            }
            mftc::mbar_arrive_expect_tx(&full[stage], STAGE);
            if (crt)  // MN-major residue planes: (row, K index, modulus)
              mftc::tma_load_3d(sA + stage * A_STAGE, &tmA, &full[stage], it.tm * BM, kb * BK, s);
            else
              mftc::tma_load_3d(sA + stage * A_STAGE, &tmA, &full[stage], kb * BK, it.tm * BM, s);
            mftc::tma_load_3d(sB + stage * B_STAGE, &tmB, &full[stage], kb * BK, it.tn * BN, t);
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
      // ---- MMA issuer ----
      // CRT residues are unsigned, and A's planes MN-major (a K step of 32 rows is 4096 bytes)
      const uint32_t idesc = crt ? mftc::idesc_u8(BM, BN) | mftc::IDESC_A_MN : mftc::idesc_i8(BM, BN);
      const uint32_t a_kstep = crt ? 32 * 128 : UMMA_K;
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      for (int w = blockIdx.x; w < items && ok; w += gridDim.x) {
        Item it = decode(w, G, nkc, ntm, ntiles);
        int kb0 = it.kc * KC_BLOCKS, kb1 = min(kblocks, kb0 + KC_BLOCKS);
        if (!wait_bar(&tempty[acc], acc_phase ^ 1, abort_flag, wait_ns)) {
          fail(2);
          break;
        }
        mftc::tc_fence_after();
        const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
        uint32_t accumulate = 0;
        for (int s = crt ? it.g : 0; s <= it.g && ok; ++s) {
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
      // every MMA issued by this thread has finished once `drain` flips
      mftc::umma_commit(drain);
      uint64_t t0 = globaltimer();
      while (!mftc::mbar_try_wait(drain, 0) && globaltimer() - t0 < WAIT_NS) {
      }
    }
  } else {
    // ---- epilogue: warps 2..5, TMEM lane quadrant = warp % 4 ----
    const int quad = warp & 3;
    const int row = quad * 32 + lane;
    int acc = 0;
    uint32_t acc_phase = 0;
    for (int w = blockIdx.x; w < items; w += gridDim.x) {
      Item it = decode(w, G, nkc, ntm, ntiles);
      bool got = wait_bar(&tfull[acc], acc_phase, abort_flag, wait_ns);
      if (!__all_sync(0xffffffffu, got)) {
        if (lane == 0) fail(8);
        break;
      }
      mftc::tc_fence_after();
      const int64_t off = ((int64_t)(it.g * nkc + it.kc) * N_pad + (int64_t)it.tn * BN) * M_pad +
                          (int64_t)it.tm * BM + row;
      const uint32_t tm_addr = tmem_base + ((uint32_t)(quad * 32) << 16) + (uint32_t)(acc * BN);
      if (crt) {  // residues modulo m_g, four columns per 32-bit word (crt_device.cuh)
        uint32_t *dst = reinterpret_cast<uint32_t *>(D) + crt_word_index(off, M_pad);
#pragma unroll 1
        for (int chunk = 0; chunk < BN / 32; ++chunk) {
          uint32_t r[32];
          mftc::tmem_ld_32x32b_x32(tm_addr + (uint32_t)(chunk * 32), r);
          mftc::tmem_wait_ld();
#pragma unroll
          for (int g = 0; g < 8; ++g) {
            __stcs(dst, crt_pack4(r[4 * g], r[4 * g + 1], r[4 * g + 2], r[4 * g + 3], it.g));
            dst += M_pad;
          }
        }
      } else {
        int32_t *dst = D + off;
#pragma unroll 1
        for (int chunk = 0; chunk < BN / 32; ++chunk) {
          uint32_t r[32];
          mftc::tmem_ld_32x32b_x32(tm_addr + (uint32_t)(chunk * 32), r);
          mftc::tmem_wait_ld();
#pragma unroll
          for (int q = 0; q < 32; ++q) {
            __stcs(dst, (int32_t)r[q]);  // evict-first: keep L2 for the slices
            dst += M_pad;
          }
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
    // an abort can leave copies in flight that no MMA consumed; they land
    // before the CTA's shared memory is released
    if (warp == 0 && lane == 0) arm.drain(full, NSTAGE);
    __syncthreads();
  }
  if (warp == 1) mftc::tmem_dealloc(tmem_base, TMEM_COLS);
}

// ---------------------------------------------------------------------------
// 4b. the same work on CTA pairs: 256 x 256 or 256 x 512 output tiles
// ---------------------------------------------------------------------------
// A cluster of two CTAs (neighbouring SMs) owns a 256 x (256 nsub) tile,
// nsub = 1 or 2.  Per pipeline stage each CTA loads its own 128 rows of the A
// slice and its own 128 rows (output columns) of each 256-column half of the
// B slice, and one thread of the even CTA issues, per K step, nsub M = 256,
// N = 256 MMAs that read both CTAs' shared memory; each CTA's tensor memory
// holds its 128 rows of the accumulator, and each CTA drains its own rows.
// Bytes loaded per SM per unit of tensor work: 2/3 (nsub = 1) or 1/2
// (nsub = 2) of the single-CTA kernel's, and the deeper ring in flight per
// byte of work hides more L2 / DRAM latency.  nsub = 1 keeps two 256-column
// accumulators (the drain of one item overlaps the next item's MMAs); nsub = 2
// uses all 512 columns for one accumulator, so the MMAs of the next item wait
// for the drain (~1% of an item's tensor time) while the loads run ahead.
//
// Barriers: every TMA load of both CTAs completes on the even CTA's full[s]
// (armed by the even CTA with both CTAs' bytes); each stage's MMAs are
// committed to empty[s] of both CTAs and each accumulator to tfull[a] of both
// CTAs (commit arrive fan-out, mask 0b11); the eight epilogue warps of the
// pair arrive on the even CTA's tempty[a].  All waits are bounded.
//
// Work is dealt in super-items of equal length: (q, K chunk, tile) runs the
// diagonal G-q and then the diagonal q of its tile ((G-q+1) + (q+1) = S+1
// slice products; a single diagonal when G-q == q).  Round r gives pair p the
// super-item r P + p of a q-major list, so all pairs start and finish their
// super-items together and, at any moment, multiply the same slice pair (s,
// t) of different tiles: the slices they read are shared through L2 instead
// of being fetched from DRAM once per pair.
// Threads of the pair kernel: warp 0 TMA, warp 1 MMA, warps 2-9 epilogue (two
// warps per TMEM lane quadrant, each draining half of the accumulator's
// columns, so the drain the next item's MMAs wait for takes half as long).
constexpr int PAIR_THREADS = 320;
constexpr int PAIR_EPI_WARPS = 8;
constexpr int P_STAGE_A = 128 * BK;  // 16 KiB: this CTA's 128 rows of A
constexpr int P_HALF_B = 128 * BK;   // 16 KiB: this CTA's 128 rows of one B half
constexpr int BM_PAIR = 256;
constexpr int PAIR_SMEM = 6 * (P_STAGE_A + P_HALF_B) + 1024 + 256;  // >= 4 * (16 + 32) KiB + extras

__host__ __device__ constexpr int pair_stages(int nsub) { return nsub == 1 ? 6 : 4; }

// Sequence of (diagonal, K chunk, tile) items of one pair (see above).
// Tiles are those of column tiles tn0 .. of the output (a column panel).
// In the CRT form every item is one product of equal length, so no pairing
// is needed: round r gives pair p item r P + p of a modulus-major list, and
// at any moment the pairs read the residue planes of at most two moduli
// (2 x 2 x 16.8 MB at 4096^3), which stay in L2 for all their tiles.
struct PairSched {
  int p, np, G, nkc, ntm, ntiles, tn0, nsuper;
  bool crt;
  int r = 0, half = 0;
  __device__ PairSched(int p_, int np_, int G_, int nkc_, int ntm_, int ntiles_, int tn0_, bool crt_)
      : p(p_), np(np_), G(G_), nkc(nkc_), ntm(ntm_), ntiles(ntiles_), tn0(tn0_),
        nsuper(crt_ ? (G_ + 1) * nkc_ * ntiles_ : ((G_ + 2) / 2) * nkc_ * ntiles_), crt(crt_) {}
  __device__ bool next(Item &it) {
    if (crt) {
      const int u = r * np + p;
      if (u >= nsuper) return false;
      ++r;
      const int per_g = nkc * ntiles;
      const int rem = u % per_g, tile = rem % ntiles;
      it.g = u / per_g;
      it.kc = rem / ntiles;
      it.tm = tile % ntm;
      it.tn = tn0 + tile / ntm;
      return true;
    }
    while (true) {
      const int u = r * np + p;
      if (u >= nsuper) return false;
      const int per_q = nkc * ntiles;
      const int q = u / per_q, rem = u % per_q;
      if (half == 1 && q == G - q) {  // the middle diagonal stands alone
        half = 0;
        ++r;
        continue;
      }
      it.g = half == 0 ? G - q : q;
      it.kc = rem / ntiles;
      const int tile = rem % ntiles;
      it.tm = tile % ntm;
      it.tn = tn0 + tile / ntm;
      if (half == 0) {
        half = 1;
      } else {
        half = 0;
        ++r;
      }
      return true;
    }
  }
};

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(PAIR_THREADS, 1)
    split_mma_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                          const Plan *plan, int32_t *__restrict__ D, int M_pad, int N_pad, int nkc,
                          int kblocks, int nsub, int tn0, int ntn, int *status, uint64_t wait_ns) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int nst = pair_stages(nsub);
  const int stage_b = nsub * P_HALF_B;
  const int stage_bytes = P_STAGE_A + stage_b;
  uint8_t *sA = smem;
  uint8_t *sB = smem + nst * P_STAGE_A;
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + nst * stage_bytes);
  uint64_t *empty = full + 6;
  uint64_t *tfull = empty + 6;
  uint64_t *tempty = tfull + 2;
  uint64_t *drain = tempty + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = mftc::cluster_rank();
  const bool leader = rank == 0;
  const int pair_id = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  const int S = plan->S, G = S - 1;
  const bool crt = plan->crt != 0;  // CRT form: item g is the single product A_g B_g
  const int tn_cols = BN * nsub;
  const int ntm = M_pad / BM_PAIR, ntiles = ntm * ntn;  // column tiles tn0 .. tn0 + ntn - 1
  const int nacc = 2 / nsub;             // accumulators
  const int acc_cols = BN * nsub;        // columns per accumulator

  if (threadIdx.x == 0) {
    for (int s = 0; s < nst; ++s) {
      mftc::mbar_init(&full[s], 1);
      mftc::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mftc::mbar_init(&tfull[a], 1);
      mftc::mbar_init(&tempty[a], 2 * PAIR_EPI_WARPS);  // every epilogue warp of both CTAs
    }
    mftc::mbar_init(drain, 1);
    *abort_flag = 0;
    mftc::fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    mftc::prefetch_tmap(&tmA);
    mftc::prefetch_tmap(&tmB);
  }
  if (warp == 1) {
    mftc::tmem_alloc_pair(tmem_slot, TMEM_COLS);
    mftc::tmem_relinquish_pair();
  }
  __syncwarp();
  mftc::tc_fence_before();
  mftc::cluster_sync();  // both CTAs' barriers are initialised before any cross-CTA signal
  mftc::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  // the peer CTA's abort flag (written before the closing cluster barrier,
  // while both CTAs are running): an abort in either CTA stops both
  const uint32_t peer_abort = mftc::cluster_addr((const void *)abort_flag, rank ^ 1u);
  auto fail = [&](int code) {
    *abort_flag = 1;
    mftc::st_cluster_u32(peer_abort, 1u);
    record_abort(status, code);
  };
  ArmedStages<6> arm;  // stages the even CTA's producer armed
  arm.clear();

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer (both CTAs) ----
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      PairSched sched(pair_id, npairs, G, nkc, ntm, ntiles, tn0, crt);
      Item it;
      while (ok && sched.next(it)) {
        int kb0 = it.kc * KC_BLOCKS, kb1 = min(kblocks, kb0 + KC_BLOCKS);
        const int arow = it.tm * BM_PAIR + (int)rank * 128;
        const int brow = it.tn * tn_cols + (int)rank * 128;
        for (int s = crt ? it.g : 0; s <= it.g && ok; ++s) {
          int t = crt ? s : it.g - s;
          for (int kb = kb0; kb < kb1; ++kb) {
            if (!wait_bar(&empty[stage], phase ^ 1, abort_flag, wait_ns)) {
              fail(1);
              ok = false;
              break;
            }
            if (leader) {
              mftc::mbar_arrive_expect_tx(&full[stage], 2 * stage_bytes);
              arm.arm(stage, phase);
            }
            const uint32_t fb = mftc::cluster_addr(&full[stage], 0);
            if (crt)  // MN-major residue planes: (row, K index, modulus)
              mftc::tma_load_3d_pair(sA + stage * P_STAGE_A, &tmA, fb, arow, kb * BK, s);
            else
              mftc::tma_load_3d_pair(sA + stage * P_STAGE_A, &tmA, fb, kb * BK, arow, s);
            for (int h = 0; h < nsub; ++h)
              mftc::tma_load_3d_pair(sB + stage * stage_b + h * P_HALF_B, &tmB, fb, kb * BK, brow + h * BN, t);
            if (++stage == nst) {
              stage = 0;
              phase ^= 1;
            }
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && leader) {
      // ---- MMA issuer (even CTA) ----
      // CRT residues are unsigned, and A's planes MN-major (a K step of 32 rows is 4096 bytes)
      const uint32_t idesc = crt ? mftc::idesc_u8(BM_PAIR, BN) | mftc::IDESC_A_MN : mftc::idesc_i8(BM_PAIR, BN);
      const uint64_t a_kstep = crt ? 32 * 128 / 16 : UMMA_K / 16;  // descriptor units of 16 bytes
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      PairSched sched(pair_id, npairs, G, nkc, ntm, ntiles, tn0, crt);
      Item it;
      // nsub = 2: one 512-column accumulator whose two 256-column halves are
      // handed back separately (tempty[0], tempty[1]).  The epilogue drains
      // half 0 first, so an item's half-0 MMAs start while half 1 of the
      // previous item still drains; the stages consumed meanwhile are held
      // (pend) and their half-1 MMAs issued, and the stages released in ring
      // order, as soon as half 1 is free -- at the latest when every stage of
      // the ring is held.
      int pend[6];
      int npend = 0;
      uint32_t acc1 = 0;
      auto half1 = [&](int st) {
        const uint64_t ad = mftc::smem_desc_k_sw128(mftc::smem_u32(sA + st * P_STAGE_A));
        const uint64_t bd = mftc::smem_desc_k_sw128(mftc::smem_u32(sB + st * stage_b));
#pragma unroll
        for (int kk = 0; kk < BK / UMMA_K; ++kk) {
          mftc::umma_i8_pair(tmem_base + (uint32_t)BN, ad + (uint64_t)kk * a_kstep,
                             bd + (uint64_t)((P_HALF_B + kk * UMMA_K) / 16), idesc, acc1);
          acc1 = 1;
        }
        mftc::umma_commit_pair(&empty[st], 0x3);
      };
      while (ok && nsub == 2 && sched.next(it)) {
        const int kb0 = it.kc * KC_BLOCKS, kb1 = min(kblocks, kb0 + KC_BLOCKS);
        if (!wait_bar(&tempty[0], acc_phase ^ 1, abort_flag, wait_ns)) {
          fail(2);
          break;
        }
        mftc::tc_fence_after();
        bool h1 = false;  // half 1 handed back for this item
        uint32_t acc0 = 0;
        acc1 = 0;
        auto catch_up = [&]() {
          for (int q = 0; q < npend; ++q) half1(pend[q]);
          npend = 0;
        };
        for (int s = crt ? it.g : 0; s <= it.g && ok; ++s) {
          for (int kb = kb0; kb < kb1; ++kb) {
            if (!h1 && npend == nst) {  // every stage held: half 1 first
              if (!wait_bar(&tempty[1], acc_phase ^ 1, abort_flag, wait_ns)) {
                fail(2);
                ok = false;
                break;
              }
              mftc::tc_fence_after();
              h1 = true;
              catch_up();
            }
            if (!wait_bar(&full[stage], phase, abort_flag, wait_ns)) {
              fail(4);
              ok = false;
              break;
            }
            mftc::tc_fence_after();
            const uint64_t ad0 = mftc::smem_desc_k_sw128(mftc::smem_u32(sA + stage * P_STAGE_A));
            const uint64_t bd0 = mftc::smem_desc_k_sw128(mftc::smem_u32(sB + stage * stage_b));
#pragma unroll
            for (int kk = 0; kk < BK / UMMA_K; ++kk) {
              mftc::umma_i8_pair(tmem_base, ad0 + (uint64_t)kk * a_kstep, bd0 + (uint64_t)(kk * UMMA_K / 16),
                                 idesc, acc0);
              acc0 = 1;
            }
            if (!h1 && mftc::mbar_test_wait(&tempty[1], acc_phase ^ 1)) {
              mftc::tc_fence_after();
              h1 = true;
              catch_up();
            }
            if (h1)
              half1(stage);
            else
              pend[npend++] = stage;
            if (++stage == nst) {
              stage = 0;
              phase ^= 1;
            }
          }
        }
        if (!ok) break;
        if (!h1) {
          if (!wait_bar(&tempty[1], acc_phase ^ 1, abort_flag, wait_ns)) {
            fail(2);
            break;
          }
          mftc::tc_fence_after();
          catch_up();
        }
        mftc::umma_commit_pair(&tfull[0], 0x3);
        acc_phase ^= 1;
      }
      while (ok && nsub == 1 && sched.next(it)) {
        int kb0 = it.kc * KC_BLOCKS, kb1 = min(kblocks, kb0 + KC_BLOCKS);
        if (!wait_bar(&tempty[acc], acc_phase ^ 1, abort_flag, wait_ns)) {
          fail(2);
          break;
        }
        mftc::tc_fence_after();
        const uint32_t d_tmem = tmem_base + (uint32_t)(acc * acc_cols);
        uint32_t accumulate = 0;
        for (int s = crt ? it.g : 0; s <= it.g && ok; ++s) {
          for (int kb = kb0; kb < kb1; ++kb) {
            if (!wait_bar(&full[stage], phase, abort_flag, wait_ns)) {
              fail(4);
              ok = false;
              break;
            }
            mftc::tc_fence_after();
            // stage descriptors built once; a K step or the second B half only moves
            // the start-address field (address / 16, far below its 14-bit limit)
            const uint64_t ad0 = mftc::smem_desc_k_sw128(mftc::smem_u32(sA + stage * P_STAGE_A));
            const uint64_t bd0 = mftc::smem_desc_k_sw128(mftc::smem_u32(sB + stage * stage_b));
#pragma unroll
            for (int kk = 0; kk < BK / UMMA_K; ++kk) {
              const uint64_t adesc = ad0 + (uint64_t)kk * a_kstep;
              mftc::umma_i8_pair(d_tmem, adesc, bd0 + (uint64_t)(kk * UMMA_K / 16), idesc, accumulate);
              accumulate = 1;
            }
            mftc::umma_commit_pair(&empty[stage], 0x3);
            if (++stage == nst) {
              stage = 0;
              phase ^= 1;
            }
          }
        }
        if (!ok) break;
        mftc::umma_commit_pair(&tfull[acc], 0x3);
        if (++acc == nacc) {
          acc = 0;
          acc_phase ^= 1;
        }
      }
      // every MMA issued by this thread has finished once `drain` flips; the
      // odd CTA is held by the closing cluster barrier until then
      mftc::umma_commit_pair(drain, 0x1);
      uint64_t t0 = globaltimer();
      while (!mftc::mbar_try_wait(drain, 0) && globaltimer() - t0 < WAIT_NS) {
      }
    }
  } else {
    // ---- epilogue: warps 2..9 of both CTAs, TMEM lane quadrant = warp % 4;
    // the two warps of a quadrant split each 256-column half of the
    // accumulator.  nsub = 2: half 0 is drained and handed back (tempty[0])
    // before half 1 (tempty[1]); nsub = 1: each accumulator is one half. ----
    const int quad = warp & 3;
    const int row = quad * 32 + lane;
    const int sel = (warp - 2) / 4;  // which 4 of a half's 8 32-column chunks
    int acc = 0;
    uint32_t acc_phase = 0;
    PairSched sched(pair_id, npairs, G, nkc, ntm, ntiles, tn0, crt);
    Item it;
    while (sched.next(it)) {
      bool got = wait_bar(&tfull[acc], acc_phase, abort_flag, wait_ns);
      if (!__all_sync(0xffffffffu, got)) {
        if (lane == 0) fail(8);
        break;
      }
      mftc::tc_fence_after();
      const int64_t off = ((int64_t)(it.g * nkc + it.kc) * N_pad + (int64_t)it.tn * tn_cols) * M_pad +
                          (int64_t)it.tm * BM_PAIR + (int64_t)rank * 128 + row;
      const uint32_t tm_addr = tmem_base + ((uint32_t)(quad * 32) << 16) + (uint32_t)(acc * acc_cols);
      // chunks [c0, c0 + 4) of the accumulator (32 columns each) to the scratch
      auto drain = [&](int c0) {
        if (crt) {  // residues modulo m_g, four columns per 32-bit word (crt_device.cuh)
          uint32_t *dst = reinterpret_cast<uint32_t *>(D) + crt_word_index(off, M_pad) + (int64_t)c0 * 8 * M_pad;
#pragma unroll 1
          for (int chunk = c0; chunk < c0 + 4; ++chunk) {
            uint32_t v[32];
            mftc::tmem_ld_32x32b_x32(tm_addr + (uint32_t)(chunk * 32), v);
            mftc::tmem_wait_ld();
#pragma unroll
            for (int g = 0; g < 8; ++g) {
              __stcs(dst, crt_pack4(v[4 * g], v[4 * g + 1], v[4 * g + 2], v[4 * g + 3], it.g));
              dst += M_pad;
            }
          }
        } else {
          int32_t *dst = D + off + (int64_t)c0 * 32 * M_pad;
#pragma unroll 1
          for (int chunk = c0; chunk < c0 + 4; ++chunk) {
            uint32_t v[32];
            mftc::tmem_ld_32x32b_x32(tm_addr + (uint32_t)(chunk * 32), v);
            mftc::tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 32; ++q) {
              __stcs(dst, (int32_t)v[q]);  // evict-first: keep L2 for the slices
              dst += M_pad;
            }
          }
        }
        mftc::tc_fence_before();
        __syncwarp();
      };
      if (nsub == 2) {
        drain(4 * sel);
        if (lane == 0) mftc::mbar_arrive_cluster(mftc::cluster_addr(&tempty[0], 0));
        drain(8 + 4 * sel);
        if (lane == 0) mftc::mbar_arrive_cluster(mftc::cluster_addr(&tempty[1], 0));
        acc_phase ^= 1;
      } else {
        drain(4 * sel);
        if (lane == 0) mftc::mbar_arrive_cluster(mftc::cluster_addr(&tempty[acc], 0));
        if (++acc == nacc) {
          acc = 0;
          acc_phase ^= 1;
        }
      }
    }
  }

  __syncwarp();
  mftc::tc_fence_before();
  mftc::cluster_sync();  // no CTA leaves while its peer may still signal it or read its shared memory
  mftc::tc_fence_after();
  // An abort in either CTA set both flags before the barrier: the flag read
  // after it has the same value in every thread of the pair.
  if (*abort_flag) {
    if (warp == 0 && lane == 0) {
      // copies in flight that no MMA consumed land before shared memory is
      // released: the even CTA waits for every stage it armed (both CTAs'
      // copies complete there); a copy the odd CTA issued for a stage the even
      // CTA gave up before arming completes on no barrier anyone waits for,
      // so both also give in-flight copies time to land (a 16 KiB tile takes
      // a few microseconds)
      if (leader) arm.drain(full, nst);
      settle_ns(50000);
    }
    __syncwarp();
    mftc::cluster_sync();
  }
  if (warp == 1) mftc::tmem_dealloc_pair(tmem_base, TMEM_COLS);
}

// ---------------------------------------------------------------------------
// 5. combine
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) combine_kernel(const int32_t *__restrict__ D, const Plan *plan,
                                                      const int *sigA, const int *flagA, const int *sigB,
                                                      const int *flagB, int64_t M, int64_t N,
                                                      int64_t M_pad, int64_t N_pad, int nkc,
                                                      double *__restrict__ C, int64_t cstride, int mode) {
  combine4_body(D, plan, sigA, flagA, sigB, flagB, M, N, M_pad, N_pad, nkc, C, cstride, mode,
                (int64_t)blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y);
}
constexpr int COMBINE_THREADS = 128;

// ---------------------------------------------------------------------------
// CRT form (crt_device.cuh): plan, residue slicing, reconstruction
// ---------------------------------------------------------------------------
// bits_dev (may be NULL): read the operand width there instead (ranks that
// agreed on one through a collective).
__global__ void crt_plan_kernel(StatSet st, int bits, double target, int64_t k, Plan *plan, CrtConst *cc,
                                const int *bits_dev) {
  crt_plan_body(st, bits_dev ? *bits_dev : bits, target, k, plan, cc);
}
// Block (x, y): column x (a K index) of A, rows 2048 y ..; MN-major planes.
__global__ void __launch_bounds__(256) crt_slice_a_kernel(const double *__restrict__ A, int64_t M, int64_t K,
                                                          int64_t stride, int64_t M_pad, int64_t K_pad,
                                                          const int *sig, const int *flag, const Plan *plan,
                                                          int8_t *__restrict__ As) {
  const int64_t i8 = ((int64_t)blockIdx.y * blockDim.x + threadIdx.x) * 8;
  if (i8 >= M_pad) return;
  crt_slice_a_mn_one(A, M, K, stride, M_pad, K_pad, sig, flag, plan, As, i8, blockIdx.x);
}
__global__ void __launch_bounds__(256) crt_slice_b_kernel(const double *__restrict__ B, int64_t K, int64_t N,
                                                          int64_t stride, int64_t N_pad, int64_t K_pad,
                                                          const int *sig, const int *flag, const Plan *plan,
                                                          int8_t *__restrict__ Bs, int64_t j0) {
  const int64_t p8 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 8;
  if (p8 >= K_pad) return;
  crt_slice_b_one(B, K, N, stride, N_pad, K_pad, sig, flag, plan, Bs, j0 + blockIdx.y, p8);  // column j0 + y
}
// Reconstruction fed by TMA (crt_recon_body): persistent, one CTA per SM;
// units of 32 rows x one column quad, rows below M, quads qbase .. (columns
// below N).  Dynamic shared memory cr_smem(ceil(moduli / 32)).
__global__ void __launch_bounds__(CR_THREADS, 1) crt_recon_kernel(
    const __grid_constant__ CUtensorMap tmD, const Plan *plan, const CrtConst *cc, const int *sigA,
    const int *flagA, const int *sigB, const int *flagB, int64_t M, int64_t N, int64_t qbase, int64_t nrb,
    int64_t units, int64_t k, double *__restrict__ C, int64_t cstride, int mode, int *status, uint64_t wait_ns) {
  extern __shared__ uint8_t cr_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(cr_raw) + 1023) & ~uintptr_t(1023));
  crt_recon_body(&tmD, plan, cc, sigA, flagA, sigB, flagB, M, N, qbase, nrb, units, k, C, cstride, mode, smem,
                 status, wait_ns);
}
// K chunks of the residue products folded into chunk 0 (block row y =
// modulus), words w0 .. w1 - 1 of each plane (the column quads of a panel:
// folding is not idempotent, so each word is folded once).
__global__ void __launch_bounds__(256) crt_fold_kernel(uint32_t *D, const Plan *plan, int nkc,
                                                       int64_t plane_words, int64_t w0, int64_t w1) {
  const int64_t w = w0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w < w1) crt_fold_body(D, plan, nkc, plane_words, (int)blockIdx.y, w);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// Workspace of one call with nA A-side operands (m x k) and nB B-side
// operands (k x n): per operand its exponent statistics and SMAX slices, one
// INT32 diagonal scratch shared by the products, the plan and a status word.
struct Layout {
  int64_t M_pad, N_pad, K_pad, kblocks, nkc;
  int nA, nB;
  int nsl;    // slices per operand allocated (digit slices, or CRT moduli)
  bool pair;  // 256 x (256 nsub) tiles on CTA pairs (m > 128), else 128 x 256 tiles
  int nsub;   // 256-column halves per pair tile: 2 when n > 256
  size_t off_plan, off_crt, off_stats[4], off_slices[4], off_D, total;
};

static int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// CTA pairs unless m fits one 128-row tile; MFCUDA_SPLIT_PAIR=0 selects the
// single-CTA kernel for every shape (same results, bit for bit).
static bool use_pair(int64_t m) {
  static const bool enabled = [] {
    const char *e = getenv("MFCUDA_SPLIT_PAIR");
    return !(e && e[0] == '0');
  }();
  return enabled && m > BM;
}

// Output columns per pair tile in 256-column halves (1 or 2; 2 halves the
// operand bytes per tensor op).  MFCUDA_SPLIT_NSUB=1 or 2 overrides.
static int pair_nsub() {
  static const int v = [] {
    const char *e = getenv("MFCUDA_SPLIT_NSUB");
    return (e && e[0] == '1') ? 1 : 2;
  }();
  return v;
}

static Layout layout(int64_t m, int64_t k, int64_t n, int nA, int nB, int nsl = SMAX, bool crt = false) {
  Layout L;
  L.nsl = nsl;
  L.pair = use_pair(m);
  L.nsub = L.pair && n > BN ? pair_nsub() : 1;
  L.M_pad = round_up(m < 1 ? 1 : m, L.pair ? BM_PAIR : BM);
  L.N_pad = round_up(n < 1 ? 1 : n, BN * L.nsub);
  L.K_pad = round_up(k < 1 ? 1 : k, BK);
  L.kblocks = L.K_pad / BK;
  L.nkc = (L.kblocks + KC_BLOCKS - 1) / KC_BLOCKS;
  L.nA = nA;
  L.nB = nB;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = (size_t)round_up((int64_t)(off + bytes), 1024);
    return o;
  };
  L.off_plan = take(sizeof(Plan));
  L.off_crt = take(sizeof(CrtConst));
  for (int o = 0; o < nA + nB; ++o) {
    int64_t rows = o < nA ? L.M_pad : L.N_pad;
    L.off_stats[o] = take(3 * sizeof(int) * rows);
    L.off_slices[o] = take((size_t)nsl * rows * L.K_pad);
  }
  // INT32 diagonal sums, or (CRT) one residue byte per output, modulus and K chunk
  L.off_D = take((size_t)nsl * L.nkc * L.N_pad * L.M_pad * (crt ? 1 : sizeof(int32_t)));
  L.total = off + 256 /* status word */;
  return L;
}

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
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
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
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// The residue scratch of the CRT form as the reconstruction's TMA source:
// bytes of (quad, rows) lines (4 M_pad per quad), quads, moduli (chunk 0 of
// each, nkc chunks apart); boxes of 128 bytes x 1 quad x 32 moduli with the
// 128-byte swizzle (planes beyond nsl read as zero).
static bool make_residue_map(CUtensorMap *map, void *D8, int64_t M_pad, int64_t N_pad, int64_t nkc, int nsl) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)(4 * M_pad), (cuuint64_t)(N_pad / 4), (cuuint64_t)nsl};
  cuuint64_t strides[2] = {(cuuint64_t)(4 * M_pad), (cuuint64_t)(nkc * N_pad * M_pad)};
  cuuint32_t box[3] = {128, 1, 32};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, D8, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Phase profiling (per host thread): while enabled, every call records five
// library-owned events on its stream -- before the scan, before the slicing,
// before and after the tensor-core kernel, after the recombination -- and
// mfcuda_phase_profile_end sums the four intervals over the recorded calls.
struct PhaseRec {
  cudaEvent_t ev[5];
};
static thread_local std::vector<PhaseRec> t_recs;
static thread_local size_t t_used = 0;
static thread_local bool t_prof = false;
static thread_local PhaseRec *t_cur = nullptr;
static void mark(int i, cudaStream_t s) {
  if (t_cur) cudaEventRecord(t_cur->ev[i], s);
}
static void prof_call_begin() {
  t_cur = nullptr;
  if (!t_prof) return;
  if (t_used == t_recs.size()) {
    PhaseRec r;
    for (int i = 0; i < 5; ++i)
      if (cudaEventCreate(&r.ev[i]) != cudaSuccess) return;
    t_recs.push_back(r);
  }
  t_cur = &t_recs[t_used++];
}
void profile_begin() {
  t_prof = true;
  t_used = 0;
}
int profile_end(double *sums, int64_t *calls) {
  t_prof = false;
  t_cur = nullptr;
  for (int i = 0; i < 4; ++i) sums[i] = 0.0;
  *calls = (int64_t)t_used;
  for (size_t c = 0; c < t_used; ++c) {
    if (cudaEventSynchronize(t_recs[c].ev[4]) != cudaSuccess) return MFCUDA_ERR_CUDA;
    for (int i = 0; i < 4; ++i) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, t_recs[c].ev[i], t_recs[c].ev[i + 1]) != cudaSuccess)
        return MFCUDA_ERR_CUDA;
      sums[i] += ms;
    }
  }
  t_used = 0;
  return MFCUDA_OK;
}

size_t workspace_size(int64_t m, int64_t k, int64_t n, bool complex_operands) {
  int no = complex_operands ? 2 : 1;
  return layout(m, k, n, no, no).total;
}
size_t crt_workspace_size(int64_t m, int64_t k, int64_t n, int bits, bool complex_operands) {
  int no = complex_operands ? 2 : 1;
  return layout(m, k, n, no, no, crt_slices_max(k, bits), true).total;
}

static std::once_flag g_attr_once;

// Persistent grid of the pair kernel: two CTAs per co-resident cluster.
static int pair_grid() {
  static int grid = [] {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * (unsigned)sm_count(), 1, 1);
    cfg.blockDim = dim3(PAIR_THREADS, 1, 1);
    cfg.dynamicSmemBytes = PAIR_SMEM;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, split_mma_pair_kernel, &cfg) != cudaSuccess || clusters < 1) {
      cudaGetLastError();
      clusters = sm_count() / 2;
    }
    return 2 * clusters;
  }();
  return grid;
}

// A product of one A-side operand with one B-side operand, written into a
// strided output view with the given mode (see combine_kernel).
struct Product {
  int a, b;
  double *out;
  int64_t ostride;
  int mode;
};

// Runs the whole split pipeline for `nprod` products of the operands
// A-side views (aview[o], stride astride[o]) and B-side views.  info (may be
// NULL) receives {S, rho_A, rho_B}; a non-NULL info waits for completion.
// crt = 1 runs the CRT form with `slices` read as the operand bits W (0 = from
// the target); info then receives {moduli, rho_A, rho_B, W}.
// A caller that takes the output in column panels (the host-pointer calls
// copy each panel to the host while later panels are computed): after every
// product of output columns [j0, j1) has been enqueued on stream s,
// done(ctx, j0, j1, s) is called.  Used by the CRT form on CTA pairs; other
// calls report the whole output as one panel.  Results are the same bit for
// bit for any panel count.
struct PanelSink {
  int panels;
  void (*done)(void *ctx, int64_t j0, int64_t j1, cudaStream_t s);
  void *ctx;
};
// Agreement between ranks that compute column panels of one product:
// fn(ctx, v, s) replaces the int at device address v (the plan's slice count
// or operand width) by its maximum over the ranks, enqueued on stream s;
// returns an MFCUDA status.
struct Agree {
  int (*fn)(void *ctx, int *v, cudaStream_t s);
  void *ctx;
};

static int run_products(const double *const *aview, const int64_t *astride, int nA,
                        const double *const *bview, const int64_t *bstride, int nB,
                        const Product *prods, int nprod, int64_t m, int64_t k, int64_t n, int slices,
                        double target, void *ws, size_t ws_bytes, cudaStream_t s, int *info, int crt = 0,
                        const PanelSink *sink = nullptr, const Agree *agree = nullptr) {
  Layout L = layout(m, k, n, nA, nB, crt ? crt_slices_max(k, slices) : SMAX, crt != 0);
  if (L.M_pad > INT32_MAX / 2 || L.N_pad > INT32_MAX / 2 || L.kblocks > INT32_MAX / 2 ||
      L.N_pad > 65535 || L.K_pad / 64 > 65535)
    return MFCUDA_ERR_UNSUPPORTED;
  void *own = nullptr;
  if (!ws) {
    MF_TRY(ws_alloc(&own, L.total, s));
    ws = own;
  } else if (ws_bytes < L.total) {
    return MFCUDA_ERR_WORKSPACE;
  }
  uint8_t *base = static_cast<uint8_t *>(ws);
  Plan *plan = reinterpret_cast<Plan *>(base + L.off_plan);
  CrtConst *cc = reinterpret_cast<CrtConst *>(base + L.off_crt);
  int32_t *D = reinterpret_cast<int32_t *>(base + L.off_D);
  int *status = reinterpret_cast<int *>(base + L.total - 256);
  const int nops = nA + nB;
  int *sig[4], *mu[4], *flag[4];
  int8_t *sl[4];
  for (int o = 0; o < nops; ++o) {
    int64_t rows = o < nA ? L.M_pad : L.N_pad;
    sig[o] = reinterpret_cast<int *>(base + L.off_stats[o]);
    mu[o] = sig[o] + rows;
    flag[o] = mu[o] + rows;
    sl[o] = reinterpret_cast<int8_t *>(base + L.off_slices[o]);
  }
  const uint64_t wait_ns = wait_limit_ns();
  int rc = MFCUDA_OK;
  do {
    std::call_once(g_attr_once, [] {
      cudaFuncSetAttribute(split_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, MMA_SMEM);
      cudaFuncSetAttribute(split_mma_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, PAIR_SMEM);
      cudaFuncSetAttribute(crt_recon_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           cr_smem((CRT_NMAX + 31) / 32));
    });
    prof_call_begin();
    mark(0, s);
    cudaMemsetAsync(status, 0, sizeof(int), s);
    const int kch = 64;
    StatSet st;
    st.n = nops;
    for (int o = 0; o < nops; ++o) {
      const bool aside = o < nA;
      int64_t rows = aside ? L.M_pad : L.N_pad;
      init_stats_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(sig[o], mu[o], flag[o], rows);
      if (aside)
        scan_a_kernel<<<dim3((unsigned)((m + 255) / 256), (unsigned)((k + kch - 1) / kch)), 256, 0, s>>>(
            aview[o], m, k, astride[o], kch, sig[o], mu[o], flag[o]);
      else
        scan_b_kernel<<<dim3((unsigned)((k + 2047) / 2048), (unsigned)n), 256, 0, s>>>(
            bview[o - nA], k, n, bstride[o - nA], sig[o], mu[o], flag[o]);
      st.sig[o] = sig[o];
      st.mu[o] = mu[o];
      st.count[o] = aside ? m : n;
      st.side[o] = aside ? 0 : 1;
    }
    if (crt)
      crt_plan_kernel<<<1, 1024, 0, s>>>(st, slices, target, k, plan, cc, nullptr);
    else
      plan_kernel<<<1, 1024, 0, s>>>(st, slices, target, plan, nullptr);
    if (agree) {
      // ranks holding other column panels of the same product agree on the
      // largest slice count / operand width (the one the single call would
      // pick from all of B) before anything depends on it
      int *val = crt ? &plan->W : &plan->S;
      rc = agree->fn(agree->ctx, val, s);
      if (rc != MFCUDA_OK) break;
      if (crt)
        crt_plan_kernel<<<1, 1024, 0, s>>>(st, slices, target, k, plan, cc, val);
      else
        plan_kernel<<<1, 1024, 0, s>>>(st, slices, target, plan, val);
    }
    mark(1, s);
    const dim3 ga((unsigned)(L.M_pad / 32), (unsigned)(L.K_pad / 64));
    const dim3 gb((unsigned)((L.K_pad / 8 + 255) / 256), (unsigned)L.N_pad);
    const dim3 gca((unsigned)L.K_pad, (unsigned)((L.M_pad / 8 + 255) / 256));
    // column panels (CRT form on CTA pairs, when a sink wants the output panel
    // by panel): B's residues, every product and the reconstruction of panel p,
    // then the sink, then panel p + 1
    const int tn_cols = BN * L.nsub;
    const int ntn_all = (int)(L.N_pad / tn_cols);
    const int npan = (sink && crt && L.pair) ? std::max(1, std::min(sink->panels, ntn_all)) : 1;
    for (int o = 0; o < nops; ++o) {
      if (o >= nA && npan > 1) continue;  // sliced panel by panel below
      if (o < nA && crt)
        crt_slice_a_kernel<<<gca, 256, 0, s>>>(aview[o], m, k, astride[o], L.M_pad, L.K_pad, sig[o], flag[o], plan,
                                               sl[o]);
      else if (o < nA)
        slice_a_kernel<<<ga, 256, 0, s>>>(aview[o], m, k, astride[o], L.M_pad, L.K_pad, sig[o], flag[o], plan,
                                          sl[o]);
      else if (crt)
        crt_slice_b_kernel<<<gb, 256, 0, s>>>(bview[o - nA], k, n, bstride[o - nA], L.N_pad, L.K_pad, sig[o],
                                              flag[o], plan, sl[o], 0);
      else
        slice_b_kernel<<<gb, 256, 0, s>>>(bview[o - nA], k, n, bstride[o - nA], L.N_pad, L.K_pad, sig[o],
                                          flag[o], plan, sl[o]);
    }
    const int tile_m = L.pair ? BM_PAIR : BM;
    int items_max = L.nsl * (int)L.nkc * (int)((L.M_pad / tile_m) * (L.N_pad / (BN * L.nsub)));
    int grid = sm_count();
    if (L.pair) {
      // super-items (pairs of diagonals) or, in the CRT form, single products of the largest plan
      const int supers_max = crt ? items_max
                                 : ((L.nsl + 1) / 2) * (int)L.nkc * (int)((L.M_pad / tile_m) * (L.N_pad / (BN * L.nsub)));
      grid = pair_grid();
      if (grid > 2 * supers_max) grid = 2 * supers_max;
    } else if (grid > items_max) {
      grid = items_max;
    }
    const unsigned cgx = (unsigned)(((m + 3) / 4 + COMBINE_THREADS - 1) / COMBINE_THREADS);
    mark(2, s);
    CUtensorMap tmA[4], tmB[4], tmD;
    if (crt && !make_residue_map(&tmD, D, L.M_pad, L.N_pad, L.nkc, L.nsl)) rc = MFCUDA_ERR_CUDA;
    for (int q = 0; q < nprod; ++q)
      if (!(crt ? make_map_mn(&tmA[q], sl[prods[q].a], L.M_pad, L.K_pad, L.nsl)
                : make_map(&tmA[q], sl[prods[q].a], L.M_pad, L.K_pad, BM, L.nsl)) ||
          !make_map(&tmB[q], sl[nA + prods[q].b], L.N_pad, L.K_pad, L.pair ? 128 : BN, L.nsl))
        rc = MFCUDA_ERR_CUDA;
    for (int pp = 0; pp < npan && rc == MFCUDA_OK; ++pp) {
      const int tn0 = (int)((int64_t)ntn_all * pp / npan), tn1 = (int)((int64_t)ntn_all * (pp + 1) / npan);
      const int64_t j0 = npan == 1 ? 0 : (int64_t)tn0 * tn_cols;
      const int64_t j1 = npan == 1 ? n : std::min<int64_t>(n, (int64_t)tn1 * tn_cols);
      if (npan > 1)  // this panel's columns of B (padding columns included)
        for (int o = nA; o < nops; ++o)
          crt_slice_b_kernel<<<dim3(gb.x, (unsigned)((tn1 - tn0) * tn_cols)), 256, 0, s>>>(
              bview[o - nA], k, n, bstride[o - nA], L.N_pad, L.K_pad, sig[o], flag[o], plan, sl[o],
              (int64_t)tn0 * tn_cols);
      int pgrid = grid;
      if (L.pair && npan > 1) {
        const int supers = (crt ? L.nsl : (L.nsl + 1) / 2) * (int)L.nkc * (int)(L.M_pad / tile_m) * (tn1 - tn0);
        pgrid = std::min(pair_grid(), 2 * supers);
      }
      for (int q = 0; q < nprod && rc == MFCUDA_OK; ++q) {
        const int ia = prods[q].a, ib = nA + prods[q].b;
        if (L.pair)
          split_mma_pair_kernel<<<pgrid, PAIR_THREADS, PAIR_SMEM, s>>>(
              tmA[q], tmB[q], plan, D, (int)L.M_pad, (int)L.N_pad, (int)L.nkc, (int)L.kblocks, L.nsub, tn0,
              npan == 1 ? ntn_all : tn1 - tn0, status, wait_ns);
        else
          split_mma_kernel<<<pgrid, MMA_THREADS, MMA_SMEM, s>>>(tmA[q], tmB[q], plan, D, (int)L.M_pad,
                                                                (int)L.N_pad, (int)L.nkc, (int)L.kblocks,
                                                                status, wait_ns);
        if (q == nprod - 1 && pp == npan - 1) mark(3, s);
        if (crt) {
          const int64_t q0 = j0 / 4, q1 = (j1 + 3) / 4, nrb = (m + 31) / 32, units = nrb * (q1 - q0);
          if (L.nkc > 1) {
            const int64_t plane_words = L.N_pad * L.M_pad / 4, nw = (q1 - q0) * L.M_pad;
            crt_fold_kernel<<<dim3((unsigned)((nw + 255) / 256), (unsigned)L.nsl), 256, 0, s>>>(
                reinterpret_cast<uint32_t *>(D), plan, (int)L.nkc, plane_words, q0 * L.M_pad, q1 * L.M_pad);
          }
          crt_recon_kernel<<<(unsigned)std::min<int64_t>(units, sm_count()), CR_THREADS, cr_smem((L.nsl + 31) / 32),
                             s>>>(tmD, plan, cc, sig[ia], flag[ia], sig[ib], flag[ib], m, j1, q0, nrb, units, k,
                                  prods[q].out, prods[q].ostride, prods[q].mode, status, wait_ns);
        } else
          combine_kernel<<<dim3(cgx, (unsigned)n), COMBINE_THREADS, 0, s>>>(
              D, plan, sig[ia], flag[ia], sig[ib], flag[ib], m, n, L.M_pad, L.N_pad, (int)L.nkc, prods[q].out,
              prods[q].ostride, prods[q].mode);
      }
      if (sink && rc == MFCUDA_OK) sink->done(sink->ctx, j0, j1, s);
    }
    mark(4, s);
    if (rc == MFCUDA_OK && cudaGetLastError() != cudaSuccess) rc = MFCUDA_ERR_CUDA;
    if (info && rc == MFCUDA_OK) {
      Plan hp;
      if (cudaMemcpyAsync(&hp, plan, sizeof(Plan), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess) {
        rc = MFCUDA_ERR_CUDA;
      } else {
        int stv = 0;
        cudaMemcpy(&stv, status, sizeof(int), cudaMemcpyDeviceToHost);
        if (stv) rc = MFCUDA_ERR_TIMEOUT;
        info[0] = hp.S;
        info[1] = hp.rho_a;
        info[2] = hp.rho_b;
        if (crt) info[3] = hp.W;
      }
    }
  } while (0);
  if (own) ws_free(own, s);
  return rc;
}

static int check_args(const void *a, const void *b, const void *c, int64_t m, int64_t k, int64_t n,
                      int slices, double target) {
  if (m < 0 || k < 0 || n < 0 || !mul_ok(m, k) || !mul_ok(k, n) || !mul_ok(m, n))
    return MFCUDA_ERR_INVALID_ARG;
  if (slices < 0 || slices > SMAX || slices == 1) return MFCUDA_ERR_INVALID_ARG;
  if (!(target > 0.0)) return MFCUDA_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return -1;  // nothing to do
  if (!c || (k > 0 && (!a || !b))) return MFCUDA_ERR_INVALID_ARG;
  if ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) | reinterpret_cast<uintptr_t>(c)) & 15)
    return MFCUDA_ERR_UNSUPPORTED;  // the split form wants 16-byte aligned operands
  return MFCUDA_OK;
}

int run(const float64x2 *a, const float64x2 *b, float64x2 *c, int64_t m, int64_t k, int64_t n,
        int slices, double target, void *ws, size_t ws_bytes, cudaStream_t s, int *info) {
  int rc = check_args(a, b, c, m, k, n, slices, target);
  if (rc == -1) return MFCUDA_OK;
  MF_TRY(rc);
  MF_TRY(require_device());
  if (k == 0) {
    MF_TRY_CUDA(cudaMemsetAsync(c, 0, (size_t)(m * n) * sizeof(float64x2), s));
    if (info) info[0] = info[1] = info[2] = 0;
    return MFCUDA_OK;
  }
  const double *av[1] = {reinterpret_cast<const double *>(a)};
  const double *bv[1] = {reinterpret_cast<const double *>(b)};
  int64_t one[1] = {1};
  Product p = {0, 0, reinterpret_cast<double *>(c), 1, 0};
  return run_products(av, one, 1, bv, one, 1, &p, 1, m, k, n, slices, target, ws, ws_bytes, s, info);
}

// CRT form of run(): bits = W (0: from the target); info = {moduli, rho_A, rho_B, W}.
int run_crt(const float64x2 *a, const float64x2 *b, float64x2 *c, int64_t m, int64_t k, int64_t n,
            int bits, double target, void *ws, size_t ws_bytes, cudaStream_t s, int *info,
            const PanelSink *sink = nullptr) {
  int rc = check_args(a, b, c, m, k, n, 0, target);
  if (bits < 0 || (bits > 0 && bits < 8) || bits > CRT_WMAX) return MFCUDA_ERR_INVALID_ARG;
  if (rc == -1) return MFCUDA_OK;
  MF_TRY(rc);
  MF_TRY(require_device());
  if (k == 0) {
    MF_TRY_CUDA(cudaMemsetAsync(c, 0, (size_t)(m * n) * sizeof(float64x2), s));
    if (info) info[0] = info[1] = info[2] = info[3] = 0;
    return MFCUDA_OK;
  }
  const double *av[1] = {reinterpret_cast<const double *>(a)};
  const double *bv[1] = {reinterpret_cast<const double *>(b)};
  int64_t one[1] = {1};
  Product p = {0, 0, reinterpret_cast<double *>(c), 1, 0};
  return run_products(av, one, 1, bv, one, 1, &p, 1, m, k, n, bits, target, ws, ws_bytes, s, info, 1, sink);
}

// One rank's column panel (n columns of B and C) of a real product computed
// by several ranks, which agree on the plan through `agree` before it is used
// (crt: the CRT form, arg = bits; else the digit-sliced form, arg = slices).
// k == 0 and m == 0 return before the agreement: every rank sees the same m
// and k, so every rank skips it alike.  n must be positive (a rank with an
// empty panel takes part in the agreement on its own).
int run_panel(bool crt, const float64x2 *a, const float64x2 *b, float64x2 *c, int64_t m, int64_t k, int64_t n,
              int arg, double target, void *ws, size_t ws_bytes, cudaStream_t s, int *info, const Agree *agree) {
  int rc = check_args(a, b, c, m, k, n, crt ? 0 : arg, target);
  if (crt && (arg < 0 || (arg > 0 && arg < 8) || arg > CRT_WMAX)) return MFCUDA_ERR_INVALID_ARG;
  if (rc == -1) return MFCUDA_OK;
  MF_TRY(rc);
  MF_TRY(require_device());
  if (k == 0) {
    MF_TRY_CUDA(cudaMemsetAsync(c, 0, (size_t)(m * n) * sizeof(float64x2), s));
    if (info) {
      info[0] = info[1] = info[2] = 0;
      if (crt) info[3] = 0;
    }
    return MFCUDA_OK;
  }
  const double *av[1] = {reinterpret_cast<const double *>(a)};
  const double *bv[1] = {reinterpret_cast<const double *>(b)};
  int64_t one[1] = {1};
  Product p = {0, 0, reinterpret_cast<double *>(c), 1, 0};
  return run_products(av, one, 1, bv, one, 1, &p, 1, m, k, n, arg, target, ws, ws_bytes, s, info, crt ? 1 : 0,
                      nullptr, agree);
}

// Complex: re = Ar Br - Ai Bi, im = Ar Bi + Ai Br (the Fortran cdd_matmul_mm
// composition, fsrc/multifloats.fypp:2609-2621), each real product in split form
// with one slice count S for all four; the four operands are sliced once.
int run_complex(const complex64x2 *a, const complex64x2 *b, complex64x2 *c, int64_t m, int64_t k,
                int64_t n, int slices, double target, void *ws, size_t ws_bytes, cudaStream_t s,
                int *info) {
  int rc = check_args(a, b, c, m, k, n, slices, target);
  if (rc == -1) return MFCUDA_OK;
  MF_TRY(rc);
  MF_TRY(require_device());
  if (k == 0) {
    MF_TRY_CUDA(cudaMemsetAsync(c, 0, (size_t)(m * n) * sizeof(complex64x2), s));
    if (info) info[0] = info[1] = info[2] = 0;
    return MFCUDA_OK;
  }
  const double *A = reinterpret_cast<const double *>(a);
  const double *B = reinterpret_cast<const double *>(b);
  double *Cd = reinterpret_cast<double *>(c);
  const double *av[2] = {A, A + 2};
  const double *bv[2] = {B, B + 2};
  int64_t two[2] = {2, 2};
  Product p[4] = {{0, 0, Cd, 2, 0},       // re  = Ar Br
                  {1, 1, Cd, 2, 1},       // re -= Ai Bi
                  {0, 1, Cd + 2, 2, 0},   // im  = Ar Bi
                  {1, 0, Cd + 2, 2, 2}};  // im += Ai Br
  return run_products(av, two, 2, bv, two, 2, p, 4, m, k, n, slices, target, ws, ws_bytes, s, info);
}

// Complex CRT form: the four real products of run_complex with one W and one
// moduli set for all four (planned from all four operands), the four parts
// reduced to residues once.
int run_complex_crt(const complex64x2 *a, const complex64x2 *b, complex64x2 *c, int64_t m, int64_t k,
                    int64_t n, int bits, double target, void *ws, size_t ws_bytes, cudaStream_t s, int *info,
                    const PanelSink *sink = nullptr) {
  int rc = check_args(a, b, c, m, k, n, 0, target);
  if (bits < 0 || (bits > 0 && bits < 8) || bits > CRT_WMAX) return MFCUDA_ERR_INVALID_ARG;
  if (rc == -1) return MFCUDA_OK;
  MF_TRY(rc);
  MF_TRY(require_device());
  if (k == 0) {
    MF_TRY_CUDA(cudaMemsetAsync(c, 0, (size_t)(m * n) * sizeof(complex64x2), s));
    if (info) info[0] = info[1] = info[2] = info[3] = 0;
    return MFCUDA_OK;
  }
  const double *A = reinterpret_cast<const double *>(a);
  const double *B = reinterpret_cast<const double *>(b);
  double *Cd = reinterpret_cast<double *>(c);
  const double *av[2] = {A, A + 2};
  const double *bv[2] = {B, B + 2};
  int64_t two[2] = {2, 2};
  Product p[4] = {{0, 0, Cd, 2, 0},       // re  = Ar Br
                  {1, 1, Cd, 2, 1},       // re -= Ai Bi
                  {0, 1, Cd + 2, 2, 0},   // im  = Ar Bi
                  {1, 0, Cd + 2, 2, 2}};  // im += Ai Br
  return run_products(av, two, 2, bv, two, 2, p, 4, m, k, n, bits, target, ws, ws_bytes, s, info, 1, sink);
}

}  // namespace split

namespace batch {
int wait_sticky_batched(bool clear);  // batched.cu
}

// MFCUDA_ERR_TIMEOUT when a tensor-core kernel of this file or of the
// grouped pipeline gave up a bounded wait on the current device.
static int timeout_status(bool clear) {
  MF_TRY(require_device());
  const int a = split::take_wait_sticky(clear), b = batch::wait_sticky_batched(clear);
  if (a < 0 || b < 0) return MFCUDA_ERR_CUDA;
  return (a | b) ? MFCUDA_ERR_TIMEOUT : MFCUDA_OK;
}

template <bool CPLX>
static int split_host(const void *a, const void *b, void *c, int64_t m, int64_t k, int64_t n, int slices,
                      double *bound_out) {
  const size_t elem = CPLX ? sizeof(complex64x2) : sizeof(float64x2);
  if (m < 0 || k < 0 || n < 0 || !mul_ok(m, k) || !mul_ok(k, n) || !mul_ok(m, n))
    return MFCUDA_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return MFCUDA_OK;
  if (!c || (k > 0 && (!a || !b))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  size_t ba = (size_t)(m * k) * elem, bb = (size_t)(k * n) * elem, bc = (size_t)(m * n) * elem;
  size_t wsb = split::workspace_size(m, k, n, CPLX);
  size_t sz[4] = {ba, bb, bc, wsb};
  Staging st;
  MF_TRY(staging_acquire(st, sz));
  if (ba) MF_TRY_CUDA(cudaMemcpyAsync(st.buf[0], a, ba, cudaMemcpyHostToDevice, st.stream));
  if (bb) MF_TRY_CUDA(cudaMemcpyAsync(st.buf[1], b, bb, cudaMemcpyHostToDevice, st.stream));
  int info[3] = {0, 0, 0};
  if (CPLX)
    MF_TRY(split::run_complex(static_cast<complex64x2 *>(st.buf[0]), static_cast<complex64x2 *>(st.buf[1]),
                              static_cast<complex64x2 *>(st.buf[2]), m, k, n, slices, 8.0, st.buf[3],
                              wsb, st.stream, info));
  else
    MF_TRY(split::run(static_cast<float64x2 *>(st.buf[0]), static_cast<float64x2 *>(st.buf[1]),
                      static_cast<float64x2 *>(st.buf[2]), m, k, n, slices, 8.0, st.buf[3], wsb,
                      st.stream, info));
  MF_TRY_CUDA(cudaMemcpyAsync(c, st.buf[2], bc, cudaMemcpyDeviceToHost, st.stream));
  MF_TRY_CUDA(cudaStreamSynchronize(st.stream));
  if (bound_out) {
    int S = info[0];
    *bound_out = S > 0 ? (S + 1) * ldexp(1.0, 106 - 8 * S + info[1] + info[2]) : 0.0;
  }
  return MFCUDA_OK;
}

// Device-to-host copies of the output, one per finished column panel, on the
// staging copy stream (each waits for its panel through an event).
struct PanelCopies {
  char *host;
  const char *dev;
  size_t col_bytes;  // bytes per output column
  cudaStream_t copy;
  cudaEvent_t *ev;
  int nev, used = 0;
  int64_t next = 0;  // columns [0, next) are on their way
  int rc = MFCUDA_OK;
};
static void copy_panel(void *ctx, int64_t j0, int64_t j1, cudaStream_t s) {
  auto *pc = static_cast<PanelCopies *>(ctx);
  if (pc->rc != MFCUDA_OK || j1 <= j0) return;
  cudaStream_t cs = s;
  if (pc->used < pc->nev) {  // otherwise copied on the compute stream itself
    cudaEvent_t e = pc->ev[pc->used++];
    if (cudaEventRecord(e, s) != cudaSuccess || cudaStreamWaitEvent(pc->copy, e, 0) != cudaSuccess) {
      pc->rc = MFCUDA_ERR_CUDA;
      return;
    }
    cs = pc->copy;
  }
  if (cudaMemcpyAsync(pc->host + j0 * pc->col_bytes, pc->dev + j0 * pc->col_bytes, (j1 - j0) * pc->col_bytes,
                      cudaMemcpyDeviceToHost, cs) != cudaSuccess)
    pc->rc = MFCUDA_ERR_CUDA;
  pc->next = j1;
}

// The host-pointer CRT call: operands copied in, the product computed in
// kPanels column panels, each panel copied back as soon as it is complete
// (overlapping the copy with the remaining panels' tensor-core work).
template <bool CPLX>
static int crt_host(const void *a, const void *b, void *c, int64_t m, int64_t k, int64_t n, int bits,
                    double *bound_out) {
  const size_t elem = CPLX ? sizeof(complex64x2) : sizeof(float64x2);
  if (m < 0 || k < 0 || n < 0 || !mul_ok(m, k) || !mul_ok(k, n) || !mul_ok(m, n))
    return MFCUDA_ERR_INVALID_ARG;
  if (bits < 0 || (bits > 0 && bits < 8) || bits > split::CRT_WMAX) return MFCUDA_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return MFCUDA_OK;
  if (!c || (k > 0 && (!a || !b))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  size_t ba = (size_t)(m * k) * elem, bb = (size_t)(k * n) * elem, bc = (size_t)(m * n) * elem;
  size_t wsb = split::crt_workspace_size(m, k, n, bits, CPLX);
  size_t sz[4] = {ba, bb, bc, wsb};
  Staging st;
  MF_TRY(staging_acquire(st, sz));
  if (ba) MF_TRY_CUDA(cudaMemcpyAsync(st.buf[0], a, ba, cudaMemcpyHostToDevice, st.stream));
  if (bb) MF_TRY_CUDA(cudaMemcpyAsync(st.buf[1], b, bb, cudaMemcpyHostToDevice, st.stream));
  int info[4] = {0, 0, 0, 0};
  PanelCopies pc;
  pc.host = static_cast<char *>(c);
  pc.dev = static_cast<const char *>(st.buf[2]);
  pc.col_bytes = (size_t)m * elem;
  pc.copy = st.copy;
  pc.ev = st.ev;
  pc.nev = kStagingEvents;
  constexpr int kPanels = 8;  // small panels: the first copy starts early (copy-bound call)
  const split::PanelSink sink = {kPanels, copy_panel, &pc};
  int rc;
  if (CPLX)
    rc = split::run_complex_crt(static_cast<complex64x2 *>(st.buf[0]), static_cast<complex64x2 *>(st.buf[1]),
                                static_cast<complex64x2 *>(st.buf[2]), m, k, n, bits, 8.0, st.buf[3], wsb,
                                st.stream, info, &sink);
  else
    rc = split::run_crt(static_cast<float64x2 *>(st.buf[0]), static_cast<float64x2 *>(st.buf[1]),
                        static_cast<float64x2 *>(st.buf[2]), m, k, n, bits, 8.0, st.buf[3], wsb, st.stream, info,
                        &sink);
  if (rc == MFCUDA_OK && pc.rc == MFCUDA_OK && pc.next < n)  // columns no panel reported (k = 0)
    copy_panel(&pc, pc.next, n, st.stream);
  // no copy may still be writing the caller's memory when this returns
  const cudaError_t e1 = cudaStreamSynchronize(st.stream), e2 = cudaStreamSynchronize(st.copy);
  MF_TRY(rc);
  MF_TRY(pc.rc);
  MF_TRY_CUDA(e1);
  MF_TRY_CUDA(e2);
  if (bound_out) *bound_out = info[0] > 0 ? split::crt_bound(info[3], info[1], info[2], k) : 0.0;
  return MFCUDA_OK;
}

}  // namespace mfcuda

extern "C" {

MULTIFLOATS_CUDA_API size_t mfcuda_crt_workspace_size(int64_t m, int64_t k, int64_t n, int bits) {
  if (m < 0 || k < 0 || n < 0 || bits < 0 || bits > mfcuda::split::CRT_WMAX) return 0;
  return mfcuda::split::crt_workspace_size(m, k, n, bits, false);
}
MULTIFLOATS_CUDA_API int mfcuda_matmuldd_mm_crt(const float64x2 *a, const float64x2 *b, float64x2 *c,
                                                int64_t m, int64_t k, int64_t n, int bits, double target,
                                                void *workspace, size_t workspace_bytes, int *info_out,
                                                void *stream) {
  return mfcuda::split::run_crt(a, b, c, m, k, n, bits, target, workspace, workspace_bytes,
                                mfcuda::as_stream(stream), info_out);
}
MULTIFLOATS_CUDA_API void matmuldd_mm_crt(const float64x2 *a, const float64x2 *b, float64x2 *c, int64_t m,
                                          int64_t k, int64_t n, int bits, double *max_err_bound_out) {
  mfcuda::set_last_error(mfcuda::crt_host<false>(a, b, c, m, k, n, bits, max_err_bound_out));
}
MULTIFLOATS_CUDA_API size_t mfcuda_ccrt_workspace_size(int64_t m, int64_t k, int64_t n, int bits) {
  if (m < 0 || k < 0 || n < 0 || bits < 0 || bits > mfcuda::split::CRT_WMAX) return 0;
  return mfcuda::split::crt_workspace_size(m, k, n, bits, true);
}
MULTIFLOATS_CUDA_API int mfcuda_cmatmuldd_mm_crt(const complex64x2 *a, const complex64x2 *b, complex64x2 *c,
                                                 int64_t m, int64_t k, int64_t n, int bits, double target,
                                                 void *workspace, size_t workspace_bytes, int *info_out,
                                                 void *stream) {
  return mfcuda::split::run_complex_crt(a, b, c, m, k, n, bits, target, workspace, workspace_bytes,
                                        mfcuda::as_stream(stream), info_out);
}
MULTIFLOATS_CUDA_API void cmatmuldd_mm_crt(const complex64x2 *a, const complex64x2 *b, complex64x2 *c,
                                           int64_t m, int64_t k, int64_t n, int bits,
                                           double *max_err_bound_out) {
  mfcuda::set_last_error(mfcuda::crt_host<true>(a, b, c, m, k, n, bits, max_err_bound_out));
}
MULTIFLOATS_CUDA_API double mfcuda_crt_bound(int bits, int rho_a, int rho_b, int64_t k) {
  if (bits < 8 || bits > mfcuda::split::CRT_WMAX || k < 1) return -1.0;
  return mfcuda::split::crt_bound(bits, rho_a, rho_b, k);
}

MULTIFLOATS_CUDA_API int mfcuda_timeout_status(int clear) { return mfcuda::timeout_status(clear != 0); }

MULTIFLOATS_CUDA_API void mfcuda_phase_profile_begin(void) { mfcuda::split::profile_begin(); }
MULTIFLOATS_CUDA_API int mfcuda_phase_profile_end(double *phase_ms_sum, int64_t *calls) {
  if (!phase_ms_sum || !calls) return MFCUDA_ERR_INVALID_ARG;
  return mfcuda::split::profile_end(phase_ms_sum, calls);
}

MULTIFLOATS_CUDA_API size_t mfcuda_split_workspace_size(int64_t m, int64_t k, int64_t n) {
  if (m < 0 || k < 0 || n < 0) return 0;
  return mfcuda::split::workspace_size(m, k, n, false);
}
MULTIFLOATS_CUDA_API size_t mfcuda_csplit_workspace_size(int64_t m, int64_t k, int64_t n) {
  if (m < 0 || k < 0 || n < 0) return 0;
  return mfcuda::split::workspace_size(m, k, n, true);
}
MULTIFLOATS_CUDA_API int mfcuda_cmatmuldd_mm_split(const complex64x2 *a, const complex64x2 *b,
                                                   complex64x2 *c, int64_t m, int64_t k, int64_t n,
                                                   int slices, double target, void *workspace,
                                                   size_t workspace_bytes, int *info_out,
                                                   void *stream) {
  return mfcuda::split::run_complex(a, b, c, m, k, n, slices, target, workspace, workspace_bytes,
                                    mfcuda::as_stream(stream), info_out);
}
MULTIFLOATS_CUDA_API void cmatmuldd_mm_split(const complex64x2 *a, const complex64x2 *b,
                                             complex64x2 *c, int64_t m, int64_t k, int64_t n,
                                             int slices, double *max_err_bound_out) {
  mfcuda::set_last_error(mfcuda::split_host<true>(a, b, c, m, k, n, slices, max_err_bound_out));
}

MULTIFLOATS_CUDA_API int mfcuda_matmuldd_mm_split(const float64x2 *a, const float64x2 *b,
                                                  float64x2 *c, int64_t m, int64_t k, int64_t n,
                                                  int slices, double target, void *workspace,
                                                  size_t workspace_bytes, int *info_out,
                                                  void *stream) {
  return mfcuda::split::run(a, b, c, m, k, n, slices, target, workspace, workspace_bytes,
                            mfcuda::as_stream(stream), info_out);
}

MULTIFLOATS_CUDA_API void matmuldd_mm_split(const float64x2 *a, const float64x2 *b, float64x2 *c,
                                            int64_t m, int64_t k, int64_t n, int slices,
                                            double *max_err_bound_out) {
  mfcuda::set_last_error(mfcuda::split_host<false>(a, b, c, m, k, n, slices, max_err_bound_out));
}

}  // extern "C"
