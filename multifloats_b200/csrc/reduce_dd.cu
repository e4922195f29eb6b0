// DD reductions: sum, dot_product, norm2 (real and complex).
//
// The reference has these only as Fortran generics (fsrc/multifloats.fypp):
//   dd_sum_1d      :1980-2019  Neumaier update, final fast two-sum
//   cdd_sum_1d     :2094-2158  same on re and im, final full two-sum
//   dd_dot_product :2254-2308  compensated update with cross = ah*bl + al*bh
//                              (two roundings), fast renorm after every block
//                              of renorm_interval elements including the last,
//                              final fast two-sum
//   cdd_dot_product:2321-2331  conj(a).b from four real dots + DD add/sub
//   dd_norm2_1d    :2338-2352  s = s + a*a with the DD operators, then sqrt
// All of them are serial loops.  On the device every thread g of a fixed grid
// of T threads runs exactly that serial update over its strided subsequence
// x[g], x[g+T], x[g+2T], ... ; the per-thread results are combined with the
// DD operator+ in a fixed tree (warp shuffle-down tree, then the warps of the
// block, then one final block over the block partials in the same pattern).
// The grid depends only on n (mfcuda_reduce_geometry), so results are
// reproducible run to run and across devices, and a CPU restatement of the
// same order reproduces them bit for bit.  Bound: HBM bandwidth.
#include "common.cuh"
#include "dd_device.cuh"

namespace mfcuda {

constexpr int kRThreads = 256;
constexpr int64_t kRMaxBlocks = 2048;
constexpr int64_t kRPerThreadMin = 16;

void reduce_geometry(int64_t n, int64_t *blocks, int64_t *threads) {
  int64_t per_block = kRThreads * kRPerThreadMin;
  int64_t b = (n + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > kRMaxBlocks) b = kRMaxBlocks;
  *blocks = b;
  *threads = kRThreads;
}

using mfdev::dd;
using mfdev::add;
using mfdev::sub;
using mfdev::mul;

// ---- per-element updates (Fortran semantics) -------------------------------
struct SumAcc {
  double hi = 0.0, lo = 0.0;
  __device__ __forceinline__ void step(double xh, double xl) {
    double t = add(hi, xh);
    double bp = sub(t, hi);
    double ap = sub(t, bp);
    double aerr = sub(hi, ap);
    double berr = sub(xh, bp);
    lo = add(lo, add(add(xl, aerr), berr));
    hi = t;
  }
  // real sum: fast two-sum (fypp:2004-2006)
  __device__ __forceinline__ dd finish_fast() const {
    double t = add(hi, lo);
    double bp = sub(t, hi);
    return mfdev::make(t, sub(lo, bp));
  }
  // complex sum: full two-sum (fypp:2143-2152)
  __device__ __forceinline__ dd finish_full() const {
    double t = add(hi, lo);
    double bp = sub(t, hi);
    double ap = sub(t, bp);
    double aerr = sub(hi, ap);
    double berr = sub(lo, bp);
    return mfdev::make(t, add(aerr, berr));
  }
};

struct DotAcc {
  double hi = 0.0, lo = 0.0;
  __device__ __forceinline__ void step(double ah, double al, double bh, double bl) {
    double p = mul(ah, bh);
    double e = mfdev::fma_(ah, bh, -p);
    double cross = add(mul(ah, bl), mul(al, bh));
    double t = add(hi, p);
    double bp = sub(t, hi);
    double ap = sub(t, bp);
    double aerr = sub(hi, ap);
    double berr = sub(p, bp);
    lo = add(lo, add(add(add(e, cross), aerr), berr));
    hi = t;
  }
  __device__ __forceinline__ void block_renorm() {
    double t = add(hi, lo);
    double bp = sub(t, hi);
    hi = t;
    lo = sub(lo, bp);
  }
  __device__ __forceinline__ dd finish() const {
    double t = add(hi, lo);
    double bp = sub(t, hi);
    return mfdev::make(t, sub(lo, bp));
  }
};

// ---- fixed-order combine -----------------------------------------------------
__device__ __forceinline__ dd shfl_down_dd(dd v, int off) {
  dd r;
  r.hi = __shfl_down_sync(0xffffffffu, v.hi, off);
  r.lo = __shfl_down_sync(0xffffffffu, v.lo, off);
  return r;
}
// Reduce NV values per thread over the block; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_combine(dd (&v)[NV]) {
  __shared__ dd warp_part[kRThreads / 32][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1)
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      dd o = shfl_down_dd(v[q], off);
      if (lane < off) v[q] = mfdev::dd_add(v[q], o);
    }
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) warp_part[warp][q] = v[q];
  __syncthreads();
  if (warp == 0) {
    constexpr int NW = kRThreads / 32;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = lane < NW ? warp_part[lane][q] : mfdev::make(0.0, 0.0);
#pragma unroll
    for (int off = NW / 2; off >= 1; off >>= 1)
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        dd o = shfl_down_dd(v[q], off);
        if (lane < off) v[q] = mfdev::dd_add(v[q], o);
      }
  }
}

// KIND: 0 sum, 1 dot, 2 norm2, 3 csum, 4 cdot, 5 cnorm2.
template <int KIND>
struct KindInfo;
template <> struct KindInfo<0> { static constexpr int NV = 1, ELEM = 2; };
template <> struct KindInfo<1> { static constexpr int NV = 1, ELEM = 2; };
template <> struct KindInfo<2> { static constexpr int NV = 1, ELEM = 2; };
template <> struct KindInfo<3> { static constexpr int NV = 2, ELEM = 4; };
template <> struct KindInfo<4> { static constexpr int NV = 4, ELEM = 4; };
template <> struct KindInfo<5> { static constexpr int NV = 1, ELEM = 4; };

// Stage 1: per-thread serial update over the strided subsequence, block tree,
// one partial (NV DD values) per block.
template <int KIND, bool ALIGNED>
__global__ void __launch_bounds__(kRThreads) reduce_stage1(const double *__restrict__ x,
                                                           const double *__restrict__ y,
                                                           int64_t n, int64_t ri,
                                                           dd *__restrict__ partials) {
  constexpr int NV = KindInfo<KIND>::NV;
  constexpr int E = KindInfo<KIND>::ELEM;  // doubles per element
  const int64_t T = (int64_t)gridDim.x * blockDim.x;
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;

  auto ld2 = [&](const double *p, int64_t i, int part) -> double2 {
    const double *q = p + E * i + 2 * part;
    if constexpr (ALIGNED) return __ldcs(reinterpret_cast<const double2 *>(q));
    return make_double2(q[0], q[1]);
  };

  dd v[NV];
  if constexpr (KIND == 0 || KIND == 3) {
    SumAcc s[NV];
    for (int64_t i = g; i < n; i += T) {
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        double2 a = ld2(x, i, q);
        s[q].step(a.x, a.y);
      }
    }
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = (KIND == 0) ? s[q].finish_fast() : s[q].finish_full();
  } else if constexpr (KIND == 1 || KIND == 4) {
    DotAcc d[NV];
    int64_t cnt = 0;
    for (int64_t i = g; i < n; i += T) {
      if constexpr (KIND == 1) {
        double2 a = ld2(x, i, 0), b = ld2(y, i, 0);
        d[0].step(a.x, a.y, b.x, b.y);
      } else {
        double2 ar = ld2(x, i, 0), ai = ld2(x, i, 1);
        double2 br = ld2(y, i, 0), bi = ld2(y, i, 1);
        d[0].step(ar.x, ar.y, br.x, br.y);  // re.re
        d[1].step(ai.x, ai.y, bi.x, bi.y);  // im.im
        d[2].step(ar.x, ar.y, bi.x, bi.y);  // re.im
        d[3].step(ai.x, ai.y, br.x, br.y);  // im.re
      }
      if (ri > 0 && ++cnt == ri) {
        cnt = 0;
#pragma unroll
        for (int q = 0; q < NV; ++q) d[q].block_renorm();
      }
    }
    // the last, partial block is renormalised too (fypp:2301-2302)
    if (ri > 0 && cnt > 0)
#pragma unroll
      for (int q = 0; q < NV; ++q) d[q].block_renorm();
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = d[q].finish();
  } else {
    dd s = mfdev::make(0.0, 0.0);
    for (int64_t i = g; i < n; i += T) {
      double2 a = ld2(x, i, 0);
      dd ad = mfdev::make(a.x, a.y);
      s = mfdev::dd_add(s, mfdev::dd_mul(ad, ad));
      if constexpr (KIND == 5) {
        double2 b = ld2(x, i, 1);
        dd bd = mfdev::make(b.x, b.y);
        s = mfdev::dd_add(s, mfdev::dd_mul(bd, bd));
      }
    }
    v[0] = s;
  }
  block_combine<NV>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) partials[(int64_t)blockIdx.x * NV + q] = v[q];
}

// The final step of each kind, applied to the fully combined NV values.
template <int KIND>
__device__ __forceinline__ void finish_kind(const dd *v, dd *out) {
  if constexpr (KIND == 0 || KIND == 1) {
    out[0] = v[0];
  } else if constexpr (KIND == 2 || KIND == 5) {
    out[0] = mfdev::dd_sqrt(v[0]);
  } else if constexpr (KIND == 3) {
    out[0] = v[0];
    out[1] = v[1];
  } else {
    out[0] = mfdev::dd_add(v[0], v[1]);  // re = rr + ii
    out[1] = mfdev::dd_sub(v[2], v[3]);  // im = ri - ir
  }
}

// Stage 2: one block folds the block partials (thread t: p[t], p[t+256], ...
// in order with DD add), same tree, then the final combination (FINAL) or the
// NV combined values themselves (a partial for a later cross-device combine).
template <int KIND, bool FINAL = true>
__global__ void __launch_bounds__(kRThreads) reduce_stage2(const dd *__restrict__ partials,
                                                           int64_t nblocks, dd *__restrict__ out) {
  constexpr int NV = KindInfo<KIND>::NV;
  dd v[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = mfdev::make(0.0, 0.0);
  for (int64_t b = threadIdx.x; b < nblocks; b += blockDim.x) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      dd p = partials[b * NV + q];
      v[q] = (b == threadIdx.x) ? p : mfdev::dd_add(v[q], p);
    }
  }
  block_combine<NV>(v);
  if (threadIdx.x == 0) {
    if constexpr (FINAL) {
      finish_kind<KIND>(v, out);
    } else {
#pragma unroll
      for (int q = 0; q < NV; ++q) out[q] = v[q];
    }
  }
}

// Cross-device combine: the partials of `count` devices (NV values each, in
// rank order) folded left to right with DD add, then the final step.
template <int KIND>
__global__ void combine_ranks_kernel(const dd *__restrict__ parts, int64_t count, dd *__restrict__ out) {
  constexpr int NV = KindInfo<KIND>::NV;
  dd v[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = parts[q];
  for (int64_t r = 1; r < count; ++r)
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = mfdev::dd_add(v[q], parts[r * NV + q]);
  finish_kind<KIND>(v, out);
}

size_t reduce_ws_size(int64_t n) {
  int64_t b, t;
  reduce_geometry(n < 0 ? 0 : n, &b, &t);
  return (size_t)b * 4 * sizeof(dd);
}

template <int KIND, bool FINAL = true>
static int reduce_dev(const double *x, const double *y, int64_t n, int64_t ri, void *out,
                      void *ws, size_t ws_bytes, cudaStream_t s) {
  constexpr int E = KindInfo<KIND>::ELEM;
  if (!size_ok(n, E * sizeof(double))) return MFCUDA_ERR_INVALID_ARG;
  if (!out || (n > 0 && (!x || ((KIND == 1 || KIND == 4) && !y)))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  int64_t blocks, threads;
  reduce_geometry(n, &blocks, &threads);
  size_t need = reduce_ws_size(n);
  void *own = nullptr;
  if (!ws) {
    MF_TRY(ws_alloc(&own, need, s));
    ws = own;
  } else if (ws_bytes < need) {
    return MFCUDA_ERR_WORKSPACE;
  }
  bool aligned = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
  dd *part = static_cast<dd *>(ws);
  if (aligned)
    reduce_stage1<KIND, true><<<(unsigned)blocks, (unsigned)threads, 0, s>>>(x, y, n, ri, part);
  else
    reduce_stage1<KIND, false><<<(unsigned)blocks, (unsigned)threads, 0, s>>>(x, y, n, ri, part);
  cudaError_t e1 = cudaGetLastError();
  if (e1 == cudaSuccess) {
    reduce_stage2<KIND, FINAL><<<1, kRThreads, 0, s>>>(part, blocks, static_cast<dd *>(out));
    e1 = cudaGetLastError();
  }
  if (own) ws_free(own, s);
  if (e1 != cudaSuccess) return MFCUDA_ERR_CUDA;
  return MFCUDA_OK;
}

// Host-pointer form: inputs copied to staging, result copied back.
template <int KIND>
static int reduce_host(const void *x, const void *y, int64_t n, int64_t ri, void *result) {
  constexpr int E = KindInfo<KIND>::ELEM;
  if (!size_ok(n, E * sizeof(double))) return MFCUDA_ERR_INVALID_ARG;
  if (n > 0 && (!x || ((KIND == 1 || KIND == 4) && !y))) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  size_t bx = (size_t)n * E * sizeof(double);
  size_t by = (KIND == 1 || KIND == 4) ? bx : 0;
  size_t ws = reduce_ws_size(n);
  size_t sz[4] = {bx, by, ws, 64};
  Staging st;
  MF_TRY(staging_acquire(st, sz));
  if (bx) MF_TRY_CUDA(cudaMemcpyAsync(st.buf[0], x, bx, cudaMemcpyHostToDevice, st.stream));
  if (by) MF_TRY_CUDA(cudaMemcpyAsync(st.buf[1], y, by, cudaMemcpyHostToDevice, st.stream));
  MF_TRY(reduce_dev<KIND>(static_cast<const double *>(st.buf[0]),
                          static_cast<const double *>(st.buf[1]), n, ri, st.buf[3], st.buf[2], ws,
                          st.stream));
  size_t rbytes = (KIND == 3 || KIND == 4) ? 2 * sizeof(dd) : sizeof(dd);
  MF_TRY_CUDA(cudaMemcpyAsync(result, st.buf[3], rbytes, cudaMemcpyDeviceToHost, st.stream));
  MF_TRY_CUDA(cudaStreamSynchronize(st.stream));
  return MFCUDA_OK;
}

// Kind-dispatched partial and cross-device combine.
static int reduce_partial(int kind, const double *x, const double *y, int64_t n, int64_t ri, void *out,
                          void *ws, size_t wsb, cudaStream_t s) {
  switch (kind) {
    case 0: return reduce_dev<0, false>(x, nullptr, n, 0, out, ws, wsb, s);
    case 1: return reduce_dev<1, false>(x, y, n, ri, out, ws, wsb, s);
    case 2: return reduce_dev<2, false>(x, nullptr, n, 0, out, ws, wsb, s);
    case 3: return reduce_dev<3, false>(x, nullptr, n, 0, out, ws, wsb, s);
    case 4: return reduce_dev<4, false>(x, y, n, ri, out, ws, wsb, s);
    case 5: return reduce_dev<5, false>(x, nullptr, n, 0, out, ws, wsb, s);
    default: return MFCUDA_ERR_INVALID_ARG;
  }
}
static int partial_values(int kind) {
  switch (kind) {
    case 0: return KindInfo<0>::NV;
    case 1: return KindInfo<1>::NV;
    case 2: return KindInfo<2>::NV;
    case 3: return KindInfo<3>::NV;
    case 4: return KindInfo<4>::NV;
    case 5: return KindInfo<5>::NV;
    default: return 0;
  }
}
static int reduce_combine(int kind, const void *parts, int64_t count, void *out, cudaStream_t s) {
  if (kind < 0 || kind > 5 || count < 1 || !parts || !out) return MFCUDA_ERR_INVALID_ARG;
  MF_TRY(require_device());
  const dd *p = static_cast<const dd *>(parts);
  dd *o = static_cast<dd *>(out);
  switch (kind) {
    case 0: combine_ranks_kernel<0><<<1, 1, 0, s>>>(p, count, o); break;
    case 1: combine_ranks_kernel<1><<<1, 1, 0, s>>>(p, count, o); break;
    case 2: combine_ranks_kernel<2><<<1, 1, 0, s>>>(p, count, o); break;
    case 3: combine_ranks_kernel<3><<<1, 1, 0, s>>>(p, count, o); break;
    case 4: combine_ranks_kernel<4><<<1, 1, 0, s>>>(p, count, o); break;
    default: combine_ranks_kernel<5><<<1, 1, 0, s>>>(p, count, o); break;
  }
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

static float64x2 nan_dd() {
  float64x2 r;
  r.limbs[0] = __builtin_nan("");
  r.limbs[1] = 0.0;
  return r;
}

// ---- dot product that allocates nothing --------------------------------------
// Some callers cannot let a library call cudaMalloc: a host application that
// hands the whole GPU memory to its own pool and forbids allocations behind
// its back, or code on a latency-critical path where cudaMalloc / cudaFree
// would synchronise the device.  mfcuda_dotdd_noalloc serves them with the
// block partials of the reduction kept in this fixed device array (16 KiB,
// held by every GPU that loads the library until the process exits).  The
// array holds kNoAllocMaxPartials partials, which limits n to
// kNoAllocMaxPartials * 4096 elements (the launch geometry gives one partial
// per 4096 elements).
constexpr int64_t kNoAllocMaxPartials = 1024;
static __device__ __align__(256) dd g_noalloc_partials[kNoAllocMaxPartials];

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static void *g_noalloc_addr[kNoAllocMaxDevices];

// Device address of g_noalloc_partials on the current device.  In host code
// the array's name only stands in for the symbol, so the address is looked up
// with the device current.  Outside stream capture it is looked up on every
// call (a cheap query), so an address cached before a cudaDeviceReset or the
// re-creation of the primary context is never reused; inside a capture the
// address cached by an earlier call on this device is used (the first call
// on a device must therefore come before any capture).
static int noalloc_scratch(void **p, cudaStream_t s) {
  int dev = 0;
  MF_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return MFCUDA_ERR_NO_DEVICE;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {  // e.g. the legacy stream while another captures
    (void)cudaGetLastError();
    cap = cudaStreamCaptureStatusActive;  // treat as capturing: no query, the cached address
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (cap == cudaStreamCaptureStatusNone || !g_noalloc_addr[dev]) {
    void *addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_partials);
    if (e != cudaSuccess || !addr) {
      (void)cudaGetLastError();
      return MFCUDA_ERR_CUDA;
    }
    g_noalloc_addr[dev] = addr;
  }
  *p = g_noalloc_addr[dev];
  return MFCUDA_OK;
}

static int dot_noalloc(const double *x, const double *y, int64_t n, int64_t ri, float64x2 *out,
                       cudaStream_t s) {
  if (!size_ok(n, 2 * sizeof(double))) return MFCUDA_ERR_INVALID_ARG;
  if (!out || (n > 0 && (!x || !y))) return MFCUDA_ERR_INVALID_ARG;
  int64_t blocks, threads;
  reduce_geometry(n, &blocks, &threads);
  if (blocks > kNoAllocMaxPartials) return MFCUDA_ERR_UNSUPPORTED;
  MF_TRY(require_device());
  void *scratch = nullptr;
  MF_TRY(noalloc_scratch(&scratch, s));
  // Every partial slot [0, blocks) is written by stage 1 before stage 2 reads
  // it, so the contents left by an earlier call never leak into this one.
  dd *part = static_cast<dd *>(scratch);
  bool aligned = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
  if (aligned)
    reduce_stage1<1, true><<<(unsigned)blocks, (unsigned)threads, 0, s>>>(x, y, n, ri, part);
  else
    reduce_stage1<1, false><<<(unsigned)blocks, (unsigned)threads, 0, s>>>(x, y, n, ri, part);
  MF_TRY_CUDA(cudaGetLastError());
  reduce_stage2<1><<<1, kRThreads, 0, s>>>(part, blocks, reinterpret_cast<dd *>(out));
  MF_TRY_CUDA(cudaGetLastError());
  return MFCUDA_OK;
}

}  // namespace mfcuda

extern "C" {

MULTIFLOATS_CUDA_API void mfcuda_reduce_geometry(int64_t n, int64_t *blocks, int64_t *threads) {
  mfcuda::reduce_geometry(n < 0 ? 0 : n, blocks, threads);
}
MULTIFLOATS_CUDA_API size_t mfcuda_reduce_workspace_size(int64_t n) {
  return mfcuda::reduce_ws_size(n);
}

#define MF_D(p) reinterpret_cast<const double *>(p)
MULTIFLOATS_CUDA_API int mfcuda_sumdd(const float64x2 *x, int64_t n, float64x2 *out, void *ws,
                                      size_t wsb, void *stream) {
  return mfcuda::reduce_dev<0>(MF_D(x), nullptr, n, 0, out, ws, wsb, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_dotdd(const float64x2 *a, const float64x2 *b, int64_t n, int64_t ri,
                                      float64x2 *out, void *ws, size_t wsb, void *stream) {
  return mfcuda::reduce_dev<1>(MF_D(a), MF_D(b), n, ri, out, ws, wsb, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_dotdd_noalloc(const float64x2 *a, const float64x2 *b, int64_t n,
                                              int64_t ri, float64x2 *out, void *stream) {
  return mfcuda::dot_noalloc(MF_D(a), MF_D(b), n, ri, out, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_norm2dd(const float64x2 *x, int64_t n, float64x2 *out, void *ws,
                                        size_t wsb, void *stream) {
  return mfcuda::reduce_dev<2>(MF_D(x), nullptr, n, 0, out, ws, wsb, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_csumdd(const complex64x2 *x, int64_t n, complex64x2 *out, void *ws,
                                       size_t wsb, void *stream) {
  return mfcuda::reduce_dev<3>(MF_D(x), nullptr, n, 0, out, ws, wsb, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_cdotdd(const complex64x2 *a, const complex64x2 *b, int64_t n,
                                       int64_t ri, complex64x2 *out, void *ws, size_t wsb,
                                       void *stream) {
  return mfcuda::reduce_dev<4>(MF_D(a), MF_D(b), n, ri, out, ws, wsb, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_cnorm2dd(const complex64x2 *x, int64_t n, float64x2 *out, void *ws,
                                         size_t wsb, void *stream) {
  return mfcuda::reduce_dev<5>(MF_D(x), nullptr, n, 0, out, ws, wsb, mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_reduce_partial_values(int kind) { return mfcuda::partial_values(kind); }
MULTIFLOATS_CUDA_API int mfcuda_reduce_partial(int kind, const void *x, const void *y, int64_t n,
                                               int64_t renorm_interval, void *out, void *ws, size_t wsb,
                                               void *stream) {
  return mfcuda::reduce_partial(kind, MF_D(x), MF_D(y), n, renorm_interval, out, ws, wsb,
                                mfcuda::as_stream(stream));
}
MULTIFLOATS_CUDA_API int mfcuda_reduce_combine(int kind, const void *parts, int64_t count, void *out,
                                               void *stream) {
  return mfcuda::reduce_combine(kind, parts, count, out, mfcuda::as_stream(stream));
}
#undef MF_D

MULTIFLOATS_CUDA_API float64x2 sumdd_array(const float64x2 *x, int64_t n) {
  float64x2 r = mfcuda::nan_dd();
  mfcuda::set_last_error(mfcuda::reduce_host<0>(x, nullptr, n, 0, &r));
  return r;
}
MULTIFLOATS_CUDA_API float64x2 dotdd_array(const float64x2 *a, const float64x2 *b, int64_t n,
                                           int64_t ri) {
  float64x2 r = mfcuda::nan_dd();
  mfcuda::set_last_error(mfcuda::reduce_host<1>(a, b, n, ri, &r));
  return r;
}
MULTIFLOATS_CUDA_API float64x2 norm2dd_array(const float64x2 *x, int64_t n) {
  float64x2 r = mfcuda::nan_dd();
  mfcuda::set_last_error(mfcuda::reduce_host<2>(x, nullptr, n, 0, &r));
  return r;
}
MULTIFLOATS_CUDA_API complex64x2 csumdd_array(const complex64x2 *x, int64_t n) {
  complex64x2 r;
  r.re = r.im = mfcuda::nan_dd();
  mfcuda::set_last_error(mfcuda::reduce_host<3>(x, nullptr, n, 0, &r));
  return r;
}
MULTIFLOATS_CUDA_API complex64x2 cdotdd_array(const complex64x2 *a, const complex64x2 *b, int64_t n,
                                              int64_t ri) {
  complex64x2 r;
  r.re = r.im = mfcuda::nan_dd();
  mfcuda::set_last_error(mfcuda::reduce_host<4>(a, b, n, ri, &r));
  return r;
}
MULTIFLOATS_CUDA_API float64x2 cnorm2dd_array(const complex64x2 *x, int64_t n) {
  float64x2 r = mfcuda::nan_dd();
  mfcuda::set_last_error(mfcuda::reduce_host<5>(x, nullptr, n, 0, &r));
  return r;
}

}  // extern "C"
