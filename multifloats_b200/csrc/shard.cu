// The DD array path over several GPUs behind the C ABI: one process (rank)
// per GPU, the ranks of an NCCL communicator.  No reference counterpart (the
// reference is single-process); the sharding follows the path's structure:
//
//   * one product C = A B in column panels: rank r of P computes the columns
//     [j0, j1) = mfcuda_shard_bounds(n, r, P) of C from all of A and the same
//     columns of B.  K is never split, so every output equals the
//     single-device call bit for bit.  The split forms first agree on the plan:
//     each rank plans its panel, one MAX all-reduce of the slice count / the
//     operand width (an int in the workspace, on the stream) gives every rank
//     the value the single call derives from all of B, and the plan is
//     recomputed from it -- no host synchronisation.  Optionally the panels
//     are then broadcast so that every rank holds all of C.
//   * reductions: each rank reduces its contiguous shard to a few DD values
//     (mfcuda_reduce_partial), the values are all-gathered in rank order and
//     folded left to right with DD addition (mfcuda_reduce_combine).  NCCL's
//     own sum would round away the compensation, so only an all-gather moves
//     data.
//
// NCCL is resolved at run time (dlopen) from the library the process already
// loaded (the caller created the communicator with it), else libnccl.so.2:
// the library has no link-time dependency on NCCL.  Every rank must make the
// same calls with the same m, k, n, form and flags; each call takes the same
// collectives in the same order on every rank, including ranks whose panel
// is empty.
#include <dlfcn.h>
#include <nccl.h>  // types only; the functions are resolved at run time

#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace mfcuda {
namespace split {
struct Agree {
  int (*fn)(void *ctx, int *v, cudaStream_t s);
  void *ctx;
};
int run_panel(bool crt, const float64x2 *a, const float64x2 *b, float64x2 *c, int64_t m, int64_t k, int64_t n,
              int arg, double target, void *ws, size_t ws_bytes, cudaStream_t s, int *info, const Agree *agree);
}  // namespace split

namespace shard {

struct NcclApi {
  decltype(&ncclAllReduce) all_reduce;
  decltype(&ncclAllGather) all_gather;
  decltype(&ncclBroadcast) broadcast;
  decltype(&ncclGroupStart) group_start;
  decltype(&ncclGroupEnd) group_end;
  decltype(&ncclCommCount) comm_count;
  decltype(&ncclCommUserRank) comm_user_rank;
};

static const NcclApi *nccl() {
  static NcclApi api;
  static const bool ok = [] {
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    if (!h) return false;
    api.all_reduce = reinterpret_cast<decltype(api.all_reduce)>(dlsym(h, "ncclAllReduce"));
    api.all_gather = reinterpret_cast<decltype(api.all_gather)>(dlsym(h, "ncclAllGather"));
    api.broadcast = reinterpret_cast<decltype(api.broadcast)>(dlsym(h, "ncclBroadcast"));
    api.group_start = reinterpret_cast<decltype(api.group_start)>(dlsym(h, "ncclGroupStart"));
    api.group_end = reinterpret_cast<decltype(api.group_end)>(dlsym(h, "ncclGroupEnd"));
    api.comm_count = reinterpret_cast<decltype(api.comm_count)>(dlsym(h, "ncclCommCount"));
    api.comm_user_rank = reinterpret_cast<decltype(api.comm_user_rank)>(dlsym(h, "ncclCommUserRank"));
    return api.all_reduce && api.all_gather && api.broadcast && api.group_start && api.group_end &&
           api.comm_count && api.comm_user_rank;
  }();
  return ok ? &api : nullptr;
}

#define MF_TRY_NCCL(expr)                               \
  do {                                                  \
    if ((expr) != ncclSuccess) return MFCUDA_ERR_CUDA;  \
  } while (0)

// Contiguous shard [j0, j1) of n items for `rank` of `world`: the first
// n % world ranks get one item more.
static void bounds(int64_t n, int rank, int world, int64_t *j0, int64_t *j1) {
  const int64_t q = n / world, r = n % world;
  *j0 = rank * q + std::min<int64_t>(rank, r);
  *j1 = *j0 + q + (rank < r ? 1 : 0);
}

static int comm_info(void *comm, int *rank, int *world) {
  const NcclApi *N = nccl();
  if (!N) return MFCUDA_ERR_UNSUPPORTED;
  if (!comm) return MFCUDA_ERR_INVALID_ARG;
  ncclComm_t c = static_cast<ncclComm_t>(comm);
  MF_TRY_NCCL(N->comm_count(c, world));
  MF_TRY_NCCL(N->comm_user_rank(c, rank));
  if (*world < 1 || *rank < 0 || *rank >= *world) return MFCUDA_ERR_CUDA;
  return MFCUDA_OK;
}

// In-place MAX all-reduce of one device int (the plan agreement).
struct AgreeCtx {
  ncclComm_t comm;
};
static int agree_max(void *ctx, int *v, cudaStream_t s) {
  const NcclApi *N = nccl();
  if (!N) return MFCUDA_ERR_UNSUPPORTED;
  MF_TRY_NCCL(N->all_reduce(v, v, 1, ncclInt32, ncclMax, static_cast<AgreeCtx *>(ctx)->comm, s));
  return MFCUDA_OK;
}

static int matmul(int form, const float64x2 *a, const float64x2 *b, float64x2 *c, int64_t m, int64_t k, int64_t n,
                  int64_t ri, double target, int flags, void *ws, size_t ws_bytes, int *info, void *comm_p,
                  cudaStream_t s) {
  if (form != MFCUDA_FORM_PLAIN && form != MFCUDA_FORM_SPLIT && form != MFCUDA_FORM_CRT)
    return MFCUDA_ERR_INVALID_ARG;
  if ((flags & ~(MFCUDA_SHARD_PANELS | MFCUDA_SHARD_GATHER)) ||
      ((flags & MFCUDA_SHARD_PANELS) && (flags & MFCUDA_SHARD_GATHER)))
    return MFCUDA_ERR_INVALID_ARG;
  if (m < 0 || k < 0 || n < 0 || !mul_ok(m, k) || !mul_ok(k, n) || !mul_ok(m, n)) return MFCUDA_ERR_INVALID_ARG;
  int rank = 0, world = 1;
  MF_TRY(comm_info(comm_p, &rank, &world));
  MF_TRY(require_device());
  ncclComm_t comm = static_cast<ncclComm_t>(comm_p);
  int64_t j0, j1;
  bounds(n, rank, world, &j0, &j1);
  const int64_t np = j1 - j0;
  const bool panels = (flags & MFCUDA_SHARD_PANELS) != 0;
  const float64x2 *bp = panels ? b : b + k * j0;  // this rank's columns of B
  float64x2 *cp = panels ? c : c + m * j0;        // and of C
  if (info) info[0] = info[1] = info[2] = info[3] = 0;
  if (form == MFCUDA_FORM_PLAIN) {
    if (np > 0 && m > 0) MF_TRY(mfcuda_matmuldd_mm(a, bp, cp, m, k, np, ri, s));
  } else if (m > 0 && k > 0) {
    // every rank takes part in the agreement, an empty panel included
    AgreeCtx ctx = {comm};
    const split::Agree agree = {agree_max, &ctx};
    const bool crt = form == MFCUDA_FORM_CRT;
    if (np > 0) {
      MF_TRY(split::run_panel(crt, a, bp, cp, m, k, np, (int)ri, target, ws, ws_bytes, s, info, &agree));
    } else {
      void *tmp = nullptr;
      MF_TRY(ws_alloc(&tmp, sizeof(int), s));
      int rc = cudaMemsetAsync(tmp, 0, sizeof(int), s) == cudaSuccess ? agree_max(&ctx, static_cast<int *>(tmp), s)
                                                                      : MFCUDA_ERR_CUDA;
      ws_free(tmp, s);
      MF_TRY(rc);
    }
  } else if (m > 0 && np > 0) {  // k == 0: C = 0
    MF_TRY_CUDA(cudaMemsetAsync(cp, 0, (size_t)(m * np) * sizeof(float64x2), s));
  }
  if (flags & MFCUDA_SHARD_GATHER) {
    // every rank broadcasts its panel; afterwards every rank holds all of C
    const NcclApi *N = nccl();
    MF_TRY_NCCL(N->group_start());
    ncclResult_t r = ncclSuccess;
    for (int q = 0; q < world && r == ncclSuccess; ++q) {
      int64_t q0, q1;
      bounds(n, q, world, &q0, &q1);
      if (q1 == q0 || m == 0) continue;
      double *panel = reinterpret_cast<double *>(c + m * q0);
      r = N->broadcast(panel, panel, (size_t)(2 * m * (q1 - q0)), ncclFloat64, q, comm, s);
    }
    const ncclResult_t r2 = N->group_end();
    if (r != ncclSuccess || r2 != ncclSuccess) return MFCUDA_ERR_CUDA;
  }
  return MFCUDA_OK;
}

static int reduce(int kind, const void *x, const void *y, int64_t n, int64_t ri, void *out, void *comm_p,
                  cudaStream_t s) {
  const int pv = mfcuda_reduce_partial_values(kind);
  if (pv <= 0) return MFCUDA_ERR_INVALID_ARG;
  if (n < 0 || !out || (n > 0 && (!x || ((kind == MFCUDA_RED_DOT || kind == MFCUDA_RED_CDOT) && !y))))
    return MFCUDA_ERR_INVALID_ARG;
  int rank = 0, world = 1;
  MF_TRY(comm_info(comm_p, &rank, &world));
  MF_TRY(require_device());
  const NcclApi *N = nccl();
  const size_t part_doubles = 2 * (size_t)pv;
  void *buf = nullptr;
  MF_TRY(ws_alloc(&buf, sizeof(double) * part_doubles * (1 + (size_t)world), s));
  double *part = static_cast<double *>(buf), *all = part + part_doubles;
  int rc = mfcuda_reduce_partial(kind, x, y, n, ri, part, nullptr, 0, s);
  if (rc == MFCUDA_OK &&
      N->all_gather(part, all, part_doubles, ncclFloat64, static_cast<ncclComm_t>(comm_p), s) != ncclSuccess)
    rc = MFCUDA_ERR_CUDA;
  if (rc == MFCUDA_OK) rc = mfcuda_reduce_combine(kind, all, world, out, s);
  ws_free(buf, s);
  return rc;
}

}  // namespace shard
}  // namespace mfcuda

extern "C" {

MULTIFLOATS_CUDA_API void mfcuda_shard_bounds(int64_t n, int rank, int world, int64_t *start, int64_t *stop) {
  if (!start || !stop) return;
  if (n < 0 || world < 1 || rank < 0 || rank >= world) {
    *start = *stop = 0;
    return;
  }
  mfcuda::shard::bounds(n, rank, world, start, stop);
}

MULTIFLOATS_CUDA_API int mfcuda_nccl_available(void) { return mfcuda::shard::nccl() ? 1 : 0; }

MULTIFLOATS_CUDA_API int mfcuda_matmuldd_mm_nccl(int form, const float64x2 *a, const float64x2 *b, float64x2 *c,
                                                 int64_t m, int64_t k, int64_t n, int64_t param, double target,
                                                 int flags, void *workspace, size_t workspace_bytes,
                                                 int *info_out, void *nccl_comm, void *stream) {
  return mfcuda::shard::matmul(form, a, b, c, m, k, n, param, target, flags, workspace, workspace_bytes,
                               info_out, nccl_comm, mfcuda::as_stream(stream));
}

MULTIFLOATS_CUDA_API int mfcuda_reduce_nccl(int kind, const void *x, const void *y, int64_t n,
                                            int64_t renorm_interval, void *out, void *nccl_comm, void *stream) {
  return mfcuda::shard::reduce(kind, x, y, n, renorm_interval, out, nccl_comm, mfcuda::as_stream(stream));
}

}  // extern "C"
