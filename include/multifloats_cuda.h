/* libmultifloats_cuda -- B200 (sm_100a) implementation of the multifloats
 * double-double array hot path behind a plain C ABI.
 *
 * Two families of entry points:
 *
 *  1. Drop-in symbols with the reference's own names and signatures
 *     (matmuldd_mm, matmuldd_mv, matmuldd_vm and their matmulf64x2_* aliases),
 *     plus array forms of the Fortran-only reductions and elemental functions
 *     (expdd_array, dotdd_array, ...).  They take HOST pointers, copy to the
 *     GPU, run the kernel and copy back before returning (synchronous).  Like
 *     the reference they return no status: NaN-in-NaN-out for the data; a CUDA
 *     or argument failure is latched per thread and read with
 *     mfcuda_last_error().
 *
 *  2. mfcuda_* entry points taking DEVICE pointers and a cudaStream_t (passed
 *     as void*), returning 0 on success or an MFCUDA_ERR_* code.  They are
 *     asynchronous on the stream.
 *
 * Layout: float64x2 is two back-to-back binary64 limbs {hi, lo} (16 bytes),
 * complex64x2 is {re, im} (32 bytes), matrices are column-major with the
 * leading dimension equal to the first extent, exactly as in the reference
 * (include/multifloats/float64x2.h:125-186, :348-378, :654-696).
 *
 * Reference citations are paths inside multifloats 0.10.3.
 */
#ifndef MULTIFLOATS_CUDA_H
#define MULTIFLOATS_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__) || defined(__clang__)
#define MULTIFLOATS_CUDA_API __attribute__((visibility("default")))
#else
#define MULTIFLOATS_CUDA_API
#endif

/* Interchange types.  When the reference header multifloats/float64x2.h has
 * already been included (it defines MULTIFLOATS_ABI_VERSION) its identical
 * structs are used instead: in C they are the global struct float64x2 /
 * complex64x2; in C++ the reference declares them in namespace multifloats
 * (include/multifloats/float64x2.h:72, :125, :348), so they are brought into
 * the global namespace here for the declarations below. */
#ifndef MULTIFLOATS_ABI_VERSION
struct float64x2 {
  double limbs[2];
};
struct complex64x2 {
  struct float64x2 re;
  struct float64x2 im;
};
#ifndef __cplusplus
typedef struct float64x2 float64x2;
typedef struct complex64x2 complex64x2;
#endif
#elif defined(__cplusplus)
using multifloats::complex64x2;
using multifloats::float64x2;
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status ------------------------------------------------------------- */
enum {
  MFCUDA_OK = 0,
  MFCUDA_ERR_INVALID_ARG = 1,   /* negative size, NULL pointer with size > 0, overflow */
  MFCUDA_ERR_CUDA = 2,          /* a CUDA runtime call failed */
  MFCUDA_ERR_ALLOC = 3,         /* device or host allocation failed */
  MFCUDA_ERR_NO_DEVICE = 4,     /* no sm_100 device visible */
  MFCUDA_ERR_TIMEOUT = 5,       /* a bounded device-side wait expired */
  MFCUDA_ERR_WORKSPACE = 6,     /* caller workspace too small */
  MFCUDA_ERR_UNSUPPORTED = 7    /* shape/parameter outside what the kernel supports */
};
/* Status of the calling thread's last drop-in call (0 = success). */
MULTIFLOATS_CUDA_API int mfcuda_last_error(void);
MULTIFLOATS_CUDA_API const char *mfcuda_error_string(int code);
/* Library version, e.g. "0.1.0". */
MULTIFLOATS_CUDA_API const char *mfcuda_version(void);

/* ==========================================================================
 * 1. Drop-in symbols (host pointers, synchronous)
 * ========================================================================== */

/* Compensated DD matmul, column-major, C overwritten.  Replaces
 * matmuldd_mm / matmuldd_mv / matmuldd_vm (include/multifloats/float64x2.h:682-696,
 * src/float64x2/abi.inc:133-149, kernels src/float64x2/matmul.inc:6-239).
 * Bit-identical to the reference: every output runs the reference MAC over
 * p = 0..k-1 in order with the same renormalisation cadence. */
MULTIFLOATS_CUDA_API void matmuldd_mm(const float64x2 *a, const float64x2 *b, float64x2 *c,
                                      int64_t m, int64_t k, int64_t n,
                                      int64_t renorm_interval);
MULTIFLOATS_CUDA_API void matmuldd_mv(const float64x2 *a, const float64x2 *x, float64x2 *y,
                                      int64_t m, int64_t k, int64_t renorm_interval);
MULTIFLOATS_CUDA_API void matmuldd_vm(const float64x2 *x, const float64x2 *b, float64x2 *y,
                                      int64_t k, int64_t n, int64_t renorm_interval);
/* f64x2-tagged spellings (src/float64x2/f64x2_aliases.inc:114-116). */
MULTIFLOATS_CUDA_API void matmulf64x2_mm(const float64x2 *a, const float64x2 *b, float64x2 *c,
                                         int64_t m, int64_t k, int64_t n,
                                         int64_t renorm_interval);
MULTIFLOATS_CUDA_API void matmulf64x2_mv(const float64x2 *a, const float64x2 *x, float64x2 *y,
                                         int64_t m, int64_t k, int64_t renorm_interval);
MULTIFLOATS_CUDA_API void matmulf64x2_vm(const float64x2 *x, const float64x2 *b, float64x2 *y,
                                         int64_t k, int64_t n, int64_t renorm_interval);

/* Complex matmul as 4 real compensated products combined with DD -/+, the
 * Fortran cdd_matmul_mm (fsrc/multifloats.fypp:2609-2621), fused in one pass.
 * Bit-identical to that composition. */
MULTIFLOATS_CUDA_API void cmatmuldd_mm(const complex64x2 *a, const complex64x2 *b,
                                       complex64x2 *c, int64_t m, int64_t k, int64_t n,
                                       int64_t renorm_interval);

/* Elementwise y[i] = f(x[i]): the Fortran elemental exp/log/sin/cos/sqrt over an
 * array (fsrc/multifloats.fypp:792-798, :1407-1412), one expdd / logdd / sindd /
 * cosdd / sqrtdd per element (src/float64x2/abi.inc:30, :53, :59, :67, :68).
 * Bit-identical per element.  x and y may alias. */
MULTIFLOATS_CUDA_API void expdd_array(const float64x2 *x, float64x2 *y, int64_t n);
MULTIFLOATS_CUDA_API void logdd_array(const float64x2 *x, float64x2 *y, int64_t n);
MULTIFLOATS_CUDA_API void sindd_array(const float64x2 *x, float64x2 *y, int64_t n);
MULTIFLOATS_CUDA_API void cosdd_array(const float64x2 *x, float64x2 *y, int64_t n);
MULTIFLOATS_CUDA_API void sqrtdd_array(const float64x2 *x, float64x2 *y, int64_t n);
/* exp2dd / log2dd / log10dd (src/float64x2/exp_log.inc:109-128, :311-326,
 * :344-353) per element; bit-identical. */
MULTIFLOATS_CUDA_API void exp2dd_array(const float64x2 *x, float64x2 *y, int64_t n);
MULTIFLOATS_CUDA_API void log2dd_array(const float64x2 *x, float64x2 *y, int64_t n);
MULTIFLOATS_CUDA_API void log10dd_array(const float64x2 *x, float64x2 *y, int64_t n);
/* Fused sine and cosine: sincosdd (src/float64x2/abi.inc:123-125,
 * trig.inc:216-236) per element, one range reduction for both outputs;
 * equal bit for bit to sindd / cosdd. */
MULTIFLOATS_CUDA_API void sincosdd_array(const float64x2 *x, float64x2 *s, float64x2 *c, int64_t n);
/* z[i] = cos x[i] + i sin x[i]: cexpidd (abi.inc:226-229). */
MULTIFLOATS_CUDA_API void cexpidd_array(const float64x2 *x, complex64x2 *z, int64_t n);
/* w[i] = exp(z[i]): cexpdd (src/complex64x2/abi.inc:189, the std::exp
 * specialisation of src/complex64x2/std.inc:20-74, C99 Annex G special values). */
MULTIFLOATS_CUDA_API void cexpdd_array(const complex64x2 *z, complex64x2 *w, int64_t n);

/* Reductions: the Fortran-only sum / dot_product / norm2 generics
 * (fsrc/multifloats.fypp:1980-2019, :2094-2158, :2254-2331, :2338-2352) as
 * C entry points.  Each thread of the device runs the reference's per-element
 * compensated update over a fixed strided subsequence; partials are combined
 * with DD addition in a fixed tree that depends only on n, so results are
 * run-to-run reproducible and bit-identical to the CPU restatement of that order. */
MULTIFLOATS_CUDA_API float64x2 sumdd_array(const float64x2 *x, int64_t n);
MULTIFLOATS_CUDA_API float64x2 dotdd_array(const float64x2 *a, const float64x2 *b, int64_t n,
                                           int64_t renorm_interval);
MULTIFLOATS_CUDA_API float64x2 norm2dd_array(const float64x2 *x, int64_t n);
MULTIFLOATS_CUDA_API complex64x2 csumdd_array(const complex64x2 *x, int64_t n);
/* conj(a) . b, as the Fortran cdd_dot_product (fypp:2321-2331). */
MULTIFLOATS_CUDA_API complex64x2 cdotdd_array(const complex64x2 *a, const complex64x2 *b,
                                              int64_t n, int64_t renorm_interval);
/* sqrt(sum re^2 + im^2): norm2 of the array viewed as 2n reals (re0, im0, re1, ...). */
MULTIFLOATS_CUDA_API float64x2 cnorm2dd_array(const complex64x2 *x, int64_t n);

/* Split-INT8 DD matmul (no reference counterpart): the product matmuldd_mm
 * computes, to a stated bound instead of bit for bit.  Each row of A and
 * column of B is scaled by a power of two, every entry is rounded to a
 * (8S-2)-bit integer and cut into S signed 8-bit slices, all slice pairs on
 * anti-diagonals s + t <= S-1 are multiplied on the tcgen05 INT8 tensor cores
 * with exact INT32 accumulation, and the diagonals are summed back into DD.
 * slices = 0 picks S (<= 14) from the operands' exponent ranges so that the
 * a-priori bound meets err_ij <= 8 k 2^-104 (|A||B|)_ij; *max_err_bound_out
 * (may be NULL) receives that a-priori bound in units of k 2^-104 (|A||B|)_ij.
 * A row of A or column of B holding Inf/NaN yields NaN in the affected
 * outputs.  Host pointers, synchronous. */
MULTIFLOATS_CUDA_API void matmuldd_mm_split(const float64x2 *a, const float64x2 *b, float64x2 *c,
                                            int64_t m, int64_t k, int64_t n, int slices,
                                            double *max_err_bound_out);
/* Complex split form: the four real products of the Fortran cdd_matmul_mm
 * composition (fsrc/multifloats.fypp:2609-2621) -- re = Ar Br - Ai Bi,
 * im = Ar Bi + Ai Br, combined with the DD operators -- each in split form
 * with one slice count for all four (the four parts are sliced once).  The
 * bound applies to each real product. */
MULTIFLOATS_CUDA_API void cmatmuldd_mm_split(const complex64x2 *a, const complex64x2 *b,
                                             complex64x2 *c, int64_t m, int64_t k, int64_t n,
                                             int slices, double *max_err_bound_out);
/* CRT (modular) split-INT8 DD matmul (no reference counterpart): the same
 * product, to the same kind of stated bound, from fewer tensor-core products.
 * Each row of A / column of B is scaled by a power of two and every entry
 * rounded to a W-bit integer (as in matmuldd_mm_split); the exact integer
 * product is recovered from its residues modulo N pairwise-coprime moduli
 * <= 256 (one INT8 GEMM per modulus on the tcgen05 tensor cores, exact INT32
 * accumulation) by the Chinese remainder theorem, then rounded to DD and
 * scaled.  bits = 0 picks the smallest W whose a-priori bound meets
 * err_ij <= 8 k 2^-104 (|A||B|)_ij (W = 92, N = 26 at k = 4096 for operands
 * spanning one binade per row / column); 8..110 = fixed W.  *max_err_bound_out
 * (may be NULL) receives the bound in units of k 2^-104 (|A||B|)_ij.  Inf/NaN
 * in a row of A or column of B yields NaN in the affected outputs.  Host
 * pointers, synchronous. */
MULTIFLOATS_CUDA_API void matmuldd_mm_crt(const float64x2 *a, const float64x2 *b, float64x2 *c,
                                          int64_t m, int64_t k, int64_t n, int bits,
                                          double *max_err_bound_out);
/* Complex CRT form: re = Ar Br - Ai Bi, im = Ar Bi + Ai Br (the Fortran
 * cdd_matmul_mm composition) with one W and moduli set for all four real
 * products (planned from all four parts, each part reduced once); the bound
 * applies to each real product. */
MULTIFLOATS_CUDA_API void cmatmuldd_mm_crt(const complex64x2 *a, const complex64x2 *b, complex64x2 *c,
                                           int64_t m, int64_t k, int64_t n, int bits,
                                           double *max_err_bound_out);

/* ==========================================================================
 * 2. Device-pointer API (asynchronous on `stream`, a cudaStream_t; NULL = legacy
 *    default stream).  Return MFCUDA_OK or an error code.
 * ========================================================================== */
MULTIFLOATS_CUDA_API int mfcuda_matmuldd_mm(const float64x2 *a, const float64x2 *b, float64x2 *c,
                                            int64_t m, int64_t k, int64_t n,
                                            int64_t renorm_interval, void *stream);
MULTIFLOATS_CUDA_API int mfcuda_matmuldd_mv(const float64x2 *a, const float64x2 *x, float64x2 *y,
                                            int64_t m, int64_t k, int64_t renorm_interval,
                                            void *stream);
MULTIFLOATS_CUDA_API int mfcuda_matmuldd_vm(const float64x2 *x, const float64x2 *b, float64x2 *y,
                                            int64_t k, int64_t n, int64_t renorm_interval,
                                            void *stream);
MULTIFLOATS_CUDA_API int mfcuda_cmatmuldd_mm(const complex64x2 *a, const complex64x2 *b,
                                             complex64x2 *c, int64_t m, int64_t k, int64_t n,
                                             int64_t renorm_interval, void *stream);

/* Split-INT8 form on device pointers (16-byte aligned).  slices: 0 = choose
 * from the exponent ranges for `target` (bound in units of k 2^-104 (|A||B|)_ij,
 * 8 in the drop-in), 2..14 = fixed.  `workspace` may be NULL (stream-ordered
 * allocation) or hold mfcuda_split_workspace_size(m, k, n) bytes.  info_out may
 * be NULL or point to int[3] receiving {S, rho_A, rho_B} (slices used and the
 * operands' exponent spreads); a non-NULL info_out makes the call wait for the
 * result and report MFCUDA_ERR_TIMEOUT if a bounded device wait expired. */
MULTIFLOATS_CUDA_API size_t mfcuda_split_workspace_size(int64_t m, int64_t k, int64_t n);
/* CRT form on device pointers (16-byte aligned).  bits: 0 = W from `target`
 * (units of k 2^-104 (|A||B|)_ij), 8..110 = fixed.  `workspace` may be NULL or
 * hold mfcuda_crt_workspace_size(m, k, n, bits) bytes.  info_out may be NULL or
 * point to int[4] receiving {N moduli, rho_A, rho_B, W} (waits for the result,
 * MFCUDA_ERR_TIMEOUT if a bounded device wait expired).  mfcuda_crt_bound gives
 * the a-priori bound for W, the spreads and k (-1 for invalid arguments). */
MULTIFLOATS_CUDA_API size_t mfcuda_crt_workspace_size(int64_t m, int64_t k, int64_t n, int bits);
MULTIFLOATS_CUDA_API int mfcuda_matmuldd_mm_crt(const float64x2 *a, const float64x2 *b, float64x2 *c,
                                                int64_t m, int64_t k, int64_t n, int bits, double target,
                                                void *workspace, size_t workspace_bytes, int *info_out,
                                                void *stream);
MULTIFLOATS_CUDA_API double mfcuda_crt_bound(int bits, int rho_a, int rho_b, int64_t k);
MULTIFLOATS_CUDA_API size_t mfcuda_ccrt_workspace_size(int64_t m, int64_t k, int64_t n, int bits);
MULTIFLOATS_CUDA_API int mfcuda_cmatmuldd_mm_crt(const complex64x2 *a, const complex64x2 *b, complex64x2 *c,
                                                 int64_t m, int64_t k, int64_t n, int bits, double target,
                                                 void *workspace, size_t workspace_bytes, int *info_out,
                                                 void *stream);
MULTIFLOATS_CUDA_API int mfcuda_matmuldd_mm_split(const float64x2 *a, const float64x2 *b,
                                                  float64x2 *c, int64_t m, int64_t k, int64_t n,
                                                  int slices, double target, void *workspace,
                                                  size_t workspace_bytes, int *info_out,
                                                  void *stream);
MULTIFLOATS_CUDA_API size_t mfcuda_csplit_workspace_size(int64_t m, int64_t k, int64_t n);
MULTIFLOATS_CUDA_API int mfcuda_cmatmuldd_mm_split(const complex64x2 *a, const complex64x2 *b,
                                                   complex64x2 *c, int64_t m, int64_t k, int64_t n,
                                                   int slices, double target, void *workspace,
                                                   size_t workspace_bytes, int *info_out,
                                                   void *stream);

/* Phase profiling of the split form for the calling host thread.  Between
 * begin and end, every mfcuda_matmuldd_mm_split / matmuldd_mm_split call
 * records events (owned by the library) on its stream around its phases;
 * end waits for them and writes the summed milliseconds of
 * {exponent scan, slicing, tensor-core kernel, recombination} to
 * phase_ms_sum[0..3] and the number of calls to *calls. */
MULTIFLOATS_CUDA_API void mfcuda_phase_profile_begin(void);
MULTIFLOATS_CUDA_API int mfcuda_phase_profile_end(double *phase_ms_sum, int64_t *calls);

/* Bounded waits of the tensor-core kernels (split and CRT forms, single calls
 * and batches).  No reference counterpart (the reference runs on the CPU).
 * Every wait of these kernels for a pipeline stage, an accumulator hand-off or
 * the reconstruction's own MMAs gives up after a limit (2 s by default),
 * records the failure and lets the kernel leave once its own copies and MMAs
 * in flight have finished, so the context stays usable; the call's outputs
 * are then unspecified.  A call given info_out reports MFCUDA_ERR_TIMEOUT.
 *
 * mfcuda_set_wait_limit_ns sets the limit, process-wide, for kernels launched
 * (and batch plans created) from then on; 0 restores the default.  It
 * returns the previous setting (0 = default).  It exists to test the failure
 * path: a limit far below a kernel's running time makes its waits give up.
 *
 * mfcuda_timeout_status returns MFCUDA_ERR_TIMEOUT if any of these kernels
 * gave up a wait on the current device since the last clearing query, else
 * MFCUDA_OK (MFCUDA_ERR_CUDA if the query itself fails); clear != 0 resets
 * the record.  For callers of the device-pointer forms that passed
 * info_out = NULL, and for batch runs: synchronise the streams of the calls
 * in question first. */
MULTIFLOATS_CUDA_API uint64_t mfcuda_set_wait_limit_ns(uint64_t ns);
MULTIFLOATS_CUDA_API int mfcuda_timeout_status(int clear);

/* op: 0 exp, 1 log, 2 sin, 3 cos, 4 sqrt */
enum {
  MFCUDA_EXP = 0,
  MFCUDA_LOG = 1,
  MFCUDA_SIN = 2,
  MFCUDA_COS = 3,
  MFCUDA_SQRT = 4,
  MFCUDA_EXP2 = 5,  /* exp2dd, src/float64x2/exp_log.inc:109-128 */
  MFCUDA_LOG2 = 6,  /* log2dd, exp_log.inc:311-326 */
  MFCUDA_LOG10 = 7  /* log10dd, exp_log.inc:344-353 */
};
/* Device forms of sincosdd_array, cexpidd_array, cexpdd_array. */
MULTIFLOATS_CUDA_API int mfcuda_sincos_dd(const float64x2 *x, float64x2 *s, float64x2 *c, int64_t n,
                                          void *stream);
MULTIFLOATS_CUDA_API int mfcuda_cexpi_dd(const float64x2 *x, complex64x2 *z, int64_t n, void *stream);
MULTIFLOATS_CUDA_API int mfcuda_cexp_dd(const complex64x2 *z, complex64x2 *w, int64_t n, void *stream);
MULTIFLOATS_CUDA_API int mfcuda_unary_dd(int op, const float64x2 *x, float64x2 *y, int64_t n,
                                         void *stream);

/* Reductions write their result to DEVICE memory `out`.  `workspace` may be
 * NULL (stream-ordered allocation inside) or point to at least
 * mfcuda_reduce_workspace_size(n) bytes of device memory. */
MULTIFLOATS_CUDA_API size_t mfcuda_reduce_workspace_size(int64_t n);
MULTIFLOATS_CUDA_API int mfcuda_sumdd(const float64x2 *x, int64_t n, float64x2 *out,
                                      void *workspace, size_t workspace_bytes, void *stream);
MULTIFLOATS_CUDA_API int mfcuda_dotdd(const float64x2 *a, const float64x2 *b, int64_t n,
                                      int64_t renorm_interval, float64x2 *out, void *workspace,
                                      size_t workspace_bytes, void *stream);
MULTIFLOATS_CUDA_API int mfcuda_norm2dd(const float64x2 *x, int64_t n, float64x2 *out,
                                        void *workspace, size_t workspace_bytes, void *stream);
MULTIFLOATS_CUDA_API int mfcuda_csumdd(const complex64x2 *x, int64_t n, complex64x2 *out,
                                       void *workspace, size_t workspace_bytes, void *stream);
MULTIFLOATS_CUDA_API int mfcuda_cdotdd(const complex64x2 *a, const complex64x2 *b, int64_t n,
                                       int64_t renorm_interval, complex64x2 *out,
                                       void *workspace, size_t workspace_bytes, void *stream);
MULTIFLOATS_CUDA_API int mfcuda_cnorm2dd(const complex64x2 *x, int64_t n, float64x2 *out,
                                         void *workspace, size_t workspace_bytes, void *stream);

/* Real dot product a . b that allocates nothing.  No counterpart in
 * the reference: it exists for callers that cannot let a library allocate
 * device memory -- a host application that gives the whole GPU memory to its
 * own pool and forbids allocations behind its back, or code on a
 * latency-critical path where cudaMalloc / cudaFree would synchronise the
 * device.  Same arguments, order of operations and result (bit for bit) as
 * mfcuda_dotdd with a NULL workspace, but the block partials live in a fixed
 * 16 KiB device array inside the library, so:
 *   - n is limited to 4,194,304 elements; larger n returns
 *     MFCUDA_ERR_UNSUPPORTED without launching anything;
 *   - every call outside stream capture looks up that array's device
 *     address on the current device (so a cudaDeviceReset between calls is
 *     harmless); a call inside a capture reuses the address found by an
 *     earlier call on that device, so make the first call on each device
 *     before any stream capture;
 *   - all calls share the one array, so calls that overlap on the GPU (for
 *     example on two streams at once) race and corrupt each other's result;
 *     serialise them.  No state carries from one call to the next.
 * The array is held on every GPU that loads the library until process exit. */
MULTIFLOATS_CUDA_API int mfcuda_dotdd_noalloc(const float64x2 *a, const float64x2 *b, int64_t n,
                                              int64_t renorm_interval, float64x2 *out,
                                              void *stream);

/* ---- reductions sharded over several devices --------------------------------
 * No reference counterpart (the reference is single-process).  Each device
 * reduces its contiguous shard with mfcuda_reduce_partial, which runs the same
 * two kernels as the single-device call but stops before the final step and
 * writes mfcuda_reduce_partial_values(kind) DD values to `out` (sum, dot: the
 * DD sum; norm2, cnorm2: the sum of squares before the square root; csum: re,
 * im; cdot: the four component dots rr, ii, ri, ir).  After an all-gather of
 * those partials in rank order, mfcuda_reduce_combine folds them left to
 * right with DD addition and applies the final step, writing the result in
 * the single call's format.  The result is deterministic for a given shard
 * split and within the single call's error bound (not bit-identical to it,
 * whose fold order differs).  kind: MFCUDA_RED_*; x, y, parts, out: device
 * pointers; y only for the dot kinds. */
enum {
  MFCUDA_RED_SUM = 0,
  MFCUDA_RED_DOT = 1,
  MFCUDA_RED_NORM2 = 2,
  MFCUDA_RED_CSUM = 3,
  MFCUDA_RED_CDOT = 4,
  MFCUDA_RED_CNORM2 = 5
};
MULTIFLOATS_CUDA_API int mfcuda_reduce_partial_values(int kind);
MULTIFLOATS_CUDA_API int mfcuda_reduce_partial(int kind, const void *x, const void *y, int64_t n,
                                               int64_t renorm_interval, void *out, void *workspace,
                                               size_t workspace_bytes, void *stream);
MULTIFLOATS_CUDA_API int mfcuda_reduce_combine(int kind, const void *parts, int64_t count, void *out,
                                               void *stream);

/* ---- batched ragged work ---------------------------------------------------
 * Many independent problems in grouped launches captured once in a CUDA graph
 * (no reference counterpart; each problem computes what the single call
 * computes, bit for bit).  A plan binds the problems' DEVICE pointers at
 * creation; mfcuda_batch_run replays the graph on a stream (refill the same
 * buffers between runs, or create a new plan for new buffers).
 *   form MFCUDA_FORM_PLAIN: one persistent grouped kernel over every output
 *     tile of every problem (longest K first, dynamic scheduling); per problem a
 *     tile shape of 64x64, 32x32 or 16x16 outputs.  renorm_interval as in
 *     matmuldd_mm; slices/target unused.
 *   form MFCUDA_FORM_SPLIT: the split-INT8 pipeline, each phase one grouped
 *     launch; one persistent tcgen05 kernel over every (diagonal, K chunk, tile)
 *     item of every problem; per problem a tile width N of 256, 128 or 64 and a
 *     shared K chunk (split-K when the batch is too small to fill the GPU);
 *     slices/target as in mfcuda_matmuldd_mm_split.  Operands 16-byte aligned.
 *   form MFCUDA_FORM_CRT: the CRT (modular) split pipeline of
 *     mfcuda_matmuldd_mm_crt in the same grouped launches (one item per
 *     modulus, K chunk and tile); `slices` is the operand bits W (0, or 8 ..
 *     110) and target as there.  Bit-identical to the single call for every
 *     K chunk (residues of chunk sums add modulo each modulus).
 * tune != 0 times the candidate tile shapes of every new shape bucket on
 * synthetic problems and caches the winners in MFCUDA_AUTOTUNE_CACHE (default
 * $HOME/.cache/multifloats_b200/autotune.txt); tune == 0 uses cached winners or
 * a built-in heuristic. */
typedef struct mfcuda_gemm_desc {
  const void *a; /* float64x2, column-major m x k */
  const void *b; /* float64x2, column-major k x n */
  void *c;       /* float64x2, column-major m x n (overwritten) */
  int64_t m, k, n;
} mfcuda_gemm_desc;
typedef struct mfcuda_batch mfcuda_batch;
enum { MFCUDA_FORM_PLAIN = 0, MFCUDA_FORM_SPLIT = 1, MFCUDA_FORM_CRT = 2 };
MULTIFLOATS_CUDA_API int mfcuda_batch_create_gemm(const mfcuda_gemm_desc *descs, int64_t count,
                                                  int form, int64_t renorm_interval, int slices,
                                                  double target, int tune, mfcuda_batch **plan);
/* The same for complex64x2 problems (a, b, c of each descriptor point to
 * complex64x2 matrices): MFCUDA_FORM_PLAIN runs every 32 x 32 output tile with
 * the tile code of mfcuda_cmatmuldd_mm (bit-identical to it);
 * MFCUDA_FORM_SPLIT runs each problem as the four real products of
 * mfcuda_cmatmuldd_mm_split (one slice count from all four operands, each
 * operand sliced once, re = ArBr - AiBi and im = ArBi + AiBr combined in that
 * order), bit-identical to it when the plan's K chunk (mfcuda_batch_kchunk)
 * is the single call's 73 x 128; MFCUDA_FORM_CRT runs the four products of
 * mfcuda_cmatmuldd_mm_crt the same way (bit-identical to it). */
MULTIFLOATS_CUDA_API int mfcuda_batch_create_cgemm(const mfcuda_gemm_desc *descs, int64_t count,
                                                   int form, int64_t renorm_interval, int slices,
                                                   double target, int tune, mfcuda_batch **plan);
/* Ragged elementwise batch: y_a[i] = op(x_a[i]) for every array a (lengths
 * ns[a], device pointers), one grid-stride launch over all elements. */
MULTIFLOATS_CUDA_API int mfcuda_batch_create_unary(int op, const float64x2 *const *xs,
                                                   float64x2 *const *ys, const int64_t *ns,
                                                   int64_t count, mfcuda_batch **plan);
MULTIFLOATS_CUDA_API int mfcuda_batch_run(mfcuda_batch *plan, void *stream);
/* Waits for the device and reports MFCUDA_ERR_TIMEOUT if a bounded device-side
 * wait of the plan's last run expired. */
MULTIFLOATS_CUDA_API int mfcuda_batch_status(mfcuda_batch *plan);
/* Tile edge (plain) or tile width N (split) chosen for problem i; -1 if none. */
MULTIFLOATS_CUDA_API int64_t mfcuda_batch_config(const mfcuda_batch *plan, int64_t i);
/* Work items of the plan's main grouped launch (tiles, diagonal items or elements). */
MULTIFLOATS_CUDA_API int64_t mfcuda_batch_work_items(const mfcuda_batch *plan);
/* Split form: the K chunk (elements) whose INT32 partials are summed in DD; -1 otherwise. */
MULTIFLOATS_CUDA_API int64_t mfcuda_batch_kchunk(const mfcuda_batch *plan);
MULTIFLOATS_CUDA_API void mfcuda_batch_destroy(mfcuda_batch *plan);
/* One-shot ragged elementwise call on a stream (no plan, no graph). */
MULTIFLOATS_CUDA_API int mfcuda_unary_dd_ragged(int op, const float64x2 *const *xs,
                                                float64x2 *const *ys, const int64_t *ns,
                                                int64_t count, void *stream);

/* ---- one process per GPU over an NCCL communicator ---------------------------
 * No reference counterpart (the reference is single-process).  nccl_comm is
 * the caller's ncclComm_t (one rank per GPU, this rank's device current);
 * NCCL is found at run time in the process (the library that created the
 * communicator), else as libnccl.so.2 -- mfcuda_nccl_available() says whether
 * it was.  Every rank makes the same calls with the same sizes, form, flags
 * and target, on streams of its own device; each call enqueues the same
 * collectives in the same order on every rank (an empty shard included) and
 * is asynchronous on the stream unless info_out is given.
 *
 * mfcuda_shard_bounds: the contiguous shard [start, stop) of n items that
 * rank `rank` of `world` owns (the first n % world ranks own one more).
 *
 * mfcuda_matmuldd_mm_nccl: C = A B (column-major DD, device pointers) in
 * column panels: this rank computes columns [j0, j1) = shard_bounds(n) of C
 * from all of A and the same columns of B.  K is never split, so every
 * output equals the single-device call of `form` bit for bit:
 *   MFCUDA_FORM_PLAIN  mfcuda_matmuldd_mm,        param = renorm_interval;
 *   MFCUDA_FORM_SPLIT  mfcuda_matmuldd_mm_split,  param = slices (0 = from target);
 *   MFCUDA_FORM_CRT    mfcuda_matmuldd_mm_crt,    param = bits (0 = from target).
 * For the split forms the ranks agree on the slice count / operand width the
 * single call derives from all of B (one MAX all-reduce of an int on the
 * stream; no host synchronisation).  flags:
 *   0                    b and c are the full k x n and m x n matrices; only
 *                        this rank's columns of B are read and of C written;
 *   MFCUDA_SHARD_PANELS  b and c hold only this rank's columns (k x (j1-j0),
 *                        m x (j1-j0));
 *   MFCUDA_SHARD_GATHER  full matrices, and afterwards every rank's c holds
 *                        all of C (each panel broadcast by its owner).
 * workspace: NULL (allocated on the stream) or at least the single call's
 * workspace size for (m, k, max panel width).  info_out: NULL or 4 ints, the
 * single call's info for this rank's panel (plan values after agreement).
 *
 * mfcuda_reduce_nccl: a reduction (kind MFCUDA_RED_*) of the array whose
 * contiguous shard of n elements this rank holds (x, y device pointers): the
 * per-shard partials (mfcuda_reduce_partial) are all-gathered in rank order
 * and folded left to right (mfcuda_reduce_combine); every rank's out (device,
 * the single call's format) receives the result, deterministic for a given
 * shard split and within the single call's error bound.
 *
 * Errors: MFCUDA_ERR_UNSUPPORTED when NCCL cannot be found, MFCUDA_ERR_CUDA
 * when an NCCL or CUDA call fails.  Argument errors are the same on every
 * rank (they depend on the common arguments only), so no rank is left
 * waiting in a collective the others skipped. */
enum { MFCUDA_SHARD_PANELS = 1, MFCUDA_SHARD_GATHER = 2 };
MULTIFLOATS_CUDA_API void mfcuda_shard_bounds(int64_t n, int rank, int world, int64_t *start, int64_t *stop);
MULTIFLOATS_CUDA_API int mfcuda_nccl_available(void);
MULTIFLOATS_CUDA_API int mfcuda_matmuldd_mm_nccl(int form, const float64x2 *a, const float64x2 *b, float64x2 *c,
                                                 int64_t m, int64_t k, int64_t n, int64_t param, double target,
                                                 int flags, void *workspace, size_t workspace_bytes,
                                                 int *info_out, void *nccl_comm, void *stream);
MULTIFLOATS_CUDA_API int mfcuda_reduce_nccl(int kind, const void *x, const void *y, int64_t n,
                                            int64_t renorm_interval, void *out, void *nccl_comm, void *stream);

/* ---- BLAS-style shims over DD matrices ------------------------------------
 * DGEMM / DTRSM argument semantics as in the reference's BLAS shims
 * test/integration/blas/wgemm.f90 and wtrsm.f90 (the `blas-multifloat`
 * library, CMakeLists.txt:377-380): column-major operands with leading
 * dimensions, transposition letters 'N' / 'T' / 'C' (C = T for real DD),
 * alpha / beta as one DD each (HOST memory), uplo 'U' / 'L', diag 'U' / 'N',
 * letters case-insensitive.  Results are bit-identical to the Fortran loops
 * with the DD operators, including the quick returns, the alpha = 0 / beta = 0
 * / beta = 1 branches (C, resp. B, is not read when beta = 0, resp. alpha = 0)
 * and the zero tests that skip a wtrsm update.
 *
 *   wgemm:  C := alpha op(A) op(B) + beta C,  op(A) m x k, op(B) k x n
 *   wtrsm:  B := alpha inv(op(A)) B  (side 'L', A m x m)  or
 *           B := alpha B inv(op(A))  (side 'R', A n x n),  A triangular
 *
 * Device-pointer forms: an invalid argument returns MFCUDA_ERR_INVALID_ARG
 * without launching anything and stores the BLAS info code (the parameter
 * position the reference hands to xerbla) in *info when info is not NULL;
 * *info = 0 otherwise. */
MULTIFLOATS_CUDA_API int mfcuda_wgemm_dd(char transa, char transb, int64_t m, int64_t n, int64_t k,
                                         const float64x2 *alpha, const float64x2 *a, int64_t lda,
                                         const float64x2 *b, int64_t ldb, const float64x2 *beta,
                                         float64x2 *c, int64_t ldc, int *info, void *stream);
MULTIFLOATS_CUDA_API int mfcuda_wtrsm_dd(char side, char uplo, char transa, char diag, int64_t m,
                                         int64_t n, const float64x2 *alpha, const float64x2 *a,
                                         int64_t lda, float64x2 *b, int64_t ldb, int *info,
                                         void *stream);
/* Fortran-callable drop-ins for the shim library's SUBROUTINE wgemm / wtrsm
 * (gfortran calling convention: every argument by reference, default INTEGER,
 * hidden CHARACTER lengths appended), HOST pointers, synchronous.  On an
 * invalid argument they call the caller's xerbla_ when one is linked (as the
 * reference does) and latch MFCUDA_ERR_INVALID_ARG in mfcuda_last_error(). */
MULTIFLOATS_CUDA_API void wgemm_(const char *transa, const char *transb, const int *m, const int *n,
                                 const int *k, const float64x2 *alpha, const float64x2 *a,
                                 const int *lda, const float64x2 *b, const int *ldb,
                                 const float64x2 *beta, float64x2 *c, const int *ldc,
                                 size_t transa_len, size_t transb_len);
MULTIFLOATS_CUDA_API void wtrsm_(const char *side, const char *uplo, const char *transa,
                                 const char *diag, const int *m, const int *n,
                                 const float64x2 *alpha, const float64x2 *a, const int *lda,
                                 float64x2 *b, const int *ldb, size_t side_len, size_t uplo_len,
                                 size_t transa_len, size_t diag_len);

/* Fixed launch geometry of the reductions for a given n (it depends on n only,
 * never on the device), exposed so a CPU restatement can follow the same order:
 * *blocks = number of thread blocks, *threads = threads per block. */
MULTIFLOATS_CUDA_API void mfcuda_reduce_geometry(int64_t n, int64_t *blocks, int64_t *threads);

#ifdef __cplusplus
}
#endif
#endif /* MULTIFLOATS_CUDA_H */
