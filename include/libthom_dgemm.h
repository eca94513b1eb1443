/*
 * libthom_dgemm.h — C ABI of the sm_100a (B200) DGEMM library for libthom's `dgemm` routine.
 *
 * Every matrix is row-major and contiguous, as in the reference: A[i*K+k], B[k*N+j], C[i*N+j],
 * C = alpha*A*B + beta*C (routines/dgemm/dgemm.h:9, routines/dgemm/dgemm.cpp:36,122-133).
 * Pointers are device pointers unless a function says otherwise. When beta == 0, C is not read
 * (BLAS convention; the reference computes 0*C, which differs only if C holds NaN or Inf).
 *
 * Two families of entry points:
 *  - dgemm_<impl>(...) -> float: the reference's implementation contract (dgemm.h:9): synchronous
 *    on the legacy default stream, returns the elapsed milliseconds measured with CUDA events
 *    around every pass of the implementation. Failures are printed to stderr, as the reference
 *    wrappers do (e.g. routines/dgemm/dgemm_final.cu:204-207), and recorded for
 *    lt_get_last_error().
 *  - lt_*(...) -> int: asynchronous on the given stream (NULL = legacy default stream),
 *    returning an LT_* status code.
 */
#ifndef LIBTHOM_DGEMM_H
#define LIBTHOM_DGEMM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------------- */
#define LT_OK 0
#define LT_ERR_INVALID_ARGUMENT 1 /* bad size, null pointer, slice count out of range */
#define LT_ERR_UNALIGNED 2        /* a pointer is not 16-byte aligned where a kernel needs it */
#define LT_ERR_CUDA 3             /* a CUDA runtime call failed (message: lt_last_error_message) */
#define LT_ERR_NO_MEMORY 4        /* workspace allocation failed or a caller workspace is too small */
#define LT_ERR_DEVICE_TIMEOUT 5   /* a bounded device-side wait gave up (pipeline fault) */
#define LT_ERR_UNSUPPORTED 6      /* not an sm_100 device, or a feature missing on it */
#define LT_ERR_NOT_FOUND 7        /* unknown implementation / config name, missing file */

/* Last status recorded by any entry point of this library on the calling host thread. */
int lt_get_last_error(void);
const char* lt_error_string(int code);
const char* lt_last_error_message(void);
/* Reads (and clears) the device error words written by bounded waits inside the kernels — the
 * library's per-device word and, once lt_dgemm_ozaki_noalloc has run on the device, that entry
 * point's static word — on the current device; call after a synchronize. Allocates nothing.
 * Returns LT_OK or LT_ERR_DEVICE_TIMEOUT. */
int lt_check_device_status(void);
/* Failure-detection self-test (no reference counterpart): launches one small kernel whose wait, the
 * same bounded mbarrier wait every pipeline uses, is on a barrier that nothing arrives at, with a
 * limit of `limit_ms` (0.001 .. 1000) instead of the pipelines' 2 s. The wait gives up, records
 * LT_ERR_DEVICE_TIMEOUT with tag 99 in the device error word (read by lt_check_device_status after
 * a synchronize) and the kernel returns: the context stays usable. Nothing faults or hangs. */
int lt_selftest_wait_timeout(double limit_ms, void* stream);
int lt_version(void);

/* ---- reference-contract implementations (routines/dgemm/dgemm.h:8-42 registry entries) ------ */
/* Native FP64 tensor-core DGEMM: TMA-staged, warp-specialised DMMA (no reference counterpart;
 * replaces the reference's best kernel dgemm_final, routines/dgemm/dgemm_final.cu:175-213). */
float dgemm_tc100(const double* A, const double* B, double* C, size_t M, size_t N, size_t K,
                  double alpha, double beta);
/* Ozaki INT8-slice DGEMM with s = 3..10 slices (tcgen05 kind::i8 products, FP64 recombination). */
float dgemm_ozaki3(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);
float dgemm_ozaki4(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);
float dgemm_ozaki5(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);
float dgemm_ozaki6(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);
float dgemm_ozaki7(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);
float dgemm_ozaki8(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);
float dgemm_ozaki9(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);
float dgemm_ozaki10(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);
/* Ozaki DGEMM whose slice count is picked per call by the learned selector (analytic fallback);
 * the target tolerance is lt_set_ozaki_tolerance() (default 1e-15). */
float dgemm_ozaki_auto(const double* A, const double* B, double* C, size_t M, size_t N, size_t K,
                       double alpha, double beta);
/* DGEMM in whichever form this GPU runs faster for the shape: native FP64 or Ozaki with the
 * learned selector's slice count (lt_dgemm_auto below). No reference counterpart. */
float dgemm_auto(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha,
                 double beta);
/* The reference's cuBLAS baseline, same call (routines/dgemm/dgemm_cublas_tc.cu:4-33):
 * cublasGemmEx, CUBLAS_COMPUTE_64F, row-major through the transposition trick. */
float dgemm_cublas_tc(const double* A, const double* B, double* C, size_t M, size_t N, size_t K,
                      double alpha, double beta);

/* ---- stream-ordered API --------------------------------------------------------------------- */
/* The calls below run on `stream` (NULL = legacy default stream) and return a status. Scratch
 * memory (Ozaki slices, FP64 partial sums of the K split and stream-K schedules, packed copies) is
 * a per-device cache that the library grows on demand and keeps until exit, shared by all calls on
 * that device: calls whose work can overlap on the GPU (other streams, other host threads) must be
 * ordered by the caller, or use lt_dgemm_ozaki_ws with a workspace of their own. */
/* Native FP64 tensor-core DGEMM; the tile shape and schedule (whole tiles, K split or stream-K)
 * follow a cost model of the shape unless a tuning table holds a choice. */
int lt_dgemm_fp64(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                  double alpha, double beta, void* stream);
/* Runs one specific FP64 kernel configuration (index into lt_fp64_config_name); -1 = tuned choice. */
int lt_dgemm_fp64_config(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                         double alpha, double beta, int config, void* stream);
int lt_fp64_num_configs(void);
const char* lt_fp64_config_name(int config);

#define LT_OZAKI_MAX_SLICES 12
/* Ozaki DGEMM using the library's cached per-device workspace (grown with cudaMalloc on demand). */
int lt_dgemm_ozaki(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                   double alpha, double beta, int slices, void* stream);
/* Same, with a caller-provided device workspace of at least lt_ozaki_workspace_size() bytes,
 * 256-byte aligned. Performs no allocation. */
size_t lt_ozaki_workspace_size(int64_t M, int64_t N, int64_t K, int slices);
int lt_dgemm_ozaki_ws(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                      double alpha, double beta, int slices, void* workspace, size_t workspace_bytes,
                      void* stream);
/* The two stages of lt_dgemm_ozaki_ws, for callers that time or overlap them separately:
 * lt_ozaki_split writes the exponents and INT8 slices of A and B into the workspace;
 * lt_ozaki_product runs the tensor-core slice products and the fused FP64 recombination into C.
 * The same workspace (and M, N, K, slices) must be passed to both. */
int lt_ozaki_split(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int slices,
                   void* workspace, size_t workspace_bytes, void* stream);
int lt_ozaki_product(double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int slices,
                     const void* workspace, size_t workspace_bytes, void* stream);
int lt_dgemm_cublas(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                    double alpha, double beta, void* stream);
/* BLAS-style DGEMM on row-major matrices: C = alpha op(A) op(B) + beta C with op(X) = X ('N') or
 * X^T ('T'; 'C' is accepted as 'T'), op(A) M x K, op(B) K x N, C M x N, every matrix row-major with
 * its own row stride: A is M x K (lda >= K) or, transposed, K x M (lda >= M); B is K x N (ldb >= N)
 * or N x K (ldb >= K); ldc >= N (columns N .. ldc-1 of C are not touched). `form` LT_FORM_FP64
 * (native tensor cores; `slices` ignored) or LT_FORM_OZAKI (`slices` slices; results bit-identical
 * to lt_dgemm_ozaki on the packed op(A), op(B)). Generalises the reference's contract
 * (routines/dgemm/dgemm.h:9: packed, untransposed, tile-multiple operands only) toward a BLAS
 * dgemm(transA, transB, lda, ...). Stream-ordered; uses the cached workspaces. */
int lt_dgemm_ex(int form, char transa, char transb, int64_t M, int64_t N, int64_t K, double alpha,
                const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C, int64_t ldc,
                int slices, void* stream);
/* Ozaki DGEMM on HOST memory: A, B and C are host pointers (C holds C0 on entry when beta != 0 and
 * the result on return). Replaces the reference harness's copy-in / kernel / copy-out sequence
 * (main.cpp and routines/dgemm/dgemm.cpp:135-170 copy whole matrices before and after the call)
 * with one pipelined call: B is copied and split first, then row panels of A and C0 are copied
 * while earlier panels are split and multiplied and finished panels of C are copied back, so the
 * PCIe transfers overlap the kernels. Overlap needs page-locked host buffers (cudaMallocHost or
 * cudaHostRegister); pageable buffers work but serialise. Uses the cached device workspace, grown
 * to hold A, B and C as well. Results are bit-identical to lt_dgemm_ozaki. Synchronous: returns
 * when C is in host memory; `stream` is ordered before and after the call's work. */
int lt_dgemm_ozaki_host(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                        double alpha, double beta, int slices, void* stream);

/* Allocation-free Ozaki DGEMM. No counterpart in the reference. For callers that cannot allocate
 * device memory (a framework whose own pool owns the GPU, a service that must not allocate on its
 * request path, a process under a hard memory cap): its scratch is a fixed device array of
 * LT_OZAKI_NOALLOC_BYTES that the library holds on every GPU it is loaded on until the process exits,
 * so no call allocates or frees anything. Problems whose scratch would exceed that size
 * (lt_ozaki_workspace_size) are rejected with LT_ERR_INVALID_ARGUMENT. The first call on a device
 * looks up the array's device address (once per device). All calls on a device share the array:
 * calls whose work overlaps on the GPU (other streams, other host threads) race on it. Results are
 * bit-identical to lt_dgemm_ozaki. Stream-ordered like lt_dgemm_ozaki. */
#define LT_OZAKI_NOALLOC_BYTES (32ll << 20)
int lt_dgemm_ozaki_noalloc(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                           double alpha, double beta, int slices, void* stream);
/* Failure-detection self-test of the allocation-free path (no reference counterpart): as
 * lt_selftest_wait_timeout, but the wait that gives up reports into lt_dgemm_ozaki_noalloc's static
 * error word (set up here if no call has done it yet), which lt_check_device_status then reads. */
int lt_selftest_wait_timeout_noalloc(double limit_ms, void* stream);

/* ---- Ozaki scheme II: the CRT form (no reference counterpart) ------------------------------- */
/* C = alpha*A*B + beta*C from `moduli` INT8 tensor-core products. Each row of A and column of B is
 * scaled by a power of two, taken from an integer bound on its 2-norm, and truncated to integers V, W
 * with |V|_2 |W|_2 < Mprod / 2 (Mprod the product of the moduli), so by the Cauchy-Schwarz inequality
 * no dot product of V and W reaches Mprod / 2; each product multiplies the residues of those integers
 * modulo one of the first `moduli` of the pairwise-coprime moduli 256, 255, 253, 251, 247, 241, 239,
 * 233, 229, 227, 223, 217, 211, 199, 197, 193, 191, 181, 179, 173 exactly, and the Chinese remainder
 * theorem recovers the exact integer product, which FP64 scales back (Ozaki, Uchino and Imamura's
 * scheme II). The only error is the truncation of A and B: on U[-1,1) entries at K = 8192, 14 moduli
 * are as accurate as native FP64; each further modulus adds about 8 bits. Rows of A or columns of B
 * holding NaN or Inf give NaN in their row / column of C. K up to 8388480. Bit-identical to the CPU
 * restatement. */
#define LT_OZAKI_CRT_MIN_MODULI 8
#define LT_OZAKI_CRT_MAX_MODULI 20
/* Uses the library's cached per-device workspace (grown with cudaMalloc on demand). */
int lt_dgemm_ozaki_crt(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                       double beta, int moduli, void* stream);
/* Same with a caller-provided device workspace (256-byte aligned, at least lt_ozaki_crt_workspace_size
 * bytes); performs no allocation. */
size_t lt_ozaki_crt_workspace_size(int64_t M, int64_t N, int64_t K, int moduli);
int lt_dgemm_ozaki_crt_ws(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                          double beta, int moduli, void* workspace, size_t workspace_bytes, void* stream);
/* The two stages, for callers that time or overlap them: scaling shifts and residues of A and B into
 * the workspace; then the products, the reconstruction and the alpha/beta epilogue into C. */
int lt_ozaki_crt_split(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int moduli, void* workspace,
                       size_t workspace_bytes, void* stream);
int lt_ozaki_crt_product(double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int moduli,
                         const void* workspace, size_t workspace_bytes, void* stream);
/* lt_ozaki_crt_product in its two launches: the INT8 products into the workspace's residue planes of
 * C, then the reconstruction of C from them (with alpha and beta). */
int lt_ozaki_crt_multiply(int64_t M, int64_t N, int64_t K, int moduli, void* workspace, size_t workspace_bytes,
                          void* stream);
int lt_ozaki_crt_reconstruct(double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int moduli,
                             const void* workspace, size_t workspace_bytes, void* stream);
/* The CRT form on HOST memory (A, B, C host pointers; C holds C0 on entry when beta != 0 and the
 * result on return), the CRT counterpart of lt_dgemm_ozaki_host: B is copied and split first, then row
 * panels of A and C0 are copied while earlier panels are multiplied and finished panels of C copied
 * back. Overlap needs page-locked host buffers. Bit-identical to lt_dgemm_ozaki_crt. Synchronous. */
int lt_dgemm_ozaki_crt_host(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                            double alpha, double beta, int moduli, void* stream);
/* The norm bounds of the CRT form with `moduli` moduli (each row of A is scaled to integers of 2-norm
 * at most 2^ta, each column of B to at most 2^tb; ta + tb is the largest T with 2^T <= Mprod (1 - 2^-20)
 * / 2, Mprod the product of the moduli) and the moduli themselves (moduli_out: `moduli` ints; any
 * pointer may be NULL). Host arithmetic only. */
int lt_ozaki_crt_info(int moduli, int* ta, int* tb, int* moduli_out);
/* Reference-contract entry points (routines/dgemm/dgemm.h:9 signature) with 14..18 moduli. */
float dgemm_ozaki_crt14(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);
float dgemm_ozaki_crt15(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);
float dgemm_ozaki_crt16(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);
float dgemm_ozaki_crt17(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);
float dgemm_ozaki_crt18(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, double beta);

/* ---- automatic form ------------------------------------------------------------------------- */
/* C = alpha*A*B + beta*C at FP64 accuracy in the faster form for this call: the learned selector
 * picks the slice count s that meets lt_set_ozaki_tolerance() (default 1e-15), then a cost model of
 * this GPU (lt_dgemm_estimate_ms) compares Ozaki with s slices against native FP64. Shapes where
 * native FP64 wins even against s = 3 (small, or HBM-bound like a 65536 x 64 x 4096 product) skip
 * the selector. Results are bit-identical to lt_dgemm_fp64, or to lt_dgemm_ozaki with the chosen s.
 * `form` (LT_FORM_FP64 / LT_FORM_OZAKI) and `slices` (0 for FP64) report the choice when non-NULL.
 * Stream-ordered except that running the selector reads its answer on the host. */
int lt_dgemm_auto(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                  double beta, int* form, int* slices, void* stream);
/* The cost model's predicted milliseconds for one DGEMM on a B200 (host arithmetic only, no GPU
 * needed); -1 for an unknown form or a slice count outside 1..12. */
double lt_dgemm_estimate_ms(int form, int64_t M, int64_t N, int64_t K, int slices);

/* ---- grouped / batched DGEMM (the `dgemmb` routine) ----------------------------------------- */
typedef struct lt_gemm_problem {
  int64_t M, N, K;
  const double* A; /* device, row-major M x K */
  const double* B; /* device, row-major K x N */
  double* C;       /* device, row-major M x N */
  double alpha, beta;
} lt_gemm_problem;

#define LT_FORM_FP64 0
#define LT_FORM_OZAKI 1
typedef struct lt_grouped_plan lt_grouped_plan;
/* Builds the device-side problem table and tile queue for `count` problems (host array). */
int lt_grouped_plan_create(const lt_gemm_problem* problems, int count, int form, int slices,
                           lt_grouped_plan** plan);
/* One persistent grouped launch (FP64) or split + grouped INT8 + recombine launches (Ozaki). */
int lt_grouped_plan_run(lt_grouped_plan* plan, void* stream);
/* Captures lt_grouped_plan_run into a CUDA graph once, then replays it on `stream`. */
int lt_grouped_plan_run_graph(lt_grouped_plan* plan, void* stream);
int lt_grouped_plan_info(const lt_grouped_plan* plan, int64_t* tiles, double* flops);
/* Autotunes the plan's FP64 tile configuration on its own problems (validated against cuBLAS FP64,
 * median of `iters` timed runs, scratch outputs): every single tile shape, and two size classes
 * (problems with min(M, N) at or above a threshold of 64, 96, 192 or 384 on one configuration, the
 * rest on a smaller tile or one that runs more CTAs per SM, as two persistent launches); no-op for
 * the Ozaki form. Synchronous. Untuned plans use 64x64 tiles at two CTAs per SM for both classes
 * (TMA at min(M, N) >= 96, cp.async below). */
int lt_grouped_plan_tune(lt_grouped_plan* plan, int iters, float* best_ms);
/* Name of the kernel configuration the plan runs. */
int lt_grouped_plan_config(const lt_grouped_plan* plan, char* name, int name_len);
/* FP64 grouped tile configurations (index -> name), and setting a plan's explicitly, e.g. to
 * re-apply a tuned choice: `cfg` for problems with min(M, N) >= split_mn and `cfg_small` for the
 * others, or `cfg_small` = -1 for one configuration for all. No-op for the Ozaki form. */
int lt_grouped_num_configs(void);
const char* lt_grouped_config_name(int cfg);
int lt_grouped_plan_set_fp64(lt_grouped_plan* plan, int cfg, int cfg_small, int64_t split_mn);
void lt_grouped_plan_destroy(lt_grouped_plan* plan);
/* Convenience: create, run once, destroy. */
int lt_dgemm_grouped(const lt_gemm_problem* problems, int count, int form, int slices, void* stream);

/* ---- autotuner ------------------------------------------------------------------------------ */
typedef struct lt_tune_entry {
  int config;        /* chosen FP64 config index */
  float ms;          /* median time of the chosen config */
  float max_rel_err; /* validation error of the chosen config vs cuBLAS FP64 */
} lt_tune_entry;
/* Validates every FP64 candidate on an M x N x K problem (against cuBLAS FP64), times the valid
 * ones (median of `iters`), records the winner for the shape class and returns it. */
int lt_tune_fp64(int64_t M, int64_t N, int64_t K, int iters, lt_tune_entry* best);
int lt_tuner_save(const char* path);
int lt_tuner_load(const char* path);
int lt_tuner_lookup(int64_t M, int64_t N, int64_t K);

/* ---- learned slice-count selector ---------------------------------------------------------- */
#define LT_SEL_FEATURES 34
#define LT_SEL_HIDDEN 64
#define LT_SEL_CLASSES 8 /* slice counts 3..10 */
#define LT_SEL_PARAMS (LT_SEL_FEATURES * LT_SEL_HIDDEN + LT_SEL_HIDDEN + LT_SEL_HIDDEN * LT_SEL_HIDDEN + LT_SEL_HIDDEN + LT_SEL_HIDDEN * LT_SEL_CLASSES + LT_SEL_CLASSES)
/* Features of one problem (device output, 34 floats): 16-bin histogram of the row exponent spreads
 * of A, 16-bin histogram of the column exponent spreads of B, log2 K, log10 tol. */
int lt_ozaki_features(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol,
                      float* features, void* stream);
/* MLP 34 -> 64 -> 64 -> 8 (GELU, tanh form), softmax over slice counts 3..10. Parameters are one
 * flat float array of LT_SEL_PARAMS (W1, b1, W2, b2, W3, b3; W row-major [out][in]). */
int lt_mlp_forward(const float* params, const float* x, int batch, float* probs, void* stream);
/* One Adam step on a batch: x [batch][34], labels [batch] in 0..7; grads and moments are
 * device arrays of LT_SEL_PARAMS floats. Writes the mean cross-entropy loss to *loss (device). */
int lt_mlp_train_step(float* params, float* m, float* v, float* grads, const float* x, const int* labels,
                      int batch, float lr, int step, float* loss, void* stream);
/* Gradient only (for the gradient check against the CPU oracle). */
int lt_mlp_backward(const float* params, const float* x, const int* labels, int batch, float* grads,
                    float* loss, void* stream);
/* Installs selector weights (host array of LT_SEL_PARAMS floats) used by dgemm_ozaki_auto;
 * NULL removes them, leaving the analytic fallback. */
int lt_selector_set_params(const float* host_params);
void lt_set_ozaki_tolerance(double tol);
/* Analytic (conservative) slice count for a tolerance, where gap_bits is the largest exponent gap
 * (e(max) - e(min nonzero)) within a row of A plus the largest within a column of B. Returns 0 on
 * bad arguments. */
int lt_ozaki_analytic_slices(double tol, int gap_bits);
/* gap_bits of a problem (the analytic count's input), measured on the device. Synchronous. */
int lt_ozaki_gap_bits(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int* gap_bits,
                      void* stream);
/* Slice count the selector picks for this problem: the learned choice when weights are installed,
 * the network is confident and predicts fewer than 10 slices; the analytic count otherwise.
 * Synchronous. */
int lt_ozaki_select_slices(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol,
                           int* slices, void* stream);
/* Same, also reporting whether the learned choice was used and the measured gap_bits (-1 when the
 * learned choice was used and no gap was measured). */
int lt_ozaki_select_info(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol,
                         int* slices, int* learned, int* gap_bits, void* stream);
/* Selection on the device (no reference counterpart): a plan holds one problem's pointers and sizes
 * (the data behind them may change between runs) and a CUDA graph that runs the selector's feature
 * kernels and network, the exponent-gap pass only when the network is not confident, picks the slice
 * count on the device with the same rule as lt_ozaki_select_slices, and runs the slice form's split
 * and product for that count through a switch node. forms = LT_AUTO_PLAN_OZAKI: always the slice
 * form; LT_AUTO_PLAN_ANY_FORM: native FP64 instead wherever lt_dgemm_auto's cost model predicts it
 * faster than the chosen count (for shapes where it wins even against 3 slices the plan is the FP64
 * kernel alone, with no selection). A run is one graph launch with no host synchronisation
 * (replayable; it can be captured into a caller's graph as a child). The workspace is sized for
 * LT_OZAKI_MAX_SLICES slices. A plan's runs use its own buffers, so runs of one plan must be ordered
 * (one stream, or events); different plans may run concurrently. lt_ozaki_auto_plan_choice reads the
 * last run's choice (slices = 0: native FP64 ran; synchronous). */
#define LT_AUTO_PLAN_OZAKI 0
#define LT_AUTO_PLAN_ANY_FORM 1
typedef struct lt_ozaki_auto_plan lt_ozaki_auto_plan;
int lt_ozaki_auto_plan_create(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                              double alpha, double beta, double tol, int forms, lt_ozaki_auto_plan** plan);
int lt_ozaki_auto_plan_run(lt_ozaki_auto_plan* plan, void* stream);
int lt_ozaki_auto_plan_choice(lt_ozaki_auto_plan* plan, int* slices, int* learned);
void lt_ozaki_auto_plan_destroy(lt_ozaki_auto_plan* plan);

/* ---- harness helpers (replace the reference's cuRAND fill, routines/dgemm/dgemm.cpp:100-119) -- */
/* X[i] = u 2^e, u ~ U[-1,1), e ~ U{-phi..phi}; counter-based, identical to the CPU oracle. */
int lt_fill(double* X, int64_t n, uint64_t seed, uint64_t stream_id, int phi, void* stream);
int lt_scale_rows(double* X, int64_t rows, int64_t cols, uint64_t seed, uint64_t stream_id, int smax, void* stream);
int lt_scale_cols(double* X, int64_t rows, int64_t cols, uint64_t seed, uint64_t stream_id, int smax, void* stream);
/* Componentwise error of C against Cref with denominator den (all device, n elements):
 * out_host[0] = max |C-Cref|/den, out_host[1] = count of elements above `tol`. Synchronous. */
int lt_componentwise_error(const double* C, const double* Cref, const double* den, int64_t n, double tol,
                           double* out_host, void* stream);
/* Compensated reference of sampled rows on the device: for each of the nrows row indices in rows[]
 * (device array, each in [0, M), nrows <= 65535), Cref[i][c] = alpha*A[r]B[:,c] + beta*C0[r][c] with
 * error-free products and double-double sums in k order (Ogita-Rump-Oishi Dot2), rounded once,
 * and den[i][c] = |alpha| sum_k |A[r][k]||B[k][c]| + |beta||C0[r][c]| (nrows x N each, row-major).
 * The extension of the reference's host check (routines/dgemm/dgemm.cpp:122-159) used to measure
 * componentwise errors without the host. Asynchronous on `stream`. */
int lt_dot2_rows(const double* A, const double* B, const double* C0, double alpha, double beta, int64_t M,
                 int64_t N, int64_t K, const int64_t* rows, int64_t nrows, double* Cref, double* den, void* stream);
/* den = |alpha| |A||B| + |beta| |C0| on the device (FP64 kernel on absolute values). */
int lt_abs_denominator(const double* A, const double* B, const double* C0, double* den, int64_t M, int64_t N,
                       int64_t K, double alpha, double beta, void* stream);
/* Writes over the whole L2 (twice its size), as the reference's flushL2 (routines/common.cpp:12-24). */
int lt_flush_l2(void* stream);

/* ---- measured tensor-pipe peaks (roofline denominators; no counterpart in the reference) ------ */
#define LT_PEAK_FP64_MMA 0      /* mma.sync m16n8k16 f64, operands in registers: FP64 FLOP/s */
#define LT_PEAK_INT8_MMA_N128 1 /* tcgen05.mma kind::i8 M128 N128 K32, one CTA per SM: INT8 op/s */
#define LT_PEAK_INT8_MMA_N256 2 /* tcgen05.mma kind::i8 M128 N256 K32, one CTA per SM */
#define LT_PEAK_INT8_MMA_PAIR 3 /* tcgen05.mma.cta_group::2 kind::i8 M256 N128 K32, CTA pairs */
#define LT_PEAK_SUSTAINED 0x10  /* OR into a kind: rate after 0.5 s of back-to-back launches (power- and
                                   clock-limited), timed over the next 0.5 s; without it one launch */
/* Runs a loop of the named tensor instruction with its operands on chip (registers, or one
 * shared-memory tile per operand) on every SM and returns the measured rate of the current device
 * in *ops_per_second (2 per multiply-add). The tcgen05 kinds first run a check launch with known
 * operands and return LT_ERR_UNSUPPORTED if any accumulator checked is wrong. Synchronous. */
int lt_measure_peak(int kind, double* ops_per_second, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LIBTHOM_DGEMM_H */
