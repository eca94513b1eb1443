// capi.cu — extern "C" entry points of the DGEMM library: the reference-contract wrappers
// (float dgemm_<impl>(...) returning milliseconds, routines/dgemm/dgemm.h:9) and the
// stream-ordered lt_* API.
#include <cublas_v2.h>
#include <cuda_fp16.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/libthom_hgemm.h"
#include "lt_internal.h"
#include "lt_runtime.cuh"

namespace lt {
namespace {

int check_gemm_args(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K) {
  if (M < 0 || N < 0 || K < 0) return set_error(LT_ERR_INVALID_ARGUMENT, "negative dimension");
  if (M > 0x7fffffff || N > 0x7fffffff || K > 0x7fffffff)
    return set_error(LT_ERR_INVALID_ARGUMENT, "dimension above 2^31-1");
  if ((M > 0 && K > 0 && A == nullptr) || (K > 0 && N > 0 && B == nullptr) || (M > 0 && N > 0 && C == nullptr))
    return set_error(LT_ERR_INVALID_ARGUMENT, "null matrix pointer");
  if (((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(C)) & 7) != 0)
    return set_error(LT_ERR_UNALIGNED, "matrix pointers must be 8-byte aligned");
  return LT_OK;
}

std::mutex g_cublas_mutex;
cublasHandle_t g_cublas[64] = {};

int cublas_handle(cublasHandle_t* out) {
  int dev = 0;
  LT_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_cublas_mutex);
  if (g_cublas[dev] == nullptr) {
    if (cublasCreate(&g_cublas[dev]) != CUBLAS_STATUS_SUCCESS) return set_error(LT_ERR_CUDA, "cublasCreate failed");
    cublasSetMathMode(g_cublas[dev], CUBLAS_DEFAULT_MATH);
  }
  *out = g_cublas[dev];
  return LT_OK;
}

// Times `fn` on the legacy default stream with CUDA events, synchronously, as the reference's
// implementation wrappers do (e.g. routines/dgemm/dgemm_final.cu:175-213). Errors are printed and
// recorded; the elapsed time is returned regardless.
template <class F>
float timed(const char* name, F&& fn) {
  cudaEvent_t start, stop;
  cudaEventCreate(&start);
  cudaEventCreate(&stop);
  cudaEventRecord(start, 0);
  int rc = fn();
  cudaEventRecord(stop, 0);
  cudaEventSynchronize(stop);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, start, stop);
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  if (rc == LT_OK) rc = lt_check_device_status();
  if (rc != LT_OK) {
    fprintf(stderr, "Kernel launch error (%s): %s: %s\n", name, lt_error_string(rc), last_message());
    set_error(rc, "%s", last_message());
  }
  return ms;
}

}  // namespace

int dgemm_fp64_dispatch(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                        double beta, int config, cudaStream_t stream, const fp64::ScratchUse* scratch) {
  LT_TRY(check_gemm_args(A, B, C, M, N, K));
  if (M == 0 || N == 0) return ok();
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  const bool tma = K > 0 && fp64::tma_compatible(A, B, N, K);  // no tensor map over zero columns
  if (config < 0) config = tuner::lookup(M, N, K, tma);
  if (config < 0) config = fp64::heuristic_config(A, B, M, N, K, ctx->sm_count);
  if (fp64::config_is_tma(config) && !tma)
    return set_error(LT_ERR_UNALIGNED, "config %s needs 16-byte aligned A/B and even N, K", fp64::config_name(config));
  LT_TRY(fp64::run_config(config, A, B, C, M, N, K, alpha, beta, stream, scratch));
  return ok();
}

}  // namespace lt

extern "C" {

int lt_dgemm_fp64(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                  double beta, void* stream) {
  return lt::dgemm_fp64_dispatch(A, B, C, M, N, K, alpha, beta, -1, lt::as_stream(stream), nullptr);
}

int lt_dgemm_fp64_config(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                         double beta, int config, void* stream) {
  if (config >= lt::fp64::num_configs()) return lt::set_error(LT_ERR_NOT_FOUND, "no FP64 config %d", config);
  return lt::dgemm_fp64_dispatch(A, B, C, M, N, K, alpha, beta, config, lt::as_stream(stream), nullptr);
}

int lt_fp64_num_configs(void) { return lt::fp64::num_configs(); }
const char* lt_fp64_config_name(int config) { return lt::fp64::config_name(config); }

int lt_dgemm_cublas(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                    double beta, void* stream) {
  LT_TRY(lt::check_gemm_args(A, B, C, M, N, K));
  if (M == 0 || N == 0) return lt::ok();
  cublasHandle_t h;
  LT_TRY(lt::cublas_handle(&h));
  cublasSetStream(h, lt::as_stream(stream));
  // Row-major C = A B computed as column-major C^T = B^T A^T (routines/dgemm/dgemm_cublas_tc.cu:10-20).
  cublasStatus_t st = cublasGemmEx(h, CUBLAS_OP_N, CUBLAS_OP_N, static_cast<int>(N), static_cast<int>(M),
                                   static_cast<int>(K), &alpha, B, CUDA_R_64F, static_cast<int>(N > 0 ? N : 1), A,
                                   CUDA_R_64F, static_cast<int>(K > 0 ? K : 1), &beta, C, CUDA_R_64F,
                                   static_cast<int>(N > 0 ? N : 1), CUBLAS_COMPUTE_64F, CUBLAS_GEMM_DEFAULT);
  if (st != CUBLAS_STATUS_SUCCESS) return lt::set_error(LT_ERR_CUDA, "cublasGemmEx failed: %d", static_cast<int>(st));
  return lt::ok();
}

int lt_dgemm_ozaki(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                   double beta, int slices, void* stream) {
  LT_TRY(lt::check_gemm_args(A, B, C, M, N, K));
  if (slices < 1 || slices > LT_OZAKI_MAX_SLICES)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d outside [1, %d]", slices, LT_OZAKI_MAX_SLICES);
  if (M == 0 || N == 0) return lt::ok();
  lt::DeviceContext* ctx = lt::context();
  if (ctx == nullptr) return lt::last_error();
  size_t bytes = lt::ozaki::workspace_size(M, N, K, slices);
  void* ws = nullptr;
  LT_TRY(lt::ensure_workspace(ctx, bytes, &ws));
  LT_TRY(lt::ozaki::run(A, B, C, M, N, K, alpha, beta, slices, ws, bytes, lt::as_stream(stream)));
  return lt::ok();
}

int lt_dgemm_ozaki_host(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                        double beta, int slices, void* stream) {
  LT_TRY(lt::check_gemm_args(A, B, C, M, N, K));
  if (slices < 1 || slices > LT_OZAKI_MAX_SLICES)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d outside [1, %d]", slices, LT_OZAKI_MAX_SLICES);
  if (M == 0 || N == 0) return lt::ok();
  LT_TRY(lt::ozaki::host_run(A, B, C, M, N, K, alpha, beta, slices, lt::as_stream(stream)));
  return lt::ok();
}

size_t lt_ozaki_workspace_size(int64_t M, int64_t N, int64_t K, int slices) {
  if (M < 0 || N < 0 || K < 0 || slices < 1 || slices > LT_OZAKI_MAX_SLICES) return 0;
  return lt::ozaki::workspace_size(M, N, K, slices);
}

int lt_dgemm_ozaki_ws(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                      double beta, int slices, void* workspace, size_t workspace_bytes, void* stream) {
  LT_TRY(lt::check_gemm_args(A, B, C, M, N, K));
  if (slices < 1 || slices > LT_OZAKI_MAX_SLICES)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d outside [1, %d]", slices, LT_OZAKI_MAX_SLICES);
  if (M == 0 || N == 0) return lt::ok();
  size_t need = lt::ozaki::workspace_size(M, N, K, slices);
  if (workspace == nullptr || workspace_bytes < need)
    return lt::set_error(LT_ERR_NO_MEMORY, "workspace of %zu bytes given, %zu needed", workspace_bytes, need);
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
    return lt::set_error(LT_ERR_UNALIGNED, "workspace must be 256-byte aligned");
  if (lt::context() == nullptr) return lt::last_error();
  LT_TRY(lt::ozaki::run(A, B, C, M, N, K, alpha, beta, slices, workspace, workspace_bytes, lt::as_stream(stream)));
  return lt::ok();
}

static int check_ws(int64_t M, int64_t N, int64_t K, int slices, const void* workspace, size_t workspace_bytes) {
  if (M < 0 || N < 0 || K < 0) return lt::set_error(LT_ERR_INVALID_ARGUMENT, "negative dimension");
  if (slices < 1 || slices > LT_OZAKI_MAX_SLICES)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d outside [1, %d]", slices, LT_OZAKI_MAX_SLICES);
  size_t need = lt::ozaki::workspace_size(M, N, K, slices);
  if (workspace == nullptr || workspace_bytes < need)
    return lt::set_error(LT_ERR_NO_MEMORY, "workspace of %zu bytes given, %zu needed", workspace_bytes, need);
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
    return lt::set_error(LT_ERR_UNALIGNED, "workspace must be 256-byte aligned");
  return LT_OK;
}

int lt_ozaki_split(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int slices, void* workspace,
                   size_t workspace_bytes, void* stream) {
  LT_TRY(lt::check_gemm_args(A, B, reinterpret_cast<double*>(8), M, N, K));
  LT_TRY(check_ws(M, N, K, slices, workspace, workspace_bytes));
  if (M == 0 || N == 0) return lt::ok();
  LT_TRY(lt::ozaki::split(A, B, M, N, K, slices, workspace, workspace_bytes, lt::as_stream(stream)));
  return lt::ok();
}

int lt_ozaki_product(double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int slices,
                     const void* workspace, size_t workspace_bytes, void* stream) {
  LT_TRY(lt::check_gemm_args(reinterpret_cast<const double*>(8), reinterpret_cast<const double*>(8), C, M, N, K));
  LT_TRY(check_ws(M, N, K, slices, workspace, workspace_bytes));
  if (M == 0 || N == 0) return lt::ok();
  LT_TRY(lt::ozaki::product(C, M, N, K, alpha, beta, slices, workspace, workspace_bytes, lt::as_stream(stream)));
  return lt::ok();
}

// ---- reference-contract wrappers ----------------------------------------------------------------
float dgemm_tc100(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha,
                  double beta) {
  return lt::timed("tc100", [&] {
    return lt_dgemm_fp64(A, B, C, static_cast<int64_t>(M), static_cast<int64_t>(N), static_cast<int64_t>(K), alpha,
                         beta, nullptr);
  });
}

int lt_hgemm_cublas(const lt_half* A, const lt_half* B, lt_half* C, int64_t M, int64_t N, int64_t K, float alpha,
                    float beta, int compute_f32, void* stream) {
  if (M < 0 || N < 0 || K < 0 || M > 0x7fffffff || N > 0x7fffffff || K > 0x7fffffff)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "bad dimension");
  if ((M > 0 && K > 0 && A == nullptr) || (K > 0 && N > 0 && B == nullptr) || (M > 0 && N > 0 && C == nullptr))
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "null matrix pointer");
  if (M == 0 || N == 0) return lt::ok();
  cublasHandle_t h;
  LT_TRY(lt::cublas_handle(&h));
  cublasSetStream(h, lt::as_stream(stream));
  // Row-major C = A B as column-major C^T = B^T A^T (routines/hgemm/hgemm_cublas.cu:10-22).
  const __half ha = __float2half_rn(alpha), hb = __float2half_rn(beta);
  const int n = static_cast<int>(N), m = static_cast<int>(M), k = static_cast<int>(K);
  const int ldb = n > 0 ? n : 1, lda = k > 0 ? k : 1;
  cublasStatus_t st =
      compute_f32 ? cublasGemmEx(h, CUBLAS_OP_N, CUBLAS_OP_N, n, m, k, &alpha, B, CUDA_R_16F, ldb, A, CUDA_R_16F, lda,
                                 &beta, C, CUDA_R_16F, ldb, CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT)
                  : cublasGemmEx(h, CUBLAS_OP_N, CUBLAS_OP_N, n, m, k, &ha, B, CUDA_R_16F, ldb, A, CUDA_R_16F, lda,
                                 &hb, C, CUDA_R_16F, ldb, CUBLAS_COMPUTE_16F, CUBLAS_GEMM_DEFAULT);
  if (st != CUBLAS_STATUS_SUCCESS) return lt::set_error(LT_ERR_CUDA, "cublasGemmEx failed: %d", static_cast<int>(st));
  return lt::ok();
}

static float half_bits_to_float(lt_half x) { return __half2float(__ushort_as_half(x)); }

float hgemm_tc100(const lt_half* A, const lt_half* B, lt_half* C, size_t M, size_t N, size_t K, lt_half alpha,
                  lt_half beta) {
  return lt::timed("hgemm tc100", [&] {
    return lt_hgemm(A, B, C, static_cast<int64_t>(M), static_cast<int64_t>(N), static_cast<int64_t>(K),
                    half_bits_to_float(alpha), half_bits_to_float(beta), nullptr);
  });
}

float hgemm_cublas(const lt_half* A, const lt_half* B, lt_half* C, size_t M, size_t N, size_t K, lt_half alpha,
                   lt_half beta) {
  return lt::timed("hgemm cublas", [&] {
    return lt_hgemm_cublas(A, B, C, static_cast<int64_t>(M), static_cast<int64_t>(N), static_cast<int64_t>(K),
                           half_bits_to_float(alpha), half_bits_to_float(beta), 0, nullptr);
  });
}

float dgemm_cublas_tc(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha,
                      double beta) {
  return lt::timed("cublas_tc", [&] {
    return lt_dgemm_cublas(A, B, C, static_cast<int64_t>(M), static_cast<int64_t>(N), static_cast<int64_t>(K), alpha,
                           beta, nullptr);
  });
}

#define LT_OZAKI_WRAPPER(S)                                                                                    \
  float dgemm_ozaki##S(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha, \
                       double beta) {                                                                          \
    return lt::timed("ozaki" #S, [&] {                                                                         \
      return lt_dgemm_ozaki(A, B, C, static_cast<int64_t>(M), static_cast<int64_t>(N), static_cast<int64_t>(K), \
                            alpha, beta, S, nullptr);                                                          \
    });                                                                                                        \
  }
LT_OZAKI_WRAPPER(3)
LT_OZAKI_WRAPPER(4)
LT_OZAKI_WRAPPER(5)
LT_OZAKI_WRAPPER(6)
LT_OZAKI_WRAPPER(7)
LT_OZAKI_WRAPPER(8)
LT_OZAKI_WRAPPER(9)
LT_OZAKI_WRAPPER(10)
#undef LT_OZAKI_WRAPPER

#define LT_CRT_WRAPPER(NM)                                                                                  \
  float dgemm_ozaki_crt##NM(const double* A, const double* B, double* C, size_t M, size_t N, size_t K,        \
                            double alpha, double beta) {                                                   \
    return lt::timed("ozaki_crt" #NM, [&] {                                                                 \
      return lt_dgemm_ozaki_crt(A, B, C, static_cast<int64_t>(M), static_cast<int64_t>(N),                  \
                                static_cast<int64_t>(K), alpha, beta, NM, nullptr);                         \
    });                                                                                                     \
  }
LT_CRT_WRAPPER(14)
LT_CRT_WRAPPER(15)
LT_CRT_WRAPPER(16)
LT_CRT_WRAPPER(17)
LT_CRT_WRAPPER(18)
#undef LT_CRT_WRAPPER

}  // extern "C"
