// gemm_ex.cu — lt_dgemm_ex: the BLAS-style form of the library's DGEMM on row-major matrices, with
// row strides (lda, ldb, ldc) and transposed operands, for both the native FP64 and the Ozaki form.
//
// The reference's kernels take packed, untransposed, tile-multiple operands only
// (routines/dgemm/dgemm.h:9, dgemm_final.cu:184); this is the step toward a BLAS-style
// dgemm(transA, transB, lda, ...) call. Ozaki form: transposes cost nothing (ozaki.cu, run_ex).
// FP64 form: strides go straight to the TMA tensor maps and the cp.async staging; a transposed
// operand is first written packed by a tiled transpose kernel (16 bytes of traffic per element,
// about 0.5 % of an 8192^3 product).
#include <cctype>

#include "lt_internal.h"
#include "lt_runtime.cuh"

namespace lt {
namespace {

// out (cols x rows, packed) = in^T, in being rows x cols with row stride ld. 32 x 32 tiles through
// shared memory (one column of padding against bank conflicts), 32 x 8 threads.
__global__ void transpose_kernel(const double* __restrict__ in, int64_t rows, int64_t cols, int64_t ld,
                                 double* __restrict__ out) {
  __shared__ double tile[32][33];
  const int64_t r0 = static_cast<int64_t>(blockIdx.y) * 32, c0 = static_cast<int64_t>(blockIdx.x) * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int64_t r = r0 + i, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[i][threadIdx.x] = in[r * ld + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int64_t c = c0 + i, r = r0 + threadIdx.x;
    if (c < cols && r < rows) out[c * rows + r] = tile[threadIdx.x][i];
  }
}

int transpose(const double* in, int64_t rows, int64_t cols, int64_t ld, double* out, cudaStream_t stream) {
  if (rows <= 0 || cols <= 0) return LT_OK;
  const dim3 grid(static_cast<unsigned>((cols + 31) / 32), static_cast<unsigned>((rows + 31) / 32));
  transpose_kernel<<<grid, dim3(32, 8), 0, stream>>>(in, rows, cols, ld, out);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

int parse_trans(char t, bool* trans) {
  const char u = static_cast<char>(toupper(static_cast<unsigned char>(t)));
  if (u == 'N') *trans = false;
  else if (u == 'T' || u == 'C') *trans = true;  // real data: conjugate transpose = transpose
  else return set_error(LT_ERR_INVALID_ARGUMENT, "transpose flag '%c' is not N or T", t);
  return LT_OK;
}

}  // namespace
}  // namespace lt

extern "C" int lt_dgemm_ex(int form, char transa, char transb, int64_t M, int64_t N, int64_t K, double alpha,
                           const double* A, int64_t lda, const double* B, int64_t ldb, double beta, double* C,
                           int64_t ldc, int slices, void* stream_) {
  using namespace lt;
  bool ta = false, tb = false;
  LT_TRY(parse_trans(transa, &ta));
  LT_TRY(parse_trans(transb, &tb));
  if (form != LT_FORM_FP64 && form != LT_FORM_OZAKI) return set_error(LT_ERR_INVALID_ARGUMENT, "unknown form %d", form);
  if (form == LT_FORM_OZAKI && (slices < 1 || slices > LT_OZAKI_MAX_SLICES))
    return set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d outside [1, %d]", slices, LT_OZAKI_MAX_SLICES);
  if (M < 0 || N < 0 || K < 0 || M > 0x7fffffff || N > 0x7fffffff || K > 0x7fffffff)
    return set_error(LT_ERR_INVALID_ARGUMENT, "bad dimensions");
  const int64_t a_cols = ta ? M : K, b_cols = tb ? K : N;
  if (lda < (a_cols > 1 ? a_cols : 1) || ldb < (b_cols > 1 ? b_cols : 1) || ldc < (N > 1 ? N : 1))
    return set_error(LT_ERR_INVALID_ARGUMENT, "row stride below the row length (lda %lld, ldb %lld, ldc %lld)",
                     static_cast<long long>(lda), static_cast<long long>(ldb), static_cast<long long>(ldc));
  if ((M > 0 && K > 0 && A == nullptr) || (K > 0 && N > 0 && B == nullptr) || (M > 0 && N > 0 && C == nullptr))
    return set_error(LT_ERR_INVALID_ARGUMENT, "null matrix pointer");
  if (((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(C)) & 7) != 0)
    return set_error(LT_ERR_UNALIGNED, "matrix pointers must be 8-byte aligned");
  if (M == 0 || N == 0) return ok();
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  cudaStream_t stream = as_stream(stream_);
  if (form == LT_FORM_OZAKI) {
    const size_t bytes = ozaki::workspace_size(M, N, K, slices);
    void* ws = nullptr;
    LT_TRY(ensure_workspace(ctx, bytes, &ws));
    LT_TRY(ozaki::run_ex(ta, tb, A, lda, B, ldb, C, ldc, M, N, K, alpha, beta, slices, ws, bytes, stream));
    return ok();
  }
  // FP64: transposed operands packed first.
  const double* a = A;
  const double* b = B;
  int64_t la = lda, lb = ldb;
  if ((ta || tb) && K > 0) {
    const size_t need = static_cast<size_t>((ta ? M * K : 0) + (tb ? K * N : 0));
    void* t = nullptr;
    LT_TRY(ensure_transpose_workspace(ctx, need * sizeof(double), &t));
    double* p = static_cast<double*>(t);
    if (ta) {
      LT_TRY(transpose(A, K, M, lda, p, stream));  // stored K x M -> packed M x K
      a = p;
      la = K;
      p += M * K;
    }
    if (tb) {
      LT_TRY(transpose(B, N, K, ldb, p, stream));  // stored N x K -> packed K x N
      b = p;
      lb = N;
    }
  }
  const bool tma = K > 0 && fp64::tma_compatible(a, b, lb, la);  // no tensor map over zero columns
  int cfg = tuner::lookup(M, N, K, tma);
  if (cfg < 0 || (fp64::config_is_tma(cfg) && !tma)) cfg = fp64::heuristic_config_for(M, N, K, ctx->sm_count, tma);
  LT_TRY(fp64::run_config_ld(cfg, a, la, b, lb, C, ldc, M, N, K, alpha, beta, stream));
  return ok();
}
