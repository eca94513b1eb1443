// ref_final_shim.cu — exposes the reference's best CUDA DGEMM, dgemm_final
// (routines/dgemm/dgemm_final.cu:65-213: cp.async double buffering, mma.sync m8n8k4 f64,
// 64 x 128 x 16 block tiles, 8 warps), compiled for sm_100a where it lies (include path set by
// oracle/Makefile), as a C symbol. Nothing of it is copied. Test infrastructure only: the GPU test
// that compares it with this library's kernels. The kernel needs M % 64 == 0, N % 128 == 0 and
// K % 16 == 0 (the reference's own precondition, dgemm_final.cu:184).
#define LIB_HAS_DGEMM_FINAL 1
#include "routines/dgemm/dgemm_final.cu"

extern "C" float ref_dgemm_final(const double* A, const double* B, double* C, size_t M, size_t N, size_t K,
                                 double alpha, double beta) {
  return dgemm_final(A, B, C, M, N, K, alpha, beta);
}
