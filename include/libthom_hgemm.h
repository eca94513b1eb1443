/*
 * libthom_hgemm.h — C ABI of the sm_100a (B200) HGEMM of libthom's `hgemm` routine
 * (routines/hgemm/hgemm.h:6-7, routines/hgemm/hgemm.cu:34-46), exported by the same library as
 * libthom_dgemm.h.
 *
 * Every matrix is row-major FP16 (IEEE binary16), as in the reference: A[i*K+k] (M x K),
 * B[k*N+j] (K x N), C[i*N+j] (M x N), C = alpha*A*B + beta*C. Products are accumulated in FP32 on
 * the tensor cores; the epilogue computes alpha*acc + beta*C in FP32 and rounds once to FP16, the
 * arithmetic of the reference's own host check (routines/hgemm/hgemm.cu:135-149). When beta == 0,
 * C is not read. Pointers are device pointers.
 *
 * lt_half is the 16-bit pattern of an FP16 value. The reference passes alpha and beta as CUDA
 * `__half` by value; on x86-64 and AArch64 a `__half` argument is passed exactly like a uint16_t,
 * and `__half_as_ushort` / `__ushort_as_half` convert explicitly.
 */
#ifndef LIBTHOM_HGEMM_H
#define LIBTHOM_HGEMM_H

#include <stddef.h>
#include <stdint.h>

#include "libthom_dgemm.h" /* status codes, lt_get_last_error, lt_check_device_status */

#ifdef __cplusplus
extern "C" {
#endif

typedef uint16_t lt_half;

/* ---- reference-contract implementations (routines/hgemm/hgemm.h:17-30 registry entries) ------ */
/* tcgen05 kind::f16 HGEMM: CTA-pair tiles, TMA-staged operands, FP32 accumulators in TMEM.
 * Replaces the reference's mma.sync kernels hgemm_final (routines/hgemm/hgemm_final.cu:257-294)
 * and hgemm_better_reuse (routines/hgemm/hgemm_better_reuse.cu:357-...). Synchronous on the legacy
 * default stream; returns the elapsed milliseconds of its CUDA events, prints
 * "Kernel launch error (...)" on failure like the reference wrappers. Any M, N, K. */
float hgemm_tc100(const lt_half* A, const lt_half* B, lt_half* C, size_t M, size_t N, size_t K, lt_half alpha,
                  lt_half beta);
/* The reference's cuBLAS baseline, the same call (cublasGemmEx, CUBLAS_COMPUTE_16F:
 * routines/hgemm/hgemm_cublas.cu:4-33). */
float hgemm_cublas(const lt_half* A, const lt_half* B, lt_half* C, size_t M, size_t N, size_t K, lt_half alpha,
                   lt_half beta);

/* ---- stream-ordered API --------------------------------------------------------------------- */
/* C = alpha*A*B + beta*C on `stream` (NULL = legacy default stream). Any M, N, K >= 0; pointers
 * 2-byte aligned. A and B are read through tensor maps when they are 16-byte aligned with row
 * pitches that are multiples of 8 elements; otherwise they are first packed into a cached
 * workspace with such pitches. */
int lt_hgemm(const lt_half* A, const lt_half* B, lt_half* C, int64_t M, int64_t N, int64_t K, float alpha,
             float beta, void* stream);
/* Same with an explicit tile configuration (-1 = automatic, else 0..lt_hgemm_num_configs()-1). */
int lt_hgemm_config(const lt_half* A, const lt_half* B, lt_half* C, int64_t M, int64_t N, int64_t K, float alpha,
                    float beta, int config, void* stream);
int lt_hgemm_num_configs(void);
const char* lt_hgemm_config_name(int config);
/* The configuration lt_hgemm would choose for this shape. */
int lt_hgemm_default_config(int64_t M, int64_t N, int64_t K);
/* cuBLAS baseline on `stream`: compute_f32 = 0 is the reference's call (CUBLAS_COMPUTE_16F, FP16
 * accumulation), 1 accumulates in FP32 like lt_hgemm. */
int lt_hgemm_cublas(const lt_half* A, const lt_half* B, lt_half* C, int64_t M, int64_t N, int64_t K, float alpha,
                    float beta, int compute_f32, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LIBTHOM_HGEMM_H */
