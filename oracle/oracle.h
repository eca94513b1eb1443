/*
 * oracle.h — CPU oracle for the libthom DGEMM hot path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product path (libthom_b200/, include/, the C-ABI
 * library) links, loads or calls this code. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py use it, and only as the checker.
 *
 * What it restates (reference paths are relative to the thom-gg/libthom project root):
 *   - oracle_dgemm_naive: the reference's host check, routines/dgemm/dgemm.cpp:122-133
 *     (row-major i-j-k loop, C = alpha*sum + beta*C).
 *   - oracle_dgemm_blocked: the same contract (dgemm.h:9, dgemm.cpp:36), blocked and
 *     multithreaded; summation reordered, FMA contraction allowed.
 *   - oracle_dgemm_dot2_rows: a compensated (double-double, Ogita-Rump-Oishi 2005 "Dot2")
 *     version of the same loop for componentwise error measurement.
 *   - oracle_fill_*: the seeded counter-based input generator that replaces the reference's
 *     cuRAND fill (dgemm.cpp:100-119) so host and device produce identical inputs.
 *   - oracle_hgemm_ref: the reference's HGEMM host check, routines/hgemm/hgemm.cu:135-149 (FP16
 *     inputs widened to float, float i-j-k loop, alpha*sum + beta*C in float, one rounding to
 *     FP16), with its own FP16 <-> float conversions (oracle_half_to_float, oracle_float_to_half).
 *   - oracle_ozaki_*: a CPU restatement of this project's Ozaki INT8-slice DGEMM (no reference
 *     counterpart; the method follows Ozaki, Ogita, Oishi, Rump 2012 and Ootomo, Ozaki,
 *     Yokota 2024), bit-for-bit the same arithmetic as the CUDA path.
 *
 * Parity pin: oracle_dgemm_naive and oracle_hgemm_ref are checked bit-exactly against the
 * reference's own getReferenceResults loops (compiled from its sources into oracle/_ref by
 * oracle/Makefile) and against the golden fixtures in tests/golden/ that were produced by them.
 */
#ifndef LIBTHOM_ORACLE_H
#define LIBTHOM_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- FP16 (IEEE binary16) ---- */
float oracle_half_to_float(uint16_t h);
/* Round to nearest, ties to even; overflow to +-Inf; NaN to the canonical quiet NaN 0x7e00. */
uint16_t oracle_float_to_half(float f);
/* routines/hgemm/hgemm.cu:135-149 on FP16 bit patterns: rows `rows[0..nrows)` (all M rows when rows
 * is NULL) of C = alpha*A*B + beta*C0, written to Cout (nrows x N, or M x N). */
void oracle_hgemm_ref(const uint16_t* A, const uint16_t* B, const uint16_t* C0, uint16_t* Cout, int64_t M,
                      int64_t N, int64_t K, float alpha, float beta, const int64_t* rows, int64_t nrows);
/* Same rows in float64 with the componentwise denominator |alpha| sum |a||b| + |beta||c| (for error
 * bounds of FP32-accumulating kernels). */
void oracle_hgemm_exact_rows(const uint16_t* A, const uint16_t* B, const uint16_t* C0, double* Cexact, double* den,
                             int64_t M, int64_t N, int64_t K, double alpha, double beta, const int64_t* rows,
                             int64_t nrows);

/* ---- seeded generator ---- */
uint64_t oracle_mix64(uint64_t z);
uint64_t oracle_bits(uint64_t seed, uint64_t stream, uint64_t idx);
double oracle_uniform(uint64_t seed, uint64_t stream, uint64_t idx);
/* X[i] = u * 2^e, u ~ U[-1,1), e ~ U{-phi..phi} (e = 0 when phi == 0), i in [0, n). */
void oracle_fill(double* X, int64_t n, uint64_t seed, uint64_t stream, int phi);
/* Multiply row r (of a rows x cols row-major matrix) by 2^s_r, s_r ~ U{-smax..smax}. */
void oracle_scale_rows(double* X, int64_t rows, int64_t cols, uint64_t seed, uint64_t stream, int smax);
/* Multiply column c by 2^s_c, s_c ~ U{-smax..smax}. */
void oracle_scale_cols(double* X, int64_t rows, int64_t cols, uint64_t seed, uint64_t stream, int smax);

/* ---- FP64 GEMM oracles (row-major, C = alpha*A*B + beta*C) ---- */
void oracle_dgemm_naive(const double* A, const double* B, double* C, int M, int N, int K,
                        double alpha, double beta);
void oracle_dgemm_blocked(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                          double alpha, double beta, int nthreads);
/* For each listed row r = rows[i]: Cref[i*N + j] = round(alpha*sum_k A[r,k]B[k,j] + beta*C0[r,j]) evaluated
 * in double-double, den[i*N + j] = |alpha| sum_k |A[r,k]||B[k,j]| + |beta||C0[r,j]|. */
void oracle_dgemm_dot2_rows(const double* A, const double* B, const double* C0, double* Cref, double* den,
                            int64_t M, int64_t N, int64_t K, double alpha, double beta,
                            const int64_t* rows, int64_t nrows, int nthreads);
/* Componentwise error statistics of C (rows subset, as laid out by dot2_rows) against Cref/den.
 * out[0] = max, out[1] = median, out[2] = mean, out[3] = count of non-finite mismatches. */
void oracle_componentwise_error(const double* C, const double* Cref, const double* den, int64_t n,
                                double* out);

/* ---- Ozaki INT8-slice restatement ---- */
/* Largest INT32-safe number of (k, pair) products in one accumulator: floor((2^31-1)/127^2). */
#define ORACLE_OZAKI_KPAIR_LIMIT 131071 /* floor((2^31 - 1) / 128^2): digits are in [-128, 127] */
#define ORACLE_OZAKI_KCHUNK 32 /* K elements (bytes of an INT8 row) per MMA step */
#define ORACLE_OZAKI_BAND 4    /* diagonals whose INT32 accumulators are live together */
void oracle_ozaki_row_exponents(const double* A, int64_t M, int64_t K, int32_t* sigma);
void oracle_ozaki_col_exponents(const double* B, int64_t K, int64_t N, int32_t* tau);
/* slices[(p*M + i)*Kp + k], p in [0,s): slice p+1 of row i; zero for k >= K; Kp = K rounded up to 32. */
void oracle_ozaki_split_rows(const double* A, int64_t M, int64_t K, const int32_t* sigma, int s,
                             int8_t* slices, int64_t Kp);
/* slices[(p*N + j)*Kp + k]: slice p+1 of column j of B (K-major); zero for k >= K. */
void oracle_ozaki_split_cols(const double* B, int64_t K, int64_t N, const int32_t* tau, int s,
                             int8_t* slices, int64_t Kp);
/* Full Ozaki DGEMM, triangular pair set p+q <= s+1, same accumulation order as the CUDA path. */
void oracle_ozaki_dgemm(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                        double alpha, double beta, int s, int nthreads);
/* Analytic slice count for a target componentwise tolerance (the selector's conservative fallback);
 * gap_bits = largest exponent gap within a row of A plus the largest within a column of B. */
int oracle_ozaki_analytic_slices(double tol, int gap_bits);
int oracle_max_gap(const double* X, int64_t rows, int64_t cols, int by_rows);

/* ---- Ozaki scheme II (CRT form) restatement ---- */
/* scaling shift of one row (stride 1) or column (stride N) of K entries, chunks of `chunk` consecutive
   k (512 for the rows of A, 128 for the columns of B): trunc(a 2^s) has 2-norm at most 2^t; 0 for a
   row without nonzero entries, 0x7fffffff when it holds NaN or Inf */
int32_t oracle_crt_shift(const double* p, int64_t stride, int64_t K, int t, int64_t chunk);
void oracle_crt_row_shifts(const double* A, int64_t M, int64_t K, int t, int32_t* shift);
void oracle_crt_col_shifts(const double* B, int64_t K, int64_t N, int t, int32_t* shift);
/* residues out[(l*M + i)*Kp + k] of trunc(A[i,k] 2^shift_i) modulo mods[l] (symmetric) */
void oracle_crt_split_rows(const double* A, int64_t M, int64_t K, const int32_t* shift, int n,
                           const int32_t* mods, int8_t* out, int64_t Kp);
/* the same for the columns of B, transposed: out[(l*N + j)*Kp + k] */
void oracle_crt_split_cols(const double* B, int64_t K, int64_t N, const int32_t* shift, int n,
                           const int32_t* mods, int8_t* out, int64_t Kp);
/* Full CRT-form DGEMM with the caller's constants (n moduli, nl limbs of w bits, norm bounds 2^ta
   for the rows of A and 2^tb for the columns of B). */
void oracle_crt_dgemm(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                      double beta, int n, int nl, int w, int ta, int tb, const int32_t* mods, const double* P,
                      const double* Mk, double f_hi, double f_lo, int nthreads);

/* ---- learned slice selector restatements ---- */
void oracle_features(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol, float* feat);
void oracle_mlp_forward(const float* params, const float* x, int batch, float* probs);
double oracle_mlp_backward(const float* params, const float* x, const int* labels, int batch, double* grads);

#ifdef __cplusplus
}
#endif
#endif
