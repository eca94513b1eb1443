/*
 * oracle_blocked.c — multithreaded blocked FP64 DGEMM on the host cores (TEST INFRASTRUCTURE ONLY:
 * the fast CPU oracle and the timed host baseline; see oracle.h).
 *
 * Contract: routines/dgemm/dgemm.h:9 / dgemm.cpp:36 — row-major C = alpha*A*B + beta*C.
 * Summation order differs from the reference loop (dgemm.cpp:122-133): K is blocked and each
 * partial product is accumulated with fused multiply-add. Packing: B panels of 16 columns,
 * micro-tile 6 x 16 held in eight-wide vectors; the widest vector ISA of the running CPU is chosen
 * at load time (target_clones), so the same build runs on hosts with or without AVX-512.
 */
#include "oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef double v8d __attribute__((vector_size(64), aligned(64)));

#define MR 6
#define NR 16
#define KC 256
#define NC 512
#define MC 96

__attribute__((target_clones("arch=x86-64-v4", "arch=x86-64-v3", "default")))
static void micro_6x16(int64_t kc, const double* a, int64_t lda, const double* bp, double* t, int64_t ldt) {
  v8d c[MR][2];
  for (int r = 0; r < MR; ++r) { c[r][0] = (v8d){0}; c[r][1] = (v8d){0}; }
  for (int64_t k = 0; k < kc; ++k) {
    v8d b0, b1;
    memcpy(&b0, bp + k * NR, 64);
    memcpy(&b1, bp + k * NR + 8, 64);
    for (int r = 0; r < MR; ++r) {
      double av = a[r * lda + k];
      v8d ab = {av, av, av, av, av, av, av, av};
      c[r][0] += ab * b0;
      c[r][1] += ab * b1;
    }
  }
  for (int r = 0; r < MR; ++r) {
    v8d t0, t1;
    memcpy(&t0, t + r * ldt, 64);
    memcpy(&t1, t + r * ldt + 8, 64);
    t0 += c[r][0];
    t1 += c[r][1];
    memcpy(t + r * ldt, &t0, 64);
    memcpy(t + r * ldt + 8, &t1, 64);
  }
}

typedef struct {
  const double *A, *B;
  double* C;
  int64_t M, N, K;
  double alpha, beta;
  int tid, nthreads;
} blk_job_t;

static void* blk_worker(void* arg) {
  blk_job_t* j = (blk_job_t*)arg;
  const int64_t M = j->M, N = j->N, K = j->K;
  double* bp = (double*)aligned_alloc(64, sizeof(double) * KC * NC);
  double* T = (double*)aligned_alloc(64, sizeof(double) * MC * NC);
  int64_t nblocks = (M + MC - 1) / MC;
  for (int64_t ib = j->tid; ib < nblocks; ib += j->nthreads) {
    int64_t i0 = ib * MC, mc = (M - i0 < MC) ? M - i0 : MC;
    for (int64_t j0 = 0; j0 < N; j0 += NC) {
      int64_t nc = (N - j0 < NC) ? N - j0 : NC;
      int64_t ncfull = nc / NR * NR;
      memset(T, 0, sizeof(double) * MC * NC);
      for (int64_t p0 = 0; p0 < K; p0 += KC) {
        int64_t kc = (K - p0 < KC) ? K - p0 : KC;
        /* pack the full-width column panels of B[p0:p0+kc, j0:j0+ncfull] */
        for (int64_t jp = 0; jp < ncfull; jp += NR)
          for (int64_t k = 0; k < kc; ++k)
            memcpy(bp + jp * kc + k * NR, j->B + (p0 + k) * N + j0 + jp, sizeof(double) * NR);
        int64_t mfull = mc / MR * MR;
        for (int64_t ir = 0; ir < mfull; ir += MR)
          for (int64_t jp = 0; jp < ncfull; jp += NR)
            micro_6x16(kc, j->A + (i0 + ir) * K + p0, K, bp + jp * kc, T + ir * NC + jp, NC);
        /* ragged rows and columns */
        for (int64_t ir = 0; ir < mc; ++ir) {
          int64_t jstart = (ir < mfull) ? ncfull : 0;
          for (int64_t jj = jstart; jj < nc; ++jj) {
            double s = 0;
            for (int64_t k = 0; k < kc; ++k) s += j->A[(i0 + ir) * K + p0 + k] * j->B[(p0 + k) * N + j0 + jj];
            T[ir * NC + jj] += s;
          }
        }
      }
      for (int64_t ir = 0; ir < mc; ++ir) {
        double* crow = j->C + (i0 + ir) * N + j0;
        for (int64_t jj = 0; jj < nc; ++jj)
          crow[jj] = (j->beta != 0.0) ? j->alpha * T[ir * NC + jj] + j->beta * crow[jj] : j->alpha * T[ir * NC + jj];
      }
    }
  }
  free(bp);
  free(T);
  return NULL;
}

void oracle_dgemm_blocked(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                          double alpha, double beta, int nthreads) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  blk_job_t jobs[256];
  for (int t = 0; t < nthreads; ++t) {
    blk_job_t j = {A, B, C, M, N, K, alpha, beta, t, nthreads};
    jobs[t] = j;
    pthread_create(&th[t], NULL, blk_worker, &jobs[t]);
  }
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
}
