/*
 * oracle.c — CPU oracle for the libthom DGEMM hot path (TEST INFRASTRUCTURE ONLY; see oracle.h).
 *
 * Compiled with -ffp-contract=off so that every a*b+c below rounds twice, exactly as written;
 * the blocked (fast) DGEMM lives in oracle_blocked.c where contraction is allowed.
 */
#include "oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------ */
/* Seeded counter-based generator. splitmix64 finaliser (Steele, Lea, Flood 2014), keyed by     */
/* (seed, stream) and indexed by element position so any element is reproducible anywhere.    */
/* The CUDA generator in libthom_b200/csrc/gen.cu computes the same bits.                      */
/* ------------------------------------------------------------------------------------------ */
uint64_t oracle_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

static uint64_t stream_key(uint64_t seed, uint64_t stream) {
  return oracle_mix64(seed ^ oracle_mix64(stream));
}

uint64_t oracle_bits(uint64_t seed, uint64_t stream, uint64_t idx) {
  return oracle_mix64(stream_key(seed, stream) + idx * 0xD1B54A32D192ED03ULL);
}

static double bits_to_uniform(uint64_t h) {
  /* 53 random bits -> k * 2^-52 - 1, exactly representable, in [-1, 1). */
  return (double)(h >> 11) * 0x1p-52 - 1.0;
}

double oracle_uniform(uint64_t seed, uint64_t stream, uint64_t idx) {
  return bits_to_uniform(oracle_bits(seed, stream, idx));
}

static int bits_to_exponent(uint64_t h, int phi) {
  if (phi <= 0) return 0;
  uint64_t e = oracle_mix64(h ^ 0x5851F42D4C957F2DULL) % (uint64_t)(2 * phi + 1);
  return (int)e - phi;
}

void oracle_fill(double* X, int64_t n, uint64_t seed, uint64_t stream, int phi) {
  uint64_t key = stream_key(seed, stream);
  for (int64_t i = 0; i < n; ++i) {
    uint64_t h = oracle_mix64(key + (uint64_t)i * 0xD1B54A32D192ED03ULL);
    X[i] = ldexp(bits_to_uniform(h), bits_to_exponent(h, phi));
  }
}

static int scale_exponent(uint64_t key, int64_t i, int smax) {
  if (smax <= 0) return 0;
  uint64_t h = oracle_mix64(key + (uint64_t)i * 0xD1B54A32D192ED03ULL);
  return (int)(h % (uint64_t)(2 * smax + 1)) - smax;
}

void oracle_scale_rows(double* X, int64_t rows, int64_t cols, uint64_t seed, uint64_t stream, int smax) {
  uint64_t key = stream_key(seed, stream);
  for (int64_t r = 0; r < rows; ++r) {
    int e = scale_exponent(key, r, smax);
    for (int64_t c = 0; c < cols; ++c) X[r * cols + c] = ldexp(X[r * cols + c], e);
  }
}

void oracle_scale_cols(double* X, int64_t rows, int64_t cols, uint64_t seed, uint64_t stream, int smax) {
  uint64_t key = stream_key(seed, stream);
  for (int64_t c = 0; c < cols; ++c) {
    int e = scale_exponent(key, c, smax);
    for (int64_t r = 0; r < rows; ++r) X[r * cols + c] = ldexp(X[r * cols + c], e);
  }
}

/* ------------------------------------------------------------------------------------------ */
/* Reference host check, restated: routines/dgemm/dgemm.cpp:122-133. Same loop order, same   */
/* operations (double sum, += a*b, then alpha*sum + beta*C), no contraction.                   */
/* ------------------------------------------------------------------------------------------ */
void oracle_dgemm_naive(const double* A, const double* B, double* C, int M, int N, int K,
                        double alpha, double beta) {
  for (int row = 0; row < M; row++) {
    for (int col = 0; col < N; col++) {
      double sum = 0;
      for (int k = 0; k < K; k++) sum += A[(int64_t)row * K + k] * B[(int64_t)k * N + col];
      C[(int64_t)row * N + col] = alpha * sum + beta * C[(int64_t)row * N + col];
    }
  }
}

/* ------------------------------------------------------------------------------------------ */
/* Double-double helpers (error-free transformations: Knuth TwoSum, FMA-based TwoProduct).    */
/* ------------------------------------------------------------------------------------------ */
typedef struct { double hi, lo; } dd_t;

static inline dd_t two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  double e = (a - (s - bb)) + (b - bb);
  dd_t r = {s, e};
  return r;
}
static inline dd_t two_prod(double a, double b) {
  double p = a * b;
  double e = fma(a, b, -p);
  dd_t r = {p, e};
  return r;
}
static inline dd_t dd_add(dd_t x, dd_t y) {
  dd_t s = two_sum(x.hi, y.hi);
  double lo = s.lo + x.lo + y.lo;
  return two_sum(s.hi, lo);
}
static inline dd_t dd_mul_d(dd_t x, double a) {
  dd_t p = two_prod(x.hi, a);
  double lo = p.lo + x.lo * a;
  return two_sum(p.hi, lo);
}

typedef struct {
  const double *A, *B, *C0;
  double *Cref, *den;
  int64_t M, N, K;
  double alpha, beta;
  const int64_t* rows;
  int64_t nrows;
  int tid, nthreads;
} dot2_job_t;

static void* dot2_worker(void* arg) {
  dot2_job_t* j = (dot2_job_t*)arg;
  const int64_t N = j->N, K = j->K;
  dd_t* acc = (dd_t*)malloc(sizeof(dd_t) * (size_t)N);
  double* aab = (double*)malloc(sizeof(double) * (size_t)N);
  for (int64_t ri = j->tid; ri < j->nrows; ri += j->nthreads) {
    int64_t r = j->rows[ri];
    for (int64_t c = 0; c < N; ++c) { acc[c].hi = 0; acc[c].lo = 0; aab[c] = 0; }
    /* i-k-j order: row r of A times B, each product error-free, sums in double-double. */
    for (int64_t k = 0; k < K; ++k) {
      double a = j->A[r * K + k];
      const double* brow = j->B + k * N;
      double aa = fabs(a);
      for (int64_t c = 0; c < N; ++c) {
        dd_t p = two_prod(a, brow[c]);
        acc[c] = dd_add(acc[c], p);
        aab[c] += aa * fabs(brow[c]);
      }
    }
    for (int64_t c = 0; c < N; ++c) {
      dd_t v = dd_mul_d(acc[c], j->alpha);
      double den = fabs(j->alpha) * aab[c];
      if (j->beta != 0.0) {
        double c0 = j->C0[r * N + c];
        v = dd_add(v, two_prod(j->beta, c0));
        den += fabs(j->beta) * fabs(c0);
      }
      j->Cref[ri * N + c] = v.hi + v.lo;
      j->den[ri * N + c] = den;
    }
  }
  free(acc);
  free(aab);
  return NULL;
}

void oracle_dgemm_dot2_rows(const double* A, const double* B, const double* C0, double* Cref, double* den,
                            int64_t M, int64_t N, int64_t K, double alpha, double beta,
                            const int64_t* rows, int64_t nrows, int nthreads) {
  (void)M;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  dot2_job_t jobs[256];
  for (int t = 0; t < nthreads; ++t) {
    dot2_job_t j = {A, B, C0, Cref, den, M, N, K, alpha, beta, rows, nrows, t, nthreads};
    jobs[t] = j;
    pthread_create(&th[t], NULL, dot2_worker, &jobs[t]);
  }
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
}

static int cmp_double(const void* a, const void* b) {
  double x = *(const double*)a, y = *(const double*)b;
  return (x > y) - (x < y);
}

void oracle_componentwise_error(const double* C, const double* Cref, const double* den, int64_t n,
                                double* out) {
  double* e = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double mx = 0, sum = 0, bad = 0;
  for (int64_t i = 0; i < n; ++i) {
    double d = fabs(C[i] - Cref[i]);
    double v;
    if (!isfinite(C[i]) || !isfinite(Cref[i])) {
      v = (C[i] == Cref[i] || (isnan(C[i]) && isnan(Cref[i]))) ? 0.0 : INFINITY;
      if (v != 0.0) bad += 1;
    } else if (den[i] > 0) {
      v = d / den[i];
    } else {
      v = (d == 0.0) ? 0.0 : INFINITY;
    }
    e[i] = v;
    if (v > mx) mx = v;
    sum += v;
  }
  qsort(e, (size_t)n, sizeof(double), cmp_double);
  out[0] = mx;
  out[1] = n > 0 ? e[n / 2] : 0.0;
  out[2] = n > 0 ? sum / (double)n : 0.0;
  out[3] = bad;
  free(e);
}

/* ------------------------------------------------------------------------------------------ */
/* Ozaki INT8-slice DGEMM restatement. Same arithmetic, same order as the CUDA kernels:       */
/*  1. sigma_i = frexp exponent of max_k |A[i,k]| (0 for an all-zero row), tau_j likewise for  */
/*     the columns of B, so |A[i,k] 2^-sigma_i| < 1.                                             */
/*  2. V = trunc(A[i,k] 2^(8s-2-sigma_i)) in balanced base-256 digits q_1..q_s (split_value),   */
/*     so A[i,k] = 2^(sigma_i+2) sum_p q_p 256^-p up to the truncation.                            */
/*  3. D = sum over pairs (p,q) with p+q = d and over a K group of q_p(A) q_q(B) in INT32.      */
/*  4. acc = sum D 2^(-8d) in the band / group / diagonal order described at ozaki_worker.        */
/*  5. C = fma(alpha, acc 2^(sigma_i+2) 2^(tau_j+2), beta*C0)   (alpha * t when beta == 0).      */
/* ------------------------------------------------------------------------------------------ */
static double pow2i(int e) {
  /* exact 2^e for e in [-1022, 1023] */
  uint64_t bits = (uint64_t)(e + 1023) << 52;
  double r;
  memcpy(&r, &bits, sizeof r);
  return r;
}

static double scale_pow2(double x, int e) {
  while (e > 1023) { x *= pow2i(1023); e -= 1023; }
  while (e < -1022) { x *= pow2i(-1022); e += 1022; }
  return x * pow2i(e);
}

static int32_t exponent_of_max(double amax) {
  if (!(amax > 0.0)) return 0;          /* zero row (or NaN: handled by NaN propagation in C) */
  if (isinf(amax)) return 0;
  int e;
  frexp(amax, &e);                       /* amax = m 2^e, m in [0.5, 1) -> amax < 2^e */
  return (int32_t)e;
}

void oracle_ozaki_row_exponents(const double* A, int64_t M, int64_t K, int32_t* sigma) {
  for (int64_t i = 0; i < M; ++i) {
    double m = 0;
    for (int64_t k = 0; k < K; ++k) { double v = fabs(A[i * K + k]); if (v > m) m = v; }
    sigma[i] = exponent_of_max(m);
  }
}

void oracle_ozaki_col_exponents(const double* B, int64_t K, int64_t N, int32_t* tau) {
  for (int64_t j = 0; j < N; ++j) {
    double m = 0;
    for (int64_t k = 0; k < K; ++k) { double v = fabs(B[k * N + j]); if (v > m) m = v; }
    tau[j] = exponent_of_max(m);
  }
}

/* Balanced base-256 digits of V = trunc(a 2^(8s-2-e)) (|V| < 2^(8s-2)), from the IEEE fields:
 * |a| = m 2^t, |V| = floor(m 2^(t-e+8s-2)). D = V + sum_{i<s-1} 128 * 256^i; digit i (0 = least
 * significant) = byte_i(D) - 128 for i < s-1 and floor(D / 256^(s-1)) (in [-64, 64]) for the top
 * one; slice p (0-based, most significant first) holds digit s-1-p. */
static void split_value(double a, int32_t e, int s, int8_t* out, int64_t stride) {
  uint64_t bits;
  memcpy(&bits, &a, sizeof bits);
  const uint64_t mag = bits & 0x7fffffffffffffffull;
  const int E = (int)(mag >> 52);
  unsigned __int128 X = 0;
  if (mag != 0 && E != 0x7ff) {
    uint64_t m = mag & 0x000fffffffffffffull;
    int t;
    if (E == 0) {
      t = -1074;
    } else {
      m |= 0x0010000000000000ull;
      t = E - 1075;
    }
    const int sh = t - e + 8 * s - 2;
    if (sh >= 0) X = (unsigned __int128)m << sh;
    else X = (-sh >= 128) ? 0 : ((unsigned __int128)m >> (-sh));
  }
  __int128 D = (bits >> 63) ? -(__int128)X : (__int128)X;
  for (int i = 0; i < s - 1; ++i) D += (__int128)128 << (8 * i);
  for (int i = 0; i < s; ++i) {
    const uint8_t byte = (uint8_t)(D >> (8 * i));
    out[(s - 1 - i) * stride] = (int8_t)(i < s - 1 ? (uint8_t)(byte ^ 0x80u) : byte);
  }
}

void oracle_ozaki_split_rows(const double* A, int64_t M, int64_t K, const int32_t* sigma, int s,
                             int8_t* slices, int64_t Kp) {
  memset(slices, 0, (size_t)(s * M * Kp));
  for (int64_t i = 0; i < M; ++i)
    for (int64_t k = 0; k < K; ++k)
      split_value(A[i * K + k], sigma[i], s, slices + i * Kp + k, M * Kp);
}

void oracle_ozaki_split_cols(const double* B, int64_t K, int64_t N, const int32_t* tau, int s,
                             int8_t* slices, int64_t Kp) {
  memset(slices, 0, (size_t)(s * N * Kp));
  for (int64_t k = 0; k < K; ++k)
    for (int64_t j = 0; j < N; ++j)
      split_value(B[k * N + j], tau[j], s, slices + j * Kp + k, N * Kp);
}

typedef struct {
  const int8_t *sa, *sb;
  const int32_t *sigma, *tau;
  const double *A, *B;
  double* C;
  int64_t M, N, K, Kp;
  double alpha, beta;
  int s, tid, nthreads;
} ozaki_job_t;

/* Band schedule shared with the CUDA kernel: diagonals d = s+1 .. 2 are taken in bands of
 * ORACLE_OZAKI_BAND consecutive diagonals (highest first); each band runs over K in 32-byte chunks,
 * split into groups whose INT32 sums cannot overflow: a group holds
 * floor(ORACLE_OZAKI_KPAIR_LIMIT / (32 * max pairs of a diagonal in the band)) chunks.
 * FP64 accumulation order: band, then group, then diagonal (highest first). */
static void* ozaki_worker(void* arg) {
  ozaki_job_t* j = (ozaki_job_t*)arg;
  const int s = j->s;
  const int64_t M = j->M, N = j->N, K = j->K, Kp = j->Kp;
  const int64_t nkc = Kp / ORACLE_OZAKI_KCHUNK;
  for (int64_t i = j->tid; i < M; i += j->nthreads) {
    int row_bad = 0;
    for (int64_t k = 0; k < K; ++k) if (!isfinite(j->A[i * K + k])) { row_bad = 1; break; }
    for (int64_t c = 0; c < N; ++c) {
      int col_bad = row_bad;
      if (!col_bad) for (int64_t k = 0; k < K; ++k) if (!isfinite(j->B[k * N + c])) { col_bad = 1; break; }
      double acc = 0.0;
      for (int dhi = s + 1; dhi >= 2; dhi -= ORACLE_OZAKI_BAND) {
        int dlo = dhi - ORACLE_OZAKI_BAND + 1 < 2 ? 2 : dhi - ORACLE_OZAKI_BAND + 1;
        int maxp = 0;
        for (int d = dhi; d >= dlo; --d) {
          int plo = d - s > 1 ? d - s : 1, phi = d - 1 < s ? d - 1 : s;
          if (phi - plo + 1 > maxp) maxp = phi - plo + 1;
        }
        int64_t gchunks = ORACLE_OZAKI_KPAIR_LIMIT / (ORACLE_OZAKI_KCHUNK * maxp);
        for (int64_t c0 = 0; c0 < nkc; c0 += gchunks) {
          int64_t c1 = c0 + gchunks < nkc ? c0 + gchunks : nkc;
          int64_t k0 = c0 * ORACLE_OZAKI_KCHUNK, k1 = c1 * ORACLE_OZAKI_KCHUNK;
          for (int d = dhi; d >= dlo; --d) {
            int plo = d - s > 1 ? d - s : 1, phi = d - 1 < s ? d - 1 : s;
            int32_t D = 0;
            for (int p = plo; p <= phi; ++p) {
              int q = d - p;
              const int8_t* ar = j->sa + ((int64_t)(p - 1) * M + i) * Kp;
              const int8_t* bc = j->sb + ((int64_t)(q - 1) * N + c) * Kp;
              for (int64_t k = k0; k < k1; ++k) D += (int32_t)ar[k] * (int32_t)bc[k];
            }
            acc = acc + (double)D * pow2i(-8 * d);
          }
        }
      }
      double t = scale_pow2(scale_pow2(acc, j->sigma[i] + 2), j->tau[c] + 2);
      double out;
      if (j->beta != 0.0) out = fma(j->alpha, t, j->beta * j->C[i * N + c]);
      else out = j->alpha * t;
      if (col_bad) out = NAN;
      j->C[i * N + c] = out;
    }
  }
  return NULL;
}

void oracle_ozaki_dgemm(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                        double alpha, double beta, int s, int nthreads) {
  int64_t Kp = (K + ORACLE_OZAKI_KCHUNK - 1) / ORACLE_OZAKI_KCHUNK * ORACLE_OZAKI_KCHUNK;
  int32_t* sigma = (int32_t*)malloc(sizeof(int32_t) * (size_t)(M > 0 ? M : 1));
  int32_t* tau = (int32_t*)malloc(sizeof(int32_t) * (size_t)(N > 0 ? N : 1));
  int8_t* sa = (int8_t*)malloc((size_t)(s * M * Kp + 1));
  int8_t* sb = (int8_t*)malloc((size_t)(s * N * Kp + 1));
  oracle_ozaki_row_exponents(A, M, K, sigma);
  oracle_ozaki_col_exponents(B, K, N, tau);
  oracle_ozaki_split_rows(A, M, K, sigma, s, sa, Kp);
  oracle_ozaki_split_cols(B, K, N, tau, s, sb, Kp);
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  ozaki_job_t jobs[256];
  for (int t = 0; t < nthreads; ++t) {
    ozaki_job_t j = {sa, sb, sigma, tau, A, B, C, M, N, K, Kp, alpha, beta, s, t, nthreads};
    jobs[t] = j;
    pthread_create(&th[t], NULL, ozaki_worker, &jobs[t]);
  }
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  free(sigma); free(tau); free(sa); free(sb);
}

/* Conservative slice count (same rule as the library's selector fallback). gap_bits = largest
 * exponent gap e(max) - e(min nonzero) within a row of A plus the largest within a column of B. An
 * entry with gap g keeps at least 8s - 2 - g - 1 bits after truncation, so the two truncated tails
 * and the dropped pairs p + q > s + 1 bound the componentwise error by (s + 3) 2^(gap_bits + 4 - 8s);
 * the FP64 recombination and epilogue add at most 4u. The smallest s in [1, 12] meeting tol. */
int oracle_ozaki_analytic_slices(double tol, int gap_bits) {
  for (int s = 1; s <= 12; ++s) {
    double bound = (double)(s + 3) * ldexp(1.0, gap_bits + 4 - 8 * s) + 4.0 * ldexp(1.0, -53);
    if (bound <= tol) return s;
  }
  return 12;
}

/* Largest exponent gap of any row (by_rows) or column of a rows x cols row-major matrix. */
int oracle_max_gap(const double* X, int64_t rows, int64_t cols, int by_rows) {
  int best = 0;
  int64_t outer = by_rows ? rows : cols, inner = by_rows ? cols : rows;
  for (int64_t o = 0; o < outer; ++o) {
    int emax = -100000, emin = 100000;
    for (int64_t i = 0; i < inner; ++i) {
      double v = fabs(by_rows ? X[o * cols + i] : X[i * cols + o]);
      if (v != 0.0 && isfinite(v)) {
        int e;
        frexp(v, &e);
        if (e > emax) emax = e;
        if (e < emin) emin = e;
      }
    }
    if (emax >= emin && emax - emin > best) best = emax - emin;
  }
  return best;
}

/* ------------------------------------------------------------------------------------------ */
/* Selector restatements: features and the 34-64-64-8 GELU MLP (forward, backward), in double. */
/* ------------------------------------------------------------------------------------------ */
static int gap_bin(int g) { return g >= 60 ? 15 : (g < 0 ? 0 : g >> 2); }

void oracle_features(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol, float* feat) {
  double hist[32];
  memset(hist, 0, sizeof hist);
  int rows = (int)(M < 128 ? M : 128);
  for (int r = 0; r < rows; ++r) {
    int64_t row = rows > 1 ? ((int64_t)r * (M - 1)) / (rows - 1) : 0;
    int em = -100000;
    for (int64_t k = 0; k < K; ++k) {
      double v = fabs(A[row * K + k]);
      if (v != 0.0 && isfinite(v)) { int e; frexp(v, &e); if (e > em) em = e; }
    }
    for (int64_t k = 0; k < K; ++k) {
      double v = fabs(A[row * K + k]);
      int b = 0;
      if (v != 0.0 && isfinite(v)) { int e; frexp(v, &e); b = gap_bin(em - e); }
      hist[b] += 1;
    }
  }
  int groups = (int)((N + 31) / 32 < 4 ? (N + 31) / 32 : 4);
  int64_t span = N > 32 ? N - 32 : 0;
  for (int gI = 0; gI < groups; ++gI) {
    int64_t c0 = groups > 1 ? ((int64_t)gI * span) / (groups - 1) : 0;
    for (int l = 0; l < 32; ++l) {
      int64_t col = c0 + l;
      if (col >= N) continue;
      int em = -100000;
      for (int64_t k = 0; k < K; ++k) {
        double v = fabs(B[k * N + col]);
        if (v != 0.0 && isfinite(v)) { int e; frexp(v, &e); if (e > em) em = e; }
      }
      for (int64_t k = 0; k < K; ++k) {
        double v = fabs(B[k * N + col]);
        int b = 0;
        if (v != 0.0 && isfinite(v)) { int e; frexp(v, &e); b = gap_bin(em - e); }
        hist[16 + b] += 1;
      }
    }
  }
  for (int h = 0; h < 2; ++h) {
    double tot = 0;
    for (int i = 0; i < 16; ++i) tot += hist[16 * h + i];
    for (int i = 0; i < 16; ++i) feat[16 * h + i] = tot > 0 ? (float)(hist[16 * h + i] / tot) : 0.f;
  }
  feat[32] = (float)(log2((double)(K > 0 ? K : 1)) / 16.0);
  feat[33] = (float)(-log10(tol) / 16.0);
}

#define SEL_F 34
#define SEL_H 64
#define SEL_C 8
#define OW1 0
#define OB1 (OW1 + SEL_H * SEL_F)
#define OW2 (OB1 + SEL_H)
#define OB2 (OW2 + SEL_H * SEL_H)
#define OW3 (OB2 + SEL_H)
#define OB3 (OW3 + SEL_C * SEL_H)
#define SEL_P (OB3 + SEL_C)

static double gelu_d(double x) {
  const double k = 0.7978845608028654;
  return 0.5 * x * (1.0 + tanh(k * (x + 0.044715 * x * x * x)));
}
static double gelu_grad_d(double x) {
  const double k = 0.7978845608028654;
  double t = tanh(k * (x + 0.044715 * x * x * x));
  return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * k * (1.0 + 3.0 * 0.044715 * x * x);
}

static void mlp_fwd1(const float* p, const float* x, double* h1, double* a1, double* h2, double* a2, double* prob) {
  for (int j = 0; j < SEL_H; ++j) {
    double acc = p[OB1 + j];
    for (int i = 0; i < SEL_F; ++i) acc += (double)p[OW1 + j * SEL_F + i] * x[i];
    h1[j] = acc; a1[j] = gelu_d(acc);
  }
  for (int j = 0; j < SEL_H; ++j) {
    double acc = p[OB2 + j];
    for (int i = 0; i < SEL_H; ++i) acc += (double)p[OW2 + j * SEL_H + i] * a1[i];
    h2[j] = acc; a2[j] = gelu_d(acc);
  }
  double lg[SEL_C], mx = -1e300, sum = 0;
  for (int c = 0; c < SEL_C; ++c) {
    double acc = p[OB3 + c];
    for (int i = 0; i < SEL_H; ++i) acc += (double)p[OW3 + c * SEL_H + i] * a2[i];
    lg[c] = acc; if (acc > mx) mx = acc;
  }
  for (int c = 0; c < SEL_C; ++c) { prob[c] = exp(lg[c] - mx); sum += prob[c]; }
  for (int c = 0; c < SEL_C; ++c) prob[c] /= sum;
}

void oracle_mlp_forward(const float* params, const float* x, int batch, float* probs) {
  double h1[SEL_H], a1[SEL_H], h2[SEL_H], a2[SEL_H], pr[SEL_C];
  for (int b = 0; b < batch; ++b) {
    mlp_fwd1(params, x + (int64_t)b * SEL_F, h1, a1, h2, a2, pr);
    for (int c = 0; c < SEL_C; ++c) probs[(int64_t)b * SEL_C + c] = (float)pr[c];
  }
}

/* Mean cross-entropy gradient over the batch (double accumulation); returns the mean loss. */
double oracle_mlp_backward(const float* p, const float* x, const int* labels, int batch, double* grads) {
  double h1[SEL_H], a1[SEL_H], h2[SEL_H], a2[SEL_H], pr[SEL_C], d3[SEL_C], d2[SEL_H], d1[SEL_H];
  double loss = 0;
  memset(grads, 0, sizeof(double) * SEL_P);
  for (int b = 0; b < batch; ++b) {
    const float* xb = x + (int64_t)b * SEL_F;
    mlp_fwd1(p, xb, h1, a1, h2, a2, pr);
    int y = labels[b];
    loss += -log(pr[y] > 1e-30 ? pr[y] : 1e-30);
    for (int c = 0; c < SEL_C; ++c) d3[c] = pr[c] - (c == y ? 1.0 : 0.0);
    for (int c = 0; c < SEL_C; ++c) {
      for (int i = 0; i < SEL_H; ++i) grads[OW3 + c * SEL_H + i] += d3[c] * a2[i];
      grads[OB3 + c] += d3[c];
    }
    for (int i = 0; i < SEL_H; ++i) {
      double acc = 0;
      for (int c = 0; c < SEL_C; ++c) acc += (double)p[OW3 + c * SEL_H + i] * d3[c];
      d2[i] = acc * gelu_grad_d(h2[i]);
    }
    for (int j = 0; j < SEL_H; ++j) {
      for (int i = 0; i < SEL_H; ++i) grads[OW2 + j * SEL_H + i] += d2[j] * a1[i];
      grads[OB2 + j] += d2[j];
    }
    for (int i = 0; i < SEL_H; ++i) {
      double acc = 0;
      for (int j = 0; j < SEL_H; ++j) acc += (double)p[OW2 + j * SEL_H + i] * d2[j];
      d1[i] = acc * gelu_grad_d(h1[i]);
    }
    for (int j = 0; j < SEL_H; ++j) {
      for (int i = 0; i < SEL_F; ++i) grads[OW1 + j * SEL_F + i] += d1[j] * xb[i];
      grads[OB1 + j] += d1[j];
    }
  }
  for (int i = 0; i < SEL_P; ++i) grads[i] /= batch;
  return loss / batch;
}

/* ------------------------------------------------------------------------------------------------
 * FP16 HGEMM host check (routines/hgemm/hgemm.cu:135-149): float accumulation in k order,
 * res = alpha*sum + beta*C in float (no contraction), one rounding to FP16.
 * ---------------------------------------------------------------------------------------------- */
float oracle_half_to_float(uint16_t h) {
  const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
  const uint32_t e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
  float f;
  if (e == 0) {
    f = ldexpf((float)m, -24); /* zero or subnormal: m * 2^-24, exact */
    return sign ? -f : f;
  }
  uint32_t bits;
  if (e == 31) bits = sign | 0x7f800000u | (m << 13); /* Inf, NaN (payload kept) */
  else bits = sign | ((e + 112u) << 23) | (m << 13);
  memcpy(&f, &bits, sizeof f);
  return f;
}

uint16_t oracle_float_to_half(float f) {
  uint32_t x;
  memcpy(&x, &f, sizeof x);
  const uint16_t sign = (uint16_t)((x >> 16) & 0x8000u);
  const uint32_t ax = x & 0x7fffffffu;
  if (ax > 0x7f800000u) return sign | 0x7e00u;  /* NaN */
  if (ax >= 0x477ff000u) return sign | 0x7c00u; /* >= 65520 (Inf included) rounds to Inf */
  if (ax >= 0x38800000u) {                      /* normal half: rebias, round mantissa to 10 bits */
    uint32_t r = ax - (112u << 23);
    r += 0xfffu + ((r >> 13) & 1u);
    return sign | (uint16_t)(r >> 13);
  }
  /* subnormal half (or zero): round(|f| * 2^24) to an integer in [0, 1024] */
  const int e = (int)(ax >> 23);
  const int s = 126 - e; /* |f| * 2^24 = mant24 >> s */
  if (e == 0 || s > 24) return sign;
  const uint32_t mant = (ax & 0x7fffffu) | 0x800000u;
  uint32_t q = mant >> s;
  const uint32_t rem = mant & ((1u << s) - 1u), halfway = 1u << (s - 1);
  if (rem > halfway || (rem == halfway && (q & 1u))) ++q;
  return sign | (uint16_t)q;
}

void oracle_hgemm_ref(const uint16_t* A, const uint16_t* B, const uint16_t* C0, uint16_t* Cout, int64_t M,
                      int64_t N, int64_t K, float alpha, float beta, const int64_t* rows, int64_t nrows) {
  const int64_t nr = rows ? nrows : M;
  for (int64_t i = 0; i < nr; ++i) {
    const int64_t row = rows ? rows[i] : i;
    for (int64_t col = 0; col < N; ++col) {
      float sum = 0.0f;
      for (int64_t k = 0; k < K; ++k)
        sum += oracle_half_to_float(A[row * K + k]) * oracle_half_to_float(B[k * N + col]);
      const float res = alpha * sum + beta * oracle_half_to_float(C0[row * N + col]);
      Cout[i * N + col] = oracle_float_to_half(res);
    }
  }
}

void oracle_hgemm_exact_rows(const uint16_t* A, const uint16_t* B, const uint16_t* C0, double* Cexact, double* den,
                             int64_t M, int64_t N, int64_t K, double alpha, double beta, const int64_t* rows,
                             int64_t nrows) {
  const int64_t nr = rows ? nrows : M;
  for (int64_t i = 0; i < nr; ++i) {
    const int64_t row = rows ? rows[i] : i;
    for (int64_t col = 0; col < N; ++col) {
      /* products of FP16 values are exact in double; the double sum's rounding error (about
       * K * 2^-53 relative to den) is far below FP32 and FP16 resolution */
      double s = 0.0, a = 0.0;
      for (int64_t k = 0; k < K; ++k) {
        const double p = (double)oracle_half_to_float(A[row * K + k]) * (double)oracle_half_to_float(B[k * N + col]);
        s += p;
        a += fabs(p);
      }
      const double c = (double)oracle_half_to_float(C0[row * N + col]);
      Cexact[i * N + col] = alpha * s + beta * c;
      den[i * N + col] = fabs(alpha) * a + fabs(beta) * fabs(c);
    }
  }
}

/* ------------------------------------------------------------------------------------------ */
/* Ozaki scheme II restated (integer residues and the Chinese remainder theorem), the arithmetic  */
/* of the library's CRT form (no reference counterpart; the reference's DGEMM contract is        */
/* routines/dgemm/dgemm.h:9, its host check routines/dgemm/dgemm.cpp:122-133):                    */
/*  1. Scaling by a bound on each row's (column's) 2-norm. Per entry a != 0: e = its frexp        */
/*     exponent and x = floor(|a| 2^(15-e)) + 1 (subnormals: e = -1021, x = 2^14 + 1), so         */
/*     |a| < x 2^(e-15). Per chunk (512 consecutive k of a row of A, 128 of a column of B):       */
/*     E_c = the largest e, S_c = the sum of ceil(x^2 4^(e-E_c)); per row: sigma = the largest    */
/*     E_c, S = the sum over chunks of ceil(S_c / 4^(sigma-E_c)) (integer sums: their order is    */
/*     immaterial), so that |row|_2^2 < S 2^(2 sigma - 30). The shift                            */
/*     s = t + 15 - sigma - ceil(bitlen(S - 1) / 2) makes V = trunc(a 2^s) satisfy |V|_2 <= 2^t;  */
/*     a row without nonzero entries takes s = 0, one holding NaN or Inf the sentinel 0x7fffffff. */
/*  2. t = ta for the rows of A, tb for the columns of B: ta + tb = Tc, the largest integer with  */
/*     2^Tc <= Mprod (1 - 2^-20) / 2 (Mprod = product of the moduli), split evenly, each at most  */
/*     62. By the Cauchy-Schwarz inequality |sum_k V W| <= |V|_2 |W|_2 <= 2^Tc < Mprod / 2, with   */
/*     a margin of 2^-21 Mprod for the rounding of the quotient estimate in step 4.              */
/*  3. For each modulus m_l: symmetric residues of V and W, their exact integer product over K,  */
/*     reduced to its residue r_l in [0, m_l).                                                    */
/*  4. C' = the integer in (-Mprod/2, Mprod/2) with C' = r_l mod m_l, through FP64 limb sums:      */
/*     L_k = K_k + sum_l r_l P_lk (exact; K_k = -128 sum_l P_lk, +128 in limb 0, keeps them below */
/*     2^53), Q = rint(L_hi F_hi + L_lo F_lo), D_k = fma(-Q, M_k, L_k),                           */
/*     t = Horner of the D_k in base 2^w. The constants (moduli, limbs P_lk of the CRT basis,     */
/*     limbs M_k of Mprod, F = 2^(w k) / Mprod) come from the caller (oracle/__init__.py derives  */
/*     them with exact integer arithmetic).                                                        */
/*  5. C = fma(alpha, t 2^(-s_i) 2^(-s_j), beta*C0)  (alpha * that when beta == 0); NaN where the */
/*     row of A or the column of B holds NaN or Inf.                                              */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  int n, nl, w;
  const int32_t* mods;   /* n moduli */
  const double* P;       /* n x nl limbs of the CRT basis P_l = (Mprod/m_l) ((Mprod/m_l)^-1 mod m_l) */
  const double* Mk;      /* nl limbs of Mprod */
  double f_hi, f_lo;     /* 2^(w (nl-1)) / Mprod_d and 2^(w (nl-2)) / Mprod_d */
} crt_consts_t;

#define CRT_CHUNK_ROWS 512 /* chunk of a row of A */
#define CRT_CHUNK_COLS 128 /* chunk of a column of B */
#define CRT_BAD 0x7fffffff
#define CRT_EMPTY INT32_MIN

/* exponent e and 15-bit bound x of a finite nonzero a: |a| < x 2^(e-15) */
static void crt_entry_bound(double a, int* e, uint64_t* x) {
  uint64_t bits;
  memcpy(&bits, &a, sizeof bits);
  const int E = (int)((bits >> 52) & 0x7ff);
  if (E == 0) {
    *e = -1021;
    *x = (1u << 14) + 1;
  } else {
    *e = E - 1022;
    *x = (1u << 14) + ((bits & 0x000fffffffffffffull) >> 38) + 1;
  }
}

/* ceil(v / 2^d) for d >= 0 and v < 2^62 */
static uint64_t crt_ceil_shr(uint64_t v, int d) {
  if (d == 0) return v;
  if (d >= 63) return v != 0;
  return (v + ((1ull << d) - 1)) >> d;
}

/* The scaling shift of one row (stride 1) or column (stride N) of K entries for the bound 2^t, with
   chunks of `chunk` consecutive k */
int32_t oracle_crt_shift(const double* p, int64_t stride, int64_t K, int t, int64_t chunk) {
  const int64_t nch = (K + chunk - 1) / chunk;
  int32_t sigma = CRT_EMPTY;
  uint64_t S = 0;
  int32_t* Ec = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nch > 0 ? nch : 1));
  uint64_t* Sc = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(nch > 0 ? nch : 1));
  for (int64_t c = 0; c < nch; ++c) {
    const int64_t k1 = (c + 1) * chunk < K ? (c + 1) * chunk : K;
    int32_t E = CRT_EMPTY;
    for (int64_t k = c * chunk; k < k1; ++k) {
      const double a = p[k * stride];
      if (!isfinite(a)) { free(Ec); free(Sc); return CRT_BAD; }
      if (a != 0.0) {
        int e;
        uint64_t x;
        crt_entry_bound(a, &e, &x);
        if (e > E) E = e;
      }
    }
    uint64_t sum = 0;
    if (E != CRT_EMPTY) {
      for (int64_t k = c * chunk; k < k1; ++k) {
        const double a = p[k * stride];
        if (a == 0.0) continue;
        int e;
        uint64_t x;
        crt_entry_bound(a, &e, &x);
        sum += crt_ceil_shr(x * x, 2 * (E - e));
      }
    }
    Ec[c] = E;
    Sc[c] = sum;
    if (E > sigma) sigma = E;
  }
  if (sigma != CRT_EMPTY)
    for (int64_t c = 0; c < nch; ++c)
      if (Ec[c] != CRT_EMPTY) S += crt_ceil_shr(Sc[c], 2 * (sigma - Ec[c]));
  free(Ec);
  free(Sc);
  if (sigma == CRT_EMPTY) return 0;
  int b = 0;
  while (b < 64 && ((S - 1) >> b) != 0) ++b; /* bitlen(S - 1) */
  return t + 15 - sigma - (b + 1) / 2;
}

void oracle_crt_row_shifts(const double* A, int64_t M, int64_t K, int t, int32_t* shift) {
  for (int64_t i = 0; i < M; ++i) shift[i] = oracle_crt_shift(A + i * K, 1, K, t, CRT_CHUNK_ROWS);
}

void oracle_crt_col_shifts(const double* B, int64_t K, int64_t N, int t, int32_t* shift) {
  for (int64_t j = 0; j < N; ++j) shift[j] = oracle_crt_shift(B + j, N, K, t, CRT_CHUNK_COLS);
}

/* trunc(a 2^s) from the IEEE fields (|result| <= 2^62 under the shifts above); zero for zero */
static int64_t crt_scaled_int(double a, int32_t s) {
  uint64_t bits;
  memcpy(&bits, &a, sizeof bits);
  const uint64_t mag = bits & 0x7fffffffffffffffull;
  const int E = (int)(mag >> 52);
  if (mag == 0 || E == 0x7ff) return 0;
  uint64_t m = mag & 0x000fffffffffffffull;
  int t;
  if (E == 0) {
    t = -1074;
  } else {
    m |= 0x0010000000000000ull;
    t = E - 1075;
  }
  const int sh = t + s;
  uint64_t X;
  if (sh >= 0) X = m << sh;
  else X = (-sh >= 64) ? 0 : (m >> (-sh));
  return (bits >> 63) ? -(int64_t)X : (int64_t)X;
}

/* symmetric residue: [-(m-1)/2, (m-1)/2] for odd m, [-128, 127] for m = 256 */
static int32_t crt_residue(int64_t v, int32_t m) {
  int64_t r = v % m;
  if (r < 0) r += m;
  if (m == 256) return r >= 128 ? (int32_t)(r - 256) : (int32_t)r;
  return r > m / 2 ? (int32_t)(r - m) : (int32_t)r;
}

/* residues of the scaled rows of A: out[l][i][k] (Kp >= K, zero padded) */
void oracle_crt_split_rows(const double* A, int64_t M, int64_t K, const int32_t* shift, int n,
                           const int32_t* mods, int8_t* out, int64_t Kp) {
  memset(out, 0, (size_t)(n * M * Kp));
  for (int64_t i = 0; i < M; ++i) {
    if (shift[i] == CRT_BAD) continue;
    for (int64_t k = 0; k < K; ++k) {
      const int64_t v = crt_scaled_int(A[i * K + k], shift[i]);
      for (int l = 0; l < n; ++l) out[((int64_t)l * M + i) * Kp + k] = (int8_t)crt_residue(v, mods[l]);
    }
  }
}

/* residues of the scaled columns of B, transposed: out[l][j][k] */
void oracle_crt_split_cols(const double* B, int64_t K, int64_t N, const int32_t* shift, int n,
                           const int32_t* mods, int8_t* out, int64_t Kp) {
  memset(out, 0, (size_t)(n * N * Kp));
  for (int64_t j = 0; j < N; ++j) {
    if (shift[j] == CRT_BAD) continue;
    for (int64_t k = 0; k < K; ++k) {
      const int64_t v = crt_scaled_int(B[k * N + j], shift[j]);
      for (int l = 0; l < n; ++l) out[((int64_t)l * N + j) * Kp + k] = (int8_t)crt_residue(v, mods[l]);
    }
  }
}

/* C' (as a double) from the residues r[0..n-1] in [0, m_l): the limb sums start from
   K_k = -128 sum_l P_lk (+128 in limb 0), so that L = sum_l (r_l - 128) P_l + 128 = C' (mod Mprod)
   (sum_l P_l = 1 mod Mprod) and every partial sum stays below 2^53 in magnitude */
double oracle_crt_reconstruct(const int32_t* r, const crt_consts_t* cc) {
  double L[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int nl = cc->nl;
  for (int k = 0; k < nl; ++k) {
    int64_t sp = 0;
    for (int l = 0; l < cc->n; ++l) sp += (int64_t)cc->P[l * nl + k];
    L[k] = -128.0 * (double)sp + (k == 0 ? 128.0 : 0.0);
  }
  for (int l = 0; l < cc->n; ++l)
    for (int k = 0; k < nl; ++k) L[k] = fma((double)r[l], cc->P[l * nl + k], L[k]);
  const double s = fma(L[nl - 1], cc->f_hi, L[nl - 2] * cc->f_lo);
  const double Q = rint(s);
  double D[8];
  for (int k = 0; k < nl; ++k) D[k] = fma(-Q, cc->Mk[k], L[k]);
  const double base = ldexp(1.0, cc->w);
  double t = D[nl - 1];
  for (int k = nl - 2; k >= 0; --k) t = fma(t, base, D[k]);
  return t;
}

typedef struct {
  const int8_t *ra, *rb;
  const int32_t *sa, *sb; /* row / column shifts */
  double* C;
  int64_t M, N, K, Kp;
  double alpha, beta;
  const crt_consts_t* cc;
  int tid, nthreads;
} crt_job_t;

static void* crt_worker(void* arg) {
  crt_job_t* j = (crt_job_t*)arg;
  const crt_consts_t* cc = j->cc;
  const int64_t M = j->M, N = j->N, K = j->K, Kp = j->Kp;
  int32_t c[32];
  for (int64_t i = j->tid; i < M; i += j->nthreads) {
    for (int64_t col = 0; col < N; ++col) {
      const int bad = j->sa[i] == CRT_BAD || j->sb[col] == CRT_BAD;
      for (int l = 0; l < cc->n; ++l) {
        const int8_t* a = j->ra + ((int64_t)l * M + i) * Kp;
        const int8_t* b = j->rb + ((int64_t)l * N + col) * Kp;
        int64_t acc = 0;
        for (int64_t k = 0; k < K; ++k) acc += (int64_t)a[k] * (int64_t)b[k];
        c[l] = (int32_t)(((acc % cc->mods[l]) + cc->mods[l]) % cc->mods[l]); /* residue in [0, m) */
      }
      double out = NAN;
      if (!bad) {
        const double t = scale_pow2(scale_pow2(oracle_crt_reconstruct(c, cc), -j->sa[i]), -j->sb[col]);
        if (j->beta != 0.0) out = fma(j->alpha, t, j->beta * j->C[i * N + col]);
        else out = j->alpha * t;
      }
      j->C[i * N + col] = out;
    }
  }
  return NULL;
}

void oracle_crt_dgemm(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                      double beta, int n, int nl, int w, int ta, int tb, const int32_t* mods, const double* P,
                      const double* Mk, double f_hi, double f_lo, int nthreads) {
  crt_consts_t cc = {n, nl, w, mods, P, Mk, f_hi, f_lo};
  const int64_t Kp = K > 0 ? K : 1;
  int32_t* sa = (int32_t*)malloc(sizeof(int32_t) * (size_t)(M > 0 ? M : 1));
  int32_t* sb = (int32_t*)malloc(sizeof(int32_t) * (size_t)(N > 0 ? N : 1));
  int8_t* ra = (int8_t*)malloc((size_t)(n * M * Kp + 1));
  int8_t* rb = (int8_t*)malloc((size_t)(n * N * Kp + 1));
  oracle_crt_row_shifts(A, M, K, ta, sa);
  oracle_crt_col_shifts(B, K, N, tb, sb);
  oracle_crt_split_rows(A, M, K, sa, n, mods, ra, Kp);
  oracle_crt_split_cols(B, K, N, sb, n, mods, rb, Kp);
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  crt_job_t jobs[256];
  for (int t = 0; t < nthreads; ++t) {
    crt_job_t jb = {ra, rb, sa, sb, C, M, N, K, Kp, alpha, beta, &cc, t, nthreads};
    jobs[t] = jb;
    pthread_create(&th[t], NULL, crt_worker, &jobs[t]);
  }
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  free(sa); free(sb); free(ra); free(rb);
}
