// gen.cu — device side of the seeded counter-based input generator (replaces the reference's
// cuRAND uniform fill, routines/dgemm/dgemm.cpp:100-119) and the componentwise-error helpers,
// including a compensated (double-double) reference for sampled rows.
// The bit recipe is the CPU oracle's (splitmix64 finaliser keyed by seed and stream, indexed by
// element), so host and device inputs are identical.
#include <cmath>

#include "lt_internal.h"
#include "lt_runtime.cuh"

namespace lt {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ inline uint64_t host_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
uint64_t stream_key(uint64_t seed, uint64_t stream) { return host_mix64(seed ^ host_mix64(stream)); }

__global__ void fill_kernel(double* X, int64_t n, uint64_t key, int phi) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint64_t h = mix64(key + static_cast<uint64_t>(i) * 0xD1B54A32D192ED03ull);
    double u = static_cast<double>(h >> 11) * 0x1p-52 - 1.0;
    int e = 0;
    if (phi > 0) e = static_cast<int>(mix64(h ^ 0x5851F42D4C957F2Dull) % static_cast<uint64_t>(2 * phi + 1)) - phi;
    X[i] = scale_pow2(u, e);
  }
}

// Error-free transformations (Knuth TwoSum, FMA-based TwoProduct) with every operation rounded
// explicitly, so that nothing is contracted or reassociated: the double-double arithmetic is the
// same step for step as the CPU oracle's Dot2 (oracle/oracle.c, oracle_dgemm_dot2_rows).
struct DD {
  double hi, lo;
};
__device__ __forceinline__ DD two_sum(double a, double b) {
  const double s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  const double e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
  return DD{s, e};
}
__device__ __forceinline__ DD two_prod(double a, double b) {
  const double p = __dmul_rn(a, b);
  return DD{p, fma(a, b, -p)};
}
__device__ __forceinline__ DD dd_add(DD x, DD y) {
  const DD s = two_sum(x.hi, y.hi);
  return two_sum(s.hi, __dadd_rn(__dadd_rn(s.lo, x.lo), y.lo));
}
__device__ __forceinline__ DD dd_mul_d(DD x, double a) {
  const DD p = two_prod(x.hi, a);
  return two_sum(p.hi, __dadd_rn(p.lo, __dmul_rn(x.lo, a)));
}

// One thread per (sampled row, column): Cref = alpha*sum_k A[r,k] B[k,c] + beta*C0[r,c] with every
// product error-free and the sums in double-double, in k order, rounded once to double at the end;
// den = |alpha| sum_k |A[r,k]||B[k,c]| + |beta||C0[r,c]|.
__global__ void dot2_rows_kernel(const double* __restrict__ A, const double* __restrict__ B,
                                 const double* __restrict__ C0, const int64_t* __restrict__ rows, int64_t N, int64_t K,
                                 double alpha, double beta, double* __restrict__ Cref, double* __restrict__ den) {
  const int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (c >= N) return;
  const int64_t ri = blockIdx.y;
  const int64_t r = rows[ri];
  const double* arow = A + r * K;
  DD acc{0.0, 0.0};
  double aab = 0.0;
  for (int64_t k = 0; k < K; ++k) {
    const double a = arow[k];
    const double b = B[k * N + c];
    acc = dd_add(acc, two_prod(a, b));
    aab = __dadd_rn(aab, __dmul_rn(fabs(a), fabs(b)));
  }
  DD v = dd_mul_d(acc, alpha);
  double d = __dmul_rn(fabs(alpha), aab);
  if (beta != 0.0) {
    const double c0 = C0[r * N + c];
    v = dd_add(v, two_prod(beta, c0));
    d = __dadd_rn(d, __dmul_rn(fabs(beta), fabs(c0)));
  }
  Cref[ri * N + c] = __dadd_rn(v.hi, v.lo);
  den[ri * N + c] = d;
}

__device__ __forceinline__ int scale_exp(uint64_t key, int64_t i, int smax) {
  if (smax <= 0) return 0;
  uint64_t h = mix64(key + static_cast<uint64_t>(i) * 0xD1B54A32D192ED03ull);
  return static_cast<int>(h % static_cast<uint64_t>(2 * smax + 1)) - smax;
}

__global__ void scale_kernel(double* X, int64_t rows, int64_t cols, uint64_t key, int smax, int by_rows) {
  const int64_t n = rows * cols;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t idx = by_rows ? i / cols : i % cols;
    X[i] = scale_pow2(X[i], scale_exp(key, idx, smax));
  }
}

__global__ void cwise_error_kernel(const double* C, const double* R, const double* D, int64_t n, double tol,
                                   unsigned long long* max_bits, unsigned long long* above) {
  double mx = 0.0;
  unsigned long long cnt = 0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double c = C[i], r = R[i], d = D[i];
    double e;
    if (!isfinite(c) || !isfinite(r)) {
      e = (c == r || (isnan(c) && isnan(r))) ? 0.0 : INFINITY;
    } else {
      double diff = fabs(c - r);
      e = d > 0.0 ? diff / d : (diff == 0.0 ? 0.0 : INFINITY);
    }
    if (e > mx) mx = e;
    if (e > tol) ++cnt;
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  }
  if ((threadIdx.x & 31) == 0) {
    // non-negative doubles order like their bit patterns
    atomicMax(max_bits, static_cast<unsigned long long>(__double_as_longlong(mx)));
    atomicAdd(above, cnt);
  }
}

__global__ void abs_kernel(const double* X, double* Y, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    Y[i] = fabs(X[i]);
}

unsigned grid_for(int64_t n, int sms) {
  int64_t g = (n + 255) / 256;
  int64_t cap = static_cast<int64_t>(sms) * 16;
  return static_cast<unsigned>(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace
}  // namespace lt

extern "C" {

int lt_fill(double* X, int64_t n, uint64_t seed, uint64_t stream_id, int phi, void* stream) {
  if (n < 0 || (n > 0 && X == nullptr) || phi < 0 || phi > 1000)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_fill: bad arguments");
  lt::DeviceContext* ctx = lt::context();
  if (ctx == nullptr) return lt::last_error();
  if (n == 0) return lt::ok();
  lt::fill_kernel<<<lt::grid_for(n, ctx->sm_count), 256, 0, lt::as_stream(stream)>>>(X, n, lt::stream_key(seed, stream_id),
                                                                                      phi);
  LT_CUDA_TRY(cudaGetLastError());
  return lt::ok();
}

static int scale_impl(double* X, int64_t rows, int64_t cols, uint64_t seed, uint64_t stream_id, int smax, int by_rows,
                      void* stream) {
  if (rows < 0 || cols < 0 || (rows * cols > 0 && X == nullptr) || smax < 0 || smax > 1000)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_scale: bad arguments");
  lt::DeviceContext* ctx = lt::context();
  if (ctx == nullptr) return lt::last_error();
  if (rows * cols == 0) return lt::ok();
  lt::scale_kernel<<<lt::grid_for(rows * cols, ctx->sm_count), 256, 0, lt::as_stream(stream)>>>(
      X, rows, cols, lt::stream_key(seed, stream_id), smax, by_rows);
  LT_CUDA_TRY(cudaGetLastError());
  return lt::ok();
}

int lt_scale_rows(double* X, int64_t rows, int64_t cols, uint64_t seed, uint64_t stream_id, int smax, void* stream) {
  return scale_impl(X, rows, cols, seed, stream_id, smax, 1, stream);
}
int lt_scale_cols(double* X, int64_t rows, int64_t cols, uint64_t seed, uint64_t stream_id, int smax, void* stream) {
  return scale_impl(X, rows, cols, seed, stream_id, smax, 0, stream);
}

int lt_componentwise_error(const double* C, const double* Cref, const double* den, int64_t n, double tol,
                           double* out_host, void* stream) {
  if (n < 0 || out_host == nullptr || (n > 0 && (C == nullptr || Cref == nullptr || den == nullptr)))
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_componentwise_error: bad arguments");
  lt::DeviceContext* ctx = lt::context();
  if (ctx == nullptr) return lt::last_error();
  unsigned long long* buf = nullptr;
  LT_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&buf), 2 * sizeof(unsigned long long), lt::as_stream(stream)));
  cudaError_t e = cudaMemsetAsync(buf, 0, 2 * sizeof(unsigned long long), lt::as_stream(stream));
  if (e == cudaSuccess && n > 0) {
    lt::cwise_error_kernel<<<lt::grid_for(n, ctx->sm_count), 256, 0, lt::as_stream(stream)>>>(C, Cref, den, n, tol, buf,
                                                                                               buf + 1);
    e = cudaGetLastError();
  }
  unsigned long long h[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, buf, sizeof h, cudaMemcpyDeviceToHost, lt::as_stream(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(lt::as_stream(stream));
  cudaFreeAsync(buf, lt::as_stream(stream));
  if (e != cudaSuccess) return lt::set_error(LT_ERR_CUDA, "lt_componentwise_error: %s", cudaGetErrorString(e));
  double mx;
  memcpy(&mx, &h[0], sizeof mx);
  out_host[0] = mx;
  out_host[1] = static_cast<double>(h[1]);
  return lt::ok();
}

int lt_dot2_rows(const double* A, const double* B, const double* C0, double alpha, double beta, int64_t M,
                 int64_t N, int64_t K, const int64_t* rows, int64_t nrows, double* Cref, double* den, void* stream) {
  if (M < 0 || N < 0 || K < 0 || nrows < 0 || nrows > 65535 ||
      (nrows > 0 && N > 0 && (rows == nullptr || Cref == nullptr || den == nullptr)) ||
      (K > 0 && nrows > 0 && N > 0 && (A == nullptr || B == nullptr)) || (beta != 0.0 && C0 == nullptr && nrows > 0))
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_dot2_rows: bad arguments");
  if (nrows == 0 || N == 0) return lt::ok();
  if (lt::context() == nullptr) return lt::last_error();
  const dim3 grid(static_cast<unsigned>((N + 255) / 256), static_cast<unsigned>(nrows));
  lt::dot2_rows_kernel<<<grid, 256, 0, lt::as_stream(stream)>>>(A, B, C0, rows, N, K, alpha, beta, Cref, den);
  LT_CUDA_TRY(cudaGetLastError());
  return lt::ok();
}

int lt_abs_denominator(const double* A, const double* B, const double* C0, double* den, int64_t M, int64_t N,
                       int64_t K, double alpha, double beta, void* stream) {
  if (M < 0 || N < 0 || K < 0 || den == nullptr)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_abs_denominator: bad arguments");
  lt::DeviceContext* ctx = lt::context();
  if (ctx == nullptr) return lt::last_error();
  cudaStream_t s = lt::as_stream(stream);
  double *absA = nullptr, *absB = nullptr;
  LT_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&absA), sizeof(double) * (M * K + 2), s));
  LT_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&absB), sizeof(double) * (K * N + 2), s));
  if (M * K > 0) lt::abs_kernel<<<lt::grid_for(M * K, ctx->sm_count), 256, 0, s>>>(A, absA, M * K);
  if (K * N > 0) lt::abs_kernel<<<lt::grid_for(K * N, ctx->sm_count), 256, 0, s>>>(B, absB, K * N);
  if (beta != 0.0 && C0 != nullptr && M * N > 0) {
    lt::abs_kernel<<<lt::grid_for(M * N, ctx->sm_count), 256, 0, s>>>(C0, den, M * N);
  }
  int cfg = lt::fp64::heuristic_config(absA, absB, M, N, K, ctx->sm_count);
  int rc = lt::fp64::run_config(cfg, absA, absB, den, M, N, K, fabs(alpha), (beta != 0.0 && C0 != nullptr) ? fabs(beta) : 0.0, s);
  cudaFreeAsync(absA, s);
  cudaFreeAsync(absB, s);
  if (rc != LT_OK) return rc;
  return lt::ok();
}

}  // extern "C"
