// gen.cu — device side of the seeded counter-based input generator (replaces the reference's
// cuRAND uniform fill, routines/dgemm/dgemm.cpp:100-119) and the componentwise-error helpers.
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
