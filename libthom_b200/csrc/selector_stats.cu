// selector_stats.cu — matrix statistics for the Ozaki slice-count selector: the learned selector's
// features (exponent-gap histograms of sampled rows of A and columns of B) and the analytic
// fallback's input (the largest exponent gap of any row of A and of any column of B).
//
// A gap is how many binades an entry sits below the largest entry of its row (column):
// g = e(max) - e(x) with e the frexp exponent; zeros and non-finite entries do not count toward the
// extremes and fall in histogram bin 0. Every pass is a 2-D grid (rows or column groups x K
// segments), so short, wide and tall matrices all fill the GPU; extremes meet through integer
// atomics and histograms through shared-memory then global atomic counts, so the results do not
// depend on scheduling (the CPU oracle, oracle_features / oracle_max_gap, gives the same numbers).
#include <cmath>

#include "lt_internal.h"
#include "lt_runtime.cuh"

namespace lt {
namespace sel {

constexpr int kSampleRows = 128;  // rows of A sampled for the features (evenly spaced)
constexpr int kColGroups = 4;     // groups of 32 consecutive columns of B sampled for the features
constexpr int kNone = -0x7f7f7f80;  // memset(0x80) pattern: "no nonzero entry seen" for a max
constexpr int kNoneMin = 0x7f7f7f7f;  // memset(0x7f) pattern for a min

__device__ __forceinline__ int exp_of(double v) {
  int e;
  frexp(v, &e);
  return e;
}
__device__ __forceinline__ bool counts(double v) { return v != 0.0 && isfinite(v); }
__device__ __forceinline__ int gap_bin(int g) { return g >= 60 ? 15 : (g < 0 ? 0 : g >> 2); }

__device__ __forceinline__ int64_t sampled_row(int i, int rows, int64_t M) {
  return rows > 1 ? (static_cast<int64_t>(i) * (M - 1)) / (rows - 1) : 0;
}
__device__ __forceinline__ int64_t sampled_col0(int g, int groups, int64_t N) {
  const int64_t span = N > 32 ? N - 32 : 0;
  return groups > 1 ? (static_cast<int64_t>(g) * span) / (groups - 1) : 0;
}

// ---- features: pass 1 (largest exponent), pass 2 (gap histogram) ----
// Rows: grid (sampled row, K segment), 256 threads stride the segment.
template <bool kHist>
__global__ void feat_rows_kernel(const double* __restrict__ A, int64_t M, int64_t K, int rows, int64_t kseg,
                                 int* __restrict__ rmax, unsigned int* __restrict__ hist) {
  __shared__ unsigned int sh[16];
  const int64_t row = sampled_row(blockIdx.x, rows, M);
  const int64_t k0 = static_cast<int64_t>(blockIdx.y) * kseg;
  const int64_t k1 = k0 + kseg < K ? k0 + kseg : K;
  const double* a = A + row * K;
  if (kHist) {
    if (threadIdx.x < 16) sh[threadIdx.x] = 0;
    __syncthreads();
    const int em = rmax[blockIdx.x];
    for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
      const double v = fabs(a[k]);
      atomicAdd(&sh[counts(v) ? gap_bin(em - exp_of(v)) : 0], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 16 && sh[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
  } else {
    int m = kNone;
    for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
      const double v = fabs(a[k]);
      if (counts(v)) m = max(m, exp_of(v));
    }
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m != kNone) atomicMax(&rmax[blockIdx.x], m);
  }
}

// Columns: grid (sampled group of 32 columns, K segment), 8 warps; lane = column, warps stride K.
template <bool kHist>
__global__ void feat_cols_kernel(const double* __restrict__ B, int64_t K, int64_t N, int groups, int64_t kseg,
                                 int* __restrict__ cmax, unsigned int* __restrict__ hist) {
  __shared__ unsigned int sh[16];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int64_t col = sampled_col0(blockIdx.x, groups, N) + lane;
  const int64_t k0 = static_cast<int64_t>(blockIdx.y) * kseg;
  const int64_t k1 = k0 + kseg < K ? k0 + kseg : K;
  int* cm = cmax + blockIdx.x * 32 + lane;
  if (kHist) {
    if (threadIdx.x < 16) sh[threadIdx.x] = 0;
    __syncthreads();
    if (col < N) {
      const int em = *cm;
      for (int64_t k = k0 + warp; k < k1; k += nwarps) {
        const double v = fabs(B[k * N + col]);
        atomicAdd(&sh[counts(v) ? gap_bin(em - exp_of(v)) : 0], 1u);
      }
    }
    __syncthreads();
    if (threadIdx.x < 16 && sh[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
  } else if (col < N) {
    int m = kNone;
    for (int64_t k = k0 + warp; k < k1; k += nwarps) {
      const double v = fabs(B[k * N + col]);
      if (counts(v)) m = max(m, exp_of(v));
    }
    if (m != kNone) atomicMax(cm, m);
  }
}

__global__ void features_finish_kernel(const unsigned int* __restrict__ hist, int64_t K, double tol,
                                       float* __restrict__ feat) {
  const int t = threadIdx.x;
  if (t < 32) {
    const unsigned int* h = hist + (t < 16 ? 0 : 16);
    unsigned long long tot = 0;
    for (int i = 0; i < 16; ++i) tot += h[i];
    feat[t] = tot ? static_cast<float>(static_cast<double>(hist[t]) / static_cast<double>(tot)) : 0.f;
  } else if (t == 32) {
    feat[32] = static_cast<float>(log2(static_cast<double>(K > 0 ? K : 1)) / 16.0);
  } else if (t == 33) {
    feat[33] = static_cast<float>(-log10(tol) / 16.0);
  }
}

// ---- largest exponent gap of any row of A / column of B ----
// Rows: grid (8-row block, K segment), one warp per row.
__global__ void gap_rows_kernel(const double* __restrict__ A, int64_t M, int64_t K, int64_t kseg,
                                int* __restrict__ emax, int* __restrict__ emin) {
  const int lane = threadIdx.x & 31;
  const int64_t row = static_cast<int64_t>(blockIdx.x) * 8 + (threadIdx.x >> 5);
  if (row >= M) return;
  const int64_t k0 = static_cast<int64_t>(blockIdx.y) * kseg;
  const int64_t k1 = k0 + kseg < K ? k0 + kseg : K;
  int hi = kNone, lo = kNoneMin;
  for (int64_t k = k0 + lane; k < k1; k += 32) {
    const double v = fabs(A[row * K + k]);
    if (counts(v)) {
      const int e = exp_of(v);
      hi = max(hi, e);
      lo = min(lo, e);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
  }
  if (lane == 0 && hi != kNone) {
    atomicMax(&emax[row], hi);
    atomicMin(&emin[row], lo);
  }
}

// Columns: grid (256-column block, K segment), one thread per column.
__global__ void gap_cols_kernel(const double* __restrict__ B, int64_t K, int64_t N, int64_t kseg,
                                int* __restrict__ emax, int* __restrict__ emin) {
  const int64_t col = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (col >= N) return;
  const int64_t k0 = static_cast<int64_t>(blockIdx.y) * kseg;
  const int64_t k1 = k0 + kseg < K ? k0 + kseg : K;
  int hi = kNone, lo = kNoneMin;
  for (int64_t k = k0; k < k1; ++k) {
    const double v = fabs(B[k * N + col]);
    if (counts(v)) {
      const int e = exp_of(v);
      hi = max(hi, e);
      lo = min(lo, e);
    }
  }
  if (hi != kNone) {
    atomicMax(&emax[col], hi);
    atomicMin(&emin[col], lo);
  }
}

__global__ void gap_reduce_kernel(const int* __restrict__ emax, const int* __restrict__ emin, int64_t n,
                                  int* __restrict__ out) {
  int best = 0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    if (emax[i] != kNone) best = max(best, emax[i] - emin[i]);
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

// K segment length giving about `target` blocks for `outer` independent rows/columns.
int64_t k_segment(int64_t K, int64_t outer, int64_t target, int64_t align) {
  int64_t split = (target + outer - 1) / (outer > 0 ? outer : 1);
  if (split < 1) split = 1;
  int64_t seg = (K + split - 1) / split;
  seg = (seg + align - 1) / align * align;
  return seg < align ? align : seg;
}

}  // namespace sel

// Features into `feat` (device, 34 floats). `scratch` must hold kStatsScratchBytes.
int features_into(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol, float* feat,
                  void* scratch, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  auto* hist = static_cast<unsigned int*>(scratch);                 // 32
  int* rmax = reinterpret_cast<int*>(hist + 32);                   // kSampleRows
  int* cmax = rmax + sel::kSampleRows;                              // 32 * kColGroups
  LT_CUDA_TRY(cudaMemsetAsync(hist, 0, 32 * sizeof(unsigned int), stream));
  LT_CUDA_TRY(cudaMemsetAsync(rmax, 0x80, (sel::kSampleRows + 32 * sel::kColGroups) * sizeof(int), stream));
  const int rows = static_cast<int>(M < sel::kSampleRows ? M : sel::kSampleRows);
  const int groups = static_cast<int>((N + 31) / 32 < sel::kColGroups ? (N + 31) / 32 : sel::kColGroups);
  const int64_t target = 4LL * ctx->sm_count;
  const int64_t kr = sel::k_segment(K, rows, target, 256), kc = sel::k_segment(K, groups, target, 64);
  const dim3 gr(rows, static_cast<unsigned>((K + kr - 1) / kr)), gc(groups, static_cast<unsigned>((K + kc - 1) / kc));
  sel::feat_rows_kernel<false><<<gr, 256, 0, stream>>>(A, M, K, rows, kr, rmax, hist);
  sel::feat_cols_kernel<false><<<gc, 256, 0, stream>>>(B, K, N, groups, kc, cmax, hist + 16);
  sel::feat_rows_kernel<true><<<gr, 256, 0, stream>>>(A, M, K, rows, kr, rmax, hist);
  sel::feat_cols_kernel<true><<<gc, 256, 0, stream>>>(B, K, N, groups, kc, cmax, hist + 16);
  sel::features_finish_kernel<<<1, 64, 0, stream>>>(hist, K, tol, feat);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

// Largest row gap of A + largest column gap of B into *out (device int, zero on entry);
// `scratch` must hold 8 (M + N) bytes.
int gap_into(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int* out, void* scratch,
             cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  int* rmax = static_cast<int*>(scratch);
  int* rmin = rmax + M;
  int* cmax = rmin + M;
  int* cmin = cmax + N;
  LT_CUDA_TRY(cudaMemsetAsync(rmax, 0x80, M * sizeof(int), stream));
  LT_CUDA_TRY(cudaMemsetAsync(rmin, 0x7f, M * sizeof(int), stream));
  LT_CUDA_TRY(cudaMemsetAsync(cmax, 0x80, N * sizeof(int), stream));
  LT_CUDA_TRY(cudaMemsetAsync(cmin, 0x7f, N * sizeof(int), stream));
  const int64_t target = 4LL * ctx->sm_count;
  const int64_t rb = (M + 7) / 8, cb = (N + 255) / 256;
  const int64_t kr = sel::k_segment(K, rb, target, 256), kc = sel::k_segment(K, cb, target, 16);
  sel::gap_rows_kernel<<<dim3(static_cast<unsigned>(rb), static_cast<unsigned>((K + kr - 1) / kr)), 256, 0, stream>>>(
      A, M, K, kr, rmax, rmin);
  sel::gap_cols_kernel<<<dim3(static_cast<unsigned>(cb), static_cast<unsigned>((K + kc - 1) / kc)), 256, 0, stream>>>(
      B, K, N, kc, cmax, cmin);
  // both reductions add into *out: max row gap + max column gap
  sel::gap_reduce_kernel<<<ctx->sm_count, 256, 0, stream>>>(rmax, rmin, M, out);
  sel::gap_reduce_kernel<<<ctx->sm_count, 256, 0, stream>>>(cmax, cmin, N, out + 1);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

}  // namespace lt

extern "C" {

int lt_ozaki_features(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol, float* features,
                      void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || A == nullptr || B == nullptr || features == nullptr || !(tol > 0.0))
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_ozaki_features: bad arguments");
  if (lt::context() == nullptr) return lt::last_error();
  cudaStream_t s = lt::as_stream(stream);
  void* scratch = nullptr;
  LT_CUDA_TRY(cudaMallocAsync(&scratch, lt::kStatsScratchBytes, s));
  int rc = lt::features_into(A, B, M, N, K, tol, features, scratch, s);
  cudaFreeAsync(scratch, s);
  if (rc != LT_OK) return rc;
  return lt::ok();
}

int lt_ozaki_gap_bits(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int* gap_bits,
                      void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || A == nullptr || B == nullptr || gap_bits == nullptr)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_ozaki_gap_bits: bad arguments");
  if (lt::context() == nullptr) return lt::last_error();
  cudaStream_t s = lt::as_stream(stream);
  void* scratch = nullptr;
  LT_CUDA_TRY(cudaMallocAsync(&scratch, 8 * (M + N) + 256, s));
  int* out = reinterpret_cast<int*>(static_cast<uint8_t*>(scratch) + 8 * (M + N));
  cudaError_t e = cudaMemsetAsync(out, 0, 2 * sizeof(int), s);
  int rc = e == cudaSuccess ? lt::gap_into(A, B, M, N, K, out, scratch, s) : LT_ERR_CUDA;
  int h[2] = {0, 0};
  if (rc == LT_OK) e = cudaMemcpyAsync(h, out, sizeof h, cudaMemcpyDeviceToHost, s);
  if (rc == LT_OK && e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFreeAsync(scratch, s);
  if (rc != LT_OK) return rc;
  if (e != cudaSuccess) return lt::set_error(LT_ERR_CUDA, "lt_ozaki_gap_bits: %s", cudaGetErrorString(e));
  *gap_bits = h[0] + h[1];
  return lt::ok();
}

}  // extern "C"
