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
#include <cstring>
#include <mutex>

#include "lt_internal.h"
#include "lt_runtime.cuh"
#include "selector_common.cuh"

namespace lt {
namespace sel {

// ---- features: pass 1 (largest exponent), pass 2 (gap histogram) ----
// Row piece: sampled row i, K segment `seg` of length kseg; 256 threads stride the segment.
template <bool kHist>
__device__ __forceinline__ void rows_piece(const double* __restrict__ A, int64_t M, int64_t K, int rows, int64_t kseg,
                                           int i, int64_t seg, int* __restrict__ rmax, unsigned int* __restrict__ hist,
                                           unsigned int* sh) {
  const int64_t row = sampled_row(i, rows, M);
  const int64_t k0 = seg * kseg;
  const int64_t k1 = k0 + kseg < K ? k0 + kseg : K;
  const double* a = A + row * K;
  if (kHist) {
    if (threadIdx.x < 16) sh[threadIdx.x] = 0;
    __syncthreads();
    const int em = __ldcg(&rmax[i]);
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
    if ((threadIdx.x & 31) == 0 && m != kNone) atomicMax(&rmax[i], m);
  }
}

// Column piece: sampled group g of 32 columns, K segment `seg`; 8 warps, lane = column, warps
// stride K.
template <bool kHist>
__device__ __forceinline__ void cols_piece(const double* __restrict__ B, int64_t K, int64_t N, int groups, int64_t kseg,
                                           int g, int64_t seg, int* __restrict__ cmax, unsigned int* __restrict__ hist,
                                           unsigned int* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int64_t col = sampled_col0(g, groups, N) + lane;
  const int64_t k0 = seg * kseg;
  const int64_t k1 = k0 + kseg < K ? k0 + kseg : K;
  int* cm = cmax + g * 32 + lane;
  if (kHist) {
    if (threadIdx.x < 16) sh[threadIdx.x] = 0;
    __syncthreads();
    if (col < N) {
      const int em = __ldcg(cm);
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

// Rows: grid (sampled row, K segment). Columns: grid (sampled group of 32 columns, K segment).
template <bool kHist>
__global__ void feat_rows_kernel(const double* __restrict__ A, int64_t M, int64_t K, int rows, int64_t kseg,
                                 int* __restrict__ rmax, unsigned int* __restrict__ hist) {
  __shared__ unsigned int sh[16];
  rows_piece<kHist>(A, M, K, rows, kseg, blockIdx.x, blockIdx.y, rmax, hist, sh);
}
template <bool kHist>
__global__ void feat_cols_kernel(const double* __restrict__ B, int64_t K, int64_t N, int groups, int64_t kseg,
                                 int* __restrict__ cmax, unsigned int* __restrict__ hist) {
  __shared__ unsigned int sh[16];
  cols_piece<kHist>(B, K, N, groups, kseg, blockIdx.x, blockIdx.y, cmax, hist, sh);
}

// Feature i < 32 from the two 16-bin histograms (each normalised by its own total), then
// log2 K / 16 and -log10(tol) / 16.
__device__ __forceinline__ float feature_value(const unsigned int* hist, int t, int64_t K, double tol) {
  if (t < 32) {
    const unsigned int* h = hist + (t < 16 ? 0 : 16);
    unsigned long long tot = 0;
    for (int i = 0; i < 16; ++i) tot += __ldcg(&h[i]);
    return tot ? static_cast<float>(static_cast<double>(__ldcg(&hist[t])) / static_cast<double>(tot)) : 0.f;
  }
  if (t == 32) return static_cast<float>(log2(static_cast<double>(K > 0 ? K : 1)) / 16.0);
  return static_cast<float>(-log10(tol) / 16.0);
}

// ---- the selector's one-call statistics: two launches over a combined grid (row pieces, then
// column pieces) on a persistent per-device scratch. The second launch's last block (an atomic
// count, no block waits for another) turns the histograms into features, runs the network when
// given its parameters, and resets the scratch for the next call. ----
struct FeatGrid {
  int rows, groups, rseg, cseg;
  int64_t kr, kc;
};

struct SelScratch {
  unsigned int hist[32];
  int rmax[kSampleRows];
  int cmax[32 * kColGroups];
  unsigned int done;
  unsigned int pad[3];
  float out[64];  // features [0, 34), probabilities [48, 56)
};

__global__ void feat_max_fused_kernel(const double* __restrict__ A, const double* __restrict__ B, int64_t M, int64_t N,
                                      int64_t K, FeatGrid g, SelScratch* __restrict__ sc) {
  __shared__ unsigned int sh[16];
  const int nr = g.rows * g.rseg;
  const int b = blockIdx.x;
  if (b < nr)
    rows_piece<false>(A, M, K, g.rows, g.kr, b / g.rseg, b % g.rseg, sc->rmax, nullptr, sh);
  else
    cols_piece<false>(B, K, N, g.groups, g.kc, (b - nr) / g.cseg, (b - nr) % g.cseg, sc->cmax, nullptr, sh);
}

__global__ void feat_hist_fused_kernel(const double* __restrict__ A, const double* __restrict__ B, int64_t M,
                                       int64_t N, int64_t K, FeatGrid g, double tol,
                                       const float* __restrict__ params, SelScratch* __restrict__ sc) {
  __shared__ unsigned int sh[16];
  __shared__ float fx[F];
  __shared__ Acts acts;
  __shared__ int last;
  const int nr = g.rows * g.rseg;
  const int b = blockIdx.x;
  if (b < nr)
    rows_piece<true>(A, M, K, g.rows, g.kr, b / g.rseg, b % g.rseg, sc->rmax, sc->hist, sh);
  else
    cols_piece<true>(B, K, N, g.groups, g.kc, (b - nr) / g.cseg, (b - nr) % g.cseg, sc->cmax, sc->hist + 16, sh);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&sc->done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int t = threadIdx.x; t < F; t += blockDim.x) {
    fx[t] = feature_value(sc->hist, t, K, tol);
    sc->out[t] = fx[t];
  }
  __syncthreads();
  if (params != nullptr) {
    forward_block(params, fx, acts);
    if (threadIdx.x < C) sc->out[48 + threadIdx.x] = acts.prob[threadIdx.x];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 32; t += blockDim.x) sc->hist[t] = 0u;
  for (int t = threadIdx.x; t < kSampleRows; t += blockDim.x) sc->rmax[t] = kNone;
  for (int t = threadIdx.x; t < 32 * kColGroups; t += blockDim.x) sc->cmax[t] = kNone;
  if (threadIdx.x == 0) sc->done = 0u;
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

namespace {
std::mutex g_sel_mutex;
sel::SelScratch* g_sel_scratch[64] = {};
float* g_sel_host[64] = {};
}  // namespace

// A feature scratch of one's own (a plan's), in its initial state; the feature kernels leave it so.
size_t selector_scratch_bytes() { return sizeof(sel::SelScratch); }

int selector_scratch_init(void* scratch, cudaStream_t stream) {
  auto* sc = static_cast<sel::SelScratch*>(scratch);
  LT_CUDA_TRY(cudaMemsetAsync(sc, 0, sizeof(sel::SelScratch), stream));
  LT_CUDA_TRY(cudaMemsetAsync(sc->rmax, 0x80, sizeof(sc->rmax) + sizeof(sc->cmax), stream));  // kNone
  return LT_OK;
}

// The two feature kernels (sampled rows and column groups, then the network's forward pass) on
// `stream` with the caller's scratch; no host synchronisation. The class probabilities are left at
// selector_probs(scratch).
int selector_features_async(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol,
                            const float* params, void* scratch, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  auto* sc = static_cast<sel::SelScratch*>(scratch);
  sel::FeatGrid g;
  g.rows = static_cast<int>(M < sel::kSampleRows ? M : sel::kSampleRows);
  g.groups = static_cast<int>((N + 31) / 32 < sel::kColGroups ? (N + 31) / 32 : sel::kColGroups);
  const int64_t target = 4LL * ctx->sm_count;
  g.kr = sel::k_segment(K, g.rows, target, 256);
  g.kc = sel::k_segment(K, g.groups, target, 64);
  g.rseg = static_cast<int>((K + g.kr - 1) / g.kr);
  g.cseg = static_cast<int>((K + g.kc - 1) / g.kc);
  const unsigned blocks = static_cast<unsigned>(g.rows * g.rseg + g.groups * g.cseg);
  sel::feat_max_fused_kernel<<<blocks, 256, 0, stream>>>(A, B, M, N, K, g, sc);
  LT_CUDA_TRY(cudaGetLastError());
  sel::feat_hist_fused_kernel<<<blocks, 256, 0, stream>>>(A, B, M, N, K, g, tol, params, sc);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

const float* selector_probs(const void* scratch) { return static_cast<const sel::SelScratch*>(scratch)->out + 48; }

int selector_infer(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol, const float* params,
                   float* feat_dev, float* probs_host, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  // One selection at a time per process: the scratch is per device, and every call synchronises
  // before it returns, so no two calls' kernels overlap on the GPU.
  std::lock_guard<std::mutex> lock(g_sel_mutex);
  const int dev = ctx->device;
  if (g_sel_scratch[dev] == nullptr) {
    sel::SelScratch* sc = nullptr;
    LT_CUDA_TRY(cudaMalloc(&sc, sizeof(sel::SelScratch)));
    cudaError_t e = cudaMemset(sc, 0, sizeof(sel::SelScratch));
    if (e == cudaSuccess) e = cudaMemset(sc->rmax, 0x80, sizeof(sc->rmax) + sizeof(sc->cmax));  // kNone
    float* h = nullptr;
    if (e == cudaSuccess) e = cudaMallocHost(&h, 64 * sizeof(float));
    if (e != cudaSuccess) {
      cudaFree(sc);
      return set_error(LT_ERR_CUDA, "selector scratch: %s", cudaGetErrorString(e));
    }
    g_sel_scratch[dev] = sc;
    g_sel_host[dev] = h;
  }
  sel::SelScratch* sc = g_sel_scratch[dev];
  LT_TRY(selector_features_async(A, B, M, N, K, tol, params, sc, stream));
  if (feat_dev != nullptr)
    LT_CUDA_TRY(cudaMemcpyAsync(feat_dev, sc->out, sel::F * sizeof(float), cudaMemcpyDeviceToDevice, stream));
  float* h = g_sel_host[dev];
  if (probs_host != nullptr)
    LT_CUDA_TRY(cudaMemcpyAsync(h, sc->out + 48, sel::C * sizeof(float), cudaMemcpyDeviceToHost, stream));
  LT_CUDA_TRY(cudaStreamSynchronize(stream));
  if (probs_host != nullptr) memcpy(probs_host, h, sel::C * sizeof(float));
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
  LT_TRY(lt::selector_infer(A, B, M, N, K, tol, nullptr, features, nullptr, lt::as_stream(stream)));
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
