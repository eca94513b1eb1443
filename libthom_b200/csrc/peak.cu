// peak.cu — measured tensor-pipe throughput of the current GPU (lt_measure_peak): the FP64
// mma.sync path the native DGEMM runs on and the INT8 tcgen05 shapes the Ozaki GEMM can use.
// The loops keep their operands on chip (registers or one shared-memory tile), so they measure
// the math pipe alone. Each tcgen05 kind first runs a short launch with known operand values and
// checks the accumulators it produced, so the CTA-pair form is verified before it is timed.
#include <cuda_runtime.h>

#include "lt_common.cuh"
#include "lt_internal.h"
#include "lt_runtime.cuh"

namespace lt {
namespace peak {

// ---------------------------------------------------------------------------------------------
// FP64: four independent m16n8k16 accumulator chains per warp, operands in registers.
// ---------------------------------------------------------------------------------------------
constexpr int kDmmaThreads = 256;

__global__ void __launch_bounds__(kDmmaThreads) dmma_loop(double* out, int iters) {
  double a[8], b[4], c[4][4];
  for (int i = 0; i < 8; ++i) a[i] = 1e-3 * (threadIdx.x + i);
  for (int i = 0; i < 4; ++i) b[i] = 1e-3 * (static_cast<int>(threadIdx.x) - i);
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i) c[j][i] = 0.0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      asm volatile(
          "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
          "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
          : "+d"(c[j][0]), "+d"(c[j][1]), "+d"(c[j][2]), "+d"(c[j][3])
          : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
            "d"(b[1]), "d"(b[2]), "d"(b[3]));
    }
  }
  double s = 0.0;
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i) s += c[j][i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// ---------------------------------------------------------------------------------------------
// INT8 tcgen05: one elected thread issues `iters` MMAs over one A tile and one B tile held in
// shared memory, rotating over 512 / N TMEM accumulators.
//   kMode 0: cta_group::1, M128 N128 K32      kMode 1: cta_group::1, M128 N256 K32
//   kMode 2: cta_group::2, M256 N128 K32 (cluster of two CTAs, each holding 128 rows of A and
//            64 rows of B)
// Check launch (`verify`): A = 1 in CTA rank 0 and 3 in rank 1; B rows n < N/2 hold 1, the others
// 2, so after k MMAs into an accumulator column j of row m holds 32 k a_m b_j.
// ---------------------------------------------------------------------------------------------
constexpr int kI8Threads = 128;
// Dynamic shared memory requested (and left unused) so that no two CTAs share an SM: each CTA
// allocates all 512 TMEM columns of its SM.
constexpr int kI8SmemPad = 120 * 1024;

template <int kMode>
__global__ void __launch_bounds__(kI8Threads, 1) i8_loop(int iters, int verify, int* mismatches, DeviceStatus* st) {
  constexpr bool kPair = kMode == 2;
  constexpr int kN = kMode == 1 ? 256 : 128;
  constexpr int kM = kPair ? 256 : 128;
  constexpr int kBRows = kPair ? kN / 2 : kN;  // rows of B held by this CTA
  constexpr int kAcc = 512 / kN;
  __shared__ __align__(1024) uint8_t sa[128 * 32];
  __shared__ __align__(1024) uint8_t sb[256 * 32];
  __shared__ __align__(8) uint64_t done;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = kPair ? cluster_ctarank() : 0u;

  auto hash = [](uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    return x ^ (x >> 16);
  };
  const uint32_t a_val = rank ? 3u : 1u;
  for (int i = threadIdx.x; i < 128 * 32 / 4; i += kI8Threads)
    reinterpret_cast<uint32_t*>(sa)[i] = verify ? a_val * 0x01010101u : hash(i + 7919u * blockIdx.x);
  for (int i = threadIdx.x; i < kBRows * 32 / 4; i += kI8Threads) {
    const int n = (kPair ? static_cast<int>(rank) * kBRows : 0) + (i * 4) / 32;
    reinterpret_cast<uint32_t*>(sb)[i] = verify ? (n < kN / 2 ? 1u : 2u) * 0x01010101u : hash(i + 104729u * blockIdx.x);
  }
  fence_proxy_async_smem();
  if (threadIdx.x == 0) {
    mbar_init(&done, 1);
    abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0) {
    if constexpr (kPair) {
      tmem_alloc_pair(&tmem_slot, 512);
      tmem_relinquish_pair();
    } else {
      tmem_alloc(&tmem_slot, 512);
      tmem_relinquish();
    }
  }
  tc_fence_before();
  __syncthreads();
  if constexpr (kPair) cluster_sync();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (rank == 0 && warp == 0) {
    if (elect_one_sync()) {
      const uint64_t da = smem_desc_k_sw32(smem_u32(sa));
      const uint64_t db = smem_desc_k_sw32(smem_u32(sb));
      constexpr uint32_t idesc = idesc_i8_s32(kM, kN);
      for (int i = 0; i < iters; ++i) {
        const uint32_t d = tmem + static_cast<uint32_t>((i % kAcc) * kN);
        if constexpr (kPair)
          mma_i8_pair(d, da, db, idesc, i >= kAcc ? 1u : 0u);
        else
          mma_i8(d, da, db, idesc, i >= kAcc ? 1u : 0u);
      }
      if constexpr (kPair) {
        mma_commit_pair(cluster_addr(&done, 0));
        mma_commit_pair(cluster_addr(&done, 1));
      } else {
        mma_commit(&done);
      }
    }
    __syncwarp();
  }
  const bool ok = kPair ? mbar_wait_cluster(&done, 0, &abort_flag, st, 91) : mbar_wait(&done, 0, &abort_flag, st, 90);
  tc_fence_after();
  if (ok && verify) {
    const uint32_t k = static_cast<uint32_t>(iters / kAcc);
    const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
    uint32_t v[32];
    int bad = 0;
    tmem_ld_32x32b_x32(tmem + lane_base, v);  // accumulator 0, columns 0..31 (B value 1)
    tmem_ld_wait();
    for (int i = 0; i < 32; ++i) bad += v[i] != 32u * k * a_val;
    tmem_ld_32x32b_x32(tmem + lane_base + static_cast<uint32_t>(kN - 32), v);  // last 32 columns (B value 2)
    tmem_ld_wait();
    for (int i = 0; i < 32; ++i) bad += v[i] != 64u * k * a_val;
    if (bad) atomicAdd(mismatches, bad);
  }
  (void)lane;
  tc_fence_before();
  __syncthreads();
  if constexpr (kPair) cluster_sync();
  if (warp == 0) {
    tc_fence_after();
    if constexpr (kPair)
      tmem_dealloc_pair(tmem, 512);
    else
      tmem_dealloc(tmem, 512);
  }
}

template <int kMode>
int launch_i8(int blocks, int iters, int verify, int* mismatches, DeviceContext* ctx, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  cfg.gridDim = dim3(static_cast<unsigned>(blocks));
  cfg.blockDim = dim3(kI8Threads);
  cfg.dynamicSmemBytes = kI8SmemPad;
  cfg.stream = stream;
  static bool attr_set[64] = {};
  if (!attr_set[ctx->device]) {
    LT_CUDA_TRY(cudaFuncSetAttribute(i8_loop<kMode>, cudaFuncAttributeMaxDynamicSharedMemorySize, kI8SmemPad));
    attr_set[ctx->device] = true;
  }
  if (kMode == 2) {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  LT_CUDA_TRY(cudaLaunchKernelEx(&cfg, i8_loop<kMode>, iters, verify, mismatches, ctx->status));
  return LT_OK;
}

// Grid for one CTA (or CTA pair) per SM: the SM count, or twice the number of co-resident pairs.
int i8_blocks(int mode, DeviceContext* ctx, int* blocks) {
  if (mode != 2) {
    *blocks = ctx->sm_count;
    return LT_OK;
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  cfg.gridDim = dim3(static_cast<unsigned>(ctx->sm_count & ~1));
  cfg.blockDim = dim3(kI8Threads);
  cfg.dynamicSmemBytes = kI8SmemPad;
  LT_CUDA_TRY(cudaFuncSetAttribute(i8_loop<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kI8SmemPad));
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  LT_CUDA_TRY(cudaOccupancyMaxActiveClusters(&clusters, i8_loop<2>, &cfg));
  if (clusters <= 0) return set_error(LT_ERR_UNSUPPORTED, "no CTA pair fits on this device");
  *blocks = 2 * (clusters < ctx->sm_count / 2 ? clusters : ctx->sm_count / 2);
  return LT_OK;
}

int run_i8(int mode, int blocks, int iters, int verify, int* mismatches, DeviceContext* ctx, cudaStream_t stream) {
  switch (mode) {
    case 0: return launch_i8<0>(blocks, iters, verify, mismatches, ctx, stream);
    case 1: return launch_i8<1>(blocks, iters, verify, mismatches, ctx, stream);
    default: return launch_i8<2>(blocks, iters, verify, mismatches, ctx, stream);
  }
}

// Times `launch` with CUDA events on `stream`: one warm-up launch, then `reps` launches (after
// `warm` more untimed ones). Returns milliseconds per launch.
template <class F>
int time_ms(F&& launch, cudaStream_t stream, float* ms, int warm = 0, int reps = 1) {
  cudaEvent_t e0, e1;
  LT_CUDA_TRY(cudaEventCreate(&e0));
  LT_CUDA_TRY(cudaEventCreate(&e1));
  int rc = launch();
  for (int i = 0; i < warm && rc == LT_OK; ++i) rc = launch();
  cudaError_t e = cudaSuccess;
  if (rc == LT_OK) e = cudaEventRecord(e0, stream);
  for (int i = 0; i < reps && rc == LT_OK && e == cudaSuccess; ++i) rc = launch();
  if (rc == LT_OK && e == cudaSuccess) e = cudaEventRecord(e1, stream);
  if (rc == LT_OK && e == cudaSuccess) e = cudaEventSynchronize(e1);
  if (rc == LT_OK && e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != LT_OK) return rc;
  LT_CUDA_TRY(e);
  *ms /= static_cast<float>(reps);
  return LT_OK;
}

// Burst: one timed launch after one warm-up. Sustained: about 0.5 s of launches back to back,
// then 0.5 s timed, so power and clock limits have settled.
template <class F>
int measure(F&& launch, cudaStream_t stream, bool sustained, float* ms) {
  int rc = time_ms(launch, stream, ms);
  if (rc != LT_OK || !sustained) return rc;
  const int n = static_cast<int>(500.0f / (*ms > 0.01f ? *ms : 0.01f)) + 1;
  return time_ms(launch, stream, ms, n, n);
}

}  // namespace peak
}  // namespace lt

extern "C" int lt_measure_peak(int kind, double* ops_per_second, void* stream_) {
  using namespace lt;
  using namespace lt::peak;
  const bool sustained = (kind & LT_PEAK_SUSTAINED) != 0;
  kind &= ~LT_PEAK_SUSTAINED;
  if (ops_per_second == nullptr || kind < LT_PEAK_FP64_MMA || kind > LT_PEAK_INT8_MMA_PAIR)
    return set_error(LT_ERR_INVALID_ARGUMENT, "lt_measure_peak: bad kind %d or null output", kind);
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  cudaStream_t stream = as_stream(stream_);
  *ops_per_second = 0.0;
  float ms = 0.f;
  if (kind == LT_PEAK_FP64_MMA) {
    const int blocks = 2 * ctx->sm_count, iters = 4096;
    double* out = nullptr;
    LT_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&out), sizeof(double) * blocks * kDmmaThreads, stream));
    int rc = measure(
        [&]() -> int {
          dmma_loop<<<blocks, kDmmaThreads, 0, stream>>>(out, iters);
          LT_CUDA_TRY(cudaGetLastError());
          return LT_OK;
        },
        stream, sustained, &ms);
    cudaFreeAsync(out, stream);
    if (rc != LT_OK) return rc;
    const double flops = 2.0 * 16 * 8 * 16 * 4.0 * iters * (kDmmaThreads / 32) * static_cast<double>(blocks);
    *ops_per_second = flops / (ms * 1e-3);
    return ok();
  }
  if (ctx->cc_major != 10) return set_error(LT_ERR_UNSUPPORTED, "tcgen05 needs an sm_100 device");
  const int mode = kind - LT_PEAK_INT8_MMA_N128;
  int blocks = 0;
  int rc = i8_blocks(mode, ctx, &blocks);
  if (rc != LT_OK) return rc;
  int* bad = nullptr;
  LT_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&bad), sizeof(int), stream));
  int hbad = 0;
  cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(int), stream);
  if (e == cudaSuccess) rc = run_i8(mode, blocks, 64, 1, bad, ctx, stream);
  if (e == cudaSuccess && rc == LT_OK) e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess && rc == LT_OK) e = cudaStreamSynchronize(stream);
  cudaFreeAsync(bad, stream);
  if (rc != LT_OK) return rc;
  LT_CUDA_TRY(e);
  rc = lt_check_device_status();
  if (rc != LT_OK) return rc;
  if (hbad != 0)
    return set_error(LT_ERR_UNSUPPORTED, "lt_measure_peak: check launch of kind %d produced %d wrong accumulators",
                     kind, hbad);
  const int iters = 32768;
  rc = measure([&]() { return run_i8(mode, blocks, iters, 0, nullptr, ctx, stream); }, stream, sustained, &ms);
  if (rc != LT_OK) return rc;
  rc = lt_check_device_status();
  if (rc != LT_OK) return rc;
  const int m = mode == 2 ? 256 : 128, n = mode == 1 ? 256 : 128;
  const double units = mode == 2 ? blocks / 2.0 : static_cast<double>(blocks);
  *ops_per_second = 2.0 * m * n * 32.0 * iters * units / (ms * 1e-3);
  return ok();
}
