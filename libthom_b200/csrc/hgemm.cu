// hgemm.cu — FP16 GEMM of libthom's `hgemm` routine (routines/hgemm/hgemm.h:6-7) on sm_100a tensor
// cores: tcgen05.mma.cta_group::2.kind::f16 with FP32 accumulators in TMEM.
//
// Operands stay in the caller's row-major layout. A (M x K) is K-major for the tensor core and B
// (K x N) is N-major ("MN-major"); tiled TMA copies with 128-byte swizzle stage both, and the MMA
// reads them through shared-memory descriptors of the matching kinds (K-major SW128 for A,
// MN-major SW128 for B), so there is no transpose pass.
//
// Kernel: persistent CTA pairs (clusters of two CTAs on two SMs). A pair computes a 256 x BN tile
// of C (BN = 512, 256 or 128) over 64-wide K blocks: each CTA stages its 128 rows of A and BN/2
// columns of B per block, rank 0's MMA warp issues the pair MMAs (M = 256, N = min(BN, 256),
// K = 16: four per block and column block), and each CTA's TMEM receives its own 128 rows. With
// BN <= 256 the accumulators are double-buffered in TMEM, so the epilogue of one tile overlaps
// the main loop of the next; BN = 512 fills TMEM with one tile and moves a quarter less operand
// data per flop, which is what counts when the power cap sets the clock.
//
// Roles (320 threads per CTA):
//   warp 0      TMA producer (one lane), both CTAs
//   warp 1      rank 0: MMA issuer for the pair; rank 1: forwards each landed stage to rank 0
//   warps 2..9  epilogue: TMEM -> registers, alpha*acc + beta*C in FP32, one rounding to FP16
// Barriers (per CTA):
//   full[s]      rank 0: count 2 (own expect_tx arrival + the arrival relayed by rank 1);
//                rank 1: count 1
//   empty[s]     count 1: rank 0's MMA warp commits to both CTAs after the stage's MMAs
//   acc_full[b]  count 1: committed to both CTAs after a tile's last MMA into buffer b
//   acc_empty[b] rank 0 only, count 16: every epilogue warp of both CTAs arrives after reading b
// Every wait is bounded (LT_WAIT_TIMEOUT_NS); a wait that gives up records LT_ERR_DEVICE_TIMEOUT,
// and the MMA warp lets its issued MMAs finish before TMEM is released.
#include <cuda.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "../../include/libthom_hgemm.h"
#include "lt_common.cuh"
#include "lt_internal.h"
#include "lt_runtime.cuh"

namespace lt {
namespace hgemm {

constexpr int kBM = 128;                    // rows of C per CTA (256 per pair)
constexpr int kBK = 64;                     // K per stage: one 128-byte swizzle row of FP16
constexpr int kMmaK = 16;                   // K of one kind::f16 MMA
constexpr int kEpilogueWarps = 8;          // two per TMEM lane quarter, each half of the columns
constexpr int kThreads = 64 + 32 * kEpilogueWarps;
constexpr int kMaxSmem = 232448;            // 227 KB opt-in per CTA
constexpr int kABytes = kBM * kBK * 2;      // 16 KB: 128 rows x 64 K
constexpr int kBBlockBytes = kBK * 64 * 2;  // 8 KB: 64 K rows x 64 columns of B
constexpr int kOverhead = 1024 + 256;       // alignment slack + barriers
constexpr int kStoreRows = 32;              // one epilogue warp's TMEM lane quarter
constexpr int kStoreCols = 32;              // 64 bytes of FP16: one 64-byte swizzle row
constexpr int kStoreBytes = kStoreRows * kStoreCols * 2;          // 2 KB staging box
constexpr int kStoreBoxes = 2;                                     // per epilogue warp, alternating
constexpr int kEpilogueBytes = kEpilogueWarps * kStoreBoxes * kStoreBytes;  // 32 KB

// BN = 128 or 256: one pair MMA of N = BN per K step, accumulators double-buffered in TMEM.
// BN = 512: two pair MMAs of N = 256 per K step into two accumulators that fill TMEM (single
// buffer); a quarter less A/B traffic per flop than BN = 256.
template <int BN>
struct Geo {
  static constexpr int kMmaN = BN < 256 ? BN : 256;  // N of one pair MMA
  static constexpr int kMmas = BN / kMmaN;           // MMAs per K step (column blocks of the tile)
  static constexpr int kHalfN = BN / 2;              // columns of B staged by each CTA
  static constexpr int kBBlocks = kHalfN / 64;       // 64-column TMA boxes of B per CTA and stage
  static constexpr int kBPerMma = kBBlocks / kMmas;  // of which one MMA reads
  static constexpr int kStageBytes = kABytes + kBBlocks * kBBlockBytes;
  static constexpr int kFit = (kMaxSmem - kOverhead - kEpilogueBytes) / kStageBytes;
  static constexpr int kStages = kFit > 8 ? 8 : kFit;
  static constexpr int kSmem = kStages * kStageBytes + kEpilogueBytes + kOverhead;
  static constexpr int kAccBufs = BN <= 256 ? 2 : 1;  // TMEM holds 512 FP32 columns
  static constexpr int kTmemCols = kAccBufs * BN;
  static_assert(kHalfN % 64 == 0 && kStageBytes % 1024 == 0, "tile geometry");
  static_assert(kStages >= 2, "shared-memory ring too small");
  static_assert(kTmemCols <= 512 && (kTmemCols & (kTmemCols - 1)) == 0, "TMEM allocation");
};

struct Problem {
  uint16_t* C;
  int64_t M, N, ldc;
  float alpha, beta;
  int tiles_m, tiles_n;  // 256-row pair blocks, BN-column blocks
  int kblocks;           // ceil(K / 64)
  int vec;               // rows of C are 16-byte aligned: 16-byte loads and stores
  int group;             // pair-rows per raster group
  int tma_store;         // C 16-byte aligned (p.vec): staged tiles written by TMA stores
};

// Pair tiles in groups of p.group pair-rows, column-major inside a group, so the CTAs resident at
// one time share A row panels and B column panels in L2.
__device__ __forceinline__ void tile_coords(const Problem& p, int64_t t, int bn, int* m0, int* n0) {
  const int64_t G = p.group;
  const int64_t group = t / (G * p.tiles_n), first_m = group * G;
  const int64_t gsize = (p.tiles_m - first_m) < G ? (p.tiles_m - first_m) : G;
  const int64_t in_group = t - group * G * p.tiles_n;
  *m0 = static_cast<int>((first_m + in_group % gsize) * 2 * kBM);
  *n0 = static_cast<int>((in_group / gsize) * bn);
}

__device__ __forceinline__ float h2f(uint32_t bits) { return __half2float(__ushort_as_half(static_cast<unsigned short>(bits))); }
__device__ __forceinline__ uint32_t f2h(float x) { return __half_as_ushort(__float2half_rn(x)); }

// alpha*acc + beta*c with separately rounded products and sum (no contraction), the order of the
// reference's host check (routines/hgemm/hgemm.cu:145).
__device__ __forceinline__ float epilogue_value(float acc, float alpha, float beta, uint32_t cbits) {
  const float t = __fmul_rn(alpha, acc);
  return beta != 0.f ? __fadd_rn(t, __fmul_rn(beta, h2f(cbits))) : t;
}

// Writes 32 accumulators (columns col0..col0+31 of one row) to C.
__device__ __forceinline__ void store_row_chunk(const Problem& p, int64_t row, int64_t col0, const uint32_t (&v)[32]) {
  uint16_t* crow = p.C + row * p.ldc;
  const float alpha = p.alpha, beta = p.beta;
  if (p.vec && col0 + 32 <= p.N) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint4* dst = reinterpret_cast<uint4*>(crow + col0 + q * 8);
      uint4 cin = make_uint4(0u, 0u, 0u, 0u);
      if (beta != 0.f) cin = *dst;
      const uint32_t cw[4] = {cin.x, cin.y, cin.z, cin.w};
      uint32_t ow[4];
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const float lo = epilogue_value(__uint_as_float(v[q * 8 + 2 * h]), alpha, beta, cw[h] & 0xffffu);
        const float hi = epilogue_value(__uint_as_float(v[q * 8 + 2 * h + 1]), alpha, beta, cw[h] >> 16);
        ow[h] = f2h(lo) | (f2h(hi) << 16);
      }
      *dst = make_uint4(ow[0], ow[1], ow[2], ow[3]);
    }
  } else {
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const int64_t col = col0 + i;
      if (col < p.N) {
        const uint32_t cb = beta != 0.f ? crow[col] : 0u;
        crow[col] = static_cast<uint16_t>(f2h(epilogue_value(__uint_as_float(v[i]), alpha, beta, cb)));
      }
    }
  }
}

// 32 FP16 values of C (one row, columns col0..col0+31) as four 16-byte words, zero past the matrix
// edges. Needs p.vec (row pitch a multiple of 8 elements, so a word is wholly inside or outside).
// Streaming loads: each value of C is read once, just before the TMA store that overwrites it.
__device__ __forceinline__ void load_c_chunk(const Problem& p, int64_t row, int64_t col0, uint4 (&c)[4]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    c[q] = make_uint4(0u, 0u, 0u, 0u);
    if (row < p.M && col0 + q * 8 < p.N) c[q] = __ldcs(reinterpret_cast<const uint4*>(p.C + row * p.ldc + col0 + q * 8));
  }
}

// One 32 x 32 box of the output through shared memory: each lane (one row) converts its 32
// accumulators (with beta != 0, alpha*acc + beta*C from the prefetched words `cin`) to FP16 pairs
// and writes them into the staging box in the 64-byte swizzled order of the tensor map (16-byte
// chunk q of row r at r*64 + 16*(q ^ ((r >> 1) & 3)): four wavefronts per 32-lane 16-byte store,
// the minimum), then one lane issues the TMA store. A warp alternates between two boxes; a box is
// rewritten only after the store issued from it two chunks earlier has finished reading it, so
// each store overlaps the next chunk's conversion.
__device__ __forceinline__ void store_box_tma(const CUtensorMap* tmC, uint8_t* box, int lane, float alpha,
                                              const uint32_t (&v)[32], const uint4 (&cin)[4], int x, int y,
                                              const Problem& p) {
  if (lane == 0) bulk_wait_group_read1();
  __syncwarp();
  uint8_t* row = box + lane * 64;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint32_t w[4];
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      float lo = __uint_as_float(v[q * 8 + 2 * h]), hi = __uint_as_float(v[q * 8 + 2 * h + 1]);
      if (p.beta != 0.f) {
        const uint32_t cw = h == 0 ? cin[q].x : h == 1 ? cin[q].y : h == 2 ? cin[q].z : cin[q].w;
        lo = epilogue_value(lo, alpha, p.beta, cw & 0xffffu);
        hi = epilogue_value(hi, alpha, p.beta, cw >> 16);
      } else if (alpha != 1.f) {
        lo = __fmul_rn(alpha, lo);
        hi = __fmul_rn(alpha, hi);
      }
      const __half2 h2 = __floats2half2_rn(lo, hi);  // one cvt.rn.f16x2.f32
      w[h] = *reinterpret_cast<const uint32_t*>(&h2);
    }
    *reinterpret_cast<uint4*>(row + 16 * (q ^ ((lane >> 1) & 3))) = make_uint4(w[0], w[1], w[2], w[3]);
  }
  fence_proxy_async_smem();  // the generic-proxy writes above become visible to the TMA engine
  __syncwarp();
  if (lane == 0 && x < p.N && y < p.M) {  // boxes wholly past the matrix edge are not issued
    tma_store_2d(tmC, box, x, y);
  }
  if (lane == 0) bulk_commit_group();  // (an empty group when nothing was issued)
}

template <int BN>
__global__ void __launch_bounds__(kThreads, 1)
    hgemm_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const __grid_constant__ CUtensorMap tmC, Problem p, DeviceStatus* status) {
  using G = Geo<BN>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* staging = smem + G::kStages * G::kStageBytes;  // kEpilogueWarps boxes of kStoreBytes
  uint64_t* full = reinterpret_cast<uint64_t*>(staging + kEpilogueBytes);
  uint64_t* empty = full + G::kStages;
  uint64_t* acc_full = empty + G::kStages;  // [2]
  uint64_t* acc_empty = acc_full + 2;       // [2]
  uint64_t* drain = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const int64_t tiles = static_cast<int64_t>(p.tiles_m) * p.tiles_n;
  const int64_t first = cluster_id_x(), stride = num_clusters_x();
  const int kblocks = p.kblocks;

  if (threadIdx.x == 0) {
    for (int i = 0; i < G::kStages; ++i) {
      mbar_init(&full[i], rank == 0 ? 2 : 1);
      mbar_init(&empty[i], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 2 * kEpilogueWarps);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_desc(&tmA);
    tma_prefetch_desc(&tmB);
    if (p.tma_store) tma_prefetch_desc(&tmC);
  }
  if (warp == 1) {
    tmem_alloc_pair(tmem_slot, G::kTmemCols);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync();  // both CTAs' barriers exist before any arrival crosses the pair
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ------------------------------ TMA producer (both CTAs) ------------------------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int64_t t = first; t < tiles && ok; t += stride) {
        int m0, n0;
        tile_coords(p, t, BN, &m0, &n0);
        const int arow = m0 + static_cast<int>(rank) * kBM;
        // column block h of the tile: this CTA stages columns h*kMmaN + rank*kMmaN/2 .. +kMmaN/2
        const int bcol = n0 + static_cast<int>(rank) * (G::kMmaN / 2);
        for (int kb = 0; kb < kblocks; ++kb) {
          if (!mbar_wait_cluster(&empty[stage], phase ^ 1, abort_flag, status, 61)) { ok = false; break; }
          uint8_t* st = smem + stage * G::kStageBytes;
          mbar_arrive_expect_tx(&full[stage], G::kStageBytes);
          tma_load_2d(st, &tmA, &full[stage], kb * kBK, arow);
#pragma unroll
          for (int j = 0; j < G::kBBlocks; ++j)
            tma_load_2d(st + kABytes + j * kBBlockBytes, &tmB, &full[stage],
                        bcol + (j / G::kBPerMma) * G::kMmaN + (j % G::kBPerMma) * 64, kb * kBK);
          if (++stage == G::kStages) { stage = 0; phase ^= 1; }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1 && rank != 0) {
    // ------------------------ rank 1: forward each landed stage to rank 0 ------------------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int64_t t = first; t < tiles && ok; t += stride) {
        for (int kb = 0; kb < kblocks; ++kb) {
          if (!mbar_wait(&full[stage], phase, abort_flag, status, 62)) { ok = false; break; }
          // The copies into this CTA's stage have landed (complete_tx observed above); the forwarded
          // arrival carries no data of this thread, so relaxed ordering suffices.
          mbar_arrive_cluster_relaxed(cluster_addr(&full[stage], 0));
          if (++stage == G::kStages) { stage = 0; phase ^= 1; }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------ rank 0: MMA issuer for the pair ------------------------------
    // Warp-convergent loop: waits are made warp-uniform with __all_sync, one elected lane issues.
    constexpr uint32_t idesc = idesc_f16_f32(2 * kBM, G::kMmaN, /*b_mn_major=*/true);
    const uint64_t a_desc0 = smem_desc_k_sw128(smem_u32(smem));
    const uint64_t b_desc0 = smem_desc_mn_sw128(smem_u32(smem + kABytes), kBBlockBytes, 1024);
    constexpr uint64_t kStageStep = static_cast<uint64_t>(G::kStageBytes >> 4);
    constexpr uint64_t kAStepK = static_cast<uint64_t>((kMmaK * 2) >> 4);    // 32 bytes along a row
    constexpr uint64_t kBStepK = static_cast<uint64_t>((kMmaK * 128) >> 4);  // 16 rows of 128 bytes
    constexpr uint64_t kBStepN = static_cast<uint64_t>((G::kBPerMma * kBBlockBytes) >> 4);
    int stage = 0;
    uint32_t phase = 0;
    uint32_t iter = 0;
    bool ok = true;
    for (int64_t t = first; t < tiles && ok; t += stride, ++iter) {
      const uint32_t buf = iter % G::kAccBufs, use = iter / G::kAccBufs;
      if (!__all_sync(0xffffffffu, mbar_wait_cluster(&acc_empty[buf], (use & 1) ^ 1, abort_flag, status, 63))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t d_tmem = tmem_base + buf * BN;
      for (int kb = 0; kb < kblocks; ++kb) {
        if (!__all_sync(0xffffffffu, mbar_wait_cluster(&full[stage], phase, abort_flag, status, 64))) {
          ok = false;
          break;
        }
        tc_fence_after();
        if (elect_one_sync()) {
          const uint64_t a0 = a_desc0 + static_cast<uint64_t>(stage) * kStageStep;
          const uint64_t b0 = b_desc0 + static_cast<uint64_t>(stage) * kStageStep;
#pragma unroll
          for (int k = 0; k < kBK / kMmaK; ++k)
#pragma unroll
            for (int h = 0; h < G::kMmas; ++h)
              mma_f16_pair(d_tmem + h * G::kMmaN, a0 + k * kAStepK, b0 + h * kBStepN + k * kBStepK, idesc,
                           (kb > 0 || k > 0) ? 1u : 0u);
          mma_commit_pair(cluster_addr(&empty[stage], 0));
          mma_commit_pair(cluster_addr(&empty[stage], 1));
        }
        __syncwarp();
        if (++stage == G::kStages) { stage = 0; phase ^= 1; }
      }
      if (!ok) break;
      if (elect_one_sync()) {
        mma_commit_pair(cluster_addr(&acc_full[buf], 0));
        mma_commit_pair(cluster_addr(&acc_full[buf], 1));
      }
      __syncwarp();
    }
    if (!ok && elect_one_sync()) {
      // Let every MMA already issued finish before TMEM is released.
      mma_commit_pair(cluster_addr(drain, 0));
      const uint64_t t0 = globaltimer();
      while (!mbar_try_wait(drain, 0) && globaltimer() - t0 < LT_WAIT_TIMEOUT_NS) {
      }
    }
    __syncwarp();
  } else {
    // --------------------------------- epilogue (8 warps per CTA) ---------------------------------
    const int quarter = warp & 3;         // TMEM lanes 32*quarter .. +31 are visible to this warp
    const int colhalf = (warp - 2) >> 2;  // columns colhalf*BN/2 .. +BN/2 of the tile
    const int row_in_tile = quarter * 32 + lane;
    const uint32_t acc_empty_r0[2] = {cluster_addr(&acc_empty[0], 0), cluster_addr(&acc_empty[1], 0)};
    constexpr int kChunks = BN / 64;  // 32-column chunks per warp
    uint32_t iter = 0;
    for (int64_t t = first; t < tiles; t += stride, ++iter) {
      const uint32_t buf = iter % G::kAccBufs, use = iter / G::kAccBufs;
      int m0, n0;
      tile_coords(p, t, BN, &m0, &n0);
      const int64_t row = static_cast<int64_t>(m0) + static_cast<int64_t>(rank) * kBM + row_in_tile;
      const int col_base = colhalf * (BN / 2);
      uint4 c_cur[4] = {}, c_next[4] = {}, c_ahead[4] = {};  // C of chunks c, c+1, c+2
      if (p.tma_store && p.beta != 0.f) {
        load_c_chunk(p, row, static_cast<int64_t>(n0) + col_base, c_cur);
        if (kChunks > 1) load_c_chunk(p, row, static_cast<int64_t>(n0) + col_base + 32, c_next);
      }
      if (!mbar_wait_cluster(&acc_full[buf], use & 1, abort_flag, status, 65)) break;
      tc_fence_after();
      const uint32_t lane_base =
          tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) + buf * BN + static_cast<uint32_t>(col_base);
      if (p.tma_store) {
        // 32-column boxes staged in shared memory and written by TMA stores (clipped at the matrix
        // edges by the tensor map). With beta != 0 each lane reads its row's 32 values of C two
        // chunks ahead of the one it converts, so the load latency (longer than one chunk's
        // conversion) stays off the path from the TMEM reads (which free the accumulator buffer) to
        // the stores.
        uint8_t* boxes = staging + (warp - 2) * kStoreBoxes * kStoreBytes;
        const int y = m0 + static_cast<int>(rank) * kBM + quarter * 32;
#pragma unroll 1
        for (int c = 0; c < kChunks; ++c) {
          if (c + 2 < kChunks && p.beta != 0.f)
            load_c_chunk(p, row, static_cast<int64_t>(n0) + col_base + (c + 2) * 32, c_ahead);
          uint32_t v[32];
          tmem_ld_32x32b_x32(lane_base + static_cast<uint32_t>(c * 32), v);
          tmem_ld_wait();
          if (c == kChunks - 1) {
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(acc_empty_r0[buf]);
          }
          store_box_tma(&tmC, boxes + (c & 1) * kStoreBytes, lane, p.alpha, v, c_cur, n0 + col_base + c * 32, y, p);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            c_cur[q] = c_next[q];
            c_next[q] = c_ahead[q];
          }
        }
      } else {
#pragma unroll 1
        for (int c = 0; c < kChunks; ++c) {
          uint32_t v[32];
          tmem_ld_32x32b_x32(lane_base + static_cast<uint32_t>(c * 32), v);
          tmem_ld_wait();
          if (c == kChunks - 1) {
            // The whole accumulator is in registers: hand the buffer back before the last stores.
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(acc_empty_r0[buf]);
          }
          if (row < p.M) store_row_chunk(p, row, static_cast<int64_t>(n0) + col_base + c * 32, v);
        }
      }
    }
    if (p.tma_store && lane == 0) bulk_wait_group0();  // the last stores have been performed
    __syncwarp();
  }

  tc_fence_before();
  __syncthreads();
  cluster_sync();  // rank 0's MMAs read rank 1's shared memory and write its TMEM until here
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, G::kTmemCols);
  }
}

// C = beta*C (zero when beta == 0): the whole product when K == 0 or alpha == 0.
__global__ void scale_kernel(uint16_t* C, int64_t M, int64_t N, int64_t ldc, float beta) {
  const int64_t n = M * N;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint16_t* c = C + (i / N) * ldc + (i % N);
    *c = beta != 0.f ? static_cast<uint16_t>(f2h(__fmul_rn(beta, h2f(*c)))) : 0;
  }
}

// Copies a rows x cols matrix (row pitch lds) into a buffer with row pitch ldd >= cols.
__global__ void pack_kernel(const uint16_t* src, int64_t rows, int64_t cols, int64_t lds, uint16_t* dst, int64_t ldd) {
  const int64_t n = rows * cols;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / cols, c = i % cols;
    dst[r * ldd + c] = src[r * lds + c];
  }
}

constexpr int kNumConfigs = 3;
constexpr int kConfigBN[kNumConfigs] = {512, 256, 128};
const char* const kConfigNames[kNumConfigs] = {"pair_256x512", "pair_256x256", "pair_256x128"};

int num_configs() { return kNumConfigs; }
const char* config_name(int c) { return (c >= 0 && c < kNumConfigs) ? kConfigNames[c] : nullptr; }

// Wave-count cost model: waves x tile width / relative efficiency of the tile shape (wider tiles
// move less operand data per flop; 512 loses the epilogue overlap).
int default_config(int64_t M, int64_t N, int sm_count) {
  const int64_t clusters = std::max(1, sm_count / 2);
  int best = 0;
  double best_cost = 0.0;
  const double eff[kNumConfigs] = {1.0, 0.97, 0.85};
  for (int c = 0; c < kNumConfigs; ++c) {
    const int bn = kConfigBN[c];
    const int64_t tiles = ((M + 255) / 256) * ((N + bn - 1) / bn);
    const int64_t waves = (tiles + clusters - 1) / clusters;
    const double cost = static_cast<double>(waves) * bn / eff[c];
    if (c == 0 || cost < best_cost) { best = c; best_cost = cost; }
  }
  return best;
}

template <int BN>
int launch(const CUtensorMap& tmA, const CUtensorMap& tmB, const CUtensorMap& tmC, const Problem& p,
           DeviceContext* ctx, cudaStream_t stream) {
  using G = Geo<BN>;
  static std::once_flag once[64];
  static cudaError_t attr_err[64];
  static int max_clusters[64];
  auto config = [&](cudaLaunchConfig_t* cfg, cudaLaunchAttribute* attr, unsigned grid) {
    *cfg = cudaLaunchConfig_t{};
    cfg->gridDim = dim3(grid);
    cfg->blockDim = dim3(kThreads);
    cfg->dynamicSmemBytes = G::kSmem;
    cfg->stream = stream;
    attr->id = cudaLaunchAttributeClusterDimension;
    attr->val.clusterDim.x = 2;
    attr->val.clusterDim.y = 1;
    attr->val.clusterDim.z = 1;
    cfg->attrs = attr;
    cfg->numAttrs = 1;
  };
  std::call_once(once[ctx->device], [&] {
    attr_err[ctx->device] =
        cudaFuncSetAttribute(hgemm_pair_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::kSmem);
    if (attr_err[ctx->device] != cudaSuccess) return;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr;
    config(&cfg, &attr, static_cast<unsigned>(ctx->sm_count & ~1));
    attr_err[ctx->device] = cudaOccupancyMaxActiveClusters(&max_clusters[ctx->device], hgemm_pair_kernel<BN>, &cfg);
  });
  LT_CUDA_TRY(attr_err[ctx->device]);
  const int64_t tiles = static_cast<int64_t>(p.tiles_m) * p.tiles_n;
  const int64_t clusters = std::min<int64_t>(std::min<int64_t>(tiles, max_clusters[ctx->device]), ctx->sm_count / 2);
  if (clusters <= 0) return set_error(LT_ERR_UNSUPPORTED, "no CTA pair of the HGEMM kernel fits on this device");
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute attr;
  config(&cfg, &attr, static_cast<unsigned>(2 * clusters));
  LT_CUDA_TRY(cudaLaunchKernelEx(&cfg, hgemm_pair_kernel<BN>, tmA, tmB, tmC, p, ctx->status));
  return LT_OK;
}

// Pair-rows per raster group, or LIBTHOM_HGEMM_GROUP (1..64). Measured at 8192^3: with 512-wide
// tiles, groups of 16 pair-rows (4096 rows of C) read 0.85 GB from DRAM per launch against 0.91 GB
// for 8 and 1.18 GB for 4, and the power-capped clock rises with the saving (1380 vs 1350 vs
// 1327 MHz); 256- and 128-wide tiles do as well with 8.
int raster_group(int bn) {
  static const int g = [] {
    const char* e = getenv("LIBTHOM_HGEMM_GROUP");
    const int v = e != nullptr ? atoi(e) : 0;
    return (v >= 1 && v <= 64) ? v : 0;
  }();
  return g != 0 ? g : (bn >= 512 ? 16 : 8);
}

int check_args(const uint16_t* A, const uint16_t* B, uint16_t* C, int64_t M, int64_t N, int64_t K) {
  if (M < 0 || N < 0 || K < 0) return set_error(LT_ERR_INVALID_ARGUMENT, "negative dimension");
  // tile origins (up to a 256-row / 256-column block past the edge) stay within int32 coordinates
  if (M > 0x7ffffe00 || N > 0x7ffffe00 || K > 0x7ffffe00)
    return set_error(LT_ERR_INVALID_ARGUMENT, "dimension above 2^31-512");
  if ((M > 0 && K > 0 && A == nullptr) || (K > 0 && N > 0 && B == nullptr) || (M > 0 && N > 0 && C == nullptr))
    return set_error(LT_ERR_INVALID_ARGUMENT, "null matrix pointer");
  if (((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(C)) & 1) != 0)
    return set_error(LT_ERR_UNALIGNED, "matrix pointers must be 2-byte aligned");
  return LT_OK;
}

int run(const uint16_t* A, const uint16_t* B, uint16_t* C, int64_t M, int64_t N, int64_t K, float alpha, float beta,
        int config, cudaStream_t stream) {
  LT_TRY(check_args(A, B, C, M, N, K));
  if (config >= kNumConfigs) return set_error(LT_ERR_NOT_FOUND, "no HGEMM config %d", config);
  if (M == 0 || N == 0) return ok();
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  if (K == 0 || alpha == 0.f) {
    const int64_t blocks = std::min<int64_t>((M * N + 255) / 256, 8 * static_cast<int64_t>(ctx->sm_count));
    scale_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(C, M, N, N, beta);
    LT_CUDA_TRY(cudaGetLastError());
    return ok();
  }
  // Tensor maps need 16-byte aligned bases and row pitches; otherwise pack into padded copies.
  int64_t lda = K, ldb = N;
  const uint16_t* a = A;
  const uint16_t* b = B;
  const bool a_ok = (reinterpret_cast<uintptr_t>(A) & 15) == 0 && (K % 8) == 0;
  const bool b_ok = (reinterpret_cast<uintptr_t>(B) & 15) == 0 && (N % 8) == 0;
  if (!a_ok || !b_ok) {
    const int64_t lda_p = (K + 7) / 8 * 8, ldb_p = (N + 7) / 8 * 8;
    const size_t a_bytes = a_ok ? 0 : static_cast<size_t>(M * lda_p * 2 + 256) / 256 * 256;
    const size_t b_bytes = b_ok ? 0 : static_cast<size_t>(K * ldb_p * 2 + 256) / 256 * 256;
    void* ws = nullptr;
    LT_TRY(ensure_pack_workspace(ctx, a_bytes + b_bytes, &ws));
    uint8_t* w = static_cast<uint8_t*>(ws);
    const unsigned blocks = static_cast<unsigned>(8 * ctx->sm_count);
    if (!a_ok) {
      uint16_t* pa = reinterpret_cast<uint16_t*>(w);
      pack_kernel<<<blocks, 256, 0, stream>>>(A, M, K, K, pa, lda_p);
      LT_CUDA_TRY(cudaGetLastError());
      a = pa;
      lda = lda_p;
    }
    if (!b_ok) {
      uint16_t* pb = reinterpret_cast<uint16_t*>(w + a_bytes);
      pack_kernel<<<blocks, 256, 0, stream>>>(B, K, N, N, pb, ldb_p);
      LT_CUDA_TRY(cudaGetLastError());
      b = pb;
      ldb = ldb_p;
    }
  }
  if (config < 0) config = default_config(M, N, ctx->sm_count);
  const int bn = kConfigBN[config];
  CUtensorMap tmA, tmB;
  LT_TRY(make_tmap_2d(&tmA, a, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, static_cast<uint64_t>(M), static_cast<uint64_t>(K),
                      static_cast<uint64_t>(lda) * 2, kBM, kBK));
  LT_TRY(make_tmap_2d(&tmB, b, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, static_cast<uint64_t>(K), static_cast<uint64_t>(N),
                      static_cast<uint64_t>(ldb) * 2, kBK, 64));
  Problem p{};
  p.C = C;
  p.M = M;
  p.N = N;
  p.ldc = N;
  p.alpha = alpha;
  p.beta = beta;
  p.tiles_m = static_cast<int>((M + 2 * kBM - 1) / (2 * kBM));
  p.tiles_n = static_cast<int>((N + bn - 1) / bn);
  p.kblocks = static_cast<int>((K + kBK - 1) / kBK);
  p.vec = ((reinterpret_cast<uintptr_t>(C) & 15) == 0 && (N % 8) == 0) ? 1 : 0;
  p.group = raster_group(bn);
  p.tma_store = p.vec;
  CUtensorMap tmC = tmA;  // not read unless p.tma_store
  if (p.tma_store)
    LT_TRY(make_tmap_2d(&tmC, C, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, static_cast<uint64_t>(M),
                        static_cast<uint64_t>(N), static_cast<uint64_t>(N) * 2, kStoreRows, kStoreCols,
                        CU_TENSOR_MAP_SWIZZLE_64B));
  if (bn == 512) LT_TRY((launch<512>(tmA, tmB, tmC, p, ctx, stream)));
  else if (bn == 256) LT_TRY((launch<256>(tmA, tmB, tmC, p, ctx, stream)));
  else LT_TRY((launch<128>(tmA, tmB, tmC, p, ctx, stream)));
  return ok();
}

}  // namespace hgemm
}  // namespace lt

extern "C" {

int lt_hgemm(const lt_half* A, const lt_half* B, lt_half* C, int64_t M, int64_t N, int64_t K, float alpha, float beta,
             void* stream) {
  return lt::hgemm::run(A, B, C, M, N, K, alpha, beta, -1, lt::as_stream(stream));
}

int lt_hgemm_config(const lt_half* A, const lt_half* B, lt_half* C, int64_t M, int64_t N, int64_t K, float alpha,
                    float beta, int config, void* stream) {
  return lt::hgemm::run(A, B, C, M, N, K, alpha, beta, config, lt::as_stream(stream));
}

int lt_hgemm_num_configs(void) { return lt::hgemm::num_configs(); }
const char* lt_hgemm_config_name(int config) { return lt::hgemm::config_name(config); }

int lt_hgemm_default_config(int64_t M, int64_t N, int64_t K) {
  (void)K;
  lt::DeviceContext* ctx = lt::context();
  return lt::hgemm::default_config(M, N, ctx != nullptr ? ctx->sm_count : 148);
}

}  // extern "C"
