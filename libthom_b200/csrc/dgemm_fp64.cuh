// dgemm_fp64.cuh — native FP64 tensor-core DGEMM for sm_100a.
//
// Replaces the reference's register-fed sm_80 kernels (routines/dgemm/dgemm_final.cu:65-173:
// 64x128x16 tiles, 2-stage cp.async, mma.sync m8n8k4) with a warp-specialised, persistent design:
//   * one producer warp stages A (BM x 16) and B (16 x BN) k-blocks into a STAGES-deep ring of
//     128-byte-swizzled shared-memory tiles, either with TMA (cp.async.bulk.tensor, when the
//     row strides are 16-byte multiples) or with zero-filling cp.async for arbitrary shapes;
//   * full/empty mbarrier pairs hand each stage to the consumer warps and back;
//   * consumer warps each own a 32 x 32 sub-tile and issue mma.sync m16n8k16 FP64 (2048 FMAs per
//     instruction) from fragments read with 128-bit shared loads;
//   * the alpha/beta epilogue writes 16-byte vectors straight from the accumulators (C0 fetched
//     into L2 at the start of each tile and loaded before any store of its half-block);
//   * tiles come from a Source: one problem's tiles in raster order (whole tiles, a K split, or a
//     stream-K schedule of equal k-block ranges per CTA), or a grouped launch's tile list with
//     per-problem tensor maps.
// Tensor cores compute in FP64 throughout (tcgen05 has no FP64 kind on sm_100a; FP64 MMA is the
// warp-level instruction).
//
// Shared-memory layout of one stage (all offsets multiples of 1024 bytes):
//   A: BM rows x 128 bytes (16 doubles of K); 16-byte chunk c of row r sits at chunk c ^ (r & 7).
//   B: BN/16 boxes, each 16 k-rows x 128 bytes (16 doubles of N); chunk c of k-row k sits at
//      chunk c ^ (k & 7).
// This is exactly what TMA's SWIZZLE_128B writes for boxes {16, BM} and {16, 16}.
//
// K-permutation: within a 16-wide k-block, thread t of a quad feeds the MMA's logical k = t+4i
// with physical k = 4t+i (i = 0..3), for A and B alike. The sum over k is unchanged and every A
// fragment becomes two contiguous 32-byte row segments (128-bit loads). The B fragment loads (64-bit,
// served in half-warps) then meet k rows i and i + 8 of one swizzle phase in the same half-warp and
// take 4 wavefronts instead of 2. A permutation without those conflicts exists (thread t reading the
// chunks c1 = 2t + (t >> 1) and c1 ^ 1): it removed the replays (404 M -> 270 M wavefronts at 4096^3)
// but ran 3 % slower at 8192^3 (33.1 against 34.0 TF/s, same box): the replays only cost issue slots
// in a kernel the DMMA pipe bounds, and its per-thread chunk offsets cost address arithmetic under
// the 168-register cap. Not kept.
//
// Register cap: 8 consumer warps + the producer warp put 3 warps on one SM sub-partition, hence
// ptxas's 168 registers a thread and a few spills. Issuing the TMA loads from lane 0 of a consumer
// warp instead (8 warps, 220 registers, no spills; 240 with a second fragment set loaded while the
// current block's MMAs run) was bit-identical and slower at 8192^3: 32.2 and 29.7 against 34.7
// TF/s. The producer warp stays.
#pragma once
#include <cuda.h>

#include "lt_common.cuh"

namespace lt {
namespace fp64 {

struct Params {
  const double* A;
  const double* B;
  double* C;
  int64_t M, N, K;
  double alpha, beta;
  DeviceStatus* status;
  int64_t lda, ldb, ldc;  // row strides of A (M x K), B (K x N), C (M x N)
  // K split: `splits` > 1 cuts the k-blocks of every tile into that many contiguous ranges; the
  // unit for range s writes its raw sums to W + s*M*N (row stride N) and splitk_reduce forms C.
  int splits;
  double* W;
  // Stream-K (`streamk` = 1, splits = 1): the tiles x k-blocks sequence is cut into gridDim.x equal
  // contiguous ranges, one per CTA. A tile that one CTA covers whole goes straight to C; the pieces
  // of a tile shared by several CTAs go to per-CTA slots (W + (2b + j)*BM*BN for CTA b, j = 0 for
  // its first tile, 1 for its last) and streamk_fixup sums them in K order.
  int streamk;
};

template <int BM_, int BN_, int STAGES_, bool TMA_, int MINB_ = 1>
struct Config {
  static constexpr int BM = BM_, BN = BN_, STAGES = STAGES_;
  static constexpr int MIN_BLOCKS = MINB_;  // CTAs per SM the register budget is sized for
  static constexpr bool kTMA = TMA_;
  static constexpr int BK = 16;  // doubles of K per stage: one 128-byte swizzle row
  static constexpr int WM = 32, WN = 32;
  static constexpr int WARPS_M = BM / WM, WARPS_N = BN / WN;
  static constexpr int CONSUMERS = WARPS_M * WARPS_N;
  // cp.async staging issues one copy per 16 bytes from the producer warps' own registers, so tiles
  // with four or more consumer warps get two producer warps (measured: 128x64 10.9 -> 20.7 TF/s at
  // 8192^3 with 16-byte copies and two producers); TMA needs one thread.
  static constexpr int PRODUCERS = (TMA_ || CONSUMERS < 4) ? 1 : 2;
  static constexpr int THREADS = (CONSUMERS + PRODUCERS) * 32;
  static constexpr int A_BYTES = BM * 128;
  static constexpr int B_BYTES = BN * 128;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*alignment slack*/ + 256 /*barriers*/;
  static_assert(BM % WM == 0 && BN % WN == 0, "tile must be a multiple of the warp tile");
  static_assert(BN % 16 == 0 && BM % 8 == 0, "tile shape");
};

// Byte offset of the 16-byte chunk holding A(row, 2c..2c+1) in an A stage.
__device__ __forceinline__ uint32_t a_off(int row, int chunk) {
  return static_cast<uint32_t>(row * 128 + ((chunk ^ (row & 7)) << 4));
}
// Byte offset of B(k, n) (one double) in a B stage.
__device__ __forceinline__ uint32_t b_off(int k, int n) {
  int box = n >> 4, col = n & 15;
  return static_cast<uint32_t>(box * 2048 + k * 128 + ((((col >> 1) ^ (k & 7)) << 4)) + ((col & 1) << 3));
}

__device__ __forceinline__ void mma_m16n8k16(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

__device__ __forceinline__ void lds128(double& x, double& y, uint32_t addr) {
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(x), "=d"(y) : "r"(addr));
}
__device__ __forceinline__ double lds64(uint32_t addr) {
  double x;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(x) : "r"(addr));
  return x;
}

// Tile order: groups of 8 tile-rows are walked column by column so that consecutive CTAs share
// B panels and A panels in L2.
__device__ __forceinline__ void tile_coords(int64_t t, int64_t tiles_m, int64_t tiles_n, int64_t& tm, int64_t& tn) {
  const int64_t G = 8;
  int64_t group = t / (G * tiles_n);
  int64_t first_m = group * G;
  int64_t gsize = (tiles_m - first_m) < G ? (tiles_m - first_m) : G;
  int64_t in_group = t - group * G * tiles_n;
  tm = first_m + in_group % gsize;
  tn = in_group / gsize;
}

// One output tile of one problem, over k-blocks kb0..kb1-1. W != nullptr: write the raw sums
// there (partial sums: element (row, col) at W[(row - wr0)*ldw + col - wc0]) instead of
// alpha*acc + beta*C.
struct Job {
  const double* A;
  const double* B;
  double* C;
  int64_t M, N, K;
  double alpha, beta;
  int64_t m0, n0;
  int kb0, kb1;
  double* W;
  int64_t lda, ldb, ldc;
  const CUtensorMap* tmA;  // TMA configurations: the tensor maps of this job's A and B
  const CUtensorMap* tmB;
  int64_t ldw, wr0, wc0;
};

// Stream-K: first iteration (tile x k-block) of CTA b's range, b in 0..G.
__host__ __device__ __forceinline__ int64_t streamk_first(int64_t b, int64_t total, int64_t G) {
  return b * total / G;
}
// The CTA whose range holds iteration i (ranges are non-empty: total >= G).
__host__ __device__ __forceinline__ int64_t streamk_owner(int64_t i, int64_t total, int64_t G) {
  int64_t b = i * G / total;
  while (b + 1 < G && streamk_first(b + 1, total, G) <= i) ++b;
  while (b > 0 && streamk_first(b, total, G) > i) --b;
  return b;
}

// Tiles of a single problem, walked in grouped raster order.
// With a K split, unit u covers range u / tiles of tile u % tiles, so each wave spans all tiles of
// one range before the next range starts. With stream-K, CTA b walks the tiles its iteration range
// touches, in order (the units are then tile indices).
template <class Cfg>
struct SingleSource {
  Params p;
  int64_t tiles_m, tiles_n;
  const CUtensorMap* tmA;
  const CUtensorMap* tmB;
  __device__ int64_t count() const { return tiles_m * tiles_n * p.splits; }
  __device__ int64_t nkb() const { return (p.K + Cfg::BK - 1) / Cfg::BK; }
  __device__ int64_t total() const { return tiles_m * tiles_n * nkb(); }
  __device__ int64_t begin() const {
    return p.streamk ? streamk_first(blockIdx.x, total(), gridDim.x) / nkb() : static_cast<int64_t>(blockIdx.x);
  }
  __device__ int64_t end() const {
    return p.streamk ? (streamk_first(blockIdx.x + 1, total(), gridDim.x) - 1) / nkb() + 1 : count();
  }
  __device__ int64_t step() const { return p.streamk ? 1 : static_cast<int64_t>(gridDim.x); }
  __device__ Job get(int64_t u) const {
    if (p.streamk) {
      const int64_t nk = nkb(), it0 = streamk_first(blockIdx.x, total(), gridDim.x);
      const int64_t it1 = streamk_first(blockIdx.x + 1, total(), gridDim.x);
      int64_t tm, tn;
      tile_coords(u, tiles_m, tiles_n, tm, tn);
      const int64_t kb0 = it0 > u * nk ? it0 - u * nk : 0;
      const int64_t kb1 = it1 - u * nk < nk ? it1 - u * nk : nk;
      double* w = nullptr;
      if (kb0 > 0 || kb1 < nk)
        w = p.W + (2 * static_cast<int64_t>(blockIdx.x) + (u == it0 / nk ? 0 : 1)) * (Cfg::BM * Cfg::BN);
      return Job{p.A, p.B, p.C, p.M, p.N, p.K, p.alpha, p.beta, tm * Cfg::BM, tn * Cfg::BN,
                 static_cast<int>(kb0), static_cast<int>(kb1), w, p.lda, p.ldb, p.ldc, tmA, tmB,
                 Cfg::BN, tm * Cfg::BM, tn * Cfg::BN};
    }
    const int64_t tiles = tiles_m * tiles_n;
    const int64_t sp = u / tiles, t = u - sp * tiles;
    int64_t tm, tn;
    tile_coords(t, tiles_m, tiles_n, tm, tn);
    const int nkb = static_cast<int>((p.K + Cfg::BK - 1) / Cfg::BK);
    const int per = (nkb + p.splits - 1) / p.splits;
    const int kb0 = static_cast<int>(sp) * per;
    const int kb1 = kb0 + per < nkb ? kb0 + per : nkb;
    double* w = p.splits > 1 ? p.W + sp * p.M * p.N : nullptr;
    return Job{p.A, p.B, p.C, p.M, p.N, p.K, p.alpha, p.beta, tm * Cfg::BM, tn * Cfg::BN, kb0, kb1, w,
               p.lda, p.ldb, p.ldc, tmA, tmB, p.N, 0, 0};
  }
};

// Grouped launch: a device table of problems and a tile list (sorted by decreasing K on the host
// so that the static round-robin over CTAs hands out the expensive tiles first). TMA
// configurations read A and B through per-problem tensor maps held in device memory (written by
// the host before any launch, null when K == 0).
struct GroupProblem {
  const double* A;
  const double* B;
  double* C;
  int64_t M, N, K;
  double alpha, beta;
  const CUtensorMap* tmA;
  const CUtensorMap* tmB;
};
struct GroupTile {
  int problem;
  int m0, n0;
  int pad;
};
struct GroupedSource {
  const GroupProblem* problems;
  const GroupTile* tiles;
  int64_t ntiles;
  __device__ int64_t count() const { return ntiles; }
  __device__ int64_t begin() const { return blockIdx.x; }
  __device__ int64_t end() const { return ntiles; }
  __device__ int64_t step() const { return gridDim.x; }
  __device__ Job get(int64_t t) const {
    const GroupTile gt = tiles[t];
    const GroupProblem& pr = problems[gt.problem];
    return Job{pr.A,  pr.B,  pr.C,  pr.M, pr.N,
               pr.K,  pr.alpha, pr.beta, gt.m0, gt.n0,
               0,     static_cast<int>((pr.K + 15) / 16), nullptr, pr.K, pr.N, pr.N,
               pr.tmA, pr.tmB, 0, 0, 0};
  }
};

template <class Cfg, class Source>
__device__ __forceinline__ void gemm_body(const CUtensorMap* tmA, const CUtensorMap* tmB, const Source& src,
                                          DeviceStatus* status) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + Cfg::STAGES * Cfg::STAGE_BYTES);
  uint64_t* empty = full + Cfg::STAGES;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + Cfg::STAGES);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t t_begin = src.begin(), t_end = src.end(), t_step = src.step();

  if (threadIdx.x == 0) {
    for (int s = 0; s < Cfg::STAGES; ++s) {
      mbar_init(&full[s], Cfg::kTMA ? 1 : 32 * Cfg::PRODUCERS);
      mbar_init(&empty[s], Cfg::CONSUMERS);
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();

  if (warp >= Cfg::CONSUMERS) {
    // ------------------------------- producer warp(s) -------------------------------
    const int pt = (warp - Cfg::CONSUMERS) * 32 + lane;  // producer thread index
    constexpr int kPT = 32 * Cfg::PRODUCERS;
    if (Cfg::kTMA && tmA != nullptr) {  // single problem: the maps are kernel parameters
      if (lane == 0) {
        tma_prefetch_desc(tmA);
        tma_prefetch_desc(tmB);
      }
    }
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (int64_t t = t_begin; t < t_end && ok; t += t_step) {
      const Job J = src.get(t);
      const int64_t m0 = J.m0, n0 = J.n0;
      for (int kb = J.kb0; kb < J.kb1; ++kb) {
        if (!mbar_wait(&empty[stage], phase ^ 1, abort_flag, status, 1)) { ok = false; break; }
        uint8_t* sa = smem + stage * Cfg::STAGE_BYTES;
        uint8_t* sb = sa + Cfg::A_BYTES;
        const int k0 = kb * Cfg::BK;
        if (Cfg::kTMA) {
          if (lane == 0) {
            mbar_arrive_expect_tx(&full[stage], Cfg::STAGE_BYTES);
            tma_load_2d(sa, J.tmA, &full[stage], k0, static_cast<int>(m0));
#pragma unroll
            for (int j = 0; j < Cfg::BN / 16; ++j)
              tma_load_2d(sb + j * 2048, J.tmB, &full[stage], static_cast<int>(n0) + 16 * j, k0);
            // Grouped launches keep each problem's tensor maps in device memory and consecutive
            // tiles of a CTA mostly belong to different problems: once this tile's first loads are
            // out, the next tile's maps are brought into the descriptor cache.
            if (tmA == nullptr && kb == J.kb0 && t + t_step < t_end) {
              const Job Jn = src.get(t + t_step);
              if (Jn.tmA != nullptr) {
                tma_prefetch_desc(Jn.tmA);
                tma_prefetch_desc(Jn.tmB);
              }
            }
          }
        } else {
          // A: BM rows x 16 doubles as 16-byte pairs (one shared-memory chunk each): one 16-byte
          // cp.async when both doubles are in range and the source is 16-byte aligned (every row
          // when K is even and A aligned, every other row when K is odd), else two 8-byte ones
          // with zero fill (ragged rows and K).
          for (int e = pt; e < Cfg::BM * 8; e += kPT) {
            const int r = e >> 3, c = e & 7;
            const int64_t gr = m0 + r, gk = k0 + 2 * c;
            uint8_t* dst = sa + a_off(r, c);
            const double* gp = J.A + gr * J.lda + gk;
            if (gr < J.M && gk + 1 < J.K && (reinterpret_cast<uintptr_t>(gp) & 15) == 0) {
              cp_async_16(dst, gp, true);
            } else {
              const bool v0 = (gr < J.M) && (gk < J.K), v1 = (gr < J.M) && (gk + 1 < J.K);
              cp_async_8(dst, v0 ? gp : J.A, v0);
              cp_async_8(dst + 8, v1 ? gp + 1 : J.A, v1);
            }
          }
          // B: 16 k-rows x BN doubles, the same way over column pairs (n, n + 1), which share a
          // 16-byte chunk of the stage layout.
          for (int e = pt; e < 16 * (Cfg::BN / 2); e += kPT) {
            const int k = e / (Cfg::BN / 2), n = 2 * (e % (Cfg::BN / 2));
            const int64_t gk = k0 + k, gn = n0 + n;
            uint8_t* dst = sb + b_off(k, n);
            const double* gp = J.B + gk * J.ldb + gn;
            if (gk < J.K && gn + 1 < J.N && (reinterpret_cast<uintptr_t>(gp) & 15) == 0) {
              cp_async_16(dst, gp, true);
            } else {
              const bool v0 = (gk < J.K) && (gn < J.N), v1 = (gk < J.K) && (gn + 1 < J.N);
              cp_async_8(dst, v0 ? gp : J.B, v0);
              cp_async_8(dst + 8, v1 ? gp + 1 : J.B, v1);
            }
          }
          cp_async_mbar_arrive_noinc(&full[stage]);
        }
        if (++stage == Cfg::STAGES) { stage = 0; phase ^= 1; }
      }
    }
    if (!Cfg::kTMA) asm volatile("cp.async.wait_all;" ::: "memory");
  } else {
    // ------------------------------- consumer warps -------------------------------
    const int wm = warp / Cfg::WARPS_N, wn = warp % Cfg::WARPS_N;
    const int g = lane >> 2, tq = lane & 3;
    const uint32_t smem_base = smem_u32(smem);
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (int64_t t = t_begin; t < t_end && ok; t += t_step) {
      const Job J = src.get(t);
      if (J.W == nullptr && J.beta != 0.0) {
        // The C block this warp's epilogue reads (32 rows of 32 doubles, one row per lane) is
        // fetched into L2 while the main loop runs, so the epilogue waits for L2, not DRAM.
        const int64_t row = J.m0 + wm * Cfg::WM + lane, col = J.n0 + wn * Cfg::WN;
        if (row < J.M && col < J.N) {
          const double* cp = J.C + row * J.ldc + col;
          prefetch_l2(cp);
          if (col + 16 < J.N) prefetch_l2(cp + 16);
          if (col + 31 < J.N) prefetch_l2(cp + 31);
        }
      }
      double acc[2][4][4];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;

      for (int kb = J.kb0; kb < J.kb1; ++kb) {
        if (!mbar_wait(&full[stage], phase, abort_flag, status, 2)) { ok = false; break; }
        const uint32_t sa = smem_base + stage * Cfg::STAGE_BYTES;
        const uint32_t sb = sa + Cfg::A_BYTES;
        double af[2][8], bf[4][4];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int r0 = wm * Cfg::WM + i * 16 + g;
          // physical k 4tq..4tq+3 = chunks 2tq, 2tq+1 of rows r0 and r0+8
          double x0, x1, x2, x3, y0, y1, y2, y3;
          lds128(x0, x1, sa + a_off(r0, 2 * tq));
          lds128(x2, x3, sa + a_off(r0, 2 * tq + 1));
          lds128(y0, y1, sa + a_off(r0 + 8, 2 * tq));
          lds128(y2, y3, sa + a_off(r0 + 8, 2 * tq + 1));
          af[i][0] = x0; af[i][1] = y0; af[i][2] = x1; af[i][3] = y1;
          af[i][4] = x2; af[i][5] = y2; af[i][6] = x3; af[i][7] = y3;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int n = wn * Cfg::WN + j * 8 + g;
#pragma unroll
          for (int i = 0; i < 4; ++i) bf[j][i] = lds64(sb + b_off(4 * tq + i, n));
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[stage]);
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) mma_m16n8k16(acc[i][j], af[i], bf[j]);
        if (++stage == Cfg::STAGES) { stage = 0; phase ^= 1; }
      }
      if (!ok) break;

      // ---- epilogue: C = alpha*acc + beta*C0 (or the raw sums into W), 16-byte vectors where the
      // row stride allows ----
      const int64_t m0 = J.m0 + wm * Cfg::WM, n0 = J.n0 + wn * Cfg::WN;
      if (J.W != nullptr) {
        const bool wvec = (J.ldw & 1) == 0;  // W and its slots are 16-byte aligned
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int64_t row = m0 + i * 16 + g + 8 * h;
            if (row >= J.M) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int64_t col = n0 + j * 8 + 2 * tq;
              double* wp = J.W + (row - J.wr0) * J.ldw + (col - J.wc0);
              if (wvec && col + 1 < J.N) {
                *reinterpret_cast<double2*>(wp) = make_double2(acc[i][j][2 * h], acc[i][j][2 * h + 1]);
              } else {
                if (col < J.N) wp[0] = acc[i][j][2 * h];
                if (col + 1 < J.N) wp[1] = acc[i][j][2 * h + 1];
              }
            }
          }
        continue;
      }
      const bool vec = ((J.ldc & 1) == 0) && ((reinterpret_cast<uintptr_t>(J.C) & 15) == 0);
      const bool use_c = J.beta != 0.0;
      // Per 16-row half of the warp's block, every C0 value is loaded before the first store: the
      // stores go through the same pointer, so a load written after one could not be moved ahead
      // of it, and each 16-byte pair would wait for its own round trip to memory.
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        double c0[2][4][2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int64_t row = m0 + i * 16 + g + 8 * h;
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int64_t col = n0 + j * 8 + 2 * tq;
            c0[h][j][0] = c0[h][j][1] = 0.0;
            if (use_c && row < J.M) {
              const double* cp = J.C + row * J.ldc + col;
              if (vec && col + 1 < J.N) {
                const double2 c = *reinterpret_cast<const double2*>(cp);
                c0[h][j][0] = c.x;
                c0[h][j][1] = c.y;
              } else {
                if (col < J.N) c0[h][j][0] = cp[0];
                if (col + 1 < J.N) c0[h][j][1] = cp[1];
              }
            }
          }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int64_t row = m0 + i * 16 + g + 8 * h;
          if (row >= J.M) continue;
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int64_t col = n0 + j * 8 + 2 * tq;
            const double v0 = acc[i][j][2 * h], v1 = acc[i][j][2 * h + 1];
            const double o0 = use_c ? fma(J.alpha, v0, J.beta * c0[h][j][0]) : J.alpha * v0;
            const double o1 = use_c ? fma(J.alpha, v1, J.beta * c0[h][j][1]) : J.alpha * v1;
            double* cp = J.C + row * J.ldc + col;
            if (vec && col + 1 < J.N) {
              *reinterpret_cast<double2*>(cp) = make_double2(o0, o1);
            } else {
              if (col < J.N) cp[0] = o0;
              if (col + 1 < J.N) cp[1] = o1;
            }
          }
        }
      }
    }
  }
}

template <class Cfg>
__global__ void __launch_bounds__(Cfg::THREADS, Cfg::MIN_BLOCKS)
    dgemm_fp64_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Params p) {
  SingleSource<Cfg> src{p, (p.M + Cfg::BM - 1) / Cfg::BM, (p.N + Cfg::BN - 1) / Cfg::BN, &tmA, &tmB};
  gemm_body<Cfg>(&tmA, &tmB, src, p.status);
}

// C = alpha * (W_0 + W_1 + ... + W_{splits-1}) + beta * C, summed in split order; W is packed
// (M x N), C has row stride ldc.
__global__ void splitk_reduce_kernel(const double* __restrict__ W, double* __restrict__ C, int64_t n, int64_t N,
                                     int64_t ldc, int splits, double alpha, double beta) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = W[i];
    for (int k = 1; k < splits; ++k) s += W[k * n + i];
    double* c = C + (i / N) * ldc + (i % N);
    *c = (beta != 0.0) ? fma(alpha, s, beta * *c) : alpha * s;
  }
}

// Stream-K fix-up: for every tile that several CTAs shared, C = alpha * (their partial sums added
// in K order, i.e. in CTA order) + beta * C. Tiles that one CTA covered whole are already in C.
// 256 threads; each holds BM*BN/256 elements of the tile (consecutive threads on consecutive
// elements), so each slot's index is worked out once per tile and CTA, not per element.
constexpr int kFixupThreads = 256;
template <int BM, int BN>
__global__ void __launch_bounds__(kFixupThreads)
    streamk_fixup_kernel(const double* __restrict__ W, double* __restrict__ C, int64_t M, int64_t N, int64_t ldc,
                         int64_t tiles_m, int64_t tiles_n, int64_t nkb, int64_t G, double alpha, double beta) {
  constexpr int kPer = BM * BN / kFixupThreads;
  static_assert(BM * BN % kFixupThreads == 0, "tile size");
  const int64_t tiles = tiles_m * tiles_n, total = tiles * nkb;
  for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int64_t b_lo = streamk_owner(t * nkb, total, G), b_hi = streamk_owner((t + 1) * nkb - 1, total, G);
    if (b_lo == b_hi) continue;
    double s[kPer];
    for (int64_t b = b_lo; b <= b_hi; ++b) {
      const int64_t slot = 2 * b + (t == streamk_first(b, total, G) / nkb ? 0 : 1);
      const double* __restrict__ w = W + slot * (BM * BN) + threadIdx.x;
#pragma unroll
      for (int k = 0; k < kPer; ++k) {
        const double v = w[k * kFixupThreads];
        s[k] = (b == b_lo) ? v : s[k] + v;
      }
    }
    int64_t tm, tn;
    tile_coords(t, tiles_m, tiles_n, tm, tn);
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int e = threadIdx.x + k * kFixupThreads;
      const int64_t row = tm * BM + e / BN, col = tn * BN + e % BN;
      if (row >= M || col >= N) continue;
      double* c = C + row * ldc + col;
      *c = (beta != 0.0) ? fma(alpha, s[k], beta * *c) : alpha * s[k];
    }
  }
}

template <class Cfg>
__global__ void __launch_bounds__(Cfg::THREADS, Cfg::MIN_BLOCKS)
    dgemm_fp64_grouped_kernel(GroupedSource src, DeviceStatus* status) {
  gemm_body<Cfg>(nullptr, nullptr, src, status);
}

}  // namespace fp64
}  // namespace lt
