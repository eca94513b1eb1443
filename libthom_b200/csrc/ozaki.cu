// ozaki.cu — Ozaki-scheme DGEMM on INT8 tensor cores (tcgen05 kind::i8) for sm_100a.
//
// No reference counterpart: this is a new implementation behind the reference's dgemm contract
// (routines/dgemm/dgemm.h:9). Method: error-free splitting of Ozaki, Ogita, Oishi and Rump (2012)
// with INT8 slices as in Ootomo, Ozaki and Yokota (2024); the code is written from the mathematics.
//
//   1. amax pass (HBM-bound): per row of A and per column of B, the largest |x| as IEEE bits
//      (NaN/Inf order above every finite value, so one atomicMax finds both). sigma_i / tau_j are
//      the frexp exponents of those maxima, so |A[i,k] 2^-sigma_i| < 1.
//   2. split pass (HBM-bound): x = a 2^-sigma; for p = 1..s: y = 128 x, q_p = trunc(y), x = y - q_p.
//      Every step is exact in FP64; q_p in [-127, 127] is stored as int8. A slices are laid out
//      [s][M][Kp] and B slices [s][N][Kp] (B transposed to K-major), Kp = K rounded up to 32.
//   3. product pass (tensor cores): for the triangular pair set p + q <= s + 1, INT8 x INT8 -> INT32
//      MMAs. Diagonals d = p + q share a power of two, so all pairs of a diagonal accumulate into one
//      INT32 TMEM accumulator. Four diagonals ("a band") are live at once (4 x 128 TMEM columns),
//      so every 32-wide K chunk of each slice is loaded into shared memory once per band and feeds
//      all pairs of the band that use it. K is cut into groups short enough that no INT32 sum can
//      overflow (|q| <= 127).
//   4. fused recombination: eight epilogue warps keep the 128 x 128 tile of FP64 partial sums in
//      registers; after each group they read the band's accumulators from TMEM and add
//      D * 2^(-7d) in a fixed order; at the end of the tile they write
//      C = fma(alpha, acc 2^sigma_i 2^tau_j, beta C0).
// The CPU oracle (oracle/oracle.c, oracle_ozaki_dgemm) performs the same arithmetic in the same
// order, so results are bit-identical.
#include <cmath>
#include <cstring>
#include <mutex>

#include "lt_internal.h"
#include "lt_runtime.cuh"

namespace lt {
namespace ozaki {

constexpr int kTileM = 128;
constexpr int kTileN = 128;
constexpr int kChunk = 32;                       // K elements per MMA (= bytes of an INT8 row)
constexpr int kTileBytes = kTileM * kChunk;      // one 128 x 32 INT8 tile
constexpr int kBand = 4;                         // live diagonal accumulators (4 x 128 TMEM cols)
constexpr int kKPairLimit = 133144;              // floor((2^31 - 1) / 127^2)
constexpr int kThreads = 320;                    // warp 0 TMA, warp 1 MMA, warps 2..9 epilogue
constexpr int kEpilogueWarps = 8;
constexpr int kMaxSmem = 232448;                 // sm_100 opt-in dynamic shared memory per block
constexpr int kSentinel = 0x7fffffff;            // exponent of a row/column holding NaN or Inf

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// ---------------------------------------------------------------------------------------------
// Workspace: [amaxA: M u64][amaxB: N u64][A slices: s*M*Kp][B slices: s*N*Kp], 256-byte aligned.
// ---------------------------------------------------------------------------------------------
struct Layout {
  int64_t Kp;
  size_t off_amax_a, off_amax_b, off_sa, off_sb, total;
};

Layout layout_for(int64_t M, int64_t N, int64_t K, int s) {
  Layout L;
  L.Kp = round_up(K > 0 ? K : 1, kChunk);
  size_t o = 0;
  L.off_amax_a = o; o += round_up(8 * M, 256);
  L.off_amax_b = o; o += round_up(8 * N, 256);
  L.off_sa = o;     o += round_up(static_cast<int64_t>(s) * M * L.Kp, 256);
  L.off_sb = o;     o += round_up(static_cast<int64_t>(s) * N * L.Kp, 256);
  L.total = o;
  return L;
}

size_t workspace_size(int64_t M, int64_t N, int64_t K, int slices) { return layout_for(M, N, K, slices).total; }

// ---------------------------------------------------------------------------------------------
// Exponent helpers
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ int exponent_of_maxbits(unsigned long long bits) {
  if (bits == 0ull) return 0;
  if (bits >= 0x7ff0000000000000ull) return kSentinel;
  int e;
  frexp(__longlong_as_double(static_cast<long long>(bits)), &e);
  return e;
}

__device__ __forceinline__ unsigned long long abs_bits(double v) {
  return static_cast<unsigned long long>(__double_as_longlong(v)) & 0x7fffffffffffffffull;
}

// Row maxima of A: blockIdx.x covers 8 rows (one warp each), blockIdx.y a K segment.
__global__ void amax_rows_kernel(const double* __restrict__ A, int64_t M, int64_t K, int64_t kseg,
                                 unsigned long long* __restrict__ amax) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = static_cast<int64_t>(blockIdx.x) * 8 + warp;
  if (row >= M) return;
  const int64_t k0 = static_cast<int64_t>(blockIdx.y) * kseg;
  const int64_t k1 = (k0 + kseg < K) ? k0 + kseg : K;
  const double* a = A + row * K;
  unsigned long long m = 0;
  for (int64_t k = k0 + lane; k < k1; k += 32) {
    unsigned long long b = abs_bits(__ldg(a + k));
    m = b > m ? b : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long x = __shfl_xor_sync(0xffffffffu, m, o);
    m = x > m ? x : m;
  }
  if (lane == 0 && m != 0) atomicMax(&amax[row], m);
}

// Column maxima of B: blockIdx.x covers 256 columns (one per thread), blockIdx.y a K segment.
__global__ void amax_cols_kernel(const double* __restrict__ B, int64_t K, int64_t N, int64_t kseg,
                                 unsigned long long* __restrict__ amax) {
  const int64_t col = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (col >= N) return;
  const int64_t k0 = static_cast<int64_t>(blockIdx.y) * kseg;
  const int64_t k1 = (k0 + kseg < K) ? k0 + kseg : K;
  unsigned long long m = 0;
  for (int64_t k = k0; k < k1; ++k) {
    unsigned long long b = abs_bits(__ldg(B + k * N + col));
    m = b > m ? b : m;
  }
  if (m != 0) atomicMax(&amax[col], m);
}

// Splits one value into S slices q_1..q_S, OR-ing byte j of each into packed[p][j / 4].
template <int S>
__device__ __forceinline__ void split_value(double a, int e, int j, uint32_t (&packed)[S][8]) {
  if (e == kSentinel || !isfinite(a)) return;  // all-zero slices
  double x = scale_pow2(a, -e);
#pragma unroll
  for (int p = 0; p < S; ++p) {
    double y = __dmul_rn(x, 128.0);
    double q = trunc(y);
    x = __dsub_rn(y, q);
    packed[p][j >> 2] |= (static_cast<uint32_t>(static_cast<int>(q)) & 0xffu) << (8 * (j & 3));
  }
}

// A rows -> slices [s][M][Kp]. Each thread: one row, 32 consecutive k (32 bytes per slice).
template <int S>
__global__ void split_rows_kernel(const double* __restrict__ A, int64_t M, int64_t K, int64_t Kp,
                                  const unsigned long long* __restrict__ amax, int8_t* __restrict__ out) {
  const int64_t chunks = Kp / kChunk;
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= M * chunks) return;
  const int64_t row = idx / chunks, c = idx % chunks;
  const int e = exponent_of_maxbits(amax[row]);
  const int64_t k0 = c * kChunk;
  const double* a = A + row * K;
  uint32_t packed[S][8];
#pragma unroll
  for (int p = 0; p < S; ++p)
#pragma unroll
    for (int w = 0; w < 8; ++w) packed[p][w] = 0u;
#pragma unroll
  for (int j = 0; j < kChunk; ++j) {
    const int64_t k = k0 + j;
    const double v = (k < K) ? __ldg(a + k) : 0.0;
    split_value<S>(v, e, j, packed);
  }
#pragma unroll
  for (int p = 0; p < S; ++p) {
    uint4* dst = reinterpret_cast<uint4*>(out + (static_cast<int64_t>(p) * M + row) * Kp + k0);
    dst[0] = make_uint4(packed[p][0], packed[p][1], packed[p][2], packed[p][3]);
    dst[1] = make_uint4(packed[p][4], packed[p][5], packed[p][6], packed[p][7]);
  }
}

// B columns -> slices [s][N][Kp] (K-major). Each thread: one column, 32 consecutive k; the loads
// of a warp are 32 consecutive doubles of one row of B.
template <int S>
__global__ void split_cols_kernel(const double* __restrict__ B, int64_t K, int64_t N, int64_t Kp,
                                  const unsigned long long* __restrict__ amax, int8_t* __restrict__ out) {
  const int64_t col = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (col >= N) return;
  const int e = exponent_of_maxbits(amax[col]);
  for (int64_t kc = blockIdx.y; kc < Kp / kChunk; kc += gridDim.y) {
  const int64_t k0 = kc * kChunk;
  uint32_t packed[S][8];
#pragma unroll
  for (int p = 0; p < S; ++p)
#pragma unroll
    for (int w = 0; w < 8; ++w) packed[p][w] = 0u;
#pragma unroll
  for (int j = 0; j < kChunk; ++j) {
    const int64_t k = k0 + j;
    const double v = (k < K) ? __ldg(B + k * N + col) : 0.0;
    split_value<S>(v, e, j, packed);
  }
#pragma unroll
  for (int p = 0; p < S; ++p) {
    uint4* dst = reinterpret_cast<uint4*>(out + (static_cast<int64_t>(p) * N + col) * Kp + k0);
    dst[0] = make_uint4(packed[p][0], packed[p][1], packed[p][2], packed[p][3]);
    dst[1] = make_uint4(packed[p][4], packed[p][5], packed[p][6], packed[p][7]);
  }
  }
}

// ---------------------------------------------------------------------------------------------
// Product + recombination kernel
// ---------------------------------------------------------------------------------------------
struct GemmParams {
  int64_t M, N, nkc;  // nkc = Kp / 32
  int s, stages, stage_tiles;
  double alpha, beta;
  double* C;
  const unsigned long long* amax_a;
  const unsigned long long* amax_b;
  DeviceStatus* status;
};

// Band b of s slices: diagonals dhi = s + 1 - 4b down to dlo; A/B slices 1..nsl are involved.
struct Band {
  int dhi, dlo, nsl, maxp, gchunks, cps;
};

__device__ __forceinline__ int pair_lo(int d, int s) { return d - s > 1 ? d - s : 1; }
__device__ __forceinline__ int pair_hi(int d, int s) { return d - 1 < s ? d - 1 : s; }

__device__ __forceinline__ Band make_band(int b, int s, int stage_tiles) {
  Band B;
  B.dhi = s + 1 - kBand * b;
  B.dlo = B.dhi - kBand + 1 < 2 ? 2 : B.dhi - kBand + 1;
  B.nsl = B.dhi - 1 < s ? B.dhi - 1 : s;
  B.maxp = 0;
  for (int d = B.dhi; d >= B.dlo; --d) {
    int np = pair_hi(d, s) - pair_lo(d, s) + 1;
    B.maxp = np > B.maxp ? np : B.maxp;
  }
  B.gchunks = kKPairLimit / (kChunk * B.maxp);
  B.cps = stage_tiles / (2 * B.nsl);
  return B;
}

__device__ __forceinline__ int num_bands(int s) { return (s + kBand - 1) / kBand; }

// Shared-memory matrix descriptor, K-major, 32-byte swizzle: rows of 32 bytes, 8-row groups
// 256 bytes apart (SBO), layout type SWIZZLE_32B (6), descriptor version 1.
__device__ __forceinline__ uint64_t desc_k_sw32(uint32_t addr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>(1u) << 16;
  d |= static_cast<uint64_t>(256u >> 4) << 32;
  d |= static_cast<uint64_t>(1u) << 46;
  d |= static_cast<uint64_t>(6u) << 61;
  return d;
}

__global__ void __launch_bounds__(kThreads, 1)
    ozaki_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmParams p) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int stage_bytes = p.stage_tiles * kTileBytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + p.stages * stage_bytes);
  uint64_t* empty = full + p.stages;
  uint64_t* acc_full = empty + p.stages;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* drain = acc_empty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t tiles_m = (p.M + kTileM - 1) / kTileM, tiles_n = (p.N + kTileN - 1) / kTileN;
  const int64_t tiles = tiles_m * tiles_n;
  const int nb = num_bands(p.s);

  if (threadIdx.x == 0) {
    for (int i = 0; i < p.stages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, kEpilogueWarps);
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ----------------------------------- TMA producer -----------------------------------
    if (lane == 0) {
      tma_prefetch_desc(&tmA);
      tma_prefetch_desc(&tmB);
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        int64_t tm, tn;
        {
          const int64_t G = 8;
          int64_t group = t / (G * tiles_n), first_m = group * G;
          int64_t gsize = (tiles_m - first_m) < G ? (tiles_m - first_m) : G;
          int64_t in_group = t - group * G * tiles_n;
          tm = first_m + in_group % gsize;
          tn = in_group / gsize;
        }
        const int m0 = static_cast<int>(tm * kTileM), n0 = static_cast<int>(tn * kTileN);
        for (int b = 0; b < nb && ok; ++b) {
          const Band bd = make_band(b, p.s, p.stage_tiles);
          for (int64_t c0 = 0; c0 < p.nkc && ok; c0 += bd.gchunks) {
            const int64_t c1 = (c0 + bd.gchunks < p.nkc) ? c0 + bd.gchunks : p.nkc;
            for (int64_t cs = c0; cs < c1; cs += bd.cps) {
              const int64_t ce = (cs + bd.cps < c1) ? cs + bd.cps : c1;
              if (!mbar_wait(&empty[stage], phase ^ 1, abort_flag, p.status, 11)) { ok = false; break; }
              uint8_t* st = smem + stage * stage_bytes;
              mbar_arrive_expect_tx(&full[stage], static_cast<uint32_t>((ce - cs) * 2 * bd.nsl * kTileBytes));
              for (int64_t c = cs; c < ce; ++c) {
                uint8_t* base = st + (c - cs) * 2 * bd.nsl * kTileBytes;
                const int x = static_cast<int>(c * kChunk);
                for (int q = 0; q < bd.nsl; ++q) tma_load_3d(base + q * kTileBytes, &tmA, &full[stage], x, m0, q);
                for (int q = 0; q < bd.nsl; ++q)
                  tma_load_3d(base + (bd.nsl + q) * kTileBytes, &tmB, &full[stage], x, n0, q);
              }
              if (++stage == p.stages) { stage = 0; phase ^= 1; }
            }
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------ MMA issuer ------------------------------------
    constexpr uint32_t idesc = idesc_i8_s32(kTileM, kTileN);
    const uint32_t smem_base = smem_u32(smem);
    int stage = 0;
    uint32_t phase = 0;
    uint32_t group = 0;
    bool ok = true;
    for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
      for (int b = 0; b < nb && ok; ++b) {
        const Band bd = make_band(b, p.s, p.stage_tiles);
        for (int64_t c0 = 0; c0 < p.nkc && ok; c0 += bd.gchunks) {
          const int64_t c1 = (c0 + bd.gchunks < p.nkc) ? c0 + bd.gchunks : p.nkc;
          if (!mbar_wait(acc_empty, (group & 1) ^ 1, abort_flag, p.status, 12)) { ok = false; break; }
          tc_fence_after();
          for (int64_t cs = c0; cs < c1; cs += bd.cps) {
            const int64_t ce = (cs + bd.cps < c1) ? cs + bd.cps : c1;
            if (!mbar_wait(&full[stage], phase, abort_flag, p.status, 13)) { ok = false; break; }
            tc_fence_after();
            if (lane == 0) {
              const uint32_t st = smem_base + stage * stage_bytes;
              for (int64_t c = cs; c < ce; ++c) {
                const uint32_t base = st + static_cast<uint32_t>((c - cs) * 2 * bd.nsl * kTileBytes);
                for (int j = 0; j < kBand; ++j) {
                  const int d = bd.dhi - j;
                  if (d < bd.dlo) break;
                  const int plo = pair_lo(d, p.s), phi = pair_hi(d, p.s);
                  for (int pp = plo; pp <= phi; ++pp) {
                    const int qq = d - pp;
                    const uint64_t adesc = desc_k_sw32(base + (pp - 1) * kTileBytes);
                    const uint64_t bdesc = desc_k_sw32(base + (bd.nsl + qq - 1) * kTileBytes);
                    const uint32_t accum = (c == c0 && pp == plo) ? 0u : 1u;
                    mma_i8(tmem_base + static_cast<uint32_t>(j * kTileN), adesc, bdesc, idesc, accum);
                  }
                }
              }
              mma_commit(&empty[stage]);
            }
            __syncwarp();
            if (++stage == p.stages) { stage = 0; phase ^= 1; }
          }
          if (!ok) break;
          if (lane == 0) mma_commit(acc_full);
          __syncwarp();
          ++group;
        }
      }
    }
    if (!ok && lane == 0) {
      // Let every MMA already issued finish before TMEM is released.
      mma_commit(drain);
      uint64_t t0 = globaltimer();
      while (!mbar_try_wait(drain, 0) && globaltimer() - t0 < LT_WAIT_TIMEOUT_NS) {
      }
    }
    __syncwarp();
  } else {
    // ------------------------------- epilogue (8 warps) -------------------------------
    const int ew = warp - 2;
    const int quarter = warp & 3;         // TMEM lanes 32*quarter .. +31 are visible to this warp
    const int half = ew >> 2;             // columns 64*half .. +63 of the tile
    const int row_in_tile = quarter * 32 + lane;
    uint32_t group = 0;
    bool ok = true;
    for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
      int64_t tm, tn;
      {
        const int64_t G = 8;
        int64_t grp = t / (G * tiles_n), first_m = grp * G;
        int64_t gsize = (tiles_m - first_m) < G ? (tiles_m - first_m) : G;
        int64_t in_group = t - grp * G * tiles_n;
        tm = first_m + in_group % gsize;
        tn = in_group / gsize;
      }
      double acc[64];
#pragma unroll
      for (int i = 0; i < 64; ++i) acc[i] = 0.0;
      for (int b = 0; b < nb && ok; ++b) {
        const Band bd = make_band(b, p.s, p.stage_tiles);
        for (int64_t c0 = 0; c0 < p.nkc; c0 += bd.gchunks) {
          if (!mbar_wait(acc_full, group & 1, abort_flag, p.status, 14)) { ok = false; break; }
          tc_fence_after();
          for (int j = 0; j < kBand; ++j) {
            const int d = bd.dhi - j;
            if (d < bd.dlo) break;
            const double sc = pow2i(-7 * d);
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
              uint32_t v[32];
              const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) +
                                     static_cast<uint32_t>(j * kTileN + half * 64 + cc * 32);
              tmem_ld_32x32b_x32(taddr, v);
              tmem_ld_wait();
#pragma unroll
              for (int i = 0; i < 32; ++i)
                acc[cc * 32 + i] = __dadd_rn(acc[cc * 32 + i], __dmul_rn(static_cast<double>(static_cast<int32_t>(v[i])), sc));
            }
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(acc_empty);
          ++group;
        }
      }
      if (!ok) break;
      // ---- C = fma(alpha, acc 2^sigma 2^tau, beta C0) ----
      const int64_t row = tm * kTileM + row_in_tile;
      if (row < p.M) {
        const int sig = exponent_of_maxbits(p.amax_a[row]);
        const int64_t col0 = tn * kTileN + half * 64;
        double* crow = p.C + row * p.N;
#pragma unroll
        for (int i = 0; i < 64; ++i) {
          const int64_t col = col0 + i;
          if (col < p.N) {
            const int tau = exponent_of_maxbits(p.amax_b[col]);
            double out;
            if (sig == kSentinel || tau == kSentinel) {
              out = __longlong_as_double(0x7ff8000000000000ll);
            } else {
              const double tv = scale_pow2(scale_pow2(acc[i], sig), tau);
              out = (p.beta != 0.0) ? fma(p.alpha, tv, __dmul_rn(p.beta, crow[col])) : __dmul_rn(p.alpha, tv);
            }
            crow[col] = out;
          }
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, 512);
  }
}

// ---------------------------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------------------------
template <int S>
int launch_split_s(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int64_t Kp,
                   const unsigned long long* amax_a, const unsigned long long* amax_b, int8_t* sa, int8_t* sb,
                   cudaStream_t stream) {
  const int64_t chunks = Kp / kChunk;
  const int64_t n = M * chunks;
  if (n > 0) split_rows_kernel<S><<<static_cast<unsigned>((n + 127) / 128), 128, 0, stream>>>(A, M, K, Kp, amax_a, sa);
  LT_CUDA_TRY(cudaGetLastError());
  if (N > 0)
    split_cols_kernel<S><<<dim3(static_cast<unsigned>((N + 127) / 128), static_cast<unsigned>(chunks < 65535 ? chunks : 65535)), 128, 0, stream>>>(
        B, K, N, Kp, amax_b, sb);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

int launch_split(int s, const double* A, const double* B, int64_t M, int64_t N, int64_t K, int64_t Kp,
                 const unsigned long long* amax_a, const unsigned long long* amax_b, int8_t* sa, int8_t* sb,
                 cudaStream_t stream) {
  switch (s) {
#define LT_SPLIT_CASE(S) \
  case S: return launch_split_s<S>(A, B, M, N, K, Kp, amax_a, amax_b, sa, sb, stream);
    LT_SPLIT_CASE(1) LT_SPLIT_CASE(2) LT_SPLIT_CASE(3) LT_SPLIT_CASE(4) LT_SPLIT_CASE(5) LT_SPLIT_CASE(6)
    LT_SPLIT_CASE(7) LT_SPLIT_CASE(8) LT_SPLIT_CASE(9) LT_SPLIT_CASE(10) LT_SPLIT_CASE(11) LT_SPLIT_CASE(12)
#undef LT_SPLIT_CASE
    default: return set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d unsupported", s);
  }
}

// Stage 1+2: exponents and slices of A and B into the workspace.
int split(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int s, void* workspace,
          size_t workspace_bytes, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  const Layout L = layout_for(M, N, K, s);
  if (workspace_bytes < L.total) return set_error(LT_ERR_NO_MEMORY, "Ozaki workspace too small");
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  auto* amax_a = reinterpret_cast<unsigned long long*>(ws + L.off_amax_a);
  auto* amax_b = reinterpret_cast<unsigned long long*>(ws + L.off_amax_b);
  auto* sa = reinterpret_cast<int8_t*>(ws + L.off_sa);
  auto* sb = reinterpret_cast<int8_t*>(ws + L.off_sb);

  LT_CUDA_TRY(cudaMemsetAsync(ws, 0, L.off_sa, stream));
  const int sms = ctx->sm_count;
  if (K > 0) {
    // amax of A rows: 8 rows per block, K split so that the grid covers the GPU.
    int64_t row_blocks = (M + 7) / 8;
    int64_t ksplit = (4 * sms + row_blocks - 1) / row_blocks;
    ksplit = ksplit < 1 ? 1 : ksplit;
    int64_t kseg = round_up((K + ksplit - 1) / ksplit, 256);
    ksplit = (K + kseg - 1) / kseg;
    amax_rows_kernel<<<dim3(static_cast<unsigned>(row_blocks), static_cast<unsigned>(ksplit)), 256, 0, stream>>>(
        A, M, K, kseg, amax_a);
    LT_CUDA_TRY(cudaGetLastError());
    int64_t col_blocks = (N + 255) / 256;
    int64_t ksplit_b = (8 * sms + col_blocks - 1) / col_blocks;
    ksplit_b = ksplit_b < 1 ? 1 : ksplit_b;
    int64_t kseg_b = (K + ksplit_b - 1) / ksplit_b;
    ksplit_b = (K + kseg_b - 1) / kseg_b;
    amax_cols_kernel<<<dim3(static_cast<unsigned>(col_blocks), static_cast<unsigned>(ksplit_b)), 256, 0, stream>>>(
        B, K, N, kseg_b, amax_b);
    LT_CUDA_TRY(cudaGetLastError());
  }
  LT_TRY(launch_split(s, A, B, M, N, K, L.Kp, amax_a, amax_b, sa, sb, stream));
  return LT_OK;
}

// Stage 3+4: slice products on the tensor cores and the fused FP64 recombination into C.
int product(double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int s, const void* workspace,
            size_t workspace_bytes, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  const Layout L = layout_for(M, N, K, s);
  if (workspace_bytes < L.total) return set_error(LT_ERR_NO_MEMORY, "Ozaki workspace too small");
  const uint8_t* ws = static_cast<const uint8_t*>(workspace);
  const auto* amax_a = reinterpret_cast<const unsigned long long*>(ws + L.off_amax_a);
  const auto* amax_b = reinterpret_cast<const unsigned long long*>(ws + L.off_amax_b);
  const auto* sa = reinterpret_cast<const int8_t*>(ws + L.off_sa);
  const auto* sb = reinterpret_cast<const int8_t*>(ws + L.off_sb);
  const int sms = ctx->sm_count;
  const int64_t chunks = L.Kp / kChunk;

  // Slices as 3-D tensors [s][rows][Kp] of bytes; one TMA box = 32 K x 128 rows of one slice.
  CUtensorMap tmA, tmB;
  LT_TRY(make_tmap_3d(&tmA, sa, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, static_cast<uint64_t>(s), static_cast<uint64_t>(M),
                      static_cast<uint64_t>(L.Kp), static_cast<uint64_t>(L.Kp), static_cast<uint64_t>(M * L.Kp),
                      kTileM, kChunk, CU_TENSOR_MAP_SWIZZLE_32B));
  LT_TRY(make_tmap_3d(&tmB, sb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, static_cast<uint64_t>(s), static_cast<uint64_t>(N),
                      static_cast<uint64_t>(L.Kp), static_cast<uint64_t>(L.Kp), static_cast<uint64_t>(N * L.Kp),
                      kTileN, kChunk, CU_TENSOR_MAP_SWIZZLE_32B));

  GemmParams gp;
  gp.M = M;
  gp.N = N;
  gp.nkc = chunks;
  gp.s = s;
  gp.stage_tiles = 2 * s;
  const int stage_bytes = gp.stage_tiles * kTileBytes;
  const int overhead = 1024 + 256;
  gp.stages = (kMaxSmem - overhead) / stage_bytes;
  if (gp.stages > 6) gp.stages = 6;
  if (gp.stages < 2) return set_error(LT_ERR_UNSUPPORTED, "slice count %d needs more shared memory", s);
  gp.alpha = alpha;
  gp.beta = beta;
  gp.C = C;
  gp.amax_a = amax_a;
  gp.amax_b = amax_b;
  gp.status = ctx->status;
  const int smem = gp.stages * stage_bytes + overhead;

  static std::once_flag once[64];
  static cudaError_t attr_err[64];
  std::call_once(once[ctx->device], [&] {
    attr_err[ctx->device] =
        cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
  });
  LT_CUDA_TRY(attr_err[ctx->device]);
  const int64_t tiles = ((M + kTileM - 1) / kTileM) * ((N + kTileN - 1) / kTileN);
  const int64_t grid = tiles < sms ? tiles : sms;
  ozaki_gemm_kernel<<<static_cast<unsigned>(grid), kThreads, smem, stream>>>(tmA, tmB, gp);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

int run(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int s,
        void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  LT_TRY(split(A, B, M, N, K, s, workspace, workspace_bytes, stream));
  return product(C, M, N, K, alpha, beta, s, workspace, workspace_bytes, stream);
}

}  // namespace ozaki
}  // namespace lt
