// ozaki.cu — Ozaki-scheme DGEMM on INT8 tensor cores (tcgen05 kind::i8) for sm_100a.
//
// No reference counterpart: this is a new implementation behind the reference's dgemm contract
// (routines/dgemm/dgemm.h:9). Method: error-free splitting of Ozaki, Ogita, Oishi and Rump (2012)
// with INT8 slices as in Ootomo, Ozaki and Yokota (2024); the code is written from the mathematics.
//
//   1. amax pass (HBM-bound): per row of A and per column of B, the largest |x| as IEEE bits
//      (NaN/Inf order above every finite value, so one max finds both). sigma_i / tau_j are the
//      frexp exponents of those maxima, so |A[i,k] 2^-sigma_i| < 1.
//   2. split pass (HBM-bound): V = trunc(a 2^(8s-2-sigma)), an integer with |V| < 2^(8s-2), is
//      written in balanced base-256 digits q_1..q_s (q_1 in [-64, 64], the others in [-128, 127]):
//      a = 2^(sigma+2) sum_p q_p 256^-p up to the truncation. Each q_p is stored as int8; the digits
//      are the bytes of V + sum_{i<s-1} 128 * 256^i with the top bit flipped in all but the top one.
//   3. product pass (tensor cores): for the triangular pair set p + q <= s + 1, INT8 x INT8 -> INT32
//      MMAs. Diagonals d = p + q share a power of two, so all pairs of a diagonal accumulate into one
//      INT32 TMEM accumulator. Four diagonals ("a band") are live at once (4 x 128 TMEM columns),
//      so every 32-wide K chunk of each slice is loaded into shared memory once per band and feeds
//      all pairs of the band that use it. K is cut into groups short enough that no INT32 sum can
//      overflow (|q| <= 128).
//   4. fused recombination: eight epilogue warps keep the 128 x 128 tile of FP64 partial sums in
//      registers; after each group they read the band's accumulators from TMEM and add
//      D * 2^(-8d) in a fixed order; at the end of the tile they write
//      C = fma(alpha, acc 2^(sigma_i+2) 2^(tau_j+2), beta C0).
// The CPU oracle (oracle/oracle.c, oracle_ozaki_dgemm) performs the same arithmetic in the same
// order, so results are bit-identical.
//
// Slice layout in HBM ("tiles"): every 128-row x 32-byte block of one slice — exactly one MMA
// operand — is stored as a contiguous 4 KB tile, already in the 32-byte-swizzled K-major order the
// tensor core reads from shared memory (16-byte half h of row r at r*32 + 16*(h ^ ((r >> 2) & 1))).
// Tiles are stored chunk-major: tile (p, rb, c) of an operand with NC chunks and S slices sits at
// ((rb*NC + c)*S + p)*4 KB, so the tiles of slices 1..n of one K chunk are one contiguous n*4 KB
// block and the producer moves them with a single 1-D bulk copy (cp.async.bulk). Each bulk copy
// costs the issuing thread about 100 cycles whatever its size (measured on B200), so copies per
// stage, not bytes, set the producer's pace. B slices that the CTA-pair kernel reads are stored
// half-major inside each chunk block (rows 0..63 of every slice's tile, then rows 64..127), so each
// CTA of the pair loads its halves of all slices with one copy too. Rows beyond M (N) in the last
// block are zero.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include "lt_internal.h"
#include "lt_runtime.cuh"

namespace lt {
namespace ozaki {

constexpr int kTileM = 128;
constexpr int kTileN = 128;
constexpr int kChunk = 32;                       // K elements per MMA (= bytes of an INT8 row)
constexpr int kTileBytes = kTileM * kChunk;      // one 128 x 32 INT8 tile
constexpr int kHalfTileBytes = kTileBytes / 2;   // 64 rows of a tile (one CTA's share of a B tile)
constexpr int kBand = 4;                         // live diagonal accumulators (4 x 128 TMEM cols)
constexpr int kKPairLimit = 131071;              // floor((2^31 - 1) / 128^2)
constexpr int kThreads = 320;                    // warp 0 loads, warp 1 MMA, warps 2..9 epilogue
constexpr int kEpilogueWarps = 8;
constexpr int kMaxSmem = 232448;                 // sm_100 opt-in dynamic shared memory per block
constexpr int kSmemOverhead = 1024 + 256;        // alignment slack + barriers

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }
inline int64_t ceil_div(int64_t x, int64_t m) { return (x + m - 1) / m; }

// ---------------------------------------------------------------------------------------------
// Workspace: [amaxA: M u64][amaxB: N u64][A tiles: s*RBa*NC*4K][B tiles: s*RBb*NC*4K], 256-aligned.
// ---------------------------------------------------------------------------------------------
struct Layout {
  int64_t NC, RBa, RBb;
  size_t off_amax_a, off_amax_b, off_sa, off_sb, total;
};

Layout layout_for(int64_t M, int64_t N, int64_t K, int s) {
  Layout L;
  L.NC = ceil_div(K > 0 ? K : 1, kChunk);
  L.RBa = ceil_div(M, kTileM);
  L.RBb = ceil_div(N, kTileN);
  size_t o = 0;
  L.off_amax_a = o; o += round_up(8 * M, 256);
  L.off_amax_b = o; o += round_up(8 * N, 256);
  L.off_sa = o;     o += static_cast<size_t>(s) * L.RBa * L.NC * kTileBytes;
  L.off_sb = o;     o += static_cast<size_t>(s) * L.RBb * L.NC * kTileBytes;
  L.total = o;
  return L;
}

size_t workspace_size(int64_t M, int64_t N, int64_t K, int slices) { return layout_for(M, N, K, slices).total; }

// ---------------------------------------------------------------------------------------------
// Exponents
// ---------------------------------------------------------------------------------------------
// Row maxima of A: block (bx, by) covers 8 rows (one warp each) and K segment by.
__device__ __forceinline__ void amax_rows_block(const double* __restrict__ A, int64_t M, int64_t K, int64_t lda,
                                                int64_t kseg, unsigned long long* __restrict__ amax, int64_t bx,
                                                int64_t by) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = bx * 8 + warp;
  if (row >= M) return;
  const int64_t k0 = by * kseg;
  const int64_t k1 = (k0 + kseg < K) ? k0 + kseg : K;
  const double* a = A + row * lda;
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

__global__ void amax_rows_kernel(const double* __restrict__ A, int64_t M, int64_t K, int64_t lda, int64_t kseg,
                                 unsigned long long* __restrict__ amax) {
  amax_rows_block(A, M, K, lda, kseg, amax, blockIdx.x, blockIdx.y);
}

// Column maxima of B: block (bx, by) covers 256 columns (one per thread) and K segment by. With
// 16-byte aligned rows (B aligned, N even) each thread reads two adjacent columns per load and the
// block covers 512 columns (`pairs` set by the launcher).
__device__ __forceinline__ void amax_cols_block(const double* __restrict__ B, int64_t K, int64_t N, int64_t ldb,
                                                int64_t kseg, unsigned long long* __restrict__ amax, int pairs,
                                                int64_t bx, int64_t by) {
  const int64_t k0 = by * kseg;
  const int64_t k1 = (k0 + kseg < K) ? k0 + kseg : K;
  if (pairs) {
    const int64_t col = 2 * (bx * blockDim.x + threadIdx.x);
    if (col >= N) return;
    unsigned long long m0 = 0, m1 = 0;
    const double* bp = B + k0 * ldb + col;
#pragma unroll 4
    for (int64_t k = k0; k < k1; ++k, bp += ldb) {
      const double2 v = __ldg(reinterpret_cast<const double2*>(bp));
      const unsigned long long b0 = abs_bits(v.x), b1 = abs_bits(v.y);
      m0 = b0 > m0 ? b0 : m0;
      m1 = b1 > m1 ? b1 : m1;
    }
    if (m0 != 0) atomicMax(&amax[col], m0);
    if (m1 != 0) atomicMax(&amax[col + 1], m1);
    return;
  }
  const int64_t col = bx * blockDim.x + threadIdx.x;
  if (col >= N) return;
  unsigned long long m = 0;
  for (int64_t k = k0; k < k1; ++k) {
    unsigned long long b = abs_bits(__ldg(B + k * ldb + col));
    m = b > m ? b : m;
  }
  if (m != 0) atomicMax(&amax[col], m);
}

__global__ void amax_cols_kernel(const double* __restrict__ B, int64_t K, int64_t N, int64_t ldb, int64_t kseg,
                                 unsigned long long* __restrict__ amax, int pairs) {
  amax_cols_block(B, K, N, ldb, kseg, amax, pairs, blockIdx.x, blockIdx.y);
}

// Both sides' maxima in one launch (256 threads): blocks 0 .. ra*ka-1 are A's row blocks (ra of
// them per K segment, ka segments), the rest B's column blocks (rb per segment).
__global__ void amax_both_kernel(const double* __restrict__ A, int64_t M, int64_t K, int64_t kseg_a, int64_t ra,
                                 int64_t ka, unsigned long long* __restrict__ amax_a, const double* __restrict__ B,
                                 int64_t N, int64_t kseg_b, int64_t rb, int pairs,
                                 unsigned long long* __restrict__ amax_b) {
  const int64_t id = blockIdx.x;
  if (id < ra * ka) {
    amax_rows_block(A, M, K, K, kseg_a, amax_a, id % ra, id / ra);
  } else {
    const int64_t j = id - ra * ka;
    amax_cols_block(B, K, N, N, kseg_b, amax_b, pairs, j % rb, j / rb);
  }
}

// ---------------------------------------------------------------------------------------------
// Split
// ---------------------------------------------------------------------------------------------
// Balanced base-256 digits. With |a| = m 2^t (m the significand with its hidden bit) and e the row's
// (column's) exponent (|a| < 2^e), V = +-floor(|a| 2^(8S-2-e)) = +-floor(m 2^(t-e+8S-2)) is an
// integer with |V| < 2^(8S-2) and the sign of a (truncation toward zero). D = V + C with
// C = sum_{i < S-1} 128 * 256^i, as a two's-complement integer of 8S bits, gives the digits:
// digit i (i = 0 least significant) = byte_i(D) - 128 in [-128, 127] for i < S-1, and
// floor(D / 256^(S-1)) in [-64, 64] for the top one, so that V = sum_i digit_i 256^i and
// a = 2^(e+2) sum_{p=1..S} q_p 256^-p with q_p = digit S-p. As int8 bytes: the bytes of D with the
// top bit flipped in bytes 0..S-2, and byte S-1 of D as it is. D fits 64 signed bits for S <= 8
// (|D| < 2^62 + 2^56) and is computed in 128 bits above.
template <int S>
using DigitInt = typename std::conditional<(S <= 8), long long, __int128>::type;

template <int S>
__host__ __device__ constexpr DigitInt<S> digit_offset() {
  DigitInt<S> c = 0;
  for (int i = 0; i < S - 1; ++i) c += static_cast<DigitInt<S>>(128) << (8 * i);
  return c;
}

// D of one value; a zero or non-finite entry gives V = 0, i.e. D = C, whose digits are all zero.
template <int S>
__device__ __forceinline__ DigitInt<S> digit_string(double a, int e) {
  using X = DigitInt<S>;
  using U = typename std::conditional<(S <= 8), unsigned long long, unsigned __int128>::type;
  const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(a));
  const unsigned long long mag = bits & 0x7fffffffffffffffull;
  const int E = static_cast<int>(mag >> 52);
  if (mag == 0ull || E == 0x7ff) return digit_offset<S>();
  unsigned long long m = mag & 0x000fffffffffffffull;
  int t;
  if (E == 0) {
    t = -1074;
  } else {
    m |= 0x0010000000000000ull;
    t = E - 1075;
  }
  const int sh = t - e + 8 * S - 2;
  constexpr int kBits = 8 * static_cast<int>(sizeof(U));
  U mg;
  if (sh >= 0) mg = U(m) << sh;
  else mg = (-sh >= kBits) ? U(0) : (U(m) >> (-sh));
  const X v = (bits >> 63) ? -static_cast<X>(mg) : static_cast<X>(mg);
  return v + digit_offset<S>();
}

// Bytes 4j .. 4j+3 of the digit string D as an int8 word (top bit flipped in the bytes of the
// lower S-1 digits).
template <int S>
__device__ __forceinline__ uint32_t digit_word(DigitInt<S> D, int j) {
  uint32_t mask = 0u;
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (4 * j + i < S - 1) mask |= 0x80u << (8 * i);
  return static_cast<uint32_t>(D >> (32 * j)) ^ mask;
}

// Splits one value into S slices q_1..q_S, OR-ing byte j of each into packed[p][j / 4].
template <int S>
__device__ __forceinline__ void split_value(double a, int e, int j, uint32_t (&packed)[S][8]) {
  if (e == kSentinel) return;  // NaN/Inf somewhere in the row/column: zero slices, NaN output
  const DigitInt<S> D = digit_string<S>(a, e);
#pragma unroll
  for (int p = 0; p < S; ++p) {
    const int i = S - 1 - p;  // digit index of slice p
    const uint32_t byte = static_cast<uint32_t>(D >> (8 * i)) & 0xffu;
    const uint32_t q = (i < S - 1) ? (byte ^ 0x80u) : byte;
    packed[p][j >> 2] |= q << (8 * (j & 3));
  }
}

// 4 x 4 byte transpose: on return w[i] byte j = (input w[j]) byte i.
__device__ __forceinline__ void transpose4x4(uint32_t (&w)[4]) {
  const uint32_t t0 = __byte_perm(w[0], w[1], 0x5140), t1 = __byte_perm(w[0], w[1], 0x7362);
  const uint32_t t2 = __byte_perm(w[2], w[3], 0x5140), t3 = __byte_perm(w[2], w[3], 0x7362);
  w[0] = __byte_perm(t0, t2, 0x5410);
  w[1] = __byte_perm(t0, t2, 0x7632);
  w[2] = __byte_perm(t1, t3, 0x5410);
  w[3] = __byte_perm(t1, t3, 0x7632);
}

// Slices of four consecutive values v[0..3] (K positions 4w .. 4w+3 of one row): sets word w of
// every slice, packed[p][w] byte i = digit p of v[i] as a two's-complement byte. Word j of value
// i's digit string holds digits 4j .. 4j+3 counted from the least significant, i.e. slices
// S-1-4j .. S-4-4j; a 4 x 4 byte transpose turns four such words into four slice words. A zero or
// non-finite entry has D = C, whose digits are all zero.
template <int S>
__device__ __forceinline__ void split4(const double (&v)[4], int e, int w, uint32_t (&packed)[S][8]) {
  constexpr int NW = (S + 3) / 4;  // words of four digits
  uint32_t dw[NW][4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const DigitInt<S> D = digit_string<S>(v[i], e);
#pragma unroll
    for (int j = 0; j < NW; ++j) dw[j][i] = digit_word<S>(D, j);
  }
#pragma unroll
  for (int j = 0; j < NW; ++j) {
    transpose4x4(dw[j]);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      constexpr int kS = S;
      const int p = kS - 1 - (4 * j + i);
      if (p >= 0) packed[p >= 0 ? p : 0][w] = dw[j][i];
    }
  }
}

// Writes row r (32 bytes per slice) of tile (rb, c) of every slice, in the swizzled tile order.
// The chunk block (rb, c) holds the S tiles of the chunk. Tile-major (half_major = 0): tile p at
// p * 4 KB, its rows 0..127 contiguous, as the one-CTA kernel reads a 128-row operand. Half-major
// (B slices of the CTA-pair kernel): rows 64h .. 64h+63 of every tile, slices 0..S-1 in turn, form
// half h (S * 2 KB), so the pair's CTA of rank h finds the halves of all slices it needs in one
// contiguous run and loads them with one bulk copy.
template <int S>
__device__ __forceinline__ void store_tile_row(int8_t* out, int64_t RB, int64_t NC, int64_t rb, int64_t c, int r,
                                               const uint32_t (&packed)[S][8], int half_major) {
  const int flip = (r >> 2) & 1;
  (void)RB;
  int8_t* block = out + (rb * NC + c) * S * kTileBytes;
  int64_t step;
  if (half_major) {
    block += (r >> 6) * S * kHalfTileBytes + (r & 63) * 32;
    step = kHalfTileBytes;
  } else {
    block += r * 32;
    step = kTileBytes;
  }
#pragma unroll
  for (int p = 0; p < S; ++p) {
    int8_t* tile = block + p * step;
    uint4 lo = make_uint4(packed[p][0], packed[p][1], packed[p][2], packed[p][3]);
    uint4 hi = make_uint4(packed[p][4], packed[p][5], packed[p][6], packed[p][7]);
    reinterpret_cast<uint4*>(tile)[flip] = lo;
    reinterpret_cast<uint4*>(tile)[flip ^ 1] = hi;
  }
}

// Tile (rb, c) of A: thread r handles row rb*128 + r, K elements 32c .. 32c + 31.
template <int S>
__device__ __forceinline__ void split_rows_tile(const double* __restrict__ A, int64_t M, int64_t K, int64_t lda,
                                                int64_t NC,
                                                int64_t RB, const unsigned long long* __restrict__ amax,
                                                int8_t* __restrict__ out, int64_t rb, int64_t c, int r,
                                                int half_major = 0) {
  const int64_t row = rb * kTileM + r;
  uint32_t packed[S][8];
#pragma unroll
  for (int p = 0; p < S; ++p)
#pragma unroll
    for (int w = 0; w < 8; ++w) packed[p][w] = 0u;
  if (row < M) {
    const int e = exponent_of_maxbits(amax[row]);
    const double* a = A + row * lda;
    const int64_t k0 = c * kChunk;
    if constexpr (S <= LT_OZAKI_MAX_SLICES) {
      if (e != kSentinel) {
        // The whole 32-value chunk is loaded before any digit is extracted, so each thread keeps
        // 256 bytes in flight (memory-level parallelism for an HBM-bound pass). 16-byte loads when
        // the row is 16-byte aligned and the chunk is whole: each lane's two doubles share one L1
        // sector, half the tag lookups of scalar loads across 32 rows.
        const bool vec = ((reinterpret_cast<uintptr_t>(a + k0) & 15) == 0) && (k0 + kChunk <= K);
        double v[kChunk];
        if (vec) {
#pragma unroll
          for (int j = 0; j < kChunk / 2; ++j) {
            const double2 x = __ldg(reinterpret_cast<const double2*>(a + k0 + 2 * j));
            v[2 * j] = x.x;
            v[2 * j + 1] = x.y;
          }
        } else {
#pragma unroll
          for (int j = 0; j < kChunk; ++j) {
            const int64_t k = k0 + j;
            v[j] = (k < K) ? __ldg(a + k) : 0.0;
          }
        }
#pragma unroll
        for (int w = 0; w < 8; ++w) {
          const double q[4] = {v[4 * w], v[4 * w + 1], v[4 * w + 2], v[4 * w + 3]};
          split4<S>(q, e, w, packed);
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < kChunk; ++j) {
        const int64_t k = k0 + j;
        const double v = (k < K) ? __ldg(a + k) : 0.0;
        split_value<S>(v, e, j, packed);
      }
    }
  }
  store_tile_row<S>(out, RB, NC, rb, c, r, packed, half_major);
}

// Tile (rb, c) of B (transposed to K-major): thread r handles column rb*128 + r.
template <int S>
__device__ __forceinline__ void split_cols_tile(const double* __restrict__ B, int64_t K, int64_t N, int64_t ldb,
                                                int64_t NC,
                                                int64_t RB, const unsigned long long* __restrict__ amax,
                                                int8_t* __restrict__ out, int64_t rb, int64_t c, int r,
                                                int half_major = 0) {
  const int64_t col = rb * kTileN + r;
  uint32_t packed[S][8];
#pragma unroll
  for (int p = 0; p < S; ++p)
#pragma unroll
    for (int w = 0; w < 8; ++w) packed[p][w] = 0u;
  if (col < N) {
    const int e = exponent_of_maxbits(amax[col]);
    const int64_t k0 = c * kChunk;
    if constexpr (S <= LT_OZAKI_MAX_SLICES) {
      if (e != kSentinel) {
        const double* bp = B + k0 * ldb + col;
        const bool whole = k0 + kChunk <= K;  // no bounds test per load
        // All 32 loads first (memory-level parallelism), then the digits.
        double v[kChunk];
#pragma unroll
        for (int kk = 0; kk < kChunk; ++kk) v[kk] = (whole || k0 + kk < K) ? __ldg(bp + kk * ldb) : 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) {
          const double q[4] = {v[4 * w], v[4 * w + 1], v[4 * w + 2], v[4 * w + 3]};
          split4<S>(q, e, w, packed);
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < kChunk; ++j) {
        const int64_t k = k0 + j;
        const double v = (k < K) ? __ldg(B + k * ldb + col) : 0.0;
        split_value<S>(v, e, j, packed);
      }
    }
  }
  store_tile_row<S>(out, RB, NC, rb, c, r, packed, half_major);
}

// One block (128 threads) per tile; tiles walked with a grid stride.
template <int S>
__global__ void __launch_bounds__(128) split_rows_kernel(const double* __restrict__ A, int64_t M, int64_t K, int64_t lda,
                                                         int64_t NC, int64_t RB,
                                                         const unsigned long long* __restrict__ amax,
                                                         int8_t* __restrict__ out, int half_major) {
  for (int64_t t = blockIdx.x; t < RB * NC; t += gridDim.x)
    split_rows_tile<S>(A, M, K, lda, NC, RB, amax, out, t / NC, t % NC, threadIdx.x, half_major);
}

template <int S>
__global__ void __launch_bounds__(128) split_cols_kernel(const double* __restrict__ B, int64_t K, int64_t N, int64_t ldb,
                                                         int64_t NC, int64_t RB,
                                                         const unsigned long long* __restrict__ amax,
                                                         int8_t* __restrict__ out, int half_major) {
  for (int64_t t = blockIdx.x; t < RB * NC; t += gridDim.x)
    split_cols_tile<S>(B, K, N, ldb, NC, RB, amax, out, t / NC, t % NC, threadIdx.x, half_major);
}

// Both sides' slices in one launch: blocks 0 .. ga-1 walk A's row tiles (stride ga), the rest B's
// column tiles (stride gb); row pitches K and N.
template <int S>
__global__ void __launch_bounds__(128)
    split_both_kernel(const double* __restrict__ A, int64_t M, const double* __restrict__ B, int64_t N, int64_t K,
                      int64_t NC, int64_t RBa, int64_t RBb, const unsigned long long* __restrict__ amax_a,
                      const unsigned long long* __restrict__ amax_b, int8_t* __restrict__ sa,
                      int8_t* __restrict__ sb, int64_t ga, int64_t gb, int half_major_b) {
  if (blockIdx.x < ga) {
    for (int64_t t = blockIdx.x; t < RBa * NC; t += ga)
      split_rows_tile<S>(A, M, K, K, NC, RBa, amax_a, sa, t / NC, t % NC, threadIdx.x, 0);
  } else {
    for (int64_t t = blockIdx.x - ga; t < RBb * NC; t += gb)
      split_cols_tile<S>(B, K, N, N, NC, RBb, amax_b, sb, t / NC, t % NC, threadIdx.x, half_major_b);
  }
}

// ---------------------------------------------------------------------------------------------
// Product + recombination kernel
// ---------------------------------------------------------------------------------------------
// One problem: its slice tiles, exponents, C and scalars.
struct OzProblem {
  const int8_t* sa;
  const int8_t* sb;
  double* C;
  const unsigned long long* amax_a;
  const unsigned long long* amax_b;
  int64_t M, N, nkc, rba, rbb;
  double alpha, beta;
  int64_t ldc;     // row stride of C (>= N)
  int group = 8;   // pair-rows per raster group of the CTA-pair kernel
  int pair = 0;    // 1: CTA-pair kernel, B slices stored half-major (see store_tile_row)
};

// One row's 64 results (columns col0 .. col0+63 of C, row < M):
// C = fma(alpha, acc 2^(sigma+2) 2^(tau+2), beta C0), NaN where the row's or the column's exponent
// is the non-finite sentinel. C0 is read 8 values at a time (16-byte loads where the row segment
// is 16-byte aligned and whole), all before those values' stores: the stores go through the same
// pointer, so a load written after one could not be moved ahead of it, and every value would wait
// for its own round trip to memory.
__device__ __forceinline__ void store_c_row64(const OzProblem& pr, int64_t row, int64_t col0,
                                              const double (&acc)[64]) {
  const int sig = exponent_of_maxbits(pr.amax_a[row]);
  double* crow = pr.C + row * pr.ldc;
  const int64_t N = pr.N;
  const double alpha = pr.alpha, beta = pr.beta;
  const bool vec = col0 + 64 <= N && (reinterpret_cast<uintptr_t>(crow + col0) & 15) == 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    double c0[8] = {};
    if (beta != 0.0) {
      if (vec) {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const double2 x = *reinterpret_cast<const double2*>(crow + col0 + q * 8 + 2 * v);
          c0[2 * v] = x.x;
          c0[2 * v + 1] = x.y;
        }
      } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int64_t col = col0 + q * 8 + i;
          if (col < N) c0[i] = crow[col];
        }
      }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      double out[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = q * 8 + 2 * v + h;
        const int64_t col = col0 + i;
        const int tau = col < N ? exponent_of_maxbits(pr.amax_b[col]) : 0;
        if (sig == kSentinel || tau == kSentinel) {
          out[h] = __longlong_as_double(0x7ff8000000000000ll);
        } else {
          const double tv = scale_pow2(scale_pow2(acc[i], sig + 2), tau + 2);
          out[h] = (beta != 0.0) ? fma(alpha, tv, __dmul_rn(beta, c0[2 * v + h])) : __dmul_rn(alpha, tv);
        }
      }
      const int64_t col = col0 + q * 8 + 2 * v;
      if (vec) {
        *reinterpret_cast<double2*>(crow + col) = make_double2(out[0], out[1]);
      } else {
        if (col < N) crow[col] = out[0];
        if (col + 1 < N) crow[col + 1] = out[1];
      }
    }
  }
}

// Fetches the 512 bytes of C0 that store_c_row64 will read for (row, col0) into L2, when beta != 0
// and the tile is short (K <= 4096): for longer tiles the lines would leave L2 before the epilogue
// reads them (8192^3: 0.87 GB of extra DRAM reads per launch), and the epilogue already hides
// behind the next tile's first band there.
__device__ __forceinline__ void prefetch_c_row64(const OzProblem& pr, int64_t row, int64_t col0) {
  if (pr.beta == 0.0 || row >= pr.M || pr.nkc > 128) return;
  const double* crow = pr.C + row * pr.ldc;
#pragma unroll
  for (int q = 0; q < 64; q += 16)
    if (col0 + q < pr.N) prefetch_l2(crow + col0 + q);
  if (col0 + 63 < pr.N) prefetch_l2(crow + col0 + 63);
}

// One output tile of one problem.
struct OzJob {
  const OzProblem* pr;
  int m0, n0;
};

struct OzSingleSource {
  const OzProblem* pr;
  int64_t tiles_m, tiles_n;
  __device__ int64_t count() const { return tiles_m * tiles_n; }
  __device__ OzJob get(int64_t t) const {
    const int64_t G = 8;
    int64_t group = t / (G * tiles_n), first_m = group * G;
    int64_t gsize = (tiles_m - first_m) < G ? (tiles_m - first_m) : G;
    int64_t in_group = t - group * G * tiles_n;
    const int64_t tm = first_m + in_group % gsize, tn = in_group / gsize;
    return OzJob{pr, static_cast<int>(tm * kTileM), static_cast<int>(tn * kTileN)};
  }
};

struct OzTile {
  int problem;
  int m0, n0;
  int pad;
};

// Grouped launch: a device table of problems and a tile list sorted by decreasing K on the host.
struct OzGroupedSource {
  const OzProblem* problems;
  const OzTile* tiles;
  int64_t ntiles;
  __device__ int64_t count() const { return ntiles; }
  __device__ OzJob get(int64_t t) const {
    const OzTile ot = tiles[t];
    return OzJob{problems + ot.problem, ot.m0, ot.n0};
  }
};

// Band b of s slices: diagonals dhi = s + 1 - 4b down to dlo; A/B slices 1..nsl are involved.
struct Band {
  int dhi, dlo, nsl, maxp;
};

__host__ __device__ constexpr int pair_lo(int d, int s) { return d - s > 1 ? d - s : 1; }
__host__ __device__ constexpr int pair_hi(int d, int s) { return d - 1 < s ? d - 1 : s; }
__host__ __device__ constexpr int num_bands(int s) { return (s + kBand - 1) / kBand; }
__host__ __device__ constexpr Band band_of(int s, int b) {
  Band B{0, 0, 0, 0};
  B.dhi = s + 1 - kBand * b;
  B.dlo = B.dhi - kBand + 1 < 2 ? 2 : B.dhi - kBand + 1;
  B.nsl = B.dhi - 1 < s ? B.dhi - 1 : s;
  for (int d = B.dhi; d >= B.dlo; --d) {
    const int np = pair_hi(d, s) - pair_lo(d, s) + 1;
    if (np > B.maxp) B.maxp = np;
  }
  return B;
}

// Pipeline geometry for S slices: a stage holds the 2*nsl tiles of one 32-wide K chunk of the
// widest band (nsl = S), narrower bands pack several chunks into a stage.
template <int S>
struct Geo {
  static constexpr int kStageTiles = 2 * S;
  static constexpr int kStageBytes = kStageTiles * kTileBytes;
  static constexpr int kStagesFit = (kMaxSmem - kSmemOverhead) / kStageBytes;
  static constexpr int kStages = kStagesFit > 8 ? 8 : kStagesFit;
  static constexpr int kSmem = kStages * kStageBytes + kSmemOverhead;
  static_assert(kStages >= 2, "slice count too large for the shared-memory ring");
  __host__ __device__ static constexpr int gchunks(int b) { return kKPairLimit / (kChunk * band_of(S, b).maxp); }
  __host__ __device__ static constexpr int cps(int b) { return kStageTiles / (2 * band_of(S, b).nsl); }
};

// Tile descriptors: smem_desc_k_sw32 (lt_common.cuh). The start address (bits 0..13, in 16-byte
// units) of consecutive 4 KB tiles differs by 256, so tile t of a stage is desc(stage) + 256 t.
__device__ __forceinline__ uint64_t desc_k_sw32(uint32_t addr) { return smem_desc_k_sw32(addr); }

// Contiguous global -> shared bulk copy, completion counted in bytes on `bar`.
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gsrc, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(smem_dst)), "l"(reinterpret_cast<uint64_t>(gsrc)), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// All MMAs of band B for one K chunk, unrolled at compile time: diagonal J of the band (d = dhi - J)
// accumulates pairs (PP, d - PP) into TMEM columns J*128 .. +127. A tiles sit at slots 0..nsl-1 of
// the chunk, B tiles at nsl..2nsl-1. The first pair of each diagonal overwrites when `first`.
template <int S, int B, int J, int PP>
__device__ __forceinline__ void issue_pairs(uint64_t a0, uint32_t tmem, uint32_t accumulate_first) {
  constexpr Band bd = band_of(S, B);
  constexpr int d = bd.dhi - J;
  if constexpr (J < kBand && d >= bd.dlo) {
    if constexpr (PP <= pair_hi(d, S)) {
      constexpr uint32_t idesc = idesc_i8_s32(kTileM, kTileN);
      constexpr uint64_t a_off = static_cast<uint64_t>((PP - 1) * (kTileBytes >> 4));
      constexpr uint64_t b_off = static_cast<uint64_t>((bd.nsl + d - PP - 1) * (kTileBytes >> 4));
      mma_i8(tmem + static_cast<uint32_t>(J * kTileN), a0 + a_off, a0 + b_off, idesc,
             PP == pair_lo(d, S) ? accumulate_first : 1u);
      issue_pairs<S, B, J, PP + 1>(a0, tmem, accumulate_first);
    } else {
      issue_pairs<S, B, J + 1, pair_lo(d - 1, S)>(a0, tmem, accumulate_first);
    }
  }
}

template <int S, int B>
__device__ __forceinline__ void issue_chunk(uint64_t a0, uint32_t tmem, uint32_t accumulate_first) {
  if constexpr (B < num_bands(S)) issue_pairs<S, B, 0, pair_lo(band_of(S, B).dhi, S)>(a0, tmem, accumulate_first);
}

template <int S, class Source>
__device__ __forceinline__ void ozaki_body(const Source& src, DeviceStatus* status) {
  using G = Geo<S>;
  constexpr int NB = num_bands(S);
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + G::kStages * G::kStageBytes);
  uint64_t* empty = full + G::kStages;
  uint64_t* acc_full = empty + G::kStages;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* drain = acc_empty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t tiles = src.count();

  if (threadIdx.x == 0) {
    for (int i = 0; i < G::kStages; ++i) {
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
    // ---------------------------------- bulk-copy producer ----------------------------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const OzJob J = src.get(t);
        const OzProblem& pr = *J.pr;
        const int64_t nkc = pr.nkc;
        constexpr int64_t kChunkBlock = static_cast<int64_t>(S) * kTileBytes;  // all slices of one chunk
        const int8_t* a_blk = pr.sa + static_cast<int64_t>(J.m0 / kTileM) * nkc * kChunkBlock;
        const int8_t* b_blk = pr.sb + static_cast<int64_t>(J.n0 / kTileN) * nkc * kChunkBlock;
        for (int b = 0; b < NB && ok; ++b) {
          const Band bd = band_of(S, b);
          const int gch = G::gchunks(b), cps = G::cps(b);
          for (int64_t c0 = 0; c0 < nkc && ok; c0 += gch) {
            const int64_t c1 = (c0 + gch < nkc) ? c0 + gch : nkc;
            for (int64_t cs = c0; cs < c1; cs += cps) {
              const int64_t ce = (cs + cps < c1) ? cs + cps : c1;
              if (!mbar_wait(&empty[stage], phase ^ 1, abort_flag, status, 11)) { ok = false; break; }
              uint8_t* st = smem + stage * G::kStageBytes;
              mbar_arrive_expect_tx(&full[stage], static_cast<uint32_t>((ce - cs) * 2 * bd.nsl * kTileBytes));
              // slices 1..nsl of chunk c: one copy per operand
              for (int64_t c = cs; c < ce; ++c) {
                uint8_t* base = st + (c - cs) * 2 * bd.nsl * kTileBytes;
                bulk_load(base, a_blk + c * kChunkBlock, bd.nsl * kTileBytes, &full[stage]);
                bulk_load(base + bd.nsl * kTileBytes, b_blk + c * kChunkBlock, bd.nsl * kTileBytes, &full[stage]);
              }
              if (++stage == G::kStages) { stage = 0; phase ^= 1; }
            }
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------ MMA issuer ------------------------------------
    // The whole warp runs the loop and one elected lane issues: under elect.sync the per-MMA
    // descriptor arithmetic stays in uniform registers (gated by a plain lane test it does not, and
    // the issue rate drops by a third, measured). Wait results are made warp-uniform. Right after a
    // stage's MMAs are queued the warp peeks at the next stage's barrier while they run, so a stage
    // whose copies have landed is issued without a blocking wait in between.
    {
      const uint64_t desc0 = desc_k_sw32(smem_u32(smem));
      int stage = 0;
      uint32_t phase = 0;
      uint32_t group = 0;
      bool ok = true;
      bool ready = false;  // full[stage] seen complete for `phase` by the last peek
      for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int64_t nkc = src.get(t).pr->nkc;
        for (int b = 0; b < NB && ok; ++b) {
          const Band bd = band_of(S, b);
          const int gch = G::gchunks(b), cps = G::cps(b);
          const uint64_t chunk_step = static_cast<uint64_t>(2 * bd.nsl * (kTileBytes >> 4));
          for (int64_t c0 = 0; c0 < nkc && ok; c0 += gch) {
            const int64_t c1 = (c0 + gch < nkc) ? c0 + gch : nkc;
            if (!__all_sync(0xffffffffu, mbar_wait(acc_empty, (group & 1) ^ 1, abort_flag, status, 12))) {
              ok = false;
              break;
            }
            tc_fence_after();
            for (int64_t cs = c0; cs < c1; cs += cps) {
              const int64_t ce = (cs + cps < c1) ? cs + cps : c1;
              if (!ready && !__all_sync(0xffffffffu, mbar_wait(&full[stage], phase, abort_flag, status, 13))) {
                ok = false;
                break;
              }
              tc_fence_after();
              if (elect_one_sync()) {
                uint64_t a0 = desc0 + static_cast<uint64_t>(stage) * (G::kStageBytes >> 4);
                for (int64_t c = cs; c < ce; ++c, a0 += chunk_step) {
                  const uint32_t acc_first = (c == c0) ? 0u : 1u;
                  switch (b) {
                    case 0: issue_chunk<S, 0>(a0, tmem_base, acc_first); break;
                    case 1: issue_chunk<S, 1>(a0, tmem_base, acc_first); break;
                    default: issue_chunk<S, 2>(a0, tmem_base, acc_first); break;
                  }
                }
                mma_commit(&empty[stage]);
              }
              __syncwarp();
              const int next = stage + 1 == G::kStages ? 0 : stage + 1;
              const uint32_t next_phase = stage + 1 == G::kStages ? phase ^ 1 : phase;
              ready = __all_sync(0xffffffffu, mbar_try_wait(&full[next], next_phase));
              stage = next;
              phase = next_phase;
            }
            if (!ok) break;
            if (elect_one_sync()) mma_commit(acc_full);
            __syncwarp();
            ++group;
          }
        }
      }
      if (!ok && elect_one_sync()) {
        // Let every MMA already issued finish before TMEM is released.
        mma_commit(drain);
        uint64_t t0 = globaltimer();
        while (!mbar_try_wait(drain, 0) && globaltimer() - t0 < LT_WAIT_TIMEOUT_NS) {
        }
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
      const OzJob J = src.get(t);
      const int64_t nkc = J.pr->nkc;
      prefetch_c_row64(*J.pr, J.m0 + row_in_tile, J.n0 + half * 64);
      double acc[64];
#pragma unroll
      for (int i = 0; i < 64; ++i) acc[i] = 0.0;
      for (int b = 0; b < NB && ok; ++b) {
        const Band bd = band_of(S, b);
        const int gch = G::gchunks(b);
        for (int64_t c0 = 0; c0 < nkc; c0 += gch) {
          if (!mbar_wait(acc_full, group & 1, abort_flag, status, 14)) { ok = false; break; }
          tc_fence_after();
          for (int j = 0; j < kBand; ++j) {
            const int d = bd.dhi - j;
            if (d < bd.dlo) break;
            const double sc = pow2i(-8 * d);
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
              uint32_t v[32];
              const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) +
                                     static_cast<uint32_t>(j * kTileN + half * 64 + cc * 32);
              tmem_ld_32x32b_x32(taddr, v);
              tmem_ld_wait();
#pragma unroll
              for (int i = 0; i < 32; ++i)
                acc[cc * 32 + i] =
                    __dadd_rn(acc[cc * 32 + i], __dmul_rn(static_cast<double>(static_cast<int32_t>(v[i])), sc));
            }
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(acc_empty);
          ++group;
        }
      }
      if (!ok) break;
      // ---- C = fma(alpha, acc 2^(sigma+2) 2^(tau+2), beta C0) ----
      const int64_t row = J.m0 + row_in_tile;
      if (row < J.pr->M) store_c_row64(*J.pr, row, J.n0 + half * 64, acc);
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, 512);
  }
}

// 10 warps per CTA put 3 warps on two of the four SM sub-partitions, whose register files hold
// 16K registers each: 168 registers per thread is the most a launch can use.
template <int S>
__global__ void __launch_bounds__(kThreads, 1) ozaki_gemm_kernel(OzProblem pr, DeviceStatus* status) {
  OzSingleSource src{&pr, (pr.M + kTileM - 1) / kTileM, (pr.N + kTileN - 1) / kTileN};
  ozaki_body<S>(src, status);
}

template <int S>
__global__ void __launch_bounds__(kThreads, 1) ozaki_gemm_grouped_kernel(OzGroupedSource src, DeviceStatus* status) {
  ozaki_body<S>(src, status);
}

// ---------------------------------------------------------------------------------------------
// CTA-pair product kernel (single problem with more than one 128-row block). A cluster of two CTAs
// computes a 256 x 128 tile with tcgen05.mma.cta_group::2 (M256 N128 K32): CTA rank r holds row
// block 2i + r of the A slices and rows 64r .. 64r + 63 of the B tile, so each SM's shared memory
// feeds 6 KB of operands per 64-cycle MMA instead of the 8 KB of a one-CTA M128 N128 MMA, which
// is the whole 128 B/clk of the port before the bulk copies are counted. Each CTA's TMEM holds its
// 128 rows of the band's diagonal accumulators and its eight epilogue warps recombine and write
// those rows. The arithmetic of every output element (pairs, K order, FP64 order) is that of
// ozaki_body, so both kernels give bit-identical C.
//
// Synchronisation (barriers at the same shared-memory offsets in both CTAs):
//   full[s]   rank 0: its own expect_tx arrival + one relayed arrival from rank 1 (count 2);
//             rank 1: its own expect_tx arrival (count 1). Rank 1's warp 1 waits on its full[s]
//             and forwards one arrival (relaxed) to rank 0's, so rank 0's MMA sees both halves
//             landed.
//   empty[s]  count 1 in each CTA: rank 0's MMA warp commits to both after the stage's MMAs.
//   acc_full  count 1 in each CTA: committed to both after a group's last MMA.
//   acc_empty rank 0 only, count 16: every epilogue warp of both CTAs arrives after reading TMEM.
// ---------------------------------------------------------------------------------------------
constexpr int kPairChunkBytes = kTileBytes + kHalfTileBytes;  // one slice, one chunk, one CTA

template <int S>
struct PairGeo {
  static constexpr int kStageBytes = S * kPairChunkBytes;
  static constexpr int kStagesFit = (kMaxSmem - kSmemOverhead) / kStageBytes;
  static constexpr int kStages = kStagesFit > 8 ? 8 : kStagesFit;
  static constexpr int kSmem = kStages * kStageBytes + kSmemOverhead;
  static_assert(kStages >= 2, "slice count too large for the shared-memory ring");
  __host__ __device__ static constexpr int cps(int b) { return S / band_of(S, b).nsl; }
};

// Pair tiles in groups of G pair-rows, column-major inside a group.
struct OzPairSource {
  int64_t tiles_m, tiles_n;  // 256-row pair blocks, 128-column blocks
  int64_t G;                 // pair-rows per raster group
  __device__ int64_t count() const { return tiles_m * tiles_n; }
  __device__ void get(int64_t t, int* m0, int* n0) const {
    int64_t group = t / (G * tiles_n), first_m = group * G;
    int64_t gsize = (tiles_m - first_m) < G ? (tiles_m - first_m) : G;
    int64_t in_group = t - group * G * tiles_n;
    *m0 = static_cast<int>((first_m + in_group % gsize) * 2 * kTileM);
    *n0 = static_cast<int>((in_group / gsize) * kTileN);
  }
};

// As issue_pairs, for the pair layout of a chunk: A tiles (4 KB) at slots 0..nsl-1, then the B
// half tiles (2 KB) of slices 1..nsl.
template <int S, int B, int J, int PP>
__device__ __forceinline__ void issue_pairs2(uint64_t a0, uint32_t tmem, uint32_t accumulate_first) {
  constexpr Band bd = band_of(S, B);
  constexpr int d = bd.dhi - J;
  if constexpr (J < kBand && d >= bd.dlo) {
    if constexpr (PP <= pair_hi(d, S)) {
      constexpr uint32_t idesc = idesc_i8_s32(2 * kTileM, kTileN);
      constexpr uint64_t a_off = static_cast<uint64_t>((PP - 1) * (kTileBytes >> 4));
      constexpr uint64_t b_off =
          static_cast<uint64_t>(bd.nsl * (kTileBytes >> 4) + (d - PP - 1) * (kHalfTileBytes >> 4));
      mma_i8_pair(tmem + static_cast<uint32_t>(J * kTileN), a0 + a_off, a0 + b_off, idesc,
                  PP == pair_lo(d, S) ? accumulate_first : 1u);
      issue_pairs2<S, B, J, PP + 1>(a0, tmem, accumulate_first);
    } else {
      issue_pairs2<S, B, J + 1, pair_lo(d - 1, S)>(a0, tmem, accumulate_first);
    }
  }
}

template <int S, int B>
__device__ __forceinline__ void issue_chunk2(uint64_t a0, uint32_t tmem, uint32_t accumulate_first) {
  if constexpr (B < num_bands(S)) issue_pairs2<S, B, 0, pair_lo(band_of(S, B).dhi, S)>(a0, tmem, accumulate_first);
}

template <int S>
__device__ __forceinline__ void ozaki_pair_body(const OzProblem& pr, DeviceStatus* status) {
  using G = PairGeo<S>;
  constexpr int NB = num_bands(S);
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + G::kStages * G::kStageBytes);
  uint64_t* empty = full + G::kStages;
  uint64_t* acc_full = empty + G::kStages;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* drain = acc_empty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const OzPairSource src{(pr.rba + 1) / 2, pr.rbb, pr.group};
  const int64_t tiles = src.count();
  const int64_t first = cluster_id_x(), stride = num_clusters_x();
  const int64_t nkc = pr.nkc;

  if (threadIdx.x == 0) {
    for (int i = 0; i < G::kStages; ++i) {
      mbar_init(&full[i], rank == 0 ? 2 : 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, 2 * kEpilogueWarps);
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc_pair(tmem_slot, 512);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync();  // both CTAs' barriers exist before any arrival crosses the pair
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ------------------------- bulk-copy producer (both CTAs) -------------------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      constexpr int64_t kChunkBlock = static_cast<int64_t>(S) * kTileBytes;  // all slices of one chunk
      for (int64_t t = first; t < tiles && ok; t += stride) {
        int m0, n0;
        src.get(t, &m0, &n0);
        const int64_t rb = m0 / kTileM + rank;  // this CTA's row block; past the end: no A copies
        const bool has_a = rb < pr.rba;
        const int8_t* a_blk = pr.sa + (has_a ? rb : 0) * nkc * kChunkBlock;
        // B slices are half-major (store_tile_row): this CTA's 64-row halves of all slices of a chunk
        // are one contiguous run, S * 2 KB past the chunk block's start for rank 1.
        const int8_t* b_blk = pr.sb + static_cast<int64_t>(n0 / kTileN) * nkc * kChunkBlock + rank * S * kHalfTileBytes;
        const uint32_t chunk_bytes = (has_a ? kTileBytes : 0) + kHalfTileBytes;
        for (int b = 0; b < NB && ok; ++b) {
          const Band bd = band_of(S, b);
          const int gch = Geo<S>::gchunks(b), cps = G::cps(b);
          for (int64_t c0 = 0; c0 < nkc && ok; c0 += gch) {
            const int64_t c1 = (c0 + gch < nkc) ? c0 + gch : nkc;
            for (int64_t cs = c0; cs < c1; cs += cps) {
              const int64_t ce = (cs + cps < c1) ? cs + cps : c1;
              if (!mbar_wait_cluster(&empty[stage], phase ^ 1, abort_flag, status, 21)) { ok = false; break; }
              uint8_t* st = smem + stage * G::kStageBytes;
              mbar_arrive_expect_tx(&full[stage], static_cast<uint32_t>((ce - cs) * bd.nsl) * chunk_bytes);
              for (int64_t c = cs; c < ce; ++c) {
                uint8_t* base = st + (c - cs) * bd.nsl * kPairChunkBytes;
                if (has_a) bulk_load(base, a_blk + c * kChunkBlock, bd.nsl * kTileBytes, &full[stage]);
                // this CTA's halves of the band's B tiles (slices 1..nsl): one copy
                bulk_load(base + bd.nsl * kTileBytes, b_blk + c * kChunkBlock, bd.nsl * kHalfTileBytes, &full[stage]);
              }
              if (++stage == G::kStages) { stage = 0; phase ^= 1; }
            }
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1 && rank != 0) {
    // ------------------- rank 1: forward each landed stage to rank 0 -------------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int64_t t = first; t < tiles && ok; t += stride) {
        for (int b = 0; b < NB && ok; ++b) {
          const int gch = Geo<S>::gchunks(b), cps = G::cps(b);
          for (int64_t c0 = 0; c0 < nkc && ok; c0 += gch) {
            const int64_t c1 = (c0 + gch < nkc) ? c0 + gch : nkc;
            for (int64_t cs = c0; cs < c1; cs += cps) {
              if (!mbar_wait(&full[stage], phase, abort_flag, status, 22)) { ok = false; break; }
              // The copies into this CTA's stage have landed (complete_tx observed above); the
              // forwarded arrival carries no data of this thread, so relaxed ordering suffices.
              mbar_arrive_cluster_relaxed(cluster_addr(&full[stage], 0));
              if (++stage == G::kStages) { stage = 0; phase ^= 1; }
            }
          }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // --------------------------- rank 0: MMA issuer for the pair ---------------------------
    // Warp-convergent loop, one elected lane issues, as in ozaki_body.
    {
      const uint64_t desc0 = smem_desc_k_sw32(smem_u32(smem));
      int stage = 0;
      uint32_t phase = 0;
      uint32_t group = 0;
      bool ok = true;
      bool ready = false;
      for (int64_t t = first; t < tiles && ok; t += stride) {
        for (int b = 0; b < NB && ok; ++b) {
          const Band bd = band_of(S, b);
          const int gch = Geo<S>::gchunks(b), cps = G::cps(b);
          const uint64_t chunk_step = static_cast<uint64_t>(bd.nsl * (kPairChunkBytes >> 4));
          for (int64_t c0 = 0; c0 < nkc && ok; c0 += gch) {
            const int64_t c1 = (c0 + gch < nkc) ? c0 + gch : nkc;
            if (!__all_sync(0xffffffffu, mbar_wait_cluster(acc_empty, (group & 1) ^ 1, abort_flag, status, 23))) {
              ok = false;
              break;
            }
            tc_fence_after();
            for (int64_t cs = c0; cs < c1; cs += cps) {
              const int64_t ce = (cs + cps < c1) ? cs + cps : c1;
              if (!ready &&
                  !__all_sync(0xffffffffu, mbar_wait_cluster(&full[stage], phase, abort_flag, status, 24))) {
                ok = false;
                break;
              }
              tc_fence_after();
              if (elect_one_sync()) {
                uint64_t a0 = desc0 + static_cast<uint64_t>(stage) * (G::kStageBytes >> 4);
                for (int64_t c = cs; c < ce; ++c, a0 += chunk_step) {
                  const uint32_t acc_first = (c == c0) ? 0u : 1u;
                  switch (b) {
                    case 0: issue_chunk2<S, 0>(a0, tmem_base, acc_first); break;
                    case 1: issue_chunk2<S, 1>(a0, tmem_base, acc_first); break;
                    default: issue_chunk2<S, 2>(a0, tmem_base, acc_first); break;
                  }
                }
                mma_commit_pair(cluster_addr(&empty[stage], 0));
                mma_commit_pair(cluster_addr(&empty[stage], 1));
              }
              __syncwarp();
              const int next = stage + 1 == G::kStages ? 0 : stage + 1;
              const uint32_t next_phase = stage + 1 == G::kStages ? phase ^ 1 : phase;
              ready = __all_sync(0xffffffffu, mbar_try_wait_cluster(&full[next], next_phase));
              stage = next;
              phase = next_phase;
            }
            if (!ok) break;
            if (elect_one_sync()) {
              mma_commit_pair(cluster_addr(acc_full, 0));
              mma_commit_pair(cluster_addr(acc_full, 1));
            }
            __syncwarp();
            ++group;
          }
        }
      }
      if (!ok && elect_one_sync()) {
        // Let every MMA already issued finish before TMEM is released.
        mma_commit_pair(cluster_addr(drain, 0));
        uint64_t t0 = globaltimer();
        while (!mbar_try_wait(drain, 0) && globaltimer() - t0 < LT_WAIT_TIMEOUT_NS) {
        }
      }
    }
    __syncwarp();
  } else {
    // ------------------------------- epilogue (8 warps per CTA) -------------------------------
    const int ew = warp - 2;
    const int quarter = warp & 3;  // TMEM lanes 32*quarter .. +31 are visible to this warp
    const int half = ew >> 2;      // columns 64*half .. +63 of the tile
    const int row_in_tile = quarter * 32 + lane;
    const uint32_t acc_empty_r0 = cluster_addr(acc_empty, 0);
    uint32_t group = 0;
    bool ok = true;
    for (int64_t t = first; t < tiles && ok; t += stride) {
      int m0, n0;
      src.get(t, &m0, &n0);
      prefetch_c_row64(pr, m0 + static_cast<int64_t>(rank) * kTileM + row_in_tile, n0 + half * 64);
      double acc[64];
#pragma unroll
      for (int i = 0; i < 64; ++i) acc[i] = 0.0;
      for (int b = 0; b < NB && ok; ++b) {
        const Band bd = band_of(S, b);
        const int gch = Geo<S>::gchunks(b);
        for (int64_t c0 = 0; c0 < nkc; c0 += gch) {
          if (!mbar_wait_cluster(acc_full, group & 1, abort_flag, status, 25)) { ok = false; break; }
          tc_fence_after();
          for (int j = 0; j < kBand; ++j) {
            const int d = bd.dhi - j;
            if (d < bd.dlo) break;
            const double sc = pow2i(-8 * d);
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
              uint32_t v[32];
              const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) +
                                     static_cast<uint32_t>(j * kTileN + half * 64 + cc * 32);
              tmem_ld_32x32b_x32(taddr, v);
              tmem_ld_wait();
#pragma unroll
              for (int i = 0; i < 32; ++i)
                acc[cc * 32 + i] =
                    __dadd_rn(acc[cc * 32 + i], __dmul_rn(static_cast<double>(static_cast<int32_t>(v[i])), sc));
            }
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive_cluster(acc_empty_r0);
          ++group;
        }
      }
      if (!ok) break;
      // ---- C = fma(alpha, acc 2^(sigma+2) 2^(tau+2), beta C0) for this CTA's 128 rows ----
      const int64_t row = m0 + static_cast<int64_t>(rank) * kTileM + row_in_tile;
      if (row < pr.M) store_c_row64(pr, row, n0 + half * 64, acc);
    }
  }

  tc_fence_before();
  __syncthreads();
  cluster_sync();  // rank 0's MMAs read rank 1's shared memory and write its TMEM until here
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, 512);
  }
}

template <int S>
__global__ void __launch_bounds__(kThreads, 1) ozaki_pair_kernel(OzProblem pr, DeviceStatus* status) {
  ozaki_pair_body<S>(pr, status);
}

// Launches the product kernel for S slices over `src` (single problem or grouped tile list).
template <int S, bool kGrouped, class Src>
int launch_gemm_s(const Src& src, int64_t ntiles, DeviceContext* ctx, cudaStream_t stream) {
  using G = Geo<S>;
  static std::once_flag once[64];
  static cudaError_t attr_err[64];
  std::call_once(once[ctx->device], [&] {
    if (kGrouped)
      attr_err[ctx->device] =
          cudaFuncSetAttribute(ozaki_gemm_grouped_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::kSmem);
    else
      attr_err[ctx->device] =
          cudaFuncSetAttribute(ozaki_gemm_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::kSmem);
  });
  LT_CUDA_TRY(attr_err[ctx->device]);
  if (ntiles <= 0) return LT_OK;
  const int64_t grid = ntiles < ctx->sm_count ? ntiles : ctx->sm_count;
  if constexpr (kGrouped)
    ozaki_gemm_grouped_kernel<S><<<static_cast<unsigned>(grid), kThreads, G::kSmem, stream>>>(src, ctx->status);
  else
    ozaki_gemm_kernel<S><<<static_cast<unsigned>(grid), kThreads, G::kSmem, stream>>>(src, ctx->status);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

// Pair-rows per raster group of the CTA-pair kernel: 8, or LIBTHOM_OZAKI_GROUP (1..64).
int pair_group() {
  static const int g = [] {
    const char* e = getenv("LIBTHOM_OZAKI_GROUP");
    const int v = e != nullptr ? atoi(e) : 0;
    return (v >= 1 && v <= 64) ? v : 8;
  }();
  return g;
}

// Launches the CTA-pair product kernel for S slices. *launched = false (nothing launched) when no
// pair of CTAs with this kernel's shared memory fits on the device.
template <int S>
int launch_pair_s(const OzProblem& problem, DeviceContext* ctx, cudaStream_t stream, bool* launched) {
  OzProblem pr = problem;
  pr.group = pair_group();
  using G = PairGeo<S>;
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
        cudaFuncSetAttribute(ozaki_pair_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::kSmem);
    if (attr_err[ctx->device] != cudaSuccess) return;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr;
    config(&cfg, &attr, static_cast<unsigned>(ctx->sm_count & ~1));
    attr_err[ctx->device] = cudaOccupancyMaxActiveClusters(&max_clusters[ctx->device], ozaki_pair_kernel<S>, &cfg);
  });
  LT_CUDA_TRY(attr_err[ctx->device]);
  *launched = false;
  const int64_t tiles = ((pr.rba + 1) / 2) * pr.rbb;
  const int64_t clusters = std::min<int64_t>(std::min<int64_t>(tiles, max_clusters[ctx->device]), ctx->sm_count / 2);
  if (clusters <= 0) return LT_OK;
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute attr;
  config(&cfg, &attr, static_cast<unsigned>(2 * clusters));
  LT_CUDA_TRY(cudaLaunchKernelEx(&cfg, ozaki_pair_kernel<S>, pr, ctx->status));
  *launched = true;
  return LT_OK;
}

int launch_pair(int s, const OzProblem& pr, DeviceContext* ctx, cudaStream_t stream, bool* launched) {
  switch (s) {
#define LT_PAIR_CASE(S) \
  case S: return launch_pair_s<S>(pr, ctx, stream, launched);
    LT_PAIR_CASE(1) LT_PAIR_CASE(2) LT_PAIR_CASE(3) LT_PAIR_CASE(4) LT_PAIR_CASE(5) LT_PAIR_CASE(6)
    LT_PAIR_CASE(7) LT_PAIR_CASE(8) LT_PAIR_CASE(9) LT_PAIR_CASE(10) LT_PAIR_CASE(11) LT_PAIR_CASE(12)
#undef LT_PAIR_CASE
    default: return set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d unsupported", s);
  }
}

// The CTA-pair kernel serves single problems with two or more 128-row blocks unless the
// environment sets LIBTHOM_OZAKI_PAIR=0 (one-CTA kernel everywhere, for comparison).
bool pair_enabled() {
  static const bool on = [] {
    const char* v = getenv("LIBTHOM_OZAKI_PAIR");
    return v == nullptr || v[0] != '0';
  }();
  return on;
}

// Whether a single problem with `rba` row blocks of A runs on the CTA-pair kernel. The split of its
// B side and the product both ask, so the B slices are laid out for the kernel that reads them.
bool pair_path(int64_t rba) { return rba >= 2 && pair_enabled(); }

template <bool kGrouped, class Src>
int launch_gemm(int s, const Src& src, int64_t ntiles, DeviceContext* ctx, cudaStream_t stream) {
  switch (s) {
#define LT_GEMM_CASE(S) \
  case S: return launch_gemm_s<S, kGrouped>(src, ntiles, ctx, stream);
    LT_GEMM_CASE(1) LT_GEMM_CASE(2) LT_GEMM_CASE(3) LT_GEMM_CASE(4) LT_GEMM_CASE(5) LT_GEMM_CASE(6)
    LT_GEMM_CASE(7) LT_GEMM_CASE(8) LT_GEMM_CASE(9) LT_GEMM_CASE(10) LT_GEMM_CASE(11) LT_GEMM_CASE(12)
#undef LT_GEMM_CASE
    default: return set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d unsupported", s);
  }
}

// ---------------------------------------------------------------------------------------------
// Host driver (single problem)
// ---------------------------------------------------------------------------------------------
template <int S>
int launch_split_s(const double* A, const double* B, int64_t M, int64_t N, int64_t K, const Layout& L,
                   const unsigned long long* amax_a, const unsigned long long* amax_b, int8_t* sa, int8_t* sb,
                   int sms, cudaStream_t stream) {
  const int64_t cap = static_cast<int64_t>(sms) * 64;
  const int64_t ta = L.RBa * L.NC, tb = L.RBb * L.NC;
  if (ta > 0) split_rows_kernel<S><<<static_cast<unsigned>(ta < cap ? ta : cap), 128, 0, stream>>>(A, M, K, K, L.NC, L.RBa,
                                                                                                   amax_a, sa, 0);
  LT_CUDA_TRY(cudaGetLastError());
  if (tb > 0) split_cols_kernel<S><<<static_cast<unsigned>(tb < cap ? tb : cap), 128, 0, stream>>>(B, K, N, N, L.NC, L.RBb,
                                                                                                   amax_b, sb, 0);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

int launch_split(int s, const double* A, const double* B, int64_t M, int64_t N, int64_t K, const Layout& L,
                 const unsigned long long* amax_a, const unsigned long long* amax_b, int8_t* sa, int8_t* sb, int sms,
                 cudaStream_t stream) {
  switch (s) {
#define LT_SPLIT_CASE(S) \
  case S: return launch_split_s<S>(A, B, M, N, K, L, amax_a, amax_b, sa, sb, sms, stream);
    LT_SPLIT_CASE(1) LT_SPLIT_CASE(2) LT_SPLIT_CASE(3) LT_SPLIT_CASE(4) LT_SPLIT_CASE(5) LT_SPLIT_CASE(6)
    LT_SPLIT_CASE(7) LT_SPLIT_CASE(8) LT_SPLIT_CASE(9) LT_SPLIT_CASE(10) LT_SPLIT_CASE(11) LT_SPLIT_CASE(12)
#undef LT_SPLIT_CASE
    default: return set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d unsupported", s);
  }
}

template <int S>
void launch_split_rows_s(const double* A, int64_t M, int64_t K, int64_t lda, int64_t NC, const unsigned long long* amax,
                         int8_t* sa, int sms, cudaStream_t stream, int half_major) {
  const int64_t cap = static_cast<int64_t>(sms) * 64;
  const int64_t rb = ceil_div(M, kTileM), t = rb * NC;
  if (t > 0)
    split_rows_kernel<S><<<static_cast<unsigned>(t < cap ? t : cap), 128, 0, stream>>>(A, M, K, lda, NC, rb, amax, sa,
                                                                                       half_major);
}

template <int S>
void launch_split_cols_s(const double* B, int64_t K, int64_t N, int64_t ldb, int64_t NC, const unsigned long long* amax,
                         int8_t* sb, int sms, cudaStream_t stream, int half_major) {
  const int64_t cap = static_cast<int64_t>(sms) * 64;
  const int64_t rb = ceil_div(N, kTileN), t = rb * NC;
  if (t > 0)
    split_cols_kernel<S><<<static_cast<unsigned>(t < cap ? t : cap), 128, 0, stream>>>(B, K, N, ldb, NC, rb, amax, sb,
                                                                                       half_major);
}

// Row side of the split: exponents of rows 0..M-1 of A (amax must be zero on entry) and their
// slices, written as row blocks 0.. of `sa` (chunk-major, NC chunks; half_major for B slices that
// the CTA-pair kernel reads, see store_tile_row).
// Row maxima of A (M x K, row stride lda) as IEEE bits into amax (zero on entry); M, K > 0.
int exponents_rows(const double* A, int64_t M, int64_t K, int64_t lda, unsigned long long* amax, int sms,
                   cudaStream_t stream) {
  // 8 rows per block, K split so that the grid covers the GPU.
  int64_t row_blocks = (M + 7) / 8;
  int64_t ksplit = (4 * sms + row_blocks - 1) / row_blocks;
  ksplit = ksplit < 1 ? 1 : ksplit;
  int64_t kseg = round_up((K + ksplit - 1) / ksplit, 256);
  ksplit = (K + kseg - 1) / kseg;
  amax_rows_kernel<<<dim3(static_cast<unsigned>(row_blocks), static_cast<unsigned>(ksplit)), 256, 0, stream>>>(
      A, M, K, lda, kseg, amax);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

// Column maxima of B (K x N, row stride ldb) as IEEE bits into amax (zero on entry); N, K > 0.
int exponents_cols(const double* B, int64_t K, int64_t N, int64_t ldb, unsigned long long* amax, int sms,
                   cudaStream_t stream) {
  const int pairs = (N % 2 == 0) && (ldb % 2 == 0) && ((reinterpret_cast<uintptr_t>(B) & 15) == 0);
  const int64_t per_block = pairs ? 512 : 256;
  int64_t col_blocks = (N + per_block - 1) / per_block;
  int64_t ksplit_b = (8 * sms + col_blocks - 1) / col_blocks;
  ksplit_b = ksplit_b < 1 ? 1 : ksplit_b;
  int64_t kseg_b = (K + ksplit_b - 1) / ksplit_b;
  ksplit_b = (K + kseg_b - 1) / kseg_b;
  amax_cols_kernel<<<dim3(static_cast<unsigned>(col_blocks), static_cast<unsigned>(ksplit_b)), 256, 0, stream>>>(
      B, K, N, ldb, kseg_b, amax, pairs);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

int rows_stage(int s, const double* A, int64_t M, int64_t K, int64_t lda, int64_t NC, unsigned long long* amax,
               int8_t* sa, int sms, cudaStream_t stream, int half_major) {
  if (M <= 0) return LT_OK;
  if (K > 0) LT_TRY(exponents_rows(A, M, K, lda, amax, sms, stream));
  switch (s) {
#define LT_ROWS_CASE(S) \
  case S: launch_split_rows_s<S>(A, M, K, lda, NC, amax, sa, sms, stream, half_major); break;
    LT_ROWS_CASE(1) LT_ROWS_CASE(2) LT_ROWS_CASE(3) LT_ROWS_CASE(4) LT_ROWS_CASE(5) LT_ROWS_CASE(6)
    LT_ROWS_CASE(7) LT_ROWS_CASE(8) LT_ROWS_CASE(9) LT_ROWS_CASE(10) LT_ROWS_CASE(11) LT_ROWS_CASE(12)
#undef LT_ROWS_CASE
    default: return set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d unsupported", s);
  }
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

// Column side: exponents of columns 0..N-1 of B (amax zero on entry) and their slices.
int cols_stage(int s, const double* B, int64_t K, int64_t N, int64_t ldb, int64_t NC, unsigned long long* amax,
               int8_t* sb, int sms, cudaStream_t stream, int half_major) {
  if (N <= 0) return LT_OK;
  if (K > 0) LT_TRY(exponents_cols(B, K, N, ldb, amax, sms, stream));
  switch (s) {
#define LT_COLS_CASE(S) \
  case S: launch_split_cols_s<S>(B, K, N, ldb, NC, amax, sb, sms, stream, half_major); break;
    LT_COLS_CASE(1) LT_COLS_CASE(2) LT_COLS_CASE(3) LT_COLS_CASE(4) LT_COLS_CASE(5) LT_COLS_CASE(6)
    LT_COLS_CASE(7) LT_COLS_CASE(8) LT_COLS_CASE(9) LT_COLS_CASE(10) LT_COLS_CASE(11) LT_COLS_CASE(12)
#undef LT_COLS_CASE
    default: return set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d unsupported", s);
  }
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

// Both sides of the split in two launches (exponents, then slices), each launch's blocks divided
// between A's rows and B's columns: the same blocks and results as rows_stage + cols_stage with
// row pitches K and N, with two kernel boundaries fewer. M, N, K > 0; amax zero on entry.
template <int S>
void launch_split_both_s(const double* A, const double* B, int64_t M, int64_t N, int64_t K, const Layout& L,
                         const unsigned long long* amax_a, const unsigned long long* amax_b, int8_t* sa, int8_t* sb,
                         int sms, cudaStream_t stream, int half_major_b) {
  const int64_t cap = static_cast<int64_t>(sms) * 64;
  const int64_t ta = L.RBa * L.NC, tb = L.RBb * L.NC;
  const int64_t ga = ta < cap ? ta : cap, gb = tb < cap ? tb : cap;
  split_both_kernel<S><<<static_cast<unsigned>(ga + gb), 128, 0, stream>>>(A, M, B, N, K, L.NC, L.RBa, L.RBb, amax_a,
                                                                           amax_b, sa, sb, ga, gb, half_major_b);
}

// Row maxima of A and column maxima of B (row pitches K and N) in one launch, the blocks rows_stage
// and cols_stage would launch; M, N, K > 0, amax zero on entry. Shared with the CRT form.
int exponents(const double* A, const double* B, int64_t M, int64_t N, int64_t K, unsigned long long* amax_a,
              unsigned long long* amax_b, int sms, cudaStream_t stream) {
  const int64_t ra = (M + 7) / 8;
  int64_t ka = (4 * sms + ra - 1) / ra;
  ka = ka < 1 ? 1 : ka;
  const int64_t kseg_a = round_up((K + ka - 1) / ka, 256);
  ka = (K + kseg_a - 1) / kseg_a;
  const int pairs = (N % 2 == 0) && ((reinterpret_cast<uintptr_t>(B) & 15) == 0);
  const int64_t per_block = pairs ? 512 : 256;
  const int64_t rb = (N + per_block - 1) / per_block;
  int64_t kb = (8 * sms + rb - 1) / rb;
  kb = kb < 1 ? 1 : kb;
  const int64_t kseg_b = (K + kb - 1) / kb;
  kb = (K + kseg_b - 1) / kseg_b;
  amax_both_kernel<<<static_cast<unsigned>(ra * ka + rb * kb), 256, 0, stream>>>(A, M, K, kseg_a, ra, ka, amax_a, B, N,
                                                                                  kseg_b, rb, pairs, amax_b);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

int both_stage(int s, const double* A, const double* B, int64_t M, int64_t N, int64_t K, const Layout& L,
               unsigned long long* amax_a, unsigned long long* amax_b, int8_t* sa, int8_t* sb, int sms,
               cudaStream_t stream, int half_major_b) {
  LT_TRY(exponents(A, B, M, N, K, amax_a, amax_b, sms, stream));
  switch (s) {
#define LT_BOTH_CASE(S) \
  case S: launch_split_both_s<S>(A, B, M, N, K, L, amax_a, amax_b, sa, sb, sms, stream, half_major_b); break;
    LT_BOTH_CASE(1) LT_BOTH_CASE(2) LT_BOTH_CASE(3) LT_BOTH_CASE(4) LT_BOTH_CASE(5) LT_BOTH_CASE(6)
    LT_BOTH_CASE(7) LT_BOTH_CASE(8) LT_BOTH_CASE(9) LT_BOTH_CASE(10) LT_BOTH_CASE(11) LT_BOTH_CASE(12)
#undef LT_BOTH_CASE
    default: return set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d unsupported", s);
  }
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

// Stage 1+2 on a given device description (see split).
int split_on(const DeviceContext* ctx, const double* A, const double* B, int64_t M, int64_t N, int64_t K, int s,
             void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  const Layout L = layout_for(M, N, K, s);
  if (workspace_bytes < L.total) return set_error(LT_ERR_NO_MEMORY, "Ozaki workspace too small");
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  auto* amax_a = reinterpret_cast<unsigned long long*>(ws + L.off_amax_a);
  auto* amax_b = reinterpret_cast<unsigned long long*>(ws + L.off_amax_b);
  auto* sa = reinterpret_cast<int8_t*>(ws + L.off_sa);
  auto* sb = reinterpret_cast<int8_t*>(ws + L.off_sb);
  LT_CUDA_TRY(cudaMemsetAsync(ws, 0, L.off_sa, stream));
  if (M > 0 && N > 0 && K > 0)
    return both_stage(s, A, B, M, N, K, L, amax_a, amax_b, sa, sb, ctx->sm_count, stream, pair_path(L.RBa) ? 1 : 0);
  LT_TRY(rows_stage(s, A, M, K, K, L.NC, amax_a, sa, ctx->sm_count, stream, 0));
  return cols_stage(s, B, K, N, N, L.NC, amax_b, sb, ctx->sm_count, stream, pair_path(L.RBa) ? 1 : 0);
}

// Stage 1+2: exponents and slices of A and B into the workspace.
int split(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int s, void* workspace,
          size_t workspace_bytes, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  return split_on(ctx, A, B, M, N, K, s, workspace, workspace_bytes, stream);
}

// Products and recombination of one problem whose slices are in place: the CTA-pair kernel when
// pr.pair is set (B slices split half-major), the one-CTA kernel otherwise.
int launch_product(int s, const OzProblem& pr, DeviceContext* ctx, cudaStream_t stream) {
  if (pr.pair) {
    bool launched = false;
    LT_TRY(launch_pair(s, pr, ctx, stream, &launched));
    if (!launched) return set_error(LT_ERR_UNSUPPORTED, "no pair of CTAs of the Ozaki product kernel fits");
    return LT_OK;
  }
  return launch_gemm<false>(s, pr, pr.rba * pr.rbb, ctx, stream);
}

// Stage 3+4 on a given device description (see product).
int product_on(DeviceContext* ctx, double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int s,
               const void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  const Layout L = layout_for(M, N, K, s);
  if (workspace_bytes < L.total) return set_error(LT_ERR_NO_MEMORY, "Ozaki workspace too small");
  const uint8_t* ws = static_cast<const uint8_t*>(workspace);
  OzProblem pr;
  pr.sa = reinterpret_cast<const int8_t*>(ws + L.off_sa);
  pr.sb = reinterpret_cast<const int8_t*>(ws + L.off_sb);
  pr.C = C;
  pr.amax_a = reinterpret_cast<const unsigned long long*>(ws + L.off_amax_a);
  pr.amax_b = reinterpret_cast<const unsigned long long*>(ws + L.off_amax_b);
  pr.M = M;
  pr.N = N;
  pr.ldc = N;
  pr.nkc = L.NC;
  pr.rba = L.RBa;
  pr.rbb = L.RBb;
  pr.alpha = alpha;
  pr.beta = beta;
  pr.pair = pair_path(L.RBa) ? 1 : 0;
  return launch_product(s, pr, ctx, stream);
}

// Stage 3+4: slice products on the tensor cores and the fused FP64 recombination into C.
int product(double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int s, const void* workspace,
            size_t workspace_bytes, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  return product_on(ctx, C, M, N, K, alpha, beta, s, workspace, workspace_bytes, stream);
}

// Row strides and transposes (lt_dgemm_ex): op(A) = A (M x K, row stride lda) or A^T (A stored
// K x M, row stride lda), op(B) = B (K x N, ldb) or B^T (B stored N x K, ldb), C is M x N with row
// stride ldc. A transposed operand goes through the other side's kernels: the rows of op(A) = A^T
// are the columns of the stored A, which amax_cols / split_cols read, writing the same tiles the row
// kernels write (tile row = row of op(A)); op(B) = B^T goes through amax_rows / split_rows. Every
// digit and every output element is the one run() computes on packed op(A) and op(B), so results are
// bit-identical to it.
int run_ex(bool trans_a, bool trans_b, const double* A, int64_t lda, const double* B, int64_t ldb, double* C, int64_t ldc,
           int64_t M, int64_t N, int64_t K, double alpha, double beta, int s, void* workspace, size_t workspace_bytes,
           cudaStream_t stream) {
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
  const int pair = pair_path(L.RBa) ? 1 : 0;
  if (!trans_a)
    LT_TRY(rows_stage(s, A, M, K, lda, L.NC, amax_a, sa, sms, stream, 0));
  else
    LT_TRY(cols_stage(s, A, K, M, lda, L.NC, amax_a, sa, sms, stream, 0));
  if (!trans_b)
    LT_TRY(cols_stage(s, B, K, N, ldb, L.NC, amax_b, sb, sms, stream, pair));
  else
    LT_TRY(rows_stage(s, B, N, K, ldb, L.NC, amax_b, sb, sms, stream, pair));
  OzProblem pr{sa, sb, C, amax_a, amax_b, M, N, L.NC, L.RBa, L.RBb, alpha, beta, ldc};
  pr.pair = pair;
  return launch_product(s, pr, ctx, stream);
}

int run(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int s,
        void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  LT_TRY(split(A, B, M, N, K, s, workspace, workspace_bytes, stream));
  return product(C, M, N, K, alpha, beta, s, workspace, workspace_bytes, stream);
}

// ---------------------------------------------------------------------------------------------
// Host-resident operands (lt_dgemm_ozaki_host). B is copied and split first; then row panels of
// A (and of C0 when beta != 0) are copied on one stream while the previous panel is split and
// multiplied on the caller's stream and finished panels of C return on a third, so the PCIe
// copies overlap the kernels. A panel is a block of whole 128-row blocks; its slices land in the
// same place of the workspace as in run(), and every output element goes through the same
// arithmetic, so C is bit-identical to run() on the same data.
// ---------------------------------------------------------------------------------------------
// Row panels of the host-resident pipeline: 16, or LIBTHOM_OZAKI_HOST_PANELS (1..64). The step is
// bound by the host-to-device copies (A, B and C0 at about 55 GB/s); more panels shorten the tail
// (the last panel's product and copy back) that follows the last copy in. Measured at 8192^3,
// s = 7: 4 / 8 / 16 / 32 panels take 35.5 / 33.7 / 33.0 / 33.2 ms against a copy-in floor of 29.0 ms.
int host_panels() {
  static const int n = [] {
    const char* e = getenv("LIBTHOM_OZAKI_HOST_PANELS");
    const int v = e != nullptr ? atoi(e) : 0;
    return (v >= 1 && v <= 64) ? v : 16;
  }();
  return n;
}

int host_run(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
             double beta, int s, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  const Layout L = layout_for(M, N, K, s);
  const size_t off_a = round_up(static_cast<int64_t>(L.total), 256);
  const size_t off_b = off_a + round_up(8 * M * K, 256);
  const size_t off_c = off_b + round_up(8 * K * N, 256);
  const size_t total = off_c + 8 * static_cast<size_t>(M) * N;
  void* base = nullptr;
  LT_TRY(ensure_workspace(ctx, total, &base));
  uint8_t* ws = static_cast<uint8_t*>(base);
  auto* amax_a = reinterpret_cast<unsigned long long*>(ws + L.off_amax_a);
  auto* amax_b = reinterpret_cast<unsigned long long*>(ws + L.off_amax_b);
  auto* sa = reinterpret_cast<int8_t*>(ws + L.off_sa);
  auto* sb = reinterpret_cast<int8_t*>(ws + L.off_sb);
  auto* Ad = reinterpret_cast<double*>(ws + off_a);
  auto* Bd = reinterpret_cast<double*>(ws + off_b);
  auto* Cd = reinterpret_cast<double*>(ws + off_c);

  // About `host_panels()` panels (at least one 128-row block each).
  const int64_t panel = std::max<int64_t>(kTileM, round_up(ceil_div(M, host_panels()), kTileM));
  const int64_t npanels = ceil_div(M, panel);
  const int64_t chunk_block = static_cast<int64_t>(s) * kTileBytes;

  cudaStream_t h2d = nullptr, d2h = nullptr;
  std::vector<cudaEvent_t> ev(2 * npanels + 2, nullptr);
  int rc = LT_OK;
  auto cuda = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == LT_OK) rc = set_error(LT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return rc == LT_OK;
  };
  cuda(cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking), "stream");
  cuda(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking), "stream");
  for (auto& e : ev)
    if (rc == LT_OK) cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  cudaEvent_t e_start = ev[2 * npanels], e_b = ev[2 * npanels + 1];
  if (rc == LT_OK) {
    // Everything starts after the work already queued on the caller's stream.
    cuda(cudaEventRecord(e_start, stream), "record");
    cuda(cudaStreamWaitEvent(h2d, e_start, 0), "wait");
    cuda(cudaStreamWaitEvent(d2h, e_start, 0), "wait");
    cuda(cudaMemcpyAsync(Bd, B, 8 * static_cast<size_t>(K) * N, cudaMemcpyHostToDevice, h2d), "copy B");
    cuda(cudaEventRecord(e_b, h2d), "record");
    cuda(cudaMemsetAsync(ws, 0, L.off_sa, stream), "memset");
    cuda(cudaStreamWaitEvent(stream, e_b, 0), "wait");
  }
  // Every panel's product takes the same kernel (the pair kernel also serves a last panel of one
  // row block), so the B slices are split once in its layout.
  const int pair = pair_path(ceil_div(panel, kTileM)) ? 1 : 0;
  if (rc == LT_OK) rc = cols_stage(s, Bd, K, N, N, L.NC, amax_b, sb, ctx->sm_count, stream, pair);
  for (int64_t i = 0; i < npanels && rc == LT_OK; ++i) {
    const int64_t r0 = i * panel, rows = std::min(panel, M - r0);
    cudaEvent_t e_in = ev[2 * i], e_out = ev[2 * i + 1];
    cuda(cudaMemcpyAsync(Ad + r0 * K, A + r0 * K, 8 * static_cast<size_t>(rows) * K, cudaMemcpyHostToDevice, h2d),
         "copy A");
    if (beta != 0.0)
      cuda(cudaMemcpyAsync(Cd + r0 * N, C + r0 * N, 8 * static_cast<size_t>(rows) * N, cudaMemcpyHostToDevice, h2d),
           "copy C0");
    cuda(cudaEventRecord(e_in, h2d), "record");
    cuda(cudaStreamWaitEvent(stream, e_in, 0), "wait");
    if (rc != LT_OK) break;
    int8_t* sa_panel = sa + (r0 / kTileM) * L.NC * chunk_block;
    rc = rows_stage(s, Ad + r0 * K, rows, K, K, L.NC, amax_a + r0, sa_panel, ctx->sm_count, stream, 0);
    if (rc != LT_OK) break;
    OzProblem pr{sa_panel, sb, Cd + r0 * N, amax_a + r0, amax_b, rows, N, L.NC, ceil_div(rows, kTileM), L.RBb,
                 alpha, beta, N};
    pr.pair = pair;
    rc = launch_product(s, pr, ctx, stream);
    if (rc != LT_OK) break;
    cuda(cudaEventRecord(e_out, stream), "record");
    cuda(cudaStreamWaitEvent(d2h, e_out, 0), "wait");
    cuda(cudaMemcpyAsync(C + r0 * N, Cd + r0 * N, 8 * static_cast<size_t>(rows) * N, cudaMemcpyDeviceToHost, d2h),
         "copy C");
  }
  // The caller's stream is ordered after the last copy back; the call returns with C in host memory.
  if (rc == LT_OK) cuda(cudaEventRecord(e_start, d2h), "record");
  if (rc == LT_OK) cuda(cudaStreamWaitEvent(stream, e_start, 0), "wait");
  if (d2h != nullptr) cuda(cudaStreamSynchronize(d2h), "sync");
  if (h2d != nullptr) cuda(cudaStreamSynchronize(h2d), "sync");
  cuda(cudaStreamSynchronize(stream), "sync");
  for (auto& e : ev)
    if (e != nullptr) cudaEventDestroy(e);
  if (h2d != nullptr) cudaStreamDestroy(h2d);
  if (d2h != nullptr) cudaStreamDestroy(d2h);
  return rc;
}

// ---------------------------------------------------------------------------------------------
// Grouped form: many independent problems, one launch per stage.
// Workspace: [amax of every problem (one contiguous region, zeroed by one memset)]
//            [per problem: A tiles | B tiles].
// Block tables map blockIdx.x to (problem, local block) through prefix sums searched on device.
// ---------------------------------------------------------------------------------------------
struct GSplit {
  const double* A;
  const double* B;
  int64_t M, N, K, NC, RBa, RBb;
  unsigned long long* amax_a;
  unsigned long long* amax_b;
  int8_t* sa;
  int8_t* sb;
};

__device__ __forceinline__ int find_problem(const int* off, int count, int b) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// 8 rows (one warp each) per block.
__global__ void g_amax_rows_kernel(const GSplit* __restrict__ P, const int* __restrict__ off, int count) {
  const int pi = find_problem(off, count, blockIdx.x);
  const GSplit g = P[pi];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = static_cast<int64_t>(blockIdx.x - off[pi]) * 8 + warp;
  if (row >= g.M) return;
  unsigned long long m = 0;
  for (int64_t k = lane; k < g.K; k += 32) {
    unsigned long long b = abs_bits(__ldg(g.A + row * g.K + k));
    m = b > m ? b : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long x = __shfl_xor_sync(0xffffffffu, m, o);
    m = x > m ? x : m;
  }
  if (lane == 0) g.amax_a[row] = m;
}

// 256 columns (one per thread) per block.
__global__ void g_amax_cols_kernel(const GSplit* __restrict__ P, const int* __restrict__ off, int count) {
  const int pi = find_problem(off, count, blockIdx.x);
  const GSplit g = P[pi];
  const int64_t col = static_cast<int64_t>(blockIdx.x - off[pi]) * 256 + threadIdx.x;
  if (col >= g.N) return;
  unsigned long long m = 0;
  for (int64_t k = 0; k < g.K; ++k) {
    unsigned long long b = abs_bits(__ldg(g.B + k * g.N + col));
    m = b > m ? b : m;
  }
  g.amax_b[col] = m;
}

// One block (128 threads) per slice tile.
template <int S>
__global__ void __launch_bounds__(128) g_split_rows_kernel(const GSplit* __restrict__ P, const int* __restrict__ off,
                                                           int count) {
  const int pi = find_problem(off, count, blockIdx.x);
  const GSplit& g = P[pi];
  const int64_t t = blockIdx.x - off[pi];
  split_rows_tile<S>(g.A, g.M, g.K, g.K, g.NC, g.RBa, g.amax_a, g.sa, t / g.NC, t % g.NC, threadIdx.x);
}

template <int S>
__global__ void __launch_bounds__(128) g_split_cols_kernel(const GSplit* __restrict__ P, const int* __restrict__ off,
                                                           int count) {
  const int pi = find_problem(off, count, blockIdx.x);
  const GSplit& g = P[pi];
  const int64_t t = blockIdx.x - off[pi];
  split_cols_tile<S>(g.B, g.K, g.N, g.N, g.NC, g.RBb, g.amax_b, g.sb, t / g.NC, t % g.NC, threadIdx.x);
}

struct Grouped {
  int count = 0, s = 0;
  void* dev = nullptr;   // tables (one allocation)
  void* ws = nullptr;    // amax + slice tiles
  size_t amax_bytes = 0;
  GSplit* d_split = nullptr;
  int* d_off = nullptr;  // 4 x (count + 1): amax rows, amax cols, split rows, split cols
  int blocks[4] = {0, 0, 0, 0};
  OzProblem* d_problems = nullptr;
  OzTile* d_tiles = nullptr;
  int64_t ntiles = 0;
};

template <int S>
int g_split_launch(const Grouped& G, cudaStream_t stream) {
  const int n = G.count;
  if (G.blocks[2] > 0) g_split_rows_kernel<S><<<G.blocks[2], 128, 0, stream>>>(G.d_split, G.d_off + 2 * (n + 1), n);
  if (G.blocks[3] > 0) g_split_cols_kernel<S><<<G.blocks[3], 128, 0, stream>>>(G.d_split, G.d_off + 3 * (n + 1), n);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

int grouped_create(const lt_gemm_problem* problems, int count, int s, Grouped** out) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  std::vector<Layout> lay(count);
  std::vector<size_t> off_aa(count), off_ab(count), off_sa(count), off_sb(count);
  size_t o = 0;
  for (int i = 0; i < count; ++i) {
    lay[i] = layout_for(problems[i].M, problems[i].N, problems[i].K, s);
    off_aa[i] = o; o += round_up(8 * problems[i].M, 256);
    off_ab[i] = o; o += round_up(8 * problems[i].N, 256);
  }
  const size_t amax_bytes = o;
  for (int i = 0; i < count; ++i) {
    off_sa[i] = o; o += static_cast<size_t>(s) * lay[i].RBa * lay[i].NC * kTileBytes;
    off_sb[i] = o; o += static_cast<size_t>(s) * lay[i].RBb * lay[i].NC * kTileBytes;
  }
  // block counts must fit the int prefix tables
  int64_t tot[4] = {0, 0, 0, 0};
  for (int i = 0; i < count; ++i) {
    const lt_gemm_problem& p = problems[i];
    tot[0] += p.K > 0 ? (p.M + 7) / 8 : 0;
    tot[1] += p.K > 0 ? (p.N + 255) / 256 : 0;
    tot[2] += lay[i].RBa * lay[i].NC;
    tot[3] += lay[i].RBb * lay[i].NC;
  }
  for (int k = 0; k < 4; ++k)
    if (tot[k] > 0x7fffffff) return set_error(LT_ERR_INVALID_ARGUMENT, "grouped problem set too large");
  auto* G = new Grouped();
  G->count = count;
  G->s = s;
  G->amax_bytes = amax_bytes;
  cudaError_t e = cudaMalloc(&G->ws, o > 0 ? o : 256);
  if (e != cudaSuccess) {
    delete G;
    return set_error(LT_ERR_NO_MEMORY, "grouped Ozaki workspace (%zu bytes): %s", o, cudaGetErrorString(e));
  }
  uint8_t* ws = static_cast<uint8_t*>(G->ws);
  std::vector<GSplit> split(count);
  std::vector<int> offs(4 * (count + 1), 0);
  std::vector<OzProblem> probs(count);
  for (int i = 0; i < count; ++i) {
    const lt_gemm_problem& p = problems[i];
    const Layout& L = lay[i];
    GSplit& g = split[i];
    g = GSplit{p.A, p.B, p.M, p.N, p.K, L.NC, L.RBa, L.RBb,
               reinterpret_cast<unsigned long long*>(ws + off_aa[i]), reinterpret_cast<unsigned long long*>(ws + off_ab[i]),
               reinterpret_cast<int8_t*>(ws + off_sa[i]), reinterpret_cast<int8_t*>(ws + off_sb[i])};
    const int64_t nb[4] = {p.K > 0 ? (p.M + 7) / 8 : 0, p.K > 0 ? (p.N + 255) / 256 : 0, L.RBa * L.NC, L.RBb * L.NC};
    for (int k = 0; k < 4; ++k) offs[k * (count + 1) + i + 1] = offs[k * (count + 1) + i] + static_cast<int>(nb[k]);
    probs[i] = OzProblem{g.sa, g.sb, p.C, g.amax_a, g.amax_b, p.M, p.N, L.NC, L.RBa, L.RBb, p.alpha, p.beta, p.N};
    G->ntiles += L.RBa * L.RBb;
  }
  for (int k = 0; k < 4; ++k) G->blocks[k] = offs[k * (count + 1) + count];
  // tiles of the longest-K problems first (a tile's cost is proportional to its problem's NC)
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return lay[a].NC > lay[b].NC; });
  std::vector<OzTile> tiles;
  tiles.reserve(static_cast<size_t>(G->ntiles));
  for (int i : order)
    for (int64_t a = 0; a < lay[i].RBa; ++a)
      for (int64_t b = 0; b < lay[i].RBb; ++b)
        tiles.push_back(OzTile{i, static_cast<int>(a * kTileM), static_cast<int>(b * kTileN), 0});
  const size_t split_bytes = round_up(sizeof(GSplit) * count, 256);
  const size_t offs_bytes = round_up(sizeof(int) * offs.size(), 256);
  const size_t prob_bytes = round_up(sizeof(OzProblem) * count, 256);
  const size_t tile_bytes = round_up(sizeof(OzTile) * (tiles.size() + 1), 256);
  e = cudaMalloc(&G->dev, split_bytes + offs_bytes + prob_bytes + tile_bytes);
  if (e == cudaSuccess) {
    uint8_t* d = static_cast<uint8_t*>(G->dev);
    G->d_split = reinterpret_cast<GSplit*>(d);
    G->d_off = reinterpret_cast<int*>(d + split_bytes);
    G->d_problems = reinterpret_cast<OzProblem*>(d + split_bytes + offs_bytes);
    G->d_tiles = reinterpret_cast<OzTile*>(d + split_bytes + offs_bytes + prob_bytes);
    e = cudaMemcpy(G->d_split, split.data(), sizeof(GSplit) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(G->d_off, offs.data(), sizeof(int) * offs.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(G->d_problems, probs.data(), sizeof(OzProblem) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !tiles.empty())
      e = cudaMemcpy(G->d_tiles, tiles.data(), sizeof(OzTile) * tiles.size(), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaFree(G->dev);
    cudaFree(G->ws);
    delete G;
    return set_error(LT_ERR_NO_MEMORY, "grouped tables: %s", cudaGetErrorString(e));
  }
  *out = G;
  return LT_OK;
}

int grouped_run(const Grouped* G, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  const int n = G->count;
  LT_CUDA_TRY(cudaMemsetAsync(G->ws, 0, G->amax_bytes, stream));
  if (G->blocks[0] > 0) g_amax_rows_kernel<<<G->blocks[0], 256, 0, stream>>>(G->d_split, G->d_off, n);
  if (G->blocks[1] > 0) g_amax_cols_kernel<<<G->blocks[1], 256, 0, stream>>>(G->d_split, G->d_off + (n + 1), n);
  LT_CUDA_TRY(cudaGetLastError());
  switch (G->s) {
#define LT_GSPLIT_CASE(S) \
  case S: LT_TRY(g_split_launch<S>(*G, stream)); break;
    LT_GSPLIT_CASE(1) LT_GSPLIT_CASE(2) LT_GSPLIT_CASE(3) LT_GSPLIT_CASE(4) LT_GSPLIT_CASE(5) LT_GSPLIT_CASE(6)
    LT_GSPLIT_CASE(7) LT_GSPLIT_CASE(8) LT_GSPLIT_CASE(9) LT_GSPLIT_CASE(10) LT_GSPLIT_CASE(11) LT_GSPLIT_CASE(12)
#undef LT_GSPLIT_CASE
    default: return set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d unsupported", G->s);
  }
  if (G->ntiles == 0) return LT_OK;
  OzGroupedSource src{G->d_problems, G->d_tiles, G->ntiles};
  return launch_gemm<true>(G->s, src, G->ntiles, ctx, stream);
}

// Kernel attribute set-up only (ntiles = 0: nothing is launched), before a stream capture.
int grouped_prepare(const Grouped* G) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  OzGroupedSource src{G->d_problems, G->d_tiles, 0};
  return launch_gemm<true>(G->s, src, 0, ctx, nullptr);
}

void grouped_destroy(Grouped* G) {
  if (G == nullptr) return;
  cudaFree(G->dev);
  cudaFree(G->ws);
  delete G;
}

int64_t grouped_tiles(const Grouped* G) { return G->ntiles; }

// ---------------------------------------------------------------------------------------------
// Allocation-free Ozaki DGEMM (lt_dgemm_ozaki_noalloc).
//
// For callers that cannot allocate device memory themselves or let a library do it — frameworks
// whose own pool owns every byte of the GPU, services that must not allocate on their request path,
// processes under a hard memory cap — this entry point keeps its scratch (row/column exponents and
// INT8 slice tiles) in a fixed array declared at file scope below. Every GPU that loads the library
// holds LT_OZAKI_NOALLOC_BYTES of device memory for it until the process exits. The array is shared
// by every call on a device and keeps the last call's contents; each call clears the exponent
// region it needs and overwrites the slice tiles it reads, so nothing leaks between calls, but two
// calls whose work overlaps on the GPU (different streams, or host threads) race on the array.
// ---------------------------------------------------------------------------------------------
static __device__ __align__(256) uint8_t g_noalloc_scratch[LT_OZAKI_NOALLOC_BYTES];
static __device__ DeviceStatus g_noalloc_status;

namespace {

struct NoAllocDevice {
  std::once_flag once;
  cudaError_t err = cudaSuccess;
  void* scratch = nullptr;     // device address of g_noalloc_scratch on this device
  DeviceStatus* status = nullptr;
  int sm_count = 0;
  std::atomic<bool> ready{false};  // set-up done on this device: its status word may hold a report
};
NoAllocDevice g_noalloc[64];

// Per-device set-up on the first call made with that device current. In host code the symbols'
// names are host-side stand-ins, so their device addresses come from cudaGetSymbolAddress.
int noalloc_setup(int dev, NoAllocDevice** out) {
  if (dev < 0 || dev >= 64) return set_error(LT_ERR_INVALID_ARGUMENT, "device %d out of range", dev);
  NoAllocDevice& d = g_noalloc[dev];
  std::call_once(d.once, [&] {
    d.err = cudaGetSymbolAddress(&d.scratch, g_noalloc_scratch);
    if (d.err == cudaSuccess) d.err = cudaGetSymbolAddress(reinterpret_cast<void**>(&d.status), g_noalloc_status);
    if (d.err == cudaSuccess) d.err = cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (d.err == cudaSuccess) d.ready.store(true);
  });
  if (d.err != cudaSuccess)
    return set_error(LT_ERR_CUDA, "static scratch set-up failed: %s", cudaGetErrorString(d.err));
  *out = &d;
  return LT_OK;
}

}  // namespace

// Device address of the allocation-free path's error word on device `dev` (set-up included).
int noalloc_status_word(int dev, DeviceStatus** st) {
  NoAllocDevice* nd = nullptr;
  LT_TRY(noalloc_setup(dev, &nd));
  *st = nd->status;
  return LT_OK;
}

// Reads the allocation-free path's error word on device `dev` into *out and clears it; *out is
// zero when that path has not been set up on the device (nothing can have reported there).
int noalloc_take_status(int dev, DeviceStatus* out) {
  *out = DeviceStatus{0, 0, 0, 0};
  if (dev < 0 || dev >= 64 || !g_noalloc[dev].ready.load()) return LT_OK;
  DeviceStatus* st = g_noalloc[dev].status;
  LT_CUDA_TRY(cudaMemcpy(out, st, sizeof *out, cudaMemcpyDeviceToHost));
  if (out->code != 0) LT_CUDA_TRY(cudaMemset(st, 0, sizeof *out));
  return LT_OK;
}

int noalloc_run(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                double beta, int s, cudaStream_t stream) {
  int dev = -1;
  LT_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(LT_ERR_INVALID_ARGUMENT, "device %d out of range", dev);
  int major = 0;
  LT_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  if (major != 10) return set_error(LT_ERR_UNSUPPORTED, "device %d is not an sm_100 device", dev);
  const Layout L = layout_for(M, N, K, s);
  if (L.total > static_cast<size_t>(LT_OZAKI_NOALLOC_BYTES))
    return set_error(LT_ERR_INVALID_ARGUMENT,
                     "%lld x %lld x %lld with %d slices needs %zu bytes of scratch; the static scratch holds %lld",
                     static_cast<long long>(M), static_cast<long long>(N), static_cast<long long>(K), s, L.total,
                     static_cast<long long>(LT_OZAKI_NOALLOC_BYTES));
  NoAllocDevice* nd = nullptr;
  LT_TRY(noalloc_setup(dev, &nd));
  // A stack description of the device (nothing is allocated) whose status word is the static one,
  // read by lt_check_device_status. The split and the product are the stages lt_dgemm_ozaki runs,
  // with the same launch plan (CTA-pair kernel and half-major B slices where it takes them), so
  // the results are bit-identical to it.
  DeviceContext ctx;
  ctx.device = dev;
  ctx.sm_count = nd->sm_count;
  ctx.status = nd->status;
  LT_TRY(split_on(&ctx, A, B, M, N, K, s, nd->scratch, L.total, stream));
  return product_on(&ctx, C, M, N, K, alpha, beta, s, nd->scratch, L.total, stream);
}

}  // namespace ozaki
}  // namespace lt

extern "C" int lt_dgemm_ozaki_noalloc(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                                      double alpha, double beta, int slices, void* stream) {
  if (M < 0 || N < 0 || K < 0 || M > 0x7fffffff || N > 0x7fffffff || K > 0x7fffffff)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "bad dimensions");
  if ((M > 0 && K > 0 && A == nullptr) || (K > 0 && N > 0 && B == nullptr) || (M > 0 && N > 0 && C == nullptr))
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "null matrix pointer");
  if (((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(C)) & 7) != 0)
    return lt::set_error(LT_ERR_UNALIGNED, "matrix pointers must be 8-byte aligned");
  if (slices < 1 || slices > LT_OZAKI_MAX_SLICES)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "slice count %d outside [1, %d]", slices, LT_OZAKI_MAX_SLICES);
  if (M == 0 || N == 0) return lt::ok();
  LT_TRY(lt::ozaki::noalloc_run(A, B, C, M, N, K, alpha, beta, slices, reinterpret_cast<cudaStream_t>(stream)));
  return lt::ok();
}
