// ozaki_crt.cu — DGEMM in the Ozaki scheme II ("CRT form") on INT8 tensor cores for sm_100a.
//
// No reference counterpart: a new implementation behind the reference's dgemm contract
// (routines/dgemm/dgemm.h:9). Method: Ozaki, Uchino and Imamura's scheme II (integer emulation
// of a floating-point product through modular arithmetic and the Chinese remainder theorem),
// written here from the mathematics:
//
//   1. scaling (HBM-bound): row i of A is scaled by 2^s_i, column j of B by 2^s_j, the shifts taken
//      from integer bounds on the rows' and columns' 2-norms so that V = trunc(A[i,k] 2^s_i) and
//      W = trunc(B[k,j] 2^s_j) satisfy |V_i|_2 <= 2^ta and |W_j|_2 <= 2^tb, where
//      2^(ta+tb) <= Mprod (1 - 2^-20) / 2 and Mprod is the product of n pairwise-coprime moduli
//      m_l <= 256: by the Cauchy-Schwarz inequality every |sum_k V W| is below Mprod / 2.
//   2. residues (HBM-bound): V and W as n symmetric residues each (one signed byte per modulus):
//      plane l of A holds V mod m_l, row-major [M][Kp]; plane l of B holds W mod m_l transposed,
//      [N][Kp] (K-major, as the tensor core reads both operands).
//   3. products (tensor cores): for each modulus, one INT8 x INT8 -> INT32 GEMM of the residue
//      planes (exact), reduced to the residue r_l in [0, m_l) of (sum_k V W) and stored as a byte in
//      residue plane l of C.
//   4. reconstruction (FP64 ALU, its own kernel): C' = sum_k V W is the integer in (-Mprod/2,
//      Mprod/2) with C' = r_l (mod m_l). With the CRT basis P_l = (Mprod/m_l) y_l,
//      y_l = (Mprod/m_l)^-1 mod m_l, split into nl limbs of w bits: L_k = sum_l (r_l - 128) P_lk plus
//      128 in limb 0 (exact in FP64; sum_l P_l = 1 mod Mprod, so L = C' mod Mprod), Q = rint(L_hi
//      F_hi + L_lo F_lo) (F_k = 2^(w k) / Mprod), D_k = fma(-Q, M_k, L_k) and C' = Horner of the D_k
//      in base 2^w; then C = fma(alpha, C' 2^-s_i 2^-s_j, beta C0). The CPU oracle (oracle/oracle.c,
//      oracle_crt_dgemm) performs the same arithmetic, so results are bit-identical.
//
// Against the slice form (ozaki.cu) the product count is n, not s(s+1)/2: at FP64 accuracy on the
// 8192^3 workload 14 INT8 products instead of 28. Scaling by the 2-norm rather than by K times the
// largest entry gains about a bit per operand on uniformly distributed rows and more on rows whose
// entries spread over many binades: one modulus fewer for the same accuracy.
//
// Product kernel: persistent CTA pairs over (modulus, tile) work items, modulus-major; a pair runs
// the whole K loop of one modulus for one 256 x 256 or 256 x 512 tile of C with
// tcgen05.mma.cta_group::2.kind::i8 (M256 N256 K32; two MMAs per K step for the 512-wide tile), into
// one of two 256-column TMEM accumulators or one 512-column accumulator; operands staged by 3-D TMA
// (plane = the modulus) with 128-byte swizzle. Roles (320 threads per CTA):
//   warp 0      TMA producer (both CTAs)
//   warp 1      rank 0: MMA issuer for the pair; rank 1: forwards each landed stage to rank 0
//   warps 2..9  drain: TMEM -> registers, INT32 -> residue in [0, m), bytes to the residue planes,
//               then the accumulator goes back to the MMA warp
// The reconstruction runs afterwards as a separate kernel at full occupancy: done inside the product
// kernel by a few warps it was latency-bound (one warp per sub-partition, long FP64 chains, global
// round trips) and held the tensor pipe back. Every wait is bounded (LT_WAIT_TIMEOUT_NS).
#include <cuda.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "lt_internal.h"
#include "lt_runtime.cuh"

namespace lt {
namespace crt {

constexpr int kMaxMod = LT_OZAKI_CRT_MAX_MODULI;
constexpr int kMinMod = LT_OZAKI_CRT_MIN_MODULI;
// Pairwise-coprime moduli no larger than 256, largest first (256 = 2^8; 255 = 3*5*17; 253 = 11*23;
// 247 = 13*19; 217 = 7*31; the rest prime): every symmetric residue is one signed byte.
constexpr int kModuli[kMaxMod] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
                                  223, 217, 211, 199, 197, 193, 191, 181, 179, 173};
constexpr int kBM = 128;                          // rows of C per CTA (256 per pair)
constexpr int kBN = 256;                          // N of one pair MMA (columns of C)
constexpr int kBK = 128;                          // K bytes per stage (one 128-byte swizzle row)
constexpr int kMmaK = 32;                         // K of one kind::i8 MMA
constexpr int kABytes = kBM * kBK;                // 16 KB
constexpr int kBHalfBytes = (kBN / 2) * kBK;      // 16 KB: this CTA's 128 rows of one MMA's B
constexpr int kMaxSmem = 232448;
constexpr int kOverhead = 1024 + 512;
constexpr int kDrainWarps = 8;                    // two per TMEM lane quarter, each half the columns
constexpr int kThreads = 64 + 32 * kDrainWarps;
constexpr int kGroupSteps = 1023;                 // K steps per INT32 accumulation: 1023*128*128^2 < 2^31
constexpr int kPadN = 512;                        // residue planes of C: columns rounded up to this

// Pair tile of 256 x BN: BN = 256, one pair MMA per K step and two TMEM accumulators (the drain of one
// modulus overlaps the products of the next); BN = 512, two pair MMAs per K step sharing the A stage
// (a quarter less operand data per product from L2 into shared memory) into one 512-column
// accumulator, so each modulus's products wait for the drain of the previous one.
template <int BN>
struct Tile {
  static constexpr int kMmas = BN / kBN;
  static constexpr int kStageBytes = kABytes + kMmas * kBHalfBytes;
  static constexpr int kStages = std::min(8, (kMaxSmem - kOverhead) / kStageBytes);
  static constexpr int kSmem = kStages * kStageBytes + kOverhead;
  static constexpr int kAccBufs = BN == kBN ? 2 : 1;
  static_assert(kStages >= 3, "shared-memory ring too small");
  static_assert(kAccBufs * BN == 512, "TMEM holds 512 INT32 columns");
};

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }
inline int64_t ceil_div(int64_t x, int64_t m) { return (x + m - 1) / m; }

// ---------------------------------------------------------------------------------------------
// Constants of a modulus set (host arithmetic, exact)
// ---------------------------------------------------------------------------------------------
struct Consts {
  int n, nl, w, ta, tb;  // norm bounds: |V_i|_2 <= 2^ta, |W_j|_2 <= 2^tb
  int32_t m[kMaxMod];
  int32_t h[kMaxMod];             // (m - 1) / 2: the symmetric residues lie in [-h, h]
  // residues of the scaled inputs: x = dp4a(bytes of V + 2^62, coef) + add, x mod m by umulhi
  uint32_t coef_lo[kMaxMod], coef_hi[kMaxMod];  // bytes (2^(8d) mod m), d = 0..3 and 4..7
  uint32_t add[kMaxMod];                        // m - (2^62 mod m)
  uint32_t split_magic[kMaxMod];                // ceil(2^32 / m)
  // INT32 accumulators -> residues in [0, m): y = dp2a(acc ^ 2^31, 1 | c16 << 8, acc_add) < 2^24,
  // q = umulhi(y, magic) >> 7
  uint32_t c16[kMaxMod];          // 2^16 mod m
  uint32_t acc_add[kMaxMod];      // m - (2^31 mod m)
  uint32_t drain_magic[kMaxMod];  // ceil(2^39 / m)
  // reconstruction
  double P[kMaxMod][4];  // limbs of the CRT basis
  double Mk[4];          // limbs of Mprod
  double Kc[4];          // -128 sum_l P_lk, plus 128 in limb 0 (residues r in [0, m) enter as r - 128)
  double f_hi, f_lo;
};

// Unsigned integers of up to 256 bits (little-endian 32-bit words): what the constants need.
struct Big {
  uint32_t d[8] = {};
  void mul_small(uint32_t v) {
    uint64_t carry = 0;
    for (uint32_t& x : d) {
      const uint64_t t = static_cast<uint64_t>(x) * v + carry;
      x = static_cast<uint32_t>(t);
      carry = t >> 32;
    }
  }
  uint32_t divmod_small(uint32_t v) {  // *this /= v, returns the remainder
    uint64_t rem = 0;
    for (int i = 7; i >= 0; --i) {
      const uint64_t cur = (rem << 32) | d[i];
      d[i] = static_cast<uint32_t>(cur / v);
      rem = cur % v;
    }
    return static_cast<uint32_t>(rem);
  }
  int bit_length() const {
    for (int i = 7; i >= 0; --i)
      if (d[i] != 0) return 32 * i + 32 - __builtin_clz(d[i]);
    return 0;
  }
  uint64_t bits(int lo, int w) const {  // bits lo .. lo+w-1 (w <= 48)
    uint64_t r = 0;
    for (int b = 0; b < w; ++b) {
      const int i = lo + b;
      if (i < 256 && ((d[i >> 5] >> (i & 31)) & 1u)) r |= uint64_t(1) << b;
    }
    return r;
  }
};

inline uint32_t pow2_mod(int e, uint32_t m) {
  uint64_t r = 1 % m;
  for (int i = 0; i < e; ++i) r = (r * 2) % m;
  return static_cast<uint32_t>(r);
}

inline uint32_t inverse_mod(uint32_t a, uint32_t m) {  // a^-1 mod m, gcd(a, m) = 1
  int64_t t = 0, nt = 1, r = m, nr = a % m;
  while (nr != 0) {
    const int64_t q = r / nr;
    int64_t x = t - q * nt; t = nt; nt = x;
    x = r - q * nr; r = nr; nr = x;
  }
  return static_cast<uint32_t>(t < 0 ? t + m : t);
}

// Constants for n moduli: ta + tb is the largest Tc with 2^Tc <= Mprod (1 - 2^-20) / 2, split
// evenly, each at most 62 (the residues are taken from 64-bit integers). The margin keeps the
// quotient estimate of the reconstruction, whose error is far below 2^-21, from rounding the wrong way.
Consts make_consts(int n) {
  Consts c;
  std::memset(&c, 0, sizeof c);
  c.n = n;
  Big Mp;
  Mp.d[0] = 1;
  for (int l = 0; l < n; ++l) Mp.mul_small(static_cast<uint32_t>(kModuli[l]));
  c.w = n <= 16 ? 42 : 41;  // n 2^7 2^w <= 2^53: the limb sums stay exact
  c.nl = (Mp.bit_length() + c.w - 1) / c.w;
  for (int l = 0; l < n; ++l) {
    const uint32_t m = static_cast<uint32_t>(kModuli[l]);
    c.m[l] = static_cast<int32_t>(m);
    c.h[l] = static_cast<int32_t>((m - 1) / 2);
    uint32_t lo = 0, hi = 0;
    for (int b = 0; b < 4; ++b) {
      lo |= pow2_mod(8 * b, m) << (8 * b);
      hi |= pow2_mod(8 * (b + 4), m) << (8 * b);
    }
    c.coef_lo[l] = lo;
    c.coef_hi[l] = hi;
    c.add[l] = m - pow2_mod(62, m);
    c.split_magic[l] = static_cast<uint32_t>(((uint64_t(1) << 32) + m - 1) / m);
    c.c16[l] = pow2_mod(16, m);
    c.acc_add[l] = m - pow2_mod(31, m);
    c.drain_magic[l] = static_cast<uint32_t>(((uint64_t(1) << 39) + m - 1) / m);
    Big Ml = Mp;
    Ml.divmod_small(m);
    Big t = Ml;
    const uint32_t r = t.divmod_small(m);
    Big P = Ml;
    P.mul_small(inverse_mod(r, m));
    for (int k = 0; k < c.nl; ++k) c.P[l][k] = static_cast<double>(P.bits(c.w * k, c.w));
  }
  for (int k = 0; k < c.nl; ++k) {
    c.Mk[k] = static_cast<double>(Mp.bits(c.w * k, c.w));
    int64_t s = 0;
    for (int l = 0; l < n; ++l) s += static_cast<int64_t>(c.P[l][k]);
    c.Kc[k] = -128.0 * static_cast<double>(s) + (k == 0 ? 128.0 : 0.0);
  }
  double md = c.Mk[c.nl - 1];
  for (int k = c.nl - 2; k >= 0; --k) md = std::fma(md, std::ldexp(1.0, c.w), c.Mk[k]);
  c.f_hi = std::ldexp(1.0, c.w * (c.nl - 1)) / md;
  c.f_lo = std::ldexp(1.0, c.w * (c.nl - 2)) / md;
  Big q = Mp;
  q.mul_small((1u << 20) - 1u);
  q.divmod_small(1u << 21);
  const int T = q.bit_length() - 1;
  c.ta = std::min(62, T / 2);
  c.tb = std::min(62, T - T / 2);
  return c;
}

// Limbs of the reconstruction for NM moduli: ceil(bit length of Mprod / w), w = 42 up to 16 moduli
// and 41 above (make_consts derives the same count; the launchers check it).
__host__ __device__ constexpr int limbs_for(int nm) { return nm <= 10 ? 2 : (nm <= 16 ? 3 : 4); }

// The constants of every modulus count in constant memory (filled once per device), read by the
// kernels with compile-time offsets through the constant cache.
__constant__ Consts c_table[kMaxMod - kMinMod + 1];

int ensure_table(int device) {
  static std::once_flag once[64];
  static cudaError_t err[64];
  std::call_once(once[device], [&] {
    Consts host[kMaxMod - kMinMod + 1];
    for (int n = kMinMod; n <= kMaxMod; ++n) host[n - kMinMod] = make_consts(n);
    err[device] = cudaMemcpyToSymbol(c_table, host, sizeof host);
  });
  LT_CUDA_TRY(err[device]);
  return LT_OK;
}

// ---------------------------------------------------------------------------------------------
// Workspace: [chunk exponents of A: M x ncha int][chunk sums of A: M x ncha u64]
//            [the same for B: N x nchb][row shifts: M int][column shifts: N int]
//            [A residues n x M x Kp][B residues n x N x Kp]
//            [C residue planes n x Mp x Np], 256-aligned; ncha = ceil(K / 512), nchb = ceil(K / 128);
//            Mp, Np = M, N rounded up to the pair tile (the product writes whole tiles).
// ---------------------------------------------------------------------------------------------
constexpr int kChunkA = 512;  // K positions per chunk of a row of A (a warp, 16 per lane)
constexpr int kChunkB = 128;  // K positions per chunk of a column of B (a block, 16 per thread)

struct Layout {
  int64_t Kp, Mp, Np, ncha, nchb;
  size_t off_eca, off_sca, off_ecb, off_scb, off_ea, off_eb, off_ra, off_rb, off_rc, total;
};

Layout layout_for(int64_t M, int64_t N, int64_t K, int n) {
  Layout L;
  L.Kp = round_up(std::max<int64_t>(K, 1), kBK);
  L.Mp = round_up(std::max<int64_t>(M, 1), 2 * kBM);
  L.Np = round_up(std::max<int64_t>(N, 1), kPadN);
  L.ncha = ceil_div(std::max<int64_t>(K, 1), kChunkA);
  L.nchb = ceil_div(std::max<int64_t>(K, 1), kChunkB);
  size_t o = 0;
  L.off_eca = o; o += round_up(4 * M * L.ncha, 256);
  L.off_sca = o; o += round_up(8 * M * L.ncha, 256);
  L.off_ecb = o; o += round_up(4 * N * L.nchb, 256);
  L.off_scb = o; o += round_up(8 * N * L.nchb, 256);
  L.off_ea = o;  o += round_up(4 * M, 256);
  L.off_eb = o;  o += round_up(4 * N, 256);
  L.off_ra = o;  o += round_up(static_cast<int64_t>(n) * M * L.Kp, 256);
  L.off_rb = o;  o += round_up(static_cast<int64_t>(n) * N * L.Kp, 256);
  L.off_rc = o;  o += static_cast<size_t>(n) * L.Mp * L.Np;
  L.total = o;
  return L;
}

// ---------------------------------------------------------------------------------------------
// Scaling: bounds on the 2-norms of the rows of A and the columns of B
// ---------------------------------------------------------------------------------------------
// Row i of A gets the shift s_i that makes V = trunc(A[i,k] 2^s_i) satisfy |V_i|_2 <= 2^ta (columns
// of B likewise with 2^tb). The bound is computed in integers, so its value does not depend on the
// order of the reductions and the CPU oracle (oracle_crt_shift) reproduces it exactly:
//   entry a != 0: e = its frexp exponent, x = floor(|a| 2^(15 - e)) + 1 (subnormals: e = -1021,
//     x = 2^14 + 1), so |a| < x 2^(e - 15);
//   chunk (512 consecutive k of a row of A, 128 of a column of B): E_c = the largest e,
//     S_c = sum of ceil(x^2 4^(e - E_c)) (each term at most 2^30);
//   row: sigma = the largest E_c, S = sum of ceil(S_c / 4^(sigma - E_c)) (< 2^54 for K < 2^23),
//     so that |row|_2^2 < S 2^(2 sigma - 30);
//   s = t + 15 - sigma - ceil(bitlen(S - 1) / 2): |V|_2^2 < S 2^(2t - 2 ceil(bitlen(S - 1) / 2)) <= 2^2t.
// A row without nonzero entries takes s = 0, one holding NaN or Inf kSentinel.
constexpr int kEmpty = INT_MIN;  // chunk or row without a nonzero entry

// (e + 2048) << 16 | x of a finite nonzero entry, 0 for zero, 0xffffffff for NaN or Inf: the largest
// code of a chunk carries its largest exponent, or flags a non-finite entry.
__device__ __forceinline__ uint32_t entry_code(double a) {
  const unsigned long long b = abs_bits(a);
  if (b == 0ull) return 0u;
  if (b >= 0x7ff0000000000000ull) return 0xffffffffu;
  const uint32_t E = static_cast<uint32_t>(b >> 52);
  if (E == 0u) return ((2048u - 1021u) << 16) | ((1u << 14) + 1u);
  return ((E + 1026u) << 16) | ((1u << 14) + static_cast<uint32_t>((b >> 38) & 0x3fffu) + 1u);
}

// ceil(x^2 4^(e - E_c)) of an entry code; ecode = the chunk's largest code >> 16 = E_c + 2048
__device__ __forceinline__ uint32_t entry_term(uint32_t code, uint32_t ecode) {
  if (code == 0u) return 0u;
  const uint32_t x = code & 0xffffu;
  const uint32_t x2 = x * x;  // x <= 2^15
  const uint32_t d = 2u * (ecode - (code >> 16));
  if (d >= 31u) return 1u;  // 0 < x^2 <= 2^30 < 2^d
  return (x2 + ((1u << d) - 1u)) >> d;  // < 2^31 + 2^30: no overflow
}

// ceil(v / 2^d), d >= 0, v < 2^62
__device__ __forceinline__ unsigned long long ceil_shr(unsigned long long v, int d) {
  if (d == 0) return v;
  if (d >= 63) return v != 0ull ? 1ull : 0ull;
  return (v + ((1ull << d) - 1ull)) >> d;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int chunk_exponent(uint32_t mx) {
  return mx == 0xffffffffu ? kSentinel : (mx == 0u ? kEmpty : static_cast<int>(mx >> 16) - 2048);
}

// Chunk statistics of the rows of A (a warp per row and chunk of 512, 16 entries per lane; blocks
// 0..row_blocks-1) and of the columns of B (a block per 32 columns and chunk of 128, 16 entries per
// thread, as the column split reads them; the remaining blocks): ec[r * nch + c] = E_c (kEmpty, or
// kSentinel for a non-finite entry), sc[r * nch + c] = S_c. Either side may be empty (M = 0 or N = 0).
__global__ void __launch_bounds__(256) crt_stats_kernel(const double* __restrict__ A, int64_t M, int64_t lda,
                                                        int64_t ncha, const double* __restrict__ B, int64_t N,
                                                        int64_t ldb, int64_t nchb, int64_t K, int64_t row_blocks,
                                                        int* __restrict__ ec_a, unsigned long long* __restrict__ sc_a,
                                                        int* __restrict__ ec_b, unsigned long long* __restrict__ sc_b) {
  __shared__ uint32_t s_max[8][32];
  __shared__ unsigned long long s_sum[8][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t code[16];
  if (static_cast<int64_t>(blockIdx.x) < row_blocks) {
    const int64_t item = static_cast<int64_t>(blockIdx.x) * 8 + warp;  // row * ncha + chunk
    if (item >= M * ncha) return;
    const int64_t row = item / ncha, k0 = (item - row * ncha) * kChunkA + lane * 16;
    const double* a = A + row * lda + k0;
    if (k0 + 16 <= K && (reinterpret_cast<uintptr_t>(a) & 15) == 0) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const double2 x = __ldcs(reinterpret_cast<const double2*>(a) + j);
        code[2 * j] = entry_code(x.x);
        code[2 * j + 1] = entry_code(x.y);
      }
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) code[j] = (k0 + j < K) ? entry_code(__ldcs(a + j)) : 0u;
    }
    uint32_t mx = 0u;
#pragma unroll
    for (int j = 0; j < 16; ++j) mx = max(mx, code[j]);
    mx = __reduce_max_sync(0xffffffffu, mx);
    unsigned long long sum = 0ull;
    if (mx != 0u && mx != 0xffffffffu) {
#pragma unroll
      for (int j = 0; j < 16; ++j) sum += entry_term(code[j], mx >> 16);
      sum = warp_sum_u64(sum);
    }
    if (lane == 0) {
      ec_a[item] = chunk_exponent(mx);
      sc_a[item] = sum;
    }
  } else {
    const int64_t ncb = (N + 31) / 32, bi = static_cast<int64_t>(blockIdx.x) - row_blocks;
    const int64_t c = bi / ncb, col = (bi - c * ncb) * 32 + lane;
    const int64_t k0 = c * kChunkB + warp * 16;
    const double* b = B + k0 * ldb + col;
    if (col < N && k0 + 16 <= K) {
#pragma unroll
      for (int j = 0; j < 16; ++j) code[j] = entry_code(__ldcs(b + j * ldb));
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) code[j] = (col < N && k0 + j < K) ? entry_code(__ldcs(b + j * ldb)) : 0u;
    }
    uint32_t mx = 0u;
#pragma unroll
    for (int j = 0; j < 16; ++j) mx = max(mx, code[j]);
    s_max[warp][lane] = mx;
    __syncthreads();
    mx = 0u;
#pragma unroll
    for (int w = 0; w < 8; ++w) mx = max(mx, s_max[w][lane]);
    unsigned long long sum = 0ull;
    if (mx != 0u && mx != 0xffffffffu) {
#pragma unroll
      for (int j = 0; j < 16; ++j) sum += entry_term(code[j], mx >> 16);
    }
    s_sum[warp][lane] = sum;
    __syncthreads();
    if (warp == 0 && col < N) {
      unsigned long long total = 0ull;
#pragma unroll
      for (int w = 0; w < 8; ++w) total += s_sum[w][lane];
      ec_b[col * nchb + c] = chunk_exponent(mx);
      sc_b[col * nchb + c] = total;
    }
  }
}

// The shifts: a warp per row of A (warps 0..M-1) and per column of B (the next N) combines that
// row's chunk statistics.
__global__ void __launch_bounds__(256) crt_shift_kernel(const int* __restrict__ ec_a,
                                                        const unsigned long long* __restrict__ sc_a, int64_t M,
                                                        int64_t ncha, const int* __restrict__ ec_b,
                                                        const unsigned long long* __restrict__ sc_b, int64_t N,
                                                        int64_t nchb, int ta, int tb, int* __restrict__ sh_a,
                                                        int* __restrict__ sh_b) {
  const int64_t wid = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= M + N) return;
  const bool is_a = wid < M;
  const int64_t r = is_a ? wid : wid - M, nch = is_a ? ncha : nchb;
  const int* ec = is_a ? ec_a + r * ncha : ec_b + r * nchb;
  const unsigned long long* sc = is_a ? sc_a + r * ncha : sc_b + r * nchb;
  int sigma = kEmpty;
  for (int64_t c = lane; c < nch; c += 32) sigma = max(sigma, ec[c]);
  sigma = __reduce_max_sync(0xffffffffu, sigma);
  int out = 0;
  if (sigma == kSentinel) {
    out = kSentinel;
  } else if (sigma != kEmpty) {
    unsigned long long S = 0ull;
    for (int64_t c = lane; c < nch; c += 32)
      if (ec[c] != kEmpty) S += ceil_shr(sc[c], 2 * (sigma - ec[c]));
    S = warp_sum_u64(S);
    const int b = S > 1ull ? 64 - __clzll(static_cast<long long>(S - 1ull)) : 0;  // bitlen(S - 1)
    out = (is_a ? ta : tb) + 15 - sigma - (b + 1) / 2;
  }
  if (lane == 0) (is_a ? sh_a : sh_b)[r] = out;
}

// ---------------------------------------------------------------------------------------------
// Residues of the scaled operands
// ---------------------------------------------------------------------------------------------
// Four values' symmetric residues modulo modulus l as one word of two's-complement bytes, from
// U = V + 2^62 given as two words per value. Modulus 256 (l = 0): the low byte of V. Otherwise
// raw = sum_d byte_d(U) (2^(8d) mod m) + m - (2^62 mod m) is congruent to V and below 2^19, so
// q = floor((raw + h) / m) = umulhi(raw + h, ceil(2^32 / m)) exactly and raw - q m, in [-h, h], is the
// symmetric residue; PRMT packs the low bytes of four of them. Called with a constant l (unrolled
// loops), so the constants are read with fixed offsets.
__device__ __forceinline__ uint32_t residue_word(int l, const uint32_t* ulo, const uint32_t* uhi, const Consts& c) {
  if (l == 0)
    return __byte_perm(__byte_perm(ulo[0], ulo[1], 0x0040), __byte_perm(ulo[2], ulo[3], 0x0040), 0x5410);
  uint32_t r[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t raw = __dp4a(ulo[i], c.coef_lo[l], __dp4a(uhi[i], c.coef_hi[l], c.add[l]));
    const uint32_t q = __umulhi(raw + static_cast<uint32_t>(c.h[l]), c.split_magic[l]);
    r[i] = raw - q * static_cast<uint32_t>(c.m[l]);
  }
  return __byte_perm(__byte_perm(r[0], r[1], 0x0040), __byte_perm(r[2], r[3], 0x0040), 0x5410);
}

// The 16 bytes of plane l for 16 consecutive values (one thread's share).
__device__ __forceinline__ uint4 residue_plane(int l, const uint32_t (&ulo)[16], const uint32_t (&uhi)[16],
                                               const Consts& c) {
  return make_uint4(residue_word(l, ulo, uhi, c), residue_word(l, ulo + 4, uhi + 4, c),
                    residue_word(l, ulo + 8, uhi + 8, c), residue_word(l, ulo + 12, uhi + 12, c));
}

// V = trunc(a 2^s) of 16 finite entries of a row (column) with shift s, as U = V + 2^62 in two words
// each: the product by 2^s is exact whenever it is at least 1 in magnitude (a power-of-two scaling to
// a normal number) and anything smaller truncates to 0, so one multiplication (two when 2^s is above
// the double range) and a truncating conversion give V exactly; |V| <= |V_row|_2 <= 2^62. A row
// (column) holding NaN or Inf (s = kSentinel) gets V = 0.
__device__ __forceinline__ void scaled_words(const double (&v)[16], int s, uint32_t (&ulo)[16], uint32_t (&uhi)[16]) {
  if (s == kSentinel) {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      ulo[i] = 0u;
      uhi[i] = 1u << 30;
    }
    return;
  }
  const int d1 = s < 1023 ? s : 1023;  // s > -1022: the shift of the largest finite rows is above -1000
  const double s1 = pow2i(d1), s2 = pow2i(s - d1);
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    double x = __dmul_rn(v[i], s1);
    if (s > 1023) x = __dmul_rn(x, s2);
    const unsigned long long U = static_cast<unsigned long long>(__double2ll_rz(x) + (1ll << 62));
    ulo[i] = static_cast<uint32_t>(U);
    uhi[i] = static_cast<uint32_t>(U >> 32);
  }
}

// Rows of A: a warp covers 512 K positions of one row (16 per lane), a block 8 rows (blockIdx.x:
// row block, blockIdx.y: K segment). Each modulus plane receives 512 contiguous bytes per warp.
template <int NM>
__global__ void __launch_bounds__(256, 3) crt_split_rows_kernel(const double* __restrict__ A, int64_t M, int64_t K,
                                                             int64_t lda, int64_t Kp,
                                                             const int* __restrict__ shifts,
                                                             int8_t* __restrict__ out, int64_t plane) {
  const Consts& c = c_table[NM - kMinMod];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = static_cast<int64_t>(blockIdx.x) * 8 + warp;
  const int64_t k0 = static_cast<int64_t>(blockIdx.y) * 512 + lane * 16;
  if (row >= M || k0 >= Kp) return;
  const int sh = shifts[row];
  const double* a = A + row * lda + k0;
  double v[16];
  if (k0 + 16 <= K && (reinterpret_cast<uintptr_t>(a) & 15) == 0) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const double2 x = __ldcs(reinterpret_cast<const double2*>(a) + j);
      v[2 * j] = x.x;
      v[2 * j + 1] = x.y;
    }
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = (k0 + j < K) ? __ldcs(a + j) : 0.0;
  }
  uint32_t ulo[16], uhi[16];
  scaled_words(v, sh, ulo, uhi);
  int8_t* dst = out + row * Kp + k0;
#pragma unroll
  for (int l = 0; l < NM; ++l) *reinterpret_cast<uint4*>(dst + l * plane) = residue_plane(l, ulo, uhi, c);
}

// Columns of B, transposed to K-major: a block covers 32 columns (one per lane) and 128 K positions
// (16 per warp). The loads read 32 consecutive columns of a row of B; the residues pass through
// shared memory, eight planes at a time, so that each plane's 32 x 128-byte block is written as
// whole 128-byte rows.
constexpr int kColPitch = 144;  // bytes per column row in shared memory (128 + 16: no bank conflicts)
constexpr int kColPlanes = 8;   // planes staged at a time (8 x 4.5 KB)
template <int NM>
__global__ void __launch_bounds__(256, 3) crt_split_cols_kernel(const double* __restrict__ B, int64_t K, int64_t N,
                                                             int64_t ldb, int64_t Kp,
                                                             const int* __restrict__ shifts,
                                                             int8_t* __restrict__ out, int64_t plane) {
  __shared__ __align__(16) uint8_t stage[kColPlanes][32 * kColPitch];
  const Consts& c = c_table[NM - kMinMod];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t col0 = static_cast<int64_t>(blockIdx.x) * 32;
  const int64_t kb = static_cast<int64_t>(blockIdx.y) * kBK;
  const int64_t col = col0 + lane;
  const int64_t k0 = kb + warp * 16;
  const int sh = col < N ? shifts[col] : 0;
  double v[16];
  const double* b = B + k0 * ldb + col;
  if (col < N && k0 + 16 <= K) {
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __ldcs(b + j * ldb);
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = (col < N && k0 + j < K) ? __ldcs(b + j * ldb) : 0.0;
  }
  uint32_t ulo[16], uhi[16];
  scaled_words(v, sh, ulo, uhi);
  // thread t then writes 16 bytes of column t / 8 (K bytes 16 (t % 8) ..) of each staged plane
  const int cl = threadIdx.x >> 3, part = threadIdx.x & 7;
  const bool writes = col0 + cl < N;
  int8_t* dst = out + (col0 + cl) * Kp + kb + part * 16;
#pragma unroll
  for (int l0 = 0; l0 < NM; l0 += kColPlanes) {
    if (l0 > 0) __syncthreads();  // the previous group's reads are done
#pragma unroll
    for (int l = l0; l < l0 + kColPlanes && l < NM; ++l)
      *reinterpret_cast<uint4*>(&stage[l - l0][lane * kColPitch + warp * 16]) = residue_plane(l, ulo, uhi, c);
    __syncthreads();
    if (writes) {
#pragma unroll
      for (int l = l0; l < l0 + kColPlanes && l < NM; ++l)
        *reinterpret_cast<uint4*>(dst + l * plane) =
            *reinterpret_cast<const uint4*>(&stage[l - l0][cl * kColPitch + part * 16]);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Product kernel: residue planes of C
// ---------------------------------------------------------------------------------------------
struct Problem {
  uint8_t* res;         // residue planes of C: n x Mp x Np bytes
  int64_t plane, Np;    // plane size and row pitch of the residue planes
  int tiles_m, tiles_n; // 256-row pair blocks, 256-column blocks
  int ksteps;           // Kp / 128
  int kgroups;          // ceil(ksteps / kGroupSteps)
  int group;            // pair-rows per raster group
  int bn;               // tile width (256 or 512)
};

__device__ __forceinline__ void tile_coords(const Problem& p, int64_t t, int* m0, int* n0) {
  const int64_t G = p.group;
  const int64_t group = t / (G * p.tiles_n), first_m = group * G;
  const int64_t gsize = (p.tiles_m - first_m) < G ? (p.tiles_m - first_m) : G;
  const int64_t in_group = t - group * G * p.tiles_n;
  *m0 = static_cast<int>((first_m + in_group % gsize) * 2 * kBM);
  *n0 = static_cast<int>((in_group / gsize) * p.bn);
}

// Residue in [0, m) of an INT32 accumulator modulo an odd modulus m: U = acc + 2^31 (acc ^ 2^31 as an
// unsigned word) has 16-bit halves hi, lo, and y = lo + hi (2^16 mod m) + (m - 2^31 mod m), one dp2a,
// is congruent to acc and below 2^24; floor(y / m) = (y ceil(2^39 / m)) >> 39 exactly (the error term
// is below y m / 2^39 < 1 / m).
__device__ __forceinline__ uint32_t residue_odd(uint32_t acc, uint32_t coef, uint32_t add, uint32_t magic,
                                                uint32_t m) {
  const uint32_t y = __dp2a_lo(acc ^ 0x80000000u, coef, add);
  return y - (__umulhi(y, magic) >> 7) * m;
}

// 32 accumulators of one row -> their residues r in [0, m) modulo m = c.m[l], stored as bytes, two
// 16-byte words. For accumulation group g > 0 the residue of the previous groups (already in `dst`)
// is added modulo m.
__device__ __forceinline__ void drain_chunk(const uint32_t (&v)[32], int l, bool add_prev, const Consts& c,
                                            uint4* dst) {
  uint32_t w[8];
  if (l == 0) {  // m = 256: the low byte
#pragma unroll
    for (int q = 0; q < 8; ++q)
      w[q] = __byte_perm(__byte_perm(v[4 * q], v[4 * q + 1], 0x0040), __byte_perm(v[4 * q + 2], v[4 * q + 3], 0x0040),
                         0x5410);
  } else {
    const uint32_t m = static_cast<uint32_t>(c.m[l]), coef = 1u | (c.c16[l] << 8), add = c.acc_add[l],
                   magic = c.drain_magic[l];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const uint32_t r0 = residue_odd(v[4 * q], coef, add, magic, m);
      const uint32_t r1 = residue_odd(v[4 * q + 1], coef, add, magic, m);
      const uint32_t r2 = residue_odd(v[4 * q + 2], coef, add, magic, m);
      const uint32_t r3 = residue_odd(v[4 * q + 3], coef, add, magic, m);
      w[q] = __byte_perm(__byte_perm(r0, r1, 0x0040), __byte_perm(r2, r3, 0x0040), 0x5410);
    }
  }
  if (add_prev) {  // K beyond one INT32 group: add the earlier groups' residues modulo m
    const uint4 a = dst[0], b = dst[1];
    const uint32_t prev[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    const uint32_t m = static_cast<uint32_t>(c.m[l]);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      uint32_t word = 0;
#pragma unroll
      for (int b4 = 0; b4 < 4; ++b4) {
        uint32_t r = ((w[q] >> (8 * b4)) & 0xffu) + ((prev[q] >> (8 * b4)) & 0xffu);
        r = l == 0 ? (r & 0xffu) : (r >= m ? r - m : r);
        word |= r << (8 * b4);
      }
      w[q] = word;
    }
  }
  dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
  dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

template <int NM, int BN>
__global__ void __launch_bounds__(kThreads, 1)
    crt_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Problem p,
                    DeviceStatus* status) {
  using T = Tile<BN>;
  constexpr int kStages = T::kStages, kStageBytes = T::kStageBytes;
  const Consts& c = c_table[NM - kMinMod];
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* acc_full = empty + kStages;  // [2]
  uint64_t* acc_empty = acc_full + 2;    // [2]
  uint64_t* drain = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  // Work items modulus-major: every pair works on the same residue plane at a time, tile by tile in
  // raster order, so the operand strips one wave of pairs reads are shared in L2 (tile-major order,
  // each pair running all moduli of its tile, read twice the DRAM bytes at 8192^3, 16.8 against
  // 8.2 GB, in the same time), and a problem with fewer tiles than pairs still occupies every pair.
  const int64_t tiles = static_cast<int64_t>(p.tiles_m) * p.tiles_n;
  const int64_t items = tiles * NM;
  const int64_t first = cluster_id_x(), stride = num_clusters_x();
  const int ksteps = p.ksteps, kgroups = p.kgroups;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&full[i], rank == 0 ? 2 : 1);
      mbar_init(&empty[i], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 2 * kDrainWarps);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_desc(&tmA);
    tma_prefetch_desc(&tmB);
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
    // ------------------------------ TMA producer (both CTAs) ------------------------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      for (int64_t w = first; w < items && ok; w += stride) {
        const int l = static_cast<int>(w / tiles);
        int m0, n0;
        tile_coords(p, w - l * tiles, &m0, &n0);
        const int arow = m0 + static_cast<int>(rank) * kBM;
        const int brow = n0 + static_cast<int>(rank) * (kBN / 2);
        for (int ks = 0; ks < ksteps; ++ks) {
          if (!mbar_wait_cluster(&empty[stage], phase ^ 1, abort_flag, status, 81)) { ok = false; break; }
          uint8_t* st = smem + stage * kStageBytes;
          mbar_arrive_expect_tx(&full[stage], kStageBytes);
          tma_load_3d(st, &tmA, &full[stage], ks * kBK, arow, l);
#pragma unroll
          for (int h = 0; h < T::kMmas; ++h)
            tma_load_3d(st + kABytes + h * kBHalfBytes, &tmB, &full[stage], ks * kBK, brow + h * kBN, l);
          if (++stage == kStages) { stage = 0; phase ^= 1; }
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
      for (int64_t w = first; w < items && ok; w += stride) {
        for (int ks = 0; ks < ksteps; ++ks) {
          if (!mbar_wait(&full[stage], phase, abort_flag, status, 82)) { ok = false; break; }
          mbar_arrive_cluster_relaxed(cluster_addr(&full[stage], 0));
          if (++stage == kStages) { stage = 0; phase ^= 1; }
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------ rank 0: MMA issuer for the pair ------------------------------
    constexpr uint32_t idesc = idesc_i8_s32(2 * kBM, kBN);
    const uint64_t a_desc0 = smem_desc_k_sw128(smem_u32(smem));
    const uint64_t b_desc0 = smem_desc_k_sw128(smem_u32(smem + kABytes));
    constexpr uint64_t kStageStep = static_cast<uint64_t>(kStageBytes >> 4);
    constexpr uint64_t kStepK = static_cast<uint64_t>(kMmaK >> 4);  // 32 bytes along the swizzled row
    int stage = 0;
    uint32_t phase = 0;
    uint32_t pass = 0;
    bool ok = true;
    for (int64_t w = first; w < items && ok; w += stride) {
      {
        for (int g = 0; g < kgroups && ok; ++g, ++pass) {
          const uint32_t buf = pass % T::kAccBufs, use = pass / T::kAccBufs;
          if (!__all_sync(0xffffffffu, mbar_wait_cluster(&acc_empty[buf], (use & 1) ^ 1, abort_flag, status, 83))) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d_tmem = tmem_base + buf * kBN;
          const int ks0 = g * kGroupSteps, ks1 = std::min(ksteps, ks0 + kGroupSteps);
          for (int ks = ks0; ks < ks1; ++ks) {
            if (!__all_sync(0xffffffffu, mbar_wait_cluster(&full[stage], phase, abort_flag, status, 84))) {
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
                for (int h = 0; h < T::kMmas; ++h)
                  mma_i8_pair(d_tmem + h * kBN, a0 + k * kStepK, b0 + h * (kBHalfBytes >> 4) + k * kStepK, idesc,
                              (ks > ks0 || k > 0) ? 1u : 0u);
              mma_commit_pair(cluster_addr(&empty[stage], 0));
              mma_commit_pair(cluster_addr(&empty[stage], 1));
            }
            __syncwarp();
            if (++stage == kStages) { stage = 0; phase ^= 1; }
          }
          if (!ok) break;
          if (elect_one_sync()) {
            mma_commit_pair(cluster_addr(&acc_full[buf], 0));
            mma_commit_pair(cluster_addr(&acc_full[buf], 1));
          }
          __syncwarp();
        }
      }
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
    // ------------------------ drain: accumulators -> residue planes of C ------------------------
    const int quarter = warp & 3;             // TMEM lanes 32*quarter .. +31 (rows of this CTA's block)
    const int colhalf = (warp - 2) >> 2;      // columns colhalf*BN/2 .. +BN/2-1 of the tile
    const uint32_t acc_empty_r0[2] = {cluster_addr(&acc_empty[0], 0), cluster_addr(&acc_empty[1], 0)};
    uint32_t pass = 0;
    bool ok = true;
    for (int64_t w = first; w < items && ok; w += stride) {
      const int l = static_cast<int>(w / tiles);
      int m0, n0;
      tile_coords(p, w - l * tiles, &m0, &n0);
      const int64_t row = static_cast<int64_t>(m0) + static_cast<int64_t>(rank) * kBM + quarter * 32 + lane;
      uint8_t* row_base = p.res + row * p.Np + n0 + colhalf * (BN / 2);
      {
        uint8_t* dst = row_base + static_cast<int64_t>(l) * p.plane;
        for (int g = 0; g < kgroups; ++g, ++pass) {
          const uint32_t buf = pass % T::kAccBufs, use = pass / T::kAccBufs;
          if (!mbar_wait_cluster(&acc_full[buf], use & 1, abort_flag, status, 86)) { ok = false; break; }
          tc_fence_after();
          const uint32_t lane_base =
              tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) + buf * kBN + colhalf * (BN / 2);
          // Chunks of 32 columns, the TMEM load of the next issued before the current one is reduced;
          // the accumulator goes back to the MMA warp once the last load has landed.
          constexpr int kChunks = BN / 64;
          uint32_t va[32], vb[32];
          tmem_ld_32x32b_x32(lane_base, va);
          tmem_ld_wait(va);
#pragma unroll 1
          for (int ch = 0; ch < kChunks; ch += 2) {
            tmem_ld_32x32b_x32(lane_base + static_cast<uint32_t>((ch + 1) * 32), vb);
            drain_chunk(va, l, g > 0, c, reinterpret_cast<uint4*>(dst + ch * 32));
            tmem_ld_wait(vb);
            if (ch + 2 < kChunks) {
              tmem_ld_32x32b_x32(lane_base + static_cast<uint32_t>((ch + 2) * 32), va);
            } else {
              tc_fence_before();
              __syncwarp();
              if (lane == 0) mbar_arrive_cluster(acc_empty_r0[buf]);
            }
            drain_chunk(vb, l, g > 0, c, reinterpret_cast<uint4*>(dst + (ch + 1) * 32));
            if (ch + 2 < kChunks) tmem_ld_wait(va);
          }
        }
      }
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

// ---------------------------------------------------------------------------------------------
// Reconstruction kernel: residue planes -> C
// ---------------------------------------------------------------------------------------------
// C' of one element from its NM residue bytes (c + 128, byte e of each word w[l]) as a double.
template <int NM, int NL>
__device__ __forceinline__ double reconstruct(const uint32_t (&w)[NM], int e, const Consts& c) {
  double L[NL];
#pragma unroll
  for (int k = 0; k < NL; ++k) L[k] = c.Kc[k];
#pragma unroll
  for (int l = 0; l < NM; ++l) {
    const uint32_t u = __byte_perm(w[l], 0u, 0x4440u | static_cast<uint32_t>(e));  // byte e, zero-extended
    const double ud = __hiloint2double(0x43300000, static_cast<int>(u)) - 4503599627370496.0;  // exact u
#pragma unroll
    for (int k = 0; k < NL; ++k) L[k] = __fma_rn(ud, c.P[l][k], L[k]);
  }
  const double s = __fma_rn(L[NL - 1], c.f_hi, __dmul_rn(L[NL - 2], c.f_lo));
  const double Q = rint(s);
  double t = __fma_rn(-Q, c.Mk[NL - 1], L[NL - 1]);
  const double base = __longlong_as_double(static_cast<long long>(1023 + c.w) << 52);
#pragma unroll
  for (int k = NL - 2; k >= 0; --k) t = __fma_rn(t, base, __fma_rn(-Q, c.Mk[k], L[k]));
  return t;
}

// One thread per four consecutive columns of a row (blockIdx.x: a block of 4 * blockDim.x columns,
// blockIdx.y: rows with a grid stride): 4-byte loads from each residue plane and 16-byte loads /
// stores of C, coalesced across the warp (128 columns of a row).
template <int NM>
__global__ void __launch_bounds__(256) crt_recon_kernel(const uint8_t* __restrict__ res, int64_t plane, int64_t Np,
                                                        double* __restrict__ C, int64_t M, int64_t N, int64_t ldc,
                                                        const int* __restrict__ ea, const int* __restrict__ eb,
                                                        double alpha, double beta) {
  constexpr int NL = limbs_for(NM);
  const Consts& c = c_table[NM - kMinMod];
  const int64_t j0 = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) * 4;
  if (j0 >= N) return;
  for (int64_t i = blockIdx.y; i < M; i += gridDim.y) {
    uint32_t w[NM];
    const uint8_t* src = res + i * Np + j0;
#pragma unroll
    for (int l = 0; l < NM; ++l) w[l] = __ldcs(reinterpret_cast<const unsigned int*>(src + l * plane));
    double* crow = C + i * ldc;
    const bool vec = j0 + 4 <= N && (reinterpret_cast<uintptr_t>(crow + j0) & 15) == 0;
    double c0[4] = {0.0, 0.0, 0.0, 0.0};
    if (beta != 0.0) {
      if (vec) {
        const double2 x = __ldcs(reinterpret_cast<const double2*>(crow + j0));
        const double2 y = __ldcs(reinterpret_cast<const double2*>(crow + j0) + 1);
        c0[0] = x.x; c0[1] = x.y; c0[2] = y.x; c0[3] = y.y;
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (j0 + e < N) c0[e] = crow[j0 + e];
      }
    }
    const int sr = ea[i];
    int sc[4];
    if (j0 + 4 <= N) {
      const int4 t4 = *reinterpret_cast<const int4*>(eb + j0);
      sc[0] = t4.x; sc[1] = t4.y; sc[2] = t4.z; sc[3] = t4.w;
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) sc[e] = j0 + e < N ? eb[j0 + e] : 0;
    }
    // C' 2^-s_i 2^-s_j: with both factors in the double range this is two exact-factor
    // multiplications, which is what scale_pow2 does there; scale_pow2 takes the rest
    const int es = -sr;
    const bool row_fast = sr != kSentinel && es >= -1022 && es <= 1023;
    const double rs = pow2i(row_fast ? es : 0);
    double out[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (sr == kSentinel || sc[e] == kSentinel) {
        out[e] = __longlong_as_double(0x7ff8000000000000ll);
      } else {
        const double t = reconstruct<NM, NL>(w, e, c);
        const int et = -sc[e];
        const double tv = (row_fast && et >= -1022 && et <= 1023) ? __dmul_rn(__dmul_rn(t, rs), pow2i(et))
                                                                   : scale_pow2(scale_pow2(t, es), et);
        out[e] = (beta != 0.0) ? fma(alpha, tv, __dmul_rn(beta, c0[e])) : __dmul_rn(alpha, tv);
      }
    }
    if (vec) {
      __stcs(reinterpret_cast<double2*>(crow + j0), make_double2(out[0], out[1]));
      __stcs(reinterpret_cast<double2*>(crow + j0) + 1, make_double2(out[2], out[3]));
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (j0 + e < N) crow[j0 + e] = out[e];
    }
  }
}

// C = beta C0 (alpha * 0 when beta == 0) for K = 0, with the epilogue's roundings.
__global__ void k0_kernel(double* C, int64_t M, int64_t N, int64_t ldc, double alpha, double beta) {
  const int64_t n = M * N;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double* c = C + (i / N) * ldc + (i % N);
    *c = beta != 0.0 ? fma(alpha, 0.0, __dmul_rn(beta, *c)) : __dmul_rn(alpha, 0.0);
  }
}

// ---------------------------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------------------------
// Tile width of the product (LIBTHOM_CRT_TILE = 256 / 512 forces one): the smaller time of whole
// waves of (modulus, tile) work items over `clusters` CTA pairs, a 512-wide tile taking 0.92 of the time of two
// 256-wide ones (measured at 8192^3: less operand traffic per product) but filling fewer pairs when the
// problem has few tiles (2048 x 2048: 32 tiles of 512 against 64 of 256 for 74 pairs).
int tile_width(int64_t M, int64_t N, int moduli, int clusters) {
  static const int forced = [] {
    const char* e = getenv("LIBTHOM_CRT_TILE");
    const int v = e != nullptr ? atoi(e) : 0;
    return (v == 256 || v == 512) ? v : 0;
  }();
  if (forced != 0) return forced;
  const int64_t tm = ceil_div(M, 2 * kBM);
  auto cost = [&](int bn, double eff) {
    return static_cast<double>(ceil_div(moduli * tm * ceil_div(N, bn), std::max(clusters, 1))) * bn * eff;
  };
  return cost(512, 0.92) < cost(256, 1.0) ? 512 : 256;
}

int raster_group() {
  static const int g = [] {
    const char* e = getenv("LIBTHOM_CRT_GROUP");
    const int v = e != nullptr ? atoi(e) : 0;
    return (v >= 1 && v <= 64) ? v : 8;
  }();
  return g;
}

// Chunk statistics and shifts of rows 0..M-1 of A (row stride K) and of the columns of B (row
// stride N); either side may be empty. `ec_a` / `sc_a` hold ncha entries per row, `ec_b` / `sc_b`
// nchb per column.
int scale(const double* A, int64_t M, const double* B, int64_t N, int64_t K, const Layout& L, int* ec_a,
          unsigned long long* sc_a, int* ec_b, unsigned long long* sc_b, int* sh_a, int* sh_b, const Consts& c,
          cudaStream_t stream) {
  if (M + N == 0) return LT_OK;
  const int64_t row_blocks = ceil_div(M * L.ncha, 8);
  const int64_t blocks = row_blocks + ceil_div(N, 32) * L.nchb;
  crt_stats_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(A, M, K, L.ncha, B, N, N, L.nchb, K, row_blocks,
                                                                       ec_a, sc_a, ec_b, sc_b);
  LT_CUDA_TRY(cudaGetLastError());
  crt_shift_kernel<<<static_cast<unsigned>(ceil_div((M + N) * 32, 256)), 256, 0, stream>>>(
      ec_a, sc_a, M, L.ncha, ec_b, sc_b, N, L.nchb, c.ta, c.tb, sh_a, sh_b);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

// Residue planes of rows 0..M-1 of A (row stride K) into `ra` (plane stride `plane`), and of the
// columns of B (row stride N) into `rb`, for NM moduli, with the shifts `scale` wrote.
template <int NM>
int split_rows_n(const double* A, int64_t M, int64_t K, int64_t Kp, const int* shifts, int8_t* ra, int64_t plane,
                 cudaStream_t stream) {
  const dim3 grid(static_cast<unsigned>(ceil_div(M, 8)), static_cast<unsigned>(ceil_div(Kp, 512)));
  crt_split_rows_kernel<NM><<<grid, 256, 0, stream>>>(A, M, K, K, Kp, shifts, ra, plane);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

template <int NM>
int split_cols_n(const double* B, int64_t K, int64_t N, int64_t Kp, const int* shifts, int8_t* rb, int64_t plane,
                 cudaStream_t stream) {
  const dim3 grid(static_cast<unsigned>(ceil_div(N, 32)), static_cast<unsigned>(Kp / kBK));
  crt_split_cols_kernel<NM><<<grid, 256, 0, stream>>>(B, K, N, N, Kp, shifts, rb, plane);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

#define LT_CRT_DISPATCH(n, CALL)                                                                             \
  switch (n) {                                                                                              \
    case 8: return CALL(8); case 9: return CALL(9); case 10: return CALL(10); case 11: return CALL(11);     \
    case 12: return CALL(12); case 13: return CALL(13); case 14: return CALL(14); case 15: return CALL(15); \
    case 16: return CALL(16); case 17: return CALL(17); case 18: return CALL(18); case 19: return CALL(19); \
    case 20: return CALL(20);                                                                               \
    default: return set_error(LT_ERR_INVALID_ARGUMENT, "modulus count %d outside [%d, %d]", n, kMinMod, kMaxMod); \
  }

int split_rows(int n, const double* A, int64_t M, int64_t K, int64_t Kp, const int* shifts, int8_t* ra, int64_t plane,
               cudaStream_t stream) {
#define LT_CALL(NM) split_rows_n<NM>(A, M, K, Kp, shifts, ra, plane, stream)
  LT_CRT_DISPATCH(n, LT_CALL)
#undef LT_CALL
}

int split_cols(int n, const double* B, int64_t K, int64_t N, int64_t Kp, const int* shifts, int8_t* rb, int64_t plane,
               cudaStream_t stream) {
#define LT_CALL(NM) split_cols_n<NM>(B, K, N, Kp, shifts, rb, plane, stream)
  LT_CRT_DISPATCH(n, LT_CALL)
#undef LT_CALL
}

struct Scratch {  // the workspace's arrays
  int *ec_a, *ec_b, *ea, *eb;
  unsigned long long *sc_a, *sc_b;
  int8_t *ra, *rb;
};

Scratch scratch(uint8_t* ws, const Layout& L) {
  Scratch s;
  s.ec_a = reinterpret_cast<int*>(ws + L.off_eca);
  s.sc_a = reinterpret_cast<unsigned long long*>(ws + L.off_sca);
  s.ec_b = reinterpret_cast<int*>(ws + L.off_ecb);
  s.sc_b = reinterpret_cast<unsigned long long*>(ws + L.off_scb);
  s.ea = reinterpret_cast<int*>(ws + L.off_ea);
  s.eb = reinterpret_cast<int*>(ws + L.off_eb);
  s.ra = reinterpret_cast<int8_t*>(ws + L.off_ra);
  s.rb = reinterpret_cast<int8_t*>(ws + L.off_rb);
  return s;
}

int split(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int n, void* workspace,
          size_t workspace_bytes, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  const Layout L = layout_for(M, N, K, n);
  if (workspace_bytes < L.total) return set_error(LT_ERR_NO_MEMORY, "CRT workspace too small");
  if (K == 0) return LT_OK;
  LT_TRY(ensure_table(ctx->device));
  const Consts c = make_consts(n);
  const Scratch w = scratch(static_cast<uint8_t*>(workspace), L);
  LT_TRY(scale(A, M, B, N, K, L, w.ec_a, w.sc_a, w.ec_b, w.sc_b, w.ea, w.eb, c, stream));
  LT_TRY(split_rows(n, A, M, K, L.Kp, w.ea, w.ra, M * L.Kp, stream));
  return split_cols(n, B, K, N, L.Kp, w.eb, w.rb, N * L.Kp, stream);
}

// One product stage over rows 0..M-1 of residue planes `ra` (plane stride a_plane) against all N
// columns of `rb`, into the C residue planes at `res` (plane stride res_plane, row pitch Np, whole
// 256 x 256 tiles) and then, reconstructed, into C (row stride ldc).
struct ProductArgs {
  const int8_t* ra;
  int64_t a_plane;
  const int8_t* rb;
  int64_t b_plane;
  int64_t Kp;
  uint8_t* res;
  int64_t res_plane, Np;
  double* C;
  int64_t M, N, ldc, K;
  const int* ea;  // row shifts of A
  const int* eb;  // column shifts of B
  double alpha, beta;
  int n;
};

template <int NM, int BN>
int launch_product_n(const CUtensorMap& tmA, const CUtensorMap& tmB, const Problem& p, const Consts& c, double* C,
                     int64_t M, int64_t N, int64_t ldc, const int* ea, const int* eb, double alpha, double beta,
                     DeviceContext* ctx,
                     cudaStream_t stream, bool do_multiply, bool do_reconstruct) {
  if (c.nl != limbs_for(NM)) return set_error(LT_ERR_UNSUPPORTED, "CRT limb count %d, kernel built for %d", c.nl, limbs_for(NM));
  static std::once_flag once[64];
  static cudaError_t attr_err[64];
  static int max_clusters[64];
  auto config = [&](cudaLaunchConfig_t* cfg, cudaLaunchAttribute* attr, unsigned grid) {
    *cfg = cudaLaunchConfig_t{};
    cfg->gridDim = dim3(grid);
    cfg->blockDim = dim3(kThreads);
    cfg->dynamicSmemBytes = Tile<BN>::kSmem;
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
        cudaFuncSetAttribute(crt_pair_kernel<NM, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, Tile<BN>::kSmem);
    if (attr_err[ctx->device] != cudaSuccess) return;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute attr;
    config(&cfg, &attr, static_cast<unsigned>(ctx->sm_count & ~1));
    attr_err[ctx->device] = cudaOccupancyMaxActiveClusters(&max_clusters[ctx->device], crt_pair_kernel<NM, BN>, &cfg);
  });
  LT_CUDA_TRY(attr_err[ctx->device]);
  const int64_t items = static_cast<int64_t>(p.tiles_m) * p.tiles_n * NM;  // (modulus, tile) work items
  const int64_t clusters = std::min<int64_t>(std::min<int64_t>(items, max_clusters[ctx->device]), ctx->sm_count / 2);
  if (clusters <= 0) return set_error(LT_ERR_UNSUPPORTED, "no pair of CTAs of the CRT product kernel fits");
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute attr;
  config(&cfg, &attr, static_cast<unsigned>(2 * clusters));
  if (do_multiply) LT_CUDA_TRY(cudaLaunchKernelEx(&cfg, crt_pair_kernel<NM, BN>, tmA, tmB, p, ctx->status));
  if (do_reconstruct) {
    // 4 columns per thread; a narrow C takes narrower blocks so few threads idle past column N
    const int64_t quads = ceil_div(N, 4);
    const int64_t tx = std::min<int64_t>(256, round_up(quads, 32));
    const int64_t bx = ceil_div(quads, tx);
    const int64_t by = std::min<int64_t>(M, std::max<int64_t>(1, 8 * ctx->sm_count * (256 / tx) / bx));
    crt_recon_kernel<NM><<<dim3(static_cast<unsigned>(bx), static_cast<unsigned>(by)), static_cast<unsigned>(tx), 0,
                           stream>>>(p.res, p.plane, p.Np, C, M, N, ldc, ea, eb, alpha, beta);
    LT_CUDA_TRY(cudaGetLastError());
  }
  return LT_OK;
}

int run_product(const ProductArgs& a, DeviceContext* ctx, cudaStream_t stream, bool do_multiply, bool do_reconstruct) {
  LT_TRY(ensure_table(ctx->device));
  CUtensorMap tmA, tmB;
  LT_TRY(make_tmap_3d(&tmA, a.ra, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, a.n, a.M, a.Kp, a.Kp, a.a_plane, kBM, kBK,
                      CU_TENSOR_MAP_SWIZZLE_128B));
  LT_TRY(make_tmap_3d(&tmB, a.rb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, a.n, a.N, a.Kp, a.Kp, a.b_plane, kBN / 2, kBK,
                      CU_TENSOR_MAP_SWIZZLE_128B));
  Problem p;
  p.res = a.res;
  p.plane = a.res_plane;
  p.Np = a.Np;
  p.tiles_m = static_cast<int>(ceil_div(a.M, 2 * kBM));
  p.bn = tile_width(a.M, a.N, a.n, ctx->sm_count / 2);
  p.tiles_n = static_cast<int>(ceil_div(a.N, p.bn));
  p.ksteps = static_cast<int>(a.Kp / kBK);
  p.kgroups = static_cast<int>(ceil_div(p.ksteps, kGroupSteps));
  p.group = raster_group();
  const Consts c = make_consts(a.n);
#define LT_CALL(NM)                                                                                              \
  (p.bn == 512 ? launch_product_n<NM, 512>(tmA, tmB, p, c, a.C, a.M, a.N, a.ldc, a.ea, a.eb, a.alpha, a.beta, ctx, \
                                           stream, do_multiply, do_reconstruct)                                   \
               : launch_product_n<NM, 256>(tmA, tmB, p, c, a.C, a.M, a.N, a.ldc, a.ea, a.eb, a.alpha, a.beta, ctx, \
                                           stream, do_multiply, do_reconstruct))
  LT_CRT_DISPATCH(a.n, LT_CALL)
#undef LT_CALL
}

// The products into the residue planes of C (do_multiply) and the reconstruction of C from them
// (do_reconstruct); both for the whole product stage.
int product(double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int n, const void* workspace,
            size_t workspace_bytes, cudaStream_t stream, bool do_multiply = true, bool do_reconstruct = true) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  const Layout L = layout_for(M, N, K, n);
  if (workspace_bytes < L.total) return set_error(LT_ERR_NO_MEMORY, "CRT workspace too small");
  if (K == 0) {
    if (!do_reconstruct) return LT_OK;
    const int64_t total = M * N;
    const int64_t blocks = std::min<int64_t>(ceil_div(total, 256), 4 * ctx->sm_count);
    k0_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(C, M, N, N, alpha, beta);
    LT_CUDA_TRY(cudaGetLastError());
    return LT_OK;
  }
  const uint8_t* ws = static_cast<const uint8_t*>(workspace);
  ProductArgs a;
  a.ra = reinterpret_cast<const int8_t*>(ws + L.off_ra);
  a.a_plane = M * L.Kp;
  a.rb = reinterpret_cast<const int8_t*>(ws + L.off_rb);
  a.b_plane = N * L.Kp;
  a.Kp = L.Kp;
  a.res = const_cast<uint8_t*>(ws + L.off_rc);
  a.res_plane = L.Mp * L.Np;
  a.Np = L.Np;
  a.C = C;
  a.M = M;
  a.N = N;
  a.ldc = N;
  a.K = K;
  a.ea = reinterpret_cast<const int*>(ws + L.off_ea);
  a.eb = reinterpret_cast<const int*>(ws + L.off_eb);
  a.alpha = alpha;
  a.beta = beta;
  a.n = n;
  return run_product(a, ctx, stream, do_multiply, do_reconstruct);
}

// ---------------------------------------------------------------------------------------------
// Host-resident operands (lt_dgemm_ozaki_crt_host): B is copied, its shifts and residues taken;
// then row panels of A (and of C0 when beta != 0), whole 256-row pair blocks each, are copied on one
// stream while earlier panels are split, multiplied and reconstructed on the caller's stream, and
// finished panels of C go back on a third, so the PCIe copies overlap the kernels. Each panel's rows
// land where run() puts them and go through the same arithmetic: C is bit-identical to
// lt_dgemm_ozaki_crt.
// ---------------------------------------------------------------------------------------------
int host_panels() {
  static const int n = [] {
    const char* e = getenv("LIBTHOM_OZAKI_HOST_PANELS");
    const int v = e != nullptr ? atoi(e) : 0;
    return (v >= 1 && v <= 64) ? v : 16;
  }();
  return n;
}

int host_run(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta,
             int n, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  const Layout L = layout_for(M, N, K, n);
  const size_t off_a = round_up(static_cast<int64_t>(L.total), 256);
  const size_t off_b = off_a + round_up(8 * M * K, 256);
  const size_t off_c = off_b + round_up(8 * K * N, 256);
  const size_t total = off_c + 8 * static_cast<size_t>(M) * N;
  void* base = nullptr;
  LT_TRY(ensure_workspace(ctx, total, &base));
  LT_TRY(ensure_table(ctx->device));
  uint8_t* ws = static_cast<uint8_t*>(base);
  const Scratch w = scratch(ws, L);
  auto* Ad = reinterpret_cast<double*>(ws + off_a);
  auto* Bd = reinterpret_cast<double*>(ws + off_b);
  auto* Cd = reinterpret_cast<double*>(ws + off_c);
  const Consts c = make_consts(n);

  const int64_t panel = std::max<int64_t>(2 * kBM, round_up(ceil_div(M, host_panels()), 2 * kBM));
  const int64_t npanels = ceil_div(M, panel);
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
    if (K > 0) cuda(cudaMemcpyAsync(Bd, B, 8 * static_cast<size_t>(K) * N, cudaMemcpyHostToDevice, h2d), "copy B");
    cuda(cudaEventRecord(e_b, h2d), "record");
    cuda(cudaStreamWaitEvent(stream, e_b, 0), "wait");
  }
  if (rc == LT_OK && K > 0)
    rc = scale(nullptr, 0, Bd, N, K, L, nullptr, nullptr, w.ec_b, w.sc_b, nullptr, w.eb, c, stream);
  if (rc == LT_OK && K > 0) rc = split_cols(n, Bd, K, N, L.Kp, w.eb, w.rb, N * L.Kp, stream);
  for (int64_t i = 0; i < npanels && rc == LT_OK; ++i) {
    const int64_t r0 = i * panel, rows = std::min(panel, M - r0);
    cudaEvent_t e_in = ev[2 * i], e_out = ev[2 * i + 1];
    if (K > 0)
      cuda(cudaMemcpyAsync(Ad + r0 * K, A + r0 * K, 8 * static_cast<size_t>(rows) * K, cudaMemcpyHostToDevice, h2d),
           "copy A");
    if (beta != 0.0)
      cuda(cudaMemcpyAsync(Cd + r0 * N, C + r0 * N, 8 * static_cast<size_t>(rows) * N, cudaMemcpyHostToDevice, h2d),
           "copy C0");
    cuda(cudaEventRecord(e_in, h2d), "record");
    cuda(cudaStreamWaitEvent(stream, e_in, 0), "wait");
    if (rc != LT_OK) break;
    if (K == 0) {
      const int64_t blocks = std::min<int64_t>(ceil_div(rows * N, 256), 4 * ctx->sm_count);
      k0_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(Cd + r0 * N, rows, N, N, alpha, beta);
      cuda(cudaGetLastError(), "k0 kernel");
    } else {
      rc = scale(Ad + r0 * K, rows, nullptr, 0, K, L, w.ec_a + r0 * L.ncha, w.sc_a + r0 * L.ncha, nullptr, nullptr,
                 w.ea + r0, nullptr, c, stream);
      if (rc == LT_OK) rc = split_rows(n, Ad + r0 * K, rows, K, L.Kp, w.ea + r0, w.ra + r0 * L.Kp, M * L.Kp, stream);
      if (rc != LT_OK) break;
      ProductArgs a;
      a.ra = w.ra + r0 * L.Kp;
      a.a_plane = M * L.Kp;
      a.rb = w.rb;
      a.b_plane = N * L.Kp;
      a.Kp = L.Kp;
      a.res = ws + L.off_rc + r0 * L.Np;
      a.res_plane = L.Mp * L.Np;
      a.Np = L.Np;
      a.C = Cd + r0 * N;
      a.M = rows;
      a.N = N;
      a.ldc = N;
      a.K = K;
      a.ea = w.ea + r0;
      a.eb = w.eb;
      a.alpha = alpha;
      a.beta = beta;
      a.n = n;
      rc = run_product(a, ctx, stream, true, true);
      if (rc != LT_OK) break;
    }
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

size_t workspace_size(int64_t M, int64_t N, int64_t K, int n) { return layout_for(M, N, K, n).total; }

}  // namespace crt
}  // namespace lt

// ---------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------
namespace {

int check_args(const double* A, const double* B, const double* C, int64_t M, int64_t N, int64_t K, int n) {
  if (M < 0 || N < 0 || K < 0 || M > 0x7fffffff || N > 0x7fffffff || K > 0x7fffffff)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "bad dimensions");
  if ((M > 0 && K > 0 && A == nullptr) || (K > 0 && N > 0 && B == nullptr) || (M > 0 && N > 0 && C == nullptr))
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "null matrix pointer");
  if (((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(C)) & 7) != 0)
    return lt::set_error(LT_ERR_UNALIGNED, "matrix pointers must be 8-byte aligned");
  if (n < LT_OZAKI_CRT_MIN_MODULI || n > LT_OZAKI_CRT_MAX_MODULI)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "modulus count %d outside [%d, %d]", n, LT_OZAKI_CRT_MIN_MODULI,
                         LT_OZAKI_CRT_MAX_MODULI);
  if (K > 65535ll * lt::crt::kBK)  // the residue split's grid covers K in 128-wide blocks (gridDim.y)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "K = %lld above the CRT form's limit %lld", static_cast<long long>(K),
                         65535ll * lt::crt::kBK);
  return LT_OK;
}

int check_ws(int64_t M, int64_t N, int64_t K, int n, const void* workspace, size_t workspace_bytes) {
  const size_t need = lt::crt::workspace_size(M, N, K, n);
  if (workspace == nullptr || workspace_bytes < need)
    return lt::set_error(LT_ERR_NO_MEMORY, "workspace of %zu bytes given, %zu needed", workspace_bytes, need);
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
    return lt::set_error(LT_ERR_UNALIGNED, "workspace must be 256-byte aligned");
  return LT_OK;
}

}  // namespace

extern "C" {

size_t lt_ozaki_crt_workspace_size(int64_t M, int64_t N, int64_t K, int moduli) {
  if (M < 0 || N < 0 || K < 0 || moduli < LT_OZAKI_CRT_MIN_MODULI || moduli > LT_OZAKI_CRT_MAX_MODULI) return 0;
  return lt::crt::workspace_size(M, N, K, moduli);
}

int lt_ozaki_crt_info(int moduli, int* ta, int* tb, int* moduli_out) {
  if (moduli < LT_OZAKI_CRT_MIN_MODULI || moduli > LT_OZAKI_CRT_MAX_MODULI)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "modulus count %d outside [%d, %d]", moduli,
                         LT_OZAKI_CRT_MIN_MODULI, LT_OZAKI_CRT_MAX_MODULI);
  const lt::crt::Consts c = lt::crt::make_consts(moduli);
  if (ta != nullptr) *ta = c.ta;
  if (tb != nullptr) *tb = c.tb;
  if (moduli_out != nullptr)
    for (int l = 0; l < moduli; ++l) moduli_out[l] = c.m[l];
  return lt::ok();
}

int lt_ozaki_crt_split(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int moduli, void* workspace,
                       size_t workspace_bytes, void* stream) {
  LT_TRY(check_args(A, B, reinterpret_cast<const double*>(8), M, N, K, moduli));
  LT_TRY(check_ws(M, N, K, moduli, workspace, workspace_bytes));
  if (M == 0 || N == 0) return lt::ok();
  LT_TRY(lt::crt::split(A, B, M, N, K, moduli, workspace, workspace_bytes, lt::as_stream(stream)));
  return lt::ok();
}

int lt_ozaki_crt_product(double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int moduli,
                         const void* workspace, size_t workspace_bytes, void* stream) {
  LT_TRY(check_args(reinterpret_cast<const double*>(8), reinterpret_cast<const double*>(8), C, M, N, K, moduli));
  LT_TRY(check_ws(M, N, K, moduli, workspace, workspace_bytes));
  if (M == 0 || N == 0) return lt::ok();
  LT_TRY(lt::crt::product(C, M, N, K, alpha, beta, moduli, workspace, workspace_bytes, lt::as_stream(stream)));
  return lt::ok();
}

int lt_ozaki_crt_multiply(int64_t M, int64_t N, int64_t K, int moduli, void* workspace, size_t workspace_bytes,
                          void* stream) {
  LT_TRY(check_args(reinterpret_cast<const double*>(8), reinterpret_cast<const double*>(8),
                    reinterpret_cast<const double*>(8), M, N, K, moduli));
  LT_TRY(check_ws(M, N, K, moduli, workspace, workspace_bytes));
  if (M == 0 || N == 0) return lt::ok();
  LT_TRY(lt::crt::product(nullptr, M, N, K, 1.0, 0.0, moduli, workspace, workspace_bytes, lt::as_stream(stream), true,
                          false));
  return lt::ok();
}

int lt_ozaki_crt_reconstruct(double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int moduli,
                             const void* workspace, size_t workspace_bytes, void* stream) {
  LT_TRY(check_args(reinterpret_cast<const double*>(8), reinterpret_cast<const double*>(8), C, M, N, K, moduli));
  LT_TRY(check_ws(M, N, K, moduli, workspace, workspace_bytes));
  if (M == 0 || N == 0) return lt::ok();
  LT_TRY(lt::crt::product(C, M, N, K, alpha, beta, moduli, workspace, workspace_bytes, lt::as_stream(stream), false,
                          true));
  return lt::ok();
}

int lt_dgemm_ozaki_crt_host(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                            double alpha, double beta, int moduli, void* stream) {
  LT_TRY(check_args(A, B, C, M, N, K, moduli));
  if (M == 0 || N == 0) return lt::ok();
  LT_TRY(lt::crt::host_run(A, B, C, M, N, K, alpha, beta, moduli, lt::as_stream(stream)));
  return lt::ok();
}

int lt_dgemm_ozaki_crt_ws(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                          double beta, int moduli, void* workspace, size_t workspace_bytes, void* stream) {
  LT_TRY(check_args(A, B, C, M, N, K, moduli));
  LT_TRY(check_ws(M, N, K, moduli, workspace, workspace_bytes));
  if (M == 0 || N == 0) return lt::ok();
  const cudaStream_t s = lt::as_stream(stream);
  LT_TRY(lt::crt::split(A, B, M, N, K, moduli, workspace, workspace_bytes, s));
  LT_TRY(lt::crt::product(C, M, N, K, alpha, beta, moduli, workspace, workspace_bytes, s));
  return lt::ok();
}

int lt_dgemm_ozaki_crt(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                       double beta, int moduli, void* stream) {
  LT_TRY(check_args(A, B, C, M, N, K, moduli));
  if (M == 0 || N == 0) return lt::ok();
  lt::DeviceContext* ctx = lt::context();
  if (ctx == nullptr) return lt::last_error();
  const size_t bytes = lt::crt::workspace_size(M, N, K, moduli);
  void* ws = nullptr;
  LT_TRY(lt::ensure_workspace(ctx, bytes, &ws));
  const cudaStream_t s = lt::as_stream(stream);
  LT_TRY(lt::crt::split(A, B, M, N, K, moduli, ws, bytes, s));
  LT_TRY(lt::crt::product(C, M, N, K, alpha, beta, moduli, ws, bytes, s));
  return lt::ok();
}

}  // extern "C"
