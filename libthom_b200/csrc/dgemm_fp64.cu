// dgemm_fp64.cu — host launchers and configuration registry of the native FP64 DGEMM.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "dgemm_fp64.cuh"
#include "lt_runtime.cuh"
#include "lt_internal.h"

namespace lt {
namespace fp64 {

namespace {

struct Schedule {
  int splits = 1;        // K ranges per tile (1: none)
  bool streamk = false;  // stream-K (splits == 1)
  double t = 0.0;        // modelled seconds
};

// LIBTHOM_FP64_STREAMK=0 turns the stream-K schedule off (the K split and whole tiles remain).
bool streamk_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("LIBTHOM_FP64_STREAMK");
    return e == nullptr || std::atoi(e) != 0;
  }();
  return on;
}

// Schedule of one launch for tile counts that fill the GPU poorly (wave quantisation), modelled
// at the FP64 tensor rate (t_kb: one k-block of one tile on one SM) with a pipeline fill and
// epilogue of ~6 k-blocks per tile:
//  * K split S in 2..4 (ranges of >= 32 k-blocks): waves(S) x (k-blocks per range + 6), plus the
//    reduction's traffic;
//  * stream-K: the tiles x k-blocks iterations shared evenly by `cap` CTAs; each CTA pays one fill
//    and ~3 k-blocks per extra tile its range touches, plus the partial-sum slots (mostly L2
//    traffic) and the fix-up launch.
// A schedule replaces no split only when it is at least 3 % faster (stream-K with 256 or more
// k-blocks per tile: 0.5 %). Stream-K is considered only
// while enabled (LIBTHOM_FP64_STREAMK), so turning it off falls back to the best remaining schedule.
Schedule choose_schedule(int64_t tiles, int64_t cap, int64_t M, int64_t N, int64_t K, int bm, int bn) {
  Schedule best;
  const int64_t nkb = (K + 15) / 16;
  if (tiles <= 0 || nkb <= 0 || cap <= 0) return best;
  const double t_kb = 2.0 * bm * bn * 16 / (128.0 * 1.9e9);
  best.t = static_cast<double>((tiles + cap - 1) / cap) * static_cast<double>(nkb + 6) * t_kb;
  const double plain = best.t;
  for (int S = 2; S <= 4 && nkb >= 64; ++S) {
    const int64_t per = (nkb + S - 1) / S;
    if (per < 32) break;
    const int64_t waves = (tiles * S + cap - 1) / cap;
    double t = static_cast<double>(waves) * static_cast<double>(per + 6) * t_kb;
    t += (S + 2) * 8.0 * static_cast<double>(M) * static_cast<double>(N) / 6.0e12;
    if (t < std::min(best.t, plain * 0.97)) best = Schedule{S, false, t};
  }
  const int64_t total = tiles * nkb;
  if (total >= 2 && streamk_enabled()) {
    const int64_t G = std::min(cap, total);
    const int64_t per = (total + G - 1) / G;
    const int64_t touched = 1 + (per + nkb - 1) / nkb;
    double t = static_cast<double>(per + 6 + 3 * (touched - 1)) * t_kb;
    t += 4.0 * G * bm * bn * 8.0 / 20.0e12 + 3.0e-6;
    // With 256 or more k-blocks per tile the fill is amortised and the model is close (8192^3:
    // modelled 0.983 of whole tiles, measured 0.988), so a smaller margin suffices there.
    const double margin = nkb >= 256 ? 0.995 : 0.97;
    if (t < std::min(best.t, plain * margin)) best = Schedule{1, true, t};
  }
  return best;
}

template <class Cfg>
// `scratch` (host side only, kept out of the kernels' Params, whose size costs registers there): the
// caller's scratch for the K split / stream-K partial sums, or a query of the bytes needed; null: the
// per-device cache.
int launch(const Params& p0, cudaStream_t stream, DeviceContext* ctx, const ScratchUse* scratch) {
  Params p = p0;
  p.status = ctx->status;
  CUtensorMap tmA, tmB;
  memset(&tmA, 0, sizeof tmA);
  memset(&tmB, 0, sizeof tmB);
  if (Cfg::kTMA) {
    if (!tma_compatible(p.A, p.B, p.ldb, p.lda))
      return set_error(LT_ERR_UNALIGNED, "TMA configuration needs 16-byte aligned A/B and even row strides");
    LT_TRY(make_tmap_2d(&tmA, p.A, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, static_cast<uint64_t>(p.M),
                        static_cast<uint64_t>(p.K), static_cast<uint64_t>(p.lda) * 8, Cfg::BM, 16));
    LT_TRY(make_tmap_2d(&tmB, p.B, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, static_cast<uint64_t>(p.K),
                        static_cast<uint64_t>(p.N), static_cast<uint64_t>(p.ldb) * 8, 16, 16));
  }
  static std::once_flag once[64];
  static int occupancy[64];
  static cudaError_t attr_err[64];
  std::call_once(once[ctx->device], [&] {
    attr_err[ctx->device] = cudaFuncSetAttribute(dgemm_fp64_kernel<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 Cfg::SMEM_BYTES);
    int occ = 0;
    if (attr_err[ctx->device] == cudaSuccess)
      attr_err[ctx->device] = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, dgemm_fp64_kernel<Cfg>,
                                                                            Cfg::THREADS, Cfg::SMEM_BYTES);
    occupancy[ctx->device] = occ > 0 ? occ : 1;
  });
  LT_CUDA_TRY(attr_err[ctx->device]);
  const int64_t tiles_m = (p.M + Cfg::BM - 1) / Cfg::BM, tiles_n = (p.N + Cfg::BN - 1) / Cfg::BN;
  const int64_t tiles = tiles_m * tiles_n;
  const int64_t cap = static_cast<int64_t>(ctx->sm_count) * occupancy[ctx->device];
  const int64_t nkb = (p.K + Cfg::BK - 1) / Cfg::BK;
  const Schedule sched = choose_schedule(tiles, cap, p.M, p.N, p.K, Cfg::BM, Cfg::BN);
  p.splits = sched.splits;
  p.streamk = sched.streamk ? 1 : 0;
  p.W = nullptr;
  int64_t grid = tiles * p.splits < cap ? tiles * p.splits : cap;
  if (p.streamk) grid = std::min(cap, tiles * nkb);
  size_t bytes = 0;
  if (p.splits > 1 || p.streamk)
    bytes = p.streamk ? static_cast<size_t>(2 * grid) * Cfg::BM * Cfg::BN * sizeof(double)
                      : static_cast<size_t>(p.splits) * p.M * p.N * sizeof(double);
  if (scratch != nullptr && scratch->query != nullptr) {
    *scratch->query = bytes;
    return LT_OK;
  }
  if (bytes > 0) {
    void* w = scratch != nullptr ? scratch->ptr : nullptr;
    if (w != nullptr && scratch->bytes < bytes)
      return set_error(LT_ERR_NO_MEMORY, "FP64 scratch of %zu bytes given, %zu needed", scratch->bytes, bytes);
    if (w == nullptr) LT_TRY(ensure_splitk_workspace(ctx, bytes, &w));
    p.W = static_cast<double*>(w);
  }
  dgemm_fp64_kernel<Cfg><<<static_cast<unsigned>(grid), Cfg::THREADS, Cfg::SMEM_BYTES, stream>>>(tmA, tmB, p);
  LT_CUDA_TRY(cudaGetLastError());
  if (p.streamk) {
    const int64_t blocks = std::min<int64_t>(tiles, static_cast<int64_t>(ctx->sm_count) * 4);
    streamk_fixup_kernel<Cfg::BM, Cfg::BN><<<static_cast<unsigned>(blocks), kFixupThreads, 0, stream>>>(
        p.W, p.C, p.M, p.N, p.ldc, tiles_m, tiles_n, nkb, grid, p.alpha, p.beta);
    LT_CUDA_TRY(cudaGetLastError());
  }
  if (p.splits > 1) {
    const int64_t n = p.M * p.N;
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, static_cast<int64_t>(ctx->sm_count) * 16);
    splitk_reduce_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(p.W, p.C, n, p.N, p.ldc, p.splits, p.alpha,
                                                                          p.beta);
    LT_CUDA_TRY(cudaGetLastError());
  }
  return LT_OK;
}

using LaunchFn = int (*)(const Params&, cudaStream_t, DeviceContext*, const ScratchUse*);

struct Entry {
  const char* name;
  LaunchFn fn;
  int bm, bn;
  bool tma;
};

// Candidate list of the autotuner (compile-time instances, as hgemm's tuner in the reference:
// routines/hgemm/hgemm_better_reuse.cu:378-454).
const Entry kConfigs[] = {
    {"tma_128x64_s6", launch<Config<128, 64, 6, true>>, 128, 64, true},
    {"tma_64x128_s6", launch<Config<64, 128, 6, true>>, 64, 128, true},
    {"tma_64x64_s8", launch<Config<64, 64, 8, true>>, 64, 64, true},
    {"tma_64x32_s8", launch<Config<64, 32, 8, true>>, 64, 32, true},
    {"tma_32x64_s8", launch<Config<32, 64, 8, true>>, 32, 64, true},
    {"tma_128x64_s4", launch<Config<128, 64, 4, true>>, 128, 64, true},
    {"tma_64x64_s4", launch<Config<64, 64, 4, true>>, 64, 64, true},
    {"cpa_128x64_s6", launch<Config<128, 64, 6, false>>, 128, 64, false},
    {"cpa_64x64_s6", launch<Config<64, 64, 6, false>>, 64, 64, false},
    {"cpa_64x32_s6", launch<Config<64, 32, 6, false>>, 64, 32, false},
    {"cpa_32x32_s6", launch<Config<32, 32, 6, false>>, 32, 32, false},
    {"tma_64x64_s6_x2", launch<Config<64, 64, 6, true, 2>>, 64, 64, true},
};
constexpr int kNumConfigs = static_cast<int>(sizeof(kConfigs) / sizeof(kConfigs[0]));

}  // namespace

bool tma_compatible(const double* A, const double* B, int64_t N, int64_t K) {
  return ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) == 0 && (N % 2 == 0) &&
         (K % 2 == 0);
}

int num_configs() { return kNumConfigs; }
const char* config_name(int i) { return (i >= 0 && i < kNumConfigs) ? kConfigs[i].name : nullptr; }
bool config_is_tma(int i) { return i >= 0 && i < kNumConfigs && kConfigs[i].tma; }

// Default choice without a tuning table: the configuration (of the staging the pointers allow)
// minimising the modelled time of its best schedule (whole tiles, K split or stream-K, one CTA per
// SM) / tile efficiency. Efficiencies are the tiles' measured 8192^3 rates relative to 128x64
// (TMA: 34.8, 33.2, 27.6, 18.0, 18.0 TF/s for 128x64, 64x128, 64x64, 64x32, 32x64).
int heuristic_config(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int sm_count) {
  return heuristic_config_for(M, N, K, sm_count, K > 0 && tma_compatible(A, B, N, K));
}

int heuristic_config_for(int64_t M, int64_t N, int64_t K, int sm_count, bool tma) {
  auto efficiency = [](int bm, int bn) {
    if (bm == 128 && bn == 64) return 1.0;
    if (bm == 64 && bn == 128) return 0.95;
    if (bm == 64 && bn == 64) return 0.79;
    if (bm * bn == 2048) return 0.52;
    return 0.35;
  };
  int best = -1;
  double best_cost = 0.0;
  for (int i = 0; i < kNumConfigs; ++i) {
    if (kConfigs[i].tma != tma) continue;
    const int bm = kConfigs[i].bm, bn = kConfigs[i].bn;
    const int64_t tiles = ((M + bm - 1) / bm) * ((N + bn - 1) / bn);
    const double cost = choose_schedule(tiles, sm_count, M, N, K, bm, bn).t / efficiency(bm, bn);
    if (best < 0 || cost < best_cost * 0.999) {
      best = i;
      best_cost = cost;
    }
  }
  return best >= 0 ? best : kNumConfigs - 1;
}

// ---- grouped launches ----
// cp.async configurations stage tiles of any shape and alignment. TMA configurations read A and B
// through per-problem tensor maps; an operand whose base is not 16-byte aligned or whose row pitch
// (K for A, N for B) is odd cannot be described by one, so each run first copies it into a
// plan-owned buffer with an even pitch (the plan holds pointers, not values, so the copy is part
// of every run; the padding column is never read: the map's extent is the operand's own).
struct PackJob {
  const double* src;  // rows x cols, row pitch cols
  double* dst;        // rows x cols, row pitch dpitch
  int64_t rows, cols, dpitch;
  int64_t row0;  // first row of this job in the launch's row numbering
};

namespace {

// One warp per row (found by binary search over row0), consecutive lanes on consecutive doubles,
// four loads in flight per lane before their stores (one load per lane at a time held the copy at
// about half the HBM rate: rows are a few hundred doubles).
__global__ void pack_rows_kernel(const PackJob* __restrict__ jobs, int njobs, int64_t total_rows) {
  const int64_t wpb = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  for (int64_t r = blockIdx.x * wpb + (threadIdx.x >> 5); r < total_rows; r += gridDim.x * wpb) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (jobs[mid].row0 <= r) lo = mid;
      else hi = mid - 1;
    }
    const PackJob& j = jobs[lo];
    const int64_t row = r - j.row0;
    const double* __restrict__ src = j.src + row * j.cols;
    double* __restrict__ dst = j.dst + row * j.dpitch;
    for (int64_t c0 = lane; c0 < j.cols; c0 += 128) {
      double v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (c0 + 32 * u < j.cols) v[u] = src[c0 + 32 * u];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (c0 + 32 * u < j.cols) dst[c0 + 32 * u] = v[u];
    }
  }
}

// setup_only: sets the kernel's attributes and, when `ctas` is given, stores the number of CTAs a
// launch runs at most (SMs x CTAs per SM) there; no launch.
template <class Cfg>
int launch_grouped(const GroupProblem* problems, const GroupTile* tiles, int64_t ntiles, cudaStream_t stream,
                   DeviceContext* ctx, bool setup_only, int64_t* ctas = nullptr) {
  static std::once_flag once[64];
  static int occupancy[64];
  static cudaError_t attr_err[64];
  std::call_once(once[ctx->device], [&] {
    attr_err[ctx->device] = cudaFuncSetAttribute(dgemm_fp64_grouped_kernel<Cfg>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM_BYTES);
    int occ = 0;
    if (attr_err[ctx->device] == cudaSuccess)
      attr_err[ctx->device] = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, dgemm_fp64_grouped_kernel<Cfg>,
                                                                            Cfg::THREADS, Cfg::SMEM_BYTES);
    occupancy[ctx->device] = occ > 0 ? occ : 1;
  });
  LT_CUDA_TRY(attr_err[ctx->device]);
  int64_t grid = static_cast<int64_t>(ctx->sm_count) * occupancy[ctx->device];
  if (ctas != nullptr) *ctas = grid;
  if (grid > ntiles) grid = ntiles;
  if (grid < 1 || setup_only) return LT_OK;
  GroupedSource src{problems, tiles, ntiles};
  dgemm_fp64_grouped_kernel<Cfg><<<static_cast<unsigned>(grid), Cfg::THREADS, Cfg::SMEM_BYTES, stream>>>(src,
                                                                                                         ctx->status);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

using GroupedFn = int (*)(const GroupProblem*, const GroupTile*, int64_t, cudaStream_t, DeviceContext*, bool,
                          int64_t*);
struct GroupedEntry {
  const char* name;
  GroupedFn fn;
  int bm, bn;
  bool tma;
};
const GroupedEntry kGrouped[] = {
    {"grouped_cpa_128x64_s6", launch_grouped<Config<128, 64, 6, false>>, 128, 64, false},
    {"grouped_cpa_64x64_s6", launch_grouped<Config<64, 64, 6, false>>, 64, 64, false},
    {"grouped_cpa_64x32_s6", launch_grouped<Config<64, 32, 6, false>>, 64, 32, false},
    {"grouped_cpa_32x32_s6", launch_grouped<Config<32, 32, 6, false>>, 32, 32, false},
    // shallower rings leave room for more CTAs per SM (more warps to hide load latency)
    {"grouped_cpa_64x64_s3", launch_grouped<Config<64, 64, 3, false>>, 64, 64, false},
    {"grouped_cpa_64x32_s3", launch_grouped<Config<64, 32, 3, false>>, 64, 32, false},
    {"grouped_cpa_32x64_s3", launch_grouped<Config<32, 64, 3, false>>, 32, 64, false},
    {"grouped_cpa_32x32_s3", launch_grouped<Config<32, 32, 3, false>>, 32, 32, false},
    {"grouped_tma_128x64_s6", launch_grouped<Config<128, 64, 6, true>>, 128, 64, true},
    {"grouped_tma_64x64_s8", launch_grouped<Config<64, 64, 8, true>>, 64, 64, true},
    {"grouped_tma_64x32_s8", launch_grouped<Config<64, 32, 8, true>>, 64, 32, true},
    {"grouped_tma_32x64_s8", launch_grouped<Config<32, 64, 8, true>>, 32, 64, true},
    {"grouped_tma_32x32_s8", launch_grouped<Config<32, 32, 8, true>>, 32, 32, true},
    {"grouped_tma_64x64_s4", launch_grouped<Config<64, 64, 4, true>>, 64, 64, true},
    {"grouped_tma_32x64_s4", launch_grouped<Config<32, 64, 4, true>>, 32, 64, true},
    {"grouped_tma_32x32_s4", launch_grouped<Config<32, 32, 4, true>>, 32, 32, true},
    {"grouped_tma_64x64_s6_x2", launch_grouped<Config<64, 64, 6, true, 2>>, 64, 64, true},
    {"grouped_tma_64x64_s4_x2", launch_grouped<Config<64, 64, 4, true, 2>>, 64, 64, true},
    {"grouped_tma_64x32_s6_x2", launch_grouped<Config<64, 32, 6, true, 2>>, 64, 32, true},
    {"grouped_cpa_64x64_s3_x2", launch_grouped<Config<64, 64, 3, false, 2>>, 64, 64, false},
};
constexpr int kNumGrouped = static_cast<int>(sizeof(kGrouped) / sizeof(kGrouped[0]));

}  // namespace

struct GroupedFp64 {
  int cfg = 0;
  void* dev = nullptr;
  GroupProblem* d_problems = nullptr;
  GroupTile* d_tiles = nullptr;
  int64_t ntiles = 0;
  // TMA configurations: operands copied to an even pitch at the start of each run
  void* pack_buf = nullptr;
  PackJob* d_pack = nullptr;
  int npack = 0;
  int64_t pack_rows = 0;
};

int grouped_num_configs() { return kNumGrouped; }
const char* grouped_config_name(int cfg) { return (cfg >= 0 && cfg < kNumGrouped) ? kGrouped[cfg].name : nullptr; }

int grouped_create(const lt_gemm_problem* problems, int count, int cfg, GroupedFp64** out) {
  if (cfg < 0 || cfg >= kNumGrouped) return set_error(LT_ERR_INVALID_ARGUMENT, "grouped config %d", cfg);
  const int bm = kGrouped[cfg].bm, bn = kGrouped[cfg].bn;
  std::vector<GroupProblem> probs(count);
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) {
    const lt_gemm_problem& p = problems[i];
    probs[i] = GroupProblem{p.A, p.B, p.C, p.M, p.N, p.K, p.alpha, p.beta, nullptr, nullptr};
    order[i] = i;
  }
  // Longest-K problems first: with a static round-robin over the CTAs this balances the work.
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return problems[a].K > problems[b].K; });
  std::vector<GroupTile> tiles;
  for (int i : order) {
    const int64_t tm = (problems[i].M + bm - 1) / bm, tn = (problems[i].N + bn - 1) / bn;
    for (int64_t a = 0; a < tm; ++a)
      for (int64_t b = 0; b < tn; ++b) tiles.push_back(GroupTile{i, static_cast<int>(a * bm), static_cast<int>(b * bn), 0});
  }
  // CTA c of a G-CTA launch takes tiles c, c + G, c + 2G, ... Dealt in plain order, CTA 0 would get
  // the longest tile of every round and finish up to one long tile after CTA G - 1, so every other
  // full round is dealt in reverse (the tiles' K falls along the list); the partial last round
  // stays in order. Only the balance depends on G: every tile is still taken exactly once.
  {
    DeviceContext* ctx = context();
    int64_t G = 0;
    if (ctx == nullptr) return last_error();
    LT_TRY(kGrouped[cfg].fn(nullptr, nullptr, static_cast<int64_t>(tiles.size()), nullptr, ctx, true, &G));
    const int64_t n = static_cast<int64_t>(tiles.size());
    if (G > 1 && n > G) {
      std::vector<GroupTile> dealt(tiles);
      for (int64_t i = 0; i < (n / G) * G; ++i) {
        const int64_t r = i / G, j = i % G;
        dealt[r * G + ((r & 1) ? G - 1 - j : j)] = tiles[i];
      }
      tiles.swap(dealt);
    }
  }
  auto* G = new GroupedFp64();
  G->cfg = cfg;
  G->ntiles = static_cast<int64_t>(tiles.size());
  const bool tma = kGrouped[cfg].tma;
  // TMA: where each problem's A and B are read from (the caller's array or a packed copy).
  struct Operand {
    const double* src;
    int64_t rows, cols, pitch;
    size_t pack_off;  // SIZE_MAX: read in place
  };
  std::vector<Operand> ops;
  std::vector<PackJob> packs;
  size_t pack_bytes = 0;
  if (tma) {
    ops.resize(2 * static_cast<size_t>(count));
    for (int i = 0; i < count; ++i) {
      const lt_gemm_problem& p = problems[i];
      const Operand in[2] = {{p.A, p.M, p.K, p.K, SIZE_MAX}, {p.B, p.K, p.N, p.N, SIZE_MAX}};
      for (int o = 0; o < 2; ++o) {
        Operand op = in[o];
        const bool used = p.M > 0 && p.N > 0 && p.K > 0;
        if (used && (((reinterpret_cast<uintptr_t>(op.src) & 15) != 0) || (op.cols & 1) != 0)) {
          op.pitch = (op.cols + 1) & ~int64_t(1);
          op.pack_off = pack_bytes;
          pack_bytes += (static_cast<size_t>(op.rows * op.pitch) * sizeof(double) + 255) / 256 * 256;
          packs.push_back(PackJob{op.src, nullptr, op.rows, op.cols, op.pitch, G->pack_rows});
          G->pack_rows += op.rows;
        }
        ops[2 * i + o] = op;
      }
    }
  }
  const size_t pb = (sizeof(GroupProblem) * count + 255) / 256 * 256;
  const size_t mb = tma ? (sizeof(CUtensorMap) * 2 * count + 255) / 256 * 256 : 0;
  const size_t jb = (sizeof(PackJob) * packs.size() + 255) / 256 * 256;
  const size_t tb = sizeof(GroupTile) * (tiles.size() + 1);
  int rc = LT_OK;
  cudaError_t e = cudaMalloc(&G->dev, pb + mb + jb + tb);
  if (e == cudaSuccess && pack_bytes > 0) e = cudaMalloc(&G->pack_buf, pack_bytes);
  if (e == cudaSuccess) {
    uint8_t* base = static_cast<uint8_t*>(G->dev);
    G->d_problems = reinterpret_cast<GroupProblem*>(base);
    CUtensorMap* d_maps = reinterpret_cast<CUtensorMap*>(base + pb);
    G->d_pack = reinterpret_cast<PackJob*>(base + pb + mb);
    G->d_tiles = reinterpret_cast<GroupTile*>(base + pb + mb + jb);
    G->npack = static_cast<int>(packs.size());
    if (tma) {
      std::vector<CUtensorMap> maps(2 * static_cast<size_t>(count));
      int j = 0;
      for (int i = 0; i < count && rc == LT_OK; ++i) {
        const lt_gemm_problem& p = problems[i];
        if (p.M <= 0 || p.N <= 0 || p.K <= 0) continue;  // no loads: the maps stay null
        const double* src[2];
        for (int o = 0; o < 2; ++o) {
          const Operand& op = ops[2 * i + o];
          src[o] = op.src;
          if (op.pack_off != SIZE_MAX) {
            src[o] = reinterpret_cast<const double*>(static_cast<uint8_t*>(G->pack_buf) + op.pack_off);
            packs[j++].dst = const_cast<double*>(src[o]);
          }
        }
        const Operand &a = ops[2 * i], &b = ops[2 * i + 1];
        rc = make_tmap_2d(&maps[2 * i], src[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, static_cast<uint64_t>(a.rows),
                          static_cast<uint64_t>(a.cols), static_cast<uint64_t>(a.pitch) * 8, bm, 16);
        if (rc == LT_OK)
          rc = make_tmap_2d(&maps[2 * i + 1], src[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8,
                            static_cast<uint64_t>(b.rows), static_cast<uint64_t>(b.cols),
                            static_cast<uint64_t>(b.pitch) * 8, 16, 16);
        probs[i].tmA = d_maps + 2 * i;
        probs[i].tmB = d_maps + 2 * i + 1;
      }
      if (rc == LT_OK) e = cudaMemcpy(d_maps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice);
      if (rc == LT_OK && e == cudaSuccess && !packs.empty())
        e = cudaMemcpy(G->d_pack, packs.data(), sizeof(PackJob) * packs.size(), cudaMemcpyHostToDevice);
    }
    if (rc == LT_OK && e == cudaSuccess)
      e = cudaMemcpy(G->d_problems, probs.data(), sizeof(GroupProblem) * count, cudaMemcpyHostToDevice);
    if (rc == LT_OK && e == cudaSuccess && !tiles.empty())
      e = cudaMemcpy(G->d_tiles, tiles.data(), sizeof(GroupTile) * tiles.size(), cudaMemcpyHostToDevice);
  }
  if (rc != LT_OK || e != cudaSuccess) {
    cudaFree(G->pack_buf);
    cudaFree(G->dev);
    delete G;
    if (rc != LT_OK) return rc;
    return set_error(LT_ERR_NO_MEMORY, "grouped FP64 tables: %s", cudaGetErrorString(e));
  }
  *out = G;
  return LT_OK;
}

int grouped_run(const GroupedFp64* G, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  if (G->npack > 0) {
    int64_t blocks = (G->pack_rows + 7) / 8;
    if (blocks > 8 * static_cast<int64_t>(ctx->sm_count)) blocks = 8 * static_cast<int64_t>(ctx->sm_count);
    pack_rows_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(G->d_pack, G->npack, G->pack_rows);
    LT_CUDA_TRY(cudaGetLastError());
  }
  return kGrouped[G->cfg].fn(G->d_problems, G->d_tiles, G->ntiles, stream, ctx, false, nullptr);
}

// Kernel attribute set-up only (before a stream capture, which must not contain it).
int grouped_prepare(const GroupedFp64* G) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  return kGrouped[G->cfg].fn(G->d_problems, G->d_tiles, G->ntiles, nullptr, ctx, true, nullptr);
}

void grouped_destroy(GroupedFp64* G) {
  if (G == nullptr) return;
  cudaFree(G->pack_buf);
  cudaFree(G->dev);
  delete G;
}

int64_t grouped_tiles(const GroupedFp64* G) { return G->ntiles; }

int run_config(int cfg, const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
               double beta, cudaStream_t stream, const ScratchUse* scratch) {
  return run_config_ld(cfg, A, K, B, N, C, N, M, N, K, alpha, beta, stream, scratch);
}

int run_config_ld(int cfg, const double* A, int64_t lda, const double* B, int64_t ldb, double* C, int64_t ldc, int64_t M,
                  int64_t N, int64_t K, double alpha, double beta, cudaStream_t stream, const ScratchUse* scratch) {
  if (cfg < 0 || cfg >= kNumConfigs) return set_error(LT_ERR_INVALID_ARGUMENT, "FP64 config %d out of range", cfg);
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  Params p{};
  p.A = A;
  p.B = B;
  p.C = C;
  p.M = M;
  p.N = N;
  p.K = K;
  p.alpha = alpha;
  p.beta = beta;
  p.splits = 1;
  p.lda = lda;
  p.ldb = ldb;
  p.ldc = ldc;
  return kConfigs[cfg].fn(p, stream, ctx, scratch);
}

}  // namespace fp64
}  // namespace lt
