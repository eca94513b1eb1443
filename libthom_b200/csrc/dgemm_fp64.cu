// dgemm_fp64.cu — host launchers and configuration registry of the native FP64 DGEMM.
#include <algorithm>
#include <mutex>
#include <vector>

#include "dgemm_fp64.cuh"
#include "lt_runtime.cuh"
#include "lt_internal.h"

namespace lt {
namespace fp64 {

namespace {

// K split for tile counts that fill the GPU poorly (wave quantisation): the split count S in 1..4
// minimising waves(S) x (k-blocks per range + pipeline fill) at the FP64 tensor rate, plus the
// reduction's traffic, and at least 3 % better than no split; ranges keep >= 32 k-blocks.
int choose_splits(int64_t tiles, int64_t cap, int64_t M, int64_t N, int64_t K, int bm, int bn) {
  const int64_t nkb = (K + 15) / 16;
  if (nkb < 64 || cap <= 0) return 1;
  const double t_kb = 2.0 * bm * bn * 16 / (128.0 * 1.9e9);  // one k-block of one tile on one SM
  double best = 0.0;
  int best_s = 1;
  for (int S = 1; S <= 4; ++S) {
    const int64_t per = (nkb + S - 1) / S;
    if (S > 1 && per < 32) break;
    const int64_t waves = (tiles * S + cap - 1) / cap;
    double t = static_cast<double>(waves) * static_cast<double>(per + 6) * t_kb;
    if (S > 1) t += (S + 2) * 8.0 * static_cast<double>(M) * static_cast<double>(N) / 6.0e12;
    if (S == 1 || t < best * 0.97) {
      best = t;
      best_s = S;
    }
  }
  return best_s;
}

template <class Cfg>
int launch(const Params& p0, cudaStream_t stream, DeviceContext* ctx) {
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
  const int64_t tiles = ((p.M + Cfg::BM - 1) / Cfg::BM) * ((p.N + Cfg::BN - 1) / Cfg::BN);
  const int64_t cap = static_cast<int64_t>(ctx->sm_count) * occupancy[ctx->device];
  p.splits = choose_splits(tiles, cap, p.M, p.N, p.K, Cfg::BM, Cfg::BN);
  p.W = nullptr;
  if (p.splits > 1) {
    void* w = nullptr;
    LT_TRY(ensure_splitk_workspace(ctx, static_cast<size_t>(p.splits) * p.M * p.N * sizeof(double), &w));
    p.W = static_cast<double*>(w);
  }
  const int64_t units = tiles * p.splits;
  const int64_t grid = units < cap ? units : cap;
  dgemm_fp64_kernel<Cfg><<<static_cast<unsigned>(grid), Cfg::THREADS, Cfg::SMEM_BYTES, stream>>>(tmA, tmB, p);
  LT_CUDA_TRY(cudaGetLastError());
  if (p.splits > 1) {
    const int64_t n = p.M * p.N;
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, static_cast<int64_t>(ctx->sm_count) * 16);
    splitk_reduce_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(p.W, p.C, n, p.N, p.ldc, p.splits, p.alpha,
                                                                          p.beta);
    LT_CUDA_TRY(cudaGetLastError());
  }
  return LT_OK;
}

using LaunchFn = int (*)(const Params&, cudaStream_t, DeviceContext*);

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
// minimising waves x tile area / tile efficiency, one CTA per SM. Efficiencies are the tiles'
// measured 8192^3 rates relative to 128x64 (TMA: 34.8, 33.2, 27.6, 18.0, 18.0 TF/s for 128x64,
// 64x128, 64x64, 64x32, 32x64). The K split handles what remains of a poorly filled last wave.
int heuristic_config(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int sm_count) {
  return heuristic_config_for(M, N, sm_count, K > 0 && tma_compatible(A, B, N, K));
}

int heuristic_config_for(int64_t M, int64_t N, int sm_count, bool tma) {
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
    const int64_t waves = (tiles + sm_count - 1) / sm_count;
    const double cost = static_cast<double>(waves) * bm * bn / efficiency(bm, bn);
    if (best < 0 || cost < best_cost * 0.999) {
      best = i;
      best_cost = cost;
    }
  }
  return best >= 0 ? best : kNumConfigs - 1;
}

// ---- grouped launches (cp.async staging: problems have arbitrary shapes and alignment) ----
namespace {

template <class Cfg>
int launch_grouped(const GroupProblem* problems, const GroupTile* tiles, int64_t ntiles, cudaStream_t stream,
                   DeviceContext* ctx, bool setup_only) {
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
  if (grid > ntiles) grid = ntiles;
  if (grid < 1 || setup_only) return LT_OK;
  GroupedSource src{problems, tiles, ntiles};
  dgemm_fp64_grouped_kernel<Cfg><<<static_cast<unsigned>(grid), Cfg::THREADS, Cfg::SMEM_BYTES, stream>>>(src,
                                                                                                         ctx->status);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

using GroupedFn = int (*)(const GroupProblem*, const GroupTile*, int64_t, cudaStream_t, DeviceContext*, bool);
struct GroupedEntry {
  const char* name;
  GroupedFn fn;
  int bm, bn;
};
const GroupedEntry kGrouped[] = {
    {"grouped_cpa_128x64_s6", launch_grouped<Config<128, 64, 6, false>>, 128, 64},
    {"grouped_cpa_64x64_s6", launch_grouped<Config<64, 64, 6, false>>, 64, 64},
    {"grouped_cpa_64x32_s6", launch_grouped<Config<64, 32, 6, false>>, 64, 32},
    {"grouped_cpa_32x32_s6", launch_grouped<Config<32, 32, 6, false>>, 32, 32},
    // shallower rings leave room for more CTAs per SM (more warps to hide load latency)
    {"grouped_cpa_64x64_s3", launch_grouped<Config<64, 64, 3, false>>, 64, 64},
    {"grouped_cpa_64x32_s3", launch_grouped<Config<64, 32, 3, false>>, 64, 32},
    {"grouped_cpa_32x64_s3", launch_grouped<Config<32, 64, 3, false>>, 32, 64},
    {"grouped_cpa_32x32_s3", launch_grouped<Config<32, 32, 3, false>>, 32, 32},
};
constexpr int kNumGrouped = static_cast<int>(sizeof(kGrouped) / sizeof(kGrouped[0]));

}  // namespace

struct GroupedFp64 {
  int cfg = 0;
  void* dev = nullptr;
  GroupProblem* d_problems = nullptr;
  GroupTile* d_tiles = nullptr;
  int64_t ntiles = 0;
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
    probs[i] = GroupProblem{p.A, p.B, p.C, p.M, p.N, p.K, p.alpha, p.beta};
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
  auto* G = new GroupedFp64();
  G->cfg = cfg;
  G->ntiles = static_cast<int64_t>(tiles.size());
  const size_t pb = (sizeof(GroupProblem) * count + 255) / 256 * 256;
  const size_t tb = sizeof(GroupTile) * (tiles.size() + 1);
  cudaError_t e = cudaMalloc(&G->dev, pb + tb);
  if (e == cudaSuccess) {
    G->d_problems = static_cast<GroupProblem*>(G->dev);
    G->d_tiles = reinterpret_cast<GroupTile*>(static_cast<uint8_t*>(G->dev) + pb);
    e = cudaMemcpy(G->d_problems, probs.data(), sizeof(GroupProblem) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !tiles.empty())
      e = cudaMemcpy(G->d_tiles, tiles.data(), sizeof(GroupTile) * tiles.size(), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaFree(G->dev);
    delete G;
    return set_error(LT_ERR_NO_MEMORY, "grouped FP64 tables: %s", cudaGetErrorString(e));
  }
  *out = G;
  return LT_OK;
}

int grouped_run(const GroupedFp64* G, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  return kGrouped[G->cfg].fn(G->d_problems, G->d_tiles, G->ntiles, stream, ctx, false);
}

// Kernel attribute set-up only (before a stream capture, which must not contain it).
int grouped_prepare(const GroupedFp64* G) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  return kGrouped[G->cfg].fn(G->d_problems, G->d_tiles, G->ntiles, nullptr, ctx, true);
}

void grouped_destroy(GroupedFp64* G) {
  if (G == nullptr) return;
  cudaFree(G->dev);
  delete G;
}

int64_t grouped_tiles(const GroupedFp64* G) { return G->ntiles; }

int run_config(int cfg, const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
               double beta, cudaStream_t stream) {
  return run_config_ld(cfg, A, K, B, N, C, N, M, N, K, alpha, beta, stream);
}

int run_config_ld(int cfg, const double* A, int64_t lda, const double* B, int64_t ldb, double* C, int64_t ldc, int64_t M,
                  int64_t N, int64_t K, double alpha, double beta, cudaStream_t stream) {
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
  return kConfigs[cfg].fn(p, stream, ctx);
}

}  // namespace fp64
}  // namespace lt
