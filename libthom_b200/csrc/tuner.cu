// tuner.cu — autotuner of the native FP64 DGEMM (tile shape, pipeline depth, TMA vs cp.async).
//
// The reference tunes only hgemm, at run time over a compile-time Cartesian product of template
// instances, validating each candidate before timing it (routines/hgemm/hgemm.cu:257-324,
// routines/hgemm/hgemm_better_reuse.cu:378-454); its dgemm handler has no TUNE case
// (routines/dgemm/dgemm.cpp:233-240). This tuner follows the same validate-then-time rule over the
// FP64 kernel's compile-time candidates and keeps one winner per shape class; the table can be
// saved to and loaded from a text file (one "M N K tma config ms" line per class).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "lt_internal.h"
#include "lt_runtime.cuh"

namespace lt {
namespace tuner {
namespace {

// Shape class: each dimension rounded up to the next power of two (minimum 32).
int64_t bucket(int64_t x) {
  int64_t b = 32;
  while (b < x) b <<= 1;
  return b;
}

using Key = std::tuple<int64_t, int64_t, int64_t, int>;
struct Value {
  int config;
  float ms;
};
std::mutex g_mutex;
std::map<Key, Value> g_table;

Key key_of(int64_t M, int64_t N, int64_t K, bool tma) { return Key(bucket(M), bucket(N), bucket(K), tma ? 1 : 0); }

}  // namespace

int lookup(int64_t M, int64_t N, int64_t K, bool tma) {
  std::lock_guard<std::mutex> lock(g_mutex);
  auto it = g_table.find(key_of(M, N, K, tma));
  if (it == g_table.end()) return -1;
  if (fp64::config_is_tma(it->second.config) && !tma) return -1;
  return it->second.config;
}

void record(int64_t M, int64_t N, int64_t K, bool tma, int config, float ms) {
  std::lock_guard<std::mutex> lock(g_mutex);
  g_table[key_of(M, N, K, tma)] = Value{config, ms};
}

}  // namespace tuner
}  // namespace lt

namespace {

__global__ void max_rel_err_kernel(const double* C, const double* R, int64_t n, unsigned long long* out) {
  double mx = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double r = R[i], d = fabs(C[i] - r);
    double e = d / fmax(fabs(r), 1e-300);
    if (!(e <= 1e300)) e = 1e300;  // NaN -> large
    mx = fmax(mx, e);
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(mx)));
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
};

}  // namespace

extern "C" {

int lt_tune_fp64(int64_t M, int64_t N, int64_t K, int iters, lt_tune_entry* best) {
  if (M <= 0 || N <= 0 || K <= 0 || iters < 1 || best == nullptr)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_tune_fp64: bad arguments");
  lt::DeviceContext* ctx = lt::context();
  if (ctx == nullptr) return lt::last_error();
  DevBuf A, B, C, R, E;
  LT_CUDA_TRY(cudaMalloc(&A.p, sizeof(double) * M * K));
  LT_CUDA_TRY(cudaMalloc(&B.p, sizeof(double) * K * N));
  LT_CUDA_TRY(cudaMalloc(&C.p, sizeof(double) * M * N));
  LT_CUDA_TRY(cudaMalloc(&R.p, sizeof(double) * M * N));
  LT_CUDA_TRY(cudaMalloc(&E.p, sizeof(unsigned long long)));
  auto* a = static_cast<double*>(A.p);
  auto* b = static_cast<double*>(B.p);
  auto* c = static_cast<double*>(C.p);
  auto* r = static_cast<double*>(R.p);
  LT_TRY(lt_fill(a, M * K, 1234, 1, 0, nullptr));
  LT_TRY(lt_fill(b, K * N, 1234, 2, 0, nullptr));
  LT_TRY(lt_dgemm_cublas(a, b, r, M, N, K, 1.0, 0.0, nullptr));
  const bool tma = lt::fp64::tma_compatible(a, b, N, K);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best_cfg = -1;
  float best_ms = 0.f, best_err = 0.f;
  for (int cfg = 0; cfg < lt::fp64::num_configs(); ++cfg) {
    if (lt::fp64::config_is_tma(cfg) && !tma) continue;
    // validate
    LT_CUDA_TRY(cudaMemset(E.p, 0, sizeof(unsigned long long)));
    if (lt::fp64::run_config(cfg, a, b, c, M, N, K, 1.0, 0.0, nullptr) != LT_OK) continue;
    max_rel_err_kernel<<<ctx->sm_count * 4, 256>>>(c, r, M * N, static_cast<unsigned long long*>(E.p));
    unsigned long long bits = 0;
    LT_CUDA_TRY(cudaMemcpy(&bits, E.p, sizeof bits, cudaMemcpyDeviceToHost));
    if (lt_check_device_status() != LT_OK) continue;
    double err;
    memcpy(&err, &bits, sizeof err);
    // FP64 products agree with cuBLAS to a few ulps relative to |C| except under cancellation;
    // 1e-8 only rejects a broken candidate.
    if (!(err < 1e-8)) continue;
    // time (median)
    std::vector<float> ts;
    for (int it = 0; it < iters; ++it) {
      cudaEventRecord(e0);
      lt::fp64::run_config(cfg, a, b, c, M, N, K, 1.0, 0.0, nullptr);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      ts.push_back(ms);
    }
    std::sort(ts.begin(), ts.end());
    float med = ts[ts.size() / 2];
    if (best_cfg < 0 || med < best_ms) {
      best_cfg = cfg;
      best_ms = med;
      best_err = static_cast<float>(err);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best_cfg < 0) return lt::set_error(LT_ERR_NOT_FOUND, "no FP64 candidate validated");
  lt::tuner::record(M, N, K, tma, best_cfg, best_ms);
  best->config = best_cfg;
  best->ms = best_ms;
  best->max_rel_err = best_err;
  return lt::ok();
}

int lt_tuner_save(const char* path) {
  if (path == nullptr) return lt::set_error(LT_ERR_INVALID_ARGUMENT, "null path");
  FILE* f = fopen(path, "w");
  if (f == nullptr) return lt::set_error(LT_ERR_NOT_FOUND, "cannot open %s", path);
  std::lock_guard<std::mutex> lock(lt::tuner::g_mutex);
  fprintf(f, "# M N K tma config_name ms\n");
  for (const auto& kv : lt::tuner::g_table)
    fprintf(f, "%lld %lld %lld %d %s %.6f\n", static_cast<long long>(std::get<0>(kv.first)),
            static_cast<long long>(std::get<1>(kv.first)), static_cast<long long>(std::get<2>(kv.first)),
            std::get<3>(kv.first), lt::fp64::config_name(kv.second.config), kv.second.ms);
  fclose(f);
  return lt::ok();
}

int lt_tuner_load(const char* path) {
  if (path == nullptr) return lt::set_error(LT_ERR_INVALID_ARGUMENT, "null path");
  FILE* f = fopen(path, "r");
  if (f == nullptr) return lt::set_error(LT_ERR_NOT_FOUND, "cannot open %s", path);
  char line[256];
  int loaded = 0;
  while (fgets(line, sizeof line, f) != nullptr) {
    if (line[0] == '#') continue;
    long long m, n, k;
    int tma;
    char name[64];
    float ms;
    if (sscanf(line, "%lld %lld %lld %d %63s %f", &m, &n, &k, &tma, name, &ms) != 6) continue;
    for (int cfg = 0; cfg < lt::fp64::num_configs(); ++cfg) {
      if (strcmp(lt::fp64::config_name(cfg), name) == 0) {
        lt::tuner::record(m, n, k, tma != 0, cfg, ms);
        ++loaded;
        break;
      }
    }
  }
  fclose(f);
  return loaded > 0 ? lt::ok() : lt::set_error(LT_ERR_NOT_FOUND, "no usable entries in %s", path);
}

int lt_tuner_lookup(int64_t M, int64_t N, int64_t K) { return lt::tuner::lookup(M, N, K, true); }

}  // extern "C"
