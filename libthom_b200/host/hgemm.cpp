// hgemm.cpp — the `hgemm` routine of the CLI: implementation registry, runner, test/bench/tune.
//
// Reference: routines/hgemm/hgemm.cu. Same argv contract and implementation signature
// (hgemm.h:6-7), same bench sizes (hgemm.cu:17-27), same inputs (uniform (0, 1] rounded to FP16),
// alpha = 1 and beta = 0 (hgemm.cu:107-121), the same acceptance test (an entry differs when its
// relative error against max(|ref|, 1e-3) exceeds 1e-2 and its absolute error 1e-3,
// hgemm.cu:155-171) and CSV export. Differences:
//  - inputs come from a seeded host generator (splitmix64, seed LIBTHOM_HGEMM_SEED, default 1234)
//    instead of cuRAND, alpha and beta from LIBTHOM_HGEMM_{ALPHA,BETA};
//  - the check compares against cuBLAS with FP32 accumulation on the device instead of the
//    single-threaded host loop (which takes minutes at 8192^3), and prints the largest error
//    relative to |alpha| sum |a||b| + |beta||c| beside the reference's count;
//  - C is restored from C0 between runs, L2 is flushed before every timed call and the median is
//    reported beside the mean;
//  - `tune hgemm [M N K [runs]]` times this library's tile configurations instead of the
//    reference's template instances (hgemm.cu:257-324).
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <fstream>

#include "libthom_hgemm.h"
#include "routines.h"

#define BENCH_RUNS 10
#define WARMUP_RUNS 5

namespace hgemm {

static const std::vector<std::vector<int>> SIZES = {{512, 512, 512},    {1024, 1024, 1024}, {1536, 1536, 1536},
                                                    {2048, 2048, 2048}, {2560, 2560, 2560}, {3072, 3072, 3072},
                                                    {3584, 3584, 3584}, {4096, 4096, 4096}, {8192, 8192, 8192}};

using HgemmImpl = float (*)(const lt_half* A, const lt_half* B, lt_half* C, size_t M, size_t N, size_t K,
                            lt_half alpha, lt_half beta);

static const std::map<std::string, HgemmImpl> hgemmImpls = {
    {"tc100", hgemm_tc100},
    {"cublas", hgemm_cublas},
};

struct Buffers {
  lt_half *A = nullptr, *B = nullptr, *C = nullptr, *C0 = nullptr, *R = nullptr;
};

static lt_half bits(float x) { return __half_as_ushort(__float2half_rn(x)); }
static float value(lt_half h) { return __half2float(__ushort_as_half(h)); }

// Uniform (0, 1] rounded to FP16 (the reference's cuRAND fill, hgemm.cu:107-119), seeded.
static void fillHost(std::vector<lt_half>& v, unsigned long long seed, unsigned long long stream) {
  unsigned long long s = seed * 0x9E3779B97F4A7C15ull + stream;
  for (auto& x : v) {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    x = bits(static_cast<float>((z >> 40) + 1) * (1.0f / 16777216.0f));
  }
}

struct Inputs {
  float alpha, beta;
  unsigned long long seed;
};

static Inputs readInputs() {
  Inputs in;
  in.alpha = static_cast<float>(envDouble("LIBTHOM_HGEMM_ALPHA", 1.0));
  in.beta = static_cast<float>(envDouble("LIBTHOM_HGEMM_BETA", 0.0));
  in.seed = static_cast<unsigned long long>(envLong("LIBTHOM_HGEMM_SEED", 1234));
  return in;
}

static void allocate(Buffers& b, const Inputs& in, size_t M, size_t N, size_t K, bool check) {
  CUDA_CHECK(cudaMalloc(&b.A, M * K * 2 + 16));
  CUDA_CHECK(cudaMalloc(&b.B, K * N * 2 + 16));
  CUDA_CHECK(cudaMalloc(&b.C, M * N * 2 + 16));
  CUDA_CHECK(cudaMalloc(&b.C0, M * N * 2 + 16));
  if (check) CUDA_CHECK(cudaMalloc(&b.R, M * N * 2 + 16));
  std::vector<lt_half> h(std::max(M * K, std::max(K * N, M * N)));
  h.resize(M * K);
  fillHost(h, in.seed, 1);
  CUDA_CHECK(cudaMemcpy(b.A, h.data(), M * K * 2, cudaMemcpyHostToDevice));
  h.resize(K * N);
  fillHost(h, in.seed, 2);
  CUDA_CHECK(cudaMemcpy(b.B, h.data(), K * N * 2, cudaMemcpyHostToDevice));
  h.resize(M * N);
  fillHost(h, in.seed, 3);
  CUDA_CHECK(cudaMemcpy(b.C0, h.data(), M * N * 2, cudaMemcpyHostToDevice));
}

static void freeAll(Buffers& b) {
  cudaFree(b.A);
  cudaFree(b.B);
  cudaFree(b.C);
  cudaFree(b.C0);
  cudaFree(b.R);
  b = Buffers();
}

// Compares C with cuBLAS (FP32 accumulation) from the same C0 using the reference's acceptance
// test; returns the number of differing entries.
static long compareToReference(const Buffers& b, const Inputs& in, size_t M, size_t N, size_t K) {
  CUDA_CHECK(cudaMemcpy(b.R, b.C0, M * N * 2, cudaMemcpyDeviceToDevice));
  LT_CHECK(lt_hgemm_cublas(b.A, b.B, b.R, M, N, K, in.alpha, in.beta, 1, nullptr));
  std::vector<lt_half> c(M * N), r(M * N);
  CUDA_CHECK(cudaMemcpy(c.data(), b.C, M * N * 2, cudaMemcpyDeviceToHost));
  CUDA_CHECK(cudaMemcpy(r.data(), b.R, M * N * 2, cudaMemcpyDeviceToHost));
  long differ = 0;
  double worst = 0.0;
  for (size_t i = 0; i < M * N; ++i) {
    const double g = value(c[i]), ref = value(r[i]);
    const double diff = std::fabs(g - ref), rel = diff / std::max(std::fabs(ref), 1e-3);
    if (rel > 1e-2 && diff > 1e-3) {
      if (++differ <= 8) printf("row %zu col %zu | GPU: %f | cuBLAS: %f | rel_error: %f\n", i / N, i % N, g, ref, rel);
    }
    worst = std::max(worst, rel);
  }
  if (differ > 0) printf("Number of different results: %ld\n", differ);
  printf("[check] %ld entries differ from cuBLAS (FP32 accumulation); largest relative difference %.3e\n", differ,
         worst);
  return differ;
}

static double getGflops(size_t M, size_t N, size_t K, double ms) {
  return 2.0 * static_cast<double>(M) * static_cast<double>(N) * static_cast<double>(K) / (ms * 1e6);
}

// Runner shared by test and bench (reference: hgemm.cu:198-239). Returns the median GFLOP/s.
static float runner(HgemmImpl impl, std::vector<int> sizes, int nb_runs, int nb_warmup_runs, bool checkResult,
                    bool printEach) {
  const size_t M = sizes[0], N = sizes[1], K = sizes[2];
  const Inputs in = readInputs();
  Buffers b;
  allocate(b, in, M, N, K, checkResult);
  std::vector<double> gf;
  double sum = 0.0;
  for (int i = -nb_warmup_runs; i < nb_runs; i++) {
    CUDA_CHECK(cudaMemcpy(b.C, b.C0, M * N * 2, cudaMemcpyDeviceToDevice));
    flushL2();
    CUDA_CHECK(cudaDeviceSynchronize());
    float ms = impl(b.A, b.B, b.C, M, N, K, bits(in.alpha), bits(in.beta));
    if (lt_get_last_error() != LT_OK) {
      fprintf(stderr, "implementation failed: %s\n", lt_last_error_message());
      exit(EXIT_FAILURE);
    }
    if (checkResult) compareToReference(b, in, M, N, K);
    if (i >= 0) {
      double g = getGflops(M, N, K, ms);
      if (printEach) printf("[internal][iter %d]: %f GFLOP/s \n", i, g);
      gf.push_back(g);
      sum += g;
    }
  }
  freeAll(b);
  if (nb_runs > 0) printf("[summary] mean %.1f GFLOP/s, median %.1f GFLOP/s\n", sum / nb_runs, median(gf));
  return static_cast<float>(median(gf));
}

static void exportCSV(const std::map<std::vector<int>, float>& results, const std::string& filename) {
  std::ofstream file(filename);
  file << "M,N,K,gflops\n";
  for (const auto& kv : results) file << kv.first[0] << "," << kv.first[1] << "," << kv.first[2] << "," << kv.second << "\n";
}

static void listImpls() {
  fprintf(stderr, "Available implementations:");
  for (const auto& e : hgemmImpls) fprintf(stderr, " %s", e.first.c_str());
  fprintf(stderr, "\n");
}

static HgemmImpl findImpl(const char* name) {
  auto it = hgemmImpls.find(name);
  if (it == hgemmImpls.end()) {
    fprintf(stderr, "Invalid implementation. Either it doesnt exist, or it's not available for the ARCH you've compiled\n");
    listImpls();
    exit(1);
  }
  return it->second;
}

// `libthom test hgemm <impl> <M> <N> <K> <nb_iter> [check=1]` (routines/routines.h:90-130).
static void testHandler(int argc, char* argv[]) {
  const int sizeDims = 3, supposedArgc = 5 + sizeDims;
  if (argc < supposedArgc) {
    fprintf(stderr, "Missing arguments.\nUsage: ./libthom test hgemm <impl> <M> <N> <K> <nb_iter> <check_result=1>\n");
    listImpls();
    exit(1);
  }
  HgemmImpl impl = findImpl(argv[3]);
  std::vector<int> sizes = {atoi(argv[4]), atoi(argv[5]), atoi(argv[6])};
  int nb_iter = atoi(argv[7]);
  bool check = true;
  if (argc >= supposedArgc + 1) check = atoi(argv[8]) == 1;
  float gflops = runner(impl, sizes, nb_iter, 0, check, true);
  printf("# GFLOP/s: %f\n", gflops);
}

// `libthom bench hgemm <impl>` (routines/routines.h:132-169).
static void benchHandler(int argc, char* argv[]) {
  if (argc < 4) {
    fprintf(stderr, "Missing arguments.\nUsage: ./libthom bench hgemm <impl>\n");
    listImpls();
    exit(1);
  }
  HgemmImpl impl = findImpl(argv[3]);
  printf("-- Running hgemm -- %s\n", argv[3]);
  std::map<std::vector<int>, float> results;
  for (const auto& sizes : SIZES) {
    printf("\nStarting benchmark for size %d...\n", sizes[0]);
    float g = runner(impl, sizes, BENCH_RUNS, WARMUP_RUNS, false, true);
    results[sizes] = g;
    printf("[size: %d] ==> %f\n", sizes[0], g);
  }
  exportCSV(results, std::string("bench_hgemm_") + argv[3] + ".csv");
}

// `libthom tune hgemm [M N K [runs]]` (reference: hgemm.cu:257-324): validate, then time, every
// tile configuration of the library's kernel at one shape; print each result and the best.
static void tuneHandler(int argc, char* argv[]) {
  int M = 2048, N = 2048, K = 2048, runs = 30;
  if (argc != 3 && argc != 6 && argc != 7) {
    fprintf(stderr, "Usage: ./libthom tune hgemm [M N K [runs]]\n");
    return;
  }
  if (argc >= 6) {
    M = atoi(argv[3]);
    N = atoi(argv[4]);
    K = atoi(argv[5]);
  }
  if (argc == 7) runs = atoi(argv[6]);
  if (M <= 0 || N <= 0 || K <= 0 || runs <= 0) {
    fprintf(stderr, "M, N, K and runs must be positive.\n");
    return;
  }
  printf("-- Tuning hgemm tc100 for M=%d N=%d K=%d (%d measured runs) --\n", M, N, K, runs);
  const Inputs in = readInputs();
  Buffers b;
  allocate(b, in, M, N, K, true);
  cudaEvent_t e0, e1;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  int best = -1;
  double best_g = -1.0;
  for (int cfg = 0; cfg < lt_hgemm_num_configs(); ++cfg) {
    printf("[test] %s\n", lt_hgemm_config_name(cfg));
    CUDA_CHECK(cudaMemcpy(b.C, b.C0, static_cast<size_t>(M) * N * 2, cudaMemcpyDeviceToDevice));
    LT_CHECK(lt_hgemm_config(b.A, b.B, b.C, M, N, K, in.alpha, in.beta, cfg, nullptr));
    LT_CHECK(lt_check_device_status());
    if (compareToReference(b, in, M, N, K) != 0) {
      printf("[failed] %s\n", lt_hgemm_config_name(cfg));
      continue;
    }
    std::vector<double> gf;
    for (int i = -WARMUP_RUNS; i < runs; ++i) {
      flushL2();
      CUDA_CHECK(cudaEventRecord(e0));
      LT_CHECK(lt_hgemm_config(b.A, b.B, b.C, M, N, K, in.alpha, in.beta, cfg, nullptr));
      CUDA_CHECK(cudaEventRecord(e1));
      CUDA_CHECK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
      if (i >= 0) gf.push_back(getGflops(M, N, K, ms));
    }
    const double g = median(gf);
    printf("[result] %s: %.2f GFLOP/s\n", lt_hgemm_config_name(cfg), g);
    if (g > best_g) {
      best_g = g;
      best = cfg;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  freeAll(b);
  if (best < 0) {
    fprintf(stderr, "No candidate supports these dimensions.\n");
    return;
  }
  printf("[best] %s: %.2f GFLOP/s (automatic choice: %s)\n", lt_hgemm_config_name(best), best_g,
         lt_hgemm_config_name(lt_hgemm_default_config(M, N, K)));
}

}  // namespace hgemm

void hgemm_handler(RunMode runMode, int argc, char* argv[]) {
  switch (runMode) {
    case RunMode::TEST: hgemm::testHandler(argc, argv); break;
    case RunMode::BENCH: hgemm::benchHandler(argc, argv); break;
    case RunMode::TUNE: hgemm::tuneHandler(argc, argv); break;
  }
}
