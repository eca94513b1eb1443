// dgemm.cpp — the `dgemm` routine of the CLI: implementation registry, runner, test/bench/tune.
//
// Reference: routines/dgemm/dgemm.cpp. Same argv contract and implementation signature
// (dgemm.cpp:36, dgemm.h:9), same default sizes for `bench` (dgemm.cpp:17) and CSV export
// (dgemm.cpp:209-219). Differences, each an extension the reference cannot express:
//  - inputs come from the library's seeded generator (lt_fill) instead of cuRAND, with alpha, beta,
//    exponent spread, row/column scaling and seed from LIBTHOM_DGEMM_{ALPHA,BETA,PHI,SCALE_S,SEED}
//    (defaults alpha = beta = 1, phi = 0, no scaling, seed 1234 as in dgemm.cpp:100-119, 229-230);
//  - C is restored from C0 on the device between runs instead of regenerating all inputs;
//  - L2 is flushed before every timed call and the median is reported beside the mean;
//  - the check compares against cuBLAS DGEMM (CUBLAS_COMPUTE_64F, the reference's baseline) with
//    the componentwise error |C - C_cublas| / (|alpha||A||B| + |beta||C0|), reporting the maximum
//    and the count above LIBTHOM_DGEMM_TOL (default 1e-13), instead of a float-rounded relative
//    error (dgemm.cpp:137-159);
//  - `tune dgemm` runs the FP64 autotuner (the reference has no TUNE case, dgemm.cpp:233-240).
#include <cmath>
#include <fstream>

#include "routines.h"

#define BENCH_RUNS 10
#define WARMUP_RUNS 5

namespace dgemm {

static const std::vector<std::vector<int>> SIZES = {{512, 512, 512}, {1024, 1024, 1024}, {2048, 2048, 2048},
                                                    {8192, 8192, 8192}};

using DgemmImpl = float (*)(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha,
                            double beta);

static const std::map<std::string, DgemmImpl> dgemmImpls = {
    {"tc100", dgemm_tc100},         {"ozaki3", dgemm_ozaki3},   {"ozaki4", dgemm_ozaki4},
    {"ozaki5", dgemm_ozaki5},       {"ozaki6", dgemm_ozaki6},   {"ozaki7", dgemm_ozaki7},
    {"ozaki8", dgemm_ozaki8},       {"ozaki9", dgemm_ozaki9},   {"ozaki10", dgemm_ozaki10},
    {"ozaki_auto", dgemm_ozaki_auto}, {"auto", dgemm_auto},     {"cublas_tc", dgemm_cublas_tc},
    {"ozaki_crt14", dgemm_ozaki_crt14}, {"ozaki_crt15", dgemm_ozaki_crt15}, {"ozaki_crt16", dgemm_ozaki_crt16},
    {"ozaki_crt17", dgemm_ozaki_crt17}, {"ozaki_crt18", dgemm_ozaki_crt18},
};

struct Buffers {
  double *A = nullptr, *B = nullptr, *C = nullptr, *C0 = nullptr, *R = nullptr, *den = nullptr;
};

static void allocate(Buffers& b, size_t M, size_t N, size_t K, bool check) {
  CUDA_CHECK(cudaMalloc(&b.A, M * K * sizeof(double) + 8));
  CUDA_CHECK(cudaMalloc(&b.B, K * N * sizeof(double) + 8));
  CUDA_CHECK(cudaMalloc(&b.C, M * N * sizeof(double) + 8));
  CUDA_CHECK(cudaMalloc(&b.C0, M * N * sizeof(double) + 8));
  if (check) {
    CUDA_CHECK(cudaMalloc(&b.R, M * N * sizeof(double) + 8));
    CUDA_CHECK(cudaMalloc(&b.den, M * N * sizeof(double) + 8));
  }
}

static void freeAll(Buffers& b) {
  cudaFree(b.A);
  cudaFree(b.B);
  cudaFree(b.C);
  cudaFree(b.C0);
  cudaFree(b.R);
  cudaFree(b.den);
  b = Buffers();
}

struct Inputs {
  double alpha, beta, tol;
  int phi, scale_s;
  unsigned long long seed;
};

static Inputs readInputs() {
  Inputs in;
  in.alpha = envDouble("LIBTHOM_DGEMM_ALPHA", 1.0);
  in.beta = envDouble("LIBTHOM_DGEMM_BETA", 1.0);
  in.phi = static_cast<int>(envLong("LIBTHOM_DGEMM_PHI", 0));
  in.scale_s = static_cast<int>(envLong("LIBTHOM_DGEMM_SCALE_S", 0));
  in.seed = static_cast<unsigned long long>(envLong("LIBTHOM_DGEMM_SEED", 1234));
  in.tol = envDouble("LIBTHOM_DGEMM_TOL", 1e-13);
  return in;
}

static void fillInputs(const Buffers& b, const Inputs& in, size_t M, size_t N, size_t K) {
  LT_CHECK(lt_fill(b.A, static_cast<int64_t>(M * K), in.seed, 1, in.phi, nullptr));
  LT_CHECK(lt_fill(b.B, static_cast<int64_t>(K * N), in.seed, 2, in.phi, nullptr));
  LT_CHECK(lt_fill(b.C0, static_cast<int64_t>(M * N), in.seed, 3, in.phi, nullptr));
  if (in.scale_s > 0) {
    LT_CHECK(lt_scale_rows(b.A, static_cast<int64_t>(M), static_cast<int64_t>(K), in.seed, 4, in.scale_s, nullptr));
    LT_CHECK(lt_scale_cols(b.B, static_cast<int64_t>(K), static_cast<int64_t>(N), in.seed, 5, in.scale_s, nullptr));
  }
  CUDA_CHECK(cudaDeviceSynchronize());
}

// Checks C against cuBLAS FP64 from the same C0; prints and returns the max componentwise error.
static double compareToReference(const Buffers& b, const Inputs& in, size_t M, size_t N, size_t K) {
  CUDA_CHECK(cudaMemcpy(b.R, b.C0, M * N * sizeof(double), cudaMemcpyDeviceToDevice));
  LT_CHECK(lt_dgemm_cublas(b.A, b.B, b.R, M, N, K, in.alpha, in.beta, nullptr));
  LT_CHECK(lt_abs_denominator(b.A, b.B, b.C0, b.den, M, N, K, in.alpha, in.beta, nullptr));
  double out[2] = {0, 0};
  LT_CHECK(lt_componentwise_error(b.C, b.R, b.den, static_cast<int64_t>(M * N), in.tol, out, nullptr));
  printf("[check] max componentwise error vs cuBLAS FP64: %.3e (%lld elements above %.1e)\n", out[0],
         static_cast<long long>(out[1]), in.tol);
  return out[0];
}

static double getGflops(size_t M, size_t N, size_t K, double ms) {
  return 2.0 * static_cast<double>(M) * static_cast<double>(N) * static_cast<double>(K) / (ms * 1e6);
}

// Runner shared by test and bench (reference: dgemm.cpp:168-205). Returns the median GFLOP/s.
static float runner(DgemmImpl impl, std::vector<int> sizes, int nb_runs, int nb_warmup_runs, bool checkResult,
                    bool printEach) {
  const size_t M = sizes[0], N = sizes[1], K = sizes[2];
  const Inputs in = readInputs();
  Buffers b;
  allocate(b, M, N, K, checkResult);
  fillInputs(b, in, M, N, K);
  std::vector<double> gf;
  double sum = 0.0;
  for (int i = -nb_warmup_runs; i < nb_runs; i++) {
    CUDA_CHECK(cudaMemcpy(b.C, b.C0, M * N * sizeof(double), cudaMemcpyDeviceToDevice));
    flushL2();
    CUDA_CHECK(cudaDeviceSynchronize());
    float ms = impl(b.A, b.B, b.C, M, N, K, in.alpha, in.beta);
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
  for (const auto& e : dgemmImpls) fprintf(stderr, " %s", e.first.c_str());
  fprintf(stderr, "\n");
}

// `libthom test dgemm <impl> <M> <N> <K> <nb_iter> [check=1]` (routines/routines.h:90-130).
static void testHandler(int argc, char* argv[]) {
  const int sizeDims = 3, supposedArgc = 5 + sizeDims;
  if (argc < supposedArgc) {
    fprintf(stderr, "Missing arguments.\nUsage: ./libthom test dgemm <impl> <M> <N> <K> <nb_iter> <check_result=1>\n");
    listImpls();
    exit(1);
  }
  auto it = dgemmImpls.find(argv[3]);
  if (it == dgemmImpls.end()) {
    fprintf(stderr, "Invalid implementation. Either it doesnt exist, or it's not available for the ARCH you've compiled\n");
    listImpls();
    exit(1);
  }
  std::vector<int> sizes = {atoi(argv[4]), atoi(argv[5]), atoi(argv[6])};
  int nb_iter = atoi(argv[7]);
  bool check = true;
  if (argc >= supposedArgc + 1) check = atoi(argv[8]) == 1;
  float gflops = runner(it->second, sizes, nb_iter, 0, check, true);
  printf("# GFLOP/s: %f\n", gflops);
}

// `libthom bench dgemm <impl>` (routines/routines.h:132-169).
static void benchHandler(int argc, char* argv[]) {
  if (argc < 4) {
    fprintf(stderr, "Missing arguments.\nUsage: ./libthom bench dgemm <impl>\n");
    listImpls();
    exit(1);
  }
  auto it = dgemmImpls.find(argv[3]);
  if (it == dgemmImpls.end()) {
    fprintf(stderr, "Invalid implementation. Either it doesnt exist, or it's not available for the ARCH you've compiled\n");
    listImpls();
    exit(1);
  }
  printf("-- Running dgemm -- %s\n", argv[3]);
  std::map<std::vector<int>, float> results;
  for (const auto& sizes : SIZES) {
    printf("\nStarting benchmark for size %d...\n", sizes[0]);
    float g = runner(it->second, sizes, BENCH_RUNS, WARMUP_RUNS, false, true);
    results[sizes] = g;
    printf("[size: %d] ==> %f\n", sizes[0], g);
  }
  exportCSV(results, std::string("bench_dgemm_") + argv[3] + ".csv");
}

// `libthom tune dgemm [M N K]...`: validate-then-time every FP64 candidate per shape and store the
// winners (reference precedent: routines/hgemm/hgemm.cu:257-324).
static void tuneHandler(int argc, char* argv[]) {
  std::vector<std::vector<int>> shapes;
  for (int i = 3; i + 2 < argc; i += 3) shapes.push_back({atoi(argv[i]), atoi(argv[i + 1]), atoi(argv[i + 2])});
  if (shapes.empty()) shapes = {{512, 512, 512}, {1024, 1024, 1024}, {2048, 2048, 2048}, {4096, 4096, 4096}};
  const char* path = getenv("LIBTHOM_TUNE_FILE");
  std::string file = path ? path : "tunings/dgemm_fp64.txt";
  lt_tuner_load(file.c_str());  // extend an existing table
  for (const auto& s : shapes) {
    lt_tune_entry best;
    LT_CHECK(lt_tune_fp64(s[0], s[1], s[2], 5, &best));
    printf("[best] %dx%dx%d: %s %.3f ms (%.1f GFLOP/s), max rel err vs cuBLAS %.2e\n", s[0], s[1], s[2],
           lt_fp64_config_name(best.config), best.ms, getGflops(s[0], s[1], s[2], best.ms), best.max_rel_err);
  }
  if (lt_tuner_save(file.c_str()) == LT_OK) printf("saved %s\n", file.c_str());
}

}  // namespace dgemm

void dgemm_handler(RunMode runMode, int argc, char* argv[]) {
  const char* tune_file = getenv("LIBTHOM_TUNE_FILE");
  if (runMode != RunMode::TUNE && tune_file != nullptr) lt_tuner_load(tune_file);
  switch (runMode) {
    case RunMode::TEST: dgemm::testHandler(argc, argv); break;
    case RunMode::BENCH: dgemm::benchHandler(argc, argv); break;
    case RunMode::TUNE: dgemm::tuneHandler(argc, argv); break;
  }
}
