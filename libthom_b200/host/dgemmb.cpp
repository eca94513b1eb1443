// dgemmb.cpp — the `dgemmb` routine: many independent, unevenly sized DGEMMs in one grouped plan.
//
// No reference counterpart (the reference times one problem per call, routines/dgemm/dgemm.cpp:168-205);
// each problem keeps the reference's contract (dgemm.h:9). Problem sizes M, N, K are drawn
// log-uniform in [lo, hi] from a seeded generator; entries come from lt_fill (U[-1,1)).
//
//   libthom test  dgemmb <impl> <count> <lo> <hi> <nb_iter> [check=1]
//   libthom bench dgemmb <impl>                      (512 problems in [32, 1024], seed 1234)
//   libthom tune  dgemmb [count lo hi]               (tile shape of the FP64 grouped kernel)
// impl: fp64 (grouped FP64 tensor cores, default tiles), fp64_tuned (tiles chosen by the tuner on
// this problem set), ozaki<s> (grouped Ozaki INT8, s slices), cublas_loop (cuBLAS FP64, one call
// per problem). Plans run as CUDA graphs.
#include <cmath>
#include <cstring>
#include <fstream>

#include "routines.h"

namespace dgemmb {

struct Set {
  std::vector<lt_gemm_problem> probs;
  std::vector<double*> bufs;
  std::vector<double*> c0;
  double flops = 0.0;
};

static uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// round(exp(U[ln lo, ln hi])) from the i-th draw of the seeded stream.
static int64_t logUniform(uint64_t seed, uint64_t i, int64_t lo, int64_t hi) {
  double u = static_cast<double>(mix64(seed * 0x9E3779B97F4A7C15ull + i) >> 11) * 0x1p-53;
  double v = std::exp(std::log(static_cast<double>(lo)) + u * (std::log(static_cast<double>(hi)) - std::log(static_cast<double>(lo))));
  int64_t r = static_cast<int64_t>(std::llround(v));
  return r < lo ? lo : (r > hi ? hi : r);
}

static Set makeSet(int count, int64_t lo, int64_t hi, uint64_t seed) {
  Set s;
  for (int i = 0; i < count; ++i) {
    lt_gemm_problem p;
    p.M = logUniform(seed, 3 * i, lo, hi);
    p.N = logUniform(seed, 3 * i + 1, lo, hi);
    p.K = logUniform(seed, 3 * i + 2, lo, hi);
    double *A, *B, *C, *C0;
    CUDA_CHECK(cudaMalloc(&A, sizeof(double) * p.M * p.K));
    CUDA_CHECK(cudaMalloc(&B, sizeof(double) * p.K * p.N));
    CUDA_CHECK(cudaMalloc(&C, sizeof(double) * p.M * p.N));
    CUDA_CHECK(cudaMalloc(&C0, sizeof(double) * p.M * p.N));
    LT_CHECK(lt_fill(A, p.M * p.K, seed + i, 1, 0, nullptr));
    LT_CHECK(lt_fill(B, p.K * p.N, seed + i, 2, 0, nullptr));
    LT_CHECK(lt_fill(C0, p.M * p.N, seed + i, 3, 0, nullptr));
    CUDA_CHECK(cudaMemcpy(C, C0, sizeof(double) * p.M * p.N, cudaMemcpyDeviceToDevice));
    p.A = A;
    p.B = B;
    p.C = C;
    p.alpha = 1.0;
    p.beta = 0.0;
    s.probs.push_back(p);
    s.bufs.insert(s.bufs.end(), {A, B, C, C0});
    s.c0.push_back(C0);
    s.flops += 2.0 * static_cast<double>(p.M) * static_cast<double>(p.N) * static_cast<double>(p.K);
  }
  CUDA_CHECK(cudaDeviceSynchronize());
  return s;
}

static void freeSet(Set& s) {
  for (double* p : s.bufs) cudaFree(p);
  s = Set();
}

// Max componentwise error of every problem's C against cuBLAS FP64.
static double check(const Set& s, double tol) {
  double worst = 0.0;
  long long above = 0;
  for (const auto& p : s.probs) {
    double *R, *den;
    CUDA_CHECK(cudaMalloc(&R, sizeof(double) * p.M * p.N));
    CUDA_CHECK(cudaMalloc(&den, sizeof(double) * p.M * p.N));
    LT_CHECK(lt_dgemm_cublas(p.A, p.B, R, p.M, p.N, p.K, p.alpha, 0.0, nullptr));
    LT_CHECK(lt_abs_denominator(p.A, p.B, nullptr, den, p.M, p.N, p.K, p.alpha, 0.0, nullptr));
    double out[2];
    LT_CHECK(lt_componentwise_error(p.C, R, den, p.M * p.N, tol, out, nullptr));
    worst = out[0] > worst ? out[0] : worst;
    above += static_cast<long long>(out[1]);
    cudaFree(R);
    cudaFree(den);
  }
  printf("[check] max componentwise error vs cuBLAS FP64 over %zu problems: %.3e (%lld elements above %.1e)\n",
         s.probs.size(), worst, above, tol);
  return worst;
}

// Implementation names of the batched routine: the FP64 grouped plan (default or tuned tiles),
// the Ozaki grouped plan with a slice count, or one cuBLAS call per problem. Checked before any
// device memory is touched, like the reference's registry lookup (routines/routines.h:108, 149).
static bool knownImpl(const std::string& impl) {
  if (impl == "fp64" || impl == "fp64_tuned" || impl == "cublas_loop") return true;
  if (impl.rfind("ozaki", 0) != 0 || impl.size() == 5 || impl.size() > 7) return false;
  for (size_t i = 5; i < impl.size(); ++i)
    if (impl[i] < '0' || impl[i] > '9') return false;
  int sl = atoi(impl.c_str() + 5);
  return sl >= 1 && sl <= LT_OZAKI_MAX_SLICES;
}

static void requireKnownImpl(const std::string& impl) {
  if (knownImpl(impl)) return;
  fprintf(stderr, "Invalid implementation %s. Available: fp64 fp64_tuned ozaki<1..%d> cublas_loop\n", impl.c_str(),
          LT_OZAKI_MAX_SLICES);
  exit(1);
}

// Median ms of `iters` timed runs (after `warmup`) of one implementation on the set.
static double runImpl(const std::string& impl, Set& s, int iters, int warmup, bool doCheck) {
  lt_grouped_plan* plan = nullptr;
  if (impl == "fp64" || impl == "fp64_tuned") {
    LT_CHECK(lt_grouped_plan_create(s.probs.data(), static_cast<int>(s.probs.size()), LT_FORM_FP64, 0, &plan));
    if (impl == "fp64_tuned") {
      float ms = 0.f;
      LT_CHECK(lt_grouped_plan_tune(plan, 5, &ms));
    }
  } else if (impl.rfind("ozaki", 0) == 0) {
    int sl = atoi(impl.c_str() + 5);
    LT_CHECK(lt_grouped_plan_create(s.probs.data(), static_cast<int>(s.probs.size()), LT_FORM_OZAKI, sl, &plan));
  } else {
    requireKnownImpl(impl);
  }
  if (plan != nullptr) {
    char name[128];
    lt_grouped_plan_config(plan, name, sizeof name);
    int64_t tiles = 0;
    lt_grouped_plan_info(plan, &tiles, nullptr);
    printf("[plan] %s, %lld tiles\n", name, static_cast<long long>(tiles));
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  std::vector<double> ts;
  for (int it = -warmup; it < iters; ++it) {
    flushL2();
    cudaEventRecord(e0);
    if (plan != nullptr) {
      LT_CHECK(lt_grouped_plan_run_graph(plan, nullptr));
    } else {
      for (const auto& p : s.probs) LT_CHECK(lt_dgemm_cublas(p.A, p.B, p.C, p.M, p.N, p.K, p.alpha, p.beta, nullptr));
    }
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    LT_CHECK(lt_check_device_status());
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (it >= 0) ts.push_back(ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (doCheck) check(s, envDouble("LIBTHOM_DGEMM_TOL", 1e-13));
  lt_grouped_plan_destroy(plan);
  return median(ts);
}

static void testHandler(int argc, char* argv[]) {
  if (argc < 8) {
    fprintf(stderr, "Usage: ./libthom test dgemmb <impl> <count> <lo> <hi> <nb_iter> [check=1]\n");
    exit(1);
  }
  std::string impl = argv[3];
  requireKnownImpl(impl);
  int count = atoi(argv[4]);
  int64_t lo = atoll(argv[5]), hi = atoll(argv[6]);
  int iters = atoi(argv[7]);
  bool doCheck = argc < 9 ? true : atoi(argv[8]) == 1;
  if (count < 1 || lo < 1 || hi < lo || iters < 1) {
    fprintf(stderr, "bad arguments\n");
    exit(1);
  }
  Set s = makeSet(count, lo, hi, static_cast<uint64_t>(envLong("LIBTHOM_DGEMM_SEED", 1234)));
  double ms = runImpl(impl, s, iters, 1, doCheck);
  printf("# %d problems, %.4g flop, median %.4f ms, GFLOP/s: %f\n", count, s.flops, ms, s.flops / (ms * 1e6));
  freeSet(s);
}

static void benchHandler(int argc, char* argv[]) {
  if (argc < 4) {
    fprintf(stderr, "Usage: ./libthom bench dgemmb <impl>\n");
    exit(1);
  }
  std::string impl = argv[3];
  requireKnownImpl(impl);
  Set s = makeSet(512, 32, 1024, 1234);
  double ms = runImpl(impl, s, 10, 5, false);
  double gf = s.flops / (ms * 1e6);
  printf("[512 problems, %.4g flop] median %.4f ms ==> %f GFLOP/s\n", s.flops, ms, gf);
  std::ofstream f(std::string("bench_dgemmb_") + impl + ".csv");
  f << "count,lo,hi,flops,ms,gflops\n512,32,1024," << s.flops << "," << ms << "," << gf << "\n";
  freeSet(s);
}

static void tuneHandler(int argc, char* argv[]) {
  int count = argc > 3 ? atoi(argv[3]) : 512;
  int64_t lo = argc > 4 ? atoll(argv[4]) : 32, hi = argc > 5 ? atoll(argv[5]) : 1024;
  if (count < 1 || lo < 1 || hi < lo) {
    fprintf(stderr, "Usage: ./libthom tune dgemmb [count=512] [lo=32] [hi=1024]\n");
    exit(1);
  }
  Set s = makeSet(count, lo, hi, 1234);
  lt_grouped_plan* plan = nullptr;
  LT_CHECK(lt_grouped_plan_create(s.probs.data(), count, LT_FORM_FP64, 0, &plan));
  float ms = 0.f;
  LT_CHECK(lt_grouped_plan_tune(plan, 5, &ms));
  char name[128];
  lt_grouped_plan_config(plan, name, sizeof name);
  printf("[best] %d problems in [%lld, %lld]: %s %.4f ms (%.1f GFLOP/s)\n", count, static_cast<long long>(lo),
         static_cast<long long>(hi), name, ms, s.flops / (ms * 1e6));
  lt_grouped_plan_destroy(plan);
  freeSet(s);
}

}  // namespace dgemmb

void dgemmb_handler(RunMode runMode, int argc, char* argv[]) {
  switch (runMode) {
    case RunMode::TEST: dgemmb::testHandler(argc, argv); break;
    case RunMode::BENCH: dgemmb::benchHandler(argc, argv); break;
    case RunMode::TUNE: dgemmb::tuneHandler(argc, argv); break;
  }
}
