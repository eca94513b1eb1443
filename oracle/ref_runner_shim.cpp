// ref_runner_shim.cpp — the reference's own runner driving this library's entry points: a test
// program that compiles routines/dgemm/dgemm.cpp where it lies (include path set by oracle/Makefile;
// nothing of it is copied), performs dgemm_handler's set-up (routines/dgemm/dgemm.cpp:228-231: cuRAND
// generator seeded with 1234, cuBLAS handle) and hands an implementation of include/libthom_dgemm.h to
// dgemm::runner (dgemm.cpp:168-205) with the runner's result check on. The runner fills the inputs
// with cuRAND, calls the implementation through its DgemmImpl pointer, and compares every element
// against its host loop (dgemm.cpp:137-159), printing "Number of different results: n" when any
// differs. Test infrastructure only.
//
//     ref_runner <impl> M N K          (impl: tc100, ozaki7, ozaki_crt15, cublas_tc, ...)
#include "routines/dgemm/dgemm.cpp"

#include <type_traits>

#include "libthom_dgemm.h"

// The library's reference-contract entry points have the reference's implementation type.
#define LT_SAME_TYPE(fn) static_assert(std::is_same<decltype(&fn), dgemm::DgemmImpl>::value, #fn " is not a DgemmImpl")
LT_SAME_TYPE(dgemm_tc100);
LT_SAME_TYPE(dgemm_ozaki3);
LT_SAME_TYPE(dgemm_ozaki4);
LT_SAME_TYPE(dgemm_ozaki5);
LT_SAME_TYPE(dgemm_ozaki6);
LT_SAME_TYPE(dgemm_ozaki7);
LT_SAME_TYPE(dgemm_ozaki8);
LT_SAME_TYPE(dgemm_ozaki9);
LT_SAME_TYPE(dgemm_ozaki10);
LT_SAME_TYPE(dgemm_ozaki_auto);
LT_SAME_TYPE(dgemm_auto);
LT_SAME_TYPE(dgemm_cublas_tc);
LT_SAME_TYPE(dgemm_ozaki_crt14);
LT_SAME_TYPE(dgemm_ozaki_crt15);
LT_SAME_TYPE(dgemm_ozaki_crt16);
LT_SAME_TYPE(dgemm_ozaki_crt17);
LT_SAME_TYPE(dgemm_ozaki_crt18);

static const std::map<std::string, dgemm::DgemmImpl> kImpls = {
    {"tc100", dgemm_tc100},         {"ozaki7", dgemm_ozaki7},           {"ozaki8", dgemm_ozaki8},
    {"ozaki_auto", dgemm_ozaki_auto}, {"auto", dgemm_auto},             {"cublas_tc", dgemm_cublas_tc},
    {"ozaki_crt14", dgemm_ozaki_crt14}, {"ozaki_crt15", dgemm_ozaki_crt15}, {"ozaki_crt16", dgemm_ozaki_crt16},
};

int main(int argc, char* argv[]) {
  if (argc != 5 || kImpls.find(argv[1]) == kImpls.end()) {
    fprintf(stderr, "usage: ref_runner <impl> M N K\n");
    return 2;
  }
  CURAND_CHECK(curandCreateGenerator(&dgemm::gen, CURAND_RNG_PSEUDO_DEFAULT));
  CURAND_CHECK(curandSetPseudoRandomGeneratorSeed(dgemm::gen, 1234ULL));
  CUBLAS_CHECK(cublasCreate(&dgemm::cublasHandle));
  std::vector<int> sizes = {atoi(argv[2]), atoi(argv[3]), atoi(argv[4])};
  // two timed runs after one warm-up, each checked against the host loop
  const float gflops = dgemm::runner(kImpls.at(argv[1]), sizes, 2, 1, true, false, argc, argv);
  printf("[ref_runner] %s %d %d %d: %f GFLOP/s, library status %d\n", argv[1], sizes[0], sizes[1], sizes[2], gflops,
         lt_get_last_error());
  CURAND_CHECK(curandDestroyGenerator(dgemm::gen));
  CUBLAS_CHECK(cublasDestroy(dgemm::cublasHandle));
  return lt_get_last_error() == LT_OK ? 0 : 1;
}
