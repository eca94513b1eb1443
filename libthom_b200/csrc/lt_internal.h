// lt_internal.h — declarations shared between the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/libthom_dgemm.h"

namespace lt {

struct DeviceStatus;  // lt_common.cuh

int last_error();
const char* last_message();

namespace fp64 {
bool tma_compatible(const double* A, const double* B, int64_t N, int64_t K);
int num_configs();
const char* config_name(int i);
bool config_is_tma(int i);
int heuristic_config(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int sm_count);
int heuristic_config_for(int64_t M, int64_t N, int64_t K, int sm_count, bool tma);
// Scratch of a caller for the partial sums of the K split and stream-K schedules, instead of the
// growable per-device cache (whose reallocation would leave a captured graph pointing at freed memory):
// with `query` set nothing is launched and the bytes needed are reported there; otherwise `ptr` (at
// least `bytes`, null when the schedule needs none) is used.
struct ScratchUse {
  void* ptr;
  size_t bytes;
  size_t* query;
};
int run_config(int cfg, const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
               double beta, cudaStream_t stream, const ScratchUse* scratch = nullptr);
// Same with row strides (lda >= K, ldb >= N, ldc >= N).
int run_config_ld(int cfg, const double* A, int64_t lda, const double* B, int64_t ldb, double* C, int64_t ldc, int64_t M,
                  int64_t N, int64_t K, double alpha, double beta, cudaStream_t stream,
                  const ScratchUse* scratch = nullptr);
}  // namespace fp64

// Selector statistics (selector_stats.cu). selector_infer: the features of one problem (copied to
// feat_dev, 34 floats, when given) and, with the network's device parameters, its class
// probabilities (into probs_host, when given); synchronous, one call at a time per process.
// gap_into needs 8 (M + N) bytes of scratch and a zeroed pair of ints at `out` (row gap, column gap).
int selector_infer(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol, const float* params,
                   float* feat_dev, float* probs_host, cudaStream_t stream);
int gap_into(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int* out, void* scratch,
             cudaStream_t stream);
// Native FP64 DGEMM with the tuned or heuristic tile configuration (capi.cu); scratch as for
// fp64::run_config (null: the per-device cache).
int dgemm_fp64_dispatch(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                        double beta, int config, cudaStream_t stream, const fp64::ScratchUse* scratch);
// A plan's own feature scratch (selector_stats.cu): size, initial state, the two feature kernels
// without host synchronisation, and the device address of the class probabilities they leave.
size_t selector_scratch_bytes();
int selector_scratch_init(void* scratch, cudaStream_t stream);
int selector_features_async(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol,
                            const float* params, void* scratch, cudaStream_t stream);
const float* selector_probs(const void* scratch);

namespace tuner {
// Tuned FP64 config for this shape class, or -1.
int lookup(int64_t M, int64_t N, int64_t K, bool tma);
}  // namespace tuner

namespace ozaki {
size_t workspace_size(int64_t M, int64_t N, int64_t K, int slices);
// Row maxima of A (M x K, pitch K) and column maxima of B (K x N, pitch N) as IEEE bits, one launch;
// M, N, K > 0 and both arrays zero on entry.
int exponents(const double* A, const double* B, int64_t M, int64_t N, int64_t K, unsigned long long* amax_a,
              unsigned long long* amax_b, int sms, cudaStream_t stream);
// The same for one side, with a row stride.
int exponents_rows(const double* A, int64_t M, int64_t K, int64_t lda, unsigned long long* amax, int sms,
                   cudaStream_t stream);
int exponents_cols(const double* B, int64_t K, int64_t N, int64_t ldb, unsigned long long* amax, int sms,
                   cudaStream_t stream);
int split(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int slices, void* workspace,
          size_t workspace_bytes, cudaStream_t stream);
int product(double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int slices, const void* workspace,
            size_t workspace_bytes, cudaStream_t stream);
int run(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta,
        int slices, void* workspace, size_t workspace_bytes, cudaStream_t stream);
int run_ex(bool trans_a, bool trans_b, const double* A, int64_t lda, const double* B, int64_t ldb, double* C, int64_t ldc,
           int64_t M, int64_t N, int64_t K, double alpha, double beta, int s, void* workspace, size_t workspace_bytes,
           cudaStream_t stream);
int host_run(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
             double beta, int slices, cudaStream_t stream);
int noalloc_run(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                double beta, int slices, cudaStream_t stream);
// The allocation-free path's device error word (a static device variable): its address on device
// `dev` (performing that path's per-device set-up), and a read-and-clear of it that reports zero
// when the path was never set up on `dev`.
int noalloc_status_word(int dev, DeviceStatus** st);
int noalloc_take_status(int dev, DeviceStatus* out);
struct Grouped;
int grouped_create(const lt_gemm_problem* problems, int count, int slices, Grouped** out);
int grouped_run(const Grouped* G, cudaStream_t stream);
int grouped_prepare(const Grouped* G);
void grouped_destroy(Grouped* G);
int64_t grouped_tiles(const Grouped* G);
}  // namespace ozaki

namespace fp64 {
struct GroupedFp64;
int grouped_num_configs();
const char* grouped_config_name(int cfg);
int grouped_create(const lt_gemm_problem* problems, int count, int cfg, GroupedFp64** out);
int grouped_run(const GroupedFp64* G, cudaStream_t stream);
int grouped_prepare(const GroupedFp64* G);
void grouped_destroy(GroupedFp64* G);
int64_t grouped_tiles(const GroupedFp64* G);
}  // namespace fp64

}  // namespace lt
