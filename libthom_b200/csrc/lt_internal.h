// lt_internal.h — declarations shared between the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace lt {

int last_error();
const char* last_message();

namespace fp64 {
bool tma_compatible(const double* A, const double* B, int64_t N, int64_t K);
int num_configs();
const char* config_name(int i);
bool config_is_tma(int i);
int heuristic_config(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int sm_count);
int run_config(int cfg, const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
               double beta, cudaStream_t stream);
}  // namespace fp64

namespace tuner {
// Tuned FP64 config for this shape class, or -1.
int lookup(int64_t M, int64_t N, int64_t K, bool tma);
}  // namespace tuner

namespace ozaki {
size_t workspace_size(int64_t M, int64_t N, int64_t K, int slices);
int split(const double* A, const double* B, int64_t M, int64_t N, int64_t K, int slices, void* workspace,
          size_t workspace_bytes, cudaStream_t stream);
int product(double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta, int slices, const void* workspace,
            size_t workspace_bytes, cudaStream_t stream);
int run(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta,
        int slices, void* workspace, size_t workspace_bytes, cudaStream_t stream);
}  // namespace ozaki

}  // namespace lt
