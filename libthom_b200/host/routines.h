// routines.h — host harness of the `libthom` CLI: run modes, routine handlers and shared helpers.
//
// Mirrors the reference's dispatch (main.cpp:10-72, enums.h:4-8, routines/routines.h:86-170):
// `libthom <test|bench|tune> <routine> <impl> [args]`, one handler per routine, a runner per routine
// that times one implementation call and optionally checks it. Implementations are the C ABI of
// liblibthom_dgemm.so (include/libthom_dgemm.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

#include "libthom_dgemm.h"

enum RunMode { TEST, BENCH, TUNE };

void dgemm_handler(RunMode runMode, int argc, char* argv[]);
void dgemmb_handler(RunMode runMode, int argc, char* argv[]);
void hgemm_handler(RunMode runMode, int argc, char* argv[]);


// Reference behaviour kept: a CUDA error is reported as a warning and the run continues
// (routines/routines.h:44-51); library errors additionally carry the library's message.
#define CUDA_CHECK(error)                                                                               \
  do {                                                                                                  \
    cudaError_t check_cuda_error_ = (error);                                                            \
    if (check_cuda_error_ != cudaSuccess)                                                               \
      fprintf(stderr, "WARNING: CUDA error at %s:%d: %s\n", __FILE__, __LINE__,                        \
              cudaGetErrorString(check_cuda_error_));                                                   \
  } while (0)

#define LT_CHECK(call)                                                                                  \
  do {                                                                                                  \
    int lt_rc_ = (call);                                                                                \
    if (lt_rc_ != LT_OK) {                                                                              \
      fprintf(stderr, "libthom_dgemm error %d (%s) at %s:%d: %s\n", lt_rc_, lt_error_string(lt_rc_),   \
              __FILE__, __LINE__, lt_last_error_message());                                             \
      exit(EXIT_FAILURE);                                                                               \
    }                                                                                                   \
  } while (0)

// Flushes L2 by writing twice its size (routines/common.cpp:12-24).
void flushL2();
double envDouble(const char* name, double def);
long envLong(const char* name, long def);
double median(std::vector<double> v);
