// lt_runtime.cuh — host-side runtime shared by the C ABI: error state, per-device context
// (device status word, SM count, TMA descriptor encoder), cached workspace, CUDA checks.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "lt_common.cuh"

namespace lt {

// Records `code` (and a printf-style message) as the calling thread's last error; returns code.
int set_error(int code, const char* fmt, ...);
int ok();

struct DeviceContext {
  int device = -1;
  int sm_count = 0;
  int cc_major = 0, cc_minor = 0;
  size_t smem_optin = 0;
  DeviceStatus* status = nullptr;  // device memory, one per device
  void* workspace = nullptr;       // cached Ozaki workspace (grown on demand)
  size_t workspace_bytes = 0;
  void* splitk = nullptr;          // cached partial sums of K-split FP64 launches
  size_t splitk_bytes = 0;
  void* transposed = nullptr;      // cached transposed operands of lt_dgemm_ex (FP64 form)
  size_t transposed_bytes = 0;
  void* pack = nullptr;            // cached padded copies of HGEMM operands with unaligned pitches
  size_t pack_bytes = 0;
  void* l2_flush = nullptr;
  size_t l2_flush_bytes = 0;
};

// Context of the current device, created on first use. Returns nullptr (error recorded) on failure.
DeviceContext* context();
// Context of device `dev` if one has been created, else nullptr (nothing is created or recorded).
DeviceContext* existing_context(int dev);
// Ensures the cached workspace of the current device holds at least `bytes`.
int ensure_workspace(DeviceContext* ctx, size_t bytes, void** ptr);
// Same for the FP64 K-split partial sums (a buffer of its own).
int ensure_splitk_workspace(DeviceContext* ctx, size_t bytes, void** ptr);
// Same for the transposed operands of lt_dgemm_ex's FP64 form.
int ensure_transpose_workspace(DeviceContext* ctx, size_t bytes, void** ptr);
// Same for the padded operand copies of the HGEMM.
int ensure_pack_workspace(DeviceContext* ctx, size_t bytes, void** ptr);

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled();

// 2-D row-major tensor map: rows x cols elements of `elem_bytes`, row pitch `pitch_bytes`,
// box {box_cols, box_rows}, 128-byte swizzle unless given, zero fill out of bounds.
int make_tmap_2d(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, int elem_bytes, uint64_t rows,
                 uint64_t cols, uint64_t pitch_bytes, uint32_t box_rows, uint32_t box_cols,
                 CUtensorMapSwizzle swizzle = CU_TENSOR_MAP_SWIZZLE_128B);
// 3-D: [planes][rows][cols] with plane pitch and row pitch in bytes, box {box_cols, box_rows, 1}.
int make_tmap_3d(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, int elem_bytes, uint64_t planes,
                 uint64_t rows, uint64_t cols, uint64_t pitch_bytes, uint64_t plane_pitch_bytes, uint32_t box_rows,
                 uint32_t box_cols, CUtensorMapSwizzle swizzle);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace lt

#define LT_CUDA_TRY(call)                                                                          \
  do {                                                                                             \
    cudaError_t lt_e_ = (call);                                                                    \
    if (lt_e_ != cudaSuccess)                                                                      \
      return ::lt::set_error(LT_ERR_CUDA, "%s failed at %s:%d: %s", #call, __FILE__, __LINE__,   \
                             cudaGetErrorString(lt_e_));                                           \
  } while (0)

#define LT_TRY(call)                 \
  do {                               \
    int lt_rc_ = (call);             \
    if (lt_rc_ != LT_OK) return lt_rc_; \
  } while (0)
