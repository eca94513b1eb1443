// lt_runtime.cu — error state, per-device contexts, workspace cache, TMA descriptor encoding.
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "lt_internal.h"
#include "lt_runtime.cuh"

namespace lt {

namespace {
thread_local int t_last_error = LT_OK;
thread_local char t_last_message[512] = "";
std::mutex g_ctx_mutex;
DeviceContext g_ctx[64];
EncodeTiledFn g_encode = nullptr;
}  // namespace

int set_error(int code, const char* fmt, ...) {
  t_last_error = code;
  if (fmt != nullptr) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_last_message, sizeof t_last_message, fmt, ap);
    va_end(ap);
  } else {
    t_last_message[0] = '\0';
  }
  return code;
}

int ok() {
  t_last_error = LT_OK;
  t_last_message[0] = '\0';
  return LT_OK;
}

int last_error() { return t_last_error; }
const char* last_message() { return t_last_message; }

DeviceContext* context() {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    set_error(LT_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_ctx_mutex);
  DeviceContext& c = g_ctx[dev];
  if (c.device == dev) return &c;
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) {
    set_error(LT_ERR_CUDA, "cudaGetDeviceProperties failed: %s", cudaGetErrorString(e));
    return nullptr;
  }
  if (prop.major != 10) {
    set_error(LT_ERR_UNSUPPORTED, "device %d is sm_%d%d; this library is built for sm_100a only", dev, prop.major,
              prop.minor);
    return nullptr;
  }
  DeviceStatus* st = nullptr;
  e = cudaMalloc(&st, sizeof(DeviceStatus));
  if (e != cudaSuccess) {
    set_error(LT_ERR_NO_MEMORY, "device status allocation failed: %s", cudaGetErrorString(e));
    return nullptr;
  }
  e = cudaMemset(st, 0, sizeof(DeviceStatus));
  if (e != cudaSuccess) {
    cudaFree(st);
    set_error(LT_ERR_CUDA, "device status init failed: %s", cudaGetErrorString(e));
    return nullptr;
  }
  c.sm_count = prop.multiProcessorCount;
  c.cc_major = prop.major;
  c.cc_minor = prop.minor;
  c.smem_optin = prop.sharedMemPerBlockOptin;
  c.status = st;
  c.device = dev;
  return &c;
}

DeviceContext* existing_context(int dev) {
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(g_ctx_mutex);
  return g_ctx[dev].device == dev ? &g_ctx[dev] : nullptr;
}

namespace {
// Grows a cached device buffer to at least `bytes` (12.5 % headroom); the old buffer may still be in
// use by work queued on any stream, so growing synchronises the device first.
int ensure_buffer(void** buf, size_t* have, size_t bytes, void** ptr) {
  if (*have < bytes) {
    if (*buf != nullptr) {
      LT_CUDA_TRY(cudaDeviceSynchronize());
      cudaFree(*buf);
      *buf = nullptr;
      *have = 0;
    }
    size_t grow = bytes + bytes / 8;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, grow);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_error(LT_ERR_NO_MEMORY, "workspace allocation of %zu bytes failed: %s", grow, cudaGetErrorString(e));
    }
    *buf = p;
    *have = grow;
  }
  *ptr = *buf;
  return LT_OK;
}
}  // namespace

int ensure_workspace(DeviceContext* ctx, size_t bytes, void** ptr) {
  return ensure_buffer(&ctx->workspace, &ctx->workspace_bytes, bytes, ptr);
}

int ensure_splitk_workspace(DeviceContext* ctx, size_t bytes, void** ptr) {
  return ensure_buffer(&ctx->splitk, &ctx->splitk_bytes, bytes, ptr);
}

int ensure_transpose_workspace(DeviceContext* ctx, size_t bytes, void** ptr) {
  return ensure_buffer(&ctx->transposed, &ctx->transposed_bytes, bytes, ptr);
}

int ensure_pack_workspace(DeviceContext* ctx, size_t bytes, void** ptr) {
  return ensure_buffer(&ctx->pack, &ctx->pack_bytes, bytes, ptr);
}

EncodeTiledFn encode_tiled() {
  if (g_encode != nullptr) return g_encode;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
  if (e != cudaSuccess || fn == nullptr || q != cudaDriverEntryPointSuccess) {
    set_error(LT_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled not available");
    return nullptr;
  }
  g_encode = reinterpret_cast<EncodeTiledFn>(fn);
  return g_encode;
}

int make_tmap_2d(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, int elem_bytes, uint64_t rows,
                 uint64_t cols, uint64_t pitch_bytes, uint32_t box_rows, uint32_t box_cols, CUtensorMapSwizzle swizzle) {
  EncodeTiledFn enc = encode_tiled();
  if (enc == nullptr) return LT_ERR_UNSUPPORTED;
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (pitch_bytes & 15) != 0)
    return set_error(LT_ERR_UNALIGNED, "tensor map base/pitch not 16-byte aligned");
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {pitch_bytes};
  cuuint32_t box[2] = {box_cols, box_rows};
  cuuint32_t estr[2] = {1, 1};
  (void)elem_bytes;
  CUresult r = enc(map, dtype, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(LT_ERR_CUDA, "cuTensorMapEncodeTiled (2d) failed: %d", static_cast<int>(r));
  return LT_OK;
}

int make_tmap_3d(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, int elem_bytes, uint64_t planes,
                 uint64_t rows, uint64_t cols, uint64_t pitch_bytes, uint64_t plane_pitch_bytes, uint32_t box_rows,
                 uint32_t box_cols, CUtensorMapSwizzle swizzle) {
  EncodeTiledFn enc = encode_tiled();
  if (enc == nullptr) return LT_ERR_UNSUPPORTED;
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (pitch_bytes & 15) != 0 || (plane_pitch_bytes & 15) != 0)
    return set_error(LT_ERR_UNALIGNED, "tensor map base/pitch not 16-byte aligned");
  cuuint64_t dims[3] = {cols, rows, planes};
  cuuint64_t strides[2] = {pitch_bytes, plane_pitch_bytes};
  cuuint32_t box[3] = {box_cols, box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  (void)elem_bytes;
  CUresult r = enc(map, dtype, 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(LT_ERR_CUDA, "cuTensorMapEncodeTiled (3d) failed: %d", static_cast<int>(r));
  return LT_OK;
}

// Failure-detection self-test: thread 0 waits, through the pipelines' bounded wait, on an mbarrier
// that nothing arrives at. After `limit_ns` the wait gives up and records LT_ERR_DEVICE_TIMEOUT
// (tag 99) in the device status word, as a stalled pipeline stage would; the kernel then returns.
// The other warp waits on the same barrier and must leave through the raised abort flag, as the
// other roles of a pipeline do. Nothing faults or traps.
__global__ void wait_timeout_selftest_kernel(uint64_t limit_ns, DeviceStatus* st) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_wait_for(&bar, 0, &abort_flag, st, 99, limit_ns);
  } else if (threadIdx.x == 32) {
    // gives up only through the abort flag (or, failing that, after twice the limit, tag 98)
    mbar_wait_for(&bar, 0, &abort_flag, st, 98, 2 * limit_ns);
  }
}

}  // namespace lt

extern "C" {

int lt_get_last_error(void) { return lt::last_error(); }

const char* lt_last_error_message(void) { return lt::last_message(); }

const char* lt_error_string(int code) {
  switch (code) {
    case LT_OK: return "ok";
    case LT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case LT_ERR_UNALIGNED: return "unaligned pointer";
    case LT_ERR_CUDA: return "CUDA error";
    case LT_ERR_NO_MEMORY: return "out of memory / workspace too small";
    case LT_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    case LT_ERR_UNSUPPORTED: return "unsupported device or feature";
    case LT_ERR_NOT_FOUND: return "not found";
    default: return "unknown error";
  }
}

int lt_check_device_status(void) {
  // Two words can hold a report on the current device: the context's (every allocating entry
  // point) and the allocation-free path's static one. Neither is created here, so a caller that
  // only uses lt_dgemm_ozaki_noalloc still allocates nothing.
  int dev = -1;
  LT_CUDA_TRY(cudaGetDevice(&dev));
  lt::DeviceStatus st{0, 0, 0, 0};
  const char* which = "";
  if (lt::DeviceContext* ctx = lt::existing_context(dev)) {
    LT_CUDA_TRY(cudaMemcpy(&st, ctx->status, sizeof st, cudaMemcpyDeviceToHost));
    if (st.code != 0) LT_CUDA_TRY(cudaMemset(ctx->status, 0, sizeof st));
  }
  lt::DeviceStatus na{0, 0, 0, 0};
  LT_TRY(lt::ozaki::noalloc_take_status(dev, &na));
  if (st.code == 0 && na.code != 0) {
    st = na;
    which = " in the allocation-free path";
  }
  if (st.code != 0)
    return lt::set_error(st.code, "device wait gave up%s (tag %d, block %d)", which, st.where, st.block);
  return LT_OK;
}

int lt_selftest_wait_timeout(double limit_ms, void* stream) {
  if (!(limit_ms >= 0.001 && limit_ms <= 1000.0))
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "wait limit %g ms outside [0.001, 1000]", limit_ms);
  lt::DeviceContext* ctx = lt::context();
  if (ctx == nullptr) return lt::last_error();
  lt::wait_timeout_selftest_kernel<<<1, 64, 0, lt::as_stream(stream)>>>(static_cast<uint64_t>(limit_ms * 1e6),
                                                                         ctx->status);
  LT_CUDA_TRY(cudaGetLastError());
  return lt::ok();
}

int lt_selftest_wait_timeout_noalloc(double limit_ms, void* stream) {
  if (!(limit_ms >= 0.001 && limit_ms <= 1000.0))
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "wait limit %g ms outside [0.001, 1000]", limit_ms);
  int dev = -1;
  LT_CUDA_TRY(cudaGetDevice(&dev));
  lt::DeviceStatus* st = nullptr;
  LT_TRY(lt::ozaki::noalloc_status_word(dev, &st));
  lt::wait_timeout_selftest_kernel<<<1, 64, 0, lt::as_stream(stream)>>>(static_cast<uint64_t>(limit_ms * 1e6), st);
  LT_CUDA_TRY(cudaGetLastError());
  return lt::ok();
}

int lt_version(void) { return 100; }

int lt_flush_l2(void* stream) {
  lt::DeviceContext* ctx = lt::context();
  if (ctx == nullptr) return lt::last_error();
  if (ctx->l2_flush == nullptr) {
    int l2 = 0;
    LT_CUDA_TRY(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, ctx->device));
    ctx->l2_flush_bytes = 2 * static_cast<size_t>(l2);
    LT_CUDA_TRY(cudaMalloc(&ctx->l2_flush, ctx->l2_flush_bytes));
  }
  LT_CUDA_TRY(cudaMemsetAsync(ctx->l2_flush, 0, ctx->l2_flush_bytes, lt::as_stream(stream)));
  return lt::ok();
}

}  // extern "C"
