// selector.cu — learned slice-count selector for the Ozaki DGEMM (no reference counterpart).
//
// Features (34 floats per problem, computed in selector_stats.cu): a 16-bin histogram of exponent
// gaps in sampled rows of A, the same for sampled columns of B, log2 K / 16 and -log10(tol) / 16. The
// gap of a nonzero entry is how many binades it sits below the largest entry of its row (column):
// g = e(max) - e(x), bins of width 4 (g >= 60 in the last bin); zeros count in bin 0. The gap is what
// the per-row power-of-two scaling costs in precision, so the histograms carry what decides the
// slice count.
//
// Network: 34 -> 64 -> 64 -> 8, GELU (tanh form: 0.5 x (1 + tanh(sqrt(2/pi)(x + 0.044715 x^3)))),
// softmax over slice counts 3..10, cross-entropy loss, Adam. Forward, backward and the optimizer
// step are hand-written kernels: one block per sample for forward/backward (per-sample gradients
// written to a buffer), then a fixed-order reduction over the batch, so gradients are deterministic.
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "lt_internal.h"
#include "lt_runtime.cuh"
#include "selector_common.cuh"

namespace lt {
namespace sel {

__global__ void mlp_forward_kernel(const float* __restrict__ p, const float* __restrict__ x, int batch,
                                   float* __restrict__ probs) {
  __shared__ Acts s;
  const int b = blockIdx.x;
  if (b >= batch) return;
  forward_block(p, x + static_cast<int64_t>(b) * F, s);
  if (threadIdx.x < C) probs[static_cast<int64_t>(b) * C + threadIdx.x] = s.prob[threadIdx.x];
}

// Per-sample gradient of the cross-entropy loss into g[b][P]; per-sample loss into loss_b[b].
__global__ void mlp_backward_kernel(const float* __restrict__ p, const float* __restrict__ x,
                                    const int* __restrict__ labels, int batch, float* __restrict__ g,
                                    float* __restrict__ loss_b) {
  __shared__ Acts s;
  __shared__ float d3[C], d2[H], d1[H];
  const int b = blockIdx.x, t = threadIdx.x;
  if (b >= batch) return;
  forward_block(p, x + static_cast<int64_t>(b) * F, s);
  const int y = labels[b];
  float* gb = g + static_cast<int64_t>(b) * P;
  if (t < C) d3[t] = s.prob[t] - (t == y ? 1.f : 0.f);
  if (t == 0) loss_b[b] = -logf(fmaxf(s.prob[y], 1e-30f));
  __syncthreads();
  // layer 3
  for (int i = t; i < C * H; i += blockDim.x) gb[OW3 + i] = d3[i / H] * s.a2[i % H];
  if (t < C) gb[OB3 + t] = d3[t];
  if (t < H) {
    float acc = 0.f;
    for (int c = 0; c < C; ++c) acc += p[OW3 + c * H + t] * d3[c];
    d2[t] = acc * gelu_grad(s.h2[t]);
  }
  __syncthreads();
  // layer 2
  for (int i = t; i < H * H; i += blockDim.x) gb[OW2 + i] = d2[i / H] * s.a1[i % H];
  if (t < H) gb[OB2 + t] = d2[t];
  if (t < H) {
    float acc = 0.f;
    for (int j = 0; j < H; ++j) acc += p[OW2 + j * H + t] * d2[j];
    d1[t] = acc * gelu_grad(s.h1[t]);
  }
  __syncthreads();
  // layer 1
  for (int i = t; i < H * F; i += blockDim.x) gb[OW1 + i] = d1[i / F] * s.x[i % F];
  if (t < H) gb[OB1 + t] = d1[t];
}

// grads[i] = mean over the batch of g[b][i] (fixed summation order); loss = mean of loss_b.
__global__ void reduce_grads_kernel(const float* __restrict__ g, const float* __restrict__ loss_b, int batch,
                                    float* __restrict__ grads, float* __restrict__ loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const float inv = 1.f / static_cast<float>(batch);
  if (i < P) {
    float acc = 0.f;
    for (int b = 0; b < batch; ++b) acc += g[static_cast<int64_t>(b) * P + i];
    grads[i] = acc * inv;
  }
  if (i == 0 && loss != nullptr) {
    float acc = 0.f;
    for (int b = 0; b < batch; ++b) acc += loss_b[b];
    *loss = acc * inv;
  }
}

__global__ void adam_kernel(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Scratch for training (per device): per-sample gradients and losses.
struct Scratch {
  float* g = nullptr;
  float* loss_b = nullptr;
  int cap = 0;
};
std::mutex g_mutex;
Scratch g_scratch[64];
std::vector<float> g_host_params;  // installed selector weights (empty = none)
float* g_dev_params[64] = {};
bool g_dev_params_valid[64] = {};
double g_tol = 1e-15;

int ensure_scratch(int batch, Scratch** out) {
  int dev = 0;
  LT_CUDA_TRY(cudaGetDevice(&dev));
  Scratch& s = g_scratch[dev];
  if (s.cap < batch) {
    if (s.g) cudaFree(s.g);
    if (s.loss_b) cudaFree(s.loss_b);
    s.g = nullptr;
    s.loss_b = nullptr;
    s.cap = 0;
    LT_CUDA_TRY(cudaMalloc(&s.g, sizeof(float) * static_cast<size_t>(batch) * P));
    LT_CUDA_TRY(cudaMalloc(&s.loss_b, sizeof(float) * batch));
    s.cap = batch;
  }
  *out = &s;
  return LT_OK;
}

int backward(const float* params, const float* x, const int* labels, int batch, float* grads, float* loss,
             cudaStream_t stream) {
  Scratch* s = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    LT_TRY(ensure_scratch(batch, &s));
  }
  mlp_backward_kernel<<<batch, H, 0, stream>>>(params, x, labels, batch, s->g, s->loss_b);
  LT_CUDA_TRY(cudaGetLastError());
  reduce_grads_kernel<<<(P + 255) / 256, 256, 0, stream>>>(s->g, s->loss_b, batch, grads, loss);
  LT_CUDA_TRY(cudaGetLastError());
  return LT_OK;
}

// Conservative slice count. With gap_bits = (largest exponent gap within a row of A) + (largest
// within a column of B), every entry a keeps at least 8s - 2 - g_a - 1 bits after truncation, so the
// two truncated tails and the dropped pairs p + q > s + 1 (at most s + 1 of them matter) bound the
// componentwise error by (s + 3) 2^(gap_bits + 4 - 8s) relative to |A||B|; the FP64 recombination
// and the alpha/beta epilogue add at most 4u (the diagonal terms shrink by 2^-8 each).
double analytic_bound(int s, int gap_bits) {
  return (s + 3) * ldexp(1.0, gap_bits + 4 - 8 * s) + 4.0 * ldexp(1.0, -53);
}

int analytic(double tol, int gap_bits) {
  for (int s = 1; s <= LT_OZAKI_MAX_SLICES; ++s)
    if (analytic_bound(s, gap_bits) <= tol) return s;
  return LT_OZAKI_MAX_SLICES;
}

// Trained weights shipped beside the library (selector_weights.bin, LT_SEL_PARAMS floats), or the
// file named by LIBTHOM_SELECTOR_WEIGHTS; loaded once unless the caller installed weights (or
// explicitly none) with lt_selector_set_params.
bool g_params_explicit = false;
std::once_flag g_default_once;

void load_default_params() {
  std::call_once(g_default_once, [] {
    std::string path;
    if (const char* env = getenv("LIBTHOM_SELECTOR_WEIGHTS")) {
      path = env;
    } else {
      Dl_info info;
      if (dladdr(reinterpret_cast<void*>(&load_default_params), &info) != 0 && info.dli_fname != nullptr) {
        path = info.dli_fname;
        size_t slash = path.find_last_of('/');
        path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) + "/selector_weights.bin";
      }
    }
    if (path.empty()) return;
    FILE* f = fopen(path.c_str(), "rb");
    if (f == nullptr) return;
    std::vector<float> w(P);
    size_t n = fread(w.data(), sizeof(float), P, f);
    char extra;
    bool exact = n == static_cast<size_t>(P) && fread(&extra, 1, 1, f) == 0;
    fclose(f);
    std::lock_guard<std::mutex> lock(g_mutex);
    if (exact && !g_params_explicit) {
      g_host_params = w;
      for (int d = 0; d < 64; ++d) g_dev_params_valid[d] = false;
    }
  });
}

int device_params(const float** out) {
  int dev = 0;
  LT_CUDA_TRY(cudaGetDevice(&dev));
  load_default_params();
  std::lock_guard<std::mutex> lock(g_mutex);
  if (g_host_params.empty()) {
    *out = nullptr;
    return LT_OK;
  }
  if (!g_dev_params_valid[dev]) {
    if (g_dev_params[dev] == nullptr) LT_CUDA_TRY(cudaMalloc(&g_dev_params[dev], sizeof(float) * P));
    LT_CUDA_TRY(cudaMemcpy(g_dev_params[dev], g_host_params.data(), sizeof(float) * P, cudaMemcpyHostToDevice));
    g_dev_params_valid[dev] = true;
  }
  *out = g_dev_params[dev];
  return LT_OK;
}

// Learned choice from the network's class probabilities (slice counts 3..10, the last class
// standing for "10 or more"): the smallest count whose cumulative probability reaches kQuantile, if
// the network is confident (top class >= 0.5) and neither the top class nor that count is the last
// class. Returns false when the analytic fallback must decide. kQuantile = 0.999: on 800 held-out
// problems (2 400 problem-tolerance pairs, selector_train's distribution) it misses the tolerance on
// none of the reachable ones, as the analytic count does, and picks 8.2 / 9.7 / 11.9 slices on average
// at 1e-12 / 1e-14 / 1e-15 against the analytic 12.0; the 0.9 quantile saved 0.2 more slices but
// missed on 11 and 6 reachable problems at 1e-12 and 1e-14.
constexpr float kQuantile = 0.999f;
bool decide(const float* probs, int* slices) {
  int top = 0;
  for (int c = 1; c < C; ++c)
    if (probs[c] > probs[top]) top = c;
  if (!(probs[top] >= 0.5f) || top == C - 1) return false;
  float cdf = 0.f;
  for (int c = 0; c < C - 1; ++c) {
    cdf += probs[c];
    if (cdf >= kQuantile) {
      *slices = 3 + c;
      return true;
    }
  }
  return false;
}

// Slice count for one problem (synchronous: the count decides the workspace layout and launches).
// The exponent-gap pass that feeds the analytic count runs only when the learned choice is not
// used; *gap_bits is -1 then.
int select(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol, int* slices,
           bool* learned, int* gap_bits, cudaStream_t stream) {
  DeviceContext* ctx = context();
  if (ctx == nullptr) return last_error();
  const float* params = nullptr;
  LT_TRY(device_params(&params));
  *learned = false;
  *gap_bits = -1;
  const size_t head = 256;
  uint8_t* d = nullptr;
  int rc = LT_OK;
  cudaError_t e = cudaSuccess;
  if (params != nullptr) {
    float hp[C];
    rc = selector_infer(A, B, M, N, K, tol, params, nullptr, hp, stream);
    if (rc == LT_OK) *learned = decide(hp, slices);
  }
  if (rc == LT_OK && !*learned) e = cudaMallocAsync(reinterpret_cast<void**>(&d), head + 8 * (M + N), stream);
  int* gap = reinterpret_cast<int*>(d);  // 2 ints
  if (rc == LT_OK && e == cudaSuccess && !*learned) {
    e = cudaMemsetAsync(gap, 0, 2 * sizeof(int), stream);
    if (e == cudaSuccess) rc = gap_into(A, B, M, N, K, gap, d + head, stream);
    int hg[2] = {0, 0};
    if (rc == LT_OK && e == cudaSuccess) e = cudaMemcpyAsync(hg, gap, sizeof hg, cudaMemcpyDeviceToHost, stream);
    if (rc == LT_OK && e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (rc == LT_OK && e == cudaSuccess) {
      *gap_bits = hg[0] + hg[1];
      *slices = analytic(tol, *gap_bits);
    }
  }
  if (d != nullptr) cudaFreeAsync(d, stream);
  if (rc != LT_OK) return rc;
  if (e != cudaSuccess) return set_error(LT_ERR_CUDA, "slice selection: %s", cudaGetErrorString(e));
  return LT_OK;
}

}  // namespace sel
}  // namespace lt

extern "C" {

int lt_mlp_forward(const float* params, const float* x, int batch, float* probs, void* stream) {
  if (params == nullptr || x == nullptr || probs == nullptr || batch <= 0)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_mlp_forward: bad arguments");
  if (lt::context() == nullptr) return lt::last_error();
  lt::sel::mlp_forward_kernel<<<batch, LT_SEL_HIDDEN, 0, lt::as_stream(stream)>>>(params, x, batch, probs);
  LT_CUDA_TRY(cudaGetLastError());
  return lt::ok();
}

int lt_mlp_backward(const float* params, const float* x, const int* labels, int batch, float* grads, float* loss,
                    void* stream) {
  if (params == nullptr || x == nullptr || labels == nullptr || grads == nullptr || batch <= 0)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_mlp_backward: bad arguments");
  if (lt::context() == nullptr) return lt::last_error();
  LT_TRY(lt::sel::backward(params, x, labels, batch, grads, loss, lt::as_stream(stream)));
  return lt::ok();
}

int lt_mlp_train_step(float* params, float* m, float* v, float* grads, const float* x, const int* labels, int batch,
                      float lr, int step, float* loss, void* stream) {
  if (params == nullptr || m == nullptr || v == nullptr || grads == nullptr || x == nullptr || labels == nullptr ||
      batch <= 0 || step < 1 || !(lr > 0.f))
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_mlp_train_step: bad arguments");
  if (lt::context() == nullptr) return lt::last_error();
  cudaStream_t s = lt::as_stream(stream);
  LT_TRY(lt::sel::backward(params, x, labels, batch, grads, loss, s));
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, static_cast<float>(step)), c2 = 1.f - powf(b2, static_cast<float>(step));
  lt::sel::adam_kernel<<<(LT_SEL_PARAMS + 255) / 256, 256, 0, s>>>(params, m, v, grads, lr, b1, b2, 1e-8f, c1, c2);
  LT_CUDA_TRY(cudaGetLastError());
  return lt::ok();
}

int lt_selector_set_params(const float* host_params) {
  std::lock_guard<std::mutex> lock(lt::sel::g_mutex);
  lt::sel::g_params_explicit = true;
  if (host_params == nullptr) {
    lt::sel::g_host_params.clear();
  } else {
    lt::sel::g_host_params.assign(host_params, host_params + LT_SEL_PARAMS);
  }
  for (int d = 0; d < 64; ++d) lt::sel::g_dev_params_valid[d] = false;
  return lt::ok();
}

void lt_set_ozaki_tolerance(double tol) {
  if (tol > 0.0) lt::sel::g_tol = tol;
}

int lt_ozaki_analytic_slices(double tol, int gap_bits) {
  if (!(tol > 0.0) || gap_bits < 0) {
    lt::set_error(LT_ERR_INVALID_ARGUMENT, "bad tolerance or gap");
    return 0;
  }
  return lt::sel::analytic(tol, gap_bits);
}

int lt_ozaki_select_slices(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol, int* slices,
                           void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || A == nullptr || B == nullptr || slices == nullptr || !(tol > 0.0))
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_ozaki_select_slices: bad arguments");
  bool learned = false;
  int gap = 0;
  LT_TRY(lt::sel::select(A, B, M, N, K, tol, slices, &learned, &gap, lt::as_stream(stream)));
  return lt::ok();
}

int lt_ozaki_select_info(const double* A, const double* B, int64_t M, int64_t N, int64_t K, double tol, int* slices,
                         int* learned, int* gap_bits, void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || A == nullptr || B == nullptr || slices == nullptr || !(tol > 0.0))
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_ozaki_select_info: bad arguments");
  bool l = false;
  int g = 0;
  LT_TRY(lt::sel::select(A, B, M, N, K, tol, slices, &l, &g, lt::as_stream(stream)));
  if (learned) *learned = l ? 1 : 0;
  if (gap_bits) *gap_bits = g;
  return lt::ok();
}

float dgemm_ozaki_auto(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha,
                       double beta) {
  cudaEvent_t start, stop;
  cudaEventCreate(&start);
  cudaEventCreate(&stop);
  cudaEventRecord(start, 0);
  int rc = LT_OK;
  int s = 0;
  if (M > 0 && N > 0 && K > 0)
    rc = lt_ozaki_select_slices(A, B, static_cast<int64_t>(M), static_cast<int64_t>(N), static_cast<int64_t>(K),
                                lt::sel::g_tol, &s, nullptr);
  if (rc == LT_OK)
    rc = lt_dgemm_ozaki(A, B, C, static_cast<int64_t>(M), static_cast<int64_t>(N), static_cast<int64_t>(K), alpha,
                        beta, s > 0 ? s : 1, nullptr);
  cudaEventRecord(stop, 0);
  cudaEventSynchronize(stop);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, start, stop);
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  if (rc == LT_OK) rc = lt_check_device_status();
  if (rc != LT_OK) {
    fprintf(stderr, "Kernel launch error (ozaki_auto): %s: %s\n", lt_error_string(rc), lt::last_message());
    lt::set_error(rc, "%s", lt::last_message());
  }
  return ms;
}

}  // extern "C"

// ---- automatic form: native FP64 or Ozaki, whichever this GPU runs faster (no reference counterpart)
namespace lt {
namespace sel {

// Predicted milliseconds of one DGEMM in `form` on a B200 (148 SMs), from rates measured on it.
// FP64: 128x64 tiles at 34.4 TF/s over the padded tile work; with fewer than 148 tiles the K split
// (up to 4 ranges) spreads them over more SMs; 5 us fixed. Ozaki with s slices: exponent passes at
// 6.2 TB/s (8 bytes per element of A and B), splits at 5.1 TB/s (8 bytes read + s written), 30 us
// for the split stage's launches; then the s(s+1)/2 INT8 slice products on 256x128 CTA-pair
// tiles (128x128 tiles when M <= 128) in whole waves, each tile at 3.6 POP/s of the GPU plus 40 us
// (pipeline fill, two band drains, the FP64 epilogue), or the slice bytes at 6.0 TB/s when that is
// longer; 10 us for the launch. Predicted (measured) Ozaki s = 7 / FP64: 8192^3 10.4 (10.0-10.6) /
// 32.0 (32.0) ms; 2048^3 0.31 (0.30) / 0.50 (0.51); 1024^3 0.13 (0.12) / 0.067 (0.076);
// 65536x64x4096 2.0 (1.87) / 1.00 (1.04); 2048x2048x65536 6.2 (6.2) / 16.0 (16.0).
double estimate_ms(int form, int64_t M, int64_t N, int64_t K, int s) {
  if (M <= 0 || N <= 0 || K <= 0) return 0.0;
  auto cdiv = [](int64_t a, int64_t b) { return static_cast<double>((a + b - 1) / b); };
  constexpr double kSms = 148.0;
  if (form == LT_FORM_FP64) {
    const double tiles = cdiv(M, 128) * cdiv(N, 64);
    const double work = 2.0 * tiles * 128.0 * 64.0 * cdiv(K, 16) * 16.0;
    const double busy = std::min(1.0, 4.0 * tiles / kSms);
    return work / (34.4e12 * busy) * 1e3 + 0.005;
  }
  const bool pair = M > 128;
  const double tm = pair ? 256.0 : 128.0, slots = pair ? kSms / 2 : kSms;
  const double tiles = cdiv(M, static_cast<int64_t>(tm)) * cdiv(N, 128);
  const double waves = std::ceil(tiles / slots);
  const double products = s * (s + 1) / 2.0;
  const double t_tile = products * 2.0 * tm * 128.0 * cdiv(K, 32) * 32.0 / (3.6e15 / slots) + 40e-6;
  const double elems = static_cast<double>(M) * K + static_cast<double>(K) * N;
  const double t_prod = std::max(waves * t_tile, s * elems / 6.0e12) + 10e-6;
  return (8.0 * elems / 6.2e12 + (8.0 + s) * elems / 5.1e12 + 30e-6 + t_prod) * 1e3;
}

constexpr double kSelectMs = 0.035;  // the learned selector: statistics, network, one host read

int run_auto(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha, double beta,
             int* form_out, int* slices_out, cudaStream_t stream) {
  int form = LT_FORM_FP64, s = 0;
  // The selector is skipped when native FP64 wins even against the fewest slices.
  if (M > 0 && N > 0 && K > 0 &&
      estimate_ms(LT_FORM_OZAKI, M, N, K, 3) + kSelectMs < estimate_ms(LT_FORM_FP64, M, N, K, 0)) {
    bool learned = false;
    int gap = 0;
    LT_TRY(select(A, B, M, N, K, g_tol, &s, &learned, &gap, stream));
    if (estimate_ms(LT_FORM_OZAKI, M, N, K, s) < estimate_ms(LT_FORM_FP64, M, N, K, 0)) form = LT_FORM_OZAKI;
  }
  if (form == LT_FORM_OZAKI) {
    LT_TRY(lt_dgemm_ozaki(A, B, C, M, N, K, alpha, beta, s, stream));
  } else {
    s = 0;
    LT_TRY(lt_dgemm_fp64(A, B, C, M, N, K, alpha, beta, stream));
  }
  if (form_out) *form_out = form;
  if (slices_out) *slices_out = s;
  return LT_OK;
}

}  // namespace sel
}  // namespace lt

extern "C" {

double lt_dgemm_estimate_ms(int form, int64_t M, int64_t N, int64_t K, int slices) {
  if ((form != LT_FORM_FP64 && form != LT_FORM_OZAKI) || (form == LT_FORM_OZAKI && (slices < 1 || slices > 12)))
    return -1.0;
  return lt::sel::estimate_ms(form, M, N, K, slices);
}

int lt_dgemm_auto(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K, double alpha,
                  double beta, int* form, int* slices, void* stream) {
  if (M < 0 || N < 0 || K < 0) return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_dgemm_auto: negative size");
  LT_TRY(lt::sel::run_auto(A, B, C, M, N, K, alpha, beta, form, slices, lt::as_stream(stream)));
  return lt::ok();
}

float dgemm_auto(const double* A, const double* B, double* C, size_t M, size_t N, size_t K, double alpha,
                 double beta) {
  cudaEvent_t start, stop;
  cudaEventCreate(&start);
  cudaEventCreate(&stop);
  cudaEventRecord(start, 0);
  int rc = lt_dgemm_auto(A, B, C, static_cast<int64_t>(M), static_cast<int64_t>(N), static_cast<int64_t>(K), alpha,
                         beta, nullptr, nullptr, nullptr);
  cudaEventRecord(stop, 0);
  cudaEventSynchronize(stop);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, start, stop);
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  if (rc == LT_OK) rc = lt_check_device_status();
  if (rc != LT_OK) {
    fprintf(stderr, "Kernel launch error (auto): %s: %s\n", lt_error_string(rc), lt::last_message());
    lt::set_error(rc, "%s", lt::last_message());
  }
  return ms;
}

}  // extern "C"

// ---- slice selection on the device: a CUDA graph with conditional nodes (no reference counterpart)
// One plan per problem (pointers and sizes, like a grouped plan; the data may change between runs).
// Its graph runs the sampled-feature kernels and the network, then
//   decide_learned: the learned count if the network is confident (the same rule as `decide`),
//                   otherwise it turns on the IF node below;
//   IF (not confident): the exponent-gap pass over all of A and B;
//   decide_final: the analytic count from the gaps when the network was not confident; sets the
//                 SWITCH node's value to the body for that count;
//   SWITCH: body s (1..LT_OZAKI_MAX_SLICES) runs the slice form's split and product with s slices,
//           body 0 the native FP64 kernel.
// So the choice never leaves the device: one graph launch per call, no host synchronisation. With
// forms = LT_AUTO_PLAN_OZAKI the result is what lt_ozaki_select_slices followed by lt_dgemm_ozaki
// computes (same rule, same kernels); with LT_AUTO_PLAN_ANY_FORM the count is mapped to body 0 where
// the cost model of lt_dgemm_auto (estimate_ms) predicts native FP64 faster than that many slices, and
// a shape where FP64 wins even against 3 slices gets a plan of the FP64 kernel alone (no selection),
// as lt_dgemm_auto skips the selector there.
namespace lt {
namespace sel {

__device__ bool decide_dev(const float* probs, int* slices) {
  int top = 0;
  for (int c = 1; c < C; ++c)
    if (probs[c] > probs[top]) top = c;
  if (!(probs[top] >= 0.5f) || top == C - 1) return false;
  float cdf = 0.f;
  for (int c = 0; c < C - 1; ++c) {
    cdf += probs[c];
    if (cdf >= kQuantile) {
      *slices = 3 + c;
      return true;
    }
  }
  return false;
}

__device__ int analytic_dev(double tol, int gap_bits) {
  for (int s = 1; s <= LT_OZAKI_MAX_SLICES; ++s)
    if ((s + 3) * ldexp(1.0, gap_bits + 4 - 8 * s) + 4.0 * ldexp(1.0, -53) <= tol) return s;
  return LT_OZAKI_MAX_SLICES;
}

// decision = {slices, learned}; the gap pair is zeroed for the fallback pass.
__global__ void auto_decide_learned_kernel(const float* probs, int use_net, int* decision, int* gap,
                                           cudaGraphConditionalHandle fallback) {
  int s = 0;
  const bool learned = use_net != 0 && decide_dev(probs, &s);
  decision[0] = s;
  decision[1] = learned ? 1 : 0;
  gap[0] = 0;
  gap[1] = 0;
  cudaGraphSetConditional(fallback, learned ? 0u : 1u);
}

// body_of[s]: the switch body that runs s slices (s itself), or 0, native FP64, where the cost model
// predicts it faster; decision[2] = the body taken.
__global__ void auto_decide_final_kernel(double tol, int* decision, const int* gap, const int* body_of,
                                         cudaGraphConditionalHandle which) {
  if (decision[1] == 0) decision[0] = analytic_dev(tol, gap[0] + gap[1]);
  decision[2] = body_of[decision[0]];
  cudaGraphSetConditional(which, static_cast<unsigned>(decision[2]));
}

}  // namespace sel
}  // namespace lt

struct lt_ozaki_auto_plan {
  int device = -1;
  const double* A = nullptr;
  const double* B = nullptr;
  double* C = nullptr;
  int64_t M = 0, N = 0, K = 0;
  uint8_t* mem = nullptr;  // weights | feature scratch | gap scratch | gap pair, decision | slice workspace
  void* fp64_scratch = nullptr;  // partial sums of the FP64 body's K split / stream-K schedule, if any
  int* decision = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

// Adds a conditional node after the work captured so far on `s` and makes it the capture's only
// dependency; its body graphs are returned through `bodies`.
int add_conditional(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                    unsigned size, cudaGraph_t** bodies) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  LT_CUDA_TRY(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &ndeps));
  if (st != cudaStreamCaptureStatusActive) return lt::set_error(LT_ERR_CUDA, "auto plan: capture not active");
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = type;
  p.conditional.size = size;
  cudaGraphNode_t node;
  LT_CUDA_TRY(cudaGraphAddNode(&node, g, deps, ndeps, &p));
  LT_CUDA_TRY(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  *bodies = p.conditional.phGraph_out;
  return LT_OK;
}

// Captures fn(stream) into the (empty) body graph `body` on stream `s`.
template <class F>
int capture_body(cudaStream_t s, cudaGraph_t body, F fn) {
  LT_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  const int rc = fn(s);
  cudaGraph_t out = body;
  const cudaError_t e = cudaStreamEndCapture(s, &out);
  if (rc != LT_OK) return rc;
  LT_CUDA_TRY(e);
  return LT_OK;
}

int build_auto_plan(lt_ozaki_auto_plan* p, double alpha, double beta, double tol, int forms, cudaStream_t s,
                    cudaStream_t sb) {
  const float* shared_params = nullptr;
  LT_TRY(lt::sel::device_params(&shared_params));
  const size_t par_bytes = (sizeof(float) * lt::sel::P + 255) / 256 * 256;
  const size_t sc_bytes = (lt::selector_scratch_bytes() + 255) / 256 * 256;
  const size_t gap_bytes = (8 * static_cast<size_t>(p->M + p->N) + 255) / 256 * 256;
  const size_t ws_bytes = lt_ozaki_workspace_size(p->M, p->N, p->K, LT_OZAKI_MAX_SLICES);
  LT_CUDA_TRY(cudaMalloc(&p->mem, par_bytes + sc_bytes + gap_bytes + 256 + ws_bytes));
  // the plan keeps the weights installed when it was created
  float* params = shared_params != nullptr ? reinterpret_cast<float*>(p->mem) : nullptr;
  void* sc = p->mem + par_bytes;
  void* gap_scratch = p->mem + par_bytes + sc_bytes;
  int* gap = reinterpret_cast<int*>(p->mem + par_bytes + sc_bytes + gap_bytes);
  p->decision = gap + 2;                  // {slices, learned, body}
  int* body_of = gap + 8;                 // LT_OZAKI_MAX_SLICES + 1 ints
  void* ws = p->mem + par_bytes + sc_bytes + gap_bytes + 256;
  const int64_t M0 = p->M, N0 = p->N, K0 = p->K;
  const double t64 = lt::sel::estimate_ms(LT_FORM_FP64, M0, N0, K0, 0);
  int host_body[LT_OZAKI_MAX_SLICES + 1] = {0};
  for (int sl = 1; sl <= LT_OZAKI_MAX_SLICES; ++sl)
    host_body[sl] = (forms == LT_AUTO_PLAN_ANY_FORM && !(lt::sel::estimate_ms(LT_FORM_OZAKI, M0, N0, K0, sl) < t64)) ? 0 : sl;
  // native FP64 alone when it wins even against the fewest slices (as lt_dgemm_auto)
  const bool fp64_only = forms == LT_AUTO_PLAN_ANY_FORM &&
                         !(lt::sel::estimate_ms(LT_FORM_OZAKI, M0, N0, K0, 3) + lt::sel::kSelectMs < t64);
  if (params != nullptr)
    LT_CUDA_TRY(cudaMemcpyAsync(params, shared_params, sizeof(float) * lt::sel::P, cudaMemcpyDeviceToDevice, s));
  LT_TRY(lt::selector_scratch_init(sc, s));
  LT_CUDA_TRY(cudaMemsetAsync(gap, 0, 256, s));
  LT_CUDA_TRY(cudaMemcpyAsync(body_of, host_body, sizeof host_body, cudaMemcpyHostToDevice, s));
  LT_CUDA_TRY(cudaStreamSynchronize(s));
  const double *A = p->A, *B = p->B;
  double* C = p->C;
  const int64_t M = p->M, N = p->N, K = p->K;
  // The FP64 body keeps lt_dgemm_fp64's schedule with scratch of the plan's own (the per-device cache
  // may be reallocated after the capture).
  lt::fp64::ScratchUse fp64_scratch{nullptr, 0, nullptr};
  if (forms == LT_AUTO_PLAN_ANY_FORM) {
    size_t need = 0;
    lt::fp64::ScratchUse q{nullptr, 0, &need};
    LT_TRY(lt::dgemm_fp64_dispatch(A, B, C, M, N, K, alpha, beta, -1, s, &q));
    if (need > 0) LT_CUDA_TRY(cudaMalloc(&p->fp64_scratch, need));
    fp64_scratch = lt::fp64::ScratchUse{p->fp64_scratch, need, nullptr};
  }
  auto run_fp64 = [&](cudaStream_t st) {
    return lt::dgemm_fp64_dispatch(A, B, C, M, N, K, alpha, beta, -1, st, &fp64_scratch);
  };
  if (fp64_only) {  // decision stays {0, 0, 0}: native FP64
    LT_CUDA_TRY(cudaGraphCreate(&p->graph, 0));
    LT_TRY(capture_body(s, p->graph, run_fp64));
    LT_CUDA_TRY(cudaGraphInstantiate(&p->exec, p->graph, 0));
    return LT_OK;
  }

  LT_CUDA_TRY(cudaGraphCreate(&p->graph, 0));
  cudaGraphConditionalHandle h_fallback, h_slices;
  LT_CUDA_TRY(cudaGraphConditionalHandleCreate(&h_fallback, p->graph, 1, cudaGraphCondAssignDefault));
  // default: no body (a value past the switch's bodies), set by decide_final on every run
  LT_CUDA_TRY(cudaGraphConditionalHandleCreate(&h_slices, p->graph, LT_OZAKI_MAX_SLICES, cudaGraphCondAssignDefault));

  LT_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, p->graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  int rc = LT_OK;
  cudaGraph_t* fb_body = nullptr;
  cudaGraph_t* sw_bodies = nullptr;
  if (params != nullptr) rc = lt::selector_features_async(A, B, M, N, K, tol, params, sc, s);
  if (rc == LT_OK) {
    lt::sel::auto_decide_learned_kernel<<<1, 1, 0, s>>>(lt::selector_probs(sc), params != nullptr ? 1 : 0,
                                                       p->decision, gap, h_fallback);
    if (cudaGetLastError() != cudaSuccess) rc = lt::set_error(LT_ERR_CUDA, "auto plan: decide launch");
  }
  if (rc == LT_OK) rc = add_conditional(s, h_fallback, cudaGraphCondTypeIf, 1, &fb_body);
  if (rc == LT_OK) {
    lt::sel::auto_decide_final_kernel<<<1, 1, 0, s>>>(tol, p->decision, gap, body_of, h_slices);
    if (cudaGetLastError() != cudaSuccess) rc = lt::set_error(LT_ERR_CUDA, "auto plan: decide launch");
  }
  if (rc == LT_OK) rc = add_conditional(s, h_slices, cudaGraphCondTypeSwitch, LT_OZAKI_MAX_SLICES + 1, &sw_bodies);
  cudaGraph_t captured = p->graph;
  const cudaError_t e = cudaStreamEndCapture(s, &captured);
  if (rc != LT_OK) return rc;
  LT_CUDA_TRY(e);

  LT_TRY(capture_body(sb, fb_body[0],
                      [&](cudaStream_t st) { return lt::gap_into(A, B, M, N, K, gap, gap_scratch, st); }));
  bool any_fp64 = false;
  for (int sl = 1; sl <= LT_OZAKI_MAX_SLICES; ++sl) any_fp64 = any_fp64 || host_body[sl] == 0;
  if (any_fp64)
    LT_TRY(capture_body(sb, sw_bodies[0], run_fp64));
  for (int sl = 1; sl <= LT_OZAKI_MAX_SLICES; ++sl) {
    if (host_body[sl] != sl) continue;  // that count runs native FP64
    LT_TRY(capture_body(sb, sw_bodies[sl], [&](cudaStream_t st) {
      int r = lt_ozaki_split(A, B, M, N, K, sl, ws, ws_bytes, st);
      if (r == LT_OK) r = lt_ozaki_product(C, M, N, K, alpha, beta, sl, ws, ws_bytes, st);
      return r;
    }));
  }
  LT_CUDA_TRY(cudaGraphInstantiate(&p->exec, p->graph, 0));
  return LT_OK;
}

void destroy_auto_plan(lt_ozaki_auto_plan* p) {
  if (p == nullptr) return;
  if (p->exec != nullptr) cudaGraphExecDestroy(p->exec);
  if (p->graph != nullptr) cudaGraphDestroy(p->graph);
  if (p->mem != nullptr) cudaFree(p->mem);
  if (p->fp64_scratch != nullptr) cudaFree(p->fp64_scratch);
  delete p;
}

}  // namespace

extern "C" {

int lt_ozaki_auto_plan_create(const double* A, const double* B, double* C, int64_t M, int64_t N, int64_t K,
                              double alpha, double beta, double tol, int forms, lt_ozaki_auto_plan** plan) {
  if (plan == nullptr) return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_ozaki_auto_plan_create: null plan");
  *plan = nullptr;
  if (M <= 0 || N <= 0 || K <= 0 || A == nullptr || B == nullptr || C == nullptr || !(tol > 0.0) ||
      (forms != LT_AUTO_PLAN_OZAKI && forms != LT_AUTO_PLAN_ANY_FORM))
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_ozaki_auto_plan_create: bad arguments");
  if (((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(C)) & 7) != 0)
    return lt::set_error(LT_ERR_UNALIGNED, "matrix pointers must be 8-byte aligned");
  lt::DeviceContext* ctx = lt::context();
  if (ctx == nullptr) return lt::last_error();
  auto* p = new lt_ozaki_auto_plan;
  p->device = ctx->device;
  p->A = A;
  p->B = B;
  p->C = C;
  p->M = M;
  p->N = N;
  p->K = K;
  cudaStream_t s = nullptr, sb = nullptr;
  int rc = LT_OK;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&sb, cudaStreamNonBlocking) != cudaSuccess)
    rc = lt::set_error(LT_ERR_CUDA, "auto plan: stream creation");
  if (rc == LT_OK) rc = build_auto_plan(p, alpha, beta, tol, forms, s, sb);
  if (s != nullptr) cudaStreamDestroy(s);
  if (sb != nullptr) cudaStreamDestroy(sb);
  if (rc != LT_OK) {
    destroy_auto_plan(p);
    return rc;
  }
  *plan = p;
  return lt::ok();
}

int lt_ozaki_auto_plan_run(lt_ozaki_auto_plan* plan, void* stream) {
  if (plan == nullptr || plan->exec == nullptr)
    return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_ozaki_auto_plan_run: no plan");
  LT_CUDA_TRY(cudaGraphLaunch(plan->exec, lt::as_stream(stream)));
  return lt::ok();
}

int lt_ozaki_auto_plan_choice(lt_ozaki_auto_plan* plan, int* slices, int* learned) {
  if (plan == nullptr) return lt::set_error(LT_ERR_INVALID_ARGUMENT, "lt_ozaki_auto_plan_choice: no plan");
  int h[3] = {0, 0, 0};
  LT_CUDA_TRY(cudaMemcpy(h, plan->decision, sizeof h, cudaMemcpyDeviceToHost));
  if (slices != nullptr) *slices = h[2] == 0 ? 0 : h[0];  // 0: native FP64 ran
  if (learned != nullptr) *learned = h[1];
  return lt::ok();
}

void lt_ozaki_auto_plan_destroy(lt_ozaki_auto_plan* plan) { destroy_auto_plan(plan); }

}  // extern "C"
