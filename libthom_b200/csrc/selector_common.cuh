// selector_common.cuh — pieces shared by the selector's kernels (selector.cu, selector_stats.cu):
// the MLP's parameter layout and forward pass, and the exponent-gap statistics' helpers.
#pragma once
#include <cmath>
#include <cstdint>

#include "lt_common.cuh"

namespace lt {
namespace sel {

constexpr int F = LT_SEL_FEATURES, H = LT_SEL_HIDDEN, C = LT_SEL_CLASSES, P = LT_SEL_PARAMS;
constexpr int OW1 = 0, OB1 = OW1 + H * F, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + C * H;
static_assert(OB3 + C == P, "parameter layout");
// ---------------------------------------------------------------------------------------------
// MLP
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float gelu(float x) {
  const float k = 0.7978845608028654f;  // sqrt(2/pi)
  float t = tanhf(k * (x + 0.044715f * x * x * x));
  return 0.5f * x * (1.f + t);
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float k = 0.7978845608028654f;
  float u = k * (x + 0.044715f * x * x * x);
  float t = tanhf(u);
  return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * k * (1.f + 3.f * 0.044715f * x * x);
}

struct Acts {
  float x[F], h1[H], a1[H], h2[H], a2[H], logit[C], prob[C];
};

// Block of H threads computes one sample's forward pass into shared memory.
__device__ __forceinline__ void forward_block(const float* __restrict__ p, const float* __restrict__ x, Acts& s) {
  const int t = threadIdx.x;
  for (int i = t; i < F; i += blockDim.x) s.x[i] = x[i];
  __syncthreads();
  if (t < H) {
    float acc = p[OB1 + t];
    for (int i = 0; i < F; ++i) acc += p[OW1 + t * F + i] * s.x[i];
    s.h1[t] = acc;
    s.a1[t] = gelu(acc);
  }
  __syncthreads();
  if (t < H) {
    float acc = p[OB2 + t];
    for (int i = 0; i < H; ++i) acc += p[OW2 + t * H + i] * s.a1[i];
    s.h2[t] = acc;
    s.a2[t] = gelu(acc);
  }
  __syncthreads();
  if (t < C) {
    float acc = p[OB3 + t];
    for (int i = 0; i < H; ++i) acc += p[OW3 + t * H + i] * s.a2[i];
    s.logit[t] = acc;
  }
  __syncthreads();
  if (t == 0) {
    float mx = s.logit[0];
    for (int c = 1; c < C; ++c) mx = fmaxf(mx, s.logit[c]);
    float sum = 0.f;
    for (int c = 0; c < C; ++c) {
      s.prob[c] = expf(s.logit[c] - mx);
      sum += s.prob[c];
    }
    for (int c = 0; c < C; ++c) s.prob[c] /= sum;
  }
  __syncthreads();
}

constexpr int kSampleRows = 128;  // rows of A sampled for the features (evenly spaced)
constexpr int kColGroups = 4;     // groups of 32 consecutive columns of B sampled for the features
constexpr int kNone = -0x7f7f7f80;  // memset(0x80) pattern: "no nonzero entry seen" for a max
constexpr int kNoneMin = 0x7f7f7f7f;  // memset(0x7f) pattern for a min

__device__ __forceinline__ int exp_of(double v) {
  int e;
  frexp(v, &e);
  return e;
}
__device__ __forceinline__ bool counts(double v) { return v != 0.0 && isfinite(v); }
__device__ __forceinline__ int gap_bin(int g) { return g >= 60 ? 15 : (g < 0 ? 0 : g >> 2); }

__device__ __forceinline__ int64_t sampled_row(int i, int rows, int64_t M) {
  return rows > 1 ? (static_cast<int64_t>(i) * (M - 1)) / (rows - 1) : 0;
}
__device__ __forceinline__ int64_t sampled_col0(int g, int groups, int64_t N) {
  const int64_t span = N > 32 ? N - 32 : 0;
  return groups > 1 ? (static_cast<int64_t>(g) * span) / (groups - 1) : 0;
}

}  // namespace sel
}  // namespace lt
