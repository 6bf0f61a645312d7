// The sizing MLP's parameter layout and its one-vector forward pass, shared
// by the MLP kernels (mlp.cu) and the kernels that fold a prediction into
// their own work (the learned join's init, join.cu).
#pragma once

#include "common.cuh"
#include "bespoke_gpu.h"

namespace bo {

constexpr int kH = 64;       // hidden width
constexpr int kMaxF = 32;    // features
constexpr int kMaxO = 4;     // outputs
constexpr int kPredThreads = 256;

struct MlpLayout {
  int F, O;
  int w1, b1, w2, b2, w3, b3, w4, b4, P;
};

__host__ __device__ inline MlpLayout mlp_layout(int F, int O) {
  MlpLayout L;
  L.F = F;
  L.O = O;
  L.w1 = 0;
  L.b1 = L.w1 + F * kH;
  L.w2 = L.b1 + kH;
  L.b2 = L.w2 + kH * kH;
  L.w3 = L.b2 + kH;
  L.b3 = L.w3 + kH * kH;
  L.w4 = L.b3 + kH;
  L.b4 = L.w4 + kH * O;
  L.P = L.b4 + O;
  return L;
}

struct FeatureVec {
  float f[kMaxF];
};

// The network's outputs y[0..O) (log1p of the predicted counts) for one
// feature vector, computed by one block of kPredThreads threads (all must
// call it); y is shared memory, valid in every thread on return.  Thread
// (j, part) owns hidden unit j's partial dot products over inputs
// i = part (mod 4); every weight the thread uses is loaded into registers up
// front (all loads independent: one memory latency), and only the 64-wide
// activations move through shared memory between layers.
__device__ __forceinline__ void mlp_predict_block(const float* __restrict__ params, const FeatureVec& xv, int F,
                                                  int O, float* y) {
  __shared__ float a[2][kH];
  const MlpLayout L = mlp_layout(F, O);
  const int j = threadIdx.x >> 2, part = threadIdx.x & 3;
  float w1[kMaxF / 4], w2[kH / 4], w3[kH / 4], w4[2 * kMaxO];
#pragma unroll
  for (int k = 0; k < kMaxF / 4; ++k) {
    const int i = part + 4 * k;
    w1[k] = i < F ? __ldg(params + L.w1 + i * kH + j) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < kH / 4; ++k) {
    w2[k] = __ldg(params + L.w2 + (part + 4 * k) * kH + j);
    w3[k] = __ldg(params + L.w3 + (part + 4 * k) * kH + j);
  }
  const float b1 = __ldg(params + L.b1 + j), b2 = __ldg(params + L.b2 + j), b3 = __ldg(params + L.b3 + j);
  const int t = threadIdx.x;
#pragma unroll
  for (int o = 0; o < kMaxO; ++o) {
    w4[2 * o] = (t < 32 && o < O) ? __ldg(params + L.w4 + t * O + o) : 0.0f;
    w4[2 * o + 1] = (t < 32 && o < O) ? __ldg(params + L.w4 + (t + 32) * O + o) : 0.0f;
  }
  const float b4 = t < O ? __ldg(params + L.b4 + t) : 0.0f;
  if (t < kMaxF) a[1][t] = t < F ? xv.f[t] : 0.0f;
  __syncthreads();
  // layer 1: inputs a[1][0..F)
  float z = 0.0f;
#pragma unroll
  for (int k = 0; k < kMaxF / 4; ++k) z = fmaf(a[1][part + 4 * k], w1[k], z);
  z += __shfl_xor_sync(0xffffffffu, z, 1);
  z += __shfl_xor_sync(0xffffffffu, z, 2);
  z += b1;
  __syncthreads();
  if (part == 0) a[0][j] = z > 0.0f ? z : 0.0f;
  __syncthreads();
  // layer 2: a[0] -> a[1]
  z = 0.0f;
#pragma unroll
  for (int k = 0; k < kH / 4; ++k) z = fmaf(a[0][part + 4 * k], w2[k], z);
  z += __shfl_xor_sync(0xffffffffu, z, 1);
  z += __shfl_xor_sync(0xffffffffu, z, 2);
  z += b2;
  if (part == 0) a[1][j] = z > 0.0f ? z : 0.0f;
  __syncthreads();
  // layer 3: a[1] -> a[0]
  z = 0.0f;
#pragma unroll
  for (int k = 0; k < kH / 4; ++k) z = fmaf(a[1][part + 4 * k], w3[k], z);
  z += __shfl_xor_sync(0xffffffffu, z, 1);
  z += __shfl_xor_sync(0xffffffffu, z, 2);
  z += b3;
  if (part == 0) a[0][j] = z > 0.0f ? z : 0.0f;
  __syncthreads();
  if (t < 32) {
#pragma unroll
    for (int o = 0; o < kMaxO; ++o) {
      if (o >= O) break;
      float v = fmaf(a[0][t], w4[2 * o], 0.0f);
      v = fmaf(a[0][t + 32], w4[2 * o + 1], v);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      const float bo = __shfl_sync(0xffffffffu, b4, o);
      if (t == 0) y[o] = v + bo;
    }
  }
  __syncthreads();
}

// Device parameters and sizes of a host-side model handle.
int mlp_view(const bo_mlp* m, const float** params, int* F, int* O);

}  // namespace bo
