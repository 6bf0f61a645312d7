// Small FP32 MLP (n_features -> 64 -> 64 -> 64 -> n_outputs, ReLU) with
// hand-written training and inference kernels.  It predicts log1p of the row
// counts the pipelines must size for (qualifying build rows, joined rows,
// distinct groups) from predicate constants and column-sketch features; the
// predictions presize hash tables and output buffers on the device, and the
// exact-count path stays both the fallback and the judge.
//
// No reference counterpart: the reference sizes its dense arrays exactly
// (e.g. bespoke_tpch/query_q3.cpp:178-180, bespoke_ceb/query_q10a.cpp:843-856).
//
// Kernels (FP32 FMA; no tensor cores -- the matrices are 64 wide):
//   mlp_fwd_bwd  one CTA per 64 samples: the parameters live in shared memory,
//                each thread runs one sample's forward pass (activations kept
//                column-major in shared memory, padded against bank conflicts),
//                then its backward pass; the CTA reduces its per-sample
//                gradients into one partial per parameter (fixed order);
//   mlp_reduce_adam  sums the CTA partials in a fixed order (bitwise
//                deterministic training) and applies one Adam step;
//   mlp_fwd_bwd<false> is the inference kernel; mlp_predict_counts writes
//                max(expm1(y), 0) for one feature vector passed by value.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "context.cuh"
#include "mlp.cuh"

struct bo_mlp {
  int F = 0, O = 0, P = 0;
  float* params = nullptr;  // device
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* grad = nullptr;     // reduced gradient (device)
  float* partials = nullptr; // [blocks][P + 1]
  int partial_blocks = 0;
  float* loss = nullptr;     // device scalar
  int64_t step = 0;
};

namespace bo {

constexpr int kTB = 64;            // samples per CTA
constexpr int kPad = kTB + 1;      // column stride of per-sample tables in shared memory

__host__ __device__ inline size_t mlp_smem_floats(int F, int O) {
  const MlpLayout L = mlp_layout(F, O);
  return (size_t)L.P + (size_t)F * kPad + 3 * (size_t)kH * kPad * 2 + (size_t)O * kPad * 2;
}

// Forward (and, when kTrain, backward + per-CTA gradient partials).
// x: [n][F], t: [n][O] log-targets; y_out (inference): [n][O].
template <bool kTrain>
__global__ void __launch_bounds__(kTB) mlp_fwd_bwd(const float* __restrict__ params, const float* __restrict__ x,
                                                   const float* __restrict__ t, int n, int F, int O,
                                                   float* __restrict__ y_out, float* __restrict__ partials) {
  extern __shared__ float sm[];
  const MlpLayout L = mlp_layout(F, O);
  float* W = sm;
  float* xs = W + L.P;                       // [F][kPad]
  float* act = xs + F * kPad;                // 3 x [kH][kPad]
  float* del = act + 3 * kH * kPad;          // 3 x [kH][kPad]
  float* ys = del + 3 * kH * kPad;           // [O][kPad]
  float* dy = ys + O * kPad;                 // [O][kPad]
  const int tid = threadIdx.x;
  const int s = blockIdx.x * kTB + tid;
  const bool valid = s < n;
  for (int i = tid; i < L.P; i += kTB) W[i] = params[i];
  for (int i = 0; i < F; ++i) xs[i * kPad + tid] = valid ? x[(size_t)s * F + i] : 0.0f;
  __syncthreads();

  // ---- forward: each thread one sample; weights read as broadcasts.
  const float* in = xs;
  int in_dim = F;
  const int wofs[3] = {L.w1, L.w2, L.w3}, bofs[3] = {L.b1, L.b2, L.b3};
#pragma unroll 1
  for (int l = 0; l < 3; ++l) {
    float* out = act + l * kH * kPad;
    const float* Wl = W + wofs[l];
    const float* bl = W + bofs[l];
    for (int j = 0; j < kH; ++j) {
      float z = bl[j];
      for (int i = 0; i < in_dim; ++i) z = fmaf(in[i * kPad + tid], Wl[i * kH + j], z);
      out[j * kPad + tid] = z > 0.0f ? z : 0.0f;
    }
    in = out;
    in_dim = kH;
  }
  const float* a3 = act + 2 * kH * kPad;
  for (int o = 0; o < O; ++o) {
    float z = W[L.b4 + o];
    for (int j = 0; j < kH; ++j) z = fmaf(a3[j * kPad + tid], W[L.w4 + j * O + o], z);
    ys[o * kPad + tid] = z;
    if (!kTrain && valid) y_out[(size_t)s * O + o] = z;
  }
  if (!kTrain) return;

  // ---- loss 0.5 * mean (y - t)^2 over samples and outputs, and dL/dy.
  const float inv = 1.0f / ((float)n * (float)O);
  float lsum = 0.0f;
  for (int o = 0; o < O; ++o) {
    const float e = valid ? ys[o * kPad + tid] - t[(size_t)s * O + o] : 0.0f;
    dy[o * kPad + tid] = e * inv;
    lsum += 0.5f * e * e * inv;
  }
  // ---- backward through the three hidden layers (per sample).
  {
    float* d3 = del + 2 * kH * kPad;
    for (int j = 0; j < kH; ++j) {
      float g = 0.0f;
      for (int o = 0; o < O; ++o) g = fmaf(W[L.w4 + j * O + o], dy[o * kPad + tid], g);
      d3[j * kPad + tid] = a3[j * kPad + tid] > 0.0f ? g : 0.0f;
    }
    for (int l = 2; l >= 1; --l) {
      const float* dn = del + l * kH * kPad;
      float* dp = del + (l - 1) * kH * kPad;
      const float* ap = act + (l - 1) * kH * kPad;
      const float* Wl = W + wofs[l];
      for (int i = 0; i < kH; ++i) {
        float g = 0.0f;
        for (int j = 0; j < kH; ++j) g = fmaf(Wl[i * kH + j], dn[j * kPad + tid], g);
        dp[i * kPad + tid] = ap[i * kPad + tid] > 0.0f ? g : 0.0f;
      }
    }
  }
  __syncthreads();
  // ---- per-CTA gradient partials: dW[i][j] = sum_t in[i][t] * delta[j][t],
  //      summed over the CTA's samples in a fixed order.
  float* part = partials + (size_t)blockIdx.x * (L.P + 1);
  for (int p = tid; p < L.P; p += kTB) {
    const float* a;
    const float* d;
    if (p < L.b1) {
      a = xs + (p / kH) * kPad;
      d = del + (p % kH) * kPad;
    } else if (p < L.w2) {
      a = nullptr;
      d = del + (p - L.b1) * kPad;
    } else if (p < L.b2) {
      const int q = p - L.w2;
      a = act + (q / kH) * kPad;
      d = del + kH * kPad + (q % kH) * kPad;
    } else if (p < L.w3) {
      a = nullptr;
      d = del + kH * kPad + (p - L.b2) * kPad;
    } else if (p < L.b3) {
      const int q = p - L.w3;
      a = act + kH * kPad + (q / kH) * kPad;
      d = del + 2 * kH * kPad + (q % kH) * kPad;
    } else if (p < L.w4) {
      a = nullptr;
      d = del + 2 * kH * kPad + (p - L.b3) * kPad;
    } else if (p < L.b4) {
      const int q = p - L.w4;
      a = act + 2 * kH * kPad + (q / O) * kPad;
      d = dy + (q % O) * kPad;
    } else {
      a = nullptr;
      d = dy + (p - L.b4) * kPad;
    }
    float g = 0.0f;
    if (a)
      for (int k = 0; k < kTB; ++k) g = fmaf(a[k], d[k], g);
    else
      for (int k = 0; k < kTB; ++k) g += d[k];
    part[p] = g;
  }
  // loss partial, fixed-order sum over the CTA
  __syncthreads();
  ys[tid] = lsum;  // reuse ys row 0 as scratch (forward outputs no longer needed)
  __syncthreads();
  if (tid == 0) {
    float l = 0.0f;
    for (int k = 0; k < kTB; ++k) l += ys[k];
    part[L.P] = l;
  }
}

// Fixed-order sum of the CTA partials, then one Adam step (or just the
// gradient when lr == 0 and grad_only).
__global__ void mlp_reduce_adam(float* __restrict__ params, float* __restrict__ m, float* __restrict__ v,
                                float* __restrict__ grad, const float* __restrict__ partials, int blocks, int P,
                                float lr, float b1, float b2, float eps, float bc1, float bc2, int grad_only,
                                float* __restrict__ loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > P) return;
  float g = 0.0f;
  for (int b = 0; b < blocks; ++b) g += partials[(size_t)b * (P + 1) + p];
  if (p == P) {
    if (loss) *loss = g;
    return;
  }
  grad[p] = g;
  if (grad_only) return;
  const float mm = b1 * m[p] + (1.0f - b1) * g;
  const float vv = b2 * v[p] + (1.0f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  params[p] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
}

// One feature vector passed by value (no host-to-device copy): predicted
// counts = max(expm1(y), 0), written to counts[0..O) (mlp_predict_block in
// mlp.cuh does the forward pass).
__global__ void __launch_bounds__(kPredThreads) mlp_predict_counts(const float* __restrict__ params, FeatureVec xv,
                                                                   int F, int O, float* __restrict__ counts,
                                                                   float* __restrict__ y_log) {
  __shared__ float y[kMaxO];
  mlp_predict_block(params, xv, F, O, y);
  const int t = threadIdx.x;
  if (t < O) {
    if (y_log) y_log[t] = y[t];
    const float c = expm1f(y[t]);
    counts[t] = c > 0.0f ? c : 0.0f;
  }
}

int mlp_view(const bo_mlp* m, const float** params, int* F, int* O) {
  if (!m || !m->params) return BO_ERR_INVALID;
  *params = m->params;
  *F = m->F;
  *O = m->O;
  return BO_OK;
}

}  // namespace bo

using namespace bo;

namespace {

int check_mlp(bo_ctx* ctx, const bo_mlp* m) {
  if (!ctx) return BO_ERR_INVALID;
  if (!m || !m->params) return set_error(ctx, BO_ERR_INVALID, "mlp: null model");
  return BO_OK;
}

int ensure_partials(bo_ctx* ctx, bo_mlp* m, int blocks) {
  if (m->partial_blocks >= blocks) return BO_OK;
  if (m->partials) cudaFree(m->partials);
  m->partials = nullptr;
  BO_CUDA(ctx, cudaMalloc(&m->partials, sizeof(float) * (size_t)blocks * (m->P + 1)));
  m->partial_blocks = blocks;
  return BO_OK;
}

int launch_fwd(bo_ctx* ctx, const bo_mlp* m, bool train, const float* x, const float* t, int n, float* y,
               float* partials) {
  const size_t smem = sizeof(float) * mlp_smem_floats(m->F, m->O);
  const void* k = train ? reinterpret_cast<const void*>(&mlp_fwd_bwd<true>)
                        : reinterpret_cast<const void*>(&mlp_fwd_bwd<false>);
  BO_CUDA(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int blocks = (n + kTB - 1) / kTB;
  if (train)
    mlp_fwd_bwd<true><<<blocks, kTB, smem, ctx->stream>>>(m->params, x, t, n, m->F, m->O, nullptr, partials);
  else
    mlp_fwd_bwd<false><<<blocks, kTB, smem, ctx->stream>>>(m->params, x, nullptr, n, m->F, m->O, y, nullptr);
  return after_launch(ctx, "mlp_fwd_bwd");
}

// Deterministic host initialisation: He-uniform weights from a xorshift stream.
std::vector<float> init_params(int F, int O, uint64_t seed) {
  const MlpLayout L = mlp_layout(F, O);
  std::vector<float> p((size_t)L.P, 0.0f);
  uint64_t s = seed * 0x9E3779B97F4A7C15ull + 0x1234567ull;
  auto uni = [&]() {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return (double)(s >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int ofs, int fan_in, int count) {
    const double lim = std::sqrt(6.0 / (double)fan_in);
    for (int i = 0; i < count; ++i) p[(size_t)ofs + i] = (float)((2.0 * uni() - 1.0) * lim);
  };
  fill(L.w1, F, F * kH);
  fill(L.w2, kH, kH * kH);
  fill(L.w3, kH, kH * kH);
  fill(L.w4, kH, kH * O);
  return p;
}

}  // namespace

extern "C" {

int bo_mlp_create(bo_ctx* ctx, int32_t n_features, int32_t n_outputs, uint64_t seed, bo_mlp** out) {
  BO_CHECK_CTX(ctx);
  if (!out) return set_error(ctx, BO_ERR_INVALID, "mlp_create: null out");
  *out = nullptr;
  if (n_features < 1 || n_features > kMaxF || n_outputs < 1 || n_outputs > kMaxO)
    return set_error(ctx, BO_ERR_INVALID, "mlp_create: features in [1,%d], outputs in [1,%d]", kMaxF, kMaxO);
  auto* m = new bo_mlp();
  m->F = n_features;
  m->O = n_outputs;
  m->P = mlp_layout(n_features, n_outputs).P;
  const size_t bytes = sizeof(float) * (size_t)m->P;
  if (cudaMalloc(&m->params, bytes) != cudaSuccess || cudaMalloc(&m->adam_m, bytes) != cudaSuccess ||
      cudaMalloc(&m->adam_v, bytes) != cudaSuccess || cudaMalloc(&m->grad, bytes) != cudaSuccess ||
      cudaMalloc(&m->loss, sizeof(float)) != cudaSuccess) {
    bo_mlp_destroy(m);
    return set_error(ctx, BO_ERR_OOM, "mlp_create: device allocation failed");
  }
  const std::vector<float> p = init_params(n_features, n_outputs, seed);
  cudaMemcpyAsync(m->params, p.data(), bytes, cudaMemcpyHostToDevice, ctx->stream);
  cudaMemsetAsync(m->adam_m, 0, bytes, ctx->stream);
  cudaMemsetAsync(m->adam_v, 0, bytes, ctx->stream);
  cudaMemsetAsync(m->grad, 0, bytes, ctx->stream);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    bo_mlp_destroy(m);
    return set_error(ctx, BO_ERR_CUDA, "mlp_create: initialisation failed");
  }
  *out = m;
  return BO_OK;
}

void bo_mlp_destroy(bo_mlp* m) {
  if (!m) return;
  cudaFree(m->params);
  cudaFree(m->adam_m);
  cudaFree(m->adam_v);
  cudaFree(m->grad);
  cudaFree(m->partials);
  cudaFree(m->loss);
  delete m;
}

int32_t bo_mlp_num_params(const bo_mlp* m) { return m ? m->P : 0; }

int bo_mlp_get_params(bo_ctx* ctx, const bo_mlp* m, float* host_out) {
  int rc = check_mlp(ctx, m);
  if (rc) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(host_out, m->params, sizeof(float) * m->P, cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return BO_OK;
}

int bo_mlp_set_params(bo_ctx* ctx, bo_mlp* m, const float* host_in) {
  int rc = check_mlp(ctx, m);
  if (rc) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(m->params, host_in, sizeof(float) * m->P, cudaMemcpyHostToDevice, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(m->adam_m, 0, sizeof(float) * m->P, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(m->adam_v, 0, sizeof(float) * m->P, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  m->step = 0;
  return BO_OK;
}

int bo_mlp_gradients_device(bo_ctx* ctx, bo_mlp* m, const float* x, const float* t, int32_t n, float* grad_device,
                            float* loss_device) {
  int rc = check_mlp(ctx, m);
  if (rc) return rc;
  if (!x || !t || n < 1 || !grad_device) return set_error(ctx, BO_ERR_INVALID, "mlp_gradients: bad argument");
  const int blocks = (n + kTB - 1) / kTB;
  if ((rc = ensure_partials(ctx, m, blocks))) return rc;
  if ((rc = launch_fwd(ctx, m, true, x, t, n, nullptr, m->partials))) return rc;
  const int threads = 256, rb = (m->P + 1 + threads - 1) / threads;
  mlp_reduce_adam<<<rb, threads, 0, ctx->stream>>>(m->params, m->adam_m, m->adam_v, grad_device, m->partials, blocks,
                                                    m->P, 0.0f, 0.9f, 0.999f, 1e-8f, 1.0f, 1.0f, 1, loss_device);
  return after_launch(ctx, "mlp_reduce_adam");
}

int bo_mlp_train_step_device(bo_ctx* ctx, bo_mlp* m, const float* x, const float* t, int32_t n, float lr,
                             float* loss_device) {
  int rc = check_mlp(ctx, m);
  if (rc) return rc;
  if (!x || !t || n < 1) return set_error(ctx, BO_ERR_INVALID, "mlp_train_step: bad argument");
  const int blocks = (n + kTB - 1) / kTB;
  if ((rc = ensure_partials(ctx, m, blocks))) return rc;
  if ((rc = launch_fwd(ctx, m, true, x, t, n, nullptr, m->partials))) return rc;
  m->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.0f - (float)std::pow((double)b1, (double)m->step);
  const float bc2 = 1.0f - (float)std::pow((double)b2, (double)m->step);
  const int threads = 256, rb = (m->P + 1 + threads - 1) / threads;
  mlp_reduce_adam<<<rb, threads, 0, ctx->stream>>>(m->params, m->adam_m, m->adam_v, m->grad, m->partials, blocks,
                                                    m->P, lr, b1, b2, 1e-8f, bc1, bc2, 0,
                                                    loss_device ? loss_device : m->loss);
  return after_launch(ctx, "mlp_reduce_adam");
}

int bo_mlp_train_host(bo_ctx* ctx, bo_mlp* m, const float* x_host, const float* t_host, int32_t n, int32_t epochs,
                      float lr, float* final_loss) {
  int rc = check_mlp(ctx, m);
  if (rc) return rc;
  if (!x_host || !t_host || n < 1 || epochs < 1) return set_error(ctx, BO_ERR_INVALID, "mlp_train: bad argument");
  void* buf = nullptr;
  const size_t xb = sizeof(float) * (size_t)n * m->F, tb = sizeof(float) * (size_t)n * m->O;
  if ((rc = region(ctx, "mlp_train_in", xb + tb + 256, &buf))) return rc;
  float* x = static_cast<float*>(buf);
  float* t = reinterpret_cast<float*>(static_cast<char*>(buf) + ((xb + 255) & ~size_t(255)));
  BO_CUDA(ctx, cudaMemcpyAsync(x, x_host, xb, cudaMemcpyHostToDevice, ctx->stream));
  BO_CUDA(ctx, cudaMemcpyAsync(t, t_host, tb, cudaMemcpyHostToDevice, ctx->stream));
  for (int e = 0; e < epochs; ++e)
    if ((rc = bo_mlp_train_step_device(ctx, m, x, t, n, lr, m->loss))) return rc;
  if (final_loss) {
    BO_CUDA(ctx, cudaMemcpyAsync(final_loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  }
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return BO_OK;
}

int bo_mlp_infer_device(bo_ctx* ctx, const bo_mlp* m, const float* x, int32_t n, float* y) {
  int rc = check_mlp(ctx, m);
  if (rc) return rc;
  if (!x || !y || n < 1) return set_error(ctx, BO_ERR_INVALID, "mlp_infer: bad argument");
  return launch_fwd(ctx, m, false, x, nullptr, n, y, nullptr);
}

int bo_mlp_predict_counts(bo_ctx* ctx, const bo_mlp* m, const float* features_host, float* counts_device,
                          float* log_device) {
  int rc = check_mlp(ctx, m);
  if (rc) return rc;
  if (!features_host || !counts_device) return set_error(ctx, BO_ERR_INVALID, "mlp_predict: bad argument");
  FeatureVec fv;
  for (int i = 0; i < kMaxF; ++i) fv.f[i] = i < m->F ? features_host[i] : 0.0f;
  mlp_predict_counts<<<1, kPredThreads, 0, ctx->stream>>>(m->params, fv, m->F, m->O, counts_device, log_device);
  return after_launch(ctx, "mlp_predict_counts");
}

}  // extern "C"
