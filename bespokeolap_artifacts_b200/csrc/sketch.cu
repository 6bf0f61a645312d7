// Column sketches computed once per table on the device: the inputs of the
// learned sizing features (per-column min/max, a 64-bin equi-width histogram,
// an exact histogram for small domains, and HyperLogLog registers for the
// distinct-value estimate).  No reference counterpart: the reference's builder
// keeps only the min/max it needs for dense arrays (e.g.
// bespoke_tpch/builder_impl.cpp:582-596).
//
// Two passes over an int32 column: (1) min/max by block reduction, (2) the
// equi-width histogram (shared-memory counters) and HLL registers (shared
// atomicMax per register), merged into global memory once per block.
#include <algorithm>

#include "common.cuh"
#include "context.cuh"

namespace bo {

constexpr int kSketchBlock = 256;
constexpr int kHllBits = 12;
constexpr int kHllRegs = 1 << kHllBits;

__global__ void __launch_bounds__(kSketchBlock) sketch_minmax_kernel(const int32_t* __restrict__ col, int64_t n,
                                                                     int* __restrict__ mm) {
  int lo = 0x7fffffff, hi = (int)0x80000000;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int v = col[i];
    lo = min(lo, v);
    hi = max(hi, v);
  }
  __shared__ int slo[kSketchBlock / 32], shi[kSketchBlock / 32];
  lo = __reduce_min_sync(0xffffffffu, lo);
  hi = __reduce_max_sync(0xffffffffu, hi);
  if ((threadIdx.x & 31) == 0) {
    slo[threadIdx.x >> 5] = lo;
    shi[threadIdx.x >> 5] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kSketchBlock / 32; ++w) {
      lo = min(lo, slo[w]);
      hi = max(hi, shi[w]);
    }
    lo = min(lo, slo[0]);
    hi = max(hi, shi[0]);
    atomicMin(mm, lo);
    atomicMax(mm + 1, hi);
  }
}

__device__ __forceinline__ uint32_t hll_hash(uint32_t v) { return hash32(v ^ 0x2545F491u); }

__global__ void __launch_bounds__(kSketchBlock) sketch_hist_kernel(const int32_t* __restrict__ col, int64_t n,
                                                                   const int* __restrict__ mm,
                                                                   unsigned long long* __restrict__ hist,
                                                                   uint32_t* __restrict__ hll) {
  __shared__ uint32_t h[BO_SKETCH_BINS];
  __shared__ uint32_t regs[kHllRegs];
  for (int i = threadIdx.x; i < BO_SKETCH_BINS; i += blockDim.x) h[i] = 0;
  for (int i = threadIdx.x; i < kHllRegs; i += blockDim.x) regs[i] = 0;
  __syncthreads();
  const int lo = mm[0], hi = mm[1];
  const uint64_t span = (uint64_t)((int64_t)hi - (int64_t)lo) + 1;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int v = col[i];
    const uint64_t b = ((uint64_t)((int64_t)v - lo) * BO_SKETCH_BINS) / span;
    atomicAdd(&h[b], 1u);
    const uint32_t x = hll_hash((uint32_t)v);
    const uint32_t idx = x >> (32 - kHllBits);
    const uint32_t rank = __clz((x << kHllBits) | (1u << (kHllBits - 1))) + 1;
    if (regs[idx] < rank) atomicMax(&regs[idx], rank);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < BO_SKETCH_BINS; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
  for (int i = threadIdx.x; i < kHllRegs; i += blockDim.x)
    if (regs[i]) atomicMax(&hll[i], regs[i]);
}

// Exact histogram of a small-domain unsigned column (uint8 or uint16 values
// below `domain`, domain <= 65536): shared counters, then one merge per block.
template <typename T>
__global__ void __launch_bounds__(kSketchBlock) sketch_small_kernel(const T* __restrict__ col, int64_t n, int domain,
                                                                    unsigned long long* __restrict__ hist,
                                                                    uint32_t* __restrict__ err) {
  extern __shared__ uint32_t c[];
  for (int i = threadIdx.x; i < domain; i += blockDim.x) c[i] = 0;
  __syncthreads();
  uint32_t bad = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t v = col[i];
    if (v < (uint32_t)domain)
      atomicAdd(&c[v], 1u);
    else
      bad = 1;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < domain; i += blockDim.x)
    if (c[i]) atomicAdd(&hist[i], (unsigned long long)c[i]);
  if (bad) raise_error(err, kErrValueRange);
}

}  // namespace bo

using namespace bo;

namespace {

int grid_of(bo_ctx* ctx, int64_t n) {
  const int64_t g = std::min<int64_t>((n + kSketchBlock - 1) / kSketchBlock, (int64_t)ctx->num_sms * 8);
  return (int)std::max<int64_t>(g, 1);
}

double hll_estimate(const uint32_t* regs) {
  const double m = kHllRegs;
  double z = 0.0;
  int zeros = 0;
  for (int i = 0; i < kHllRegs; ++i) {
    z += std::ldexp(1.0, -(int)regs[i]);
    zeros += regs[i] == 0;
  }
  const double alpha = 0.7213 / (1.0 + 1.079 / m);
  double e = alpha * m * m / z;
  if (e <= 2.5 * m && zeros > 0) e = m * std::log(m / zeros);  // small-range correction
  return e;
}

}  // namespace

extern "C" {

int bo_sketch_i32(bo_ctx* ctx, const int32_t* col_device, int64_t n, bo_sketch* out) {
  BO_CHECK_CTX(ctx);
  if (!out || n < 0 || (n > 0 && !col_device)) return set_error(ctx, BO_ERR_INVALID, "sketch: bad argument");
  *out = bo_sketch{};
  out->n = n;
  if (n == 0) return BO_OK;
  void* p = nullptr;
  const size_t bytes = 16 + sizeof(unsigned long long) * BO_SKETCH_BINS + sizeof(uint32_t) * kHllRegs;
  int rc = region(ctx, "sketch", bytes, &p);
  if (rc) return rc;
  int* mm = static_cast<int*>(p);
  unsigned long long* hist = reinterpret_cast<unsigned long long*>(static_cast<char*>(p) + 16);
  uint32_t* hll = reinterpret_cast<uint32_t*>(hist + BO_SKETCH_BINS);
  const int init[2] = {0x7fffffff, (int)0x80000000};
  BO_CUDA(ctx, cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
  BO_CUDA(ctx, cudaMemsetAsync(hist, 0, bytes - 16, ctx->stream));
  const int g = grid_of(ctx, n);
  sketch_minmax_kernel<<<g, kSketchBlock, 0, ctx->stream>>>(col_device, n, mm);
  if ((rc = after_launch(ctx, "sketch_minmax_kernel"))) return rc;
  sketch_hist_kernel<<<g, kSketchBlock, 0, ctx->stream>>>(col_device, n, mm, hist, hll);
  if ((rc = after_launch(ctx, "sketch_hist_kernel"))) return rc;
  int h_mm[2];
  unsigned long long h_hist[BO_SKETCH_BINS];
  static thread_local uint32_t h_hll[kHllRegs];
  BO_CUDA(ctx, cudaMemcpyAsync(h_mm, mm, sizeof(h_mm), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaMemcpyAsync(h_hist, hist, sizeof(h_hist), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaMemcpyAsync(h_hll, hll, sizeof(h_hll), cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  out->min = h_mm[0];
  out->max = h_mm[1];
  for (int i = 0; i < BO_SKETCH_BINS; ++i) out->hist[i] = (int64_t)h_hist[i];
  out->distinct_estimate = hll_estimate(h_hll);
  return BO_OK;
}

int bo_histogram_small(bo_ctx* ctx, const void* col_device, int32_t elem_bytes, int64_t n, int32_t domain,
                       int64_t* hist_host) {
  BO_CHECK_CTX(ctx);
  if (!hist_host || n < 0 || (n > 0 && !col_device) || (elem_bytes != 1 && elem_bytes != 2) || domain < 1 ||
      domain > 65536)
    return set_error(ctx, BO_ERR_INVALID, "histogram_small: bad argument");
  void* p = nullptr;
  int rc = region(ctx, "sketch_small", sizeof(unsigned long long) * (size_t)domain, &p);
  if (rc) return rc;
  unsigned long long* hist = static_cast<unsigned long long*>(p);
  BO_CUDA(ctx, cudaMemsetAsync(hist, 0, sizeof(unsigned long long) * (size_t)domain, ctx->stream));
  if (n > 0) {
    const int g = grid_of(ctx, n);
    const size_t smem = sizeof(uint32_t) * (size_t)domain;
    if (elem_bytes == 1) {
      BO_CUDA(ctx, cudaFuncSetAttribute(reinterpret_cast<const void*>(&sketch_small_kernel<uint8_t>),
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      sketch_small_kernel<uint8_t><<<g, kSketchBlock, smem, ctx->stream>>>(static_cast<const uint8_t*>(col_device), n,
                                                                           domain, hist, ctx->d_err);
    } else {
      BO_CUDA(ctx, cudaFuncSetAttribute(reinterpret_cast<const void*>(&sketch_small_kernel<uint16_t>),
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      sketch_small_kernel<uint16_t><<<g, kSketchBlock, smem, ctx->stream>>>(
          static_cast<const uint16_t*>(col_device), n, domain, hist, ctx->d_err);
    }
    if ((rc = after_launch(ctx, "sketch_small_kernel"))) return rc;
  }
  BO_CUDA(ctx, cudaMemcpyAsync(hist_host, hist, sizeof(int64_t) * (size_t)domain, cudaMemcpyDeviceToHost,
                               ctx->stream));
  uint32_t bits = 0;
  if ((rc = consume_device_errors(ctx, &bits))) return rc;
  return device_error_status(ctx, bits, "histogram_small");
}

}  // extern "C"
