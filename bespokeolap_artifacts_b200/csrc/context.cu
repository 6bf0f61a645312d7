// Context, error reporting and memory helpers of the C ABI (bespoke_gpu.h).
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "context.cuh"

namespace bo {

int set_error(bo_ctx* ctx, int code, const char* fmt, ...) {
  if (!ctx) return code;
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  ctx->last_error = buf;
  return code;
}

int cuda_fail(bo_ctx* ctx, cudaError_t e, const char* what) {
  const int code = (e == cudaErrorMemoryAllocation) ? BO_ERR_OOM : BO_ERR_CUDA;
  return set_error(ctx, code, "%s failed: %s", what, cudaGetErrorString(e));
}

int region(bo_ctx* ctx, const char* name, size_t bytes, void** out) {
  auto& r = ctx->regions[name];
  if (r.bytes < bytes) {
    if (r.ptr) {
      drain_host_work(ctx);  // queued host work may still enqueue kernels that read the region
      cudaStreamSynchronize(ctx->stream);
      cudaFree(r.ptr);
      r.ptr = nullptr;
      r.bytes = 0;
    }
    const size_t rounded = (bytes + 4095) & ~size_t(4095);
    BO_CUDA(ctx, cudaMalloc(&r.ptr, rounded));
    BO_CUDA(ctx, cudaMemsetAsync(r.ptr, 0, rounded, ctx->stream));
    r.bytes = rounded;
  }
  *out = r.ptr;
  return BO_OK;
}

int host_stage(bo_ctx* ctx, size_t bytes, void** out) {
  if (ctx->h_stage_bytes < bytes) {
    if (ctx->h_stage) {
      cudaStreamSynchronize(ctx->stream);
      cudaFreeHost(ctx->h_stage);
      ctx->h_stage = nullptr;
      ctx->h_stage_bytes = 0;
    }
    const size_t rounded = (bytes + 4095) & ~size_t(4095);
    BO_CUDA(ctx, cudaHostAlloc(&ctx->h_stage, rounded, cudaHostAllocDefault));
    ctx->h_stage_bytes = rounded;
  }
  *out = ctx->h_stage;
  return BO_OK;
}

int after_launch(bo_ctx* ctx, const char* what) {
  ctx->launches.fetch_add(1, std::memory_order_relaxed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, what);
  return BO_OK;
}

int consume_device_errors(bo_ctx* ctx, uint32_t* bits_out) {
  if (int rc = drain_host_work(ctx)) return rc;
  BO_CUDA(ctx, cudaMemcpyAsync(ctx->h_err, ctx->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                               ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *bits_out = *ctx->h_err;
  if (*bits_out) {
    BO_CUDA(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), ctx->stream));
  }
  return BO_OK;
}

int device_error_status(bo_ctx* ctx, uint32_t bits, const char* op) {
  if (bits == 0) return BO_OK;
  if (bits & kErrSpinTimeout)
    return set_error(ctx, BO_ERR_TIMEOUT, "%s: a bounded device wait timed out (bits 0x%x)", op, bits);
  if (bits & kErrTableOverflow)
    return set_error(ctx, BO_ERR_OVERFLOW, "%s: table overflow (bits 0x%x)", op, bits);
  if (bits & kErrOutputOverflow)
    return set_error(ctx, BO_ERR_OVERFLOW, "%s: output buffer overflow (bits 0x%x)", op, bits);
  if (bits & kErrSumOverflow)
    return set_error(ctx, BO_ERR_OVERFLOW, "%s: a total exceeds its 64-bit result field (bits 0x%x)", op,
                     bits);
  if (bits & kErrBadGroupCode)
    return set_error(ctx, BO_ERR_DATA, "%s: group code outside the declared domain (bits 0x%x)", op, bits);
  return set_error(ctx, BO_ERR_DATA, "%s: value outside the exact-arithmetic contract (bits 0x%x)", op,
                   bits);
}

int occupancy_blocks(const void* kernel, int block, size_t smem) {
  static std::mutex mu;
  static std::unordered_map<const void*, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(kernel);
  if (it != cache.end()) return it->second;
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, block, smem) != cudaSuccess ||
      blocks < 1)
    blocks = 1;
  cache[kernel] = blocks;
  return blocks;
}

}  // namespace bo

extern "C" {

const char* bo_build_info(void) {
  return "bespoke_gpu: sm_100a (B200) build, nvcc " __DATE__;
}

int bo_device_init(int device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return BO_ERR_UNSUPPORTED;
  }
  if (device < 0 || device >= n) return BO_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess || cudaFree(nullptr) != cudaSuccess) {
    cudaGetLastError();
    return BO_ERR_CUDA;
  }
  return BO_OK;
}

int bo_create(bo_ctx** out, int device) {
  if (!out) return BO_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return BO_ERR_UNSUPPORTED;
  }
  if (device < 0 || device >= n) return BO_ERR_INVALID;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return BO_ERR_CUDA;
  if (prop.major < 10) return BO_ERR_UNSUPPORTED;  // kernels are sm_100a only
  if (cudaSetDevice(device) != cudaSuccess) return BO_ERR_CUDA;
  auto* ctx = new bo_ctx();
  ctx->device = device;
  ctx->num_sms = prop.multiProcessorCount;
  ctx->l2_bytes = prop.l2CacheSize;
  // A blocking stream: it is ordered with the legacy default stream, so data a
  // caller wrote there (PyTorch's default stream, a cudaMemcpy) is complete
  // before the context's kernels read it, without an explicit synchronise.
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamDefault) != cudaSuccess ||
      cudaMalloc(&ctx->d_err, sizeof(uint32_t)) != cudaSuccess ||
      cudaHostAlloc(&ctx->h_err, sizeof(uint32_t), cudaHostAllocDefault) != cudaSuccess ||
      cudaHostAlloc(reinterpret_cast<void**>(&ctx->h_word), 2 * sizeof(unsigned long long), cudaHostAllocDefault) !=
          cudaSuccess ||
      cudaMemset(ctx->d_err, 0, sizeof(uint32_t)) != cudaSuccess) {
    bo_destroy(ctx);
    return BO_ERR_CUDA;
  }
  ctx->stream = ctx->own_stream;
  *out = ctx;
  return BO_OK;
}

void bo_destroy(bo_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  bo::destroy_host_work(ctx);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->regions)
    if (kv.second.ptr) cudaFree(kv.second.ptr);
  if (ctx->d_err) cudaFree(ctx->d_err);
  if (ctx->h_err) cudaFreeHost(ctx->h_err);
  if (ctx->h_word) cudaFreeHost(ctx->h_word);
  if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
  if (ctx->copy_stream) {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
  }
  for (cudaEvent_t e : ctx->events) cudaEventDestroy(e);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

const char* bo_last_error(const bo_ctx* ctx) {
  if (!ctx) return "null context";
  return ctx->last_error.c_str();
}

int bo_set_stream(bo_ctx* ctx, void* cuda_stream) {
  BO_CHECK_CTX(ctx);
  ctx->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : ctx->own_stream;
  return BO_OK;
}

void* bo_get_stream(const bo_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int bo_synchronize(bo_ctx* ctx) {
  BO_CHECK_CTX(ctx);
  if (int rc = bo::drain_host_work(ctx)) return rc;
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return BO_OK;
}

int bo_num_sms(const bo_ctx* ctx) { return ctx ? ctx->num_sms : 0; }

int bo_device_alloc(bo_ctx* ctx, size_t bytes, void** out) {
  BO_CHECK_CTX(ctx);
  if (!out) return bo::set_error(ctx, BO_ERR_INVALID, "bo_device_alloc: null out");
  *out = nullptr;
  BO_CUDA(ctx, cudaMalloc(out, bytes ? bytes : 16));
  return BO_OK;
}

int bo_device_free(bo_ctx* ctx, void* ptr) {
  BO_CHECK_CTX(ctx);
  if (ptr) BO_CUDA(ctx, cudaFree(ptr));
  return BO_OK;
}

int bo_host_alloc_pinned(bo_ctx* ctx, size_t bytes, void** out) {
  BO_CHECK_CTX(ctx);
  if (!out) return bo::set_error(ctx, BO_ERR_INVALID, "bo_host_alloc_pinned: null out");
  // Mapped: kernels may also read it in place (zero-copy), e.g. the streamed join.
  BO_CUDA(ctx, cudaHostAlloc(out, bytes ? bytes : 16, cudaHostAllocMapped | cudaHostAllocPortable));
  return BO_OK;
}

int bo_host_free_pinned(bo_ctx* ctx, void* ptr) {
  BO_CHECK_CTX(ctx);
  if (ptr) BO_CUDA(ctx, cudaFreeHost(ptr));
  return BO_OK;
}

int bo_copy_h2d(bo_ctx* ctx, void* dst, const void* src, size_t bytes) {
  BO_CHECK_CTX(ctx);
  if (bytes == 0) return BO_OK;
  BO_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return BO_OK;
}

int bo_copy_d2h(bo_ctx* ctx, void* dst, const void* src, size_t bytes) {
  BO_CHECK_CTX(ctx);
  if (bytes == 0) return BO_OK;
  BO_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return BO_OK;
}

int64_t bo_launch_count(const bo_ctx* ctx) { return ctx ? ctx->launches.load() : 0; }

int bo_check_errors(bo_ctx* ctx) {
  BO_CHECK_CTX(ctx);
  uint32_t bits = 0;
  int rc = bo::consume_device_errors(ctx, &bits);
  if (rc) return rc;
  return bo::device_error_status(ctx, bits, "device");
}

}  // extern "C"
