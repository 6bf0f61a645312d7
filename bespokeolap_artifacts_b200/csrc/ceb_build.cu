// The CEB builder's fact-table order on the device
// (bespoke_ceb/builder_impl.cpp:255-360, 432-452): the reference sorts a
// row permutation with std::sort by one or two int32 columns and reorders
// every column through it.  Here the two keys become one 64-bit key
// (each int32 with its sign bit flipped, so unsigned order is signed
// order), the onesweep radix sort orders (key, row) pairs -- stably -- and
// gather kernels reorder the columns.
#include <algorithm>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kCebSortBlock = 256;

__global__ void __launch_bounds__(kCebSortBlock) ceb_key_kernel(const int32_t* __restrict__ primary,
                                                                const int32_t* __restrict__ secondary, int64_t n,
                                                                unsigned long long* __restrict__ keys,
                                                                uint32_t* __restrict__ rows) {
  const int64_t stride = (int64_t)gridDim.x * kCebSortBlock;
  for (int64_t i = (int64_t)blockIdx.x * kCebSortBlock + threadIdx.x; i < n; i += stride) {
    const uint32_t hi = (uint32_t)primary[i] ^ 0x80000000u;
    const uint32_t lo = secondary ? ((uint32_t)secondary[i] ^ 0x80000000u) : 0u;
    keys[i] = ((unsigned long long)hi << 32) | lo;
    rows[i] = (uint32_t)i;
  }
}

template <class T>
__global__ void __launch_bounds__(kCebSortBlock) ceb_gather_kernel(const T* __restrict__ src,
                                                                   const uint32_t* __restrict__ perm, int64_t n,
                                                                   T* __restrict__ dst) {
  const int64_t stride = (int64_t)gridDim.x * kCebSortBlock;
  for (int64_t i = (int64_t)blockIdx.x * kCebSortBlock + threadIdx.x; i < n; i += stride) dst[i] = src[perm[i]];
}

int ceb_sort_grid(bo_ctx* ctx, const void* k, int64_t n) {
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(k, kCebSortBlock, 0);
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + kCebSortBlock - 1) / kCebSortBlock, resident));
}

template <class T>
int ceb_gather(bo_ctx* ctx, const T* src, const uint32_t* perm, int64_t n, T* dst, const char* name) {
  BO_CHECK_CTX(ctx);
  if (n < 0 || (n > 0 && (!src || !perm || !dst))) return set_error(ctx, BO_ERR_INVALID, "%s: bad argument", name);
  if (n > 0 && src == dst) return set_error(ctx, BO_ERR_INVALID, "%s: source and destination alias", name);
  if (n == 0) return BO_OK;
  const void* k = reinterpret_cast<const void*>(&ceb_gather_kernel<T>);
  ceb_gather_kernel<T><<<ceb_sort_grid(ctx, k, n), kCebSortBlock, 0, ctx->stream>>>(src, perm, n, dst);
  return after_launch(ctx, name);
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" {

int bo_ceb_sort_rows(bo_ctx* ctx, const int32_t* primary, const int32_t* secondary, int64_t n,
                     uint32_t* perm_device) {
  BO_CHECK_CTX(ctx);
  if (n < 0 || (n > 0 && (!primary || !perm_device)) || n > 0xffffffffll)
    return set_error(ctx, BO_ERR_INVALID, "ceb_sort_rows: bad argument");
  if (n == 0) return BO_OK;
  const size_t kb = (sizeof(unsigned long long) * (size_t)n + 255) & ~size_t(255);
  void* p = nullptr;
  int rc = region(ctx, "ceb_sort", 2 * kb + sizeof(uint32_t) * (size_t)n, &p);
  if (rc) return rc;
  auto* keys = static_cast<unsigned long long*>(p);
  auto* tmp_keys = reinterpret_cast<unsigned long long*>(static_cast<char*>(p) + kb);
  auto* tmp_rows = reinterpret_cast<uint32_t*>(static_cast<char*>(p) + 2 * kb);
  const void* k = reinterpret_cast<const void*>(&ceb_key_kernel);
  ceb_key_kernel<<<ceb_sort_grid(ctx, k, n), kCebSortBlock, 0, ctx->stream>>>(primary, secondary, n, keys,
                                                                              perm_device);
  if ((rc = after_launch(ctx, "ceb_key_kernel"))) return rc;
  return radix_sort_pairs(ctx, keys, perm_device, tmp_keys, tmp_rows, n, secondary ? 0 : 32, 64, nullptr);
}

int bo_ceb_gather_i32(bo_ctx* ctx, const int32_t* src, const uint32_t* perm, int64_t n, int32_t* dst) {
  return ceb_gather<int32_t>(ctx, src, perm, n, dst, "ceb_gather_i32");
}

int bo_ceb_gather_u8(bo_ctx* ctx, const uint8_t* src, const uint32_t* perm, int64_t n, uint8_t* dst) {
  return ceb_gather<uint8_t>(ctx, src, perm, n, dst, "ceb_gather_u8");
}

}  // extern "C"
