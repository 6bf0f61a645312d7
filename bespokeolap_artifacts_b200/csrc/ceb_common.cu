// Kernels shared by the CEB pipelines (declared in ceb.cuh).
#include <algorithm>

#include "ceb.cuh"
#include "context.cuh"

namespace bo {

__global__ void __launch_bounds__(kCebBlock) ceb_dim_mask_kernel(bo_ceb_col id, bo_ceb_col code, int64_t n,
                                                                 const uint8_t* __restrict__ allowed, int32_t n_codes,
                                                                 int32_t mask_size, uint8_t* __restrict__ mask,
                                                                 unsigned int* __restrict__ any) {
  bool hit = false;
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t r = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; r < n; r += stride) {
    if (ceb_null(id, r) || ceb_null(code, r)) continue;
    const int32_t i = id.values[r], c = code.values[r];
    if (i < 0 || i >= mask_size || c < 0 || c >= n_codes || !allowed[c]) continue;
    mask[i] = 1;
    hit = true;
  }
  if (any && __any_sync(0xffffffffu, hit) && (threadIdx.x & 31) == 0) atomicOr(any, 1u);
}

__global__ void __launch_bounds__(kCebBlock) ceb_like_dict_kernel(const char* __restrict__ bytes,
                                                                  const uint32_t* __restrict__ off, int64_t n,
                                                                  int32_t type, const char* __restrict__ pat,
                                                                  int32_t len, uint8_t* __restrict__ match) {
  const int64_t stride = (int64_t)gridDim.x * kCebBlock;
  for (int64_t c = (int64_t)blockIdx.x * kCebBlock + threadIdx.x; c < n; c += stride) {
    const uint32_t b = off[c], e = off[c + 1];
    match[c] = ceb_like(type, pat, len, bytes + b, (int)(e - b)) ? 1 : 0;
  }
}

namespace {

constexpr int kScanItems = 4;                        // per thread
constexpr int kScanTile = kCebBlock * kScanItems;    // per block

// Exclusive scan of n counts: per-tile sums, a scan of the tile sums in one
// block, then each tile's scan plus its base.
__global__ void __launch_bounds__(kCebBlock) ceb_tile_sum_kernel(const unsigned int* __restrict__ in, int64_t n,
                                                                 unsigned int* __restrict__ tile_sum) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  unsigned int s = 0;
  for (int i = threadIdx.x; i < kScanTile; i += kCebBlock)
    if (base + i < n) s += in[base + i];
  s = warp_sum_u32(s);
  __shared__ unsigned int part[kCebBlock / 32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = 0;
    for (int w = 0; w < kCebBlock / 32; ++w) t += part[w];
    tile_sum[blockIdx.x] = t;
  }
}

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ unsigned int block_exclusive_scan(unsigned int v, unsigned int* total) {
  __shared__ unsigned int warp_tot[kCebBlock / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    unsigned int s = lane < kCebBlock / 32 ? warp_tot[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kCebBlock / 32) warp_tot[lane] = s;  // inclusive
  }
  __syncthreads();
  const unsigned int before = (w ? warp_tot[w - 1] : 0u) + x - v;
  *total = warp_tot[kCebBlock / 32 - 1];
  __syncthreads();
  return before;
}

__global__ void __launch_bounds__(kCebBlock) ceb_scan_tile_sums_kernel(unsigned int* __restrict__ tile_sum,
                                                                       int64_t n_tiles) {
  unsigned int carry = 0;
  for (int64_t b = 0; b < n_tiles; b += kCebBlock) {
    const int64_t i = b + threadIdx.x;
    const unsigned int v = i < n_tiles ? tile_sum[i] : 0u;
    unsigned int tot = 0;
    const unsigned int ex = block_exclusive_scan(v, &tot);
    if (i < n_tiles) tile_sum[i] = carry + ex;
    carry += tot;
  }
}

__global__ void __launch_bounds__(kCebBlock) ceb_scan_tiles_kernel(const unsigned int* __restrict__ in, int64_t n,
                                                                   const unsigned int* __restrict__ tile_base,
                                                                   unsigned int* __restrict__ out) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  unsigned int v[kScanItems], s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : 0u;
    s += v[k];
  }
  unsigned int tot = 0;
  unsigned int run = tile_base[blockIdx.x] + block_exclusive_scan(s, &tot);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == kCebBlock - 1) out[n] = run;  // the total at out[n]
}

}  // namespace

int ceb_exclusive_scan(bo_ctx* ctx, const unsigned int* in, int64_t n, unsigned int* out) {
  if (n <= 0) return BO_OK;
  const int64_t n_tiles = (n + kScanTile - 1) / kScanTile;
  if (n_tiles > 0x7fffffff) return set_error(ctx, BO_ERR_INVALID, "ceb scan: too many entries");
  void* p = nullptr;
  int rc = region(ctx, "ceb_scan_tiles", sizeof(unsigned int) * (size_t)n_tiles, &p);
  if (rc) return rc;
  auto* tiles = static_cast<unsigned int*>(p);
  ceb_tile_sum_kernel<<<(int)n_tiles, kCebBlock, 0, ctx->stream>>>(in, n, tiles);
  if ((rc = after_launch(ctx, "ceb_tile_sum_kernel"))) return rc;
  ceb_scan_tile_sums_kernel<<<1, kCebBlock, 0, ctx->stream>>>(tiles, n_tiles);
  if ((rc = after_launch(ctx, "ceb_scan_tile_sums_kernel"))) return rc;
  ceb_scan_tiles_kernel<<<(int)n_tiles, kCebBlock, 0, ctx->stream>>>(in, n, tiles, out);
  return after_launch(ctx, "ceb_scan_tiles_kernel");
}

}  // namespace bo
