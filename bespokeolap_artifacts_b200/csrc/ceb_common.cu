// Kernels shared by the CEB pipelines (declared in ceb.cuh).
#include "ceb.cuh"

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

}  // namespace bo
