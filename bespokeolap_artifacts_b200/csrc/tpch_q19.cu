// TPC-H Q19 over the storage-plan layout: run_q19 of
// bespoke_tpch/query_q19.cpp:130-338.
//
// The reference gives every partkey a 3-bit mask (one bit per brand /
// container list / size group, the last part row of a key deciding), then
// scans the lineitems of the two ship modes and the one ship instruction and
// adds extendedprice * (100 - discount) for rows whose quantity lies in the
// range of a group of their part's mask.  Here:
//   q19_mask_kernel      one thread per partkey: the mask of its last part row
//                        (per-key row map built with the database);
//   q19_lineitem_kernel  eight ship-mode and ship-instruct codes per thread
//                        from 16-byte loads; the few rows that pass read
//                        partkey, mask, quantity, price and discount; an
//                        int64 sum per thread, warp / block reduced, one
//                        atomic per block.
#include <algorithm>

#include "common.cuh"
#include "context.cuh"

namespace bo {
namespace {

constexpr int kQ19Block = 256;
constexpr int kQ19Rows = 8;
constexpr int kQ19MaxContainers = 1 << 16;

struct Q19Groups {
  int32_t brand[3];
  int32_t size_high[3];
  int32_t qty_low[3];
  int32_t mode1, mode2, instruct;
};

__global__ void __launch_bounds__(kQ19Block) q19_mask_kernel(bo_tpch_q19_tables t, Q19Groups g,
                                                             const uint8_t* __restrict__ cont_groups,
                                                             int32_t n_containers, uint8_t* __restrict__ mask) {
  const int64_t stride = (int64_t)gridDim.x * kQ19Block;
  for (int64_t k = (int64_t)blockIdx.x * kQ19Block + threadIdx.x; k < t.n_mask; k += stride) {
    uint8_t m = 0;
    const int32_t row = k < t.n_part_keys ? t.p_row_by_key[k] : -1;
    if (row >= 0 && (int64_t)row < t.n_part) {
      const int32_t brand = t.p_brand[row], cont = t.p_container[row], size = t.p_size[row];
      const uint8_t cg = cont < n_containers ? cont_groups[cont] : 0;
#pragma unroll
      for (int i = 0; i < 3; ++i)
        if (g.brand[i] >= 0 && brand == g.brand[i] && ((cg >> i) & 1u) && size >= 1 && size <= g.size_high[i])
          m |= (uint8_t)(1u << i);
    }
    mask[k] = m;
  }
}

__device__ __forceinline__ bool q19_mode_ok(uint32_t m, const Q19Groups& g) {
  return (int32_t)m == g.mode1 || (int32_t)m == g.mode2;
}

__global__ void __launch_bounds__(kQ19Block) q19_lineitem_kernel(bo_tpch_q19_tables t, Q19Groups g,
                                                                 const uint8_t* __restrict__ mask,
                                                                 unsigned long long* __restrict__ revenue) {
  long long sum = 0;
  const int64_t n = t.n_lineitem;
  const int64_t stride = (int64_t)gridDim.x * kQ19Block;
  for (int64_t c = (int64_t)blockIdx.x * kQ19Block + threadIdx.x; c * kQ19Rows < n; c += stride) {
    const int64_t r0 = c * kQ19Rows;
    uint32_t pass = 0;
    if (r0 + kQ19Rows <= n) {
      const int4 m4 = ld_stream_v4(t.l_shipmode + r0), i4 = ld_stream_v4(t.l_shipinstruct + r0);
      const uint32_t mw[4] = {(uint32_t)m4.x, (uint32_t)m4.y, (uint32_t)m4.z, (uint32_t)m4.w};
      const uint32_t iw[4] = {(uint32_t)i4.x, (uint32_t)i4.y, (uint32_t)i4.z, (uint32_t)i4.w};
#pragma unroll
      for (int k = 0; k < kQ19Rows; ++k) {
        const uint32_t m = (mw[k >> 1] >> (16 * (k & 1))) & 0xffffu, in = (iw[k >> 1] >> (16 * (k & 1))) & 0xffffu;
        pass |= (uint32_t)(q19_mode_ok(m, g) && (int32_t)in == g.instruct) << k;
      }
    } else {
      for (int k = 0; k < kQ19Rows; ++k)
        if (r0 + k < n && q19_mode_ok(t.l_shipmode[r0 + k], g) && (int32_t)t.l_shipinstruct[r0 + k] == g.instruct)
          pass |= 1u << k;
    }
    while (pass) {
      const int k = __ffs(pass) - 1;
      pass &= pass - 1;
      const int64_t r = r0 + k;
      const int32_t pk = t.l_partkey[r];
      if (pk < 0 || (int64_t)pk >= t.n_mask) continue;
      const uint32_t m = mask[pk];
      if (!m) continue;
      const int32_t q = t.l_quantity[r];
      bool hit = false;
#pragma unroll
      for (int i = 0; i < 3; ++i) hit |= ((m >> i) & 1u) && q >= g.qty_low[i] && q <= g.qty_low[i] + 1000;
      if (hit) sum += (long long)t.l_extendedprice[r] * (long long)(100 - (int32_t)t.l_discount[r]);
    }
  }
  for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  __shared__ long long part[kQ19Block / 32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int w = 0; w < kQ19Block / 32; ++w) s += part[w];
    if (s) atomicAdd(revenue, (unsigned long long)s);
  }
}

int q19_grid(bo_ctx* ctx, const void* k, int64_t threads) {
  const int64_t resident = (int64_t)ctx->num_sms * occupancy_blocks(k, kQ19Block, 0);
  return (int)std::max<int64_t>(1, std::min<int64_t>((threads + kQ19Block - 1) / kQ19Block, resident));
}

}  // namespace
}  // namespace bo

using namespace bo;

extern "C" int bo_tpch_q19(bo_ctx* ctx, const bo_tpch_q19_tables* t, const int32_t brand_code[3],
                           const uint8_t* container_groups_host, int32_t n_containers, const int32_t size_high[3],
                           const int32_t qty_low[3], int32_t mode1, int32_t mode2, int32_t instruct_code,
                           int64_t* revenue_out) {
  BO_CHECK_CTX(ctx);
  if (!t || !brand_code || !size_high || !qty_low || !revenue_out || n_containers < 0 ||
      n_containers > kQ19MaxContainers || (n_containers > 0 && !container_groups_host))
    return set_error(ctx, BO_ERR_INVALID, "q19: null argument or container count");
  *revenue_out = 0;
  if (t->n_lineitem < 0 || t->n_part < 0 || t->n_part_keys < 0 || t->n_mask < 0 || t->n_mask > 0x7fffffffll)
    return set_error(ctx, BO_ERR_INVALID, "q19: sizes");
  if (t->n_lineitem == 0 || t->n_mask == 0 || instruct_code < 0 || (mode1 < 0 && mode2 < 0)) return BO_OK;
  if (!t->l_shipmode || !t->l_shipinstruct || !t->l_partkey || !t->l_quantity || !t->l_extendedprice ||
      !t->l_discount || !aligned16(t->l_shipmode) || !aligned16(t->l_shipinstruct) ||
      (t->n_part_keys > 0 && !t->p_row_by_key) || (t->n_part > 0 && (!t->p_brand || !t->p_container || !t->p_size)))
    return set_error(ctx, BO_ERR_INVALID, "q19: null column or codes not 16-byte aligned");
  Q19Groups g;
  for (int i = 0; i < 3; ++i) {
    g.brand[i] = brand_code[i];
    g.size_high[i] = size_high[i];
    g.qty_low[i] = qty_low[i];
  }
  // A code that names no mode matches nothing (codes are 16-bit).
  g.mode1 = mode1 >= 0 ? mode1 : -2;
  g.mode2 = mode2 >= 0 ? mode2 : -2;
  g.instruct = instruct_code;
  const size_t cont_bytes = ((size_t)std::max(n_containers, 1) + 255) & ~size_t(255);
  const size_t mask_bytes = ((size_t)t->n_mask + 255) & ~size_t(255);
  void* p = nullptr;
  int rc = region(ctx, "q19_ws", 256 + cont_bytes + mask_bytes, &p);
  if (rc) return rc;
  auto* revenue = static_cast<unsigned long long*>(p);
  auto* cont = static_cast<uint8_t*>(p) + 256;
  auto* mask = cont + cont_bytes;
  BO_CUDA(ctx, cudaMemsetAsync(revenue, 0, 8, ctx->stream));
  if (n_containers > 0)
    BO_CUDA(ctx, cudaMemcpyAsync(cont, container_groups_host, (size_t)n_containers, cudaMemcpyHostToDevice,
                                 ctx->stream));
  const void* km = reinterpret_cast<const void*>(&q19_mask_kernel);
  q19_mask_kernel<<<q19_grid(ctx, km, t->n_mask), kQ19Block, 0, ctx->stream>>>(*t, g, cont, n_containers, mask);
  if ((rc = after_launch(ctx, "q19_mask_kernel"))) return rc;
  const void* kl = reinterpret_cast<const void*>(&q19_lineitem_kernel);
  q19_lineitem_kernel<<<q19_grid(ctx, kl, (t->n_lineitem + kQ19Rows - 1) / kQ19Rows), kQ19Block, 0, ctx->stream>>>(
      *t, g, mask, revenue);
  if ((rc = after_launch(ctx, "q19_lineitem_kernel"))) return rc;
  unsigned long long r = 0;
  BO_CUDA(ctx, cudaMemcpyAsync(&r, revenue, 8, cudaMemcpyDeviceToHost, ctx->stream));
  BO_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *revenue_out = (int64_t)r;
  return BO_OK;
}
