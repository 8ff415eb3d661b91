// Tensor-core self-check: one 128 x 256 x 64 bf16 GEMM on tcgen05 with the
// operand and accumulator layouts of tc.cuh, so a host test can compare it
// with a CPU product before the block matcher and the pilot network rely on
// those layouts.  C[i][j] = sum_k A[i][k] B[j][k] (row-major A: 128 x 64,
// B: 256 x 64, bf16 bits; C: 128 x 256 fp32).
#include "common.cuh"
#include "kernels.cuh"
#include "tc.cuh"

namespace gbm3d {

namespace {
constexpr int CM = 128, CN = 256, CK = 64;

__global__ void __launch_bounds__(128) k_tc_gemm_check(const uint16_t* __restrict__ A, const uint16_t* __restrict__ B,
                                                       float* __restrict__ C, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* sA = smem;                   // 128 x 64 bf16 = 16 KB
  unsigned char* sB = smem + CM * CK * 2;     // 256 x 64 bf16 = 32 KB
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sB + CN * CK * 2);
  uint32_t* taddr_s = reinterpret_cast<uint32_t*>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;

  if (warp == 0) tc::tmem_alloc(taddr_s, 256);
  if (tid == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  for (int e = tid; e < CM * CK; e += blockDim.x) {
    const int row = e / CK, k = e % CK;
    *reinterpret_cast<uint16_t*>(sA + tc::kmajor_offset(row, k, CK)) = A[e];
  }
  for (int e = tid; e < CN * CK; e += blockDim.x) {
    const int row = e / CK, k = e % CK;
    *reinterpret_cast<uint16_t*>(sB + tc::kmajor_offset(row, k, CK)) = B[e];
  }
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *taddr_s;
  if (tid == 0) {
    const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
    constexpr uint32_t idesc = tc::idesc_bf16_f32(CM, CN);
#pragma unroll
    for (int ks = 0; ks < CK / 16; ++ks) {
      const uint64_t ad = tc::desc_kmajor(a0 + ks * 256, 128, CK * 16);
      const uint64_t bd = tc::desc_kmajor(b0 + ks * 256, 128, CK * 16);
      tc::mma_bf16(tmem, ad, bd, idesc, ks > 0);
    }
    tc::commit(mbar);
  }
  const bool ok = tc::mbar_wait(mbar, 0, 2000000000LL);
  if (!ok && tid == 0) atomicOr(err, 2);
  tc::fence_after_sync();
  if (ok) {
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < CN; c0 += 32) {
      float v[32];
      tc::tmem_ld32(lane_base + c0, v);
      const int row = warp * 32 + (tid & 31);
#pragma unroll
      for (int q = 0; q < 32; ++q) C[row * CN + c0 + q] = v[q];
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 256);
}
// The same product with both operands stored MN-major (the layout of an
// NHWC activation tile read with pixels as K): core matrices of 8 K-rows x 8
// consecutive M (or N) elements, K-adjacent ones 128 bytes apart (the
// descriptor's leading byte offset), M-adjacent ones (K/8) * 128 bytes apart
// (its stride byte offset); instruction descriptor bits 15 / 16 select
// MN-major A / B.  With swap_offsets the two descriptor fields are exchanged
// (the other reading of the MN-major canonical layout); every address either
// reading implies stays inside the operand buffers.
__global__ void __launch_bounds__(128) k_tc_gemm_check_mn(const uint16_t* __restrict__ A,
                                                          const uint16_t* __restrict__ B, float* __restrict__ C,
                                                          int* __restrict__ err, int swap_offsets) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* sA = smem;
  unsigned char* sB = smem + CM * CK * 2;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sB + CN * CK * 2);
  uint32_t* taddr_s = reinterpret_cast<uint32_t*>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  auto mn_off = [](int mn, int k) -> uint32_t {
    return (uint32_t)((mn >> 3) * (CK / 8) * 128 + (k >> 3) * 128 + (k & 7) * 16 + (mn & 7) * 2);
  };
  if (warp == 0) tc::tmem_alloc(taddr_s, 256);
  if (tid == 0) {
    tc::mbar_init(mbar, 1);
    tc::fence_mbar_init();
  }
  for (int e = tid; e < CM * CK; e += blockDim.x) {
    const int row = e / CK, k = e % CK;
    *reinterpret_cast<uint16_t*>(sA + mn_off(row, k)) = A[e];
  }
  for (int e = tid; e < CN * CK; e += blockDim.x) {
    const int row = e / CK, k = e % CK;
    *reinterpret_cast<uint16_t*>(sB + mn_off(row, k)) = B[e];
  }
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *taddr_s;
  if (tid == 0) {
    const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
    constexpr uint32_t idesc = tc::idesc_bf16_f32(CM, CN) | (1u << 15) | (1u << 16);
#pragma unroll
    for (int ks = 0; ks < CK / 16; ++ks) {
      const uint32_t kstr = 128, mstr = (CK / 8) * 128;  // K-adjacent, M-adjacent core strides
      const uint32_t lbo = swap_offsets ? mstr : kstr, sbo = swap_offsets ? kstr : mstr;
      const uint64_t ad = tc::desc_kmajor(a0 + ks * 256, lbo, sbo);
      const uint64_t bd = tc::desc_kmajor(b0 + ks * 256, lbo, sbo);
      tc::mma_bf16(tmem, ad, bd, idesc, ks > 0);
    }
    tc::commit(mbar);
  }
  const bool ok = tc::mbar_wait(mbar, 0, 2000000000LL);
  if (!ok && tid == 0) atomicOr(err, 2);
  tc::fence_after_sync();
  if (ok) {
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < CN; c0 += 32) {
      float v[32];
      tc::tmem_ld32(lane_base + c0, v);
      const int row = warp * 32 + (tid & 31);
#pragma unroll
      for (int q = 0; q < 32; ++q) C[row * CN + c0 + q] = v[q];
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 256);
}
}  // namespace

cudaError_t launch_tc_gemm_check_mn(const uint16_t* A, const uint16_t* B, float* C, int* err, int swap_offsets,
                                    cudaStream_t st) {
  const size_t sm = (size_t)(CM + CN) * CK * 2 + 64;
  cudaError_t e = cudaFuncSetAttribute(k_tc_gemm_check_mn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  k_tc_gemm_check_mn<<<1, 128, sm, st>>>(A, B, C, err, swap_offsets);
  return cudaGetLastError();
}

cudaError_t launch_tc_gemm_check(const uint16_t* A, const uint16_t* B, float* C, int* err, cudaStream_t st) {
  const size_t sm = (size_t)(CM + CN) * CK * 2 + 64;
  cudaError_t e = cudaFuncSetAttribute(k_tc_gemm_check, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  k_tc_gemm_check<<<1, 128, sm, st>>>(A, B, C, err);
  return cudaGetLastError();
}

}  // namespace gbm3d
