// Forward products of the surrogate's perceptron on the fifth-generation tensor cores:
//
//   C[M, N] = A[M, K] W[N, K]^T (+ bias[n]) (GELU)     A, W: BF16, K contiguous, in HBM
//
// One CTA of sixteen warps computes a 128 x 256 tile.  The tensor memory accelerator brings
// 64-wide K slices of A (128 rows) and W (256 rows) into shared memory, swizzled by 128
// bytes, through a four-stage ring guarded by mbarriers; one thread issues tcgen05.mma
// (kind::f16: BF16 operands, FP32 accumulation) for each 16-wide K step into a 128 x 256
// FP32 accumulator held in tensor memory, and commits each stage back to its producer.
// When the ring drains, each warp reads its 32 rows of the accumulator with tcgen05.ld and
// applies the epilogue (bias, GELU, FP32 and/or BF16 stores).  Every mbarrier wait is
// bounded: a wait that gives up sets *status, and the CTA still releases its tensor memory
// before it returns.  No load is multicast.
//
// The shared-memory and instruction descriptors follow the sm_100 UMMA formats (K-major,
// 128-byte swizzle: stride between 8-row groups 1024 bytes; a 16-element K step advances
// the start address by 32 bytes inside the swizzle atom).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "solprop_b200.h"
#include "tcgen05.cuh"

namespace sp {
namespace {

constexpr int kTM = 128, kTN = 256, kTK = 64, kStages = 4;
// sixteen warps: one thread of warp 0 feeds the ring, one of warp 1 issues the products, and
// all sixteen drain the accumulator (warp w reads lanes 32 (w % 4) .. + 31, columns
// 64 (w / 4) .. + 63), so that the epilogue's arithmetic has warps to hide its latency
constexpr int kThreads = 512;
constexpr int kEpilogueColumns = kTN / (kThreads / 128);
constexpr uint32_t kABytes = kTM * kTK * 2;  // 16 KB
constexpr uint32_t kBBytes = kTN * kTK * 2;  // 32 KB
constexpr uint32_t kStageBytes = kABytes + kBBytes;
constexpr size_t kSmemBytes = (size_t)kStages * kStageBytes + 1024 + 256;
constexpr uint32_t kTmemColumns = 256;     // the FP32 accumulator: 256 columns x 128 lanes
constexpr uint32_t kIdesc = tc::idesc_bf16(kTM, kTN);
using namespace tc;

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__global__ void __launch_bounds__(kThreads, 1)
    k_mlp_gemm_tc(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_w,
                  float* C, __nv_bfloat16* C16, const float* bias, int M, int N, int K, int ldc, int ldc16,
                  int epilogue, int* status) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  unsigned char* ring = reinterpret_cast<unsigned char*>(((uintptr_t)tc_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + (size_t)kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* done = empty + kStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ int failed;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int m0 = blockIdx.y * kTM, n0 = blockIdx.x * kTN;
  const int n_k = K / kTK;
  if (threadIdx.x == 0) {
    failed = 0;
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) {  // the whole warp allocates the accumulator's columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemColumns)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (threadIdx.x == 0) {
    // producer: the K slices of A and W, stage by stage
    for (int k = 0; k < n_k; ++k) {
      const int s = k % kStages;
      const uint32_t round = k / kStages;
      if (k >= kStages && !mbar_wait(&empty[s], (round - 1) & 1)) {
        failed = 1;
        break;
      }
      unsigned char* stage = ring + (size_t)s * kStageBytes;
      mbar_expect_tx(&full[s], kStageBytes);
      tma_load_2d(stage, &map_a, &full[s], k * kTK, m0);
      tma_load_2d(stage + kABytes, &map_w, &full[s], k * kTK, n0);
    }
  } else if (threadIdx.x == 32) {
    // the MMA issuer: four 16-wide K steps per stage, the stage handed back on completion
    for (int k = 0; k < n_k; ++k) {
      const int s = k % kStages;
      const uint32_t round = k / kStages;
      if (!mbar_wait(&full[s], round & 1)) {
        failed = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const unsigned char* stage = ring + (size_t)s * kStageBytes;
      const uint64_t da = sw128_desc(stage), db = sw128_desc(stage + kABytes);
#pragma unroll
      for (int kk = 0; kk < kTK / 16; ++kk)
        umma_bf16(tmem, da + 2ull * kk, db + 2ull * kk, kIdesc, (k | kk) != 0 ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    umma_commit(done);  // every MMA issued above has completed when this arrives
  }
  __syncwarp();
  // epilogue: warp w holds accumulator lanes (rows) 32 w .. 32 w + 31; the tile goes
  // through shared memory (the drained ring, rows padded by one word against bank
  // conflicts) so that it leaves in coalesced rows
  const bool ok = mbar_wait(done, 0);
  __syncwarp();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  constexpr int kPitch = kTN + 1;
  static_assert((size_t)kTM * kPitch * 4 <= (size_t)kStages * kStageBytes, "the tile fits in the ring");
  float* tile = reinterpret_cast<float*>(ring);
  const int quarter = warp % 4;  // the accumulator lanes this warp may read
  const int row = quarter * 32 + lane;
  const int c_lo = (warp / 4) * kEpilogueColumns;
  for (int c = c_lo; c < c_lo + kEpilogueColumns; c += 32) {
    uint32_t r[32];
    __syncwarp();  // the load is warp-wide (.sync.aligned)
    tmem_load_32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c, r);
#pragma unroll
    for (int j = 0; j < 32; ++j) tile[row * kPitch + c + j] = __uint_as_float(r[j]);
  }
  __syncthreads();
  if (ok && !failed) {
    for (int rr = warp; rr < kTM && m0 + rr < M; rr += kThreads / 32) {
      const size_t m = (size_t)(m0 + rr);
      for (int cc = lane; cc < kTN; cc += 32) {
        const int n = n0 + cc;
        float v = tile[rr * kPitch + cc];
        if (epilogue >= 1 && bias) v += bias[n];
        if (epilogue == 3) {  // training: the pre-activation in FP32, the activation in BF16
          if (C) C[m * ldc + n] = v;
          if (C16) C16[m * ldc16 + n] = __float2bfloat16_rn(gelu(v));
          continue;
        }
        if (epilogue == 2) v = gelu(v);
        if (C) C[m * ldc + n] = v;
        if (C16) C16[m * ldc16 + n] = __float2bfloat16_rn(v);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemColumns) : "memory");
  if (threadIdx.x == 0 && (!ok || failed)) atomicExch(status, 1);
}

// FP32 rows -> BF16 rows (zero-padded to `cols_out` columns)
__global__ void k_to_bf16(const float* src, int ld_src, int rows, int cols, __nv_bfloat16* dst, int ld_dst,
                          int cols_out) {
  const size_t total = (size_t)rows * cols_out;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols_out), c = (int)(i % cols_out);
    dst[(size_t)r * ld_dst + c] = __float2bfloat16_rn(c < cols ? src[(size_t)r * ld_src + c] : 0.0f);
  }
}

// dst[c][r] = BF16(src[r][c]) for r < rows, zero for rows <= r < rows_pad (32 x 32 tiles
// through shared memory, both sides coalesced)
template <class T>
__global__ void k_transpose_bf16(const T* src, int ld_src, int rows, int cols, __nv_bfloat16* dst, int ld_dst,
                                 int rows_pad) {
  __shared__ float tile[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    float v = 0.0f;
    if (r < rows && c < cols) {
      if constexpr (sizeof(T) == 4) v = src[(size_t)r * ld_src + c];
      else v = __bfloat162float(src[(size_t)r * ld_src + c]);
    }
    tile[i][threadIdx.x] = v;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (c < cols && r < rows_pad) dst[(size_t)c * ld_dst + r] = __float2bfloat16_rn(tile[threadIdx.x][i]);
  }
}

// a rows x cols BF16 matrix (row pitch ld elements) as 2-D tiles of box_rows x 64
bool make_map(CUtensorMap* map, const void* base, int rows, int cols, int ld, int box_rows) {
  return tc::make_bf16_map(map, base, rows, cols, ld, box_rows, kTK);
}

}  // namespace
}  // namespace sp

extern "C" {

sp_status sp_mlp_gemm_tc(const void* A, int lda, const void* W, int ldw, float* C, int ldc, void* C16,
                         int ldc16, int M, int N, int K, const float* bias, int epilogue, int* status,
                         void* stream) {
  using namespace sp;
  if (!A || !W || (!C && !C16) || !status || M < 1 || N < 1 || K < 1 || epilogue < 0 || epilogue > 3)
    return SP_ERR_ARGUMENT;
  // the tiling's and the tensor maps' rules: whole 256-column tiles and 64-wide K slices,
  // 16-byte aligned rows
  if (N % kTN || K % kTK || lda % 8 || ldw % 8 || lda < K || ldw < K) return SP_ERR_ARGUMENT;
  if (((uintptr_t)A | (uintptr_t)W) & 15) return SP_ERR_ARGUMENT;
  CUtensorMap map_a, map_w;
  if (!make_map(&map_a, A, M, K, lda, kTM) || !make_map(&map_w, W, N, K, ldw, kTN)) return SP_ERR_CUDA;
  static std::once_flag configured;
  std::call_once(configured, [] {
    cudaFuncSetAttribute(k_mlp_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
  });
  const dim3 grid(N / kTN, (M + kTM - 1) / kTM);
  k_mlp_gemm_tc<<<grid, kThreads, kSmemBytes, (cudaStream_t)stream>>>(
      map_a, map_w, C, static_cast<__nv_bfloat16*>(C16), bias, M, N, K, ldc, ldc16, epilogue, status);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ERR_CUDA;
}

sp_status sp_mlp_transpose_bf16(const void* src, int src_bf16, int ld_src, int rows, int cols, void* dst,
                                int ld_dst, int rows_pad, void* stream) {
  if (!src || !dst || rows < 0 || cols < 0 || rows_pad < rows || ld_dst < rows_pad) return SP_ERR_ARGUMENT;
  if (!rows_pad || !cols) return SP_OK;
  const dim3 grid((cols + 31) / 32, (rows_pad + 31) / 32), block(32, 8);
  if (src_bf16)
    sp::k_transpose_bf16<__nv_bfloat16><<<grid, block, 0, (cudaStream_t)stream>>>(
        static_cast<const __nv_bfloat16*>(src), ld_src, rows, cols, static_cast<__nv_bfloat16*>(dst), ld_dst,
        rows_pad);
  else
    sp::k_transpose_bf16<float><<<grid, block, 0, (cudaStream_t)stream>>>(
        static_cast<const float*>(src), ld_src, rows, cols, static_cast<__nv_bfloat16*>(dst), ld_dst, rows_pad);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ERR_CUDA;
}

sp_status sp_mlp_to_bf16(const float* src, int ld_src, int rows, int cols, void* dst, int ld_dst, int cols_out,
                         void* stream) {
  if (!src || !dst || rows < 0 || cols < 0 || cols_out < cols) return SP_ERR_ARGUMENT;
  if (!rows || !cols_out) return SP_OK;
  const size_t total = (size_t)rows * cols_out;
  const unsigned blocks = (unsigned)((total + 255) / 256 < 148 * 16 ? (total + 255) / 256 : 148 * 16);
  sp::k_to_bf16<<<blocks, 256, 0, (cudaStream_t)stream>>>(src, ld_src, rows, cols,
                                                          static_cast<__nv_bfloat16*>(dst), ld_dst, cols_out);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ERR_CUDA;
}

}  // extern "C"
