// Forward products of the surrogate's perceptron on the fifth-generation tensor cores:
//
//   C[M, N] = A[M, K] W[N, K]^T (+ bias[n]) (GELU)     A, W: BF16, K contiguous, in HBM
//
// A persistent CTA per SM (ten warps) computes 128 x 256 tiles in turn.  The tensor memory
// accelerator brings 64-wide K slices of A (128 rows) and W (256 rows) into shared memory,
// swizzled by 128 bytes, through a four-stage ring guarded by mbarriers; one thread issues
// tcgen05.mma (kind::f16: BF16 operands, FP32 accumulation) for each 16-wide K step into a
// 128 x 256 FP32 accumulator in tensor memory -- two of them, alternating by tile -- and
// commits each stage back to its producer.  Eight warps drain the other accumulator with
// tcgen05.ld meanwhile and apply the epilogue (bias, GELU, FP32 and/or BF16 stores, staged
// through shared memory so that rows leave coalesced).  Every mbarrier wait is bounded: a
// wait that gives up sets *status, and the CTA still waits for its products and loads and
// releases its tensor memory before it returns.  No load is multicast.
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

constexpr int kTM = 128, kTN = 256, kTK = 64, kStages = 3;
// eighteen warps: one thread of warp 0 feeds the ring, one of warp 1 issues the products,
// and warps 2..17 drain the accumulators (warp w may read tensor-memory lanes 32 (w % 4) ..
// + 31; warps 2..5 take columns 0..63 of a tile, warps 6..9 columns 64..127, and so on):
// the epilogue's arithmetic (bias, GELU, conversion) per output is what bounds a tile
constexpr int kEpilogueWarps = 16;
constexpr int kThreads = 32 * (2 + kEpilogueWarps);
constexpr int kEpilogueColumns = kTN / (kEpilogueWarps / 4);
constexpr uint32_t kABytes = kTM * kTK * 2;  // 16 KB
constexpr uint32_t kBBytes = kTN * kTK * 2;  // 32 KB
constexpr uint32_t kStageBytes = kABytes + kBBytes;
// an epilogue warp's 32 x 32 FP32 staging block (rows of 128 bytes, 16-byte units swizzled)
constexpr size_t kStagingBytes = (size_t)kEpilogueWarps * 32 * 32 * 4;
constexpr size_t kSmemBytes = (size_t)kStages * kStageBytes + kStagingBytes + 1024 + 256;
static_assert(kSmemBytes + 64 <= 232448, "the ring, the staging and the barriers fit one CTA");
constexpr uint32_t kAccColumns = 256;      // one FP32 accumulator: 256 columns x 128 lanes
constexpr uint32_t kTmemColumns = 2 * kAccColumns;
constexpr uint32_t kIdesc = tc::idesc_bf16(kTM, kTN);
constexpr int kMaxProducts = 8;  // products of one launch (the ensemble's members)
using namespace tc;

// The products of one launch: the same shapes, operands and outputs of their own (the
// ensemble's members through one layer).  The tensor maps live in the kernel's parameters.
struct GemmBatch {
  CUtensorMap a[kMaxProducts], w[kMaxProducts];
  float* C[kMaxProducts];
  __nv_bfloat16* C16[kMaxProducts];
  const float* bias[kMaxProducts];
  int count;
};

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// A persistent CTA per SM walks the output tiles t = blockIdx.x, + gridDim.x, ... of every
// product of the batch in turn (the column tile fastest, so that the CTAs running together
// share A's rows in L2).  The ring
// of K slices runs on across tiles; the products of tile i go to accumulator i % 2, so that
// the epilogue warps drain one while the next tile's products fill the other:
//   full[s] / empty[s]   the ring's stages (TMA bytes in / products done reading)
//   acc_full[b]          the products of accumulator b's tile are complete (commit)
//   acc_empty[b]         the epilogue warps have read accumulator b (one arrival per warp)
// Every wait is bounded; a wait that gives up sets `failed`, which the other roles poll, and
// the CTA waits (bounded) for its own products and loads in flight before it frees its
// tensor memory.
__global__ void __launch_bounds__(kThreads, 1)
    k_mlp_gemm_tc(const __grid_constant__ GemmBatch p, int M, int N, int K, int ldc, int ldc16, int epilogue,
                  int* status) {
  extern __shared__ __align__(16) unsigned char tc_raw[];  // aligned to 1024 by hand (the slack)
  unsigned char* ring = reinterpret_cast<unsigned char*>(((uintptr_t)tc_raw + 1023) & ~(uintptr_t)1023);
  float* staging = reinterpret_cast<float*>(ring + (size_t)kStages * kStageBytes);
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + (size_t)kStages * kStageBytes + kStagingBytes);
  uint64_t* empty = full + kStages;
  uint64_t* acc_full = empty + kStages;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* drain = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  __shared__ volatile int failed;
  __shared__ int consumed;  // ring slices the products have taken (for the drain on failure)
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int n_k = K / kTK;
  const int tiles_n = N / kTN, per_product = tiles_n * ((M + kTM - 1) / kTM);
  const int tiles = per_product * p.count;
  if (threadIdx.x == 0) {
    failed = 0;
    consumed = 0;
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], kEpilogueWarps);
    }
    mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) {  // the whole warp allocates both accumulators' columns
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
    // producer: the K slices of every tile of this CTA, through the ring
    long g = 0;
    for (int t = blockIdx.x; t < tiles && !failed; t += gridDim.x) {
      const int q = t / per_product, u = t % per_product;
      const int m0 = (u / tiles_n) * kTM, n0 = (u % tiles_n) * kTN;
      for (int k = 0; k < n_k; ++k, ++g) {
        const int s = (int)(g % kStages);
        const uint32_t round = (uint32_t)(g / kStages);
        if (g >= kStages && !mbar_wait(&empty[s], (round - 1) & 1)) {
          failed = 1;
          break;
        }
        if (failed) break;
        unsigned char* stage = ring + (size_t)s * kStageBytes;
        mbar_expect_tx(&full[s], kStageBytes);
        tma_load_2d(stage, &p.a[q], &full[s], k * kTK, m0);
        tma_load_2d(stage + kABytes, &p.w[q], &full[s], k * kTK, n0);
      }
    }
    // on failure: the loads still in flight land before the CTA leaves
    if (failed)
      for (long h = consumed; h < g; ++h) mbar_wait(&full[h % kStages], (uint32_t)(h / kStages) & 1);
  } else if (threadIdx.x == 32) {
    // the MMA issuer: tile i into accumulator i % 2 once the epilogue has read it
    long g = 0;
    int it = 0;
    for (int t = blockIdx.x; t < tiles && !failed; t += gridDim.x, ++it) {
      const int b = it & 1, use = it >> 1;
      if (use >= 1 && !mbar_wait(&acc_empty[b], (use - 1) & 1)) {
        failed = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t acc = tmem + (uint32_t)b * kAccColumns;
      for (int k = 0; k < n_k; ++k, ++g) {
        const int s = (int)(g % kStages);
        const uint32_t round = (uint32_t)(g / kStages);
        if (!mbar_wait(&full[s], round & 1)) {
          failed = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const unsigned char* stage = ring + (size_t)s * kStageBytes;
        const uint64_t da = sw128_desc(stage), db = sw128_desc(stage + kABytes);
#pragma unroll
        for (int kk = 0; kk < kTK / 16; ++kk)
          umma_bf16(acc, da + 2ull * kk, db + 2ull * kk, kIdesc, (k | kk) != 0 ? 1u : 0u);
        umma_commit(&empty[s]);
        consumed = (int)(g + 1);
      }
      if (failed) break;
      umma_commit(&acc_full[b]);
    }
    umma_commit(drain);  // every product issued above has completed when this arrives
  } else if (warp >= 2) {
    // epilogue: warp w reads accumulator lanes (rows) 32 (w % 4) .. + 31, columns
    // kEpilogueColumns ((w - 2) / 4) onwards, 32 at a time: each lane applies the bias and
    // the GELU to its row's 32 values in registers, and the rows leave through the warp's
    // staging block as 16-byte stores
    const int quarter = warp % 4, slice = (warp - 2) / 4;
    float4* stg = reinterpret_cast<float4*>(staging + (size_t)(warp - 2) * 32 * 32);
    int it = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++it) {
      const int q = t / per_product, u = t % per_product;
      const int m0 = (u / tiles_n) * kTM, n0 = (u % tiles_n) * kTN;
      float* const C = p.C[q];
      __nv_bfloat16* const C16 = p.C16[q];
      const float* const bias = epilogue >= 1 ? p.bias[q] : nullptr;
      const int b = it & 1;
      const bool ok = mbar_wait(&acc_full[b], (it >> 1) & 1);
      if (!ok || failed) {
        failed = 1;
        break;
      }
      __syncwarp();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t acc = tmem + (uint32_t)b * kAccColumns + ((uint32_t)(quarter * 32) << 16);
      const int m_first = m0 + quarter * 32;
      const int rows = min(32, M - m_first);  // the rows inside the matrix
      for (int c = slice * kEpilogueColumns; c < (slice + 1) * kEpilogueColumns; c += 32) {
        uint32_t r[32];
        __syncwarp();  // the load is warp-wide (.sync.aligned)
        tmem_load_32(acc + (uint32_t)c, r);
        if (c + 32 == (slice + 1) * kEpilogueColumns) {
          // the accumulator is read: the next tile's products may overwrite it
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[b]);
        }
        const int nb = n0 + c;  // the chunk's first column
        float v[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
        if (bias) {
#pragma unroll
          for (int j4 = 0; j4 < 8; ++j4) {
            const float4 b4 = __ldg(reinterpret_cast<const float4*>(bias + nb) + j4);
            v[4 * j4] += b4.x;
            v[4 * j4 + 1] += b4.y;
            v[4 * j4 + 2] += b4.z;
            v[4 * j4 + 3] += b4.w;
          }
        }
        if (epilogue == 2) {
#pragma unroll
          for (int j = 0; j < 32; ++j) v[j] = gelu(v[j]);
        }
        if (C) {
          // FP32 rows: lane `lane` (row) writes its eight 16-byte units, unit s of row rr at
          // slot s ^ (rr & 7) (eight lanes of a wavefront, eight banks groups); then lanes
          // 8 i .. 8 i + 7 take row 4 k + i's units in turn, 16-byte stores along the row
#pragma unroll
          for (int s4 = 0; s4 < 8; ++s4)
            stg[lane * 8 + (s4 ^ (lane & 7))] = make_float4(v[4 * s4], v[4 * s4 + 1], v[4 * s4 + 2], v[4 * s4 + 3]);
          __syncwarp();
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const int rr = 4 * k + (lane >> 3), s4 = lane & 7;
            const float4 x = stg[rr * 8 + (s4 ^ (rr & 7))];
            if (rr < rows) *reinterpret_cast<float4*>(C + (size_t)(m_first + rr) * ldc + nb + 4 * s4) = x;
          }
          __syncwarp();
        }
        if (C16) {
          if (epilogue == 3) {  // training: the pre-activation above, its GELU here
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = gelu(v[j]);
          }
          // BF16 rows of 64 bytes: unit s (eight values) of row rr at slot s ^ ((rr >> 1) & 3)
          // of that row's four; lanes 4 i .. 4 i + 3 then take row 8 k + i's units
          uint4* stg16 = reinterpret_cast<uint4*>(stg);
#pragma unroll
          for (int s8 = 0; s8 < 4; ++s8) {
            uint32_t w[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
              const __nv_bfloat162 pair = __floats2bfloat162_rn(v[8 * s8 + 2 * h], v[8 * s8 + 2 * h + 1]);
              w[h] = *reinterpret_cast<const uint32_t*>(&pair);
            }
            stg16[lane * 4 + (s8 ^ ((lane >> 1) & 3))] = make_uint4(w[0], w[1], w[2], w[3]);
          }
          __syncwarp();
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int rr = 8 * k + (lane >> 2), s8 = lane & 3;
            const uint4 x = stg16[rr * 4 + (s8 ^ ((rr >> 1) & 3))];
            if (rr < rows) *reinterpret_cast<uint4*>(C16 + (size_t)(m_first + rr) * ldc16 + nb + 8 * s8) = x;
          }
          __syncwarp();
        }
      }
    }
  }
  __syncwarp();  // warps 0 and 1 wait for their producing / issuing lane before the barrier
  __syncthreads();
  // the products issued (all of them, or those before a failure) are complete
  if (threadIdx.x == 0 && !mbar_wait(drain, 0)) failed = 1;
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemColumns) : "memory");
  if (threadIdx.x == 0 && failed) atomicExch(status, 1);
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

sp_status sp_mlp_gemm_tc_batch(int count, const void* const* A, int lda, const void* const* W, int ldw,
                               float* const* C, int ldc, void* const* C16, int ldc16, int M, int N, int K,
                               const float* const* bias, int epilogue, int* status, void* stream) {
  using namespace sp;
  if (count < 1 || count > kMaxProducts || !A || !W || !status || M < 1 || N < 1 || K < 1 || epilogue < 0 ||
      epilogue > 3)
    return SP_ERR_ARGUMENT;
  // the tiling's and the tensor maps' rules: whole 256-column tiles and 64-wide K slices,
  // 16-byte aligned rows
  if (N % kTN || K % kTK || lda % 8 || ldw % 8 || lda < K || ldw < K) return SP_ERR_ARGUMENT;
  // the epilogue's 16-byte row stores and bias loads
  if ((C && ldc % 4) || (C16 && ldc16 % 8)) return SP_ERR_ARGUMENT;
  GemmBatch batch{};
  batch.count = count;
  for (int q = 0; q < count; ++q) {
    float* c = C ? C[q] : nullptr;
    void* c16 = C16 ? C16[q] : nullptr;
    if (!A[q] || !W[q] || (!c && !c16)) return SP_ERR_ARGUMENT;
    if (((uintptr_t)A[q] | (uintptr_t)W[q] | (uintptr_t)c | (uintptr_t)c16) & 15) return SP_ERR_ARGUMENT;
    if (bias && bias[q] && ((uintptr_t)bias[q] & 15)) return SP_ERR_ARGUMENT;
    if (!make_map(&batch.a[q], A[q], M, K, lda, kTM) || !make_map(&batch.w[q], W[q], N, K, ldw, kTN))
      return SP_ERR_CUDA;
    batch.C[q] = c;
    batch.C16[q] = static_cast<__nv_bfloat16*>(c16);
    batch.bias[q] = bias ? bias[q] : nullptr;
  }
  static std::once_flag configured;
  std::call_once(configured, [] {
    cudaFuncSetAttribute(k_mlp_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
  });
  static int n_sms = 0;
  if (!n_sms) {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess ||
        cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || n_sms < 1)
      return SP_ERR_CUDA;
  }
  const int tiles = count * (N / kTN) * ((M + kTM - 1) / kTM);
  k_mlp_gemm_tc<<<tiles < n_sms ? tiles : n_sms, kThreads, kSmemBytes, (cudaStream_t)stream>>>(
      batch, M, N, K, ldc, ldc16, epilogue, status);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ERR_CUDA;
}

sp_status sp_mlp_gemm_tc(const void* A, int lda, const void* W, int ldw, float* C, int ldc, void* C16,
                         int ldc16, int M, int N, int K, const float* bias, int epilogue, int* status,
                         void* stream) {
  if (!C && !C16) return SP_ERR_ARGUMENT;
  return sp_mlp_gemm_tc_batch(1, &A, lda, &W, ldw, &C, ldc, &C16, ldc16, M, N, K, &bias, epilogue, status,
                              stream);
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
