// The modal transform as dense products: the GEMM route of the source evaluation.
//
// The reference synthesises the node field E[i, t] = tau sum_m S[i, m] a[m, t] and projects
// the node streams back, P_m(t) = sum_i W[m, i] P_i(t) / tau, as matrix products
// (src/solprop/backends/numpy_ref/passes/transforms.py:87-187; the native backend's
// synthesis provider native/src/general/trial.cpp:181-315 and its GEMM wrapper
// native/include/solprop_native/transforms/gemm.hpp:55-275).  On the fused route the
// response column synthesises and projects on CUDA cores from a modal window in shared
// memory; this route takes the products out of the column, so that any number of modes
// and nodes fits:
//
//   plain form (FP64):   k_gemm_f64, a tiled FP64 product, k summed in order;
//   mixed form (FP32):   each operand split into three BF16 parts x = hi + mid + lo
//                        (hi = bf16(x), mid = bf16(x - hi), lo = bf16(x - hi - mid)), and
//                        the six leading cross products hi.hi, mid.hi, hi.mid, lo.hi,
//                        mid.mid, hi.lo accumulated in FP32 by tcgen05.mma in tensor
//                        memory -- the K loop walks the six (A part, B part) pairs, so no
//                        operand is duplicated -- which keeps the product to FP32 accuracy
//                        (the terms left out are below 2^-24 of the leading one).
//
// The tcgen05 kernel: one CTA of sixteen warps per 128 x BN output tile; TMA brings 64-wide
// K slices of the A and B parts (K-major, 128-byte swizzle, no multicast) through a
// four-stage mbarrier ring; one thread issues the MMAs; all warps drain the accumulator.
// Every wait is bounded and a give-up marks *status (the column's status slot, which the
// host reads with the norms); tensor memory is freed on every path.
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "kernels.cuh"
#include "tcgen05.cuh"

namespace sp {
namespace {

using namespace tc;

constexpr int kGM = 128, kGK = 64, kGStages = 4, kGThreads = 512;
constexpr uint32_t kGABytes = kGM * kGK * 2;  // 16 KB
template <int BN> constexpr uint32_t stage_bytes() { return kGABytes + (uint32_t)BN * kGK * 2; }
template <int BN> constexpr size_t gemm_smem() { return (size_t)kGStages * stage_bytes<BN>() + 1024 + 256; }

// the six (A part, B part) pairs, the largest products last
__constant__ int c_terms[6][2] = {{2, 0}, {0, 2}, {1, 1}, {1, 0}, {0, 1}, {0, 0}};

struct SplitMaps {
  CUtensorMap a[3];
  CUtensorMap b[3];
};

template <int BN>
__global__ void __launch_bounds__(kGThreads, 1)
    k_gemm_split3(const __grid_constant__ SplitMaps maps, float* C, int ldc, int M, int n_valid, int K,
                  int transposed, const double* scale, int divide, double* status, size_t split_stride) {
  constexpr uint32_t kStage = stage_bytes<BN>();
  constexpr uint32_t kIdescN = idesc_bf16(kGM, BN);
  extern __shared__ __align__(1024) unsigned char g_raw[];
  unsigned char* ring = reinterpret_cast<unsigned char*>(((uintptr_t)g_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + (size_t)kGStages * kStage);
  uint64_t* empty = full + kGStages;
  uint64_t* done = empty + kGStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ int failed;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int m0 = blockIdx.y * kGM, n0 = blockIdx.x * BN;
  // split K: CTA z of gridDim.z takes K slices [ks0, ks1) of every term and writes its own
  // partial tile, C + z split_stride (added in split order by k_reduce_splits)
  const int n_all = K / kGK;
  const int ks0 = (int)((long)blockIdx.z * n_all / gridDim.z), ks1 = (int)((long)(blockIdx.z + 1) * n_all / gridDim.z);
  const int n_k = ks1 - ks0;
  const int total = 6 * n_k;
  C += (size_t)blockIdx.z * split_stride;
  if (threadIdx.x == 0) {
    failed = 0;
    for (int s = 0; s < kGStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (threadIdx.x == 0) {
    for (int it = 0; it < total; ++it) {
      const int s = it % kGStages;
      const uint32_t round = it / kGStages;
      if (it >= kGStages && !mbar_wait(&empty[s], (round - 1) & 1)) {
        failed = 1;
        break;
      }
      const int term = it / n_k, ks = ks0 + it % n_k;
      unsigned char* stage = ring + (size_t)s * kStage;
      mbar_expect_tx(&full[s], kStage);
      tma_load_2d(stage, &maps.a[c_terms[term][0]], &full[s], ks * kGK, m0);
      tma_load_2d(stage + kGABytes, &maps.b[c_terms[term][1]], &full[s], ks * kGK, n0);
    }
  } else if (threadIdx.x == 32) {
    for (int it = 0; it < total; ++it) {
      const int s = it % kGStages;
      const uint32_t round = it / kGStages;
      if (!mbar_wait(&full[s], round & 1)) {
        failed = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const unsigned char* stage = ring + (size_t)s * kStage;
      const uint64_t da = sw128_desc(stage), db = sw128_desc(stage + kGABytes);
#pragma unroll
      for (int kk = 0; kk < kGK / 16; ++kk)
        umma_bf16(tmem, da + 2ull * kk, db + 2ull * kk, kIdescN, (it | kk) != 0 ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    umma_commit(done);
  }
  __syncwarp();
  const bool ok = mbar_wait(done, 0);
  __syncwarp();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // drain: warp w reads accumulator lanes 32 (w % 4) .. + 31 and a quarter of the columns
  constexpr int kPitch = BN + 1;
  static_assert((size_t)kGM * kPitch * 4 <= (size_t)kGStages * kStage, "the tile fits in the ring");
  float* tile = reinterpret_cast<float*>(ring);
  const int quarter = warp % 4;
  const int row = quarter * 32 + lane;
  constexpr int kCols = BN / 4;
  const int c_lo = (warp / 4) * kCols;
  if constexpr (kCols >= 32) {
    for (int c = c_lo; c < c_lo + kCols; c += 32) {
      uint32_t r[32];
      __syncwarp();
      tmem_load_32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c, r);
#pragma unroll
      for (int j = 0; j < 32; ++j) tile[row * kPitch + c + j] = __uint_as_float(r[j]);
    }
  } else {
    uint32_t r[16];
    __syncwarp();
    tmem_load_16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c_lo, r);
#pragma unroll
    for (int j = 0; j < 16; ++j) tile[row * kPitch + c_lo + j] = __uint_as_float(r[j]);
  }
  __syncthreads();
  if (ok && !failed && total > 0) {
    const float f = scale ? (float)(divide ? 1.0 / *scale : *scale) : 1.0f;
    if (!transposed) {
      // C[m][n]: a warp per row, lanes along n
      for (int rr = warp; rr < kGM && m0 + rr < M; rr += kGThreads / 32)
        for (int cc = lane; cc < BN && n0 + cc < n_valid; cc += 32)
          C[(size_t)(m0 + rr) * ldc + n0 + cc] = f * tile[rr * kPitch + cc];
    } else {
      // C[n][m]: a warp per column, lanes along m
      for (int cc = warp; cc < BN && n0 + cc < n_valid; cc += kGThreads / 32)
        for (int rr = lane; rr < kGM && m0 + rr < M; rr += 32)
          C[(size_t)(n0 + cc) * ldc + m0 + rr] = f * tile[rr * kPitch + cc];
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN) : "memory");
  if (threadIdx.x == 0 && (!ok || failed)) *status = 1.0;
}

// out[i] = f sum_z partials[z][i], the splits added in order; f = *scale or 1 / *scale
template <class T>
__global__ void k_reduce_splits(const T* __restrict__ partials, int splits, size_t count, size_t stride,
                                T* __restrict__ out, size_t out_stride, int rows, const double* scale,
                                int divide) {
  // `rows` blocks of `count` values, block r at r * stride in each split and r * out_stride out
  const T f = (T)(divide ? 1.0 / *scale : *scale);
  const size_t total = (size_t)rows * count;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
    const size_t r = g / count, i = g % count;
    T acc = T(0);
    for (int z = 0; z < splits; ++z) acc += partials[(size_t)z * rows * stride + r * stride + i];
    out[r * out_stride + i] = f * acc;
  }
}

// the three BF16 parts of x, in the order hi, mid, lo
template <class T>
__device__ __forceinline__ void split3(T x, __nv_bfloat16 (&p)[3]) {
  const float v = (float)x;
  p[0] = __float2bfloat16_rn(v);
  const float r1 = v - __bfloat162float(p[0]);
  p[1] = __float2bfloat16_rn(r1);
  p[2] = __float2bfloat16_rn(r1 - __bfloat162float(p[1]));
}

// out[p][r][c] = part p of src[c][r] (c < C; 0 for C <= c < ld_out), r < R; 64 (c) x 32 (r)
// tiles through shared memory: the source is read in 128-byte rows, and each warp stores a
// part's 64 columns of one row as 32 BF16 pairs, a 128-byte row.  src rows have pitch
// ld_src; ld_out is even.
template <class T>
__global__ void __launch_bounds__(256) k_split3_transpose(const T* __restrict__ src, int C, int R, int ld_src,
                                                          __nv_bfloat16* __restrict__ out, int ld_out) {
  __shared__ T tile[64][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 64;
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;  // 32 x 8
  for (int j = ty; j < 64; j += 8) {
    const int c = c0 + j, r = r0 + tx;
    tile[j][tx] = (c < C && r < R) ? src[(size_t)c * ld_src + r] : T(0);
  }
  __syncthreads();
  const size_t panel = (size_t)R * ld_out;
  for (int j = ty; j < 32; j += 8) {
    const int r = r0 + j, c = c0 + 2 * tx;
    if (r >= R || c >= ld_out) continue;
    __nv_bfloat16 a[3], b[3];
    split3(tile[2 * tx][j], a);
    split3(tile[2 * tx + 1][j], b);
    const size_t at = (size_t)r * ld_out + c;
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      __nv_bfloat162 v;
      v.x = a[p];
      v.y = b[p];
      *reinterpret_cast<__nv_bfloat162*>(out + p * panel + at) = v;
    }
  }
}

// C[M, N] = f (A[M, K] B[K, N]), row-major, f = *scale or 1 / *scale; 64 x 64 tiles, each
// thread 4 x 4 outputs, k summed in order
constexpr int kFM = 64, kFN = 64, kFK = 16;
__global__ void __launch_bounds__(256) k_gemm_f64(const double* __restrict__ A, int lda, const double* __restrict__ B,
                                                  int ldb, double* __restrict__ C, int ldc, int M, int N, int K,
                                                  const double* scale, int divide, size_t split_stride) {
  __shared__ double As[kFK][kFM + 1];
  __shared__ double Bs[kFK][kFN + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * kFM, n0 = blockIdx.x * kFN;
  // split K over gridDim.z: this CTA's slices of kFK, its partial tile at C + z split_stride
  const int n_all = (K + kFK - 1) / kFK;
  const int kb0 = (int)((long)blockIdx.z * n_all / gridDim.z), kb1 = (int)((long)(blockIdx.z + 1) * n_all / gridDim.z);
  C += (size_t)blockIdx.z * split_stride;
  double acc[4][4] = {};
  for (int k0 = kb0 * kFK; k0 < kb1 * kFK; k0 += kFK) {
    for (int i = threadIdx.x; i < kFM * kFK; i += 256) {
      const int mm = i / kFK, kk = i % kFK;
      As[kk][mm] = (m0 + mm < M && k0 + kk < K) ? A[(size_t)(m0 + mm) * lda + k0 + kk] : 0.0;
    }
    for (int i = threadIdx.x; i < kFK * kFN; i += 256) {
      const int kk = i / kFN, nn = i % kFN;
      Bs[kk][nn] = (k0 + kk < K && n0 + nn < N) ? B[(size_t)(k0 + kk) * ldb + n0 + nn] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kFK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  const double s = scale ? *scale : 1.0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 16 * i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx + 16 * j;
      if (n < N) C[(size_t)m * ldc + n] = !scale ? acc[i][j] : divide ? acc[i][j] / s : s * acc[i][j];
    }
  }
}

// split-K factor: enough CTAs for about four waves of the 148 SMs, each split at least
// `min_slices` K slices long
int splits_for(int tiles, int k_slices, int min_slices) {
  int s = 1;
  while (tiles * s < 4 * 148 && k_slices / (2 * s) >= min_slices) s *= 2;
  return s;
}

bool split_maps(SplitMaps* maps, const uint16_t* a_parts, int a_rows, const uint16_t* b_parts, int b_rows,
                int kpad, int box_n) {
  const size_t a_panel = (size_t)a_rows * kpad, b_panel = (size_t)b_rows * kpad;
  for (int p = 0; p < 3; ++p) {
    if (!make_bf16_map(&maps->a[p], a_parts + p * a_panel, a_rows, kpad, kpad, kGM, kGK)) return false;
    if (!make_bf16_map(&maps->b[p], b_parts + p * b_panel, b_rows, kpad, kpad, box_n, kGK)) return false;
  }
  return true;
}

template <class T>
cudaError_t split_transpose(const T* src, int C, int R, int ld_src, uint16_t* out, int ld_out, cudaStream_t s) {
  const dim3 grid((R + 31) / 32, (ld_out + 63) / 64);
  k_split3_transpose<T><<<grid, 256, 0, s>>>(src, C, R, ld_src, reinterpret_cast<__nv_bfloat16*>(out), ld_out);
  return cudaGetLastError();
}

}  // namespace

int modal_kpad(int k) { return ((k + kGK - 1) / kGK) * kGK; }

cudaError_t configure_modal_gemm() {
  cudaError_t e = cudaFuncSetAttribute(k_gemm_split3<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)gemm_smem<256>());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_gemm_split3<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)gemm_smem<64>());
}

void split3_host(const double* src, int rows, int cols, int ld_out, std::vector<uint16_t>& out) {
  out.assign((size_t)3 * rows * ld_out, 0);
  const size_t panel = (size_t)rows * ld_out;
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c) {
      const float v = (float)src[(size_t)r * cols + c];
      const __nv_bfloat16 hi = __float2bfloat16_rn(v);
      const float r1 = v - __bfloat162float(hi);
      const __nv_bfloat16 mid = __float2bfloat16_rn(r1);
      const __nv_bfloat16 lo = __float2bfloat16_rn(r1 - __bfloat162float(mid));
      const size_t at = (size_t)r * ld_out + c;
      out[at] = __bfloat16_as_ushort(hi);
      out[panel + at] = __bfloat16_as_ushort(mid);
      out[2 * panel + at] = __bfloat16_as_ushort(lo);
    }
}

cudaError_t modal_synthesis_f64(const double* S, const double* modal, double* E, int n_nodes, int n_modes,
                                int n_to, const double* taper, cudaStream_t s) {
  const dim3 grid((n_to + kFN - 1) / kFN, (n_nodes + kFM - 1) / kFM);
  k_gemm_f64<<<grid, 256, 0, s>>>(S, n_modes, modal, n_to, E, n_to, n_nodes, n_to, n_modes, taper, 0, 0);
  return cudaGetLastError();
}

size_t modal_projection_scratch(int n_modes, int n_nodes, int n_to) {
  const int tiles_f64 = ((n_to + kFN - 1) / kFN) * ((n_modes + kFM - 1) / kFM);
  const int tiles_tc = (n_modes + 63) / 64 * ((n_to + kGM - 1) / kGM);
  const int s = std::max(splits_for(tiles_f64, (n_nodes + kFK - 1) / kFK, 16),
                         splits_for(tiles_tc, modal_kpad(n_nodes) / kGK, 4));
  return (size_t)s * n_modes * n_to;
}

cudaError_t modal_projection_f64(const double* W, const double* node_streams, double* out, int n_streams,
                                 int n_modes, int n_nodes, int n_to, size_t out_stride, const double* taper,
                                 double* scratch, cudaStream_t s) {
  const int tiles = ((n_to + kFN - 1) / kFN) * ((n_modes + kFM - 1) / kFM);
  const int splits = splits_for(tiles, (n_nodes + kFK - 1) / kFK, 16);
  const size_t part = (size_t)n_modes * n_to;
  const dim3 grid((n_to + kFN - 1) / kFN, (n_modes + kFM - 1) / kFM, splits);
  for (int st = 0; st < n_streams; ++st) {
    k_gemm_f64<<<grid, 256, 0, s>>>(W, n_nodes, node_streams + (size_t)st * n_nodes * n_to, n_to, scratch, n_to,
                                    n_modes, n_to, n_nodes, nullptr, 1, part);
    k_reduce_splits<double><<<592, 256, 0, s>>>(scratch, splits, part, part, out + st * out_stride, part, 1,
                                                taper, 1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t modal_synthesis_split3(const uint16_t* s_parts, const double* modal, uint16_t* modal_parts, float* E,
                                   int n_nodes, int n_modes, int n_to, int kpad, const double* taper,
                                   double* status, cudaStream_t s) {
  // B = the modal field transposed, (n_to, kpad) in three parts
  cudaError_t e = split_transpose<double>(modal, n_modes, n_to, n_to, modal_parts, kpad, s);
  if (e != cudaSuccess) return e;
  SplitMaps maps;
  if (!split_maps(&maps, s_parts, n_nodes, modal_parts, n_to, kpad, 256)) return cudaErrorInvalidValue;
  const dim3 grid((n_to + 255) / 256, (n_nodes + kGM - 1) / kGM);
  k_gemm_split3<256><<<grid, kGThreads, gemm_smem<256>(), s>>>(maps, E, n_to, n_nodes, n_to, kpad, 0, taper, 0,
                                                                status, 0);
  return cudaGetLastError();
}

cudaError_t modal_projection_split3(const uint16_t* w_parts, const float* node_streams, uint16_t* node_parts,
                                    float* out, int n_streams, int n_modes, int n_nodes, int n_to, int kpad,
                                    size_t out_stride, const double* taper, double* status, float* scratch,
                                    cudaStream_t s) {
  const int tiles = (n_modes + 63) / 64 * ((n_to + kGM - 1) / kGM);
  const int splits = splits_for(tiles, kpad / kGK, 4);
  const size_t part = (size_t)n_modes * n_to;
  for (int st = 0; st < n_streams; ++st) {
    // A = the stream transposed, (n_to, kpad) in three parts
    cudaError_t e = split_transpose<float>(node_streams + (size_t)st * n_nodes * n_to, n_nodes, n_to, n_to,
                                           node_parts, kpad, s);
    if (e != cudaSuccess) return e;
    SplitMaps maps;
    if (!split_maps(&maps, node_parts, n_to, w_parts, n_modes, kpad, 64)) return cudaErrorInvalidValue;
    const dim3 grid((n_modes + 63) / 64, (n_to + kGM - 1) / kGM, splits);
    k_gemm_split3<64><<<grid, kGThreads, gemm_smem<64>(), s>>>(maps, scratch, n_to, n_to, n_modes, kpad, 1,
                                                               nullptr, 1, status, part);
    k_reduce_splits<float><<<592, 256, 0, s>>>(scratch, splits, part, part, out + st * out_stride, part, 1, taper,
                                               1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace sp
