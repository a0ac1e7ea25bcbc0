// The scan surrogate's multilayer perceptron: forward, backward and optimiser kernels.
//
// Tensors live in HBM as FP32 (row-major, leading dimensions in elements).  Every matrix
// product runs on the tensor cores in BF16 with FP32 accumulation: the tile loader
// rounds each FP32 operand to BF16 (round to nearest even) as it stages the tile in
// shared memory, and mma.sync m16n8k16 accumulates in FP32.  The forward product fuses
// its epilogue (bias, GELU, and the pre-activation kept for the backward pass); the
// backward products (dX = dZ W, dW = dZ^T X) use the same kernel with transposed
// operand views.  Reductions (bias gradients, the loss) have a fixed order.
//
//   C[M, N] = op(A)[M, K] op(B)[K, N]     op(A)(m, k) = transA ? A[k lda + m] : A[m lda + k]
//                                         op(B)(k, n) = transB ? B[n ldb + k] : B[k ldb + n]
//
// A linear layer y = x W^T + b with W (N, K) is (A = x, B = W, transB = 1).
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>

namespace sp {
namespace {

constexpr int kBM = 128, kBN = 128, kBK = 32;
constexpr int kPad = 8;               // bf16 elements of padding per shared row
constexpr int kLd = kBK + kPad;       // shared row length (k contiguous)
constexpr int kGemmThreads = 256;     // 8 warps: 2 (m) x 4 (n), each 64 x 32

// 0.5 x (1 + erf(x / sqrt 2)): the exact GELU
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

struct GemmArgs {
  const float* A;
  const float* B;
  float* C;
  const float* bias;  // (N) or null
  float* pre;         // (M, N) pre-activation kept when the epilogue applies GELU, or null
  int lda, ldb, ldc, ldpre;
  int M, N, K;
  int transA, transB;
  int epilogue;       // 0: C = AB, 1: C = AB + bias, 2: C = GELU(AB + bias)
};

// Stage op(A)[m0 : m0 + 128, k0 : k0 + 32] as As[m][k] and op(B)[k0 : k0 + 32, n0 : n0 + 128]
// as Bs[n][k], rounded to BF16; elements outside the matrices are zero.
__device__ __forceinline__ void load_tiles(const GemmArgs& g, int m0, int n0, int k0, __nv_bfloat16* As,
                                           __nv_bfloat16* Bs) {
  const int t = threadIdx.x;
  // A: 128 x 32 elements, 16 per thread; read along A's contiguous index
  if (!g.transA) {
    for (int e = t; e < kBM * kBK; e += kGemmThreads) {
      const int m = e / kBK, k = e % kBK;
      const int gm = m0 + m, gk = k0 + k;
      const float v = (gm < g.M && gk < g.K) ? g.A[(size_t)gm * g.lda + gk] : 0.0f;
      As[m * kLd + k] = __float2bfloat16_rn(v);
    }
  } else {
    for (int e = t; e < kBM * kBK; e += kGemmThreads) {
      const int k = e / kBM, m = e % kBM;
      const int gm = m0 + m, gk = k0 + k;
      const float v = (gm < g.M && gk < g.K) ? g.A[(size_t)gk * g.lda + gm] : 0.0f;
      As[m * kLd + k] = __float2bfloat16_rn(v);
    }
  }
  if (g.transB) {
    for (int e = t; e < kBN * kBK; e += kGemmThreads) {
      const int n = e / kBK, k = e % kBK;
      const int gn = n0 + n, gk = k0 + k;
      const float v = (gn < g.N && gk < g.K) ? g.B[(size_t)gn * g.ldb + gk] : 0.0f;
      Bs[n * kLd + k] = __float2bfloat16_rn(v);
    }
  } else {
    for (int e = t; e < kBN * kBK; e += kGemmThreads) {
      const int k = e / kBN, n = e % kBN;
      const int gn = n0 + n, gk = k0 + k;
      const float v = (gn < g.N && gk < g.K) ? g.B[(size_t)gk * g.ldb + gn] : 0.0f;
      Bs[n * kLd + k] = __float2bfloat16_rn(v);
    }
  }
}

__device__ __forceinline__ uint32_t smem_pair(const __nv_bfloat16* p) {
  return *reinterpret_cast<const uint32_t*>(p);
}

// mma.sync m16n8k16, row (A) x col (B), BF16 in, FP32 accumulate
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(kGemmThreads) k_mlp_gemm(GemmArgs g) {
  __shared__ __align__(16) __nv_bfloat16 As[kBM * kLd];
  __shared__ __align__(16) __nv_bfloat16 Bs[kBN * kLd];
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int wm = (warp / 4) * 64, wn = (warp % 4) * 32;  // the warp's 64 x 32 sub-tile
  const int gid = lane >> 2, tig = lane & 3;              // fragment row group, thread in group
  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0f;
  for (int k0 = 0; k0 < g.K; k0 += kBK) {
    load_tiles(g, m0, n0, k0, As, Bs);
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 16) {
      uint32_t a[4][4], b[4][2];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const __nv_bfloat16* base = As + (wm + i * 16 + gid) * kLd + kk + tig * 2;
        a[i][0] = smem_pair(base);
        a[i][1] = smem_pair(base + 8 * kLd);
        a[i][2] = smem_pair(base + 8);
        a[i][3] = smem_pair(base + 8 * kLd + 8);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const __nv_bfloat16* base = Bs + (wn + j * 8 + gid) * kLd + kk + tig * 2;
        b[j][0] = smem_pair(base);
        b[j][1] = smem_pair(base + 8);
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
  // epilogue: rows gid and gid + 8 of each m16 tile, columns 2 tig and 2 tig + 1 of each n8
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int m = m0 + wm + i * 16 + gid + (r >= 2 ? 8 : 0);
        const int n = n0 + wn + j * 8 + tig * 2 + (r & 1);
        if (m >= g.M || n >= g.N) continue;
        float v = acc[i][j][r];
        if (g.epilogue >= 1 && g.bias) v += g.bias[n];
        if (g.epilogue == 2) {
          if (g.pre) g.pre[(size_t)m * g.ldpre + n] = v;
          v = gelu(v);
        }
        g.C[(size_t)m * g.ldc + n] = v;
      }
}

__global__ void k_gelu_backward(const float* dA, const float* pre, float* dZ, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dZ[i] = dA[i] * gelu_grad(pre[i]);
}

// db[n] = sum_m dZ[m, n]: one thread per column, rows in order
__global__ void k_bias_grad(const float* dZ, int M, int N, int ld, float* db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.0f;
  for (int m = 0; m < M; ++m) s += dZ[(size_t)m * ld + n];
  db[n] = s;
}

// dY = 2 (Y - T) / (M N); per-row partial losses, summed by k_loss_total in row order
__global__ void k_mse(const float* Y, const float* T, int M, int N, float* dY, float* row_loss) {
  const int m = blockIdx.x;
  __shared__ float part[256];
  float s = 0.0f;
  const float scale = 2.0f / ((float)M * (float)N);
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    const size_t i = (size_t)m * N + n;
    const float d = Y[i] - T[i];
    dY[i] = scale * d;
    s += d * d;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) row_loss[m] = part[0];
}

__global__ void k_loss_total(const float* row_loss, int M, int N, float* loss) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int m = 0; m < M; ++m) s += row_loss[m];
  *loss = (float)(s / ((double)M * (double)N));
}

// Adam (Kingma & Ba 2015) with bias correction, FP32 master weights
__global__ void k_adam(float* w, const float* grad, float* m1, float* m2, size_t n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = grad[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
  }
}

// The ensemble's statistics of one point (one block per row): the mean over members of
// every output, and the disagreement -- the members' standard deviation of each output
// weighted by the mean spectrum's energy in that output, 10^mean (outputs are log10
// spectral densities), over the summed weights.  Y holds (members, M, N); mean (M, N).
__global__ void k_ensemble_stats(const float* Y, int members, int M, int N, float* mean, float* spread) {
  const int m = blockIdx.x;
  __shared__ float part[256];
  __shared__ float part_w[256];
  float peak = -INFINITY;
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    float mu = 0.0f;
    for (int e = 0; e < members; ++e) mu += Y[((size_t)e * M + m) * N + n];
    mu /= (float)members;
    mean[(size_t)m * N + n] = mu;
    peak = fmaxf(peak, mu);
  }
  part[threadIdx.x] = peak;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] = fmaxf(part[threadIdx.x], part[threadIdx.x + w]);
    __syncthreads();
  }
  peak = part[0];
  __syncthreads();
  float s = 0.0f, sw = 0.0f;
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    const float mu = mean[(size_t)m * N + n];
    float var = 0.0f;
    for (int e = 0; e < members; ++e) {
      const float d = Y[((size_t)e * M + m) * N + n] - mu;
      var += d * d;
    }
    const float weight = exp10f(mu - peak);
    s += weight * sqrtf(var / (float)members);
    sw += weight;
  }
  part[threadIdx.x] = s;
  part_w[threadIdx.x] = sw;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      part[threadIdx.x] += part[threadIdx.x + w];
      part_w[threadIdx.x] += part_w[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) spread[m] = part_w[0] > 0.0f ? part[0] / part_w[0] : 0.0f;
}

inline unsigned grid_for(size_t n) {
  const size_t b = (n + 255) / 256;
  return (unsigned)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

}  // namespace
}  // namespace sp

#include "solprop_b200.h"

extern "C" {

sp_status sp_mlp_gemm(const float* A, int lda, int transA, const float* B, int ldb, int transB, float* C,
                      int ldc, int M, int N, int K, const float* bias, int epilogue, float* pre,
                      void* stream) {
  if (!A || !B || !C || M < 0 || N < 0 || K < 0 || epilogue < 0 || epilogue > 2) return SP_ERR_ARGUMENT;
  if (M == 0 || N == 0) return SP_OK;
  sp::GemmArgs g{A, B, C, bias, pre, lda, ldb, ldc, ldc, M, N, K, transA, transB, epilogue};
  const dim3 grid((N + sp::kBN - 1) / sp::kBN, (M + sp::kBM - 1) / sp::kBM);
  sp::k_mlp_gemm<<<grid, sp::kGemmThreads, 0, (cudaStream_t)stream>>>(g);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ERR_CUDA;
}

sp_status sp_mlp_gelu_backward(const float* dA, const float* pre, float* dZ, size_t n, void* stream) {
  if (!dA || !pre || !dZ) return SP_ERR_ARGUMENT;
  if (!n) return SP_OK;
  sp::k_gelu_backward<<<sp::grid_for(n), 256, 0, (cudaStream_t)stream>>>(dA, pre, dZ, n);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ERR_CUDA;
}

sp_status sp_mlp_bias_grad(const float* dZ, int M, int N, float* db, void* stream) {
  if (!dZ || !db || M < 0 || N < 0) return SP_ERR_ARGUMENT;
  if (!N) return SP_OK;
  sp::k_bias_grad<<<(N + 127) / 128, 128, 0, (cudaStream_t)stream>>>(dZ, M, N, N, db);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ERR_CUDA;
}

sp_status sp_mlp_mse(const float* Y, const float* T, int M, int N, float* dY, float* row_loss,
                     float* loss, void* stream) {
  if (!Y || !T || !dY || !row_loss || !loss || M < 1 || N < 1) return SP_ERR_ARGUMENT;
  sp::k_mse<<<M, 256, 0, (cudaStream_t)stream>>>(Y, T, M, N, dY, row_loss);
  sp::k_loss_total<<<1, 32, 0, (cudaStream_t)stream>>>(row_loss, M, N, loss);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ERR_CUDA;
}

sp_status sp_mlp_adam(float* w, const float* grad, float* m1, float* m2, size_t n, float lr, float beta1,
                      float beta2, float eps, int step, void* stream) {
  if (!w || !grad || !m1 || !m2 || step < 1) return SP_ERR_ARGUMENT;
  if (!n) return SP_OK;
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  sp::k_adam<<<sp::grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, grad, m1, m2, n, lr, beta1, beta2, eps,
                                                               c1, c2);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ERR_CUDA;
}

sp_status sp_mlp_ensemble_stats(const float* Y, int members, int M, int N, float* mean, float* spread,
                                void* stream) {
  if (!Y || !mean || !spread || members < 1 || M < 0 || N < 1) return SP_ERR_ARGUMENT;
  if (!M) return SP_OK;
  sp::k_ensemble_stats<<<M, 256, 0, (cudaStream_t)stream>>>(Y, members, M, N, mean, spread);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ERR_CUDA;
}

}  // extern "C"
