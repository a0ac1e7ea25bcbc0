// The kernels of one source evaluation on the modal route (field grid): solprop's
// passes 2-7 (docs/dev/architecture.md section 8), restated for sm_100a.  The transforms
// are templates over the real type: FP64, or FP32 in the mixed-precision form, whose
// stage output still combines in FP64.
//
//   k_inverse_field   pad + c2r inverse transform of every modal column, in shared
//                     memory; epilogue writes the modal field and the in-stage
//                     absorber's stream -alpha(t) a(t) / 2      (transforms.py:31-84,
//                                                                stepping.py:286-369)
//   (the response column and the projection: column_kernels.cu)
//   k_forward_field   r2c forward transform of every stream row and the crop
//                                                                (transforms.py:190)
//   k_stage_output    held plasma assembly, prefactor, window, absorber, inverse
//                     propagator                       (plasma.py:579, stepping.py:88)
#include <algorithm>

#include "fft.cuh"
#include "kernels.cuh"
#include "stage_output.cuh"

namespace sp {

// a row's block: up to 512 threads, so that each keeps its 16 (FP32) or 8 (FP64) points
// and their twiddles in registers
constexpr int kRowThreads = 512;

// ----------------------------------------------------------------------------- K1
template <class R>
__device__ __forceinline__ void inverse_field_body(const InverseArgsT<R>& a, int col) {
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* smem_c = reinterpret_cast<C*>(smem_raw);
  const int M = a.n_to >> 1;  // complex length
  const double2* lab = a.lab + (size_t)col * a.n_omega;
  const C* tw = a.twiddles;
  // X[k] for k in [0, M]; pocketfft's irfft reads only the real part of the DC and
  // Nyquist bins, so those are taken real here too.
  // the field grid's crop is the leading bins (crop_index[j] = j) unless told otherwise,
  // so the fine spectrum is the coarse one padded: no index load on that path
  auto fine = [&](int k) -> C {
    double2 v;
    if (a.crop_identity) {
      v = k < a.n_omega ? lab[k] : make_double2(0.0, 0.0);
    } else {
      const int j = a.fine_to_coarse[k];
      v = j >= 0 ? lab[j] : make_double2(0.0, 0.0);
    }
    if (k == 0 || k == M) v.y = 0.0;
    return to_c<C>(v);
  };
  const R half = R(0.5);
#pragma unroll 4
  for (int k = threadIdx.x; k < M; k += blockDim.x) {
    C xk = fine(k), xm = cconj(fine(M - k));
    C e = cscale(half, cadd(xk, xm));
    // O[k] = (X[k] - conj X[M-k]) W^-k / 2, W^-k = conj(exp(-i pi k / M))
    C w = __ldg(tw + k);  // exp(-2 pi i k / n_to)
    C o = cscale(half, cmul(csub(xk, xm), cconj(w)));
    smem_c[row_slot<C>(k)] = cadd(e, mul_pi(o));  // Z = E + i O
  }
  __syncthreads();
  fft_dif_swizzled</*kInv=*/true>(smem_c, a.log_m, tw, a.log_n_to);
  const R inv_m = R(1.0 / (double)M);
  R* row = a.modal_t + (size_t)col * a.n_to;
  R* absorb = a.absorber_stream ? a.absorber_stream + (size_t)col * a.n_to : nullptr;
#pragma unroll 4
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    C z = smem_c[row_slot<C>(bitrev(m, a.log_m))];
    R x0 = z.x * inv_m, x1 = z.y * inv_m;
    C v;
    v.x = x0;
    v.y = x1;
    reinterpret_cast<C*>(row)[m] = v;
    if (absorb) {
      const C al = reinterpret_cast<const C*>(a.alpha)[m];
      C ab;
      ab.x = -half * al.x * x0;
      ab.y = -half * al.y * x1;
      reinterpret_cast<C*>(absorb)[m] = ab;
    }
  }
}

template <class R>
__global__ void __launch_bounds__(kRowThreads) k_inverse_field(InverseArgsT<R> a) {
  inverse_field_body(a, blockIdx.x);
}

// batched: items[blockIdx.x] = (run, column)
template <class R>
__global__ void __launch_bounds__(kRowThreads) k_inverse_field_b(const InverseArgsT<R>* args, const int2* items,
                                                         const int* flags) {
  const int2 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  inverse_field_body(own_args(args, it.x), it.y);
}

// ----------------------------------------------------------------------------- K4
// 16-byte loads of a row of complex samples: two in FP32, one in FP64
template <class R> struct Load16Of;
template <> struct Load16Of<float> { using type = float4; };
template <> struct Load16Of<double> { using type = double2; };
template <class R> using Load16 = typename Load16Of<R>::type;
__device__ __forceinline__ void split16(const float4& v, float2 (&c)[2]) {
  c[0] = make_float2(v.x, v.y);
  c[1] = make_float2(v.z, v.w);
}
__device__ __forceinline__ void split16(const double2& v, double2 (&c)[1]) { c[0] = v; }

template <class R>
__device__ __forceinline__ void forward_field_body(const ForwardArgsT<R>& a, int row_index) {
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* smem_c = reinterpret_cast<C*>(smem_raw);
  const int row = a.rows[row_index];
  const int M = a.n_to >> 1;
  if (row < a.n_partial_rows) {
    // a projected stream: the node groups' partial projections, summed in group order.
    // 16-byte loads (two complex samples in FP32, one in FP64), eight groups' loads issued
    // before their sums, so that enough bytes are in flight to stream the rows
    constexpr int kPair = 16 / (int)sizeof(C);
    constexpr int kBatch = 8;
    const size_t group_stride = (size_t)a.n_partial_rows * a.n_to / (2 * kPair);  // in 16-byte units
    using V = Load16<R>;
    const V* rows16 = reinterpret_cast<const V*>(a.partials + (size_t)row * a.n_to);
    for (int v = threadIdx.x; v < M / kPair; v += blockDim.x) {
      C acc[kPair];
#pragma unroll
      for (int h = 0; h < kPair; ++h) acc[h].x = acc[h].y = R(0);
      for (int g0 = 0; g0 < a.n_groups; g0 += kBatch) {
        V x[kBatch];
#pragma unroll
        for (int g = 0; g < kBatch; ++g)
          if (g0 + g < a.n_groups) x[g] = __ldg(rows16 + (size_t)(g0 + g) * group_stride + v);
#pragma unroll
        for (int g = 0; g < kBatch; ++g) {
          if (g0 + g >= a.n_groups) break;
          C c[kPair];
          split16(x[g], c);
#pragma unroll
          for (int h = 0; h < kPair; ++h) acc[h] = cadd(acc[h], c[h]);
        }
      }
#pragma unroll
      for (int h = 0; h < kPair; ++h) smem_c[row_slot<C>(kPair * v + h)] = acc[h];  // z = x_even + i x_odd
    }
  } else {
    const double2* x = reinterpret_cast<const double2*>(a.streams + (size_t)row * a.n_to);
#pragma unroll 4
    for (int m = threadIdx.x; m < M; m += blockDim.x) smem_c[row_slot<C>(m)] = to_c<C>(x[m]);
  }
  __syncthreads();
  fft_dif_swizzled</*kInv=*/false>(smem_c, a.log_m, a.twiddles, a.log_n_to);
  C* out = a.spectra + (size_t)row * a.n_omega;
  const R half = R(0.5);
#pragma unroll 4
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x) {
    const int k = a.crop_identity ? j : (int)a.crop_index[j];
    const int km = (k == 0) ? 0 : M - k;
    C zk = smem_c[row_slot<C>(bitrev(k == M ? 0 : k, a.log_m))];
    C zm = cconj(smem_c[row_slot<C>(bitrev(km == M ? 0 : km, a.log_m))]);
    C e = cscale(half, cadd(zk, zm));
    C o = cscale(half, mul_mi(csub(zk, zm)));  // (Z[k] - conj Z[M-k]) / (2 i)
    C w;
    if (k < M) {
      w = __ldg(a.twiddles + k);
    } else {
      w.x = R(-1);
      w.y = R(0);
    }
    out[j] = cadd(e, cmul(w, o));
  }
}

template <class R>
__global__ void __launch_bounds__(kRowThreads) k_forward_field(ForwardArgsT<R> a) {
  forward_field_body(a, blockIdx.x);
}

// batched: items[blockIdx.x] = (run, row index)
template <class R>
__global__ void __launch_bounds__(kRowThreads) k_forward_field_b(const ForwardArgsT<R>* args, const int2* items,
                                                         const int* flags) {
  const int2 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  forward_field_body(own_args(args, it.x), it.y);
}

// ----------------------------------------------------------------------------- K5
__device__ __forceinline__ void stage_output_any(const OutputArgs& a, int block) {
  const int idx = block * blockDim.x + threadIdx.x;
  if (idx < a.n_cols * a.n_omega) a.out[idx] = stage_output_value(a, idx);
}

__global__ void k_stage_output(OutputArgs a) { stage_output_any(a, blockIdx.x); }

// batched: items[blockIdx.x] = (run, block of 256 elements)
__global__ void k_stage_output_b(const OutputArgs* args, const int2* items, const int* flags) {
  const int2 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  stage_output_any(own_args(args, it.x), it.y);
}

// ----------------------------------------------------------------------------- launch
// a block per row: one thread per register group of the transform's passes (M / 16 in FP32,
// M / 8 in FP64), at least 64 and at most kRowThreads
template <class R>
static int threads_for(int m) {
  return std::min(kRowThreads, std::max(64, m >> kRadixBits<cplx<R>>));
}
template <class R>
static size_t row_smem(int m) { return row_length<cplx<R>>(m) * sizeof(cplx<R>); }

template <class R>
cudaError_t launch_inverse(const InverseArgsT<R>& a, int n_cols, cudaStream_t stream) {
  const int C = single_transform_width(a.n_to, sizeof(cplx<R>), false);
  if (C > 1) return launch_inverse_cluster(a, n_cols, C, stream);
  const int M = a.n_to >> 1;
  k_inverse_field<R><<<n_cols, threads_for<R>(M), row_smem<R>(M), stream>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_forward(const ForwardArgsT<R>& a, int n_rows, cudaStream_t stream) {
  const int C = single_transform_width(a.n_to, sizeof(cplx<R>), true);
  if (C > 1) return launch_forward_cluster(a, n_rows, C, stream);
  const int M = a.n_to >> 1;
  k_forward_field<R><<<n_rows, threads_for<R>(M), row_smem<R>(M), stream>>>(a);
  return cudaGetLastError();
}

template cudaError_t launch_inverse<double>(const InverseArgsT<double>&, int, cudaStream_t);
template cudaError_t launch_inverse<float>(const InverseArgsT<float>&, int, cudaStream_t);
template cudaError_t launch_forward<double>(const ForwardArgsT<double>&, int, cudaStream_t);
template cudaError_t launch_forward<float>(const ForwardArgsT<float>&, int, cudaStream_t);

cudaError_t launch_output(const OutputArgs& a, cudaStream_t stream) {
  const int total = a.n_cols * a.n_omega;
  k_stage_output<<<(total + 255) / 256, 256, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t configure_source_kernels() {
  const int max_shm = 200 * 1024;  // rows of up to 128 KB, and room for static shared memory
  cudaError_t e;
  const void* kernels[8] = {(const void*)k_inverse_field<double>, (const void*)k_forward_field<double>,
                            (const void*)k_inverse_field_b<double>, (const void*)k_forward_field_b<double>,
                            (const void*)k_inverse_field<float>, (const void*)k_forward_field<float>,
                            (const void*)k_inverse_field_b<float>, (const void*)k_forward_field_b<float>};
  for (const void* k : kernels) {
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, max_shm);
    if (e != cudaSuccess) return e;
  }
  e = configure_column_kernels();
  if (e != cudaSuccess) return e;
  e = configure_envelope_kernels();
  if (e != cudaSuccess) return e;
  return configure_cluster_fft();
}

}  // namespace sp

namespace sp {

template <class R>
cudaError_t launch_inverse_b(const InverseArgsT<R>* args, const int2* items, const int* flags,
                             int n_items, int n_to, cudaStream_t stream) {
  const int M = n_to >> 1;
  k_inverse_field_b<R><<<n_items, threads_for<R>(M), row_smem<R>(M), stream>>>(args, items, flags);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_forward_b(const ForwardArgsT<R>* args, const int2* items, const int* flags,
                             int n_items, int n_to, cudaStream_t stream) {
  const int M = n_to >> 1;
  k_forward_field_b<R><<<n_items, threads_for<R>(M), row_smem<R>(M), stream>>>(args, items, flags);
  return cudaGetLastError();
}

template cudaError_t launch_inverse_b<double>(const InverseArgsT<double>*, const int2*, const int*, int, int, cudaStream_t);
template cudaError_t launch_inverse_b<float>(const InverseArgsT<float>*, const int2*, const int*, int, int, cudaStream_t);
template cudaError_t launch_forward_b<double>(const ForwardArgsT<double>*, const int2*, const int*, int, int, cudaStream_t);
template cudaError_t launch_forward_b<float>(const ForwardArgsT<float>*, const int2*, const int*, int, int, cudaStream_t);

cudaError_t launch_output_b(const OutputArgs* args, const int2* items, const int* flags,
                            int n_items, cudaStream_t stream) {
  k_stage_output_b<<<n_items, 256, 0, stream>>>(args, items, flags);
  return cudaGetLastError();
}

}  // namespace sp
