// The kernels of one source evaluation on the modal route (field grid): solprop's
// passes 2-7 (docs/dev/architecture.md section 8), restated for sm_100a.
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
#include "fft.cuh"
#include "kernels.cuh"

namespace sp {

// ----------------------------------------------------------------------------- K1
__device__ __forceinline__ void inverse_field_body(const InverseArgs& a, int col) {
  extern __shared__ double2 smem_c[];
  const int M = a.n_to >> 1;  // complex length
  const double2* lab = a.lab + (size_t)col * a.n_omega;
  const double2* tw = a.twiddles;
  // X[k] for k in [0, M]; pocketfft's irfft reads only the real part of the DC and
  // Nyquist bins, so those are taken real here too.
  // the field grid's crop is the leading bins (crop_index[j] = j) unless told otherwise,
  // so the fine spectrum is the coarse one padded: no index load on that path
  auto fine = [&](int k) -> double2 {
    double2 v;
    if (a.crop_identity) {
      v = k < a.n_omega ? lab[k] : make_double2(0.0, 0.0);
    } else {
      const int j = a.fine_to_coarse[k];
      v = j >= 0 ? lab[j] : make_double2(0.0, 0.0);
    }
    if (k == 0 || k == M) v.y = 0.0;
    return v;
  };
#pragma unroll 4
  for (int k = threadIdx.x; k < M; k += blockDim.x) {
    double2 xk = fine(k), xm = cconj(fine(M - k));
    double2 e = cscale(0.5, cadd(xk, xm));
    // O[k] = (X[k] - conj X[M-k]) W^-k / 2, W^-k = conj(exp(-i pi k / M))
    double2 w = __ldg(tw + k);  // exp(-2 pi i k / n_to)
    double2 o = cscale(0.5, cmul(csub(xk, xm), cconj(w)));
    smem_c[k] = cadd(e, mul_pi(o));  // Z = E + i O
  }
  __syncthreads();
  fft_dif_inplace(smem_c, a.log_m, tw, a.log_n_to, /*inverse=*/true);
  const double inv_m = 1.0 / (double)M;
  double* row = a.modal_t + (size_t)col * a.n_to;
  double* absorb = a.absorber_stream ? a.absorber_stream + (size_t)col * a.n_to : nullptr;
#pragma unroll 4
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    double2 z = smem_c[bitrev(m, a.log_m)];
    double x0 = z.x * inv_m, x1 = z.y * inv_m;
    reinterpret_cast<double2*>(row)[m] = make_double2(x0, x1);
    if (absorb) {
      const double2 al = reinterpret_cast<const double2*>(a.alpha)[m];
      reinterpret_cast<double2*>(absorb)[m] =
          make_double2(-0.5 * al.x * x0, -0.5 * al.y * x1);
    }
  }
}

__global__ void __launch_bounds__(1024) k_inverse_field(InverseArgs a) {
  inverse_field_body(a, blockIdx.x);
}

// batched: items[blockIdx.x] = (run, column)
__global__ void __launch_bounds__(1024) k_inverse_field_b(const InverseArgs* args, const int2* items,
                                                         const int* flags) {
  const int2 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  inverse_field_body(args[it.x], it.y);
}

// ----------------------------------------------------------------------------- K4
__device__ __forceinline__ void forward_field_body(const ForwardArgs& a, int row_index) {
  extern __shared__ double2 smem_c[];
  const int row = a.rows[row_index];
  const int M = a.n_to >> 1;
  if (row < a.n_partial_rows) {
    // a projected stream: the node groups' partial projections, summed in group order
#pragma unroll 4
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
      double2 acc = make_double2(0.0, 0.0);
      for (int g = 0; g < a.n_groups; ++g) {
        const double2 v = reinterpret_cast<const double2*>(
            a.partials + ((size_t)g * a.n_partial_rows + row) * a.n_to)[m];
        acc = cadd(acc, v);
      }
      smem_c[m] = acc;  // z = x_even + i x_odd
    }
  } else {
    const double2* x = reinterpret_cast<const double2*>(a.streams + (size_t)row * a.n_to);
#pragma unroll 4
    for (int m = threadIdx.x; m < M; m += blockDim.x) smem_c[m] = x[m];
  }
  __syncthreads();
  fft_dif_inplace(smem_c, a.log_m, a.twiddles, a.log_n_to, /*inverse=*/false);
  double2* out = a.spectra + (size_t)row * a.n_omega;
#pragma unroll 4
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x) {
    const int k = a.crop_identity ? j : (int)a.crop_index[j];
    const int km = (k == 0) ? 0 : M - k;
    double2 zk = smem_c[bitrev(k == M ? 0 : k, a.log_m)];
    double2 zm = cconj(smem_c[bitrev(km == M ? 0 : km, a.log_m)]);
    double2 e = cscale(0.5, cadd(zk, zm));
    double2 o = cscale(0.5, mul_mi(csub(zk, zm)));  // (Z[k] - conj Z[M-k]) / (2 i)
    double2 w = k < M ? __ldg(a.twiddles + k) : make_double2(-1.0, 0.0);
    out[j] = cadd(e, cmul(w, o));
  }
}

__global__ void __launch_bounds__(1024) k_forward_field(ForwardArgs a) {
  forward_field_body(a, blockIdx.x);
}

// batched: items[blockIdx.x] = (run, row index)
__global__ void __launch_bounds__(1024) k_forward_field_b(const ForwardArgs* args, const int2* items,
                                                         const int* flags) {
  const int2 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  forward_field_body(args[it.x], it.y);
}

// ----------------------------------------------------------------------------- K5
__device__ __forceinline__ void stage_output_body(const OutputArgs& a, int block) {
  const int idx = block * blockDim.x + threadIdx.x;
  const int total = a.n_cols * a.n_omega;
  if (idx >= total) return;
  const int j = idx % a.n_omega;
  const StageScalarsDev& st = *a.stage;
  // prefactor = combine(weights, terms)    (translate/stage.py:292-342)
  double2 pre;
  if (st.n_pre == 1) {
    pre = a.prefactor_terms[idx];
    if (st.pre_w[0] != 1.0) pre = cscale(st.pre_w[0], pre);
  } else {
    pre = make_double2(0.0, 0.0);
    for (int p = 0; p < st.n_pre; ++p)
      pre = cadd(pre, cscale(st.pre_w[p], a.prefactor_terms[(size_t)p * total + idx]));
  }
  double2 spec = a.spectra[idx];  // stream 0: P
  const bool active = a.active_mask[j];
  if (a.plasma && active) {
    const double2 xs = a.spectra[(size_t)1 * total + idx];
    const double2 zs = a.spectra[(size_t)2 * total + idx];
    const double2 qv = make_double2(0.0, a.omega[j]);
    const double2 q2 = cmul(qv, qv);
    spec = cadd(spec, csub(cdiv(xs, qv), cdiv(zs, q2)));
  }
  double2 normalised = cmul(cscale(a.omega_window[j], pre), spec);
  if (a.absorber) {
    double2 ab = active ? a.spectra[(size_t)3 * total + idx] : make_double2(0.0, 0.0);
    normalised = cadd(normalised, ab);
  }
  if (a.inverse_propagator) normalised = cmul(a.inverse_propagator[idx], normalised);
  a.out[idx] = normalised;
}

__global__ void k_stage_output(OutputArgs a) { stage_output_body(a, blockIdx.x); }

// batched: items[blockIdx.x] = (run, block of 256 elements)
__global__ void k_stage_output_b(const OutputArgs* args, const int2* items, const int* flags) {
  const int2 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  stage_output_body(args[it.x], it.y);
}

// ----------------------------------------------------------------------------- launch
static int threads_for(int m) { return m >= 1024 ? 1024 : (m >= 32 ? m : 32); }

cudaError_t launch_inverse(const InverseArgs& a, int n_cols, cudaStream_t stream) {
  if (fft_cluster_size(a.n_to) > 1) return launch_inverse_cluster(a, n_cols, stream);
  const int M = a.n_to >> 1;
  const size_t shm = (size_t)M * sizeof(double2);
  k_inverse_field<<<n_cols, threads_for(M), shm, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_forward(const ForwardArgs& a, int n_rows, cudaStream_t stream) {
  if (fft_cluster_size(a.n_to) > 1) return launch_forward_cluster(a, n_rows, stream);
  const int M = a.n_to >> 1;
  const size_t shm = (size_t)M * sizeof(double2);
  k_forward_field<<<n_rows, threads_for(M), shm, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_output(const OutputArgs& a, cudaStream_t stream) {
  const int total = a.n_cols * a.n_omega;
  k_stage_output<<<(total + 255) / 256, 256, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t configure_source_kernels() {
  const int max_shm = 227 * 1024;
  cudaError_t e;
  e = cudaFuncSetAttribute(k_inverse_field, cudaFuncAttributeMaxDynamicSharedMemorySize, max_shm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_forward_field, cudaFuncAttributeMaxDynamicSharedMemorySize, max_shm);
  if (e != cudaSuccess) return e;
  e = configure_column_kernels();
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_inverse_field_b, cudaFuncAttributeMaxDynamicSharedMemorySize, max_shm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_forward_field_b, cudaFuncAttributeMaxDynamicSharedMemorySize, max_shm);
  if (e != cudaSuccess) return e;
  return configure_cluster_fft();
}

}  // namespace sp

namespace sp {

cudaError_t launch_inverse_b(const InverseArgs* args, const int2* items, const int* flags,
                             int n_items, int n_to, cudaStream_t stream) {
  const int M = n_to >> 1;
  k_inverse_field_b<<<n_items, threads_for(M), (size_t)M * sizeof(double2), stream>>>(args, items, flags);
  return cudaGetLastError();
}

cudaError_t launch_forward_b(const ForwardArgs* args, const int2* items, const int* flags,
                             int n_items, int n_to, cudaStream_t stream) {
  const int M = n_to >> 1;
  k_forward_field_b<<<n_items, threads_for(M), (size_t)M * sizeof(double2), stream>>>(args, items, flags);
  return cudaGetLastError();
}

cudaError_t launch_output_b(const OutputArgs* args, const int2* items, const int* flags,
                            int n_items, cudaStream_t stream) {
  k_stage_output_b<<<n_items, 256, 0, stream>>>(args, items, flags);
  return cudaGetLastError();
}

}  // namespace sp
