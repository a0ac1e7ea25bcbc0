// The Raman response on the field grid, node by node, on the modal transform's products
// route (where the node field lives in HBM): backends/numpy_ref/passes/responses.py:218-334
// (the damped kernel's spectrum, one component or a mixture's) and 395-498 (the delayed
// polarisation):
//
//   H = dt rfft(f_R sum_r u_r(s) exp(-g_r s dt)),  s in [0, 2 n_to)     once per evaluation
//   P_R(t) = eps0 rho_R E(t) irfft(H rfft(D))(t),  D = E^2 on [0, n_to), 0 above
//
// -- the drive of a field grid that keeps the harmonic, the convolution linear on the
// doubled, zero-padded grid.  P_R, gated by the window g, is added to the node's
// polarisation stream after the response column has written the Kerr part there.  Real
// transforms of length 2 n_to run as complex transforms of length n_to (even samples real,
// odd imaginary) with the usual unpacking, over the table exp(-2 pi i m / (2 n_to)),
// m < n_to -- the envelope route's arithmetic (envelope_kernels.cu), in FP64 in both forms.
#include <algorithm>

#include "fft.cuh"
#include "fft_long.cuh"
#include "kernels.cuh"

namespace sp {

namespace {

constexpr double kEps0 = 8.8541878188e-12;  // vacuum permittivity (F/m), CODATA 2022, as solprop.constants
constexpr int kRamanThreads = 1024;

// X[k] = E_k + w^k O_k of a packed real transform of length 2 n (k in [0, n]); Z in
// bit-reversed order, w = exp(-2 pi i k / 2n) = tw[k] (k < n), -1 at k = n
__device__ __forceinline__ double2 unpack(const double2* Z, const double2* tw, int k, int n, int log_n) {
  const int kk = k == n ? 0 : k;
  const int km = k == 0 ? 0 : (n - k == n ? 0 : n - k);
  const double2 zk = Z[bitrev(kk, log_n)];
  const double2 zm = cconj(Z[bitrev(km, log_n)]);
  const double2 e = cscale(0.5, cadd(zk, zm));
  const double2 o = cscale(0.5, mul_mi(csub(zk, zm)));
  const double2 w = k < n ? tw[k] : make_double2(-1.0, 0.0);
  return cadd(e, cmul(w, o));
}

// one CTA per kernel: blockIdx.x 0 the trace (or the scalar kernel), 1 the traceless
__global__ void __launch_bounds__(kRamanThreads) k_raman_kernel(RamanArgs a) {
  extern __shared__ __align__(16) double2 rk_raw[];
  const int n = a.n_to, kernel = blockIdx.x;
  double2* B = rk_raw;
  const StageScalarsDev& st = *a.stage;
  const double* weights = a.tensor_weights;  // (rows, 2), or null for one component
  // one component: f_R sum_r u_r(s) e^(-g_r s dt); a mixture (passes/responses.py:293-334):
  // sum_c rho_c f_c sum_r u_r(s) e^(-g_r s dt), rows in component order
  const bool mixture = a.n_components > 1;
  auto packed = [&](int m) {
    double v[2];
    for (int q = 0; q < 2; ++q) {
      const int s = 2 * m + q;
      const double delay = (double)s * a.dt;
      double total = 0.0;
      for (int c = 0; c < a.n_components; ++c) {
        double k = 0.0;
        for (int r = a.first_row[c]; r < a.first_row[c + 1]; ++r) {
          const double damped = a.undamped[(size_t)r * 2 * n + s] * exp(-st.raman_rates[r] * delay);
          k += weights ? weights[2 * r + kernel] * damped : damped;
        }
        total += mixture ? st.raman_densities[c] * a.fraction[c] * k : a.fraction[c] * k;
      }
      v[q] = total;
    }
    return make_double2(v[0], v[1]);
  };
  double2* spectrum = a.spectrum + (size_t)kernel * (n + 1);
  double largest = 0.0;
  if (n > kMaxEnvelopeRowF64) {
    // a row of 16 384 (the envelope grid's longest): two halves through the scratch, the
    // transform left in natural order there
    double2* gz = a.scratch + (size_t)kernel * (n + n / 2);
    long_forward(packed, B, gz, gz + n, a.twiddles, a.log_n_to - 1);
    for (int k = threadIdx.x; k <= n; k += blockDim.x) {
      const int kk = k == n ? 0 : k, km = k == 0 ? 0 : (n - k == n ? 0 : n - k);
      const double2 zk = gz[kk], zm = cconj(gz[km]);
      const double2 e = cscale(0.5, cadd(zk, zm)), o = cscale(0.5, mul_mi(csub(zk, zm)));
      const double2 w = k < n ? a.twiddles[k] : make_double2(-1.0, 0.0);
      const double2 h = cscale(a.dt, cadd(e, cmul(w, o)));
      spectrum[k] = h;
      largest = fmax(largest, fmax(fabs(h.x), fabs(h.y)));
    }
  } else {
    for (int m = threadIdx.x; m < n; m += blockDim.x) B[m] = packed(m);
    __syncthreads();
    fft_dif_inplace(B, a.log_n_to, a.twiddles, a.log_n_to + 1, /*inverse=*/false);
    for (int k = threadIdx.x; k <= n; k += blockDim.x) {
      const double2 h = cscale(a.dt, unpack(B, a.twiddles, k, n, a.log_n_to));
      spectrum[k] = h;
      largest = fmax(largest, fmax(fabs(h.x), fabs(h.y)));
    }
  }
  if (!a.spectrum32) return;
  // the mixed form's complex64 copy: a molecular gas's spectrum in SI units (about 1e-55)
  // lies below FP32's range, so it is scaled by the power of two that brings its largest
  // bin into [1, 2); the convolution takes the scale back out in FP64
  __shared__ double block_max[kRamanThreads / 32];
  for (int d = 16; d > 0; d >>= 1) largest = fmax(largest, __shfl_xor_sync(0xffffffffu, largest, d));
  if (threadIdx.x % 32 == 0) block_max[threadIdx.x / 32] = largest;
  __syncthreads();
  double all = 0.0;
  for (int w = 0; w < (int)(blockDim.x / 32); ++w) all = fmax(all, block_max[w]);
  const int shift = all > 0.0 ? -ilogb(all) : 0;
  if (threadIdx.x == 0) a.scale[kernel] = shift;
  float2* out = a.spectrum32 + (size_t)kernel * (n + 1);
  __syncthreads();  // every thread's spectrum bins are written
  for (int k = threadIdx.x; k <= n; k += blockDim.x) {
    const double2 h = spectrum[k];
    out[k] = make_float2((float)scalbn(h.x, shift), (float)scalbn(h.y, shift));
  }
}

template <class R>
__global__ void __launch_bounds__(kRamanThreads) k_raman_nodes(RamanArgs a, const R* __restrict__ field,
                                                                R* __restrict__ polarisation) {
  extern __shared__ __align__(16) double2 rn_raw[];
  const int n = a.n_to;
  double2* B = rn_raw;  // the drive's transform, then the convolution's
  double2* C = B + n;   // H D
  __shared__ double2 top;  // bin n
  const int node = blockIdx.x;
  const R* e_row = field + (size_t)node * n;
  // the drive E^2 on [0, n), zero on [n, 2n), packed
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    double v[2] = {0.0, 0.0};
    if (2 * m < n) {
      const double e0 = (double)e_row[2 * m], e1 = (double)e_row[2 * m + 1];
      v[0] = e0 * e0;
      v[1] = e1 * e1;
    }
    B[m] = make_double2(v[0], v[1]);
  }
  __syncthreads();
  fft_dif_inplace(B, a.log_n_to, a.twiddles, a.log_n_to + 1, /*inverse=*/false);
  for (int k = threadIdx.x; k <= n; k += blockDim.x) {
    const double2 y = cmul(a.spectrum[k], unpack(B, a.twiddles, k, n, a.log_n_to));
    if (k < n) C[k] = y;
    else top = y;
  }
  __syncthreads();
  // irfft of length 2n: Z_k = E_k + i O_k, E_k = (Y_k + Y*_{n-k}) / 2,
  // O_k = (Y_k - Y*_{n-k}) conj(w^k) / 2; the imaginary parts of bins 0 and n dropped
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double2 yk = C[k], ym = k == 0 ? top : C[n - k];
    if (k == 0) {
      yk.y = 0.0;
      ym.y = 0.0;
    }
    ym = cconj(ym);
    const double2 e = cscale(0.5, cadd(yk, ym));
    const double2 o = cscale(0.5, cmul(csub(yk, ym), cconj(a.twiddles[k])));
    B[k] = cadd(e, mul_pi(o));
  }
  __syncthreads();
  fft_dif_inplace(B, a.log_n_to, a.twiddles, a.log_n_to + 1, /*inverse=*/true);
  const StageScalarsDev& st = *a.stage;
  const double scale = kEps0 * (a.n_components > 1 ? 1.0 : st.raman_density);  // a mixture's are inside
  const double inv_n = 1.0 / (double)n;
  R* p_row = polarisation + (size_t)node * n;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const double2 z = B[bitrev(t >> 1, a.log_n_to)];
    const double conv = ((t & 1) ? z.y : z.x) * inv_n;  // irfft's 1 / (2n), with the packing's 2
    const double p = scale * (double)e_row[t] * conv;
    p_row[t] = (R)((double)p_row[t] + a.t_window[t] * p);
  }
}

}  // namespace

size_t raman_smem(int n_to) { return (size_t)2 * n_to * sizeof(double2); }

cudaError_t configure_raman_kernels() {
  cudaError_t e = cudaFuncSetAttribute(k_raman_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(kMaxEnvelopeRowF64 * sizeof(double2)));  // one row
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_raman_nodes<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)raman_smem(kMaxRamanSamples));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_raman_nodes<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)raman_smem(kMaxRamanSamples));
}

cudaError_t launch_raman_spectrum(const RamanArgs& a, cudaStream_t s) {
  const size_t row = (size_t)std::min(a.n_to, kMaxEnvelopeRowF64) * sizeof(double2);  // a row, or half a long one
  k_raman_kernel<<<a.tensor_weights ? a.n_kernels : 1, kRamanThreads, row, s>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_raman(const RamanArgs& a, const R* field, R* polarisation, int n_nodes, cudaStream_t s) {
  k_raman_kernel<<<1, kRamanThreads, raman_smem(a.n_to) / 2, s>>>(a);
  k_raman_nodes<R><<<n_nodes, kRamanThreads, raman_smem(a.n_to), s>>>(a, field, polarisation);
  return cudaGetLastError();
}

template cudaError_t launch_raman<double>(const RamanArgs&, const double*, double*, int, cudaStream_t);
template cudaError_t launch_raman<float>(const RamanArgs&, const float*, float*, int, cudaStream_t);

}  // namespace sp
