// The envelope grid's modal route with many modes and nodes, on the modal transform's
// products (the GEMM route): the multimode generalised NLSE of a fibre or capillary on
// complex time samples.  backends/numpy_ref/passes/transforms.py:31-233 (ifft / fft with
// the crop, synthesis and projection), responses.py:65-139 (the analytic Kerr cubic),
// responses.py:218-498 (the Raman response on the doubled grid, drive |E|^2 / 2),
// stepping.py:286-369 (the in-stage absorber):
//
//   k_env_inverse  one CTA per modal column: a(t) = ifft(pad(lab)) into the modal field,
//                  interleaved (re, im) rows of 2 n_to; the absorber's spectrum
//                  FFT[-alpha a / 2], cropped, into its spectra block
//   products       E = tau S a and P_m = sum W P / tau over the interleaved rows
//                  (modal_gemm.cu), N = 2 n_to: FP64 products, or tcgen05 products of
//                  three-part BF16 splits accumulated in FP32 in the mixed form
//   k_env_nodes    one CTA per node: the Kerr cubic, the Raman convolution, the window g
//   k_env_forward  one CTA per modal column: fft of the projected row, cropped
//
// Every transform is the shared-memory radix-4 FFT of fft.cuh over the table
// exp(-2 pi i m / (2 n_to)), m < n_to.  The inverse transform, the modal field and the
// Raman convolution are FP64 in both forms; the Kerr cubic and the forward transform run
// in the form's type R (FP32 in the mixed form).
#include "fft.cuh"
#include "kernels.cuh"

namespace sp {

namespace {

constexpr double kEps0 = 8.8541878188e-12;  // vacuum permittivity (F/m), CODATA 2022, as solprop.constants
constexpr int kEnvThreads = 1024;

// X[k] = E_k + w^k O_k of a packed real transform of length 2 n (k in [0, n]); Z in
// bit-reversed order, w = exp(-2 pi i k / 2n) = tw[k] (k < n), -1 at k = n
template <class C>
__device__ __forceinline__ C unpack_real(const C* Z, const C* tw, int k, int n, int log_n) {
  using R = decltype(C{}.x);
  const int kk = k == n ? 0 : k;
  const int km = k == 0 ? 0 : (n - k == n ? 0 : n - k);
  const C zk = Z[bitrev(kk, log_n)];
  const C zm = cconj(Z[bitrev(km, log_n)]);
  const C e = cscale(R(0.5), cadd(zk, zm));
  const C o = cscale(R(0.5), mul_mi(csub(zk, zm)));
  C w;
  if (k < n) {
    w = tw[k];
  } else {
    w.x = R(-1);
    w.y = R(0);
  }
  return cadd(e, cmul(w, o));
}

template <class R>
__global__ void __launch_bounds__(kEnvThreads) k_env_inverse(EnvModalArgsT<R> a) {
  extern __shared__ __align__(16) double2 ei_raw[];
  const int n = a.n_to, col = blockIdx.x;
  double2* A = ei_raw;
  for (int k = threadIdx.x; k < n; k += blockDim.x) A[k] = make_double2(0.0, 0.0);
  __syncthreads();
  const double2* lab = a.lab + (size_t)col * a.n_omega;
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x) A[a.crop[j]] = lab[j];
  __syncthreads();
  fft_dif_inplace(A, a.log_n_to, a.twiddles, a.log_n_to + 1, /*inverse=*/true);
  const double inv_n = 1.0 / (double)n;  // scipy's ifft carries 1 / n_to
  double2* row = reinterpret_cast<double2*>(a.modal_t + (size_t)col * 2 * n);
  for (int t = threadIdx.x; t < n; t += blockDim.x) row[t] = cscale(inv_n, A[bitrev(t, a.log_n_to)]);
  if (!a.alpha) return;
  // the in-stage absorber -alpha a / 2, transformed and cropped (stage output masks it)
  double2* B = A + n;
  for (int t = threadIdx.x; t < n; t += blockDim.x)
    B[t] = cscale(-0.5 * a.alpha[t], cscale(inv_n, A[bitrev(t, a.log_n_to)]));
  __syncthreads();
  fft_dif_inplace(B, a.log_n_to, a.twiddles, a.log_n_to + 1, /*inverse=*/false);
  cplx<R>* absorber = a.spectra + (size_t)3 * a.n_cols * a.n_omega + (size_t)col * a.n_omega;
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x)
    absorber[j] = to_c<cplx<R>>(B[bitrev((int)a.crop[j], a.log_n_to)]);
}

// The Raman convolution runs in FP64 in both forms: a molecular gas's kernel spectrum in SI
// units (about 1e-55 at a femtosecond spacing) lies below FP32's range.  With two field
// components (rows x, y of the node) the Kerr cubic sums over them and the Raman response
// is the tensor one (passes/responses.py:501-550): the trace drive |a_x|^2/2 + |a_y|^2/2 and,
// with a traceless kernel, the difference and coherence drives, three convolutions u, v, w
// whose symmetric matrix [[u + v, w], [w, u - v]] multiplies the field.
template <class R>
__global__ void __launch_bounds__(kEnvThreads) k_env_nodes(EnvModalArgsT<R> a) {
  using C = cplx<R>;
  extern __shared__ __align__(16) double2 en_raw[];
  const int n = a.n_to, node = blockIdx.x, nc = a.n_components;
  double2* B = en_raw;  // a drive's transform, then its convolution's
  double2* H = B + n;   // H D
  double* U = reinterpret_cast<double*>(H + n);  // three drives: the trace and difference convolutions
  double* V = U + n;
  __shared__ double2 top;  // bin n
  const StageScalarsDev& st = *a.stage;
  const C* Ex = reinterpret_cast<const C*>(a.node_field) + (size_t)node * nc * n;
  const C* Ey = Ex + (nc == 2 ? n : 0);
  const bool raman = a.raman_spectrum != nullptr;
  const int drives = !raman ? 0 : (nc == 2 && a.raman_kernels == 2 ? 3 : 1);
  for (int dr = 0; dr < drives; ++dr) {
    // the drive on [0, n), zero on [n, 2n), packed
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
      double v[2] = {0.0, 0.0};
      if (2 * m < n) {
        for (int q = 0; q < 2; ++q) {
          const double2 x = to_d2(Ex[2 * m + q]);
          const double xx = 0.5 * (x.x * x.x + x.y * x.y);
          if (nc == 1) {
            v[q] = xx;
          } else {
            const double2 y = to_d2(Ey[2 * m + q]);
            const double yy = 0.5 * (y.x * y.x + y.y * y.y);
            v[q] = dr == 0 ? xx + yy : dr == 1 ? xx - yy : 2.0 * 0.5 * (x.x * y.x + x.y * y.y);
          }
        }
      }
      B[m] = make_double2(v[0], v[1]);
    }
    __syncthreads();
    fft_dif_inplace(B, a.log_n_to, a.twiddles, a.log_n_to + 1, /*inverse=*/false);
    const double2* kernel = a.raman_spectrum + (dr == 0 ? 0 : (size_t)(n + 1));  // trace, then traceless
    for (int k = threadIdx.x; k <= n; k += blockDim.x) {
      const double2 y = cmul(kernel[k], unpack_real(B, a.twiddles, k, n, a.log_n_to));
      if (k < n) H[k] = y;
      else top = y;
    }
    __syncthreads();
    // irfft of length 2n: Z_k = E_k + i O_k, E_k = (Y_k + Y*_{n-k}) / 2,
    // O_k = (Y_k - Y*_{n-k}) conj(w^k) / 2; the imaginary parts of bins 0 and n dropped
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      double2 yk = H[k], ym = k == 0 ? top : H[n - k];
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
    if (dr + 1 < drives) {  // keep u and v in natural order; the last one stays in B
      double* keep = dr == 0 ? U : V;
      const double inv = 1.0 / (double)n;
      for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const double2 z = B[bitrev(t >> 1, a.log_n_to)];
        keep[t] = ((t & 1) ? z.y : z.x) * inv;
      }
      __syncthreads();
    }
  }
  // the Kerr coefficient times the density (about 1e-37 in SI units for a gas) is applied in
  // FP64 to the cubic formed in R, so that it never rounds to an FP32 subnormal
  const double factor = a.kerr ? a.kerr_coefficient * st.kerr_density : 0.0;
  const R self = R(a.kerr_self), conj = R(a.kerr_conjugate);
  const double raman_scale = kEps0 * (a.raman_mixture ? 1.0 : st.raman_density);  // a mixture's are inside
  const double inv_n = 1.0 / (double)n;
  C* Px = reinterpret_cast<C*>(a.node_streams) + (size_t)node * nc * n;
  C* Py = Px + (nc == 2 ? n : 0);
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const C x = Ex[t], y = Ey[t];
    double2 px = make_double2(0.0, 0.0), py = px;
    if (a.kerr) {  // c rho (s (sum |a|^2) a_p + q (sum a^2) a_p*), summed over the components
      R mod = x.x * x.x + x.y * x.y;
      C sq = cmul(x, x);
      if (nc == 2) {
        mod += y.x * y.x + y.y * y.y;
        sq = cadd(sq, cmul(y, y));
      }
      const C cx = cadd(cscale(self * mod, x), cscale(conj, cmul(sq, cconj(x))));
      px = make_double2(factor * (double)cx.x, factor * (double)cx.y);
      if (nc == 2) {
        const C cy = cadd(cscale(self * mod, y), cscale(conj, cmul(sq, cconj(y))));
        py = make_double2(factor * (double)cy.x, factor * (double)cy.y);
      }
    }
    if (drives > 0) {
      const double2 z = B[bitrev(t >> 1, a.log_n_to)];
      const double last = ((t & 1) ? z.y : z.x) * inv_n;  // irfft's 1 / (2n), with the packing's 2
      const double2 dx = to_d2(x), dy = to_d2(y);
      if (drives == 1) {
        px = cadd(px, cscale(raman_scale * last, dx));
        if (nc == 2) py = cadd(py, cscale(raman_scale * last, dy));
      } else {
        const double u = U[t], v = V[t], w = last;
        px = cadd(px, cscale(raman_scale, cadd(cscale(u + v, dx), cscale(w, dy))));
        py = cadd(py, cscale(raman_scale, cadd(cscale(w, dx), cscale(u - v, dy))));
      }
    }
    const double g = a.t_window[t];
    Px[t] = to_c<C>(cscale(g, px));
    if (nc == 2) Py[t] = to_c<C>(cscale(g, py));
  }
}

template <class R>
__global__ void __launch_bounds__(kEnvThreads) k_env_forward(EnvModalArgsT<R> a) {
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char ef_raw[];
  const int n = a.n_to, col = blockIdx.x;
  C* A = reinterpret_cast<C*>(ef_raw);
  const C* row = reinterpret_cast<const C*>(a.projected) + (size_t)col * n;
  for (int t = threadIdx.x; t < n; t += blockDim.x) A[t] = row[t];
  __syncthreads();
  fft_dif_inplace(A, a.log_n_to, a.twiddles_r, a.log_n_to + 1, /*inverse=*/false);
  C* spectra = a.spectra + (size_t)col * a.n_omega;
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x) spectra[j] = A[bitrev((int)a.crop[j], a.log_n_to)];
}

}  // namespace

cudaError_t configure_env_modal_kernels() {
  const int two = (int)(2 * kMaxEnvelopeSamples * sizeof(double2)), one = two / 2;
  const void* kernels[6] = {(const void*)k_env_inverse<double>, (const void*)k_env_inverse<float>,
                            (const void*)k_env_nodes<double>,   (const void*)k_env_nodes<float>,
                            (const void*)k_env_forward<double>, (const void*)k_env_forward<float>};
  const int nodes = (int)(kMaxEnvelopeSamples * (2 * sizeof(double2) + 2 * sizeof(double)));
  const int shm[6] = {two, two, nodes, nodes, one, one / 2};
  for (int i = 0; i < 6; ++i) {
    cudaError_t e = cudaFuncSetAttribute(kernels[i], cudaFuncAttributeMaxDynamicSharedMemorySize, shm[i]);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <class R>
cudaError_t launch_env_inverse(const EnvModalArgsT<R>& a, cudaStream_t s) {
  const size_t row = (size_t)a.n_to * sizeof(double2);
  k_env_inverse<R><<<a.n_cols, kEnvThreads, a.alpha ? 2 * row : row, s>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_env_nodes(const EnvModalArgsT<R>& a, int n_nodes, cudaStream_t s) {
  const bool three = a.n_components == 2 && a.raman_kernels == 2 && a.raman_spectrum;  // u, v kept
  const size_t bytes = (size_t)a.n_to * (2 * sizeof(double2) + (three ? 2 * sizeof(double) : 0));
  k_env_nodes<R><<<n_nodes, kEnvThreads, bytes, s>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_env_forward(const EnvModalArgsT<R>& a, cudaStream_t s) {
  k_env_forward<R><<<a.n_cols, kEnvThreads, (size_t)a.n_to * sizeof(cplx<R>), s>>>(a);
  return cudaGetLastError();
}

template cudaError_t launch_env_inverse<double>(const EnvModalArgsT<double>&, cudaStream_t);
template cudaError_t launch_env_inverse<float>(const EnvModalArgsT<float>&, cudaStream_t);
template cudaError_t launch_env_nodes<double>(const EnvModalArgsT<double>&, int, cudaStream_t);
template cudaError_t launch_env_nodes<float>(const EnvModalArgsT<float>&, int, cudaStream_t);
template cudaError_t launch_env_forward<double>(const EnvModalArgsT<double>&, cudaStream_t);
template cudaError_t launch_env_forward<float>(const EnvModalArgsT<float>&, cudaStream_t);

}  // namespace sp
