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
// exp(-2 pi i m / (2 n_to)), m < n_to.  The inverse transform and the modal field are FP64
// in both forms; the Kerr cubic, the Raman convolutions and the forward transform run in the
// form's type R (FP32 in the mixed form).
#include "fft.cuh"
#include "fft_long.cuh"
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
  // the in-stage absorber -alpha a / 2, transformed and cropped (stage output masks it); the
  // row of shared memory is reused, a(t) read back from the modal field just written
  __syncthreads();
  double2* B = A;
  for (int t = threadIdx.x; t < n; t += blockDim.x) B[t] = cscale(-0.5 * a.alpha[t], row[t]);
  __syncthreads();
  fft_dif_inplace(B, a.log_n_to, a.twiddles, a.log_n_to + 1, /*inverse=*/false);
  cplx<R>* absorber = a.spectra + (size_t)3 * a.n_cols * a.n_omega + (size_t)col * a.n_omega;
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x)
    absorber[j] = to_c<cplx<R>>(B[bitrev((int)a.crop[j], a.log_n_to)]);
}

constexpr int kNodeThreads = 512;  // one radix-8 butterfly per thread at 4 096 samples
constexpr int kMaxPairs = kMaxEnvelopeProducts / 2 / kNodeThreads + 1;

// Y = H X on the packed spectrum of a real drive of length 2n, and the packing of the
// inverse real transform, in place over the swizzled row: Z[j] (j < n, bit-reversed slots)
// holds the forward transform of d(2m) + i d(2m + 1).  Pair (k, n - k) needs Z[k] and
// Z[n - k] alone and gives Z'[k] and Z'[n - k] (k = 0 also makes bin n), so every thread
// reads its pairs, the block meets, and the thread writes them back in natural order:
//   X[k] = E_k + w^k O_k,  E_k = (Z[k] + Z*[n-k]) / 2,  O_k = -i (Z[k] - Z*[n-k]) / 2
//   Z'[k] = E'_k + i O'_k, E'_k = (Y[k] + Y*[n-k]) / 2, O'_k = (Y[k] - Y*[n-k]) conj(w^k) / 2
// with w = exp(-2 pi i / 2n) and the imaginary parts of Y[0] and Y[n] dropped.
// The Raman convolution's arithmetic: FP64 in the FP64 form; FP32 in the mixed form, on the
// kernel spectrum scaled by 2^scale (a molecular gas's SI spectrum, about 1e-55, lies below
// FP32's range; the scale is taken back out in FP64)
template <class R>
__device__ __forceinline__ const cplx<R>* spectrum_table(const EnvModalArgsT<R>& a) {
  if constexpr (sizeof(R) == 8) return a.twiddles;
  else return a.twiddles_r;
}
template <class R>
__device__ __forceinline__ const cplx<R>* kernel_spectrum(const EnvModalArgsT<R>& a, int kernel) {
  if constexpr (sizeof(R) == 8) return a.raman_spectrum + (size_t)kernel * (a.n_to + 1);
  else return a.raman_spectrum32 + (size_t)kernel * (a.n_to + 1);
}
template <class R>
__device__ __forceinline__ double spectrum_unscale(const EnvModalArgsT<R>& a, int kernel, double v) {
  if constexpr (sizeof(R) == 8) return v;
  else return scalbn(v, -a.raman_scale[kernel]);
}

template <class C>
__device__ __forceinline__ void spectrum_product(C* B, const C* __restrict__ H, const C* __restrict__ tw, int n,
                                                 int log_n) {
  using T = decltype(C{}.x);
  C za[kMaxPairs], zb[kMaxPairs];
  int count = 0;
  const T half = T(0.5);
  for (int k = threadIdx.x; k <= n / 2; k += blockDim.x, ++count) {
    const int km = k == 0 ? 0 : n - k;
    const C a = B[row_slot<C>(bitrev(k, log_n))];
    const C b = B[row_slot<C>(bitrev(km, log_n))];
    if (k == 0) {
      // X[0] = Re Z0 + Im Z0, X[n] = Re Z0 - Im Z0 (both real); Y's imaginary parts dropped;
      // Z'[0] = (Y0 + Yn) / 2 + i (Y0 - Yn) / 2
      C x0, xn;
      x0.x = a.x + a.y;
      x0.y = T(0);
      xn.x = a.x - a.y;
      xn.y = T(0);
      const T y0 = cmul(H[0], x0).x, yn = cmul(H[n], xn).x;
      za[count].x = half * (y0 + yn);
      za[count].y = half * (y0 - yn);
      zb[count] = za[count];
      continue;
    }
    const C e = cscale(half, cadd(a, cconj(b)));
    const C o = cscale(half, mul_mi(csub(a, cconj(b))));
    const C wk = tw[k], wm = tw[km];
    const C xk = cadd(e, cmul(wk, o));
    // X[n - k]: E_{n-k} = conj(E_k), O_{n-k} = -i (Z[n-k] - Z*[k]) / 2
    const C om = cscale(half, mul_mi(csub(b, cconj(a))));
    const C xm = cadd(cconj(e), cmul(wm, om));
    const C yk = cmul(H[k], xk), ym = cmul(H[km], xm);
    za[count] = cadd(cscale(half, cadd(yk, cconj(ym))), mul_pi(cscale(half, cmul(csub(yk, cconj(ym)), cconj(wk)))));
    zb[count] = cadd(cscale(half, cadd(ym, cconj(yk))), mul_pi(cscale(half, cmul(csub(ym, cconj(yk)), cconj(wm)))));
  }
  __syncthreads();
  count = 0;
  for (int k = threadIdx.x; k <= n / 2; k += blockDim.x, ++count) {
    B[row_slot<C>(k)] = za[count];
    if (k != 0 && k != n / 2) B[row_slot<C>(n - k)] = zb[count];
  }
  __syncthreads();
}

// One sample t of a node's gated polarisation: with drive 0 the Kerr cubic and the first
// convolution conv (already times eps0 rho) times the field; the later drives add
// conv [[1, 0], [0, -1]] (the difference) or conv [[0, 1], [1, 0]] (the coherence) times it.
template <class R>
__device__ __forceinline__ void node_sample(const EnvModalArgsT<R>& a, const cplx<R>* Ex, const cplx<R>* Ey,
                                            cplx<R>* Px, cplx<R>* Py, int t, double conv, int dr, int nc,
                                            double factor, R self, R conj) {
  using C = cplx<R>;
  const C x = Ex[t], y = Ey[t];
  const double g = a.t_window[t];
  const double2 dx = to_d2(x), dy = to_d2(y);
  if (dr == 0) {  // the Kerr cubic and the first convolution
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
    px = cadd(px, cscale(conv, dx));
    Px[t] = to_c<C>(cscale(g, px));
    if (nc == 2) {
      py = cadd(py, cscale(conv, dy));
      Py[t] = to_c<C>(cscale(g, py));
    }
  } else if (dr == 1) {  // + v [[1, 0], [0, -1]]
    Px[t] = to_c<C>(cadd(to_d2(Px[t]), cscale(g * conv, dx)));
    Py[t] = to_c<C>(csub(to_d2(Py[t]), cscale(g * conv, dy)));
  } else {  // + w [[0, 1], [1, 0]]
    Px[t] = to_c<C>(cadd(to_d2(Px[t]), cscale(g * conv, dy)));
    Py[t] = to_c<C>(cadd(to_d2(Py[t]), cscale(g * conv, dx)));
  }
}

// The nodes' responses, one CTA per node.  The Raman convolutions run in the form's type
// (the mixed form's on a scaled spectrum, above).  With two field components (rows x, y of the node) the
// Kerr cubic sums over them and the Raman response is the tensor one
// (passes/responses.py:501-550): the trace drive |a_x|^2/2 + |a_y|^2/2 and, with a
// traceless kernel, the difference and coherence drives, three convolutions u, v, w whose
// symmetric matrix [[u + v, w], [w, u - v]] multiplies the field.  Each convolution is
// added to the node's stream as it is formed (the first with the Kerr cubic), so the row
// of shared memory is the transform's alone.
template <class R>
__global__ void __launch_bounds__(kNodeThreads, 2) k_env_nodes(EnvModalArgsT<R> a) {
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char en_raw[];
  const int n = a.n_to, node = blockIdx.x, nc = a.n_components;
  C* B = reinterpret_cast<C*>(en_raw);  // a drive's transform, then its convolution's (swizzled slots)
  const StageScalarsDev& st = *a.stage;
  const C* Ex = reinterpret_cast<const C*>(a.node_field) + (size_t)node * nc * n;
  const C* Ey = Ex + (nc == 2 ? n : 0);
  C* Px = reinterpret_cast<C*>(a.node_streams) + (size_t)node * nc * n;
  C* Py = Px + (nc == 2 ? n : 0);
  const bool raman = a.raman_spectrum != nullptr;
  const int drives = !raman ? 0 : (nc == 2 && a.raman_kernels == 2 ? 3 : 1);
  // the Kerr coefficient times the density (about 1e-37 in SI units for a gas) is applied in
  // FP64 to the cubic formed in R, so that it never rounds to an FP32 subnormal
  const double factor = a.kerr ? a.kerr_coefficient * st.kerr_density : 0.0;
  const R self = R(a.kerr_self), conj = R(a.kerr_conjugate);
  const double raman_scale = kEps0 * (a.raman_mixture ? 1.0 : st.raman_density);  // a mixture's are inside
  const double inv_n = 1.0 / (double)n;
  for (int dr = 0; dr < (drives > 0 ? drives : 1); ++dr) {
    if (drives > 0) {
      // the drive on [0, n), zero on [n, 2n), packed: B[m] = d(2m) + i d(2m + 1)
      for (int m = threadIdx.x; m < n; m += blockDim.x) {
        R v[2] = {R(0), R(0)};
        if (2 * m < n) {
          for (int q = 0; q < 2; ++q) {
            const C x = Ex[2 * m + q];
            const R xx = R(0.5) * (x.x * x.x + x.y * x.y);
            if (nc == 1) {
              v[q] = xx;
            } else {
              const C y = Ey[2 * m + q];
              const R yy = R(0.5) * (y.x * y.x + y.y * y.y);
              v[q] = dr == 0 ? xx + yy : dr == 1 ? xx - yy : R(2) * R(0.5) * (x.x * y.x + x.y * y.y);
            }
          }
        }
        C packed;
        packed.x = v[0];
        packed.y = v[1];
        B[row_slot<C>(m)] = packed;
      }
      __syncthreads();
      const C* table = spectrum_table<R>(a);
      fft_dif_swizzled<false>(B, a.log_n_to, table, a.log_n_to + 1);
      spectrum_product(B, kernel_spectrum<R>(a, dr == 0 ? 0 : 1), table, n, a.log_n_to);  // trace, then traceless
      fft_dif_swizzled<true>(B, a.log_n_to, table, a.log_n_to + 1);
    }
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      double conv = 0.0;
      if (drives > 0) {
        const C z = B[row_slot<C>(bitrev(t >> 1, a.log_n_to))];
        // irfft's 1 / (2n), with the packing's 2; the mixed form's spectrum scale taken out
        conv = raman_scale * spectrum_unscale<R>(a, dr == 0 ? 0 : 1, (double)((t & 1) ? z.y : z.x) * inv_n);
      }
      node_sample<R>(a, Ex, Ey, Px, Py, t, conv, dr, nc, factor, self, conj);
    }
    __syncthreads();  // the next drive's packing overwrites the row
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

// ---- FP64 rows of 16 384 samples: the halves of fft_long.cuh over each row's scratch
// (1.5 n_to complex: the n_to-point spectrum, then the even half's transform)

__global__ void __launch_bounds__(kEnvThreads) k_env_inverse_long(EnvModalArgsT<double> a) {
  extern __shared__ __align__(16) double2 el_raw[];
  const int n = a.n_to, h = n / 2, log_h = a.log_n_to - 1, col = blockIdx.x;
  double2* S = el_raw;
  double2* gz = a.scratch + (size_t)col * (n + h);
  double2* ge = gz + n;
  for (int k = threadIdx.x; k < n; k += blockDim.x) gz[k] = make_double2(0.0, 0.0);
  __syncthreads();
  const double2* lab = a.lab + (size_t)col * a.n_omega;
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x) gz[a.crop[j]] = lab[j];
  __syncthreads();
  const double inv_n = 1.0 / (double)n;  // scipy's ifft carries 1 / n_to
  double2* row = reinterpret_cast<double2*>(a.modal_t + (size_t)col * 2 * n);
  for (int half = 0; half < 2; ++half) {
    long_inverse_half(gz, S, a.twiddles, log_h, half);
    for (int i = threadIdx.x; i < h; i += blockDim.x)
      row[2 * i + half] = cscale(inv_n, S[row_slot<double2>(bitrev(i, log_h))]);
    __syncthreads();
  }
  if (!a.alpha) return;
  long_forward([&](int m) { return cscale(-0.5 * a.alpha[m], row[m]); }, S, gz, ge, a.twiddles, log_h);
  double2* absorber = a.spectra + (size_t)3 * a.n_cols * a.n_omega + (size_t)col * a.n_omega;
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x) absorber[j] = gz[a.crop[j]];
}

// the mixed form's inverse: the same FP64 transform, the absorber's spectrum in complex64
__global__ void __launch_bounds__(kEnvThreads) k_env_inverse_long32(EnvModalArgsT<float> a) {
  extern __shared__ __align__(16) double2 em_raw[];
  const int n = a.n_to, h = n / 2, log_h = a.log_n_to - 1, col = blockIdx.x;
  double2* S = em_raw;
  double2* gz = a.scratch + (size_t)col * (n + h);
  double2* ge = gz + n;
  for (int k = threadIdx.x; k < n; k += blockDim.x) gz[k] = make_double2(0.0, 0.0);
  __syncthreads();
  const double2* lab = a.lab + (size_t)col * a.n_omega;
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x) gz[a.crop[j]] = lab[j];
  __syncthreads();
  const double inv_n = 1.0 / (double)n;
  double2* row = reinterpret_cast<double2*>(a.modal_t + (size_t)col * 2 * n);
  for (int half = 0; half < 2; ++half) {
    long_inverse_half(gz, S, a.twiddles, log_h, half);
    for (int i = threadIdx.x; i < h; i += blockDim.x)
      row[2 * i + half] = cscale(inv_n, S[row_slot<double2>(bitrev(i, log_h))]);
    __syncthreads();
  }
  if (!a.alpha) return;
  long_forward([&](int m) { return cscale(-0.5 * a.alpha[m], row[m]); }, S, gz, ge, a.twiddles, log_h);
  float2* absorber = a.spectra + (size_t)3 * a.n_cols * a.n_omega + (size_t)col * a.n_omega;
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x) absorber[j] = to_c<float2>(gz[a.crop[j]]);
}

__global__ void __launch_bounds__(kEnvThreads) k_env_forward_long(EnvModalArgsT<double> a) {
  extern __shared__ __align__(16) double2 ef_long_raw[];
  const int n = a.n_to, h = n / 2, log_h = a.log_n_to - 1, col = blockIdx.x;
  double2* gz = a.scratch + (size_t)col * (n + h);
  const double2* row = reinterpret_cast<const double2*>(a.projected) + (size_t)col * n;
  long_forward([&](int m) { return row[m]; }, ef_long_raw, gz, gz + n, a.twiddles, log_h);
  double2* spectra = a.spectra + (size_t)col * a.n_omega;
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x) spectra[j] = gz[a.crop[j]];
}

// The spectrum product of spectrum_product over a natural-order row in global memory: the
// thread of pair (k, n - k) reads and writes those two bins alone.
__device__ __forceinline__ void spectrum_product_global(double2* Z, const double2* __restrict__ H,
                                                        const double2* __restrict__ tw, int n) {
  for (int k = threadIdx.x; k <= n / 2; k += blockDim.x) {
    const int km = k == 0 ? 0 : n - k;
    const double2 a = Z[k], b = Z[km];
    if (k == 0) {
      const double y0 = cmul(H[0], make_double2(a.x + a.y, 0.0)).x, yn = cmul(H[n], make_double2(a.x - a.y, 0.0)).x;
      Z[0] = make_double2(0.5 * (y0 + yn), 0.5 * (y0 - yn));
      continue;
    }
    const double2 e = cscale(0.5, cadd(a, cconj(b)));
    const double2 o = cscale(0.5, mul_mi(csub(a, cconj(b))));
    const double2 wk = tw[k], wm = tw[km];
    const double2 xk = cadd(e, cmul(wk, o));
    const double2 om = cscale(0.5, mul_mi(csub(b, cconj(a))));
    const double2 xm = cadd(cconj(e), cmul(wm, om));
    const double2 yk = cmul(H[k], xk), ym = cmul(H[km], xm);
    Z[k] = cadd(cscale(0.5, cadd(yk, cconj(ym))), mul_pi(cscale(0.5, cmul(csub(yk, cconj(ym)), cconj(wk)))));
    if (k != n / 2)
      Z[km] = cadd(cscale(0.5, cadd(ym, cconj(yk))), mul_pi(cscale(0.5, cmul(csub(ym, cconj(yk)), cconj(wm)))));
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kNodeThreads, 1) k_env_nodes_long(EnvModalArgsT<double> a) {
  extern __shared__ __align__(16) double2 en_long_raw[];
  const int n = a.n_to, h = n / 2, log_h = a.log_n_to - 1, node = blockIdx.x, nc = a.n_components;
  double2* S = en_long_raw;
  double2* gz = a.scratch + (size_t)node * (n + h);
  double2* ge = gz + n;
  const StageScalarsDev& st = *a.stage;
  const double2* Ex = reinterpret_cast<const double2*>(a.node_field) + (size_t)node * nc * n;
  const double2* Ey = Ex + (nc == 2 ? n : 0);
  double2* Px = reinterpret_cast<double2*>(a.node_streams) + (size_t)node * nc * n;
  double2* Py = Px + (nc == 2 ? n : 0);
  const bool raman = a.raman_spectrum != nullptr;
  const int drives = !raman ? 0 : (nc == 2 && a.raman_kernels == 2 ? 3 : 1);
  const double factor = a.kerr ? a.kerr_coefficient * st.kerr_density : 0.0;
  const double self = a.kerr_self, conj = a.kerr_conjugate;
  const double raman_scale = kEps0 * (a.raman_mixture ? 1.0 : st.raman_density);
  const double inv_n = 1.0 / (double)n;
  if (drives == 0) {
    for (int t = threadIdx.x; t < n; t += blockDim.x) node_sample<double>(a, Ex, Ey, Px, Py, t, 0.0, 0, nc, factor, self, conj);
    return;
  }
  for (int dr = 0; dr < drives; ++dr) {
    // the drive on [0, n), zero on [n, 2n), packed b[m] = d(2m) + i d(2m + 1), transformed
    long_forward(
        [&](int m) {
          double v[2] = {0.0, 0.0};
          if (2 * m < n) {
            for (int q = 0; q < 2; ++q) {
              const double2 x = Ex[2 * m + q];
              const double xx = 0.5 * (x.x * x.x + x.y * x.y);
              if (nc == 1) {
                v[q] = xx;
              } else {
                const double2 y = Ey[2 * m + q];
                const double yy = 0.5 * (y.x * y.x + y.y * y.y);
                v[q] = dr == 0 ? xx + yy : dr == 1 ? xx - yy : 2.0 * 0.5 * (x.x * y.x + x.y * y.y);
              }
            }
          }
          return make_double2(v[0], v[1]);
        },
        S, gz, ge, a.twiddles, log_h);
    spectrum_product_global(gz, a.raman_spectrum + (dr == 0 ? 0 : (size_t)(n + 1)), a.twiddles, n);
    // the convolution at samples t < n: packed bins j = t >> 1 < h, j = 2 i + half
    for (int half = 0; half < 2; ++half) {
      long_inverse_half(gz, S, a.twiddles, log_h, half);
      for (int i = threadIdx.x; i < h / 2; i += blockDim.x) {
        const double2 z = S[row_slot<double2>(bitrev(i, log_h))];
        for (int q = 0; q < 2; ++q) {
          const int t = 4 * i + 2 * half + q;
          node_sample<double>(a, Ex, Ey, Px, Py, t, raman_scale * ((q ? z.y : z.x) * inv_n), dr, nc, factor,
                              self, conj);
        }
      }
      __syncthreads();  // the next half's inputs overwrite the row
    }
  }
}

}  // namespace

cudaError_t configure_env_modal_kernels() {
  const int row = (int)(kMaxEnvelopeRowF64 * sizeof(double2));  // one FP64 row (or half a long one)
  const void* kernels[10] = {(const void*)k_env_inverse<double>, (const void*)k_env_inverse<float>,
                             (const void*)k_env_nodes<double>,   (const void*)k_env_nodes<float>,
                             (const void*)k_env_forward<double>, (const void*)k_env_forward<float>,
                             (const void*)k_env_inverse_long,    (const void*)k_env_inverse_long32,
                             (const void*)k_env_forward_long,    (const void*)k_env_nodes_long};
  for (int i = 0; i < 10; ++i) {
    const int shm = row;  // an FP32 row of 16 384 samples is as long as an FP64 row of 8 192
    cudaError_t e = cudaFuncSetAttribute(kernels[i], cudaFuncAttributeMaxDynamicSharedMemorySize, shm);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <class R>
cudaError_t launch_env_inverse(const EnvModalArgsT<R>& a, cudaStream_t s) {
  if (a.n_to > kMaxEnvelopeRowF64) {
    const size_t half = (size_t)a.n_to / 2 * sizeof(double2);
    if constexpr (sizeof(R) == 8) k_env_inverse_long<<<a.n_cols, kEnvThreads, half, s>>>(a);
    else k_env_inverse_long32<<<a.n_cols, kEnvThreads, half, s>>>(a);
    return cudaGetLastError();
  }
  k_env_inverse<R><<<a.n_cols, kEnvThreads, (size_t)a.n_to * sizeof(double2), s>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_env_nodes(const EnvModalArgsT<R>& a, int n_nodes, cudaStream_t s) {
  if (sizeof(R) == 8 && a.n_to > kMaxEnvelopeRowF64) {
    if constexpr (sizeof(R) == 8)
      k_env_nodes_long<<<n_nodes, kNodeThreads, (size_t)a.n_to / 2 * sizeof(double2), s>>>(a);
    return cudaGetLastError();
  }
  k_env_nodes<R><<<n_nodes, kNodeThreads, (size_t)a.n_to * sizeof(cplx<R>), s>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_env_forward(const EnvModalArgsT<R>& a, cudaStream_t s) {
  if (sizeof(R) == 8 && a.n_to > kMaxEnvelopeRowF64) {
    if constexpr (sizeof(R) == 8)
      k_env_forward_long<<<a.n_cols, kEnvThreads, (size_t)a.n_to / 2 * sizeof(double2), s>>>(a);
    return cudaGetLastError();
  }
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
