// The source evaluation on the envelope grid (complex time samples, c2c transforms) for a
// single modal column on a single node -- the generalised NLSE of a single-mode fibre:
// passes/transforms.py:31-84 and 190-233 (ifft / fft with the crop), responses.py:65-139
// (the analytic Kerr cubic), responses.py:218-498 (the Raman response as a doubled-grid
// convolution), the projection, all in one CTA:
//
//   A <- ifft(pad(lab))                                   the envelope a(t), E = tau S a
//   B <- rfft of the damped Raman kernel (length 2 n_to)  -> H = dt rfft(f_R sum_r h_r e^{-g_r t})
//   B <- rfft of the drive |E|^2 / 2, zero-padded to 2 n_to -> Y = H D
//   B <- irfft(Y)[:n_to]                                  the convolution
//   C <- (W / tau)(Kerr + eps0 rho_R E conv) g(t), fft, crop   -> the spectrum
//
// Real transforms of length 2 n_to run as complex transforms of length n_to (even samples
// real, odd imaginary) with the usual unpacking; every transform is the shared-memory
// radix-4 FFT of fft.cuh over one twiddle table of exp(-2 pi i m / (2 n_to)), m < n_to.
#include "fft.cuh"
#include "kernels.cuh"

namespace sp {

namespace {

constexpr double kEps0 = 8.8541878188e-12;  // vacuum permittivity (F/m), CODATA 2022, as solprop.constants

// X[k] = E_k + w^k O_k of a packed real transform of length 2 n (k in [0, n]); Z in
// bit-reversed order, w = exp(-2 pi i k / 2n) = tw[k] (k < n), -1 at k = n
__device__ __forceinline__ double2 unpack_real(const double2* Z, const double2* tw, int k, int n, int log_n) {
  const int kk = k == n ? 0 : k;
  const int km = k == 0 ? 0 : (n - k == n ? 0 : n - k);
  const double2 zk = Z[bitrev(kk, log_n)];
  const double2 zm = cconj(Z[bitrev(km, log_n)]);
  const double2 e = cscale(0.5, cadd(zk, zm));
  const double2 o = cscale(0.5, mul_mi(csub(zk, zm)));
  const double2 w = k < n ? tw[k] : make_double2(-1.0, 0.0);
  return cadd(e, cmul(w, o));
}

}  // namespace

__global__ void __launch_bounds__(1024) k_envelope_source(EnvelopeArgs a) {
  extern __shared__ __align__(16) unsigned char env_raw[];
  const int n = a.n_to;
  double2* A = reinterpret_cast<double2*>(env_raw);
  double2* B = A + n;
  double2* C = B + n;
  __shared__ double2 top;  // bin n of the length-2n spectra (H, then Y)
  const StageScalarsDev& st = *a.stage;
  const double tau = st.taper;
  const double es = tau * a.synthesis;  // E = tau S a
  const double inv_n = 1.0 / (double)n;
  // (i) the envelope: pad the coarse spectrum at the crop, inverse transform (scipy's
  // ifft carries 1 / n_to)
  for (int k = threadIdx.x; k < n; k += blockDim.x) A[k] = make_double2(0.0, 0.0);
  __syncthreads();
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x) A[a.crop[j]] = a.lab[j];
  __syncthreads();
  fft_dif_inplace(A, a.log_n_to, a.twiddles, a.log_n_to + 1, /*inverse=*/true);
  auto field = [&](int t) -> double2 { return cscale(es * inv_n, A[bitrev(t, a.log_n_to)]); };
  const bool raman = a.raman_terms > 0;
  if (raman) {
    // (ii) H = dt rfft(f_R sum_r h_r(s) exp(-g_r s dt)), s in [0, 2n), packed
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
      double v[2];
      for (int q = 0; q < 2; ++q) {
        const int s = 2 * m + q;
        double k = 0.0;
        for (int r = 0; r < a.raman_terms; ++r)
          k += a.raman_undamped[(size_t)r * 2 * n + s] * exp(-st.raman_rates[r] * ((double)s * a.dt));
        v[q] = a.raman_fraction * k;
      }
      B[m] = make_double2(v[0], v[1]);
    }
    __syncthreads();
    fft_dif_inplace(B, a.log_n_to, a.twiddles, a.log_n_to + 1, /*inverse=*/false);
    for (int k = threadIdx.x; k <= n; k += blockDim.x) {
      const double2 h = cscale(a.dt, unpack_real(B, a.twiddles, k, n, a.log_n_to));
      if (k < n) C[k] = h;
      else top = h;
    }
    __syncthreads();
    // (iii) the drive d(s) = |E(s)|^2 / 2 for s < n, zero above, packed
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
      double v[2] = {0.0, 0.0};
      if (2 * m < n) {
        for (int q = 0; q < 2; ++q) {
          const double2 e = field(2 * m + q);
          v[q] = 0.5 * (e.x * e.x + e.y * e.y);
        }
      }
      B[m] = make_double2(v[0], v[1]);
    }
    __syncthreads();
    fft_dif_inplace(B, a.log_n_to, a.twiddles, a.log_n_to + 1, /*inverse=*/false);
    // (iv) Y = H D, in place over H
    for (int k = threadIdx.x; k <= n; k += blockDim.x) {
      const double2 d = unpack_real(B, a.twiddles, k, n, a.log_n_to);
      if (k < n) C[k] = cmul(C[k], d);
      else top = cmul(top, d);
    }
    __syncthreads();
    // (v) irfft of length 2n: Z_k = E_k + i O_k, E_k = (Y_k + Y*_{n-k}) / 2,
    // O_k = (Y_k - Y*_{n-k}) conj(w^k) / 2; imaginary parts of bins 0 and n dropped
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
  }
  // (vi) the polarisation, gated and projected, in natural order into C
  const double factor = a.kerr ? a.kerr_coefficient * st.kerr_density : 0.0;
  const double raman_scale = kEps0 * st.raman_density;
  const double proj = a.projection / tau;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const double2 e = field(t);
    double2 p = make_double2(0.0, 0.0);
    if (a.kerr) {
      const double mod = e.x * e.x + e.y * e.y;
      const double2 sq = cmul(e, e);
      p = cscale(factor, cadd(cscale(a.kerr_self * mod, e), cscale(a.kerr_conjugate, cmul(sq, cconj(e)))));
    }
    if (raman) {
      const double2 z = B[bitrev(t >> 1, a.log_n_to)];
      const double conv = ((t & 1) ? z.y : z.x) * inv_n;  // irfft's 1 / (2n), with the packing's 2
      p = cadd(p, cscale(raman_scale * conv, e));
    }
    C[t] = cscale(proj * a.t_window[t], p);
  }
  __syncthreads();
  // (vii) forward transform and crop
  fft_dif_inplace(C, a.log_n_to, a.twiddles, a.log_n_to + 1, /*inverse=*/false);
  for (int j = threadIdx.x; j < a.n_omega; j += blockDim.x)
    a.spectra[j] = C[bitrev((int)a.crop[j], a.log_n_to)];
}

size_t envelope_smem(int n_to) { return (size_t)3 * n_to * sizeof(double2); }

cudaError_t launch_envelope(const EnvelopeArgs& a, cudaStream_t stream) {
  k_envelope_source<<<1, 1024, envelope_smem(a.n_to), stream>>>(a);
  return cudaGetLastError();
}

cudaError_t configure_envelope_kernels() {
  return cudaFuncSetAttribute(k_envelope_source, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)envelope_smem(kMaxEnvelopeSamples));
}

}  // namespace sp
