// FP64 complex transforms of rows too long for one CTA's shared memory (n = 2h samples, an
// h-sample half in shared memory), for the envelope grid's rows of 16 384 samples: one
// radix-2 step through a global scratch row beside the swizzled shared-memory FFT of
// fft.cuh.  The forward transform is decimation in time,
//   Z[k] = E[k] + w_n^k O[k],  Z[k + h] = E[k] - w_n^k O[k],
// E and O the h-point transforms of the even and odd samples; the inverse is decimation in
// frequency, its two halves
//   X[2i] = sum_j (Z[j] + Z[j + h]) w_h^-ij,  X[2i + 1] = sum_j (Z[j] - Z[j + h]) w_n^-j w_h^-ij.
// The twiddle table is the envelope grid's exp(-2 pi i m / 2n), m < n, so w_n^k = table[2k].
// Both are unnormalised; callers scale.
#pragma once
#include "fft.cuh"

namespace sp {

// Z = FFT_n(b) into gz (natural order, n entries) through ge (h entries); b[m] = load(m).
// Ends with the block's barrier.
template <class Load>
__device__ __forceinline__ void long_forward(Load load, double2* s, double2* gz, double2* ge,
                                            const double2* __restrict__ table, int log_h) {
  const int h = 1 << log_h, log_table = log_h + 2;
  for (int i = threadIdx.x; i < h; i += blockDim.x) s[row_slot<double2>(i)] = load(2 * i);
  __syncthreads();
  fft_dif_swizzled<false>(s, log_h, table, log_table);
  for (int k = threadIdx.x; k < h; k += blockDim.x) ge[k] = s[row_slot<double2>(bitrev(k, log_h))];
  __syncthreads();
  for (int i = threadIdx.x; i < h; i += blockDim.x) s[row_slot<double2>(i)] = load(2 * i + 1);
  __syncthreads();
  fft_dif_swizzled<false>(s, log_h, table, log_table);
  for (int k = threadIdx.x; k < h; k += blockDim.x) {
    const double2 e = ge[k];
    const double2 o = cmul(__ldg(table + 2 * k), s[row_slot<double2>(bitrev(k, log_h))]);
    gz[k] = cadd(e, o);
    gz[k + h] = csub(e, o);
  }
  __syncthreads();
}

// One half of X = IFFT_n(Z) (unnormalised) from gz: s[row_slot(bitrev(i))] = X[2 i + half].
// Ends with the block's barrier (the transform's last pass).
__device__ __forceinline__ void long_inverse_half(const double2* gz, double2* s, const double2* __restrict__ table,
                                                  int log_h, int half) {
  const int h = 1 << log_h, log_table = log_h + 2;
  for (int j = threadIdx.x; j < h; j += blockDim.x) {
    const double2 x0 = gz[j], x1 = gz[j + h];
    s[row_slot<double2>(j)] = half == 0 ? cadd(x0, x1) : cmul(csub(x0, x1), cconj(__ldg(table + 2 * j)));
  }
  __syncthreads();
  fft_dif_swizzled<true>(s, log_h, table, log_table);
}

}  // namespace sp
