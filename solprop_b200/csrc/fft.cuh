// A complex FFT (FP64, or FP32 in the mixed-precision form) of one row held in shared
// memory, for power-of-two lengths.
//
// In-place decimation in frequency: natural-order input, bit-reversed output; two
// radix-2 stages are fused per pass (a radix-4 butterfly in registers), so a 2^13-point
// row takes 7 passes over shared memory.  Twiddles are read from a table of
// exp(-2 pi i m / n_table), m < n_table / 2, which the host computes in long double and
// rounds once, so every twiddle is the correctly rounded value.  The transform is
// unnormalised in both directions; callers scale.
#pragma once
#include "sp_common.cuh"

namespace sp {

__device__ __forceinline__ unsigned bitrev(unsigned k, int log_n) {
  return __brev(k) >> (32 - log_n);
}

// w_L^j for the table of n_table entries (stride = n_table / L); conj for inverse.
template <class C>
__device__ __forceinline__ C twiddle(const C* __restrict__ table, int index, bool inverse) {
  C w = __ldg(table + index);
  if (inverse) w.y = -w.y;
  return w;
}

// In-place DIF FFT of s[0..n) by the whole block; n = 2^log_n <= n_table.
template <class C>
__device__ __noinline__ static void fft_dif_inplace(C* s, int log_n, const C* __restrict__ table,
                                                    int log_table, bool inverse) {
  const int n = 1 << log_n;
  int log_len = log_n;
  // radix-4 passes: stages of span L and L/2
  for (; log_len >= 2; log_len -= 2) {
    const int L = 1 << log_len;
    const int q = L >> 2;
    const int log_q = log_len - 2;
    const int shift_L = log_table - log_len;  // w_L^j = table[j << shift_L]
    for (int p = threadIdx.x; p < (n >> 2); p += blockDim.x) {
      const int b = p >> log_q;
      const int j = p & (q - 1);
      const int base = (b << log_len) + j;
      C a0 = s[base], a1 = s[base + q], a2 = s[base + 2 * q], a3 = s[base + 3 * q];
      const C w1 = twiddle(table, j << shift_L, inverse);        // w_L^j
      const C w2 = twiddle(table, (2 * j) << shift_L, inverse);  // w_{L/2}^j
      C t0 = cadd(a0, a2);
      C t2 = cmul(csub(a0, a2), w1);
      C t1 = cadd(a1, a3);
      C d13 = csub(a1, a3);
      // w_L^{j+q} = w_L^j * (-i) forward, (+i) inverse
      C t3 = cmul(inverse ? mul_pi(d13) : mul_mi(d13), w1);
      s[base] = cadd(t0, t1);
      s[base + q] = cmul(csub(t0, t1), w2);
      s[base + 2 * q] = cadd(t2, t3);
      s[base + 3 * q] = cmul(csub(t2, t3), w2);
    }
    __syncthreads();
  }
  if (log_len == 1) {  // one radix-2 stage of span 2, twiddle 1
    for (int p = threadIdx.x; p < (n >> 1); p += blockDim.x) {
      C a = s[2 * p], b = s[2 * p + 1];
      s[2 * p] = cadd(a, b);
      s[2 * p + 1] = csub(a, b);
    }
    __syncthreads();
  }
}

}  // namespace sp
