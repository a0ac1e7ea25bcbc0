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

// ---------------------------------------------------------------------------
// The register-radix form of the same transform.  A pass fuses K radix-2 stages: each
// thread loads the 2^K points x[base + r q] (q = L / 2^K, L the current span), runs a
// 2^K-point DFT in registers, multiplies output f by w_L^(f j) and stores it back where it
// came from -- so the row ends in the same bit-reversed order as fft_dif_inplace, in
// ceil(log_n / K) passes instead of log_n / 2.  Radix 16 in FP32 and 8 in FP64 (the
// points fill 32 registers either way).  The row is stored swizzled (row_slot): the low
// bits of an index, which pick the element's place in a 128-byte line of banks, are XORed
// with every higher group of as many bits.  That is a bijection, and it keeps each pass's
// strided loads and stores and the epilogues' bit-reversed reads (stride M / 32 across a
// warp) at the minimum number of shared-memory wavefronts.

template <class C>
constexpr int kBankBits = sizeof(C) == 8 ? 4 : 3;  // log2 of the elements per 128 bytes
template <class C>
__host__ __device__ __forceinline__ int row_slot(int i) {
  constexpr int b = kBankBits<C>;
  constexpr int mask = (1 << b) - 1;
  int fold = 0;
#pragma unroll
  for (int shift = b; shift < 16; shift += b) fold ^= i >> shift;
  return i ^ (fold & mask);
}
template <class C>
__host__ __device__ constexpr size_t row_length(int n) { return (size_t)n; }
template <class C>
constexpr int kRadixBits = sizeof(C) == 8 ? 4 : 3;

template <int K>
__host__ __device__ constexpr int bitrev_const(int r) {
  int v = 0;
  for (int b = 0; b < K; ++b) v |= ((r >> b) & 1) << (K - 1 - b);
  return v;
}

// exp(-2 pi i m / span) (conjugated for the inverse) times a, for span <= 16: multiples of
// pi / 8, whose cosines are the constants below (the doubles nearest the exact values)
template <bool kInv, class C>
__device__ __forceinline__ C rotate_const(C a, int m, int span) {
  using T = decltype(a.x);
  const int e = (m * 16 / span) & 15;  // the angle in units of 2 pi / 16
  if (e == 0) return a;
  if (e == 4) return kInv ? mul_pi(a) : mul_mi(a);
  if (e == 8) { a.x = -a.x; a.y = -a.y; return a; }
  if (e == 12) return kInv ? mul_mi(a) : mul_pi(a);
  constexpr double c1 = 0.923879532511286756128183189396788933;  // cos pi/8
  constexpr double s1 = 0.382683432365089771728459984030398866;  // sin pi/8
  constexpr double h = 0.707106781186547524400844362104849039;   // cos pi/4
  const double cs[16] = {1, c1, h, s1, 0, -s1, -h, -c1, -1, -c1, -h, -s1, 0, s1, h, c1};
  const double sn[16] = {0, s1, h, c1, 1, c1, h, s1, 0, -s1, -h, -c1, -1, -c1, -h, -s1};
  C w;
  w.x = (T)cs[e];
  w.y = kInv ? (T)sn[e] : (T)-sn[e];
  return cmul(a, w);
}

// 2^K-point DFT of x in registers by K radix-2 DIF stages: x[r] ends as output bitrev(r)
template <int K, bool kInv, class C>
__device__ __forceinline__ void dft_registers(C (&x)[1 << K]) {
  constexpr int R = 1 << K;
#pragma unroll
  for (int span = R; span >= 2; span >>= 1) {
    const int half = span >> 1;
#pragma unroll
    for (int blk = 0; blk < R; blk += span) {
#pragma unroll
      for (int i = 0; i < half; ++i) {
        const C a = x[blk + i], b = x[blk + i + half];
        x[blk + i] = cadd(a, b);
        x[blk + i + half] = rotate_const<kInv>(csub(a, b), i, span);
      }
    }
  }
}

// w_L^e from the half table of exp(-2 pi i m / n_table), m < n_table / 2 (e < L)
template <bool kInv, class C>
__device__ __forceinline__ C span_twiddle(const C* __restrict__ table, int e, int shift, int half_table) {
  const int m = e << shift;
  C w;
  if (m < half_table) {
    w = __ldg(table + m);
  } else {
    w = __ldg(table + (m - half_table));
    w.x = -w.x;
    w.y = -w.y;
  }
  if (kInv) w.y = -w.y;
  return w;
}

// one pass of K fused stages at span 2^log_len over the swizzled row
template <int K, bool kInv, class C>
__device__ __forceinline__ void dif_pass(C* s, int log_n, int log_len, const C* __restrict__ table,
                                         int log_table) {
  constexpr int R = 1 << K;
  const int log_q = log_len - K;
  const int q = 1 << log_q;
  const int shift = log_table - log_len;
  const int half_table = 1 << (log_table - 1);
  for (int p = threadIdx.x; p < (1 << (log_n - K)); p += blockDim.x) {
    const int j = p & (q - 1);
    const int base = ((p >> log_q) << log_len) + j;
    C x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = s[row_slot<C>(base + r * q)];
    dft_registers<K, kInv>(x);
    if (j != 0) {
#pragma unroll
      for (int r = 1; r < R; ++r)
        x[r] = cmul(x[r], span_twiddle<kInv>(table, bitrev_const<K>(r) * j, shift, half_table));
    }
#pragma unroll
    for (int r = 0; r < R; ++r) s[row_slot<C>(base + r * q)] = x[r];
  }
  __syncthreads();
}

// The swizzled row s (s[row_slot(i)] = x[i], made visible by the caller's barrier) is
// transformed in place into bit-reversed order: s[row_slot(bitrev(k))] = X[k].  Twiddles as
// for fft_dif_inplace.
template <bool kInv, class C>
__device__ __forceinline__ void fft_dif_swizzled(C* s, int log_n, const C* __restrict__ table, int log_table) {
  constexpr int K = kRadixBits<C>;
  int log_len = log_n;
  for (; log_len >= K; log_len -= K) dif_pass<K, kInv>(s, log_n, log_len, table, log_table);
  if (K > 3 && log_len == 3) dif_pass<3, kInv>(s, log_n, 3, table, log_table);
  if (log_len == 2) dif_pass<2, kInv>(s, log_n, 2, table, log_table);
  if (log_len == 1) dif_pass<1, kInv>(s, log_n, 1, table, log_table);
}

}  // namespace sp
