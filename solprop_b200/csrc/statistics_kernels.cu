// Plane statistics of a state, formed where the state lives (the native workspace's
// statistics pass, native/src/general/statistics.cpp:106-450, and solprop's definitions in
// src/solprop/stats/definitions.py): per modal column the energy and the spectral
// centroid, the energy spectral density per bin summed over the columns, and the peak
// instantaneous power of each mode and of the whole field from the analytic signal.  Only
// the small results leave the device.
#include <cuda_runtime.h>

#include "fft.cuh"
#include "kernels.cuh"

namespace sp {
namespace {

constexpr int kStatThreads = 256;
constexpr int kPowerThreads = 512;

// the bin's weight in fourier.energy_omega: dt / n_t, times 4 for a field grid's
// interior bins (the analytic signal's doubling), 1 at its DC and Nyquist bins
__device__ __forceinline__ double energy_weight(const StatisticsArgs& a, int k) {
  const double base = a.dt / (double)a.n_t;
  if (a.envelope) return base;
  return (k == 0 || k == a.n_omega - 1) ? base : 4.0 * base;
}

__device__ __forceinline__ double block_sum(double v, double* shared) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) shared[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = lane < (int)(blockDim.x >> 5) ? shared[lane] : 0.0;
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  __syncthreads();
  return t;  // valid in warp 0
}

// one CTA per column: sum_k w_k |a_k|^2 p_k (energy), sum_k p|a|^2, sum_k omega_k p|a|^2
__global__ void k_stat_columns(StatisticsArgs a) {
  __shared__ double red[32];
  const int c = blockIdx.x;
  const double2* row = a.state + (size_t)c * a.n_omega;
  const double* pw = a.power_weight ? a.power_weight + (size_t)c * a.n_omega : nullptr;
  double e = 0.0, d = 0.0, m = 0.0;
  for (int k = threadIdx.x; k < a.n_omega; k += blockDim.x) {
    const double2 v = row[k];
    double p = v.x * v.x + v.y * v.y;
    if (pw) p *= pw[k];
    e += energy_weight(a, k) * p;
    d += p;
    m += a.omega[k] * p;
  }
  e = block_sum(e, red);
  d = block_sum(d, red);
  m = block_sum(m, red);
  if (threadIdx.x == 0) {
    a.out[kStatEnergy * a.n_cols + c] = e;
    a.out[kStatOmega0 * a.n_cols + c] = d > 0.0 ? m / d : __longlong_as_double(0x7ff8000000000000LL);
  }
}

// the energy spectral density per bin, summed over the columns (J per bin)
__global__ void k_stat_spectrum(StatisticsArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.n_omega) return;
  double s = 0.0;
  for (int c = 0; c < a.n_cols; ++c) {
    const double2 v = a.state[(size_t)c * a.n_omega + k];
    double p = v.x * v.x + v.y * v.y;
    if (a.power_weight) p *= a.power_weight[(size_t)c * a.n_omega + k];
    s += p;
  }
  a.out[a.spectrum_offset + k] = energy_weight(a, k) * s;
}

// the analytic signal's coefficient at bin k of the n_t-point transform (stats
// definitions.py analytic_field: an irfft, then scipy.signal.hilbert's weights; the
// envelope's samples are the ifft itself), including ifft's 1 / n_t
__device__ __forceinline__ double2 analytic_coefficient(const StatisticsArgs& a, const double2* row, int k) {
  const double inv_n = 1.0 / (double)a.n_t;
  if (a.envelope) return cscale(inv_n, row[k]);
  const int half = a.n_t / 2;
  if (k > half) return make_double2(0.0, 0.0);
  const double2 v = row[k];
  // irfft reads only the real parts of the DC and Nyquist bins
  if (k == 0 || k == half) return make_double2(inv_n * v.x, 0.0);
  return cscale(2.0 * inv_n, v);
}

// Instantaneous power |E_a(t)|^2 of one column at the times t = R m + r of residue class r
// (blockIdx.y), R = n_t / M: E_a(R m + r) = sum_{j<M} Y_j e^{2 pi i j m / M} with
// Y_j = e^{2 pi i j r / n_t} sum_{q<R} Z_{j+qM} e^{2 pi i q r / R}, one M-point inverse
// transform in shared memory.  The powers are written in the transform's bit-reversed
// order, the same for every column, which sums over columns and maxima do not mind.
__global__ void __launch_bounds__(kPowerThreads) k_stat_power(StatisticsArgs a) {
  extern __shared__ __align__(16) double2 row_s[];
  const int c = blockIdx.x, r = blockIdx.y;
  const int M = 1 << a.log_m, R = a.n_t >> a.log_m;
  const double2* row = a.state + (size_t)c * a.n_omega;
  for (int j = threadIdx.x; j < M; j += blockDim.x) {
    double2 acc = make_double2(0.0, 0.0);
    for (int q = 0; q < R; ++q) {
      double sn, cs;
      sincospi(2.0 * (double)((q * r) % R) / (double)R, &sn, &cs);
      acc = cadd(acc, cmul(analytic_coefficient(a, row, j + q * M), make_double2(cs, sn)));
    }
    double sn, cs;
    sincospi(2.0 * (double)(((long long)j * r) % a.n_t) / (double)a.n_t, &sn, &cs);
    row_s[j] = cmul(acc, make_double2(cs, sn));
  }
  __syncthreads();
  fft_dif_inplace(row_s, a.log_m, a.twiddles, a.log_table, true);
  double* out = a.power + (size_t)c * a.n_t + (size_t)r * M;
  for (int p = threadIdx.x; p < M; p += blockDim.x) {
    const double2 v = row_s[p];
    out[p] = v.x * v.x + v.y * v.y;
  }
}

// the peaks: per mode max_t sum_pol P, and max_t sum_columns P (stats definitions.py
// peak_power, peak_power_total)
__global__ void k_stat_peaks(StatisticsArgs a) {
  __shared__ double red[32];
  double best_total = 0.0;
  double best[kStatMaxModes];
  for (int m = 0; m < kStatMaxModes; ++m) best[m] = 0.0;
  for (int t = threadIdx.x; t < a.n_t; t += blockDim.x) {
    double total = 0.0;
    for (int m = 0; m < a.n_modes; ++m) {
      double pm = 0.0;
      for (int p = 0; p < a.n_pol; ++p) pm += a.power[(size_t)(m * a.n_pol + p) * a.n_t + t];
      if (m < kStatMaxModes) best[m] = fmax(best[m], pm);
      total += pm;
    }
    best_total = fmax(best_total, total);
  }
  auto block_max = [&](double v) {
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 32) {
      t = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
      for (int o = 16; o; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
    }
    __syncthreads();
    return t;
  };
  for (int m = 0; m < a.n_modes && m < kStatMaxModes; ++m) {
    const double v = block_max(best[m]);
    if (threadIdx.x == 0) a.out[a.peak_offset + m] = v;
  }
  const double v = block_max(best_total);
  if (threadIdx.x == 0) a.out[a.peak_offset + a.n_modes] = v;
}

}  // namespace

size_t statistics_power_smem(int log_m) { return sizeof(double2) << log_m; }

cudaError_t configure_statistics_kernels() {
  return cudaFuncSetAttribute(k_stat_power, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)statistics_power_smem(kStatLogRow));
}

cudaError_t launch_statistics(const StatisticsArgs& a, bool peaks, cudaStream_t s) {
  k_stat_columns<<<a.n_cols, kStatThreads, 0, s>>>(a);
  k_stat_spectrum<<<(a.n_omega + kStatThreads - 1) / kStatThreads, kStatThreads, 0, s>>>(a);
  if (peaks) {
    k_stat_power<<<dim3(a.n_cols, a.n_t >> a.log_m), kPowerThreads, statistics_power_smem(a.log_m), s>>>(a);
    k_stat_peaks<<<1, 1024, 0, s>>>(a);
  }
  return cudaGetLastError();
}

}  // namespace sp
