// The kernels of one source evaluation on the modal route (field grid): solprop's
// passes 2-7 (docs/dev/architecture.md section 8), restated for sm_100a.
//
//   k_inverse_field   pad + c2r inverse transform of every modal column, in shared
//                     memory; epilogue writes the modal field and the in-stage
//                     absorber's stream -alpha(t) a(t) / 2      (transforms.py:31-84,
//                                                                stepping.py:286-369)
//   k_column_field    per quadrature node, a thread-block cluster spanning the time
//                     row: synthesis, ionisation rate, the band-filtered running
//                     integrals (two cluster-wide scans over DSMEM), the fraction, the
//                     total current and the Kerr cubic, windowed     (responses.py:678,
//                                                                plasma.py:59-323)
//   k_project         deterministic projection of the node streams onto the modes
//                                                                (transforms.py:142)
//   k_forward_field   r2c forward transform of every stream row and the crop
//                                                                (transforms.py:190)
//   k_stage_output    held plasma assembly, prefactor, window, absorber, inverse
//                     propagator                       (plasma.py:579, stepping.py:88)
#include <cooperative_groups.h>

#include "fft.cuh"
#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace sp {

// ----------------------------------------------------------------------------- K1
__global__ void __launch_bounds__(1024) k_inverse_field(InverseArgs a) {
  extern __shared__ double2 smem_c[];
  const int col = blockIdx.x;
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

// ----------------------------------------------------------------------------- K2
// Block-wide exclusive scan of one double per thread; returns the thread's offset and
// writes the block total to *total (shared).
__device__ double block_exclusive_scan(double v, double* warp_sums, double* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    double y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int n_warps = blockDim.x >> 5;
    double s = lane < n_warps ? warp_sums[lane] : 0.0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      double y = __shfl_up_sync(0xffffffffu, s, d);
      if (lane >= d) s += y;
    }
    if (lane < n_warps) warp_sums[lane] = s;  // inclusive
    if (lane == n_warps - 1) *total = s;
  }
  __syncthreads();
  double before = warp > 0 ? warp_sums[warp - 1] : 0.0;
  return before + x - v;
}

// The rate lookup of translate/ionisation.py:242-323: exp of a cubic in log|E| on
// uniform knots, exactly zero below field_min and rate_max above field_max.
__device__ __forceinline__ double rate_lookup(const ColumnArgs& a, double magnitude) {
  if (magnitude > a.field_max) return a.rate_max;
  if (!(magnitude >= a.field_min)) return 0.0;
  double lf = log(magnitude);
  long idx = (long)((lf - a.log_field_min) / a.d_log_field);
  if (idx < 0) idx = 0;
  if (idx > a.rate_intervals - 1) idx = a.rate_intervals - 1;
  double local = lf - (a.log_field_min + (double)idx * a.d_log_field);
  const double* c = a.rate_coefficients;
  const int n = a.rate_intervals;
  double v = ((c[idx] * local + c[n + idx]) * local + c[2 * n + idx]) * local + c[3 * n + idx];
  return exp(v);
}

// One running integral of the band rule (nonlinear/ionisation.py:566-653) over the
// node's row, which the cluster's CTAs share: values in, exclusive prefix of the
// trapezoid increments of the filtered values out.  ybuf holds [-H, L + H] around the
// CTA's span.
template <int SPT>
__device__ void band_running_integral(const ColumnArgs& a, const double (&vals)[SPT],
                                      double (&out)[SPT], double* ybuf, double* warp_sums,
                                      double* cta_total, cg::cluster_group& cluster,
                                      int rank, int n_ranks, int L) {
  const int H = a.half_width;
  const int local0 = threadIdx.x * SPT;
#pragma unroll
  for (int q = 0; q < SPT; ++q) ybuf[local0 + q] = vals[q];
  cluster.sync();
  // halos: neighbours' samples, or the point reflections at the row's ends
  if (threadIdx.x <= H) {
    const int m = threadIdx.x;  // 0..H
    if (m >= 1) {
      if (rank > 0) {
        double* left = cluster.map_shared_rank(ybuf, rank - 1);
        ybuf[-m] = left[L - m];
      } else {
        ybuf[-m] = 2.0 * ybuf[0] - ybuf[m];
      }
    }
    if (rank < n_ranks - 1) {
      double* right = cluster.map_shared_rank(ybuf, rank + 1);
      ybuf[L + m] = right[m];
    } else if (m >= 1) {
      ybuf[L - 1 + m] = 2.0 * ybuf[L - 1] - ybuf[L - 1 - m];
    }
  }
  cluster.sync();  // remote reads done before anyone rewrites a buffer
  const double* c = a.taps;
  double filtered[SPT + 1];
#pragma unroll
  for (int q = 0; q <= SPT; ++q) {
    const int t = local0 + q;
    double f = c[0] * ybuf[t];
    for (int k = 1; k <= H; ++k) f = f + c[k] * (ybuf[t - k] + ybuf[t + k]);
    filtered[q] = f;
  }
  const int t_global0 = rank * L + local0;
  double inc[SPT];
  double sum = 0.0;
#pragma unroll
  for (int q = 0; q < SPT; ++q) {
    inc[q] = (t_global0 + q < a.n_to - 1) ? a.dt * (filtered[q + 1] + filtered[q]) / 2.0 : 0.0;
    sum += inc[q];
  }
  double offset = block_exclusive_scan(sum, warp_sums, cta_total);
  cluster.sync();
  double cta_offset = 0.0;
  for (int r = 0; r < rank; ++r) cta_offset += *cluster.map_shared_rank(cta_total, r);
  double run = cta_offset + offset;
#pragma unroll
  for (int q = 0; q < SPT; ++q) {
    out[q] = run;
    run += inc[q];
  }
  cluster.sync();  // cta_total read by the cluster before the next integral rewrites it
}

template <int SPT>
__global__ void __launch_bounds__(512) k_column_field(ColumnArgs a) {
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int n_ranks = (int)cluster.num_blocks();
  const int node = blockIdx.y;
  const int L = a.n_to / n_ranks;
  extern __shared__ double smem_d[];
  double* warp_sums = smem_d;                        // 32
  double* totals = smem_d + 32;                      // 2 (one per integral)
  double* ybuf = smem_d + 40 + a.half_width;         // [-H, L + H]
  const StageScalarsDev& st = *a.stage;
  const int t0 = rank * L + threadIdx.x * SPT;
  double E[SPT], W[SPT], F[SPT];
  // synthesis: E = sum_m (S tau)[node, m] a[m, t]   (transforms.py:87-139)
  {
    const double tau = st.taper;
#pragma unroll
    for (int q = 0; q < SPT; ++q) E[q] = 0.0;
    for (int m = 0; m < a.n_modes; ++m) {
      const double s = a.synthesis[node * a.n_modes + m] * tau;
      const double* am = a.modal_t + (size_t)m * a.n_to + t0;
#pragma unroll
      for (int q = 0; q < SPT; ++q) E[q] += s * am[q];
    }
  }
  double P[SPT], X[SPT], Z[SPT];
  const double* win = a.t_window + t0;
  const double* dwin = a.t_window_derivative + t0;
  if (a.plasma) {
#pragma unroll
    for (int q = 0; q < SPT; ++q) W[q] = rate_lookup(a, fabs(E[q]));
    double S[SPT];
    band_running_integral<SPT>(a, W, S, ybuf, warp_sums, totals + 0, cluster, rank, n_ranks, L);
    const double f0 = st.preionisation;
#pragma unroll
    for (int q = 0; q < SPT; ++q) {
      const double x = a.band ? fmax(S[q], 0.0) : S[q];
      F[q] = 1.0 - (1.0 - f0) * exp(-x);
    }
    double G[SPT], J[SPT];
#pragma unroll
    for (int q = 0; q < SPT; ++q) G[q] = F[q] * a.charge_mass_ratio * E[q];
    band_running_integral<SPT>(a, G, J, ybuf, warp_sums, totals + 1, cluster, rank, n_ranks, L);
    const double rho = st.plasma_density;
#pragma unroll
    for (int q = 0; q < SPT; ++q) {
      const double squared = fabs(E[q]) * fabs(E[q]);
      double scale = 0.0;
      if (W[q] > 0.0 && squared > 0.0) scale = a.ionisation_potential * W[q] * (1.0 - F[q]) / squared;
      const double current = rho * (J[q] + scale * E[q]);
      X[q] = win[q] * current;
      Z[q] = dwin[q] * current;
    }
  }
  // Kerr, real cubic: (c rho) E^2 E   (responses.py:65-139)
  const double factor = a.kerr ? a.kerr_coefficient * st.kerr_density : 0.0;
#pragma unroll
  for (int q = 0; q < SPT; ++q) {
    const double pk = a.kerr ? factor * (E[q] * E[q]) * E[q] : 0.0;
    P[q] = pk * win[q];
  }
  double* outP = a.node_p + (size_t)node * a.n_to + t0;
#pragma unroll
  for (int q = 0; q < SPT; ++q) outP[q] = P[q];
  if (a.plasma) {
    double* outX = a.node_x + (size_t)node * a.n_to + t0;
    double* outZ = a.node_z + (size_t)node * a.n_to + t0;
#pragma unroll
    for (int q = 0; q < SPT; ++q) {
      outX[q] = X[q];
      outZ[q] = Z[q];
    }
  }
}

// ----------------------------------------------------------------------------- K3
__global__ void __launch_bounds__(256) k_project(ProjectArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_to) return;
  const double tau = a.stage->taper;
  double acc[3][kMaxModes];
#pragma unroll
  for (int s = 0; s < 3; ++s)
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m) acc[s][m] = 0.0;
  for (int node = 0; node < a.n_nodes; ++node) {
    const size_t off = (size_t)node * a.n_to + t;
    const double p = a.node_p[off];
    const double x = a.n_streams > 1 ? a.node_x[off] : 0.0;
    const double z = a.n_streams > 1 ? a.node_z[off] : 0.0;
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m) {
      if (m < a.n_modes) {
        const double w = a.projection[m * a.n_nodes + node] / tau;
        acc[0][m] += w * p;
        acc[1][m] += w * x;
        acc[2][m] += w * z;
      }
    }
  }
#pragma unroll
  for (int m = 0; m < kMaxModes; ++m) {
    if (m < a.n_modes) {
      for (int s = 0; s < a.n_streams; ++s)
        a.streams[((size_t)s * a.n_cols + m) * a.n_to + t] = acc[s][m];
    }
  }
}

// ----------------------------------------------------------------------------- K4
__global__ void __launch_bounds__(1024) k_forward_field(ForwardArgs a) {
  extern __shared__ double2 smem_c[];
  const int row = a.rows[blockIdx.x];
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

// ----------------------------------------------------------------------------- K5
__global__ void k_stage_output(OutputArgs a) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
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

// ----------------------------------------------------------------------------- launch
template <int SPT>
static cudaError_t launch_column_spt(const ColumnArgs& a, int cluster, cudaStream_t stream) {
  const int L = a.n_to / cluster;
  const int threads = L / SPT;
  const size_t shm = (40 + (size_t)L + 2 * a.half_width + 2) * sizeof(double);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cluster, a.n_nodes, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = shm;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_column_field<SPT>, a);
}

cudaError_t launch_column(const ColumnArgs& a, cudaStream_t stream) {
  const int cluster = a.n_to > kColumnSpan ? a.n_to / kColumnSpan : 1;
  const int L = a.n_to / cluster;
  const int spt = L >= kColumnThreads ? L / kColumnThreads : 1;
  switch (spt) {
    case 1: return launch_column_spt<1>(a, cluster, stream);
    case 2: return launch_column_spt<2>(a, cluster, stream);
    case 4: return launch_column_spt<4>(a, cluster, stream);
    case 8: return launch_column_spt<8>(a, cluster, stream);
    default: return cudaErrorInvalidValue;
  }
}

static int threads_for(int m) { return m >= 1024 ? 1024 : (m >= 32 ? m : 32); }

cudaError_t launch_inverse(const InverseArgs& a, int n_cols, cudaStream_t stream) {
  if (fft_cluster_size(a.n_to) > 1) return launch_inverse_cluster(a, n_cols, stream);
  const int M = a.n_to >> 1;
  const size_t shm = (size_t)M * sizeof(double2);
  k_inverse_field<<<n_cols, threads_for(M), shm, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_project(const ProjectArgs& a, cudaStream_t stream) {
  k_project<<<(a.n_to + 255) / 256, 256, 0, stream>>>(a);
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
  e = cudaFuncSetAttribute(k_column_field<1>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_column_field<2>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_column_field<4>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_column_field<8>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

}  // namespace sp
