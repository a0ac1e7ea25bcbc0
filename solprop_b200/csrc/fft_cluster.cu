// The field grid's transforms split over a thread-block cluster: a complex FFT of
// M = n_to / 2 points as C sub-transforms of M / C points, one per CTA, and C-point
// transforms across the cluster through distributed shared memory (the four-step
// factorisation M = C x M', n = C n2 + n1, k = k1 + M' k2):
//   Y_n1[k1] = sum_n2 z[C n2 + n1] w_M'^(n2 k1)          (each CTA, in shared memory)
//   Z[k1 + M' k2] = sum_n1 w_C^(n1 k2) w_M^(n1 k1) Y_n1[k1]   (across the cluster)
// The real-to-complex and complex-to-real packing around it (x[2m] + i x[2m+1], and
// E[k] = (X[k] + X*[M-k])/2, O[k] = (X[k] - X*[M-k]) w^-k / 2) is the single-CTA
// kernels' (source_kernels.cu); the inverse prologue builds the strided Z samples
// directly from the coarse spectrum, and the forward epilogue reads Z[k] and Z[M - k]
// from whichever CTA holds them.
#include <cooperative_groups.h>

#include "fft.cuh"
#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace sp {

namespace {

constexpr int kFftCluster = 8;

// w_M^j = exp(-2 pi i j / M) from the table of n_to = 2M entries' first half
__device__ __forceinline__ double2 w_m(const double2* __restrict__ table, long j, int log_m,
                                       bool inverse) {
  const long M = 1L << log_m;
  j &= (M - 1);
  double2 w;
  if (j < M / 2) {
    w = __ldg(table + 2 * j);
  } else {
    const double2 v = __ldg(table + 2 * (j - M / 2));
    w = make_double2(-v.x, -v.y);  // w_M^(j) = -w_M^(j - M/2)
  }
  return inverse ? make_double2(w.x, -w.y) : w;
}

// The C values Y_n1[k1] of one k1, twiddled by w_M^(n1 k1), then their C-point DFT:
// out[k2] = sum_n1 w_C^(n1 k2) w_M^(n1 k1) Y_n1[k1].  All loads are issued before any use.
template <int C>
__device__ __forceinline__ void cross_dft(cg::cluster_group& cluster, double2* sc, int k1,
                                          int log_mp, const double2* __restrict__ tw, int log_m,
                                          bool inverse, double2 (&out)[C]) {
  double2 y[C], w[C];
#pragma unroll
  for (int n1 = 0; n1 < C; ++n1) y[n1] = cluster.map_shared_rank(sc, n1)[bitrev(k1, log_mp)];
#pragma unroll
  for (int n1 = 0; n1 < C; ++n1) w[n1] = w_m(tw, (long)n1 * k1, log_m, inverse);
  const int Mp = 1 << log_mp;
  double2 root[C];  // w_C^j = w_M^(j Mp)
#pragma unroll
  for (int j = 0; j < C; ++j) root[j] = w_m(tw, (long)j * Mp, log_m, inverse);
#pragma unroll
  for (int n1 = 0; n1 < C; ++n1) y[n1] = cmul(w[n1], y[n1]);
#pragma unroll
  for (int k2 = 0; k2 < C; ++k2) {
    double2 acc = y[0];
#pragma unroll
    for (int n1 = 1; n1 < C; ++n1) acc = cadd(acc, cmul(root[(n1 * k2) % C], y[n1]));
    out[k2] = acc;
  }
}

}  // namespace

// inverse (c2r): coarse spectrum -> modal field (and the absorber's stream)
__device__ __forceinline__ void inverse_cluster_body(const InverseArgs& a, int col) {
  cg::cluster_group cluster = cg::this_cluster();
  const int C = (int)cluster.num_blocks();
  const int r = (int)cluster.block_rank();
  extern __shared__ double2 sc[];
  const int M = a.n_to >> 1;
  const int Mp = M / C;
  const int log_mp = a.log_m - __ffs(C) + 1;
  const double2* lab = a.lab + (size_t)col * a.n_omega;
  const double2* tw = a.twiddles;
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
  // Z[k] = E[k] + i O[k] at k = C n2 + r
#pragma unroll 4
  for (int n2 = threadIdx.x; n2 < Mp; n2 += blockDim.x) {
    const int k = C * n2 + r;
    const double2 xk = fine(k), xm = cconj(fine(M - k));
    const double2 e = cscale(0.5, cadd(xk, xm));
    const double2 w = __ldg(tw + k);
    const double2 o = cscale(0.5, cmul(csub(xk, xm), cconj(w)));
    sc[n2] = cadd(e, mul_pi(o));
  }
  __syncthreads();
  fft_dif_inplace(sc, log_mp, tw, a.log_n_to, /*inverse=*/true);  // sc[bitrev(k1)] = Y_r[k1]
  cluster.sync();
  // this CTA's slice of k1; z[k1 + Mp k2] for every k2
  const int slice = Mp / C;
  const double inv_m = 1.0 / (double)M;
  double* row = a.modal_t + (size_t)col * a.n_to;
  double* absorb = a.absorber_stream ? a.absorber_stream + (size_t)col * a.n_to : nullptr;
  for (int kk = threadIdx.x; kk < slice; kk += blockDim.x) {
    const int k1 = r * slice + kk;
    double2 z[kFftCluster];
    cross_dft<kFftCluster>(cluster, sc, k1, log_mp, tw, a.log_m, true, z);
#pragma unroll
    for (int k2 = 0; k2 < kFftCluster; ++k2) {
      const int m = k1 + Mp * k2;
      const double x0 = z[k2].x * inv_m, x1 = z[k2].y * inv_m;
      reinterpret_cast<double2*>(row)[m] = make_double2(x0, x1);
      if (absorb) {
        const double2 al = reinterpret_cast<const double2*>(a.alpha)[m];
        reinterpret_cast<double2*>(absorb)[m] = make_double2(-0.5 * al.x * x0, -0.5 * al.y * x1);
      }
    }
  }
  cluster.sync();  // no CTA leaves while another reads its shared memory
}

__global__ void __launch_bounds__(512) k_inverse_cluster(InverseArgs a) {
  inverse_cluster_body(a, blockIdx.y);
}

// batched: items[blockIdx.y] = (run, column)
__global__ void __launch_bounds__(512) k_inverse_cluster_b(const InverseArgs* args, const int2* items,
                                                          const int* flags) {
  const int2 it = items[blockIdx.y];
  if (!flags[it.x]) return;  // uniform over the cluster: every CTA of it has this item
  inverse_cluster_body(args[it.x], it.y);
}

// forward (r2c): stream rows -> cropped coarse spectra
__device__ __forceinline__ void forward_cluster_body(const ForwardArgs& a, int row_index) {
  cg::cluster_group cluster = cg::this_cluster();
  const int C = (int)cluster.num_blocks();
  const int r = (int)cluster.block_rank();
  const int row = a.rows[row_index];
  extern __shared__ double2 sc[];
  const int M = a.n_to >> 1;
  const int Mp = M / C;
  const int log_mp = a.log_m - __ffs(C) + 1;
  double2* zb = sc + Mp;  // Z for this CTA's k1 slice: [k2][k1 - r slice]
  const int slice = Mp / C;
  // z[C n2 + r] = x[2(C n2 + r)] + i x[2(C n2 + r) + 1]
  if (row < a.n_partial_rows) {
#pragma unroll 4
    for (int n2 = threadIdx.x; n2 < Mp; n2 += blockDim.x) {
      const int m = C * n2 + r;
      double2 acc = make_double2(0.0, 0.0);
      for (int g = 0; g < a.n_groups; ++g)
        acc = cadd(acc, reinterpret_cast<const double2*>(
                            a.partials + ((size_t)g * a.n_partial_rows + row) * a.n_to)[m]);
      sc[n2] = acc;
    }
  } else {
    const double2* x = reinterpret_cast<const double2*>(a.streams + (size_t)row * a.n_to);
#pragma unroll 4
    for (int n2 = threadIdx.x; n2 < Mp; n2 += blockDim.x) sc[n2] = x[C * n2 + r];
  }
  __syncthreads();
  fft_dif_inplace(sc, log_mp, a.twiddles, a.log_n_to, /*inverse=*/false);
  cluster.sync();
  for (int kk = threadIdx.x; kk < slice; kk += blockDim.x) {
    const int k1 = r * slice + kk;
    double2 z[kFftCluster];
    cross_dft<kFftCluster>(cluster, sc, k1, log_mp, a.twiddles, a.log_m, false, z);
#pragma unroll
    for (int k2 = 0; k2 < kFftCluster; ++k2) zb[k2 * slice + kk] = z[k2];
  }
  cluster.sync();
  // X[k] = E[k] + w^k O[k] from Z[k] and Z[M - k] (Z[M] = Z[0]); bins strided by rank
  auto zat = [&](int k) -> double2 {
    if (k == M) k = 0;
    const int k1 = k % Mp, k2 = k / Mp;
    const int owner = k1 / slice;
    const double2* src = cluster.map_shared_rank(zb, owner);
    return src[k2 * slice + (k1 - owner * slice)];
  };
  double2* out = a.spectra + (size_t)row * a.n_omega;
  for (int j = r * blockDim.x + threadIdx.x; j < a.n_omega; j += C * blockDim.x) {
    const int k = a.crop_identity ? j : (int)a.crop_index[j];
    const int km = (k == 0) ? 0 : M - k;
    const double2 zk = zat(k), zm = cconj(zat(km));
    const double2 e = cscale(0.5, cadd(zk, zm));
    const double2 o = cscale(0.5, mul_mi(csub(zk, zm)));
    const double2 w = k < M ? __ldg(a.twiddles + k) : make_double2(-1.0, 0.0);
    out[j] = cadd(e, cmul(w, o));
  }
  cluster.sync();
}

__global__ void __launch_bounds__(512) k_forward_cluster(ForwardArgs a) {
  forward_cluster_body(a, blockIdx.y);
}

// batched: items[blockIdx.y] = (run, row index)
__global__ void __launch_bounds__(512) k_forward_cluster_b(const ForwardArgs* args, const int2* items,
                                                          const int* flags) {
  const int2 it = items[blockIdx.y];
  if (!flags[it.x]) return;
  forward_cluster_body(args[it.x], it.y);
}

static cudaError_t launch_cluster(const void* kernel, dim3 grid, int threads, size_t shm, int C,
                                  cudaStream_t stream, void** args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = shm;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, kernel, args);
}

int fft_cluster_size(int n_to) {
  const int M = n_to / 2;
  if (M <= 2048) return 1;
  return kFftCluster;  // portable cluster; M / 8 points per CTA
}

cudaError_t launch_inverse_cluster(const InverseArgs& a, int n_cols, cudaStream_t stream) {
  const int C = fft_cluster_size(a.n_to);
  const int Mp = (a.n_to / 2) / C;
  InverseArgs copy = a;
  void* args[] = {&copy};
  return launch_cluster((const void*)k_inverse_cluster, dim3(C, n_cols), Mp >= 512 ? 512 : Mp, (size_t)Mp * sizeof(double2),
                        C, stream, args);
}

cudaError_t launch_forward_cluster(const ForwardArgs& a, int n_rows, cudaStream_t stream) {
  const int C = fft_cluster_size(a.n_to);
  const int Mp = (a.n_to / 2) / C;
  ForwardArgs copy = a;
  void* args[] = {&copy};
  return launch_cluster((const void*)k_forward_cluster, dim3(C, n_rows), Mp >= 512 ? 512 : Mp,
                        (size_t)2 * Mp * sizeof(double2), C, stream, args);
}

cudaError_t launch_inverse_cluster_b(const InverseArgs* args, const int2* items, const int* flags,
                                     int n_items, int n_to, cudaStream_t stream) {
  const int C = fft_cluster_size(n_to);
  const int Mp = (n_to / 2) / C;
  void* params[] = {(void*)&args, (void*)&items, (void*)&flags};
  return launch_cluster((const void*)k_inverse_cluster_b, dim3(C, n_items), Mp >= 512 ? 512 : Mp,
                        (size_t)Mp * sizeof(double2), C, stream, params);
}

cudaError_t launch_forward_cluster_b(const ForwardArgs* args, const int2* items, const int* flags,
                                     int n_items, int n_to, cudaStream_t stream) {
  const int C = fft_cluster_size(n_to);
  const int Mp = (n_to / 2) / C;
  void* params[] = {(void*)&args, (void*)&items, (void*)&flags};
  return launch_cluster((const void*)k_forward_cluster_b, dim3(C, n_items), Mp >= 512 ? 512 : Mp,
                        (size_t)2 * Mp * sizeof(double2), C, stream, params);
}

cudaError_t configure_cluster_fft() {
  // rows of up to 2^15 real samples: 2048 complex points per CTA, two buffers forward
  const int shm = 2 * 2048 * (int)sizeof(double2);
  cudaError_t e;
  e = cudaFuncSetAttribute(k_inverse_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, shm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_forward_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, shm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_inverse_cluster_b, cudaFuncAttributeMaxDynamicSharedMemorySize, shm);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_forward_cluster_b, cudaFuncAttributeMaxDynamicSharedMemorySize, shm);
}

}  // namespace sp
