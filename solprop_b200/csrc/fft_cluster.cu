// The field grid's transforms split over a thread-block cluster (FP64, or FP32 in the
// mixed-precision form): a complex FFT of
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
template <class Cx>
__device__ __forceinline__ Cx w_m(const Cx* __restrict__ table, long j, int log_m, bool inverse) {
  const long M = 1L << log_m;
  j &= (M - 1);
  Cx w;
  if (j < M / 2) {
    w = __ldg(table + 2 * j);
  } else {
    w = __ldg(table + 2 * (j - M / 2));
    w.x = -w.x;  // w_M^(j) = -w_M^(j - M/2)
    w.y = -w.y;
  }
  if (inverse) w.y = -w.y;
  return w;
}

// The C values Y_n1[k1] of one k1, twiddled by w_M^(n1 k1), then their C-point DFT:
// out[k2] = sum_n1 w_C^(n1 k2) w_M^(n1 k1) Y_n1[k1].  All loads are issued before any use.
template <int C, class Cx>
__device__ __forceinline__ void cross_dft(cg::cluster_group& cluster, Cx* sc, int k1,
                                          int log_mp, const Cx* __restrict__ tw, int log_m,
                                          bool inverse, Cx (&out)[C]) {
  Cx y[C], w[C];
#pragma unroll
  for (int n1 = 0; n1 < C; ++n1) y[n1] = cluster.map_shared_rank(sc, n1)[row_slot<Cx>(bitrev(k1, log_mp))];
#pragma unroll
  for (int n1 = 0; n1 < C; ++n1) w[n1] = w_m(tw, (long)n1 * k1, log_m, inverse);
  const int Mp = 1 << log_mp;
  Cx root[C];  // w_C^j = w_M^(j Mp)
#pragma unroll
  for (int j = 0; j < C; ++j) root[j] = w_m(tw, (long)j * Mp, log_m, inverse);
#pragma unroll
  for (int n1 = 0; n1 < C; ++n1) y[n1] = cmul(w[n1], y[n1]);
#pragma unroll
  for (int k2 = 0; k2 < C; ++k2) {
    Cx acc = y[0];
#pragma unroll
    for (int n1 = 1; n1 < C; ++n1) acc = cadd(acc, cmul(root[(n1 * k2) % C], y[n1]));
    out[k2] = acc;
  }
}

}  // namespace

// inverse (c2r): coarse spectrum -> modal field (and the absorber's stream), over a
// cluster of C CTAs
template <int C, class R>
__device__ __forceinline__ void inverse_cluster_body(const InverseArgsT<R>& a, int col) {
  using Cx = cplx<R>;
  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx* sc = reinterpret_cast<Cx*>(smem_raw);
  const int M = a.n_to >> 1;
  const int Mp = M / C;
  const int log_mp = a.log_m - __ffs(C) + 1;
  const double2* lab = a.lab + (size_t)col * a.n_omega;
  const Cx* tw = a.twiddles;
  auto fine = [&](int k) -> Cx {
    double2 v;
    if (a.crop_identity) {
      v = k < a.n_omega ? lab[k] : make_double2(0.0, 0.0);
    } else {
      const int j = a.fine_to_coarse[k];
      v = j >= 0 ? lab[j] : make_double2(0.0, 0.0);
    }
    if (k == 0 || k == M) v.y = 0.0;
    return to_c<Cx>(v);
  };
  const R half = R(0.5);
  // Z[k] = E[k] + i O[k] at k = C n2 + r
#pragma unroll 4
  for (int n2 = threadIdx.x; n2 < Mp; n2 += blockDim.x) {
    const int k = C * n2 + r;
    const Cx xk = fine(k), xm = cconj(fine(M - k));
    const Cx e = cscale(half, cadd(xk, xm));
    const Cx w = __ldg(tw + k);
    const Cx o = cscale(half, cmul(csub(xk, xm), cconj(w)));
    sc[row_slot<Cx>(n2)] = cadd(e, mul_pi(o));
  }
  __syncthreads();
  fft_dif_swizzled</*kInv=*/true>(sc, log_mp, tw, a.log_n_to);  // sc[slot(bitrev(k1))] = Y_r[k1]
  cluster.sync();
  // this CTA's slice of k1; z[k1 + Mp k2] for every k2
  const int slice = Mp / C;
  const R inv_m = R(1.0 / (double)M);
  R* row = a.modal_t + (size_t)col * a.n_to;
  R* absorb = a.absorber_stream ? a.absorber_stream + (size_t)col * a.n_to : nullptr;
  for (int kk = threadIdx.x; kk < slice; kk += blockDim.x) {
    const int k1 = r * slice + kk;
    Cx z[C];
    cross_dft<C>(cluster, sc, k1, log_mp, tw, a.log_m, true, z);
#pragma unroll
    for (int k2 = 0; k2 < C; ++k2) {
      const int m = k1 + Mp * k2;
      Cx v;
      v.x = z[k2].x * inv_m;
      v.y = z[k2].y * inv_m;
      reinterpret_cast<Cx*>(row)[m] = v;
      if (absorb) {
        const Cx al = reinterpret_cast<const Cx*>(a.alpha)[m];
        Cx ab;
        ab.x = -half * al.x * v.x;
        ab.y = -half * al.y * v.y;
        reinterpret_cast<Cx*>(absorb)[m] = ab;
      }
    }
  }
  cluster.sync();  // no CTA leaves while another reads its shared memory
}

template <class R, int C>
__global__ void __launch_bounds__(512) k_inverse_cluster(InverseArgsT<R> a) {
  inverse_cluster_body<C>(a, blockIdx.y);
}

// batched: items[blockIdx.y] = (run, column)
template <class R, int C>
__global__ void __launch_bounds__(512) k_inverse_cluster_b(const InverseArgsT<R>* args, const int2* items,
                                                          const int* flags) {
  const int2 it = items[blockIdx.y];
  if (!flags[it.x]) return;  // uniform over the cluster: every CTA of it has this item
  inverse_cluster_body<C>(own_args(args, it.x), it.y);
}

// forward (r2c): stream rows -> cropped coarse spectra, over a cluster of C CTAs
template <int C, class R>
__device__ __forceinline__ void forward_cluster_body(const ForwardArgsT<R>& a, int row_index) {
  using Cx = cplx<R>;
  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  const int row = a.rows[row_index];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx* sc = reinterpret_cast<Cx*>(smem_raw);
  const int M = a.n_to >> 1;
  const int Mp = M / C;
  const int log_mp = a.log_m - __ffs(C) + 1;
  Cx* zb = sc + Mp;  // Z for this CTA's k1 slice: [k2][k1 - r slice]
  const int slice = Mp / C;
  // z[C n2 + r] = x[2(C n2 + r)] + i x[2(C n2 + r) + 1]
  if (row < a.n_partial_rows) {
    // a projected stream: the node groups' partial rows summed in group order, eight
    // groups' loads issued before their sums
    constexpr int kBatch = 8;
    const Cx* rows = reinterpret_cast<const Cx*>(a.partials + (size_t)row * a.n_to);
    const size_t group_stride = (size_t)a.n_partial_rows * a.n_to / 2;  // in complex samples
#pragma unroll 2
    for (int n2 = threadIdx.x; n2 < Mp; n2 += blockDim.x) {
      const int m = C * n2 + r;
      Cx acc;
      acc.x = R(0);
      acc.y = R(0);
      for (int g0 = 0; g0 < a.n_groups; g0 += kBatch) {
        Cx x[kBatch];
#pragma unroll
        for (int g = 0; g < kBatch; ++g)
          if (g0 + g < a.n_groups) x[g] = __ldg(rows + (size_t)(g0 + g) * group_stride + m);
#pragma unroll
        for (int g = 0; g < kBatch; ++g) {
          if (g0 + g >= a.n_groups) break;
          acc = cadd(acc, x[g]);
        }
      }
      sc[row_slot<Cx>(n2)] = acc;
    }
  } else {
    const double2* x = reinterpret_cast<const double2*>(a.streams + (size_t)row * a.n_to);
#pragma unroll 4
    for (int n2 = threadIdx.x; n2 < Mp; n2 += blockDim.x) sc[row_slot<Cx>(n2)] = to_c<Cx>(x[C * n2 + r]);
  }
  __syncthreads();
  fft_dif_swizzled</*kInv=*/false>(sc, log_mp, a.twiddles, a.log_n_to);
  cluster.sync();
  for (int kk = threadIdx.x; kk < slice; kk += blockDim.x) {
    const int k1 = r * slice + kk;
    Cx z[C];
    cross_dft<C>(cluster, sc, k1, log_mp, a.twiddles, a.log_m, false, z);
#pragma unroll
    for (int k2 = 0; k2 < C; ++k2) zb[k2 * slice + kk] = z[k2];
  }
  cluster.sync();
  // X[k] = E[k] + w^k O[k] from Z[k] and Z[M - k] (Z[M] = Z[0]); bins strided by rank
  auto zat = [&](int k) -> Cx {
    if (k == M) k = 0;
    const int k1 = k % Mp, k2 = k / Mp;
    const int owner = k1 / slice;
    const Cx* src = cluster.map_shared_rank(zb, owner);
    return src[k2 * slice + (k1 - owner * slice)];
  };
  Cx* out = a.spectra + (size_t)row * a.n_omega;
  const R half = R(0.5);
  for (int j = r * blockDim.x + threadIdx.x; j < a.n_omega; j += C * blockDim.x) {
    const int k = a.crop_identity ? j : (int)a.crop_index[j];
    const int km = (k == 0) ? 0 : M - k;
    const Cx zk = zat(k), zm = cconj(zat(km));
    const Cx e = cscale(half, cadd(zk, zm));
    const Cx o = cscale(half, mul_mi(csub(zk, zm)));
    Cx w;
    if (k < M) {
      w = __ldg(a.twiddles + k);
    } else {
      w.x = R(-1);
      w.y = R(0);
    }
    out[j] = cadd(e, cmul(w, o));
  }
  cluster.sync();
}

template <class R, int C>
__global__ void __launch_bounds__(512) k_forward_cluster(ForwardArgsT<R> a) {
  forward_cluster_body<C>(a, blockIdx.y);
}

// batched: items[blockIdx.y] = (run, row index)
template <class R, int C>
__global__ void __launch_bounds__(512) k_forward_cluster_b(const ForwardArgsT<R>* args, const int2* items,
                                                          const int* flags) {
  const int2 it = items[blockIdx.y];
  if (!flags[it.x]) return;
  forward_cluster_body<C>(own_args(args, it.x), it.y);
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

// A single run's rows are few, so its transforms are latency-bound: wider clusters cut each
// CTA's passes but add cluster barriers and DSMEM gathers.  Measured on config 2's rows (n_to
// 16 384, FP64, CUDA events per attempt): inverse over 1/2/4/8 CTAs 41.2/28.4/20.7/18.4 us,
// forward (which also adds the node groups' partial rows) 31.2/27.1/19.0/26.0 us.
int single_transform_width(int n_to, size_t complex_bytes, bool forward) {
  (void)complex_bytes;
  const int M = n_to / 2;
  if (M <= 2048) return 1;
  if (forward && M <= 8192) return 4;
  return kFftCluster;
}

template <class R>
static const void* single_inverse_kernel(int C) {
  switch (C) {
    case 2: return (const void*)k_inverse_cluster<R, 2>;
    case 4: return (const void*)k_inverse_cluster<R, 4>;
    case 8: return (const void*)k_inverse_cluster<R, 8>;
    default: return nullptr;
  }
}
template <class R>
static const void* single_forward_kernel(int C) {
  switch (C) {
    case 2: return (const void*)k_forward_cluster<R, 2>;
    case 4: return (const void*)k_forward_cluster<R, 4>;
    case 8: return (const void*)k_forward_cluster<R, 8>;
    default: return nullptr;
  }
}

template <class R>
cudaError_t launch_inverse_cluster(const InverseArgsT<R>& a, int n_cols, int C, cudaStream_t stream) {
  const void* kernel = single_inverse_kernel<R>(C);
  if (!kernel) return cudaErrorInvalidValue;
  const int Mp = (a.n_to / 2) / C;
  InverseArgsT<R> copy = a;
  void* args[] = {&copy};
  return launch_cluster(kernel, dim3(C, n_cols), Mp >= 512 ? 512 : Mp, (size_t)Mp * sizeof(cplx<R>), C,
                        stream, args);
}

template <class R>
cudaError_t launch_forward_cluster(const ForwardArgsT<R>& a, int n_rows, int C, cudaStream_t stream) {
  const void* kernel = single_forward_kernel<R>(C);
  if (!kernel) return cudaErrorInvalidValue;
  const int Mp = (a.n_to / 2) / C;
  ForwardArgsT<R> copy = a;
  void* args[] = {&copy};
  return launch_cluster(kernel, dim3(C, n_rows), Mp >= 512 ? 512 : Mp, (size_t)2 * Mp * sizeof(cplx<R>), C,
                        stream, args);
}

template <class R>
static const void* inverse_cluster_kernel(int C) {
  switch (C) {
    case 2: return (const void*)k_inverse_cluster_b<R, 2>;
    case 4: return (const void*)k_inverse_cluster_b<R, 4>;
    case 8: return (const void*)k_inverse_cluster_b<R, 8>;
    default: return nullptr;
  }
}
template <class R>
static const void* forward_cluster_kernel(int C) {
  switch (C) {
    case 2: return (const void*)k_forward_cluster_b<R, 2>;
    case 4: return (const void*)k_forward_cluster_b<R, 4>;
    case 8: return (const void*)k_forward_cluster_b<R, 8>;
    default: return nullptr;
  }
}

size_t cluster_transform_smem(int n_to, int C, size_t complex_bytes, bool forward) {
  return (size_t)(forward ? 2 : 1) * (size_t)(n_to / 2 / C) * complex_bytes;
}

template <class R>
cudaError_t launch_inverse_cluster_b(const InverseArgsT<R>* args, const int2* items, const int* flags,
                                     int n_items, int n_to, int C, cudaStream_t stream) {
  const void* kernel = inverse_cluster_kernel<R>(C);
  if (!kernel) return cudaErrorInvalidValue;
  const int Mp = (n_to / 2) / C;
  void* params[] = {(void*)&args, (void*)&items, (void*)&flags};
  return launch_cluster(kernel, dim3(C, n_items), Mp >= 512 ? 512 : Mp,
                        cluster_transform_smem(n_to, C, sizeof(cplx<R>), false), C, stream, params);
}

template <class R>
cudaError_t launch_forward_cluster_b(const ForwardArgsT<R>* args, const int2* items, const int* flags,
                                     int n_items, int n_to, int C, cudaStream_t stream) {
  const void* kernel = forward_cluster_kernel<R>(C);
  if (!kernel) return cudaErrorInvalidValue;
  const int Mp = (n_to / 2) / C;
  void* params[] = {(void*)&args, (void*)&items, (void*)&flags};
  return launch_cluster(kernel, dim3(C, n_items), Mp >= 512 ? 512 : Mp,
                        cluster_transform_smem(n_to, C, sizeof(cplx<R>), true), C, stream, params);
}

#define SP_CLUSTER_INSTANCES(R)                                                                      \
  template cudaError_t launch_inverse_cluster<R>(const InverseArgsT<R>&, int, int, cudaStream_t);    \
  template cudaError_t launch_forward_cluster<R>(const ForwardArgsT<R>&, int, int, cudaStream_t);    \
  template cudaError_t launch_inverse_cluster_b<R>(const InverseArgsT<R>*, const int2*, const int*, \
                                                   int, int, int, cudaStream_t);                     \
  template cudaError_t launch_forward_cluster_b<R>(const ForwardArgsT<R>*, const int2*, const int*, \
                                                   int, int, int, cudaStream_t);
SP_CLUSTER_INSTANCES(double)
SP_CLUSTER_INSTANCES(float)
#undef SP_CLUSTER_INSTANCES

cudaError_t configure_cluster_fft() {
  // single-run and batched kernels of every width: rows of up to kClusterSmem per CTA
  for (int C : {2, 4, 8}) {
    for (const void* k : {single_inverse_kernel<double>(C), single_forward_kernel<double>(C),
                          single_inverse_kernel<float>(C), single_forward_kernel<float>(C),
                          inverse_cluster_kernel<double>(C), forward_cluster_kernel<double>(C),
                          inverse_cluster_kernel<float>(C), forward_cluster_kernel<float>(C)}) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClusterSmem);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

}  // namespace sp
