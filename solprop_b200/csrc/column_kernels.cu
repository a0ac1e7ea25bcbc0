// The response column of the field-plasma route as three tiled passes, fused with the
// projection (passes 3-5 of docs/dev/architecture.md section 8: synthesis, the fused
// response, projection; backends/numpy_ref/passes/plasma.py:59-323, responses.py:678-819,
// transforms.py:87-187; nonlinear/ionisation.py:410-675 for the band rule).
//
// A tile is kSeg fine samples of a group of kGroup quadrature nodes, one CTA of 256
// threads: 16 threads per node, each owning kSeg/16 consecutive samples.  The two
// running integrals (the exposure int W dt and the free current int f E dt) are split
// the way the reference's native device scan splits them -- tile totals, then a rescan
// of every tile from its offset (native trial_response.inc:597-700):
//   pass 0  exposure increments of each tile, summed;
//   pass 1  offset = the predecessors' sums in tile order, exposure rescanned, fraction,
//           current increments summed;
//   pass 2  both rescans, the total current, the Kerr cubic, the temporal collar, and the
//           tile projected onto the modes (partial sums per node group).
// Each pass recomputes the synthesis and the rate on its tile and a halo of 2K + 1
// samples, staging the modal field in shared memory first.  Every sum has a fixed order,
// so the results are reproducible bit for bit.
#include "kernels.cuh"

namespace sp {

namespace {

constexpr int kLen = kSeg + 4 * kHalo + 2;  // local samples: [t0 - 2H - 1, t1 + 2H + 1)
constexpr int kThreads = 256;
constexpr int kLanes = kThreads / kGroup;    // threads per node (16)
constexpr int kPer = kSeg / kLanes;          // samples of the tile per thread (4)
constexpr int kI0 = 2 * kHalo + 1;           // local index of t0
constexpr size_t kRowBytes = sizeof(double) * kGroup * kLen;
constexpr size_t kModalBytes = sizeof(double) * kMaxModes * kLen;
constexpr size_t kPass0Smem = 3 * kRowBytes + kModalBytes;
constexpr size_t kPass1Smem = 4 * kRowBytes + kModalBytes;
constexpr size_t kPass2Smem = 5 * kRowBytes + kModalBytes;

struct Tile {
  int t0, n0, nodes, tile;
  int node, lane;  // this thread's node within the group (thread / kLanes) and lane
};

__device__ __forceinline__ Tile tile_of(const ColumnTileArgs& a, int tile, int group) {
  Tile c;
  c.tile = tile;
  c.t0 = tile * kSeg;
  c.n0 = group * kGroup;
  c.nodes = min(kGroup, a.n_nodes - c.n0);
  c.node = threadIdx.x / kLanes;
  c.lane = threadIdx.x % kLanes;
  return c;
}

__device__ __forceinline__ int local_of(int t, int t0) { return t - t0 + kI0; }

__device__ __forceinline__ double rate_of(const ColumnTileArgs& a, double magnitude) {
  if (magnitude > a.field_max) return a.rate_max;
  if (!(magnitude >= a.field_min)) return 0.0;
  const double lf = log(magnitude);
  long idx = (long)((lf - a.log_field_min) / a.d_log_field);
  if (idx < 0) idx = 0;
  if (idx > a.rate_intervals - 1) idx = a.rate_intervals - 1;
  const double local = lf - (a.log_field_min + (double)idx * a.d_log_field);
  const double* c = a.rate_coefficients;
  const int n = a.rate_intervals;
  return exp(((c[idx] * local + c[n + idx]) * local + c[2 * n + idx]) * local + c[3 * n + idx]);
}

// Stage the modal field a[m][t] for the tile's local range, then synthesise E and the
// rate W on local indices [lo, hi) of every node (each thread: its node, every 16th).
__device__ void field_and_rate(const ColumnTileArgs& a, const Tile& c, double* modal, double* E,
                               double* W, int lo, int hi, bool need_rate) {
  const int base = c.t0 - kI0;
  for (int m = 0; m < a.n_modes; ++m) {
    for (int i = threadIdx.x; i < kLen; i += blockDim.x) {
      const int t = base + i;
      modal[m * kLen + i] = (t >= 0 && t < a.n_to) ? a.modal_t[(size_t)m * a.n_to + t] : 0.0;
    }
  }
  __syncthreads();
  if (c.node < c.nodes) {
    const double tau = a.stage->taper;
    double srow[kMaxModes];
    const double* sp = a.synthesis + (c.n0 + c.node) * a.n_modes;
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m) srow[m] = m < a.n_modes ? sp[m] * tau : 0.0;
    double* e_row = E + c.node * kLen;
    double* w_row = W + c.node * kLen;
    for (int i = lo + c.lane; i < hi; i += kLanes) {
      double e = 0.0;
#pragma unroll
      for (int m = 0; m < kMaxModes; ++m)
        if (m < a.n_modes) e += srow[m] * modal[m * kLen + i];
      e_row[i] = e;
      if (need_rate) {
        const int t = base + i;
        w_row[i] = (t >= 0 && t < a.n_to) ? rate_of(a, fabs(e)) : 0.0;
      }
    }
  }
  __syncthreads();
}

// point reflection at the row's ends: y[-m] = 2 y[0] - y[m], y[N-1+m] = 2 y[N-1] - y[N-1-m]
__device__ __forceinline__ double reflected(const double* y, int t, int t0, int n_to) {
  if (t < 0) return 2.0 * y[local_of(0, t0)] - y[local_of(-t, t0)];
  if (t > n_to - 1) {
    const int m = t - (n_to - 1);
    return 2.0 * y[local_of(n_to - 1, t0)] - y[local_of(n_to - 1 - m, t0)];
  }
  return y[local_of(t, t0)];
}

// filtered value c0 y[t] + sum_k c_k (y[t-k] + y[t+k]), centre first, pairs in k order
__device__ __forceinline__ double filtered(const ColumnTileArgs& a, const double* y, int t, int t0) {
  const double* c = a.taps;
  const bool inside = t - a.half_width >= 0 && t + a.half_width <= a.n_to - 1;
  if (inside) {
    const double* p = y + local_of(t, t0);
    double f = c[0] * p[0];
    for (int k = 1; k <= a.half_width; ++k) f = f + c[k] * (p[-k] + p[k]);
    return f;
  }
  double f = c[0] * reflected(y, t, t0, a.n_to);
  for (int k = 1; k <= a.half_width; ++k)
    f = f + c[k] * (reflected(y, t - k, t0, a.n_to) + reflected(y, t + k, t0, a.n_to));
  return f;
}

// inc[t] = dt (y~[t] + y~[t+1]) / 2 for t in [lo, hi) (zero at the last sample and outside);
// ytil is scratch for y~ on [lo, hi].  Positions are global samples.
__device__ void increments(const ColumnTileArgs& a, const Tile& c, const double* y, double* ytil,
                           double* inc, int lo, int hi) {
  if (c.node < c.nodes) {
    const double* y_row = y + c.node * kLen;
    double* yt = ytil + c.node * kLen;
    for (int t = lo + c.lane; t <= hi; t += kLanes)
      if (t >= 0 && t < a.n_to) yt[local_of(t, c.t0)] = filtered(a, y_row, t, c.t0);
  }
  __syncthreads();
  if (c.node < c.nodes) {
    const double* yt = ytil + c.node * kLen;
    double* o = inc + c.node * kLen;
    const int last = a.n_to - 1;
    for (int i = c.lane; i < kLen; i += kLanes) {
      const int t = c.t0 - kI0 + i;
      double v = 0.0;
      if (t >= lo && t < hi && t >= 0 && t < last) v = a.dt * (yt[i + 1] + yt[i]) / 2.0;
      o[i] = v;
    }
  }
  __syncthreads();
}

// inclusive scan across the kLanes threads of one node (a half warp), fixed order
__device__ __forceinline__ double lanes_scan(double v, int lane) {
#pragma unroll
  for (int d = 1; d < kLanes; d <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, v, d, kLanes);
    if (lane >= d) v += y;
  }
  return v;
}

__device__ __forceinline__ double lanes_total(double v) {
#pragma unroll
  for (int d = kLanes / 2; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d, kLanes);
  return v;
}

// The tile's sum of increments over [t0, t1), per node; lane 0 writes it.
__device__ void tile_sum(const Tile& c, const double* inc, double* out, int n_tiles) {
  double s = 0.0;
  const double* in = inc + c.node * kLen + kI0 + c.lane * kPer;
#pragma unroll
  for (int q = 0; q < kPer; ++q) s += in[q];
  s = lanes_total(s);
  if (c.lane == 0 && c.node < c.nodes) out[(size_t)(c.n0 + c.node) * n_tiles + c.tile] = s;
}

// The sum of the predecessors' tile sums of this thread's node, in a fixed order: lane l
// adds tiles l, l + kLanes, ... below the tile, then the lanes are added as a tree.
__device__ double predecessors(const Tile& c, const double* sums, int n_tiles) {
  double s = 0.0;
  if (c.node < c.nodes) {
    const double* row = sums + (size_t)(c.n0 + c.node) * n_tiles;
    int k = c.lane;
    // four loads in flight, added in tile order
    for (; k + 3 * kLanes < c.tile; k += 4 * kLanes) {
      const double v0 = row[k], v1 = row[k + kLanes], v2 = row[k + 2 * kLanes],
                   v3 = row[k + 3 * kLanes];
      s += v0;
      s += v1;
      s += v2;
      s += v3;
    }
    for (; k < c.tile; k += kLanes) s += row[k];
  }
  return lanes_total(s);
}

// The running integral on [t0 - H, t1 + H] of this thread's node, into out: the
// increments on [t0 - H, t1 + H) scanned across the node's lanes, anchored so that
// out[t0] = offset.  Each lane scans 5 consecutive samples (kSeg + 2H = 80 = 16 x 5).
__device__ void rescan(const Tile& c, const double* inc, double* out, double offset) {
  constexpr int kSpan = kSeg + 2 * kHalo;
  constexpr int kEach = kSpan / kLanes;
  static_assert(kSpan % kLanes == 0, "rescan span");
  const int n = c.node;
  const int first = kI0 - kHalo + c.lane * kEach;  // local index of this lane's first
  double local[kEach];
  double s = 0.0;
  if (n < c.nodes) {
#pragma unroll
    for (int q = 0; q < kEach; ++q) {
      local[q] = inc[n * kLen + first + q];
      s += local[q];
    }
  }
  const double incl = lanes_scan(s, c.lane);
  // prefix (from t0 - H) before each of this lane's samples
  double pref[kEach + 1];
  double run = incl - s;
#pragma unroll
  for (int q = 0; q < kEach; ++q) {
    pref[q] = run;
    run += local[q];
  }
  pref[kEach] = run;
  // the prefix at t0 sits in lane kHalo / kEach, element kHalo % kEach
  constexpr int kL0 = kHalo / kEach, kQ0 = kHalo % kEach;
  const double at_t0 = __shfl_sync(0xffffffffu, pref[kQ0], kL0, kLanes);
  if (n < c.nodes) {
#pragma unroll
    for (int q = 0; q < kEach; ++q) out[n * kLen + first + q] = offset + (pref[q] - at_t0);
    if (c.lane == kLanes - 1) out[n * kLen + first + kEach] = offset + (pref[kEach] - at_t0);
  }
  __syncthreads();
}

}  // namespace

// pass 0: the exposure's tile sums
__device__ __forceinline__ void pass0_body(const ColumnTileArgs& a, int tile, int group) {
  extern __shared__ double dyn0[];
  double* E = dyn0;
  double* W = E + kGroup * kLen;
  double* T = W + kGroup * kLen;
  double* modal = T + kGroup * kLen;
  const Tile c = tile_of(a, tile, group);
  // W~ on [t0, t1] needs W on [t0 - H, t1 + H]
  field_and_rate(a, c, modal, E, W, kI0 - kHalo, kI0 + kSeg + kHalo + 1, true);
  increments(a, c, W, T, E, c.t0, c.t0 + kSeg);
  tile_sum(c, E, a.sums0, a.n_tiles);
}

// pass 1: the exposure rescanned, the fraction, the current's tile sums
__device__ __forceinline__ void pass1_body(const ColumnTileArgs& a, int tile, int group) {
  extern __shared__ double dyn1[];
  double* E = dyn1;
  double* W = E + kGroup * kLen;
  double* T = W + kGroup * kLen;
  double* S = T + kGroup * kLen;
  double* modal = S + kGroup * kLen;
  const Tile c = tile_of(a, tile, group);
  const double off0 = predecessors(c, a.sums0, a.n_tiles);
  if (c.lane == 0 && c.node < c.nodes) a.offsets0[(size_t)(c.n0 + c.node) * a.n_tiles + c.tile] = off0;
  field_and_rate(a, c, modal, E, W, 0, kLen, true);
  increments(a, c, W, T, S, c.t0 - kHalo, c.t0 + kSeg + kHalo);
  rescan(c, S, T, off0);  // T = exposure on [t0 - H, t1 + H]
  const double f0 = a.stage->preionisation;
  if (c.node < c.nodes) {
    for (int i = c.lane; i < kLen; i += kLanes) {
      const int idx = c.node * kLen + i;
      const int t = c.t0 - kI0 + i;
      double g = 0.0;
      if (t >= c.t0 - kHalo && t <= c.t0 + kSeg + kHalo && t >= 0 && t < a.n_to) {
        const double x = a.band ? fmax(T[idx], 0.0) : T[idx];
        const double f = 1.0 - (1.0 - f0) * (x == 0.0 ? 1.0 : exp(-x));
        g = f * a.charge_mass_ratio * E[idx];
      }
      W[idx] = g;  // the current's integrand
    }
  }
  __syncthreads();
  increments(a, c, W, T, S, c.t0, c.t0 + kSeg);
  tile_sum(c, S, a.sums1, a.n_tiles);
}

// pass 2: both rescans, the total current, Kerr, the collar and the projection
__device__ __forceinline__ void pass2_body(const ColumnTileArgs& a, int tile, int group) {
  extern __shared__ double dyn2[];
  double* E = dyn2;
  double* W = E + kGroup * kLen;
  double* F = W + kGroup * kLen;   // exposure, then the fraction in place
  double* Y1 = F + kGroup * kLen;  // integrand -> increments
  double* Y2 = Y1 + kGroup * kLen; // filtered scratch -> running integral
  double* modal = Y2 + kGroup * kLen;
  const Tile c = tile_of(a, tile, group);
  const bool plasma = a.plasma;
  double off1 = 0.0, off0 = 0.0;
  if (plasma) {
    off1 = predecessors(c, a.sums1, a.n_tiles);
    if (c.node < c.nodes) off0 = a.offsets0[(size_t)(c.n0 + c.node) * a.n_tiles + c.tile];
  }
  field_and_rate(a, c, modal, E, W, plasma ? 0 : kI0, plasma ? kLen : kI0 + kSeg, plasma);
  if (plasma) {
    increments(a, c, W, Y2, Y1, c.t0 - kHalo, c.t0 + kSeg + kHalo);
    rescan(c, Y1, F, off0);  // F = exposure
    const double f0 = a.stage->preionisation;
    if (c.node < c.nodes) {
      for (int i = c.lane; i < kLen; i += kLanes) {
        const int idx = c.node * kLen + i;
        const int t = c.t0 - kI0 + i;
        double f = 0.0, g = 0.0;
        if (t >= c.t0 - kHalo && t <= c.t0 + kSeg + kHalo && t >= 0 && t < a.n_to) {
          const double x = a.band ? fmax(F[idx], 0.0) : F[idx];
          f = 1.0 - (1.0 - f0) * (x == 0.0 ? 1.0 : exp(-x));
          g = f * a.charge_mass_ratio * E[idx];
        }
        F[idx] = f;
        Y1[idx] = g;
      }
    }
    __syncthreads();
    increments(a, c, Y1, Y2, Y1, c.t0, c.t0 + kSeg);  // Y1: the current's increments
    rescan(c, Y1, Y2, off1);                          // Y2: free current per unit density
  }
  // outputs on [t0, t1): P = (c rho E^2 E) g, X = g rho J, Z = g' rho J
  const StageScalarsDev& st = *a.stage;
  const double factor = a.kerr ? a.kerr_coefficient * st.kerr_density : 0.0;
  const double rho = st.plasma_density;
  double outp[kPer], outx[kPer], outz[kPer];
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int q = c.lane * kPer + k;
    const int li = c.node * kLen + kI0 + q;
    const int t = c.t0 + q;
    double p = 0.0, x = 0.0, z = 0.0;
    if (c.node < c.nodes && t < a.n_to) {
      const double e = E[li];
      const double win = a.t_window[t];
      p = (a.kerr ? factor * (e * e) * e : 0.0) * win;
      if (plasma) {
        const double w = W[li], f = F[li];
        const double squared = fabs(e) * fabs(e);
        double scale = 0.0;
        if (w > 0.0 && squared > 0.0) scale = a.ionisation_potential * w * (1.0 - f) / squared;
        const double current = rho * (Y2[li] + scale * e);
        x = win * current;
        z = a.t_window_derivative[t] * current;
      }
    }
    outp[k] = p;
    outx[k] = x;
    outz[k] = z;
  }
  __syncthreads();
  double* P = E;  // [node][kSeg] output tiles over the spent rows
  double* X = W;
  double* Z = F;
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int o = c.node * kSeg + c.lane * kPer + k;
    P[o] = outp[k];
    X[o] = outx[k];
    Z[o] = outz[k];
  }
  __syncthreads();
  // projection of the tile onto the modes: sum over the group's nodes in node order
  const double tau = st.taper;
  const int n_streams = plasma ? 3 : 1;
  const double* rows[3] = {P, X, Z};
  // weights W[m, node] / tau of the group, once
  __shared__ double wt[kMaxModes * kGroup];
  for (int k = threadIdx.x; k < a.n_modes * kGroup; k += blockDim.x) {
    const int m = k / kGroup, n = k % kGroup;
    wt[k] = n < c.nodes ? a.projection[m * a.n_nodes + c.n0 + n] / tau : 0.0;
  }
  __syncthreads();
  const int q = threadIdx.x % kSeg;  // sample of the tile
  const int t = c.t0 + q;
  for (int sm = threadIdx.x / kSeg; sm < n_streams * a.n_modes; sm += kThreads / kSeg) {
    const int s = sm / a.n_modes, m = sm - s * a.n_modes;
    if (t >= a.n_to) continue;
    const double* row = rows[s];
    double acc = 0.0;
    for (int n = 0; n < c.nodes; ++n) acc += wt[m * kGroup + n] * row[n * kSeg + q];
    a.partials[(((size_t)group * 3 + s) * a.n_cols + m) * a.n_to + t] = acc;
  }
}

__global__ void __launch_bounds__(kThreads) k_column_pass0(ColumnTileArgs a) {
  pass0_body(a, blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(kThreads) k_column_pass1(ColumnTileArgs a) {
  pass1_body(a, blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(kThreads) k_column_pass2(ColumnTileArgs a) {
  pass2_body(a, blockIdx.x, blockIdx.y);
}
// batched: items[blockIdx.x] = (run, tile, group, -)
__global__ void __launch_bounds__(kThreads) k_column_pass0_b(const ColumnTileArgs* args, const int4* items,
                                                                const int* flags) {
  const int4 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  pass0_body(args[it.x], it.y, it.z);
}
__global__ void __launch_bounds__(kThreads) k_column_pass1_b(const ColumnTileArgs* args, const int4* items,
                                                                const int* flags) {
  const int4 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  pass1_body(args[it.x], it.y, it.z);
}
__global__ void __launch_bounds__(kThreads) k_column_pass2_b(const ColumnTileArgs* args, const int4* items,
                                                                const int* flags) {
  const int4 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  pass2_body(args[it.x], it.y, it.z);
}

cudaError_t launch_column_tiled_b(const ColumnTileArgs* args, const int4* items, const int* flags,
                                  int n_items, int pass, cudaStream_t stream) {
  if (pass == 0) k_column_pass0_b<<<n_items, kThreads, kPass0Smem, stream>>>(args, items, flags);
  else if (pass == 1) k_column_pass1_b<<<n_items, kThreads, kPass1Smem, stream>>>(args, items, flags);
  else k_column_pass2_b<<<n_items, kThreads, kPass2Smem, stream>>>(args, items, flags);
  return cudaGetLastError();
}

cudaError_t launch_column_tiled(const ColumnTileArgs& a, cudaStream_t stream) {
  const dim3 grid(a.n_tiles, a.n_groups);
  if (a.plasma) {
    k_column_pass0<<<grid, kThreads, kPass0Smem, stream>>>(a);
    k_column_pass1<<<grid, kThreads, kPass1Smem, stream>>>(a);
  }
  k_column_pass2<<<grid, kThreads, kPass2Smem, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t configure_column_kernels() {
  const void* kernels[6] = {(const void*)k_column_pass0, (const void*)k_column_pass1,
                            (const void*)k_column_pass2, (const void*)k_column_pass0_b,
                            (const void*)k_column_pass1_b, (const void*)k_column_pass2_b};
  const size_t shm[6] = {kPass0Smem, kPass1Smem, kPass2Smem, kPass0Smem, kPass1Smem, kPass2Smem};
  for (int i = 0; i < 6; ++i) {
    cudaError_t e = cudaFuncSetAttribute(kernels[i], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)shm[i]);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace sp
