// The response column of the field-plasma route in one launch, fused with the
// projection (passes 3-5 of docs/dev/architecture.md section 8: synthesis, the fused
// response, projection; backends/numpy_ref/passes/plasma.py:59-323, responses.py:678-819,
// transforms.py:87-187; nonlinear/ionisation.py:410-675 for the band rule).
//
// A tile is kSeg fine samples of a group of kGroup quadrature nodes, one CTA of 256
// threads: 16 threads per node, each owning kSeg/16 consecutive samples.  The two
// running integrals (the exposure int W dt and the free current int f E dt) are split
// the way the reference's native device scan splits them -- tile totals, then every tile
// rescanned from its offset (native trial_response.inc:597-700) -- but in a single pass:
// a tile publishes its exposure sum, adds its predecessors' sums (in a fixed order) once
// they are published, rescans, publishes its current sum the same way, and goes on to the
// total current, the Kerr cubic, the temporal collar and the projection onto the modes
// (partial sums per node group).  The synthesis and the rate are computed once per tile
// and its halo of 2K + 1 samples, from the modal field staged in shared memory.  Every
// sum has a fixed order, so the results are reproducible bit for bit.
#include "kernels.cuh"

namespace sp {

namespace {

constexpr int kLen = kSeg + 4 * kHalo + 2;  // local samples: [t0 - 2H - 1, t1 + 2H + 1)
constexpr int kThreads = 256;
constexpr int kLanes = kThreads / kGroup;    // threads per node (16)
constexpr int kPer = kSeg / kLanes;          // samples of the tile per thread (4)
constexpr int kI0 = 2 * kHalo + 1;           // local index of t0
// dynamic shared memory of one tile: five node rows and the staged modal field
template <class R>
constexpr size_t chain_smem() {
  return sizeof(R) * (5 * kGroup * kLen + kMaxModes * kLen);
}

struct Tile {
  int t0, n0, nodes, tile;
  int node, lane;  // this thread's node within the group (thread / kLanes) and lane
};

template <class R>
__device__ __forceinline__ Tile tile_of(const ColumnArgsT<R>& a, int tile, int group) {
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

__device__ __forceinline__ double rate_of(const ColumnArgsT<double>& a, double magnitude) {
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

// The same lookup in FP32.  Its table is (c0, c1, c2, exp c3, 1 / knot) per interval, the
// knot being the field at the interval's start, so that W = exp(c3) exp(((c0 l + c1) l +
// c2) l) with l = log1p(|E| / knot - 1): no large logarithm or exponent is rounded to
// FP32, and the error of W is that of |E| times the rate's slope d log W / d log |E|.
__device__ __forceinline__ float rate_of(const ColumnArgsT<float>& a, float magnitude) {
  if (magnitude > (float)a.field_max) return (float)a.rate_max;
  if (!(magnitude >= (float)a.field_min)) return 0.0f;
  const int n = a.rate_intervals;
  const float pos = (__logf(magnitude) - (float)a.log_field_min) * (float)(1.0 / a.d_log_field);
  int idx = (int)pos;
  if (idx < 0) idx = 0;
  if (idx > n - 1) idx = n - 1;
  const float* c = a.rate_coefficients;
  const float local = log1pf(fmaf(magnitude, c[4 * n + idx], -1.0f));
  return c[3 * n + idx] * expf(((c[idx] * local + c[n + idx]) * local + c[2 * n + idx]) * local);
}

// Stage the modal field a[m][t] for the tile's local range, then synthesise E and the
// rate W on local indices [lo, hi) of every node (each thread: its node, every 16th).
template <class R>
__device__ void field_and_rate(const ColumnArgsT<R>& a, const Tile& c, R* modal, R* E, R* W, int lo,
                               int hi, bool need_rate) {
  const int base = c.t0 - kI0;
  for (int m = 0; m < a.n_modes; ++m) {
    for (int i = threadIdx.x; i < kLen; i += blockDim.x) {
      const int t = base + i;
      modal[m * kLen + i] = (t >= 0 && t < a.n_to) ? R(a.modal_t[(size_t)m * a.n_to + t]) : R(0);
    }
  }
  __syncthreads();
  if (c.node < c.nodes) {
    const R tau = R(a.stage->taper);
    R srow[kMaxModes];
    const R* sp = a.synthesis + (c.n0 + c.node) * a.n_modes;
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m) srow[m] = m < a.n_modes ? sp[m] * tau : R(0);
    R* e_row = E + c.node * kLen;
    R* w_row = W + c.node * kLen;
    for (int i = lo + c.lane; i < hi; i += kLanes) {
      R e = R(0);
#pragma unroll
      for (int m = 0; m < kMaxModes; ++m)
        if (m < a.n_modes) e += srow[m] * modal[m * kLen + i];
      e_row[i] = e;
      if (need_rate) {
        const int t = base + i;
        w_row[i] = (t >= 0 && t < a.n_to) ? rate_of(a, fabs(e)) : R(0);
      }
    }
  }
  __syncthreads();
}

// point reflection at the row's ends: y[-m] = 2 y[0] - y[m], y[N-1+m] = 2 y[N-1] - y[N-1-m]
template <class R>
__device__ __forceinline__ R reflected(const R* y, int t, int t0, int n_to) {
  if (t < 0) return R(2) * y[local_of(0, t0)] - y[local_of(-t, t0)];
  if (t > n_to - 1) {
    const int m = t - (n_to - 1);
    return R(2) * y[local_of(n_to - 1, t0)] - y[local_of(n_to - 1 - m, t0)];
  }
  return y[local_of(t, t0)];
}

// filtered value c0 y[t] + sum_k c_k (y[t-k] + y[t+k]), centre first, pairs in k order
template <class R>
__device__ __forceinline__ R filtered(const ColumnArgsT<R>& a, const R* y, int t, int t0) {
  const R* c = a.taps;
  const bool inside = t - a.half_width >= 0 && t + a.half_width <= a.n_to - 1;
  if (inside) {
    const R* p = y + local_of(t, t0);
    R f = c[0] * p[0];
    for (int k = 1; k <= a.half_width; ++k) f = f + c[k] * (p[-k] + p[k]);
    return f;
  }
  R f = c[0] * reflected(y, t, t0, a.n_to);
  for (int k = 1; k <= a.half_width; ++k)
    f = f + c[k] * (reflected(y, t - k, t0, a.n_to) + reflected(y, t + k, t0, a.n_to));
  return f;
}

// inc[t] = dt (y~[t] + y~[t+1]) / 2 for t in [lo, hi) (zero at the last sample and outside);
// ytil is scratch for y~ on [lo, hi].  Positions are global samples.
template <class R>
__device__ void increments(const ColumnArgsT<R>& a, const Tile& c, const R* y, R* ytil, R* inc, int lo,
                           int hi) {
  if (c.node < c.nodes) {
    const R* y_row = y + c.node * kLen;
    R* yt = ytil + c.node * kLen;
    for (int t = lo + c.lane; t <= hi; t += kLanes)
      if (t >= 0 && t < a.n_to) yt[local_of(t, c.t0)] = filtered(a, y_row, t, c.t0);
  }
  __syncthreads();
  if (c.node < c.nodes) {
    const R* yt = ytil + c.node * kLen;
    R* o = inc + c.node * kLen;
    const int last = a.n_to - 1;
    const R dt = R(a.dt);
    for (int i = c.lane; i < kLen; i += kLanes) {
      const int t = c.t0 - kI0 + i;
      R v = R(0);
      if (t >= lo && t < hi && t >= 0 && t < last) v = dt * (yt[i + 1] + yt[i]) / R(2);
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

// The tile's sum of increments over [t0, t1), per node, in FP64; lane 0 writes it.
template <class R>
__device__ void tile_sum(const Tile& c, const R* inc, double* out, int n_tiles) {
  double s = 0.0;
  const R* in = inc + c.node * kLen + kI0 + c.lane * kPer;
#pragma unroll
  for (int q = 0; q < kPer; ++q) s += in[q];
  s = lanes_total(s);
  if (c.lane == 0 && c.node < c.nodes) out[(size_t)(c.n0 + c.node) * n_tiles + c.tile] = s;
}

// The running integral on [t0 - H, t1 + H] of this thread's node, into out: the
// increments on [t0 - H, t1 + H) scanned across the node's lanes, anchored so that
// out[t0] = offset.  Each lane scans 5 consecutive samples (kSeg + 2H = 80 = 16 x 5).
// The sums are FP64 whatever the rows' type (the mixed form's compensated integral).
template <class R>
__device__ void rescan(const Tile& c, const R* inc, R* out, double offset) {
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
    for (int q = 0; q < kEach; ++q) out[n * kLen + first + q] = R(offset + (pref[q] - at_t0));
    if (c.lane == kLanes - 1) out[n * kLen + first + kEach] = R(offset + (pref[kEach] - at_t0));
  }
  __syncthreads();
}

// ---- tile order and the hand-over between tiles
// Every CTA takes a ticket from the workspace's counter; tickets are handed out in tile
// order (tile-major, node group minor), so a CTA only ever waits on tiles whose CTAs took
// their tickets earlier and are therefore resident: the waits always end.  A launch takes
// exactly n_blocks tickets, so ticket / n_blocks numbers the evaluation (its epoch) and the
// ready flags need no reset: a tile's flag reads 2 e + 1 once its exposure sums of
// evaluation e are published and 2 e + 2 once its current sums are.
constexpr long kSpinLimit = 1L << 20;  // polls of one flag before the wait gives up

__device__ __forceinline__ int load_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void store_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// publish this tile's sums (already written by the nodes' lane 0) as stage `target`
template <class R>
__device__ __forceinline__ void publish(const ColumnArgsT<R>& a, const Tile& c, int group, int target) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) store_release(a.flags + (size_t)group * a.n_tiles + c.tile, target);
}

// wait until every earlier tile of the group has published stage `target`; a wait that
// gives up marks the evaluation failed in *status (read by the host) and goes on
template <class R>
__device__ __forceinline__ void await_predecessors(const ColumnArgsT<R>& a, const Tile& c, int group,
                                                   int target) {
  const int* f = a.flags + (size_t)group * a.n_tiles;
  for (int j = threadIdx.x; j < c.tile; j += blockDim.x) {
    long polls = 0;
    while (load_acquire(f + j) < target) {
      if (++polls > kSpinLimit) {
        *a.status = 1.0;
        break;
      }
      __nanosleep(64);
    }
  }
  __threadfence();
  __syncthreads();
}

// the predecessors' sums, read past L1 (other CTAs wrote them during this launch)
__device__ double predecessors_cg(const Tile& c, const double* sums, int n_tiles) {
  double s = 0.0;
  if (c.node < c.nodes) {
    const double* row = sums + (size_t)(c.n0 + c.node) * n_tiles;
    int k = c.lane;
    for (; k + 3 * kLanes < c.tile; k += 4 * kLanes) {
      const double v0 = __ldcg(row + k), v1 = __ldcg(row + k + kLanes),
                   v2 = __ldcg(row + k + 2 * kLanes), v3 = __ldcg(row + k + 3 * kLanes);
      s += v0;
      s += v1;
      s += v2;
      s += v3;
    }
    for (; k < c.tile; k += kLanes) s += __ldcg(row + k);
  }
  return lanes_total(s);
}

// the ionised fraction f = 1 - (1 - f0) e^-x (plasma.py:104-191); in FP32 as
// f0 + (1 - f0)(1 - e^-x) through expm1, which keeps its relative accuracy for small x
__device__ __forceinline__ double fraction(double f0, double x) {
  return 1.0 - (1.0 - f0) * (x == 0.0 ? 1.0 : exp(-x));
}
__device__ __forceinline__ float fraction(float f0, float x) {
  return fmaf(1.0f - f0, -expm1f(-x), f0);
}

}  // namespace

// One tile of the column, start to finish: synthesis and rate on the tile and its halo,
// the exposure's increments and tile sum (published), the exposure from the
// predecessors' sums, the fraction and the current's increments and tile sum (published),
// the current from the predecessors' sums, then the total current, Kerr, the collar and
// the tile projected onto the modes (partial sums per node group).
template <class R>
__device__ __forceinline__ void chain_body(const ColumnArgsT<R>& a) {
  extern __shared__ __align__(16) unsigned char dyn_raw[];
  R* E = reinterpret_cast<R*>(dyn_raw);
  R* W = E + kGroup * kLen;
  R* F = W + kGroup * kLen;   // exposure, then the fraction in place
  R* Y1 = F + kGroup * kLen;  // increments
  R* Y2 = Y1 + kGroup * kLen; // filtered scratch -> running integral
  R* modal = Y2 + kGroup * kLen;
  __shared__ unsigned long long ticket;
  if (threadIdx.x == 0) ticket = atomicAdd(a.ticket, 1ull);
  __syncthreads();
  const unsigned long long epoch = ticket / (unsigned long long)a.n_blocks;
  const int index = (int)(ticket % (unsigned long long)a.n_blocks);
  const int tile = index / a.n_groups, group = index % a.n_groups;
  const Tile c = tile_of(a, tile, group);
  const bool plasma = a.plasma;
  field_and_rate(a, c, modal, E, W, plasma ? 0 : kI0, plasma ? kLen : kI0 + kSeg, plasma);
  if (plasma) {
    const int first = (int)(2 * epoch + 1);
    // exposure increments on [t0 - H, t1 + H) into Y1; the tile's own sum is published
    increments(a, c, W, Y2, Y1, c.t0 - kHalo, c.t0 + kSeg + kHalo);
    tile_sum(c, Y1, a.sums0, a.n_tiles);
    publish(a, c, group, first);
    await_predecessors(a, c, group, first);
    const double off0 = predecessors_cg(c, a.sums0, a.n_tiles);
    rescan(c, Y1, F, off0);  // F = exposure on [t0 - H, t1 + H]
    const R f0 = R(a.stage->preionisation);
    const R qm = R(a.charge_mass_ratio);
    if (c.node < c.nodes) {
      for (int i = c.lane; i < kLen; i += kLanes) {
        const int idx = c.node * kLen + i;
        const int t = c.t0 - kI0 + i;
        R f = R(0), g = R(0);
        if (t >= c.t0 - kHalo && t <= c.t0 + kSeg + kHalo && t >= 0 && t < a.n_to) {
          const R x = a.band ? fmax(F[idx], R(0)) : F[idx];
          f = fraction(f0, x);
          g = f * qm * E[idx];
        }
        F[idx] = f;
        Y1[idx] = g;
      }
    }
    __syncthreads();
    increments(a, c, Y1, Y2, Y1, c.t0, c.t0 + kSeg);  // Y1: the current's increments
    tile_sum(c, Y1, a.sums1, a.n_tiles);
    publish(a, c, group, first + 1);
    await_predecessors(a, c, group, first + 1);
    const double off1 = predecessors_cg(c, a.sums1, a.n_tiles);
    rescan(c, Y1, Y2, off1);  // Y2: free current per unit density
  }
  // outputs on [t0, t1): P = (c rho E^2 E) g, X = g rho J, Z = g' rho J
  const StageScalarsDev& st = *a.stage;
  const R factor = R(a.kerr ? a.kerr_coefficient * st.kerr_density : 0.0);
  const R rho = R(st.plasma_density);
  const R ip = R(a.ionisation_potential);
  R outp[kPer], outx[kPer], outz[kPer];
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int q = c.lane * kPer + k;
    const int li = c.node * kLen + kI0 + q;
    const int t = c.t0 + q;
    R p = R(0), x = R(0), z = R(0);
    if (c.node < c.nodes && t < a.n_to) {
      const R e = E[li];
      const R win = a.t_window[t];
      p = (a.kerr ? factor * (e * e) * e : R(0)) * win;
      if (plasma) {
        const R w = W[li], f = F[li];
        const R squared = fabs(e) * fabs(e);
        R scale = R(0);
        if (w > R(0) && squared > R(0)) scale = ip * w * (R(1) - f) / squared;
        const R current = rho * (Y2[li] + scale * e);
        x = win * current;
        z = a.t_window_derivative[t] * current;
      }
    }
    outp[k] = p;
    outx[k] = x;
    outz[k] = z;
  }
  __syncthreads();
  R* P = E;  // [node][kSeg] output tiles over the spent rows
  R* X = W;
  R* Z = F;
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int o = c.node * kSeg + c.lane * kPer + k;
    P[o] = outp[k];
    X[o] = outx[k];
    Z[o] = outz[k];
  }
  __syncthreads();
  // projection of the tile onto the modes: sum over the group's nodes in node order
  const R tau = R(st.taper);
  const int n_streams = plasma ? 3 : 1;
  const R* rows[3] = {P, X, Z};
  // weights W[m, node] / tau of the group, once
  __shared__ R wt[kMaxModes * kGroup];
  for (int k = threadIdx.x; k < a.n_modes * kGroup; k += blockDim.x) {
    const int m = k / kGroup, n = k % kGroup;
    wt[k] = n < c.nodes ? a.projection[m * a.n_nodes + c.n0 + n] / tau : R(0);
  }
  __syncthreads();
  const int q = threadIdx.x % kSeg;  // sample of the tile
  const int t = c.t0 + q;
  for (int sm = threadIdx.x / kSeg; sm < n_streams * a.n_modes; sm += kThreads / kSeg) {
    const int s = sm / a.n_modes, m = sm - s * a.n_modes;
    if (t >= a.n_to) continue;
    const R* row = rows[s];
    R acc = R(0);
    for (int n = 0; n < c.nodes; ++n) acc += wt[m * kGroup + n] * row[n * kSeg + q];
    a.partials[(((size_t)group * 3 + s) * a.n_cols + m) * a.n_to + t] = acc;
  }
}

template <class R>
__global__ void __launch_bounds__(kThreads, 3) k_column(ColumnArgsT<R> a) { chain_body(a); }

// batched: items[blockIdx.x].x = the run; a run's CTAs take their tiles from its counter
template <class R>
__global__ void __launch_bounds__(kThreads, 3) k_column_b(const ColumnArgsT<R>* args, const int4* items,
                                                          const int* flags) {
  const int run = items[blockIdx.x].x;
  if (!flags[run]) return;  // every CTA of an idle run leaves before its ticket
  chain_body(args[run]);
}

template <class R>
cudaError_t launch_column_b(const ColumnArgsT<R>* args, const int4* items, const int* flags,
                            int n_items, cudaStream_t stream) {
  k_column_b<R><<<n_items, kThreads, chain_smem<R>(), stream>>>(args, items, flags);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_column(const ColumnArgsT<R>& a, cudaStream_t stream) {
  k_column<R><<<a.n_blocks, kThreads, chain_smem<R>(), stream>>>(a);
  return cudaGetLastError();
}

template cudaError_t launch_column<double>(const ColumnArgsT<double>&, cudaStream_t);
template cudaError_t launch_column<float>(const ColumnArgsT<float>&, cudaStream_t);
template cudaError_t launch_column_b<double>(const ColumnArgsT<double>*, const int4*, const int*, int,
                                             cudaStream_t);
template cudaError_t launch_column_b<float>(const ColumnArgsT<float>*, const int4*, const int*, int,
                                            cudaStream_t);

cudaError_t configure_column_kernels() {
  const void* kernels[4] = {(const void*)k_column<double>, (const void*)k_column_b<double>,
                            (const void*)k_column<float>, (const void*)k_column_b<float>};
  const size_t shm[4] = {chain_smem<double>(), chain_smem<double>(), chain_smem<float>(),
                         chain_smem<float>()};
  for (int i = 0; i < 4; ++i) {
    cudaError_t e = cudaFuncSetAttribute(kernels[i], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)shm[i]);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace sp
