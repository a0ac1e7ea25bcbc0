// The response column of the field-plasma route in one launch, fused with the
// projection (passes 3-5 of docs/dev/architecture.md section 8: synthesis, the fused
// response, projection; backends/numpy_ref/passes/plasma.py:59-323, responses.py:678-819,
// transforms.py:87-187; nonlinear/ionisation.py:410-675 for the band rule).
//
// One warp holds one quadrature node's window of kWindow = 256 fine samples in registers,
// eight consecutive samples per lane; a CTA is kGroup = 8 warps, eight nodes over the same
// window.  The band filter's taps reach the neighbouring lanes by shuffles, so a window
// carries a halo of A = 2K + 1 samples on each side (K the filter's half-width) and owns
// the kWindow - 2A samples between them; consecutive tiles' windows overlap by 2A.
//
// The two running integrals (the exposure int W~ dt and the free current int f E~ dt)
// are split the way the reference's native device scan splits them -- tile totals, then
// every tile rescanned from its offset (native trial_response.inc:597-700) -- in a single
// pass: a tile publishes its owned increments' sum, adds its predecessors' sums in tile
// order once they are published, and rescans its window from that offset.  The sums are
// FP64 in both precisions (the mixed form's compensated integral).  The tile then forms
// the total current, the Kerr cubic and the temporal collar, and projects the owned
// samples onto the modes (a partial row per node group, added in group order by the
// forward transform).  Every sum has a fixed order, so the results are reproducible bit for
// bit.
#include "kernels.cuh"

namespace sp {

namespace {

constexpr int kThreads = 32 * kGroup;
constexpr int kPer = kWindow / 32;  // samples per lane (8)
static_assert(kPer == 8, "the filter's halo exchange assumes eight samples per lane");
static_assert(kHalo <= kPer, "a tap may reach one neighbouring lane at most");
static_assert(3 * kGroup >= kMaxModes, "the stream buffer must cover the modal window");

// Shared rows are padded by one element after every eight (pad(u) = u + u / 8), so that
// the 32 lanes of a warp, each at its own eight-sample run, hit distinct banks.
constexpr int kPitch = kWindow + kWindow / kPer;
__device__ __forceinline__ int pad(int u) { return u + (u >> 3); }

// shared memory: the modal window (n_modes rows), later the three projected streams of
// the group (3 x kGroup rows) over the same space, and one scratch row per warp for the
// point reflection at the row's ends
template <class R>
constexpr size_t column_smem() {
  return sizeof(R) * ((size_t)3 * kGroup * kPitch + (size_t)kGroup * kPitch);
}
// the sweep adds the next tile's modal window (FP64, as in global memory) and temporal
// windows, copied in while the current tile is computed
template <class R>
constexpr size_t column_sweep_smem() {
  return column_smem<R>() + sizeof(double) * (size_t)kMaxModes * kWindow + sizeof(R) * 2 * kWindow;
}

// asynchronous global -> shared copies of 4 or 8 bytes (zero-filled when !valid, which
// reads nothing), their commit and the wait for all of this thread's copies
template <int kBytes>
__device__ __forceinline__ void copy_async(void* smem, const void* gmem, bool valid) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(dst), "l"(gmem), "n"(kBytes),
               "r"(valid ? kBytes : 0)
               : "memory");
}
__device__ __forceinline__ void copy_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void copy_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The rate table's scalars, read from the argument record once per tile into registers
// (the record lives in shared memory, where every read after a shared store is a load).
template <class R>
struct RateLookup {
  R field_min, field_max, rate_max, log_field_min, step;  // step: d log|E| (FP64), 1 / d (FP32)
  const R* c;
  int n;
};
__device__ __forceinline__ RateLookup<double> rate_lookup(const ColumnArgsT<double>& a) {
  return {a.field_min, a.field_max, a.rate_max, a.log_field_min, a.d_log_field, a.rate_coefficients,
          a.rate_intervals};
}
__device__ __forceinline__ RateLookup<float> rate_lookup(const ColumnArgsT<float>& a) {
  return {(float)a.field_min, (float)a.field_max, (float)a.rate_max, (float)a.log_field_min,
          (float)(1.0 / a.d_log_field), a.rate_coefficients, a.rate_intervals};
}

__device__ __forceinline__ RateLookup<double> rate_lookup(const ChannelTableT<double>& c) {
  return {c.field_min, c.field_max, c.rate_max, c.log_field_min, c.d_log_field, c.rate_coefficients,
          c.rate_intervals};
}
__device__ __forceinline__ RateLookup<float> rate_lookup(const ChannelTableT<float>& c) {
  return {(float)c.field_min, (float)c.field_max, (float)c.rate_max, (float)c.log_field_min,
          (float)(1.0 / c.d_log_field), c.rate_coefficients, c.rate_intervals};
}

__device__ __forceinline__ double rate_of(const RateLookup<double>& a, double magnitude) {
  if (magnitude > a.field_max) return a.rate_max;
  if (!(magnitude >= a.field_min)) return 0.0;
  const double lf = log(magnitude);
  long idx = (long)((lf - a.log_field_min) / a.step);
  if (idx < 0) idx = 0;
  if (idx > a.n - 1) idx = a.n - 1;
  const double local = lf - (a.log_field_min + (double)idx * a.step);
  const double* c = a.c;
  const int n = a.n;
  return exp(((c[idx] * local + c[n + idx]) * local + c[2 * n + idx]) * local + c[3 * n + idx]);
}

// The same lookup in FP32.  Its table is (c0, c1, c2, exp c3, 1 / knot) per interval, the
// knot being the field at the interval's start, so that W = exp(c3) exp(((c0 l + c1) l +
// c2) l) with l = log1p(|E| / knot - 1): no large logarithm or exponent is rounded to
// FP32, and the error of W is that of |E| times the rate's slope d log W / d log |E|.
__device__ __forceinline__ float rate_of(const RateLookup<float>& a, float magnitude) {
  if (magnitude > a.field_max) return a.rate_max;
  if (!(magnitude >= a.field_min)) return 0.0f;
  const int n = a.n;
  const float pos = (__logf(magnitude) - a.log_field_min) * a.step;
  int idx = (int)pos;
  if (idx < 0) idx = 0;
  if (idx > n - 1) idx = n - 1;
  const float* c = a.c;
  // l = log1p(v), v = |E| / knot - 1: within an interval |v| is a few 1e-2 at most, where
  // the series to v^5 is as good as FP32 (its first omitted term, v^6 / 6, stays below
  // 6e-8 |v|)
  const float v = fmaf(magnitude, c[4 * n + idx], -1.0f);
  float local;
  if (fabsf(v) < 0.05f)
    local = v * (1.0f + v * (-0.5f + v * (1.0f / 3.0f + v * (-0.25f + v * 0.2f))));
  else
    local = log1pf(v);
  // the exponent stays small (|l| <= the interval's width), where the fast exponential
  // keeps its relative error to a few units in the last place
  return c[3 * n + idx] * __expf(((c[idx] * local + c[n + idx]) * local + c[2 * n + idx]) * local);
}

// a / b: exact in FP64; in FP32 the fast reciprocal-based division (2 ulp), for b far
// below 2^126 (here |E|^2)
__device__ __forceinline__ double divide(double a, double b) { return a / b; }
__device__ __forceinline__ float divide(float a, float b) { return __fdividef(a, b); }

// the ionised fraction f = 1 - (1 - f0) e^-x (plasma.py:104-191); in FP32 as
// f0 + (1 - f0)(1 - e^-x) through expm1, which keeps its relative accuracy for small x
__device__ __forceinline__ double fraction(double f0, double x) {
  return 1.0 - (1.0 - f0) * (x == 0.0 ? 1.0 : exp(-x));
}
__device__ __forceinline__ float fraction(float f0, float x) {
  return fmaf(1.0f - f0, -expm1f(-x), f0);
}

// ---- warp-level pieces over a window held as v[kPer] per lane (sample 8 lane + j)
template <class R>
__device__ __forceinline__ R shfl_up1(R v) { return __shfl_up_sync(0xffffffffu, v, 1); }
template <class R>
__device__ __forceinline__ R shfl_down1(R v) { return __shfl_down_sync(0xffffffffu, v, 1); }

// Point reflection at the row's ends, y[-m] = 2 y[0] - y[m] and y[N-1+m] = 2 y[N-1] -
// y[N-1-m] for m <= K, through the warp's scratch row (tiles that touch an end only).
template <class R>
__device__ __forceinline__ void reflect_ends(R (&v)[kPer], R* row, int tw, int n_to, int K, int lane) {
#pragma unroll
  for (int j = 0; j < kPer; ++j) row[pad(kPer * lane + j)] = v[j];
  __syncwarp();
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int t = tw + kPer * lane + j;
    if (t < 0 && t >= -K) v[j] = R(2) * row[pad(0 - tw)] - row[pad(-t - tw)];
    if (t > n_to - 1 && t <= n_to - 1 + K) {
      const int m = t - (n_to - 1);
      v[j] = R(2) * row[pad(n_to - 1 - tw)] - row[pad(n_to - 1 - m - tw)];
    }
  }
  __syncwarp();
}

// y~[j] = c0 y[j] + sum_{k <= K} c_k (y[j - k] + y[j + k]), centre first, pairs in k
// order; the taps reach the neighbouring lanes' samples (edge lanes' values outside the
// window are garbage and lie in the halo, which the caller does not use)
template <class R>
__device__ __forceinline__ void band_filter(const R (&y)[kPer], R (&out)[kPer], const R* taps, int K) {
  if (K == 0) {  // the trapezoid rule: the single tap (warp-uniform)
    const R c0 = taps[0];
#pragma unroll
    for (int j = 0; j < kPer; ++j) out[j] = c0 * y[j];
    return;
  }
  R ext[3 * kPer];  // the left neighbour's samples, this lane's, the right neighbour's
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    ext[j] = shfl_up1(y[j]);
    ext[kPer + j] = y[j];
    ext[2 * kPer + j] = shfl_down1(y[j]);
  }
  R c[kHalo + 1];
#pragma unroll
  for (int k = 0; k <= kHalo; ++k) c[k] = k <= K ? taps[k] : R(0);
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    R f = c[0] * ext[kPer + j];
#pragma unroll
    for (int k = 1; k <= kHalo; ++k)
      if (k <= K) f = f + c[k] * (ext[kPer + j - k] + ext[kPer + j + k]);
    out[j] = f;
  }
}

// inc[j] = dt (y~[u] + y~[u + 1]) / 2 on window samples u in [lo, hi) of the row
// (t in [0, n_to - 1)), else 0
template <class R>
__device__ __forceinline__ void trapezoid(const R (&yt)[kPer], R (&inc)[kPer], R dt, int tw, int lo, int hi,
                                          int n_to, int lane) {
  const R next0 = shfl_down1(yt[0]);
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int u = kPer * lane + j, t = tw + u;
    const R nxt = j + 1 < kPer ? yt[j + 1] : next0;
    inc[j] = (u >= lo && u < hi && t >= 0 && t < n_to - 1) ? dt * (yt[j] + nxt) / R(2) : R(0);
  }
}

__device__ __forceinline__ double warp_total(double v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

// the sum of inc over owned window samples [lo, hi), in FP64, fixed order
template <class R>
__device__ __forceinline__ double owned_sum(const R (&inc)[kPer], int lo, int hi, int lane) {
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int u = kPer * lane + j;
    if (u >= lo && u < hi) s += (double)inc[j];
  }
  return warp_total(s);
}

// P[j] = sum of inc over window samples before 8 lane + j (FP64); returns P at sample `at`
template <class R>
__device__ __forceinline__ double window_prefix(const R (&inc)[kPer], double (&P)[kPer], int at, int lane) {
  double run = 0.0;
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    P[j] = run;
    run += (double)inc[j];
  }
  double incl = run;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += y;
  }
  const double base = incl - run;
  double mine = 0.0;
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    P[j] += base;
    if (j == at % kPer) mine = P[j];
  }
  return __shfl_sync(0xffffffffu, mine, at / kPer);
}

// ---- the hand-over between tiles
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

// publish this tile's sums (already written by the warps' lane 0) as stage `target`
template <class R>
__device__ __forceinline__ void publish(const ColumnArgsT<R>& a, int group, int tile, int target) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) store_release(a.flags + (size_t)group * a.n_tiles + tile, target);
}

// wait until every earlier tile of the group has published stage `target`; a wait that
// gives up marks the evaluation failed in *status (read by the host) and goes on
template <class R>
__device__ __forceinline__ void await_predecessors(const ColumnArgsT<R>& a, int group, int tile, int target) {
  const int* f = a.flags + (size_t)group * a.n_tiles;
  for (int j = threadIdx.x; j < tile; j += blockDim.x) {
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

// the predecessors' sums of one node, read past L1 (other CTAs wrote them during this
// launch): lane l adds tiles l, l + 32, ... in order, then the lanes as a tree
__device__ __forceinline__ double predecessors(const double* sums, int node, int n_tiles, int tile, int lane) {
  const double* row = sums + (size_t)node * n_tiles;
  double s = 0.0;
  int k = lane;
  for (; k + 96 < tile; k += 128) {
    const double v0 = __ldcg(row + k), v1 = __ldcg(row + k + 32), v2 = __ldcg(row + k + 64),
                 v3 = __ldcg(row + k + 96);
    s += v0;
    s += v1;
    s += v2;
    s += v3;
  }
  for (; k < tile; k += 32) s += __ldcg(row + k);
  return warp_total(s);
}

}  // namespace

// The plasma of a gas mixture on one tile (passes/plasma.py:326-485): every channel's rate
// and exposure scan in channel order, each handed over between tiles as the single
// channel's is (channel c publishes its exposure sums as stage first + c, in its own plane
// of sums0), the weights rho_c f_c q_c and the works rho_c I_c W_c (1 - f_c) summed over the
// channels, then the one free-current integral of the summed weight times the field
// (published as stage first + n_channels).  J receives the free current, L the summed work
// (the loss current is L E / |E|^2); the densities are inside both.
template <class R>
__device__ __forceinline__ void mixture_plasma(const ColumnArgsT<R>& a, const StageScalarsDev& st,
                                               const R (&E)[kPer], R (&J)[kPer], R (&L)[kPer], int tw,
                                               int K, int owned, int own_hi, bool at_end, int node,
                                               bool live, int group, int tile, int first, R* row,
                                               int lane, bool& quiet) {
  const int n_to = a.n_to, A = a.lead;
  const R dt = R(a.dt);
  const size_t plane = (size_t)a.n_nodes * a.n_tiles;
  R weight[kPer];
#pragma unroll
  for (int j = 0; j < kPer; ++j) weight[j] = L[j] = R(0);
  bool all_dark = true;
  for (int c = 0; c < a.n_channels; ++c) {
    const ChannelTableT<R> ch = a.channels[c];
    const RateLookup<R> rates = rate_lookup(ch);
    R W[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int t = tw + kPer * lane + j;
      W[j] = (t >= 0 && t < n_to) ? rate_of(rates, fabs(E[j])) : R(0);
    }
    bool dark = true;
#pragma unroll
    for (int j = 0; j < kPer; ++j) dark = dark && W[j] == R(0);
    dark = __all_sync(0xffffffffu, dark);
    R inc[kPer];
    double s0 = 0.0;
    if (!dark) {
      R Wf[kPer];
      if (at_end) {
        R Wg[kPer];
#pragma unroll
        for (int j = 0; j < kPer; ++j) Wg[j] = W[j];
        reflect_ends(Wg, row, tw, n_to, K, lane);
        band_filter(Wg, Wf, a.taps, K);
      } else {
        band_filter(W, Wf, a.taps, K);
      }
      trapezoid(Wf, inc, dt, tw, A - K, A + owned + K, n_to, lane);
      s0 = owned_sum(inc, A, own_hi, lane);
    }
    double* sums = a.sums0 + (size_t)c * plane;
    if (lane == 0 && live) sums[(size_t)node * a.n_tiles + tile] = s0;
    publish(a, group, tile, first + c);
    await_predecessors(a, group, tile, first + c);
    const double off0 = live ? predecessors(sums, node, a.n_tiles, tile, lane) : 0.0;
    const R f0 = R(st.channel_preionisation[c]), rho = R(st.channel_density[c]);
    const R qm = R(ch.charge_mass_ratio), ip = R(ch.ionisation_potential);
    if (dark) {
      const R x = R(off0);
      const R f = fraction(f0, a.band ? fmax(x, R(0)) : x);
#pragma unroll
      for (int j = 0; j < kPer; ++j) {
        const int u = kPer * lane + j, t = tw + u;
        if (u >= A - K && u <= A + owned + K && t >= 0 && t < n_to) weight[j] += rho * f * qm;
      }
    } else {
      double P[kPer];
      const double at_t0 = window_prefix(inc, P, A, lane);
#pragma unroll
      for (int j = 0; j < kPer; ++j) {
        const int u = kPer * lane + j, t = tw + u;
        if (u >= A - K && u <= A + owned + K && t >= 0 && t < n_to) {
          const R x = R(off0 + (P[j] - at_t0));
          const R f = fraction(f0, a.band ? fmax(x, R(0)) : x);
          weight[j] += rho * f * qm;
          L[j] += rho * ip * W[j] * (R(1) - f);
        }
      }
    }
    all_dark = all_dark && dark;
  }
  R g[kPer];
#pragma unroll
  for (int j = 0; j < kPer; ++j) g[j] = weight[j] * E[j];
  bool still = true;
#pragma unroll
  for (int j = 0; j < kPer; ++j) still = still && g[j] == R(0);
  still = __all_sync(0xffffffffu, still);
  R inc[kPer];
  double s1 = 0.0;
  if (!still) {
    if (at_end) reflect_ends(g, row, tw, n_to, K, lane);
    R gf[kPer];
    band_filter(g, gf, a.taps, K);
    trapezoid(gf, inc, dt, tw, A, A + owned, n_to, lane);
    s1 = owned_sum(inc, A, own_hi, lane);
  }
  const int last = first + a.n_channels;
  if (lane == 0 && live) a.sums1[(size_t)node * a.n_tiles + tile] = s1;
  publish(a, group, tile, last);
  await_predecessors(a, group, tile, last);
  const double off1 = live ? predecessors(a.sums1, node, a.n_tiles, tile, lane) : 0.0;
  quiet = all_dark && still && off1 == 0.0;
  if (still) {
#pragma unroll
    for (int j = 0; j < kPer; ++j) J[j] = R(off1);
  } else {
    double P[kPer];
    const double at_t0 = window_prefix(inc, P, A, lane);
#pragma unroll
    for (int j = 0; j < kPer; ++j) J[j] = R(off1 + (P[j] - at_t0));
  }
}

// One tile of one node group: the window's synthesis, rate, running integrals, outputs and
// projection.  kSweep = false: the tile is one CTA's whole work and learns its running
// integrals' offsets from its predecessors' published sums (the hand-over above).
// kSweep = true: one CTA walks
// a node group through all tiles in order, so the offsets are its own running sums,
// carried per lane -- lane l holds the sum of tiles l, l + 32, ... added in tile order,
// the association predecessors() uses, so both forms give the same bits -- and every
// group keeps its own partial rows, which the forward transform adds in group order.
//
// kNodes = true is the GEMM route's form (tile-parallel only): the window's field is the
// node field a synthesis product wrote, read in place of the synthesis, and the outputs
// go to the node streams a projection product reads, in place of the projection.
//
// kMulti = true is a gas mixture's form (tile-parallel only): the channels' plasma of
// mixture_plasma in place of the single channel's.
template <class R, bool kSweep, bool kNodes = false, bool kMulti = false>
__device__ __forceinline__ void column_tile(const ColumnArgsT<R>& a, int tile, int group,
                                            unsigned long long epoch, double& carry0, double& carry1) {
  static_assert(!(kSweep && kNodes), "the node-field form is tile-parallel");
  static_assert(!(kSweep && kMulti), "a mixture's form is tile-parallel");
  extern __shared__ __align__(16) unsigned char column_raw[];
  R* modal = reinterpret_cast<R*>(column_raw);    // [m][kPitch], then the streams
  R* streams = modal;                              // [s][warp][kPitch]
  R* scratch = modal + (size_t)3 * kGroup * kPitch;
  __shared__ __align__(16) R wt[kMaxModes * kGroup];
  __shared__ R gate[kPitch], gate_d[kPitch];  // the temporal window g and g' on the window (padded)
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  // the record's scalars this tile reads, into registers once
  const int n_to = a.n_to, n_modes = a.n_modes, n_nodes = a.n_nodes, n_cols = a.n_cols;
  const int node = group * kGroup + warp;
  const bool live = node < n_nodes;
  const int K = a.half_width, A = a.lead, owned = a.owned;
  const int t0 = tile * owned, tw = t0 - A;  // owned samples [t0, t0 + owned): window [A, A + owned)
  const int own_hi = A + min(owned, n_to - t0);
  const StageScalarsDev& st = *a.stage;
  const R tau = R(st.taper);
  const bool plasma = a.plasma;
  // the modal window and the group's projection weights W[m, node] / tau
  // the sweep's copies of this tile's windows arrived during the last tile (the caller
  // waited for them before its barrier)
  double* next_modal = reinterpret_cast<double*>(column_raw + column_smem<R>());
  R* next_gate = reinterpret_cast<R*>(next_modal + (size_t)kMaxModes * kWindow);
  const bool copied = kSweep && tile > 0;
  if constexpr (kNodes) {
    // nothing modal to stage: the field is read per node below
  } else if (copied) {
    for (int i = threadIdx.x; i < n_modes * kWindow; i += blockDim.x)
      modal[(i / kWindow) * kPitch + pad(i % kWindow)] = R(next_modal[i]);
  } else {
    const double* modal_t = a.modal_t;
    for (int i = threadIdx.x; i < n_modes * kWindow; i += blockDim.x) {
      const int m = i / kWindow, u = i % kWindow, t = tw + u;
      modal[m * kPitch + pad(u)] = (t >= 0 && t < n_to) ? R(modal_t[(size_t)m * n_to + t]) : R(0);
    }
  }
  if (!kNodes && (!kSweep || tile == 0)) {  // the weights do not change along a sweep
    const R* projection = a.projection;
    for (int k = threadIdx.x; k < n_modes * kGroup; k += blockDim.x) {
      const int m = k / kGroup, w = k % kGroup, nd = group * kGroup + w;
      wt[k] = nd < n_nodes ? projection[m * n_nodes + nd] / tau : R(0);
    }
  }
  for (int u = threadIdx.x; u < kWindow; u += blockDim.x) {
    if (copied) {
      gate[pad(u)] = next_gate[u];
      gate_d[pad(u)] = next_gate[kWindow + u];
    } else {
      const int t = tw + u;
      const bool in = t >= 0 && t < n_to;
      gate[pad(u)] = in ? a.t_window[t] : R(0);
      gate_d[pad(u)] = in ? a.t_window_derivative[t] : R(0);
    }
  }
  __syncthreads();
  if (kSweep && tile + 1 < a.n_tiles) {
    // the next tile's windows, copied while this one is computed
    const int tn = tw + owned;  // the next window's first sample
    const double* modal_t = a.modal_t;
    for (int i = threadIdx.x; i < n_modes * kWindow; i += blockDim.x) {
      const int m = i / kWindow, t = tn + i % kWindow;
      const bool in = t >= 0 && t < n_to;
      copy_async<8>(next_modal + i, modal_t + (size_t)m * n_to + (in ? t : 0), in);
    }
    for (int u = threadIdx.x; u < kWindow; u += blockDim.x) {
      const int t = tn + u;
      const bool in = t >= 0 && t < n_to;
      copy_async<sizeof(R)>(next_gate + u, a.t_window + (in ? t : 0), in);
      copy_async<sizeof(R)>(next_gate + kWindow + u, a.t_window_derivative + (in ? t : 0), in);
    }
    copy_async_commit();
  }
  // synthesis and rate on the window
  R E[kPer], W[kPer];
  {
    R srow[kMaxModes];
    const R* synthesis = a.synthesis;
#pragma unroll
    for (int m = 0; m < kMaxModes; ++m)
      srow[m] = (!kNodes && live && m < n_modes) ? synthesis[node * n_modes + m] * tau : R(0);
    const RateLookup<R> rates = rate_lookup(a);
    const R* field_row = kNodes && live ? a.node_field + (size_t)node * n_to : nullptr;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int u = kPer * lane + j, t = tw + u;
      R e = R(0);
      if constexpr (kNodes) {
        if (field_row && t >= 0 && t < n_to) e = field_row[t];
      } else {
#pragma unroll
        for (int m = 0; m < kMaxModes; ++m)
          if (m < n_modes) e += srow[m] * modal[m * kPitch + pad(u)];
      }
      E[j] = e;
      W[j] = (!kMulti && plasma && t >= 0 && t < n_to) ? rate_of(rates, fabs(e)) : R(0);
    }
  }
  __syncthreads();  // the modal window's space becomes the streams'
  const bool at_end = tw < 0 || tw + kWindow > n_to;  // block-uniform
  R F[kPer], J[kPer];
#pragma unroll
  for (int j = 0; j < kPer; ++j) F[j] = J[j] = R(0);
  bool quiet = true;  // this node carries no current on the window (warp-uniform)
  if (kMulti && plasma) {
    // J: the free current, F: the summed work (both with the channel densities inside)
    const int first = (int)((unsigned long long)(a.n_channels + 1) * epoch + 1);
    mixture_plasma(a, st, E, J, F, tw, K, owned, own_hi, at_end, node, live, group, tile, first,
                   scratch + (size_t)warp * kPitch, lane, quiet);
  } else if (plasma) {
    const int first = (int)(2 * epoch + 1);
    const R dt = R(a.dt);
    R* row = scratch + (size_t)warp * kPitch;
    // A node whose rate is zero on the whole window (every tile but the few the pulse
    // ionises) has zero exposure increments: the filter, the trapezoid and the prefix
    // would return exact zeros, so they are skipped, the exposure is the offset alone and
    // the fraction one value.  Where that fraction is zero too (ahead of the pulse) the
    // current's integrand vanishes and its pass is skipped the same way.  The shortcuts
    // give the bits of the full path: its zeros may carry a sign, but every sum starts
    // from +0, which absorbs them.
    bool dark = true;
#pragma unroll
    for (int j = 0; j < kPer; ++j) dark = dark && W[j] == R(0);
    dark = __all_sync(0xffffffffu, dark);
    // exposure: W~ on [A - K, A + owned + K], increments on [A - K, A + owned + K)
    R inc[kPer];
    double s0 = 0.0;
    if (!dark) {
      R Wf[kPer];
      if (at_end) {
        R Wg[kPer];  // with the reflected ghosts, for the filter only
#pragma unroll
        for (int j = 0; j < kPer; ++j) Wg[j] = W[j];
        reflect_ends(Wg, row, tw, n_to, K, lane);
        band_filter(Wg, Wf, a.taps, K);
      } else {
        band_filter(W, Wf, a.taps, K);
      }
      trapezoid(Wf, inc, dt, tw, A - K, A + owned + K, n_to, lane);
      s0 = owned_sum(inc, A, own_hi, lane);
    }
    double off0;
    if constexpr (kSweep) {
      off0 = live ? warp_total(carry0) : 0.0;
      if (lane == (tile & 31)) carry0 += s0;
    } else {
      if (lane == 0 && live) a.sums0[(size_t)node * a.n_tiles + tile] = s0;
      publish(a, group, tile, first);
      await_predecessors(a, group, tile, first);
      off0 = live ? predecessors(a.sums0, node, a.n_tiles, tile, lane) : 0.0;
    }
    // fraction and the current's integrand on [A - K, A + owned + K]
    const R f0 = R(st.preionisation), qm = R(a.charge_mass_ratio);
    R g[kPer];
    if (dark) {
      const R x = R(off0);
      const R f_dark = fraction(f0, a.band ? fmax(x, R(0)) : x);
#pragma unroll
      for (int j = 0; j < kPer; ++j) {
        const int u = kPer * lane + j, t = tw + u;
        const bool in = u >= A - K && u <= A + owned + K && t >= 0 && t < n_to;
        F[j] = in ? f_dark : R(0);
        g[j] = in ? f_dark * qm * E[j] : R(0);
      }
    } else {
      double P[kPer];
      const double at_t0 = window_prefix(inc, P, A, lane);
#pragma unroll
      for (int j = 0; j < kPer; ++j) {
        const int u = kPer * lane + j, t = tw + u;
        R f = R(0), gv = R(0);
        if (u >= A - K && u <= A + owned + K && t >= 0 && t < n_to) {
          const R x = R(off0 + (P[j] - at_t0));
          f = fraction(f0, a.band ? fmax(x, R(0)) : x);
          gv = f * qm * E[j];
        }
        F[j] = f;
        g[j] = gv;
      }
    }
    bool still = true;
#pragma unroll
    for (int j = 0; j < kPer; ++j) still = still && g[j] == R(0);
    still = __all_sync(0xffffffffu, still);
    double s1 = 0.0;
    if (!still) {
      if (at_end) reflect_ends(g, row, tw, n_to, K, lane);
      R gf[kPer];
      band_filter(g, gf, a.taps, K);
      trapezoid(gf, inc, dt, tw, A, A + owned, n_to, lane);
      s1 = owned_sum(inc, A, own_hi, lane);
    }
    double off1;
    if constexpr (kSweep) {
      off1 = live ? warp_total(carry1) : 0.0;
      if (lane == (tile & 31)) carry1 += s1;
    } else {
      if (lane == 0 && live) a.sums1[(size_t)node * a.n_tiles + tile] = s1;
      publish(a, group, tile, first + 1);
      await_predecessors(a, group, tile, first + 1);
      off1 = live ? predecessors(a.sums1, node, a.n_tiles, tile, lane) : 0.0;
    }
    quiet = dark && still && off1 == 0.0;
    if (still) {
#pragma unroll
      for (int j = 0; j < kPer; ++j) J[j] = R(off1);
    } else {
      double P[kPer];
      const double at_t0_1 = window_prefix(inc, P, A, lane);
#pragma unroll
      for (int j = 0; j < kPer; ++j) J[j] = R(off1 + (P[j] - at_t0_1));
    }
  }
  // outputs on the owned samples: P = (c rho E^2 E) g, X = g rho J, Z = g' rho J
  {
    // The Kerr factor (coefficient times density: about 1e-39 for helium at a fifth of a bar)
    // lies among FP32's subnormals; the FP32 form carries it scaled by 2^64 and takes the
    // scale out of the cubic, both exact powers of two.  FP64 takes it as it is.
    constexpr double kKerrScale = sizeof(R) == 4 ? 18446744073709551616.0 : 1.0;  // 2^64
    const R factor = R(a.kerr ? a.kerr_coefficient * st.kerr_density * kKerrScale : 0.0);
    const R unscale = R(1.0 / kKerrScale);
    const R rho = R(st.plasma_density), ip = R(a.ionisation_potential);
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int u = kPer * lane + j;
      R p = R(0), x = R(0), z = R(0);
      if (live && u >= A && u < own_hi) {
        const R e = E[j];
        const R win = gate[pad(u)];
        p = (a.kerr ? factor * (e * e) * e * unscale : R(0)) * win;
        if (kMulti && plasma) {  // J + (L / |E|^2) E, the densities inside (plasma.py:471-485)
          const R squared = fabs(e) * fabs(e);
          const R guard = squared > R(0) ? divide(F[j], squared) : R(0);
          const R current = J[j] + guard * e;
          x = win * current;
          z = gate_d[pad(u)] * current;
        } else if (plasma) {
          const R w = W[j], f = F[j];
          const R squared = fabs(e) * fabs(e);
          R scale = R(0);
          if (w > R(0) && squared > R(0)) scale = divide(ip * w * (R(1) - f), squared);
          const R current = rho * (J[j] + scale * e);
          x = win * current;
          z = gate_d[pad(u)] * current;
        }
      }
      if constexpr (kNodes) {
        if (live && u >= A && u < own_hi) {
          const size_t at = (size_t)node * n_to + (size_t)(tw + u);
          const size_t plane = (size_t)n_nodes * n_to;
          a.node_streams[at] = p;
          if (plasma) {
            a.node_streams[plane + at] = x;
            a.node_streams[2 * plane + at] = z;
          }
        }
      } else {
        streams[(0 * kGroup + warp) * kPitch + pad(u)] = p;
        streams[(1 * kGroup + warp) * kPitch + pad(u)] = x;
        streams[(2 * kGroup + warp) * kPitch + pad(u)] = z;
      }
    }
  }
  if constexpr (kNodes) return;  // the projection product takes the node streams
  // Ahead of the pulse no node of the group carries a current: the two current streams
  // are zeros of either sign, whose projections are +0, written without the products.
  const bool currents = __syncthreads_or(!quiet) != 0;
  // projection of the owned samples onto the modes: thread u takes window sample u of
  // every stream and mode, the group's nodes summed in order
  static_assert(kThreads == kWindow, "one thread per window sample");
  const int n_streams = plasma ? 3 : 1;
  const int u = threadIdx.x;
  const bool mine = u >= A && u < own_hi;
  const size_t row_of_group = (size_t)3 * n_cols * n_to;
  R* base = a.partials + (mine ? tw + u : 0);  // sample t = tw + u of row (group 3 + s) n_cols + m
  if (mine) {
    // the three streams' samples of the group's nodes, then mode by mode: the weights
    // are read once per mode for all streams
    R v[3][kGroup];
#pragma unroll
    for (int s = 0; s < 3; ++s)
#pragma unroll
      for (int w = 0; w < kGroup; ++w)
        v[s][w] = s < n_streams && (s == 0 || currents) ? streams[(s * kGroup + w) * kPitch + pad(u)] : R(0);
    R* out = base + group * row_of_group;
    const size_t stream_stride = (size_t)n_cols * n_to;
    for (int m = 0; m < n_modes; ++m) {
      R c[kGroup];
#pragma unroll
      for (int w = 0; w < kGroup; ++w) c[w] = wt[m * kGroup + w];
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        if (s < n_streams) {
          R acc = R(0);
          if (s == 0 || currents) {
#pragma unroll
            for (int w = 0; w < kGroup; ++w) acc += c[w] * v[s][w];
          }
          out[s * stream_stride + (size_t)m * n_to] = acc;
        }
      }
    }
  }
  // the node groups' partial rows stay apart: the forward transform adds them in group order
}

template <class R, bool kNodes = false, bool kMulti = false>
__device__ __forceinline__ void column_body(const ColumnArgsT<R>& a) {
  __shared__ unsigned long long ticket;
  if (threadIdx.x == 0) ticket = atomicAdd(a.ticket, 1ull);
  __syncthreads();
  const unsigned long long epoch = ticket / (unsigned long long)a.n_blocks;
  const int index = (int)(ticket % (unsigned long long)a.n_blocks);
  double unused0 = 0.0, unused1 = 0.0;
  column_tile<R, false, kNodes, kMulti>(a, index / a.n_groups, index % a.n_groups, epoch, unused0, unused1);
}

// one node group through every tile of the row, in tile order
template <class R>
__device__ __forceinline__ void column_sweep(const ColumnArgsT<R>& a, int group) {
  double carry0 = 0.0, carry1 = 0.0;
  for (int tile = 0; tile < a.n_tiles; ++tile) {
    if (tile > 0) {
      copy_async_wait();  // this thread's copies of the tile's windows
      __syncthreads();    // everyone's, and the last tile's projection is done with the rows
    }
    column_tile<R, true>(a, tile, group, 0ull, carry0, carry1);
  }
}

// resident CTAs per SM: two in FP64 (128 registers), three in FP32 (85)
template <class R> constexpr int column_residency() { return sizeof(R) == 8 ? 2 : 3; }

template <class R>
__global__ void __launch_bounds__(kThreads, column_residency<R>()) k_column(ColumnArgsT<R> a) {
  column_body(a);
}

template <class R>
__global__ void __launch_bounds__(kThreads, column_residency<R>()) k_column_nodes(ColumnArgsT<R> a) {
  column_body<R, true>(a);
}

// a gas mixture's plasma channels, on either route
template <class R>
__global__ void __launch_bounds__(kThreads, column_residency<R>()) k_column_mix(ColumnArgsT<R> a) {
  column_body<R, false, true>(a);
}

template <class R>
__global__ void __launch_bounds__(kThreads, column_residency<R>()) k_column_nodes_mix(ColumnArgsT<R> a) {
  column_body<R, true, true>(a);
}

// batched: items[blockIdx.x].x = the run; a run's CTAs take their tiles from its counter
template <class R>
__global__ void __launch_bounds__(kThreads, column_residency<R>())
    k_column_b(const ColumnArgsT<R>* args, const int4* items, const int* flags) {
  const int run = items[blockIdx.x].x;
  if (!flags[run]) return;  // every CTA of an idle run leaves before its ticket
  column_body(own_args(args, run));
}

// batched, one CTA per (run, node group) walking the run's tiles: items[blockIdx.x] =
// (run, group), listed longest row first so that the long walks start in the first wave
template <class R>
__global__ void __launch_bounds__(kThreads, column_residency<R>())
    k_column_sweep_b(const ColumnArgsT<R>* args, const int4* items, const int* flags) {
  const int4 it = items[blockIdx.x];
  if (!flags[it.x]) return;  // block-uniform
  column_sweep(own_args(args, it.x), it.y);
}

template <class R>
cudaError_t launch_column_sweep_b(const ColumnArgsT<R>* args, const int4* items, const int* flags,
                                  int n_items, cudaStream_t stream) {
  k_column_sweep_b<R><<<n_items, kThreads, column_sweep_smem<R>(), stream>>>(args, items, flags);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_column_b(const ColumnArgsT<R>* args, const int4* items, const int* flags,
                            int n_items, cudaStream_t stream) {
  k_column_b<R><<<n_items, kThreads, column_smem<R>(), stream>>>(args, items, flags);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_column(const ColumnArgsT<R>& a, cudaStream_t stream) {
  if (a.plasma && a.n_channels > 1)
    k_column_mix<R><<<a.n_blocks, kThreads, column_smem<R>(), stream>>>(a);
  else
    k_column<R><<<a.n_blocks, kThreads, column_smem<R>(), stream>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t launch_column_nodes(const ColumnArgsT<R>& a, cudaStream_t stream) {
  if (a.plasma && a.n_channels > 1)
    k_column_nodes_mix<R><<<a.n_blocks, kThreads, column_smem<R>(), stream>>>(a);
  else
    k_column_nodes<R><<<a.n_blocks, kThreads, column_smem<R>(), stream>>>(a);
  return cudaGetLastError();
}

template cudaError_t launch_column_nodes<double>(const ColumnArgsT<double>&, cudaStream_t);
template cudaError_t launch_column_nodes<float>(const ColumnArgsT<float>&, cudaStream_t);
template cudaError_t launch_column<double>(const ColumnArgsT<double>&, cudaStream_t);
template cudaError_t launch_column<float>(const ColumnArgsT<float>&, cudaStream_t);
template cudaError_t launch_column_b<double>(const ColumnArgsT<double>*, const int4*, const int*, int,
                                             cudaStream_t);
template cudaError_t launch_column_b<float>(const ColumnArgsT<float>*, const int4*, const int*, int,
                                            cudaStream_t);
template cudaError_t launch_column_sweep_b<double>(const ColumnArgsT<double>*, const int4*, const int*,
                                                   int, cudaStream_t);
template cudaError_t launch_column_sweep_b<float>(const ColumnArgsT<float>*, const int4*, const int*,
                                                  int, cudaStream_t);

cudaError_t configure_column_kernels() {
  const void* kernels[12] = {(const void*)k_column<double>, (const void*)k_column_b<double>,
                             (const void*)k_column_sweep_b<double>, (const void*)k_column<float>,
                             (const void*)k_column_b<float>, (const void*)k_column_sweep_b<float>,
                             (const void*)k_column_nodes<double>, (const void*)k_column_nodes<float>,
                             (const void*)k_column_mix<double>, (const void*)k_column_mix<float>,
                             (const void*)k_column_nodes_mix<double>, (const void*)k_column_nodes_mix<float>};
  const size_t shm[12] = {column_smem<double>(), column_smem<double>(), column_sweep_smem<double>(),
                          column_smem<float>(), column_smem<float>(), column_sweep_smem<float>(),
                          column_smem<double>(), column_smem<float>(), column_smem<double>(),
                          column_smem<float>(), column_smem<double>(), column_smem<float>()};
  for (int i = 0; i < 12; ++i) {
    cudaError_t e = cudaFuncSetAttribute(kernels[i], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)shm[i]);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace sp
