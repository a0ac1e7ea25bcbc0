// The stepping kernels: the exponential Adams trial's predict and correct passes with
// their fused norms and the accept pass (backends/numpy_ref/adams_kernels.py:404-741,
// multistep.py:901-1070), and the DOPRI5 trial's stage input and finish
// (backends/numpy_ref/engines.py:97-181, passes/stepping.py:38-283).  Each kernel is a
// single pass over the state; the norms are two-level deterministic reductions: a fixed
// grid of kNormBlocks blocks writes one partial per block, one block adds them.
#include "kernels.cuh"
#include "stage_output.cuh"

namespace sp {

// 1 / n! for n < 32, each the double nearest the exact value
__constant__ double c_inv_fact[32] = {
    1.0, 1.0, 0.5, 0.16666666666666666,
    0.041666666666666664, 0.008333333333333333, 0.001388888888888889, 0.0001984126984126984,
    2.48015873015873e-05, 2.7557319223985893e-06, 2.755731922398589e-07, 2.505210838544172e-08,
    2.08767569878681e-09, 1.6059043836821613e-10, 1.1470745597729725e-11, 7.647163731819816e-13,
    4.779477332387385e-14, 2.8114572543455206e-15, 1.5619206968586225e-16, 8.22063524662433e-18,
    4.110317623312165e-19, 1.9572941063391263e-20, 8.896791392450574e-22, 3.868170170630684e-23,
    1.6117375710961184e-24, 6.446950284384474e-26, 2.4795962632247976e-27, 9.183689863795546e-29,
    3.279889237069838e-30, 1.1309962886447716e-31, 3.7699876288159054e-33, 1.216125041553518e-34};

// acc y + c for complex acc, y and real c
__device__ __forceinline__ double2 horner_step(double2 acc, double2 y, double c) {
  return make_double2(fma(acc.x, y.x, fma(-acc.y, y.y, c)), fma(acc.x, y.y, acc.y * y.x));
}

// phi_0(x) .. phi_order(x) (backends/exponential.py:131-224): the upward recurrence
// phi_k = (phi_{k-1} - 1/(k-1)!) / x from exp(x) beyond |x| = 3; below, x is halved sq
// times to |y| <= 1/2, phi_order(y) = sum_{m<24} y^m / (m + order)! is summed by Horner's
// rule, the lower functions follow by the downward recurrence phi_k = 1/k! + y phi_{k+1},
// and sq doublings phi_k(2y) = 2^-k (phi_0 phi_k + sum_{j=1..k} phi_j / (k - j)!) undo the
// halving.  Every index is a compile-time one (order <= kMaxWidth), so the functions stay
// in registers; the divisions are products with 1/x, 1/n! and 2^-k.
__device__ __forceinline__ void phi_functions(double2 x, int order, double2 (&out)[kMaxWidth + 1]) {
  const double mag2 = x.x * x.x + x.y * x.y;
  if (mag2 > 9.0) {
    const double s = 1.0 / mag2;
    const double2 rx = make_double2(x.x * s, -x.y * s);
    out[0] = cexp(x);
#pragma unroll
    for (int k = 1; k <= kMaxWidth; ++k) {
      if (k > order) break;
      out[k] = cmul(make_double2(out[k - 1].x - c_inv_fact[k - 1], out[k - 1].y), rx);
    }
    return;
  }
  int sq = 0;
  if (mag2 > 0.25) {  // the least sq with 2 |x| <= 2^sq
    int e;
    const double f = frexp(2.0 * sqrt(mag2), &e);
    sq = f == 0.5 ? e - 1 : e;
  }
  const double scale = ldexp(1.0, -sq);
  const double2 y = make_double2(x.x * scale, x.y * scale);
  double2 acc = make_double2(c_inv_fact[23 + order], 0.0);
#pragma unroll 4
  for (int m = 22; m >= 0; --m) acc = horner_step(acc, y, c_inv_fact[m + order]);
  // the downward recurrence from phi_order = acc
#pragma unroll
  for (int k = kMaxWidth; k >= 1; --k) {
    if (k > order) continue;
    if (k == order) {
      out[k] = acc;
    } else {
      const double2 t = cmul(y, out[k + 1]);
      out[k] = make_double2(c_inv_fact[k] + t.x, t.y);
    }
  }
  out[0] = cexp(y);
  for (int level = 0; level < sq; ++level) {
    double2 old[kMaxWidth + 1];
#pragma unroll
    for (int k = 0; k <= kMaxWidth; ++k) old[k] = out[k];
    out[0] = cmul(old[0], old[0]);
    double p2 = 1.0;
#pragma unroll
    for (int k = 1; k <= kMaxWidth; ++k) {
      if (k > order) break;
      p2 *= 0.5;
      double2 t = cmul(old[0], old[k]);
#pragma unroll
      for (int j = 1; j <= k; ++j) t = cadd(t, cscale(c_inv_fact[k - j], old[j]));
      out[k] = make_double2(t.x * p2, t.y * p2);
    }
  }
}

// sum_p w[p] terms[p][i] from +0 in term order, the loads of eight terms in flight at a time
__device__ __forceinline__ double2 contract_terms(const double* w, int n_terms, const double2* terms,
                                                  size_t n, size_t i) {
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll 8
  for (int p = 0; p < n_terms; ++p) acc = cadd(acc, cscale(w[p], terms[(size_t)p * n + i]));
  return acc;
}

__device__ __forceinline__ double2 combine_terms(const double* w, int n_terms,
                                                 const double2* terms, int n, int i) {
  // translate/stage.py:292-342: one term multiplied (or itself for a unit weight),
  // several contracted in order
  if (n_terms == 1) {
    double2 t = terms[i];
    return w[0] == 1.0 ? t : cscale(w[0], t);
  }
  return contract_terms(w, n_terms, terms, n, i);
}

// x = combine_terms(wx, ...) and r = contract_terms(wr, ...) in one pass over the rows
__device__ __forceinline__ void combine_two(const double* wx, const double* wr, int n_terms,
                                            const double2* terms, size_t n, size_t i, double2& x, double2& r) {
  if (n_terms == 1) {
    const double2 t = terms[i];
    x = wx[0] == 1.0 ? t : cscale(wx[0], t);
    r = cadd(make_double2(0.0, 0.0), cscale(wr[0], t));
    return;
  }
  double2 ax = make_double2(0.0, 0.0), ar = make_double2(0.0, 0.0);
#pragma unroll 8
  for (int p = 0; p < n_terms; ++p) {
    const double2 t = terms[(size_t)p * n + i];
    ax = cadd(ax, cscale(wx[p], t));
    ar = cadd(ar, cscale(wr[p], t));
  }
  x = ax;
  r = ar;
}

// sum of n_q values per thread into partials[q][blockIdx.x]; deterministic order
template <int NQ>
__device__ void block_partials(double (&v)[NQ], double* partials, int block) {
  __shared__ double red[NQ][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double x = v[q];
    for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
    if (lane == 0) red[q][warp] = x;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double x = lane < nw ? red[q][lane] : 0.0;
      for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
      if (lane == 0) partials[q * kNormBlocks + block] = x;
    }
  }
}

__device__ __forceinline__ void reduce_body(const double* partials, double* out, int q, int nb) {
  // one warp per quantity; fixed order
  double x = 0.0;
  for (int b = threadIdx.x; b < nb; b += 32) x += partials[q * kNormBlocks + b];
  for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
  if (threadIdx.x == 0) out[q] = x;
}

__global__ void k_reduce(const double* partials, double* out, int nq, int nb) {
  if ((int)blockIdx.x >= nq) return;
  reduce_body(partials, out, blockIdx.x, nb);
}

// batched: one block per (quantity, run); runs[blockIdx.y]
__global__ void k_reduce_b(const StepArgs* args, const int* flags, int nq) {
  if (!flags[blockIdx.y]) return;
  const StepArgs& a = args[blockIdx.y];
  if ((int)blockIdx.x >= nq) return;
  reduce_body(a.partials, a.norms, blockIdx.x, a.n_blocks);
}

// A single run's corrector reduces its own partials: every block counts itself in on the
// arrival counter once its partials are written (and fenced), and the last block to arrive
// adds every block's partials, one warp per quantity in the order reduce_body uses, then
// resets the counter for the next launch.  The partials are read from L2 (written by other SMs).
__device__ __forceinline__ void reduce_if_last(const StepArgs& a, int nq) {
  __shared__ int last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(a.norm_arrivals, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int lane = threadIdx.x & 31;
  for (int q = threadIdx.x >> 5; q < nq; q += blockDim.x >> 5) {
    double x = 0.0;
    for (int b = lane; b < a.n_blocks; b += 32) x += __ldcg(a.partials + q * kNormBlocks + b);
    for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
    if (lane == 0) a.norms[q] = x;
  }
  if (threadIdx.x == 0) *a.norm_arrivals = 0u;
}

// The trial's coefficient table, copied into shared memory once per block.  Every thread
// reads each coefficient right before its use; from global memory each such read is a
// stall of the one warp per scheduler that a single run's passes have.
static_assert(sizeof(AdamsDev) % 8 == 0, "the table is copied in 8-byte words");
__device__ __forceinline__ const AdamsDev& staged_adams(const AdamsDev* src) {
  __shared__ AdamsDev table;
  const unsigned long long* from = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* to = reinterpret_cast<unsigned long long*>(&table);
  for (int w = threadIdx.x; w < (int)(sizeof(AdamsDev) / 8); w += blockDim.x) to[w] = from[w];
  __syncthreads();
  return table;
}

// ------------------------------------------------------------------ Adams predict
// kPair: two warps per 32 elements (a single run, whose few elements leave most of the GPU
// idle): the even warp of a pair takes the phi functions, the moments and the predicted
// state, the odd warp the compensation (the carried rows, each with its own exponential,
// and the step end's rate) and hands its sums to the even warp through shared memory, the
// pair meeting at a named barrier once per trip (double-buffered, so one meeting per trip
// suffices).  Otherwise every thread takes both parts of its element.
template <bool kPair>
__device__ __forceinline__ void adams_predict_body(const StepArgs& a, int block) {
  const AdamsDev& ad = staged_adams(a.adams);
  const StageScalarsDev& st = *a.stage;
  const int width = ad.width, order = ad.order;
  const int lane = threadIdx.x & 31, warp_in_block = threadIdx.x >> 5;
  const bool main_part = !kPair || !(warp_in_block & 1);
  const bool comp_part = ad.compensated && (!kPair || (warp_in_block & 1));
  // element groups of 32: one per warp, or one per warp pair
  const int groups_per_block = kPair ? (int)(blockDim.x >> 6) : (int)(blockDim.x >> 5);
  const int group = block * groups_per_block + (kPair ? warp_in_block >> 1 : warp_in_block);
  const int n_groups = a.n_blocks * groups_per_block;
  __shared__ double2 handed[2][kPair ? 16 : 1][32];  // the odd warps' sums, by trip parity
  double v[1] = {0.0};
  int trip = 0;
  for (int base = group * 32; base < a.n; base += n_groups * 32, ++trip) {
    const int i = base + lane;
    const bool valid = i < a.n;
    double2 x = make_double2(0.0, 0.0), rate_end = make_double2(0.0, 0.0);
    double2 comp = make_double2(0.0, 0.0), lab = make_double2(0.0, 0.0), y = make_double2(0.0, 0.0);
    constexpr int kRows = 5;  // the Adams order is at most 5
    double2 rate_rows[kRows], state_rows[kRows];
    if (valid && comp_part) {  // loaded first, to overlap with the loads and work below
#pragma unroll
      for (int j = 0; j < kRows; ++j) {
        if (j < width - 1) {
          rate_rows[j] = a.rates[(size_t)ad.slots[j] * a.n + i];
          state_rows[j] = a.states[(size_t)ad.slots[j] * a.n + i];
        }
      }
    }
    if (valid && main_part) {
      // the accept of the trial before, when the host left it to this pass: the new state
      // and the source row of its free slot (which this trial's stencil reads as its newest
      // row)
      if (ad.settle) {
        const double2 adv = a.advanced[i];
        y = a.active_mask[i % a.n_omega] ? adv : make_double2(adv.x * 0.0, adv.y * 0.0);
        a.state[i] = y;
        a.store[(size_t)(ad.settle - 1) * a.n + i] = a.source[i];
      } else {
        y = a.state[i];
      }
      // every operand row is loaded up front, so that the loads overlap one another and the
      // phi functions instead of waiting in the loops below
      double2 rows[kRows];
#pragma unroll
      for (int j = 0; j < kRows; ++j)
        if (j < order) rows[j] = a.store[(size_t)ad.slots[j] * a.n + i];
      if (comp_part) combine_two(st.phi_w, ad.rate_w, st.n_phi, a.phi_terms, a.n, i, x, rate_end);
      else x = combine_terms(st.phi_w, st.n_phi, a.phi_terms, a.n, i);
      double2 phi[kMaxWidth + 1];
      phi_functions(x, width, phi);
      // beyond |x| = 3 the recurrence started from exp(x) itself
      const double2 fl = x.x * x.x + x.y * x.y > 9.0 ? phi[0] : cexp(x);
      double fact = 1.0;
      double2 mom[kMaxWidth];
#pragma unroll
      for (int k = 0; k < kMaxWidth; ++k) {
        if (k >= width) break;
        if (k > 0) fact *= (double)k;
        mom[k] = cscale(fact, phi[k + 1]);
        a.moments[(size_t)k * a.n + i] = mom[k];
      }
      a.flow[i] = fl;
      a.exponent[i] = x;
      double2 total = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < kRows; ++k) {
        if (k >= order) break;
        double2 comb = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < kRows; ++j) {
          if (j >= order) break;
          const double c = ad.pred[j][k];
          if (c != 0.0) comb = cadd(comb, cscale(c, rows[j]));
        }
        total = cadd(total, cmul(mom[k], comb));
      }
      lab = cadd(cmul(fl, y), cscale(ad.dz, total));
    } else if (valid && comp_part) {
      combine_two(st.phi_w, ad.rate_w, st.n_phi, a.phi_terms, a.n, i, x, rate_end);
    }
    if (valid && comp_part) {
      // D(z + dz) = sum_p r_p terms_p, contracted always (translate/linop.py:2332-2334), for
      // the corrector's endpoint; it and the predicted state go to the free slot's rows
      // (adams_kernels.py accept), which no row of this trial's stencil reads
      a.rates[(size_t)ad.free_slot * a.n + i] = rate_end;
      // carried rows exp((1 - theta_j) x) ((D(z_j) - x/dz) u_j)   (adams_kernels.py carry)
      const double2 ref = make_double2(x.x / ad.dz, x.y / ad.dz);
#pragma unroll
      for (int j = 0; j < kRows; ++j) {
        if (j >= width - 1) break;
        const double span = 1.0 - ad.nodes[j];
        const double2 diff = csub(rate_rows[j], ref);
        const double2 c = cmul(cexp(cscale(span, x)), cmul(diff, state_rows[j]));
        a.carried[(size_t)j * a.n + i] = c;
        if (j < order) comp = cadd(comp, cscale(ad.comp_pred_main[j], c));
      }
    }
    if (kPair) {
      double2* slot = &handed[trip & 1][warp_in_block >> 1][lane];
      if (!main_part) *slot = comp;
      // the pair's two warps: barrier 1 + pair index, 64 threads
      asm volatile("bar.sync %0, 64;" ::"r"(1 + (warp_in_block >> 1)) : "memory");
      if (main_part) comp = *slot;
    }
    if (valid && main_part) {
      if (ad.compensated) lab = cadd(lab, cscale(ad.dz, comp));
      a.lab[i] = lab;
      if (ad.compensated) a.states[(size_t)ad.free_slot * a.n + i] = lab;
      const int bin = i % a.n_omega;
      if (a.norm_mask[bin]) v[0] += y.x * y.x + y.y * y.y;
    }
  }
  block_partials<1>(v, a.partials + (size_t)kMaxOrders * kNormBlocks, block);
}

// ------------------------------------------------------------------ Adams correct
// Every loop runs to the compile-time bound (kMaxWidth, kMaxOrders) and stops at the
// trial's width and order count, so the operand rows stay in registers.
// kPair: two warps per 32 elements (a single run): the even warp forms the advanced state,
// the odd warp the defect norms; they share only their loads.  With an output record the
// source row is formed here from the transformed streams (the stage-output pass, fused) and
// written by the even warp.
template <bool kPair>
__device__ __forceinline__ void adams_correct_body(const StepArgs& a, int block, const OutputArgs* output) {
  const AdamsDev& ad = staged_adams(a.adams);
  const int width = ad.width, n_orders = ad.n_orders;
  const int lane = threadIdx.x & 31, warp_in_block = threadIdx.x >> 5;
  const bool adv_part = !kPair || !(warp_in_block & 1);
  const bool norm_part = !kPair || (warp_in_block & 1);
  const int groups_per_block = kPair ? (int)(blockDim.x >> 6) : (int)(blockDim.x >> 5);
  const int group = block * groups_per_block + (kPair ? warp_in_block >> 1 : warp_in_block);
  const int n_groups = a.n_blocks * groups_per_block;
  double v[kMaxOrders] = {0.0, 0.0, 0.0};
  for (int i = group * 32 + lane; i < a.n; i += n_groups * 32) {
    double2 xs[kMaxWidth], mom[kMaxWidth];
    if (output) {
      xs[0] = stage_output_value(*output, i);
      if (adv_part) output->out[i] = xs[0];
    } else {
      xs[0] = a.source[i];
    }
#pragma unroll
    for (int j = 1; j < kMaxWidth; ++j) {
      if (j >= width) break;
      xs[j] = a.store[(size_t)ad.slots[j - 1] * a.n + i];
    }
#pragma unroll
    for (int k = 0; k < kMaxWidth; ++k) {
      if (k >= width) break;
      mom[k] = a.moments[(size_t)k * a.n + i];
    }
    double2 endpoint = make_double2(0.0, 0.0);
    double2 carried[kMaxWidth];
    if (ad.compensated) {
      const double2 x = a.exponent[i];
      const double2 ref = make_double2(x.x / ad.dz, x.y / ad.dz);
      // D(z + dz), contracted by the predictor into the free slot's rate row
      const double2 rate_end = a.rates[(size_t)ad.free_slot * a.n + i];
      endpoint = cmul(csub(rate_end, ref), a.lab[i]);
#pragma unroll
      for (int j = 0; j < kMaxWidth - 1; ++j) {
        if (j >= width - 1) break;
        carried[j] = a.carried[(size_t)j * a.n + i];
      }
    }
    if (adv_part) {
      // advanced = flow u + dz sum_k M_k sum_j corr_jk X_j
      double2 total = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < kMaxWidth; ++k) {
        if (k >= width) break;
        double2 comb = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < kMaxWidth; ++j) {
          if (j >= width) break;
          const double c = ad.corr[j][k];
          if (c != 0.0) comb = cadd(comb, cscale(c, xs[j]));
        }
        total = cadd(total, cmul(mom[k], comb));
      }
      double2 adv = cadd(cmul(a.flow[i], a.state[i]), cscale(ad.dz, total));
      if (ad.compensated) {
        double2 c = cscale(ad.comp_corr_main[0], endpoint);
        double2 t = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < kMaxWidth - 1; ++j) {
          if (j >= ad.order) break;
          t = cadd(t, cscale(ad.comp_corr_main[j + 1], carried[j]));
        }
        adv = cadd(adv, cscale(ad.dz, cadd(t, c)));
      }
      a.advanced[i] = adv;
    }
    if (!norm_part) continue;
    const int bin = i % a.n_omega;
    const bool scored = a.norm_mask[bin];
#pragma unroll
    for (int r = 0; r < kMaxOrders; ++r) {
      if (r >= n_orders) break;
      double2 d = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < kMaxWidth; ++k) {
        if (k >= width) break;
        double2 comb = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < kMaxWidth; ++j) {
          if (j >= width) break;
          const double c = ad.rows[r][j][k];
          if (c != 0.0) comb = cadd(comb, cscale(c, xs[j]));
        }
        d = cadd(d, cmul(mom[k], comb));
      }
      d = cscale(ad.dz, d);
      if (ad.compensated) {
        // corrector(k) - predictor(k) of the compensation
        double2 tc = make_double2(0.0, 0.0), tp = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < kMaxWidth - 1; ++j) {
          if (j >= width - 1) break;
          tc = cadd(tc, cscale(ad.comp_corr[r][j + 1], carried[j]));
          tp = cadd(tp, cscale(ad.comp_pred[r][j], carried[j]));
        }
        tc = cadd(tc, cscale(ad.comp_corr[r][0], endpoint));
        d = cadd(d, csub(cscale(ad.dz, tc), cscale(ad.dz, tp)));
      }
      if (scored) v[r] += d.x * d.x + d.y * d.y;
    }
  }
  block_partials<kMaxOrders>(v, a.partials, block);
}

// The compensated rows of the free slot (the predicted state and the rate at the step's
// end) were written by the predictor; accepting adds the source row and the new state.
__device__ __forceinline__ void adams_accept_body(const StepArgs& a, int free_slot, int block) {
  for (int i = block * blockDim.x + threadIdx.x; i < a.n; i += a.n_blocks * blockDim.x) {
    const int bin = i % a.n_omega;
    const double2 adv = a.advanced[i];
    a.state[i] = a.active_mask[bin] ? adv : make_double2(adv.x * 0.0, adv.y * 0.0);
    a.store[(size_t)free_slot * a.n + i] = a.source[i];
  }
}

__device__ __forceinline__ void adams_start_body(const StepArgs& a, int write_rate, int block) {
  const AdamsDev& ad = *a.adams;
  for (int i = block * blockDim.x + threadIdx.x; i < a.n; i += a.n_blocks * blockDim.x) {
    a.store[i] = a.source[i];
    if (write_rate) {
      a.states[i] = a.state[i];
      a.rates[i] = contract_terms(ad.rate0_w, a.stage->n_phi, a.phi_terms, a.n, i);
    }
  }
}

// One run alone: the state is small and the passes are latency-bound, so the blocks are
// narrow (128 threads) to spread the elements over every SM, and each thread keeps all its
// operand rows in registers.  Batched, the passes stream far more than L2 holds and are
// bound by HBM: the register budget is capped so that more warps keep loads in flight.
constexpr int kStepThreads = 128;
__global__ void __launch_bounds__(2 * kStepThreads) k_adams_predict(StepArgs a) {
  adams_predict_body<true>(a, blockIdx.x);
}
__global__ void __launch_bounds__(2 * kStepThreads) k_adams_correct(StepArgs a, const __grid_constant__ OutputArgs o) {
  adams_correct_body<true>(a, blockIdx.x, o.out ? &o : nullptr);
  if (a.norm_arrivals) reduce_if_last(a, kMaxOrders + 1);
}
__global__ void k_adams_accept(StepArgs a, int free_slot) { adams_accept_body(a, free_slot, blockIdx.x); }
__global__ void k_adams_start(StepArgs a, int write_rate) { adams_start_body(a, write_rate, blockIdx.x); }

// batched: items[blockIdx.x] = (run, block of that run)
__global__ void __launch_bounds__(256, 2) k_adams_predict_b(const StepArgs* args, const int2* items,
                                                           const int* flags) {
  const int2 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  adams_predict_body<false>(own_args(args, it.x), it.y);
}
__global__ void __launch_bounds__(256, 4) k_adams_correct_b(const StepArgs* args, const int2* items,
                                                           const int* flags) {
  const int2 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  adams_correct_body<false>(own_args(args, it.x), it.y, nullptr);
}
__global__ void k_adams_accept_b(const StepArgs* args, const int2* items, const int* flags) {
  const int2 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  const StepArgs& a = own_args(args, it.x);
  adams_accept_body(a, a.adams->free_slot, it.y);
}
__global__ void k_adams_start_b(const StepArgs* args, const int2* items, const int* flags) {
  const int2 it = items[blockIdx.x];
  if (!flags[it.x]) return;
  const StepArgs& a = own_args(args, it.x);
  adams_start_body(a, a.states != nullptr, it.y);
}

cudaError_t launch_adams_predict(const StepArgs& a, cudaStream_t s) {
  k_adams_predict<<<a.n_blocks, 2 * kStepThreads, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_adams_correct(const StepArgs& a, const OutputArgs* output, cudaStream_t s) {
  k_adams_correct<<<a.n_blocks, 2 * kStepThreads, 0, s>>>(a, output ? *output : OutputArgs{});
  if (!a.norm_arrivals) k_reduce<<<kMaxOrders + 1, 32, 0, s>>>(a.partials, a.norms, kMaxOrders + 1, a.n_blocks);
  return cudaGetLastError();
}
cudaError_t launch_adams_accept(const StepArgs& a, int free_slot, double2*, cudaStream_t s) {
  k_adams_accept<<<a.n_blocks, 256, 0, s>>>(a, free_slot);
  return cudaGetLastError();
}
cudaError_t launch_adams_start(const StepArgs& a, cudaStream_t s) {
  k_adams_start<<<a.n_blocks, 256, 0, s>>>(a, a.states != nullptr);
  return cudaGetLastError();
}

cudaError_t launch_step_b(int which, const StepArgs* args, const int2* items, const int* flags,
                          int n_items, int n_runs, cudaStream_t s) {
  switch (which) {
    case 0: k_adams_predict_b<<<n_items, 256, 0, s>>>(args, items, flags); break;
    case 1:
      k_adams_correct_b<<<n_items, 256, 0, s>>>(args, items, flags);
      k_reduce_b<<<dim3(kMaxOrders + 1, n_runs), 32, 0, s>>>(args, flags, kMaxOrders + 1);
      break;
    case 2: k_adams_accept_b<<<n_items, 256, 0, s>>>(args, items, flags); break;
    case 3: k_adams_start_b<<<n_items, 256, 0, s>>>(args, items, flags); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// ------------------------------------------------------------------ DOPRI5
struct RkCoeffs {
  double a[8];
  int stage;
  double dz;
};

__global__ void __launch_bounds__(256) k_rk_stage_input(RkArgs a, RkCoeffs c) {
  const StageScalarsDev& st = *a.stage;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const double2 x = combine_terms(st.phi_w, st.n_phi, a.phi_terms, a.n, i);
    double2 comb = make_double2(0.0, 0.0);
    for (int j = 0; j < c.stage; ++j) comb = cadd(comb, cscale(c.a[j], a.stages[(size_t)j * a.n + i]));
    const double2 y = a.state[i];
    const double2 inner = cadd(y, cscale(c.dz, comb));
    a.lab[i] = cmul(cexp(x), inner);
    a.back[i] = cexp(make_double2(-x.x, -x.y));
  }
}

struct RkFinish {
  double b[8], e[8];
  double dz;
};

__global__ void __launch_bounds__(256) k_rk_finish(RkArgs a, RkFinish f) {
  const StageScalarsDev& st = *a.stage;
  double v[3] = {0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    double2 sol = make_double2(0.0, 0.0), err = make_double2(0.0, 0.0);
    for (int j = 0; j < 7; ++j) {
      const double2 k = a.stages[(size_t)j * a.n + i];
      sol = cadd(sol, cscale(f.b[j], k));
      err = cadd(err, cscale(f.e[j], k));
    }
    const double2 x = combine_terms(st.phi_w, st.n_phi, a.phi_terms, a.n, i);
    const double2 prop = cexp(x);
    const double2 y = a.state[i];
    const double2 adv = cmul(prop, cadd(y, cscale(f.dz, sol)));
    const double2 e = cmul(prop, cscale(f.dz, err));
    a.advanced[i] = adv;
    if (a.norm_mask[i % a.n_omega]) {
      v[0] += y.x * y.x + y.y * y.y;
      v[1] += adv.x * adv.x + adv.y * adv.y;
      v[2] += e.x * e.x + e.y * e.y;
    }
  }
  block_partials<3>(v, a.partials, blockIdx.x);
}

__global__ void k_mask_copy(double2* dst, const double2* src, const unsigned char* active, int n,
                            int n_omega) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 v = src[i];
    dst[i] = active[i % n_omega] ? v : make_double2(v.x * 0.0, v.y * 0.0);
  }
}

cudaError_t launch_rk_stage_input(const RkArgs& a, int stage, const double* coeffs, double dz,
                                  cudaStream_t s) {
  RkCoeffs c = {};
  for (int j = 0; j < stage && j < 8; ++j) c.a[j] = coeffs[j];
  c.stage = stage;
  c.dz = dz;
  k_rk_stage_input<<<kNormBlocks, 256, 0, s>>>(a, c);
  return cudaGetLastError();
}

cudaError_t launch_rk_finish(const RkArgs& a, const double* b, const double* e, double dz,
                             double, double, cudaStream_t s) {
  RkFinish f = {};
  for (int j = 0; j < 7; ++j) {
    f.b[j] = b[j];
    f.e[j] = e[j];
  }
  f.dz = dz;
  k_rk_finish<<<kNormBlocks, 256, 0, s>>>(a, f);
  k_reduce<<<3, 32, 0, s>>>(a.partials, a.norms, 3, kNormBlocks);
  return cudaGetLastError();
}

cudaError_t launch_mask_copy(double2* dst, const double2* src, const unsigned char* active, int n,
                             int n_omega, cudaStream_t s) {
  k_mask_copy<<<kNormBlocks, 256, 0, s>>>(dst, src, active, n, n_omega);
  return cudaGetLastError();
}

}  // namespace sp
