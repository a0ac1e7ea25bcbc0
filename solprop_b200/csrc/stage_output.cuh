// The stage output of one element (translate/stage.py:292-342 for the prefactor;
// backends/numpy_ref/passes/transforms.py for the assembly): the prefactor, the held
// plasma assembly P + X / (i w) - Z / (i w)^2 on the band, the spectral window, the
// absorber's row and the inverse propagator.  Shared by the stage-output pass and the
// single-run corrector, which forms its source row itself.
#pragma once
#include "kernels.cuh"

namespace sp {

template <class CS>
__device__ __forceinline__ double2 stage_output_value(const OutputArgs& a, const CS* spectra, int idx) {
  const int total = a.n_cols * a.n_omega;
  const int j = idx % a.n_omega;
  const StageScalarsDev& st = *a.stage;
  // every operand is loaded before any is used (the streams of bins off the band too, which
  // the selections below drop), so that the loads overlap
  const double2 spec0 = to_d2(spectra[idx]);  // stream 0: P
  const double2 xs = a.plasma ? to_d2(spectra[(size_t)1 * total + idx]) : make_double2(0.0, 0.0);
  const double2 zs = a.plasma ? to_d2(spectra[(size_t)2 * total + idx]) : make_double2(0.0, 0.0);
  const double2 ab_row = a.absorber ? to_d2(spectra[(size_t)3 * total + idx]) : make_double2(0.0, 0.0);
  const double2 propagator = a.inverse_propagator ? a.inverse_propagator[idx] : make_double2(0.0, 0.0);
  const bool active = a.active_mask[j];
  const double omega = a.omega[j], window = a.omega_window[j];
  double2 pre;
  if (st.n_pre == 1) {
    pre = a.prefactor_terms[idx];
    if (st.pre_w[0] != 1.0) pre = cscale(st.pre_w[0], pre);
  } else {
    pre = make_double2(0.0, 0.0);
    const int n_pre = st.n_pre;
#pragma unroll 8  // eight terms' loads in flight at a time
    for (int p = 0; p < n_pre; ++p)
      pre = cadd(pre, cscale(st.pre_w[p], a.prefactor_terms[(size_t)p * total + idx]));
  }
  double2 spec = spec0;
  if (a.plasma && active) {
    const double2 qv = make_double2(0.0, omega);
    const double2 q2 = cmul(qv, qv);
    spec = cadd(spec, csub(cdiv(xs, qv), cdiv(zs, q2)));
  }
  double2 normalised = cmul(cscale(window, pre), spec);
  if (a.absorber) {
    const double2 ab = active ? ab_row : make_double2(0.0, 0.0);
    normalised = cadd(normalised, ab);
  }
  if (a.inverse_propagator) normalised = cmul(propagator, normalised);
  return normalised;
}

__device__ __forceinline__ double2 stage_output_value(const OutputArgs& a, int idx) {
  return a.spectra32 ? stage_output_value(a, a.spectra32, idx) : stage_output_value(a, a.spectra, idx);
}

}  // namespace sp
