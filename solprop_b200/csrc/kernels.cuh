// Argument records and launchers of the device kernels.  Every per-stage scalar a
// kernel reads lives in device memory (StageScalarsDev, AttemptDev), written by one
// host-to-device copy before the launches, so that a captured CUDA graph replays with
// the values of the current attempt.
#pragma once
#include <vector>

#include "sp_common.cuh"

namespace sp {

constexpr int kMaxTerms = 64;      // stage terms of Phi or of the prefactor
constexpr int kMaxWidth = 8;       // Adams interpolation nodes (order 5 + 1, padded)
constexpr int kMaxOrders = 3;      // scored orders per trial
constexpr int kColumnStatus = kMaxOrders + 1;  // norms slot the response column marks on failure
constexpr int kMaxSlots = 8;       // history rows (order + 2)
constexpr int kNormBlocks = 148;   // partial-sum blocks of the norm reductions

// A batched kernel's argument record, copied once per CTA into shared memory: the
// kernel body reads its fields throughout, and from the global array of records each read
// would be a load of its own.  Every thread of the CTA must call it.
template <class T>
__device__ __forceinline__ const T& own_args(const T* args, int run) {
  __shared__ T own;
  if (threadIdx.x == 0) own = args[run];
  __syncthreads();
  return own;
}

constexpr int kMaxChannels = 4;    // field-plasma channels of a gas mixture
constexpr int kMaxRamanRows = 8;   // damped Raman rows over a mixture's components
constexpr int kMaxRamanComponents = 4;

struct StageScalarsDev {
  double z0, z1, taper, density, kerr_density, plasma_density, preionisation, raman_density;
  int n_pre, n_phi;
  double pre_w[kMaxTerms];
  double phi_w[kMaxTerms];   // weights of Phi(z1) - Phi(z0)
  double raman_rates[kMaxRamanRows];  // every component's rows, in order
  // a gas mixture: every plasma channel's density and initial fraction (channel 0 as
  // plasma_density and preionisation), every Raman component's density
  double channel_density[kMaxChannels], channel_preionisation[kMaxChannels];
  double raman_densities[kMaxRamanComponents];
};

// One plasma channel's rate table and constants (translate/ionisation.py:242-323): the
// coefficients are (4, n) in FP64 and the FP32 form's (5, n) table (column_kernels.cu).
template <class R>
struct ChannelTableT {
  const R* rate_coefficients;
  int rate_intervals;
  double log_field_min, d_log_field, field_min, field_max, rate_max;
  double charge_mass_ratio, ionisation_potential;  // the ratio times the electrons per event
};

// One Adams trial's tables (backends/numpy_ref/adams_tables.py, multistep.py _trial).
struct AdamsDev {
  double dz, rtol, atol;
  int order, width, n_orders, compensated;
  int slots[kMaxWidth];                 // history rows read, newest first
  double nodes[kMaxWidth];              // theta_j, newest first
  double pred[kMaxWidth][kMaxWidth];    // Lagrange coefficients c_jk of the predictor
  double corr[kMaxWidth][kMaxWidth];    // corrector over (source, newest, ...)
  double rows[kMaxOrders][kMaxWidth][kMaxWidth];  // defect rows
  // compensation (integrated Adams weights) for the predictor, corrector, per order
  double comp_pred[kMaxOrders][kMaxWidth];        // weights over carried rows
  double comp_corr[kMaxOrders][kMaxWidth + 1];    // [0] endpoint, then carried rows
  double comp_pred_main[kMaxWidth];
  double comp_corr_main[kMaxWidth + 1];
  int free_slot;               // the history row an accepted step writes
  int settle;                  // 1 + the free slot of the accepted trial before this one whose
                               // accept the predictor applies first (0: none pending)
  double rate_w[kMaxTerms];   // D(z + dz) weights (the endpoint rate, "before")
  double rate0_w[kMaxTerms];  // D(z) weights (startup)
};

// The source evaluation's argument records are templates over the real type R of the
// forward transforms and the response column: double in the plain form, float in the
// mixed form, whose inverse transform (the modal field and the absorber's stream), state,
// propagator phase, accumulation and norms stay FP64.
template <class R>
struct InverseArgsT {
  const double2* lab;            // (n_cols, n_omega), FP64 in both forms
  const int* fine_to_coarse;     // (n_to/2 + 1)
  const cplx<R>* twiddles;       // exp(-2 pi i m / n_to), m < n_to / 2
  R* modal_t;                    // (n_cols, n_to)
  R* absorber_stream;            // (n_cols, n_to) or null
  const R* alpha;                // (n_to)
  int n_omega, n_to, log_m, log_n_to;
  int crop_identity;             // crop_index[j] == j for every coarse bin
};
using InverseArgs = InverseArgsT<double>;

// The response column (column_kernels.cu): a warp holds one node's window of kWindow
// samples, a CTA kGroup nodes; a window owns column_owned(K) samples between halos of
// 2K + 1 (K the band filter's half-width, at most kHalo).
constexpr int kWindow = 256;
constexpr int kGroup = 8;
constexpr int kHalo = 8;
__host__ __device__ constexpr int column_lead(int half_width) { return 2 * half_width + 1; }
__host__ __device__ constexpr int column_owned(int half_width) {
  return kWindow - 2 * column_lead(half_width);
}

template <class R>
struct ColumnArgsT {
  const StageScalarsDev* stage;
  const double* modal_t;   // (n_modes, n_to), FP64 in both forms
  const R* synthesis;      // (n_nodes, n_modes)
  const R* projection;     // (n_modes, n_nodes)
  const R* t_window;
  const R* t_window_derivative;
  double* sums0;           // (n_nodes, n_tiles) exposure tile sums
  double* sums1;           // current tile sums
  unsigned long long* ticket;  // tiles handed out so far (n_blocks per evaluation)
  int* flags;              // (n_groups, n_tiles) publication stage of each tile
  double* status;          // set to 1 when a tile gave up waiting
  R* partials;             // (n_groups, 3, n_cols, n_to) projected streams per node group
  int n_modes, n_nodes, n_cols, n_to, n_tiles, n_groups, n_blocks;
  int lead, owned;         // a window's halo and owned samples (column_lead, column_owned)
  int kerr, plasma, band, half_width, rate_intervals;
  double kerr_coefficient, charge_mass_ratio, ionisation_potential, dt;
  double log_field_min, d_log_field, field_min, field_max, rate_max;
  const R* rate_coefficients;
  const R* taps;
  // the modal transform on the GEMM route: the node field the synthesis product wrote,
  // (n_nodes, n_to), and the node streams P, X, Z the projection product reads,
  // (3, n_nodes, n_to); null on the fused route
  const R* node_field;
  R* node_streams;
  // a gas mixture's plasma channels (n_channels > 1; sums0 then holds one plane of
  // (n_nodes, n_tiles) per channel); single-channel problems read the fields above
  int n_channels;
  const ChannelTableT<R>* channels;
};
using ColumnTileArgs = ColumnArgsT<double>;

template <class R>
cudaError_t launch_column(const ColumnArgsT<R>& a, cudaStream_t stream);
// the response column on the GEMM route: node field in, node streams out
template <class R>
cudaError_t launch_column_nodes(const ColumnArgsT<R>& a, cudaStream_t stream);
cudaError_t configure_column_kernels();

template <class R>
struct ForwardArgsT {
  const double* streams;       // rows of n_to (the absorber's), FP64 in both forms
  const R* partials;           // (n_groups, n_partial_rows, n_to): summed for rows below
  int n_groups, n_partial_rows;
  const int* rows;             // which rows to transform
  const long long* crop_index; // (n_omega)
  const cplx<R>* twiddles;
  cplx<R>* spectra;            // rows of n_omega
  int n_to, n_omega, log_m, log_n_to;
  int crop_identity;
};
using ForwardArgs = ForwardArgsT<double>;

struct OutputArgs {
  const StageScalarsDev* stage;
  const double2* spectra;          // (4, n_cols, n_omega): P, gJ, g'J, absorber
  const float2* spectra32;         // the same in complex64 (mixed form), else null
  const double2* prefactor_terms;  // (n_pre, n_cols, n_omega)
  const double* omega;
  const double* omega_window;
  const unsigned char* active_mask;
  const double2* inverse_propagator;  // (n_cols, n_omega) or null
  double2* out;
  int n_cols, n_omega, plasma, absorber;
};

// The envelope route (envelope_kernels.cu): one modal column on one node, one CTA.
constexpr int kMaxEnvelopeSamples = 4096;   // the single CTA's three rows
constexpr int kMaxEnvelopeProducts = 16384;  // the products route's rows
constexpr int kMaxEnvelopeRowF64 = 8192;     // an FP64 row in one CTA's shared memory; longer
                                             // FP64 rows take two halves and a global scratch
struct EnvelopeArgs {
  const StageScalarsDev* stage;
  const double2* lab;            // (n_omega)
  const long long* crop;         // (n_omega): coarse bin -> fine bin
  const double2* twiddles;       // exp(-2 pi i m / (2 n_to)), m < n_to
  const double* t_window;        // (n_to)
  const double* raman_undamped;  // (raman_terms, 2 n_to), or null
  double2* spectra;              // (n_omega): the projected polarisation's spectrum
  double synthesis, projection, dt;
  double kerr_coefficient, kerr_self, kerr_conjugate, raman_fraction;
  int kerr, raman_terms, n_omega, n_to, log_n_to;
};
cudaError_t launch_envelope(const EnvelopeArgs& a, cudaStream_t stream);
cudaError_t configure_envelope_kernels();

cudaError_t configure_source_kernels();

// Plane statistics (statistics_kernels.cu).  out holds [energy: n_cols][omega0: n_cols],
// then at peak_offset the peak power of each mode and of the whole field, then at
// spectrum_offset the energy spectral density (n_omega).  power: (n_cols, n_t) scratch.
constexpr int kStatEnergy = 0, kStatOmega0 = 1;
constexpr int kStatMaxModes = 32;
constexpr int kStatLogRow = 13;  // the longest row one CTA transforms: 8192 points
struct StatisticsArgs {
  const double2* state;         // (n_cols, n_omega)
  const double* power_weight;   // (n_cols, n_omega) or null for one
  const double* omega;          // (n_omega)
  const double2* twiddles;      // exp(-2 pi i m / 2^log_table), m < 2^(log_table - 1)
  double* power;                // (n_cols, n_t)
  double* out;
  int n_modes, n_pol, n_cols, n_omega, n_t, log_m, log_table, envelope;
  double dt;
  int peak_offset, spectrum_offset;
};
cudaError_t configure_statistics_kernels();

// The Raman response on the field grid (raman_kernels.cu), node by node on the GEMM route.
constexpr int kMaxRamanSamples = 4096;  // n_to: the doubled grid's packed transform in one CTA
struct RamanArgs {
  const StageScalarsDev* stage;  // the damping rates and the Raman densities at the stage
  const double* undamped;        // (rows, 2 n_to): every component's rows, in order
  double2* spectrum;             // (n_to + 1): dt rfft of the damped kernel
  const double2* twiddles;       // exp(-2 pi i m / (2 n_to)), m < n_to
  const double* t_window;        // (n_to) the window g
  int n_to, log_n_to;
  int n_components;              // > 1: a mixture, its densities inside the kernel
  int first_row[kMaxRamanComponents + 1];  // component c: rows [first_row[c], first_row[c + 1])
  double fraction[kMaxRamanComponents];
  double dt;
  // two field components: each row's trace and traceless weights (rows, 2), and the
  // kernels formed (1: the trace; 2: trace and traceless, spectra (2, n_to + 1)); null: scalar
  const double* tensor_weights;
  int n_kernels;
  // the mixed form's envelope products: the spectra also in complex64, each scaled by the
  // power of two 2^scale[kernel] that brings its largest bin near one (else null)
  float2* spectrum32;
  int* scale;
  double2* scratch;  // rows above kMaxEnvelopeRowF64: 1.5 n_to complex per kernel
};
cudaError_t configure_raman_kernels();
cudaError_t launch_raman_spectrum(const RamanArgs& a, cudaStream_t s);  // the kernel's spectrum alone

// The envelope grid's modal route with many modes and nodes on the products
// (envelope_modal.cu): complex rows interleaved (re, im), n_to <= kMaxEnvelopeProducts.  R
// is the form's real type: the inverse transform and the modal field are FP64 in both
// forms; the node field and streams, the nodes' responses, the forward transform and the
// spectra are R.
template <class R>
struct EnvModalArgsT {
  const StageScalarsDev* stage;
  const double2* lab;             // (n_cols, n_omega)
  const long long* crop;          // (n_omega): coarse bin -> fine bin
  const double2* twiddles;        // exp(-2 pi i m / (2 n_to)), m < n_to
  const cplx<R>* twiddles_r;      // the same table in the form's type
  const double* t_window;         // (n_to)
  const double* alpha;            // the in-stage absorber's rate (n_to), or null
  double* modal_t;                // (n_cols, 2 n_to): a(t)
  const R* node_field;            // (n_nodes, 2 n_to): E = tau S a
  R* node_streams;                // (n_nodes, 2 n_to): the gated polarisation
  const R* projected;             // (n_cols, 2 n_to): sum W P / tau
  cplx<R>* spectra;               // (4, n_cols, n_omega): P, -, -, absorber
  double2* scratch;               // FP64 rows above kMaxEnvelopeRowF64: 1.5 n_to per row
  const double2* raman_spectrum;  // (raman_kernels, n_to + 1), or null without Raman
  const float2* raman_spectrum32; // the mixed form: the spectra scaled by 2^raman_scale[k], complex64
  const int* raman_scale;
  int n_cols, n_omega, n_to, log_n_to, kerr, raman_mixture;
  int n_components;               // field components per node (1, or 2: rows x, y)
  int raman_kernels;              // two components: 1 (trace) or 2 (trace, traceless)
  double kerr_coefficient, kerr_self, kerr_conjugate;
};
cudaError_t configure_env_modal_kernels();
template <class R>
cudaError_t launch_env_inverse(const EnvModalArgsT<R>& a, cudaStream_t s);
template <class R>
cudaError_t launch_env_nodes(const EnvModalArgsT<R>& a, int n_nodes, cudaStream_t s);
template <class R>
cudaError_t launch_env_forward(const EnvModalArgsT<R>& a, cudaStream_t s);
template <class R>
cudaError_t launch_raman(const RamanArgs& a, const R* field, R* polarisation, int n_nodes, cudaStream_t s);

// The modal transform as products (modal_gemm.cu): the GEMM route.  The mixed form's
// operands are three BF16 parts (hi, mid, lo) per value, panel after panel, rows of kpad.
constexpr int kMaxGemmModes = 1024;  // modal columns the products take (the projection tiles them by 64)
int modal_kpad(int k);              // k rounded up to the products' 64-wide K slices
cudaError_t configure_modal_gemm();
void split3_host(const double* src, int rows, int cols, int ld_out, std::vector<uint16_t>& out);
cudaError_t modal_synthesis_f64(const double* S, const double* modal, double* E, int n_nodes, int n_modes,
                                int n_to, const double* taper, cudaStream_t s);
// scratch the projections' split-K partial tiles need (elements of either form's type)
size_t modal_projection_scratch(int n_modes, int n_nodes, int n_to);
cudaError_t modal_projection_f64(const double* W, const double* node_streams, double* out, int n_streams,
                                 int n_modes, int n_nodes, int n_to, size_t out_stride, const double* taper,
                                 double* scratch, cudaStream_t s);
cudaError_t modal_synthesis_split3(const uint16_t* s_parts, const double* modal, uint16_t* modal_parts, float* E,
                                   int n_nodes, int n_modes, int n_to, int kpad, const double* taper,
                                   double* status, cudaStream_t s);
cudaError_t modal_projection_split3(const uint16_t* w_parts, const float* node_streams, uint16_t* node_parts,
                                    float* out, int n_streams, int n_modes, int n_nodes, int n_to, int kpad,
                                    size_t out_stride, const double* taper, double* status, float* scratch,
                                    cudaStream_t s);
cudaError_t launch_statistics(const StatisticsArgs& a, bool peaks, cudaStream_t s);
int fft_cluster_size(int n_to);
// a single run's transforms: one CTA per row (1) or a cluster of 2, 4 or 8 CTAs per row
int single_transform_width(int n_to, size_t complex_bytes, bool forward);
template <class R>
cudaError_t launch_inverse_cluster(const InverseArgsT<R>& a, int n_cols, int C, cudaStream_t stream);
template <class R>
cudaError_t launch_forward_cluster(const ForwardArgsT<R>& a, int n_rows, int C, cudaStream_t stream);
template <class R>
cudaError_t launch_inverse(const InverseArgsT<R>& a, int n_cols, cudaStream_t stream);
template <class R>
cudaError_t launch_forward(const ForwardArgsT<R>& a, int n_rows, cudaStream_t stream);
cudaError_t launch_output(const OutputArgs& a, cudaStream_t stream);

// ---- batched launches over several runs: items map each block to (run, index)
cudaError_t configure_cluster_fft();
// flags[run] != 0 selects the runs a launch serves; other items return at once
template <class R>
cudaError_t launch_inverse_b(const InverseArgsT<R>* args, const int2* items, const int* flags,
                             int n_items, int n_to, cudaStream_t stream);
template <class R>
cudaError_t launch_forward_b(const ForwardArgsT<R>* args, const int2* items, const int* flags,
                             int n_items, int n_to, cudaStream_t stream);
// batched transforms over clusters of C = 2, 4 or 8 CTAs (the scan's autotuner picks);
// their dynamic shared memory (cluster_transform_smem) may be up to kClusterSmem
constexpr size_t kClusterSmem = 200 * 1024;
size_t cluster_transform_smem(int n_to, int C, size_t complex_bytes, bool forward);
template <class R>
cudaError_t launch_inverse_cluster_b(const InverseArgsT<R>* args, const int2* items, const int* flags,
                                     int n_items, int n_to, int C, cudaStream_t stream);
template <class R>
cudaError_t launch_forward_cluster_b(const ForwardArgsT<R>* args, const int2* items, const int* flags,
                                     int n_items, int n_to, int C, cudaStream_t stream);
cudaError_t launch_output_b(const OutputArgs* args, const int2* items, const int* flags,
                            int n_items, cudaStream_t stream);
template <class R>
cudaError_t launch_column_b(const ColumnArgsT<R>* args, const int4* items, const int* flags,
                            int n_items, cudaStream_t stream);
// the same column, one CTA per (run, node group) walking the run's tiles in order; each
// group leaves its own partial rows (ForwardArgsT::n_groups = the column's n_groups)
template <class R>
cudaError_t launch_column_sweep_b(const ColumnArgsT<R>* args, const int4* items, const int* flags,
                                  int n_items, cudaStream_t stream);

// ---- stepping kernels (step_kernels.cu)
struct StepArgs {
  const StageScalarsDev* stage;
  const AdamsDev* adams;
  const double2* phi_terms;   // (n_phi, n)
  const unsigned char* norm_mask;
  const unsigned char* active_mask;
  int n, n_omega;             // state elements, bins per column
  double2* state;             // (n)
  double2* store;             // (n_slots, n)
  double2* states;            // compensated: (n_slots, n)
  double2* rates;             // compensated: (n_slots, n)
  double2* moments;           // (width, n)
  double2* flow;              // (n)
  double2* exponent;          // (n)
  double2* carried;           // compensated: (width - 1, n)
  double2* lab;               // (n)
  double2* source;            // (n)
  double2* advanced;          // (n)
  double* partials;           // (kMaxOrders + 2, kNormBlocks)
  double* norms;              // (kMaxOrders + 2)
  int n_blocks;               // blocks of the grid-stride loops (<= kNormBlocks)
  unsigned* norm_arrivals;    // single run: the corrector's block count (its last block
                              // reduces the partials); null: a separate reduction launch
};

cudaError_t launch_adams_predict(const StepArgs& a, cudaStream_t stream);
// with an output record (non-null), the corrector forms the source row itself: the stage
// output pass of the source evaluation before it, fused
cudaError_t launch_adams_correct(const StepArgs& a, const OutputArgs* output, cudaStream_t stream);
cudaError_t launch_adams_accept(const StepArgs& a, int free_slot, double2* rate_out, cudaStream_t s);
cudaError_t launch_adams_start(const StepArgs& a, cudaStream_t stream);
// batched step kernels: which = 0 predict, 1 correct (+ reduction), 2 accept, 3 start
cudaError_t launch_step_b(int which, const StepArgs* args, const int2* items, const int* flags,
                          int n_items, int n_runs, cudaStream_t stream);

struct RkArgs {
  const StageScalarsDev* stage;
  const double2* phi_terms;
  const unsigned char* norm_mask;
  const unsigned char* active_mask;
  int n, n_omega, n_phi;
  double2* state;
  double2* stages;        // (7, n)
  double2* lab;
  double2* back;          // inverse propagator of the stage
  double2* advanced;
  double* partials;
  double* norms;
};
// stage_input: lab = exp(x)(y + dz sum_j a_ij k_j), back = exp(-x); coefficients by value
cudaError_t launch_rk_stage_input(const RkArgs& a, int stage, const double* coeffs, double dz,
                                  cudaStream_t stream);
cudaError_t launch_rk_finish(const RkArgs& a, const double* b, const double* e, double dz,
                             double rtol, double atol, cudaStream_t stream);
cudaError_t launch_mask_copy(double2* dst, const double2* src, const unsigned char* active,
                             int n, int n_omega, cudaStream_t stream);

}  // namespace sp
