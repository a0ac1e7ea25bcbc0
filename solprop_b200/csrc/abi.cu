// The C ABI of the library (include/solprop_b200.h): problem, workspace and session
// objects, the host evaluation of the stage scalars (translate/stage.py:413-503, the
// Clenshaw pass of translate/chebyshev.py:138-198), and the two marches -- exponential
// Adams (backends/adams_core.py, numpy_ref/marches/adams.py) and DOPRI5
// (backends/rk_core.py, numpy_ref/marches/runge_kutta.py) -- which decide on the host
// from the norms the device reduces, one device synchronisation per attempt, as the
// reference's native march does (native/src/march/adams_march.cpp, rk_march.cpp).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/solprop_b200.h"
#include "host_pool.hpp"
#include "kernels.cuh"

using namespace sp;

namespace {

thread_local std::string g_error;

struct Failure : std::runtime_error {
  sp_status code;
  int reason;  // SP_REASON_* a session reports for it
  Failure(sp_status c, const std::string& m, int r = SP_REASON_ERROR)
      : std::runtime_error(m), code(c), reason(r) {}
};

#define CUDA_CHECK(call)                                                                    \
  do {                                                                                      \
    cudaError_t _e = (call);                                                                \
    if (_e != cudaSuccess)                                                                  \
      throw Failure(SP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e));       \
  } while (0)

template <class F>
sp_status guarded(F&& f) {
  try {
    f();
    return SP_OK;
  } catch (const Failure& e) {
    g_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_error = e.what();
    return SP_ERR_ARGUMENT;
  }
}

// The source kernels' shared-memory limits are attributes of one device: every entry point
// that launches them sets them once per device, with that device current.
constexpr int kMaxDevices = 64;
std::mutex g_configure_mutex;
bool g_configured[kMaxDevices];

void ensure_configured(int device) {
  if (device < 0 || device >= kMaxDevices) throw Failure(SP_ERR_ARGUMENT, "device index out of range");
  std::lock_guard<std::mutex> lock(g_configure_mutex);
  if (g_configured[device]) return;
  CUDA_CHECK(configure_source_kernels());
  CUDA_CHECK(configure_statistics_kernels());
  CUDA_CHECK(configure_modal_gemm());
  CUDA_CHECK(configure_raman_kernels());
  CUDA_CHECK(configure_env_modal_kernels());
  g_configured[device] = true;
}

// Runs a callable when the scope ends, however it ends.
template <class F>
struct ScopeExit {
  F f;
  ~ScopeExit() { f(); }
};
template <class F>
ScopeExit<F> on_scope_exit(F f) { return ScopeExit<F>{f}; }

// ------------------------------------------------------------------ piecewise tables
struct Table {
  int n_int = 0, n_deg = 0, n_val = 0;
  std::vector<double> bp, c;
  bool present() const { return n_int > 0; }
  void load(const sp_table& t) {
    n_int = t.n_intervals;
    n_deg = t.n_deg;
    n_val = t.n_values;
    if (!n_int) return;
    if (!t.breakpoints || !t.coefficients || n_deg < 1 || n_val < 1)
      throw Failure(SP_ERR_ARGUMENT, "a table without breakpoints or coefficients");
    bp.assign(t.breakpoints, t.breakpoints + n_int + 1);
    c.assign(t.coefficients, t.coefficients + (size_t)n_int * n_deg * n_val);
  }
  int interval(double z) const {
    // searchsorted(edges, z, side="right") - 1, clamped (chebyshev.py:171-180)
    int lo = 0, hi = n_int + 1;
    while (lo < hi) {
      int mid = (lo + hi) / 2;
      if (bp[mid] <= z) lo = mid + 1; else hi = mid;
    }
    return std::min(std::max(lo - 1, 0), n_int - 1);
  }
  // chebval by Clenshaw, operation for operation (chebyshev.py:182-198)
  void eval_interval(int k, double z, double* out) const {
    const double lo = bp[k], hi = bp[k + 1];
    const double x = (2.0 * z - lo - hi) / (hi - lo);
    const double* ck = c.data() + (size_t)k * n_deg * n_val;
    for (int j = 0; j < n_val; ++j) {
      if (n_deg == 1) { out[j] = ck[j] + 0.0 * x; continue; }
      if (n_deg == 2) { out[j] = ck[j] + ck[n_val + j] * x; continue; }
      const double x2 = 2 * x;
      double c0 = ck[(n_deg - 2) * n_val + j], c1 = ck[(n_deg - 1) * n_val + j];
      for (int i = 3; i <= n_deg; ++i) {
        double tmp = c0;
        c0 = ck[(n_deg - i) * n_val + j] - c1;
        c1 = tmp + c1 * x2;
      }
      out[j] = c0 + c1 * x;
    }
  }
  void eval(double z, double* out) const { eval_interval(interval(z), z, out); }
  void eval_before(double z, double* out) const {
    int k = interval(z);
    if (k > 0 && z <= bp[k]) --k;
    eval_interval(k, z, out);
  }
  double scalar(double z, double dflt) const {
    if (!present()) return dflt;
    double v;
    eval(z, &v);
    return v;
  }
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  bool owned = true;
  void alloc(size_t count) {
    n = count;
    if (count) CUDA_CHECK(cudaMalloc(&p, count * sizeof(T)));
  }
  void upload(const void* host, size_t count, cudaStream_t s) {
    alloc(count);
    if (count) CUDA_CHECK(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void zero(cudaStream_t s) {
    if (n) CUDA_CHECK(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  ~DevBuf() {
    if (p && owned) cudaFree(p);
  }
};

int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

}  // namespace

// ====================================================================== problem
struct sp_problem {
  sp_problem_desc d{};
  int n_cols = 0, n = 0, n_fine = 0;
  int crop_identity = 0;  // crop_index[j] == j for every coarse bin
  std::vector<double> omega, omega_window, t_window, t_window_d, carrier, alpha;
  std::vector<long long> crop;
  std::vector<unsigned char> active, norm;
  std::vector<double> phi_terms, pre_terms, synthesis, projection, rate_coeff, taps;
  Table phi_weights, phi_rate, pre_weights, density, kerr_density, plasma_density, preion, taper;
  Table raman_rates[kMaxRamanRows], raman_density;
  std::vector<double> raman_undamped;  // (rows, 2 n_to): every Raman component's rows, in order
  // a gas mixture (n_extra_channels > 0): every plasma channel, channel 0 the descriptor's
  struct Channel {
    double charge_mass_ratio, ionisation_potential, log_field_min, d_log_field, field_min, field_max,
        rate_max;
    std::vector<double> coefficients;  // (4, n)
    Table density, preion;
  };
  std::vector<Channel> channels;
  // every Raman component (component 0 the descriptor's): rows, fraction, density
  std::vector<int> raman_first_row{0};
  std::vector<double> raman_fraction;
  std::vector<Table> raman_densities;
  std::vector<double> raman_weights;  // two components: (rows, 2) trace and traceless weights
  int raman_kernels = 1;              // 2 when any row has a traceless weight
  int raman_rows() const { return raman_first_row.back(); }
};

static void validate(const sp_problem_desc* d) {
  auto need = [](bool ok, const char* what) {
    if (!ok) throw Failure(SP_ERR_ARGUMENT, what);
  };
  need(d != nullptr, "problem description is NULL");
  need(d->n_modes >= 1 && d->n_pol >= 1 && d->n_omega >= 2, "bad state shape");
  need(d->n_to >= 2 * kWindow && (d->n_to & (d->n_to - 1)) == 0,
       "n_to must be a power of two >= 512 (mixed radices and shorter rows are not built)");
  need(d->n_nodes >= 1 && d->synthesis && d->projection, "synthesis/projection required");
  need(d->omega && d->crop_index && d->active_mask && d->norm_mask && d->omega_window &&
           d->t_window && d->t_window_derivative,
       "grid arrays required");
  need(d->n_phi_terms >= 1 && d->n_phi_terms <= kMaxTerms && d->phi_terms, "phi terms");
  need(d->n_prefactor_terms >= 1 && d->n_prefactor_terms <= kMaxTerms && d->prefactor_terms,
       "prefactor terms");
  if (d->grid_kind != 0 && d->grid_kind != 1) throw Failure(SP_ERR_ARGUMENT, "unknown grid kind");
  const bool envelope = d->grid_kind == 1;
  if (d->n_pol != 1 || (d->n_pol_transform != 1 && d->n_pol_transform != 2))
    throw Failure(SP_ERR_REFUSED, "a state with two polarisation columns is not built");
  if (d->n_pol_transform == 2 && !envelope)
    throw Failure(SP_ERR_REFUSED, "two field components on the field grid (vector Kerr, tensor Raman) are not built");
  if (d->n_pol_transform == 2 && d->raman_enabled) {
    need(d->raman_tensor_weights != nullptr, "two components' Raman needs its tensor weights");
    for (int c = 0; c < d->n_extra_raman; ++c)
      need(d->extra_raman[c].tensor_weights != nullptr, "two components' Raman needs its tensor weights");
  }
  if (d->n_modes * d->n_pol > kMaxGemmModes)
    throw Failure(SP_ERR_REFUSED, "more than 1024 modal columns");
  if (envelope) {
    // the envelope route: one modal column on one node in one CTA (the single-mode GNLSE),
    // or many modes and nodes on the products
    if (d->n_to > kMaxEnvelopeProducts)
      throw Failure(SP_ERR_REFUSED, "the envelope grid above 16384 samples is not built yet");
    if (d->plasma_enabled) throw Failure(SP_ERR_REFUSED, "envelope plasma is not built yet");
    if (d->kerr_enabled && (!d->kerr_analytic || d->kerr_take_real ||
                            (d->carrier && d->kerr_harmonic != 0.0)))
      throw Failure(SP_ERR_REFUSED, "the envelope route takes the analytic Kerr cubic without a harmonic");
    if (d->raman_enabled) {
      need(d->raman_terms >= 1 && d->raman_terms <= 4 && d->raman_undamped, "Raman terms");
      if (d->raman_thg) throw Failure(SP_ERR_REFUSED, "a third-harmonic Raman drive on the envelope grid");
    }
    if (d->n_extra_raman) throw Failure(SP_ERR_REFUSED, "a Raman mixture on the envelope grid");
  } else {
    if (d->raman_enabled) {
      need(d->raman_terms >= 1 && d->raman_terms <= 4 && d->raman_undamped, "Raman terms");
      if (!d->raman_thg)
        throw Failure(SP_ERR_REFUSED, "the field grid's Raman drive without the harmonic (an analytic signal)");
      if (d->n_to > kMaxRamanSamples)
        throw Failure(SP_ERR_REFUSED, "field-grid Raman above 4096 fine samples");
    }
    if (d->kerr_enabled && d->kerr_analytic)
      throw Failure(SP_ERR_REFUSED, "the analytic Kerr cubic belongs to the envelope grid");
  }
  need(d->n_extra_channels >= 0 && d->n_extra_channels < kMaxChannels, "at most four plasma channels");
  need(d->n_extra_channels == 0 || (d->plasma_enabled && d->extra_channels), "mixture channels");
  for (int c = 0; c < d->n_extra_channels; ++c)
    need(d->extra_channels[c].rate_intervals >= 1 && d->extra_channels[c].rate_coefficients &&
             d->extra_channels[c].d_log_field > 0.0,
         "a mixture channel's rate table");
  need(d->n_extra_raman >= 0 && d->n_extra_raman < kMaxRamanComponents, "at most four Raman components");
  need(d->n_extra_raman == 0 || (d->raman_enabled && d->extra_raman), "mixture Raman components");
  {
    int rows = d->raman_enabled ? d->raman_terms : 0;
    for (int c = 0; c < d->n_extra_raman; ++c) {
      need(d->extra_raman[c].terms >= 1 && d->extra_raman[c].terms <= 4 && d->extra_raman[c].undamped,
           "a mixture component's Raman terms");
      rows += d->extra_raman[c].terms;
    }
    if (rows > kMaxRamanRows) throw Failure(SP_ERR_REFUSED, "more than eight damped Raman rows in a mixture");
  }
  if (d->plasma_enabled) {
    need(d->rate_intervals >= 1 && d->rate_coefficients, "rate table");
    need(d->n_taps >= 1 && d->n_taps - 1 <= kHalo && d->taps,
         "running-integral taps: a band-rule half-width above 8 is not built");
  }
  if (d->absorber_in_stage) need(d->temporal_absorber_fine != nullptr, "absorber rate");
  const long long n_fine = envelope ? d->n_to : d->n_to / 2 + 1;
  for (int j = 0; j < d->n_omega; ++j) {
    const long long k = d->crop_index[j];
    need(k >= 0 && k < n_fine, "crop_index outside the fine spectrum");
  }
}

// ====================================================================== workspace
struct sp_workspace {
  const sp_problem* P = nullptr;
  int device = 0;
  cudaStream_t stream = nullptr;
  int log_m = 0, log_n_to = 0, launches = 0, n_rows = 0;
  DevBuf<double2> phi_terms, pre_terms, twiddles, lab, out, spectra;
  DevBuf<double> omega, omega_window, t_window, t_window_d, alpha, synthesis, projection,
      rate_coeff, taps, modal_t, streams, sums0, sums1, proj;
  DevBuf<long long> crop;
  DevBuf<int> fine_to_coarse, rows, chain_flags;
  DevBuf<unsigned long long> ticket;  // the response column's tile counter
  DevBuf<double2> env_twiddles;       // envelope route: exp(-2 pi i m / (2 n_to)), m < n_to
  DevBuf<double> raman_undamped, raman_weights;
  DevBuf<double> stat_power, stat_out, stat_weight;  // plane statistics, on first use
  DevBuf<double2> raman_spectrum;  // field-grid Raman: the damped kernel's spectrum (n_to + 1)
  DevBuf<float2> raman_spectrum32;  // the envelope products' mixed form: the spectra scaled, complex64
  DevBuf<int> raman_scale;          // ... and their powers of two
  DevBuf<double2> env_scratch;      // the envelope products' FP64 rows above 8192 samples: 1.5 n_to per row
  DevBuf<double2> raman_scratch;    // ... and the Raman kernel's spectra
  DevBuf<ChannelTableT<double>> channels;  // a mixture's plasma channels (rate_coeff holds their tables)
  // the modal transform as products (SP_MODAL_GEMM): the node field and streams in HBM;
  // the mixed form's operands in three BF16 parts, rows padded to kpad
  bool gemm = false;
  int kpad_modes = 0, kpad_nodes = 0;
  DevBuf<double> node_field, node_streams;
  DevBuf<uint16_t> s_parts, w_parts, modal_parts, node_parts;
  DevBuf<double> proj_scratch;  // the projections' split-K partial tiles (FP32 in the mixed form)
  // the mixed-precision form's FP32 copies of the source evaluation's buffers
  int precision = SP_PRECISION_FP64;
  struct {
    DevBuf<float2> twiddles, spectra;
    DevBuf<float> t_window, t_window_d, synthesis, projection, rate_coeff, taps, proj;
    DevBuf<float> node_field, node_streams;
    DevBuf<ChannelTableT<float>> channels;
    DevBuf<float2> env_twiddles;
  } f32;
  DevBuf<unsigned char> active, norm;
  DevBuf<StageScalarsDev> stage;   // kStageSlots slots
  StageScalarsDev* h_stage = nullptr;  // pinned
  // stepping state
  DevBuf<double2> state, store, states, rates, moments, flow, exponent, carried, src, adv,
      stages, back;
  DevBuf<AdamsDev> adams;
  AdamsDev* h_adams = nullptr;       // pinned
  // The trial's table then the stage slots, in one pinned and one device allocation
  // (h_adams / h_stage and adams / stage are views into them), so that a single copy
  // carries an attempt's tables
  unsigned char* h_tables = nullptr;
  DevBuf<unsigned char> tables;
  DevBuf<double> partials, norms;
  DevBuf<unsigned> norm_arrivals;    // the single-run corrector's block count (zero between launches)
  double* h_norms = nullptr;         // pinned
  // Recorded after every asynchronous copy out of h_stage and h_adams: the host waits on
  // it before it writes them again, so that a copy still in flight never reads the next
  // attempt's tables.
  cudaEvent_t host_tables_free = nullptr;
  bool tables_in_flight = false;  // a copy out of h_stage / h_adams issued since the last wait
  // The free slot of a single run's accepted trial whose accept (the new state, the source
  // row) the next predictor applies, or -1: settle_accept() writes it at once for anything
  // else that reads the state or the history rows.
  int pending_accept = -1;
  // A single run's Adams attempt phase (table uploads, predict, source, correct, the norms'
  // read-back), captured once and replayed: its launches and arguments are the same for
  // every attempt, the tables' contents change in the pinned buffers the copies read
  cudaGraph_t attempt_graph = nullptr;
  cudaGraphExec_t attempt_exec = nullptr;
  static constexpr int kStageSlots = 10;
  // per-kernel timing (sp_session_set_timing)
  bool timing = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  size_t ev_next = 0;
  double t_ms[SP_K_COUNT] = {};
  int64_t t_count[SP_K_COUNT] = {};
  cudaEvent_t next_event() {
    if (ev_next == ev_pool.size()) {
      cudaEvent_t e;
      CUDA_CHECK(cudaEventCreate(&e));
      ev_pool.push_back(e);
    }
    return ev_pool[ev_next++];
  }
  void flush_timing() {
    if (pending.empty()) return;
    CUDA_CHECK(cudaStreamSynchronize(stream));
    for (auto& p : pending) {
      float ms = 0.f;
      CUDA_CHECK(cudaEventElapsedTime(&ms, p.second.first, p.second.second));
      t_ms[p.first] += ms;
      t_count[p.first] += 1;
    }
    pending.clear();
    ev_next = 0;
  }
  // A borrowed workspace is a view over memory it does not own (the no-allocation entry
  // point's): its stream and host scalars belong to others, and it frees nothing.
  bool borrowed = false;
  ~sp_workspace() {
    if (borrowed) return;
    if (attempt_exec) cudaGraphExecDestroy(attempt_exec);
    if (attempt_graph) cudaGraphDestroy(attempt_graph);
    for (auto e : ev_pool) cudaEventDestroy(e);
    if (host_tables_free) cudaEventDestroy(host_tables_free);
    if (stream) cudaStreamSynchronize(stream);
    if (h_tables) cudaFreeHost(h_tables);
    if (h_norms) cudaFreeHost(h_norms);
    if (stream) cudaStreamDestroy(stream);
  }
};

// Records events around one launch family while timing is on.
struct KernelTimer {
  sp_workspace* ws;
  int kind;
  cudaEvent_t end{};
  KernelTimer(sp_workspace* w, int k) : ws(w), kind(k) {
    if (!ws->timing) return;
    cudaEvent_t start = ws->next_event();
    end = ws->next_event();
    CUDA_CHECK(cudaEventRecord(start, ws->stream));
    ws->pending.push_back({kind, {start, end}});
  }
  ~KernelTimer() {
    if (ws->timing) cudaEventRecord(end, ws->stream);
  }
};

// The pinned stage and Adams tables are copied to the device asynchronously: before the
// host writes them, it waits for the copies already issued from them; after issuing
// copies, it marks them.
// A wait only follows a release: the batched scan reads the per-run tables on the host and
// issues no copy from them, so its prepares make no driver call here.
static void claim_host_tables(sp_workspace* ws) {
  if (ws->host_tables_free && ws->tables_in_flight) {
    CUDA_CHECK(cudaEventSynchronize(ws->host_tables_free));
    ws->tables_in_flight = false;
  }
}
static void release_host_tables(sp_workspace* ws) {
  if (ws->host_tables_free) {
    CUDA_CHECK(cudaEventRecord(ws->host_tables_free, ws->stream));
    ws->tables_in_flight = true;
  }
}

// host evaluation of one stage's scalars into slot `slot` of the pinned buffer
static void fill_stage(sp_workspace* ws, int slot, double z0, double z1) {
  const sp_problem& P = *ws->P;
  claim_host_tables(ws);
  StageScalarsDev& s = ws->h_stage[slot];
  std::memset(&s, 0, sizeof(s));
  s.z0 = z0;
  s.z1 = z1;
  s.density = P.density.scalar(z1, 1.0);
  s.taper = P.taper.scalar(z1, 1.0);
  s.kerr_density = P.kerr_density.present() ? P.kerr_density.scalar(z1, 1.0) : s.density;
  s.plasma_density = P.plasma_density.scalar(z1, s.density);
  s.preionisation = P.preion.scalar(z1, 0.0);
  if (P.d.raman_enabled) {  // translate/stage.py scalars: the damping rates and the density
    for (int r = 0; r < P.raman_rows(); ++r) s.raman_rates[r] = P.raman_rates[r].scalar(z1, 0.0);
    s.raman_density = P.raman_density.scalar(z1, s.density);
    for (size_t c = 0; c < P.raman_densities.size(); ++c)
      s.raman_densities[c] = P.raman_densities[c].scalar(z1, s.density);
  }
  s.channel_density[0] = s.plasma_density;
  s.channel_preionisation[0] = s.preionisation;
  for (size_t c = 1; c < P.channels.size(); ++c) {  // a mixture's further channels
    s.channel_density[c] = P.channels[c].density.scalar(z1, s.density);
    s.channel_preionisation[c] = P.channels[c].preion.scalar(z1, 0.0);
  }
  s.n_phi = P.d.n_phi_terms;
  s.n_pre = P.d.n_prefactor_terms;
  if (!P.d.phi_expansion) {
    s.phi_w[0] = z1 - z0;  // Phi(z) = D z: the distance (translate/stage.py:731-734)
  } else {
    double w1[kMaxTerms], w0[kMaxTerms];
    P.phi_weights.eval(z1, w1);
    P.phi_weights.eval(z0, w0);
    for (int p = 0; p < s.n_phi; ++p) s.phi_w[p] = w1[p] - w0[p];
  }
  if (P.pre_weights.present()) P.pre_weights.eval(z1, s.pre_w);
  else s.pre_w[0] = 1.0;
}

static void upload_stages(sp_workspace* ws, int count) {
  CUDA_CHECK(cudaMemcpyAsync(ws->stage.p, ws->h_stage, count * sizeof(StageScalarsDev),
                             cudaMemcpyHostToDevice, ws->stream));
  release_host_tables(ws);
}

// The response column's tiles: windows of kWindow samples owning column_owned(K) each.
static int column_halfwidth(const sp_problem_desc& d) { return d.plasma_enabled ? d.n_taps - 1 : 0; }
static int column_tiles(const sp_problem_desc& d) {
  const int owned = column_owned(column_halfwidth(d));
  return (d.n_to + owned - 1) / owned;
}

// The buffers one source evaluation reads and writes, in the evaluation's real type.
template <class R>
struct SourceView {
  const cplx<R>* twiddles;
  cplx<R>* spectra;
  const R *t_window, *t_window_d, *synthesis, *projection, *rate_coeff, *taps;
  R* proj;
};

template <class R>
static SourceView<R> source_view(const sp_workspace* ws);
template <>
SourceView<double> source_view<double>(const sp_workspace* ws) {
  return {ws->twiddles.p, ws->spectra.p, ws->t_window.p, ws->t_window_d.p, ws->synthesis.p,
          ws->projection.p, ws->rate_coeff.p, ws->taps.p, ws->proj.p};
}
template <>
SourceView<float> source_view<float>(const sp_workspace* ws) {
  const auto& f = ws->f32;
  return {f.twiddles.p, f.spectra.p, f.t_window.p, f.t_window_d.p, f.synthesis.p,
          f.projection.p, f.rate_coeff.p, f.taps.p, f.proj.p};
}

// The argument records of one source evaluation on a workspace.  The inverse transform
// is FP64 in both forms (the FP32 noise floor of the modal field would swamp the
// absorber's stream, which lives where the field is weak).
static InverseArgs inverse_args(const sp_workspace* ws, const double2* lab, bool absorber) {
  const sp_problem& P = *ws->P;
  const sp_problem_desc& d = P.d;
  return InverseArgs{lab, ws->fine_to_coarse.p, ws->twiddles.p, ws->modal_t.p,
                     absorber ? ws->streams.p + (size_t)3 * P.n_cols * d.n_to : nullptr,
                     ws->alpha.p, d.n_omega, d.n_to, ws->log_m, ws->log_n_to, P.crop_identity};
}

template <class R = double>
static ColumnArgsT<R> column_args(const sp_workspace* ws, const StageScalarsDev* stage) {
  const sp_problem& P = *ws->P;
  const sp_problem_desc& d = P.d;
  const SourceView<R> v = source_view<R>(ws);
  ColumnArgsT<R> ca{};
  ca.stage = stage;
  ca.modal_t = ws->modal_t.p;
  ca.synthesis = v.synthesis;
  ca.projection = v.projection;
  ca.t_window = v.t_window;
  ca.t_window_derivative = v.t_window_d;
  ca.sums0 = ws->sums0.p;
  ca.sums1 = ws->sums1.p;
  ca.ticket = ws->ticket.p;
  ca.flags = ws->chain_flags.p;
  ca.status = ws->norms.p + kColumnStatus;
  ca.partials = v.proj;
  ca.n_modes = d.n_modes;
  ca.n_nodes = d.n_nodes;
  ca.n_cols = P.n_cols;
  ca.n_to = d.n_to;
  ca.half_width = column_halfwidth(d);
  ca.lead = column_lead(ca.half_width);
  ca.owned = column_owned(ca.half_width);
  ca.n_tiles = column_tiles(d);
  ca.n_groups = (d.n_nodes + kGroup - 1) / kGroup;
  ca.n_blocks = ca.n_tiles * ca.n_groups;
  ca.kerr = d.kerr_enabled;
  ca.plasma = d.plasma_enabled;
  ca.band = d.band;
  ca.rate_intervals = d.rate_intervals;
  ca.kerr_coefficient = d.kerr_coefficient;
  ca.charge_mass_ratio = d.charge_mass_ratio;
  ca.ionisation_potential = d.ionisation_potential;
  ca.dt = d.dt_fine;
  ca.log_field_min = d.log_field_min;
  ca.d_log_field = d.d_log_field;
  ca.field_min = d.field_min;
  ca.field_max = d.field_max;
  ca.rate_max = d.rate_max;
  ca.rate_coefficients = v.rate_coeff;
  ca.taps = v.taps;
  ca.n_channels = std::max<int>(1, (int)P.channels.size());
  if constexpr (sizeof(R) == 8)
    ca.channels = ws->channels.p;
  else
    ca.channels = ws->f32.channels.p;
  return ca;
}

// stream rows: P [0, nc), gJ [nc, 2nc), g'J [2nc, 3nc), absorber [3nc, 4nc). The row
// list holds [0, 4nc) for plasma runs and, at offset 4nc, [P rows, absorber rows].
static int forward_rows(const sp_workspace* ws, bool absorber) {
  const sp_problem& P = *ws->P;
  return (P.d.plasma_enabled ? 3 * P.n_cols : P.n_cols) + (absorber ? P.n_cols : 0);
}

template <class R = double>
static ForwardArgsT<R> forward_args(const sp_workspace* ws) {
  const sp_problem& P = *ws->P;
  const sp_problem_desc& d = P.d;
  const int nc = P.n_cols;
  const SourceView<R> v = source_view<R>(ws);
  // the response column leaves a partial row per node group (the products: group 0's rows
  // alone), which the transform adds in group order
  const int n_groups = ws->gemm ? 1 : (d.n_nodes + kGroup - 1) / kGroup;
  return ForwardArgsT<R>{ws->streams.p, v.proj, n_groups, 3 * nc,
                         d.plasma_enabled ? ws->rows.p : ws->rows.p + 4 * nc,
                         ws->crop.p, v.twiddles, v.spectra, d.n_to, d.n_omega, ws->log_m,
                         ws->log_n_to, P.crop_identity};
}

static OutputArgs output_args(const sp_workspace* ws, const StageScalarsDev* stage,
                              const double2* inv_prop, double2* out, bool absorber) {
  const sp_problem& P = *ws->P;
  return OutputArgs{stage, ws->spectra.p,
                    ws->precision == SP_PRECISION_MIXED ? ws->f32.spectra.p : nullptr,
                    ws->pre_terms.p, ws->omega.p, ws->omega_window.p,
                    ws->active.p, inv_prop, out, P.n_cols, P.d.n_omega, P.d.plasma_enabled,
                    absorber};
}

// The field-grid Raman pass's arguments (the doubled grid's table, the stage's rates)
static RamanArgs raman_args(const sp_workspace* ws, int slot) {
  const sp_problem_desc& d = ws->P->d;
  RamanArgs ra{};
  ra.stage = ws->stage.p + slot;
  ra.undamped = ws->raman_undamped.p;
  ra.spectrum = ws->raman_spectrum.p;
  ra.twiddles = ws->env_twiddles.p;
  ra.t_window = ws->t_window.p;
  ra.n_to = d.n_to;
  ra.log_n_to = ws->log_n_to;
  ra.n_components = (int)ws->P->raman_fraction.size();
  for (int c = 0; c <= ra.n_components; ++c) ra.first_row[c] = ws->P->raman_first_row[c];
  for (int c = 0; c < ra.n_components; ++c) ra.fraction[c] = ws->P->raman_fraction[c];
  ra.dt = d.dt_fine;
  ra.tensor_weights = ws->P->raman_weights.empty() ? nullptr : ws->raman_weights.p;
  ra.n_kernels = ws->P->raman_kernels;
  ra.scratch = ws->raman_scratch.p;
  return ra;
}

// The field grid's source on the GEMM route: inverse transforms, the synthesis product
// (node field), the response column over the node field (node streams), the projection
// products (the projected streams, group 0's rows), forward transforms.  The taper tau
// of the stage scales the synthesis and divides the projection, read on the device.
static void eval_source_gemm(sp_workspace* ws, const double2* lab, int slot, bool absorber) {
  const sp_problem& P = *ws->P;
  const sp_problem_desc& d = P.d;
  const double* taper = &(ws->stage.p + slot)->taper;
  double* status = ws->norms.p + kColumnStatus;
  const int n_streams = d.plasma_enabled ? 3 : 1;
  const size_t stride = (size_t)P.n_cols * d.n_to;  // one projected stream's rows
  const auto ia = inverse_args(ws, lab, absorber);
  { KernelTimer t(ws, SP_K_INVERSE); CUDA_CHECK(launch_inverse(ia, P.n_cols, ws->stream)); }
  if (ws->precision == SP_PRECISION_MIXED) {
    {
      KernelTimer t(ws, SP_K_PROJECT);
      CUDA_CHECK(modal_synthesis_split3(ws->s_parts.p, ws->modal_t.p, ws->modal_parts.p, ws->f32.node_field.p,
                                        d.n_nodes, d.n_modes, d.n_to, ws->kpad_modes, taper, status, ws->stream));
    }
    auto ca = column_args<float>(ws, ws->stage.p + slot);
    ca.node_field = ws->f32.node_field.p;
    ca.node_streams = ws->f32.node_streams.p;
    { KernelTimer t(ws, SP_K_COLUMN); CUDA_CHECK(launch_column_nodes(ca, ws->stream)); }
    if (d.raman_enabled) {
      KernelTimer t(ws, SP_K_COLUMN);
      CUDA_CHECK(launch_raman(raman_args(ws, slot), ws->f32.node_field.p, ws->f32.node_streams.p, d.n_nodes,
                              ws->stream));
    }
    {
      KernelTimer t(ws, SP_K_PROJECT);
      CUDA_CHECK(modal_projection_split3(ws->w_parts.p, ws->f32.node_streams.p, ws->node_parts.p,
                                         ws->f32.proj.p, n_streams, d.n_modes, d.n_nodes, d.n_to,
                                         ws->kpad_nodes, stride, taper, status,
                                         reinterpret_cast<float*>(ws->proj_scratch.p), ws->stream));
    }
    const auto fa = forward_args<float>(ws);
    { KernelTimer t(ws, SP_K_FORWARD); CUDA_CHECK(launch_forward(fa, forward_rows(ws, absorber), ws->stream)); }
  } else {
    {
      KernelTimer t(ws, SP_K_PROJECT);
      CUDA_CHECK(modal_synthesis_f64(ws->synthesis.p, ws->modal_t.p, ws->node_field.p, d.n_nodes, d.n_modes,
                                     d.n_to, taper, ws->stream));
    }
    auto ca = column_args<double>(ws, ws->stage.p + slot);
    ca.node_field = ws->node_field.p;
    ca.node_streams = ws->node_streams.p;
    { KernelTimer t(ws, SP_K_COLUMN); CUDA_CHECK(launch_column_nodes(ca, ws->stream)); }
    if (d.raman_enabled) {
      KernelTimer t(ws, SP_K_COLUMN);
      CUDA_CHECK(launch_raman(raman_args(ws, slot), ws->node_field.p, ws->node_streams.p, d.n_nodes, ws->stream));
    }
    {
      KernelTimer t(ws, SP_K_PROJECT);
      CUDA_CHECK(modal_projection_f64(ws->projection.p, ws->node_streams.p, ws->proj.p, n_streams, d.n_modes,
                                      d.n_nodes, d.n_to, stride, taper, ws->proj_scratch.p, ws->stream));
    }
    const auto fa = forward_args<double>(ws);
    { KernelTimer t(ws, SP_K_FORWARD); CUDA_CHECK(launch_forward(fa, forward_rows(ws, absorber), ws->stream)); }
  }
}

// The envelope grid's source on the products: inverse transforms into the modal field (and
// the absorber's spectrum), the synthesis product, the Raman kernel's spectrum, the nodes'
// responses, the projection product, forward transforms.  Rows are complex, interleaved:
// the products see N = 2 n_to.  The mixed form's products are the tcgen05 products of
// three-part BF16 splits; its node field, streams and spectra are FP32.
template <class R>
static EnvModalArgsT<R> env_modal_args(const sp_workspace* ws, const double2* lab, int slot, bool absorber) {
  const sp_problem& P = *ws->P;
  const sp_problem_desc& d = P.d;
  EnvModalArgsT<R> ea{};
  ea.stage = ws->stage.p + slot;
  ea.lab = lab;
  ea.crop = ws->crop.p;
  ea.twiddles = ws->env_twiddles.p;
  ea.t_window = ws->t_window.p;
  ea.alpha = absorber ? ws->alpha.p : nullptr;
  ea.modal_t = ws->modal_t.p;
  ea.scratch = ws->env_scratch.p;
  ea.raman_spectrum = d.raman_enabled ? ws->raman_spectrum.p : nullptr;
  ea.n_cols = P.n_cols;
  ea.n_omega = d.n_omega;
  ea.n_to = d.n_to;
  ea.log_n_to = ws->log_n_to;
  ea.kerr = d.kerr_enabled;
  ea.raman_mixture = P.raman_fraction.size() > 1;
  ea.kerr_coefficient = d.kerr_coefficient;
  ea.kerr_self = d.kerr_self;
  ea.kerr_conjugate = d.kerr_conjugate;
  ea.n_components = d.n_pol_transform;
  ea.raman_kernels = P.raman_kernels;
  if constexpr (sizeof(R) == 8) {
    ea.twiddles_r = ws->env_twiddles.p;
    ea.node_field = ws->node_field.p;
    ea.node_streams = ws->node_streams.p;
    ea.projected = ws->proj.p;
    ea.spectra = ws->spectra.p;
  } else {
    ea.twiddles_r = ws->f32.env_twiddles.p;
    ea.raman_spectrum32 = ws->raman_spectrum32.p;
    ea.raman_scale = ws->raman_scale.p;
    ea.node_field = ws->f32.node_field.p;
    ea.node_streams = ws->f32.node_streams.p;
    ea.projected = ws->f32.proj.p;
    ea.spectra = ws->f32.spectra.p;
  }
  return ea;
}

static void eval_source_envelope_gemm(sp_workspace* ws, const double2* lab, int slot, bool absorber) {
  const sp_problem& P = *ws->P;
  const sp_problem_desc& d = P.d;
  const double* taper = &(ws->stage.p + slot)->taper;
  double* status = ws->norms.p + kColumnStatus;
  const int n2 = 2 * d.n_to;
  const int rows = d.n_nodes * d.n_pol_transform;  // two components: rows x, y per node
  const size_t stride = (size_t)P.n_cols * n2;
  if (ws->precision == SP_PRECISION_MIXED) {
    const auto ea = env_modal_args<float>(ws, lab, slot, absorber);
    { KernelTimer t(ws, SP_K_INVERSE); CUDA_CHECK(launch_env_inverse(ea, ws->stream)); }
    {
      KernelTimer t(ws, SP_K_PROJECT);
      CUDA_CHECK(modal_synthesis_split3(ws->s_parts.p, ws->modal_t.p, ws->modal_parts.p, ws->f32.node_field.p,
                                        rows, d.n_modes, n2, ws->kpad_modes, taper, status, ws->stream));
    }
    {
      KernelTimer t(ws, SP_K_COLUMN);
      if (d.raman_enabled) {
        RamanArgs ra = raman_args(ws, slot);
        ra.spectrum32 = ws->raman_spectrum32.p;
        ra.scale = ws->raman_scale.p;
        CUDA_CHECK(launch_raman_spectrum(ra, ws->stream));
      }
      CUDA_CHECK(launch_env_nodes(ea, d.n_nodes, ws->stream));
    }
    {
      KernelTimer t(ws, SP_K_PROJECT);
      CUDA_CHECK(modal_projection_split3(ws->w_parts.p, ws->f32.node_streams.p, ws->node_parts.p, ws->f32.proj.p,
                                         1, d.n_modes, rows, n2, ws->kpad_nodes, stride, taper, status,
                                         reinterpret_cast<float*>(ws->proj_scratch.p), ws->stream));
    }
    { KernelTimer t(ws, SP_K_FORWARD); CUDA_CHECK(launch_env_forward(ea, ws->stream)); }
    return;
  }
  const auto ea = env_modal_args<double>(ws, lab, slot, absorber);
  { KernelTimer t(ws, SP_K_INVERSE); CUDA_CHECK(launch_env_inverse(ea, ws->stream)); }
  {
    KernelTimer t(ws, SP_K_PROJECT);
    CUDA_CHECK(modal_synthesis_f64(ws->synthesis.p, ws->modal_t.p, ws->node_field.p, rows, d.n_modes, n2,
                                   taper, ws->stream));
  }
  {
    KernelTimer t(ws, SP_K_COLUMN);
    if (d.raman_enabled) CUDA_CHECK(launch_raman_spectrum(raman_args(ws, slot), ws->stream));
    CUDA_CHECK(launch_env_nodes(ea, d.n_nodes, ws->stream));
  }
  {
    KernelTimer t(ws, SP_K_PROJECT);
    CUDA_CHECK(modal_projection_f64(ws->projection.p, ws->node_streams.p, ws->proj.p, 1, d.n_modes, rows,
                                    n2, stride, taper, ws->proj_scratch.p, ws->stream));
  }
  { KernelTimer t(ws, SP_K_FORWARD); CUDA_CHECK(launch_env_forward(ea, ws->stream)); }
}

// One source evaluation at lab (device), stage slot, optional inverse propagator.
// The stage output's record of a source evaluation (its last pass)
static OutputArgs source_output_args(const sp_workspace* ws, int slot, const double2* inv_prop, double2* out,
                                     bool quiet) {
  const bool absorber = ws->P->d.absorber_in_stage && !quiet;
  return output_args(ws, ws->stage.p + slot, inv_prop, out, absorber);
}

// output: false leaves the stage output (the last pass) to the caller's next kernel, which
// forms it from source_output_args (the single-run corrector)
static void eval_source(sp_workspace* ws, const double2* lab, int slot, const double2* inv_prop,
                        double2* out, bool quiet, bool output = true) {
  const sp_problem& P = *ws->P;
  const bool absorber = P.d.absorber_in_stage && !quiet;
  if (P.d.grid_kind == 1 && ws->gemm) {
    eval_source_envelope_gemm(ws, lab, slot, absorber);
  } else if (P.d.grid_kind == 1) {
    const sp_problem_desc& d = P.d;
    EnvelopeArgs ea{};
    ea.stage = ws->stage.p + slot;
    ea.lab = lab;
    ea.crop = ws->crop.p;
    ea.twiddles = ws->env_twiddles.p;
    ea.t_window = ws->t_window.p;
    ea.raman_undamped = d.raman_enabled ? ws->raman_undamped.p : nullptr;
    ea.spectra = ws->spectra.p;
    ea.synthesis = P.synthesis[0];
    ea.projection = P.projection[0];
    ea.dt = d.dt_fine;
    ea.kerr = d.kerr_enabled;
    ea.kerr_coefficient = d.kerr_coefficient;
    ea.kerr_self = d.kerr_self;
    ea.kerr_conjugate = d.kerr_conjugate;
    ea.raman_fraction = d.raman_fraction;
    ea.raman_terms = d.raman_enabled ? d.raman_terms : 0;
    ea.n_omega = d.n_omega;
    ea.n_to = d.n_to;
    ea.log_n_to = ws->log_n_to;
    { KernelTimer t(ws, SP_K_COLUMN); CUDA_CHECK(launch_envelope(ea, ws->stream)); }
  } else if (ws->gemm) {
    eval_source_gemm(ws, lab, slot, absorber);
  } else if (ws->precision == SP_PRECISION_MIXED) {
    const auto ia = inverse_args(ws, lab, absorber);
    { KernelTimer t(ws, SP_K_INVERSE); CUDA_CHECK(launch_inverse(ia, P.n_cols, ws->stream)); }
    const auto ca = column_args<float>(ws, ws->stage.p + slot);
    { KernelTimer t(ws, SP_K_COLUMN); CUDA_CHECK(launch_column(ca, ws->stream)); }
    const auto fa = forward_args<float>(ws);
    { KernelTimer t(ws, SP_K_FORWARD); CUDA_CHECK(launch_forward(fa, forward_rows(ws, absorber), ws->stream)); }
  } else {
    const auto ia = inverse_args(ws, lab, absorber);
    { KernelTimer t(ws, SP_K_INVERSE); CUDA_CHECK(launch_inverse(ia, P.n_cols, ws->stream)); }
    const auto ca = column_args<double>(ws, ws->stage.p + slot);
    { KernelTimer t(ws, SP_K_COLUMN); CUDA_CHECK(launch_column(ca, ws->stream)); }
    const auto fa = forward_args<double>(ws);
    { KernelTimer t(ws, SP_K_FORWARD); CUDA_CHECK(launch_forward(fa, forward_rows(ws, absorber), ws->stream)); }
  }
  if (!output) return;
  const OutputArgs oa = source_output_args(ws, slot, inv_prop, out, quiet);
  { KernelTimer t(ws, SP_K_OUTPUT); CUDA_CHECK(launch_output(oa, ws->stream)); }
}

template <class T>
static std::vector<float> to_float(const std::vector<T>& v) {
  return std::vector<float>(v.begin(), v.end());
}

// The mixed-precision form's FP32 tables and buffers.  The rate table becomes (c0, c1,
// c2, exp c3, 1 / knot) per interval, the form the FP32 lookup evaluates.
static void build_mixed(sp_workspace* ws, const std::vector<double2>& tw, const std::vector<double>& rc,
                        const std::vector<double>& taps) {
  const sp_problem& P = *ws->P;
  const sp_problem_desc& d = P.d;
  cudaStream_t s = ws->stream;
  auto& f = ws->f32;
  std::vector<float2> tw32(tw.size());
  for (size_t m = 0; m < tw.size(); ++m) tw32[m] = make_float2((float)tw[m].x, (float)tw[m].y);
  f.twiddles.upload(tw32.data(), tw32.size(), s);
  auto up = [&](DevBuf<float>& dst, const std::vector<float>& v) { dst.upload(v.data(), v.size(), s); };
  // the uploads are asynchronous: keep the host copies alive until the stream is synchronised
  std::vector<std::vector<float>> keep;
  keep.reserve(8);
  keep.push_back(to_float(P.t_window));
  up(f.t_window, keep.back());
  keep.push_back(to_float(P.t_window_d));
  up(f.t_window_d, keep.back());
  keep.push_back(to_float(P.synthesis));
  up(f.synthesis, keep.back());
  keep.push_back(to_float(P.projection));
  up(f.projection, keep.back());
  keep.push_back(to_float(taps));
  up(f.taps, keep.back());
  // the rate tables in the FP32 form: (c0, c1, c2, exp c3, 1 / knot) per interval, every
  // channel's in channel order
  std::vector<float> r32;
  auto convert = [&](const double* c, int n, double log_field_min, double d_log_field) {
    const size_t at = r32.size();
    r32.resize(at + (size_t)5 * n, 0.0f);
    for (int i = 0; i < n; ++i) {
      r32[at + i] = (float)c[i];
      r32[at + n + i] = (float)c[n + i];
      r32[at + 2 * n + i] = (float)c[2 * n + i];
      r32[at + 3 * n + i] = (float)std::exp(c[3 * n + i]);
      r32[at + 4 * n + i] = (float)std::exp(-(log_field_min + (double)i * d_log_field));
    }
    return at;
  };
  std::vector<size_t> offsets;
  if (!P.channels.empty()) {
    for (const auto& ch : P.channels)
      offsets.push_back(convert(ch.coefficients.data(), (int)(ch.coefficients.size() / 4), ch.log_field_min,
                                ch.d_log_field));
  } else if (rc.size() >= (size_t)4 * std::max(d.rate_intervals, 1) && d.rate_intervals >= 1) {
    convert(rc.data(), d.rate_intervals, d.log_field_min, d.d_log_field);
  } else {
    r32.assign(5, 0.0f);
  }
  keep.push_back(std::move(r32));
  up(f.rate_coeff, keep.back());
  if (!P.channels.empty()) {
    std::vector<ChannelTableT<float>> tables;
    for (size_t c = 0; c < P.channels.size(); ++c) {
      const auto& ch = P.channels[c];
      tables.push_back({f.rate_coeff.p + offsets[c], (int)(ch.coefficients.size() / 4), ch.log_field_min,
                        ch.d_log_field, ch.field_min, ch.field_max, ch.rate_max, ch.charge_mass_ratio,
                        ch.ionisation_potential});
    }
    f.channels.upload(tables.data(), tables.size(), s);
    CUDA_CHECK(cudaStreamSynchronize(s));
  }
  const size_t n_groups = ws->gemm ? 1 : (d.n_nodes + kGroup - 1) / kGroup;  // the products write group 0's rows
  f.proj.alloc(n_groups * 3 * P.n_cols * d.n_to);
  f.proj.zero(s);
  f.spectra.alloc((size_t)4 * P.n);
  f.spectra.zero(s);
  CUDA_CHECK(cudaStreamSynchronize(s));
}

static void build_workspace(sp_workspace* ws) {
  const sp_problem& P = *ws->P;
  const sp_problem_desc& d = P.d;
  cudaStream_t s = ws->stream;
  const size_t n = P.n;
  ws->log_m = ilog2(d.n_to / 2);
  ws->log_n_to = ilog2(d.n_to);
  ws->phi_terms.upload(P.phi_terms.data(), (size_t)d.n_phi_terms * n, s);
  ws->pre_terms.upload(P.pre_terms.data(), (size_t)d.n_prefactor_terms * n, s);
  // twiddles exp(-2 pi i m / n_to), m < n_to/2, in long double, rounded once
  std::vector<double2> tw(d.n_to / 2);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < d.n_to / 2; ++m) {
    long double ang = two_pi * (long double)m / (long double)d.n_to;
    tw[m] = make_double2((double)cosl(ang), (double)(-sinl(ang)));
  }
  ws->twiddles.upload(tw.data(), tw.size(), s);
  ws->omega.upload(P.omega.data(), d.n_omega, s);
  ws->omega_window.upload(P.omega_window.data(), d.n_omega, s);
  ws->t_window.upload(P.t_window.data(), d.n_to, s);
  ws->t_window_d.upload(P.t_window_d.data(), d.n_to, s);
  std::vector<double> alpha(d.n_to, 0.0);
  if (d.absorber_in_stage) alpha = P.alpha;
  ws->alpha.upload(alpha.data(), d.n_to, s);
  ws->synthesis.upload(P.synthesis.data(), P.synthesis.size(), s);
  ws->projection.upload(P.projection.data(), P.projection.size(), s);
  std::vector<double> rc = P.rate_coeff.empty() ? std::vector<double>(4, 0.0) : P.rate_coeff;
  std::vector<size_t> channel_at;  // a mixture: every channel's table, channel 0's first
  if (!P.channels.empty()) {
    rc.clear();
    for (const auto& ch : P.channels) {
      channel_at.push_back(rc.size());
      rc.insert(rc.end(), ch.coefficients.begin(), ch.coefficients.end());
    }
  }
  ws->rate_coeff.upload(rc.data(), rc.size(), s);
  if (!P.channels.empty()) {
    std::vector<ChannelTableT<double>> tables;
    for (size_t c = 0; c < P.channels.size(); ++c) {
      const auto& ch = P.channels[c];
      tables.push_back({ws->rate_coeff.p + channel_at[c], (int)(ch.coefficients.size() / 4), ch.log_field_min,
                        ch.d_log_field, ch.field_min, ch.field_max, ch.rate_max, ch.charge_mass_ratio,
                        ch.ionisation_potential});
    }
    ws->channels.upload(tables.data(), tables.size(), s);
    CUDA_CHECK(cudaStreamSynchronize(s));
  }
  std::vector<double> taps = P.taps.empty() ? std::vector<double>(1, 1.0) : P.taps;
  ws->taps.upload(taps.data(), taps.size(), s);
  ws->crop.upload(P.crop.data(), d.n_omega, s);
  // the fine spectrum's bins: n_to / 2 + 1 on the field grid, n_to on the envelope grid
  std::vector<int> f2c(d.grid_kind == 1 ? d.n_to : d.n_to / 2 + 1, -1);
  for (int j = 0; j < d.n_omega; ++j) f2c.at(P.crop[j]) = j;
  ws->fine_to_coarse.upload(f2c.data(), f2c.size(), s);
  // stream rows: [0, 3 n_cols) P X Z, then absorber [3 n_cols, 4 n_cols); a second list
  // at 4 n_cols for the no-plasma case: P rows then absorber rows
  std::vector<int> rows;
  for (int r = 0; r < 4 * P.n_cols; ++r) rows.push_back(r);
  for (int r = 0; r < P.n_cols; ++r) rows.push_back(r);
  for (int r = 0; r < P.n_cols; ++r) rows.push_back(3 * P.n_cols + r);
  ws->rows.upload(rows.data(), rows.size(), s);
  ws->active.upload(P.active.data(), d.n_omega, s);
  ws->norm.upload(P.norm.data(), d.n_omega, s);
  ws->lab.alloc(n);
  ws->out.alloc(n);
  const size_t cplx_rows = d.grid_kind == 1 ? 2 : 1;  // the envelope's rows are complex, interleaved
  ws->modal_t.alloc(cplx_rows * P.n_cols * d.n_to);
  const size_t n_tiles = column_tiles(d);
  const size_t n_groups = (d.n_nodes + kGroup - 1) / kGroup;
  ws->sums0.alloc((size_t)std::max<size_t>(1, P.channels.size()) * d.n_nodes * n_tiles);  // a plane per channel
  ws->sums1.alloc((size_t)d.n_nodes * n_tiles);
  ws->chain_flags.alloc(n_groups * n_tiles);
  ws->chain_flags.zero(s);
  ws->ticket.alloc(1);
  ws->ticket.zero(s);
  ws->proj.alloc((ws->gemm ? 1 : n_groups) * 3 * P.n_cols * d.n_to);
  ws->proj.zero(s);
  if (ws->gemm) {
    const int node_rows = d.n_nodes * d.n_pol_transform;  // two components: rows x, y per node
    const size_t field = cplx_rows * node_rows * d.n_to;
    ws->kpad_modes = modal_kpad(d.n_modes);
    ws->kpad_nodes = modal_kpad(node_rows);
    ws->proj_scratch.alloc(modal_projection_scratch(d.n_modes, node_rows, (int)cplx_rows * d.n_to));
    if (ws->precision == SP_PRECISION_MIXED) {
      ws->f32.node_field.alloc(field);
      ws->f32.node_streams.alloc(3 * field);
      ws->f32.node_streams.zero(s);
      std::vector<uint16_t> parts;
      split3_host(P.synthesis.data(), node_rows, d.n_modes, ws->kpad_modes, parts);
      ws->s_parts.upload(parts.data(), parts.size(), s);
      CUDA_CHECK(cudaStreamSynchronize(s));  // the host copy goes with this scope
      split3_host(P.projection.data(), d.n_modes, node_rows, ws->kpad_nodes, parts);
      ws->w_parts.upload(parts.data(), parts.size(), s);
      CUDA_CHECK(cudaStreamSynchronize(s));
      ws->modal_parts.alloc((size_t)3 * cplx_rows * d.n_to * ws->kpad_modes);
      ws->node_parts.alloc((size_t)3 * cplx_rows * d.n_to * ws->kpad_nodes);
    } else {
      ws->node_field.alloc(field);
      ws->node_streams.alloc(3 * field);
      ws->node_streams.zero(s);
    }
  }
  ws->streams.alloc((size_t)4 * P.n_cols * d.n_to);
  ws->streams.zero(s);
  ws->spectra.alloc((size_t)4 * n);
  ws->spectra.zero(s);
  static_assert(sizeof(AdamsDev) % alignof(StageScalarsDev) == 0, "the stage slots follow the trial's table");
  const size_t table_bytes = sizeof(AdamsDev) + sizeof(StageScalarsDev) * sp_workspace::kStageSlots;
  ws->tables.alloc(table_bytes);
  ws->adams.p = reinterpret_cast<AdamsDev*>(ws->tables.p);
  ws->adams.n = 1;
  ws->adams.owned = false;
  ws->stage.p = reinterpret_cast<StageScalarsDev*>(ws->tables.p + sizeof(AdamsDev));
  ws->stage.n = sp_workspace::kStageSlots;
  ws->stage.owned = false;
  CUDA_CHECK(cudaEventCreateWithFlags(&ws->host_tables_free, cudaEventDisableTiming));
  CUDA_CHECK(cudaMallocHost(&ws->h_tables, table_bytes));
  ws->h_adams = reinterpret_cast<AdamsDev*>(ws->h_tables);
  ws->h_stage = reinterpret_cast<StageScalarsDev*>(ws->h_tables + sizeof(AdamsDev));
  CUDA_CHECK(cudaMallocHost(&ws->h_norms, sizeof(double) * 8));
  ws->partials.alloc((kMaxOrders + 2) * kNormBlocks);
  ws->norms.alloc(kMaxOrders + 2);
  ws->norms.zero(s);
  ws->norm_arrivals.alloc(1);
  ws->norm_arrivals.zero(s);
  ws->launches = 5;
  if (ws->gemm && d.grid_kind == 1) {  // inverse, synthesis, (Raman spectrum,) nodes, projection, reduction,
    ws->launches = 6 + (d.raman_enabled ? 1 : 0) + (ws->precision == SP_PRECISION_MIXED ? 2 : 0);  // forward,
                                                                  // output; the mixed form's two split passes
  } else if (ws->gemm) {  // inverse, synthesis, column, one projection per stream, forward, output
    const int per_product = ws->precision == SP_PRECISION_MIXED ? 2 : 1;  // (split,) product
    const int streams = d.plasma_enabled ? 3 : 1;  // each: (split,) product, reduction of the K splits
    ws->launches = 4 + per_product + (per_product + 1) * streams + (d.raman_enabled ? 2 : 0);
  }
  if (ws->precision == SP_PRECISION_MIXED) build_mixed(ws, tw, rc, taps);
  if (d.grid_kind == 1 || d.raman_enabled) {  // the doubled grid's table: envelope route, Raman
    std::vector<double2> tw2(d.n_to);
    for (int m = 0; m < d.n_to; ++m) {
      long double ang = two_pi * (long double)m / (long double)(2 * d.n_to);
      tw2[m] = make_double2((double)cosl(ang), (double)(-sinl(ang)));
    }
    ws->env_twiddles.upload(tw2.data(), tw2.size(), s);
    if (ws->precision == SP_PRECISION_MIXED) {
      std::vector<float2> tw2f(tw2.size());
      for (size_t m = 0; m < tw2.size(); ++m) tw2f[m] = make_float2((float)tw2[m].x, (float)tw2[m].y);
      ws->f32.env_twiddles.upload(tw2f.data(), tw2f.size(), s);
      CUDA_CHECK(cudaStreamSynchronize(s));  // the host copy goes with this scope
    }
    if (d.raman_enabled) ws->raman_undamped.upload(P.raman_undamped.data(), P.raman_undamped.size(), s);
    if (!P.raman_weights.empty()) ws->raman_weights.upload(P.raman_weights.data(), P.raman_weights.size(), s);
    if (d.raman_enabled && (d.grid_kind == 0 || ws->gemm))
      ws->raman_spectrum.alloc((size_t)P.raman_kernels * (d.n_to + 1));
    if (d.raman_enabled && d.grid_kind == 1 && ws->gemm && ws->precision == SP_PRECISION_MIXED) {
      ws->raman_spectrum32.alloc((size_t)P.raman_kernels * (d.n_to + 1));
      ws->raman_scale.alloc(2);
    }
    if (d.grid_kind == 1 && ws->gemm && d.n_to > kMaxEnvelopeRowF64) {
      // rows of FP64 too long for one CTA: the inverse transforms' (every column), and in the
      // FP64 form the nodes' and the forward transforms'
      const size_t rows = ws->precision == SP_PRECISION_MIXED ? (size_t)P.n_cols
                                                              : std::max<size_t>(P.n_cols, d.n_nodes);
      ws->env_scratch.alloc(rows * ((size_t)d.n_to + d.n_to / 2));
      if (d.raman_enabled) ws->raman_scratch.alloc((size_t)P.raman_kernels * ((size_t)d.n_to + d.n_to / 2));
    }
    CUDA_CHECK(cudaStreamSynchronize(s));
  }
  CUDA_CHECK(cudaStreamSynchronize(s));
}

// ====================================================================== coefficient tables
// stepper/multistep.py _basis_rows: the Lagrange basis from its own roots, ascending.
// The stencils hold a few points (at most kBasis), so every list and table here is a
// fixed-size array: the per-run host work of a batch step allocates nothing.
constexpr int kBasis = kMaxWidth + 1;
struct Points {
  double v[kBasis];
  int n = 0;
  void push(double x) {
    if (n >= kBasis) throw Failure(SP_ERR_ARGUMENT, "an Adams stencil longer than the tables hold");
    v[n++] = x;
  }
};
// coef (ascending powers) and denominator of basis polynomial `index`
static int basis_poly(const Points& pts, int index, double (&coef)[kBasis + 1], double& den) {
  double prod[kBasis + 1];
  const double node = pts.v[index];
  int length = 1;
  coef[0] = 1.0;
  den = 1.0;
  for (int other = 0; other < pts.n; ++other) {
    if (other == index) continue;
    const double root = pts.v[other];
    prod[0] = 0.0;
    for (int p = 0; p < length; ++p) prod[p + 1] = coef[p];
    for (int p = 0; p < length; ++p) prod[p] -= root * coef[p];
    ++length;
    for (int p = 0; p < length; ++p) coef[p] = prod[p];
    den *= node - root;
  }
  return length;
}
// rows[i][p]: coefficient p of basis polynomial i
static void lagrange(const Points& pts, double (&rows)[kBasis][kBasis]) {
  for (int index = 0; index < pts.n; ++index) {
    double coef[kBasis + 1], den;
    const int length = basis_poly(pts, index, coef, den);
    for (int p = 0; p < length; ++p) rows[index][p] = coef[p] / den;
  }
}
// weights[i]: the integral of basis polynomial i over [0, 1]
static void integrated(const Points& pts, double (&weights)[kBasis]) {
  const double upper = 1.0;
  for (int index = 0; index < pts.n; ++index) {
    double coef[kBasis + 1], den;
    const int length = basis_poly(pts, index, coef, den);
    double integral = 0.0;
    for (int p = length - 1; p >= 0; --p) integral = (integral + coef[p] / (p + 1)) * upper;
    weights[index] = integral / den;
  }
}

// ====================================================================== session
static constexpr int kLandingUlps = 8;
static double ulp(double x) {
  x = std::fabs(x);
  return std::nextafter(x, std::numeric_limits<double>::infinity()) - x;
}
static bool reached(double pos, double target) {
  return pos >= target - kLandingUlps * ulp(std::max(std::fabs(pos), std::fabs(target)));
}

struct sp_session {
  sp_workspace* ws = nullptr;
  sp_run_desc run{};
  std::vector<double> planes, kinks, edges, schedule, sched_edges;
  double z = 0.0, proposal = 0.0;
  int64_t attempts = 0, rejected = 0, evaluations = 0;
  int plane_cursor = 0, sched_cursor = 0;
  bool finished = false, failed = false;
  // Adams
  std::vector<std::pair<double, int>> history;  // (z, row), oldest first
  int rejections = 0, order = 1;
  bool last_rejected = false;
  // the public single-run API leaves an accepted trial's accept to the next predictor
  // (sp_workspace::pending_accept); a scan's runs accept at once
  bool defer_accept = false;
  // RK
  std::vector<double> norms_hist;
  // the last attempt, for the batch's attempt rows: end, step, norm, accepted
  struct Row {
    double end = 0, step = 0, norm = 0;
    bool accepted = false;
  } row;
  // requests from other threads, polled between attempts
  std::atomic<bool> stop_requested{false}, snapshot_requested{false};
  bool stopped = false;
};

static void settle_accept(sp_workspace* ws);

static void adams_start(sp_session* S) {
  sp_workspace* ws = S->ws;
  const sp_problem& P = *ws->P;
  settle_accept(ws);  // the start reads the state
  fill_stage(ws, 1, S->z, S->z);  // source at (z, z)
  AdamsDev& ad = *ws->h_adams;
  std::memset(&ad, 0, sizeof(ad));
  const bool comp = P.d.phi_expansion;
  if (comp) P.phi_rate.eval(S->z, ad.rate0_w);
  CUDA_CHECK(cudaMemcpyAsync(ws->stage.p, ws->h_stage, 2 * sizeof(StageScalarsDev),
                             cudaMemcpyHostToDevice, ws->stream));
  CUDA_CHECK(cudaMemcpyAsync(ws->adams.p, &ad, sizeof(AdamsDev), cudaMemcpyHostToDevice, ws->stream));
  release_host_tables(ws);  // the attempt that follows refills both tables
  eval_source(ws, ws->state.p, 1, nullptr, ws->src.p, false);
  StepArgs a{};
  a.stage = ws->stage.p + 1;
  a.adams = ws->adams.p;
  a.phi_terms = ws->phi_terms.p;
  a.n = P.n;
  a.n_omega = P.d.n_omega;
  a.state = ws->state.p;
  a.store = ws->store.p;
  a.states = comp ? ws->states.p : nullptr;
  a.rates = comp ? ws->rates.p : nullptr;
  a.source = ws->src.p;
  a.n_blocks = kNormBlocks;
  { KernelTimer t(ws, SP_K_START); CUDA_CHECK(launch_adams_start(a, ws->stream)); }
  S->evaluations += 1;
  S->history.assign(1, {S->z, 0});
  S->order = S->run.variable_order ? 1 : S->run.order;
}

static double limit_step(double dz, double factor, double dz_min, double dz_max) {
  double proposed = std::min(dz * factor, dz_max);
  if (proposed < dz_min) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "step control asked for %.3e m, below the floor dz_min = %.3e m",
                  proposed, dz_min);
    throw Failure(SP_ERR_CONVERGENCE, buf, SP_REASON_FLOOR);
  }
  return proposed;
}

// One Adams attempt, split in three so that a batch of runs can share the launches:
// prepare (stencil, tables and stage scalars into the workspace's pinned records),
// the launches, and decide (the host's acceptance, order and step choice).
struct Pending {
  double dz = 0, end = 0;
  bool kink = false, fixed = false;
  int order = 1, free_slot = 0;
  int orders[kMaxOrders] = {0, 0, 0};  // the scored orders, the trial's own first
  int n_orders = 0;
};

static Pending prepare_attempt(sp_session* S, double dz, double end, bool kink, bool fixed) {
  sp_workspace* ws = S->ws;
  const sp_problem& P = *ws->P;
  const sp_run_desc& R = S->run;
  const bool comp = P.d.phi_expansion;
  Pending pd;
  pd.dz = dz;
  pd.end = end;
  pd.kink = kink;
  pd.fixed = fixed;
  // stencil (adams_core.py:150-206)
  Points nodes;
  int slots[kBasis];
  for (auto it = S->history.rbegin(); it != S->history.rend(); ++it) {
    nodes.push((it->first - S->z) / dz);
    slots[nodes.n - 1] = it->second;
  }
  const int held = nodes.n;
  const int order = std::min(S->order, held);
  const bool rising = !S->last_rejected && held > order;
  pd.orders[pd.n_orders++] = order;
  if (R.variable_order) {
    for (int o : {order - 1, order + 1})
      if (o >= 1 && o <= R.order && o <= held && (o < order || rising)) pd.orders[pd.n_orders++] = o;
  }
  pd.order = order;
  // the row an accepted step writes: the first not kept (marches/adams.py:593-596)
  {
    const size_t from = !R.order ? S->history.size()
                        : S->history.size() > (size_t)R.order ? S->history.size() - R.order : 0;
    int free_slot = 0;
    for (;; ++free_slot) {
      bool used = false;
      for (size_t e = from; e < S->history.size(); ++e) used |= S->history[e].second == free_slot;
      if (!used) break;
    }
    pd.free_slot = free_slot;
  }
  int width = 1 + *std::max_element(pd.orders, pd.orders + pd.n_orders);
  claim_host_tables(ws);
  AdamsDev& ad = *ws->h_adams;
  std::memset(&ad, 0, sizeof(ad));
  if (ws->pending_accept >= 0) {  // this trial's predictor applies the accept before it
    ad.settle = ws->pending_accept + 1;
    ws->pending_accept = -1;
  }
  ad.dz = dz;
  ad.rtol = R.rtol;
  ad.atol = R.atol;
  ad.order = order;
  ad.width = width;
  ad.n_orders = pd.n_orders;
  ad.compensated = comp;
  ad.free_slot = pd.free_slot;
  for (int j = 0; j < width - 1 && j < held; ++j) {
    ad.slots[j] = slots[j];
    ad.nodes[j] = nodes.v[j];
  }
  // the first k nodes, and the same behind the new point theta = 1
  auto stencil = [&](int k, bool with_one) {
    Points p;
    if (with_one) p.push(1.0);
    for (int j = 0; j < k; ++j) p.push(nodes.v[j]);
    return p;
  };
  double c[kBasis][kBasis];
  lagrange(stencil(order, false), c);
  for (int j = 0; j < order; ++j)
    for (int k = 0; k < order; ++k) ad.pred[j][k] = c[j][k];
  lagrange(stencil(order, true), c);
  for (int j = 0; j <= order; ++j)
    for (int k = 0; k <= order; ++k) ad.corr[j][k] = c[j][k];
  for (int r = 0; r < pd.n_orders; ++r) {
    const int k = pd.orders[r];
    const Points st = stencil(k, false), th = stencil(k, true);
    double a2[kBasis][kBasis];
    lagrange(th, c);
    lagrange(st, a2);
    for (int j = 0; j <= k; ++j)
      for (int q = 0; q <= k; ++q) ad.rows[r][j][q] = c[j][q];
    for (int j = 0; j < k; ++j)
      for (int q = 0; q < k; ++q) ad.rows[r][j + 1][q] -= a2[j][q];
    if (comp) {
      double wp[kBasis], wc[kBasis];
      integrated(st, wp);
      integrated(th, wc);
      for (int j = 0; j < k; ++j) ad.comp_pred[r][j] = wp[j];
      for (int j = 0; j <= k; ++j) ad.comp_corr[r][j] = wc[j];
    }
  }
  if (comp) {
    double wp[kBasis], wc[kBasis];
    integrated(stencil(order, false), wp);
    integrated(stencil(order, true), wc);
    for (int j = 0; j < order; ++j) ad.comp_pred_main[j] = wp[j];
    for (int j = 0; j <= order; ++j) ad.comp_corr_main[j] = wc[j];
    P.phi_rate.eval_before(S->z + dz, ad.rate_w);
  }
  fill_stage(ws, 0, S->z, S->z + dz);        // the step's exponent
  fill_stage(ws, 1, S->z + dz, S->z + dz);   // the source at the predicted field
  return pd;
}

// The host's decision on a trial from its four reduced sums (defect norms squared in
// the orders' order, then the state's squared norm); returns whether it was accepted.
static bool decide_attempt(sp_session* S, const Pending& pd, const double* sums) {
  const sp_run_desc& R = S->run;
  S->attempts += 1;
  S->evaluations += 1;
  const double magnitude = std::sqrt(sums[kMaxOrders]);
  const double scale = R.rtol * magnitude + R.atol;
  double norms[kMaxOrders];
  for (int r = 0; r < pd.n_orders; ++r) norms[r] = std::sqrt(sums[r]) / scale;
  const double norm = norms[0];
  const int order = pd.order;
  const double dz = pd.dz;
  S->row = {pd.end, dz, norm, false};
  auto factor = [&](double nm, int o, double growth) {
    if (nm <= 0.0) return growth;
    double raw = R.safety * std::pow(nm, -1.0 / (o + 1));
    return std::min(growth, std::max(R.min_factor, raw));
  };
  if (!(norm <= 1.0) && !(pd.fixed && std::isfinite(norm))) {
    S->rejected += 1;
    S->last_rejected = true;
    int count = S->rejections + 1;
    bool restart = count >= R.restart_after && S->history.size() > 1;
    double sc = !std::isfinite(norm) ? R.min_factor : factor(norm, order, R.rejection_growth);
    S->rejections = restart ? 0 : count;
    if (restart) S->history.clear();
    S->proposal = limit_step(dz, sc, R.dz_min, R.dz_max);
    return false;
  }
  // keep the newest R.order rows (none for order 0), then the new one -- in place
  {
    const size_t from = !R.order ? S->history.size()
                        : S->history.size() > (size_t)R.order ? S->history.size() - R.order : 0;
    S->history.erase(S->history.begin(), S->history.begin() + from);
    S->history.push_back({S->z + dz, pd.free_slot});
  }
  S->rejections = 0;
  // order choice (adams_core.py:256-301)
  int stored = order, control = order;
  double cnorm = norm;
  if (!R.variable_order) {
    stored = R.order;
  } else {
    auto weight = [&](double nm, int o) {
      double rate = nm <= 0.0 ? INFINITY : std::pow(nm, -1.0 / (o + 1));
      double allowed = R.safety * rate;
      double stable = INFINITY;
      if (R.collar_rate > 0.0)
        stable = R.collar_stability * R.real_intervals[o - 1] / (R.collar_rate * dz);
      return std::min(allowed, stable);
    };
    int best = pd.orders[0];
    double bw = weight(norms[0], pd.orders[0]);
    for (int r = 1; r < pd.n_orders; ++r) {
      double w = weight(norms[r], pd.orders[r]);
      if (w > bw) { bw = w; best = pd.orders[r]; }
    }
    if (best != order && bw > R.hysteresis * weight(norms[0], order)) {
      stored = control = best;
      for (int r = 0; r < pd.n_orders; ++r) if (pd.orders[r] == best) cnorm = norms[r];
    }
  }
  S->order = stored;
  S->last_rejected = false;
  S->row.accepted = true;
  S->z = pd.end;
  if (pd.kink) S->history.clear();
  S->proposal = limit_step(dz, factor(cnorm, control, R.max_growth), R.dz_min, R.dz_max);
  return true;
}

static StepArgs step_args_of(sp_workspace* ws, const AdamsDev* adams_dev, const StageScalarsDev* stage0) {
  const sp_problem& P = *ws->P;
  const bool comp = P.d.phi_expansion;
  StepArgs a{};
  a.stage = stage0;
  a.adams = adams_dev;
  a.phi_terms = ws->phi_terms.p;
  a.norm_mask = ws->norm.p;
  a.active_mask = ws->active.p;
  a.n = P.n;
  a.n_omega = P.d.n_omega;
  a.state = ws->state.p;
  a.store = ws->store.p;
  a.states = comp ? ws->states.p : nullptr;
  a.rates = comp ? ws->rates.p : nullptr;
  a.moments = ws->moments.p;
  a.flow = ws->flow.p;
  a.exponent = ws->exponent.p;
  a.carried = ws->carried.p;
  a.lab = ws->lab.p;
  a.source = ws->src.p;
  a.advanced = ws->adv.p;
  a.partials = ws->partials.p;
  a.norms = ws->norms.p;
  a.n_blocks = kNormBlocks;
  a.norm_arrivals = ws->norm_arrivals.p;
  return a;
}

// A pending accept written now (launched on the workspace's stream), for a reader of the
// state or of the history rows other than the next trial's predictor.
static void settle_accept(sp_workspace* ws) {
  if (ws->pending_accept < 0) return;
  const int slot = ws->pending_accept;
  ws->pending_accept = -1;
  const StepArgs a = step_args_of(ws, ws->adams.p, ws->stage.p);
  KernelTimer t(ws, SP_K_ACCEPT);
  CUDA_CHECK(launch_adams_accept(a, slot, nullptr, ws->stream));
}

// A response column whose tiles gave up waiting on one another marks the norms' status
// slot; the host turns that into an error (and clears the mark).
static void check_column(const double* h_norms, double* d_norms, cudaStream_t s) {
  if (h_norms[kColumnStatus] == 0.0) return;
  CUDA_CHECK(cudaMemsetAsync(d_norms + kColumnStatus, 0, sizeof(double), s));
  throw Failure(SP_ERR_CUDA, "response column: a tile gave up waiting for its predecessors");
}

// The attempt phase of a single run's Adams attempt, issued on the workspace's stream: the
// step's two stage slots and tables from the pinned buffers, the predictor, the source at the
// predicted field, the corrector with its reduction, the norms to the pinned host buffer.
static void issue_attempt(sp_workspace* ws, const StepArgs& a) {
  // the trial's table and the step's two stage slots, contiguous on both sides: one copy
  CUDA_CHECK(cudaMemcpyAsync(ws->adams.p, ws->h_adams, sizeof(AdamsDev) + 2 * sizeof(StageScalarsDev),
                             cudaMemcpyHostToDevice, ws->stream));
  { KernelTimer t(ws, SP_K_PREDICT); CUDA_CHECK(launch_adams_predict(a, ws->stream)); }
  eval_source(ws, ws->lab.p, 1, nullptr, ws->src.p, false, /*output=*/false);
  const OutputArgs oa = source_output_args(ws, 1, nullptr, ws->src.p, false);
  { KernelTimer t(ws, SP_K_CORRECT); CUDA_CHECK(launch_adams_correct(a, &oa, ws->stream)); }
  CUDA_CHECK(cudaMemcpyAsync(ws->h_norms, ws->norms.p, sizeof(double) * (kColumnStatus + 1),
                             cudaMemcpyDeviceToHost, ws->stream));
}

// One Adams attempt of a single run; returns accepted.  Without per-kernel timing the attempt
// phase is a CUDA graph, captured on the first attempt and replayed (one launch instead of
// nine); the copies out of the pinned tables are released by an event recorded after it.
static bool adams_attempt(sp_session* S, double dz, double end, bool kink, bool fixed) {
  sp_workspace* ws = S->ws;
  Pending pd = prepare_attempt(S, dz, end, kink, fixed);
  StepArgs a = step_args_of(ws, ws->adams.p, ws->stage.p);
  if (ws->timing) {
    issue_attempt(ws, a);
  } else {
    if (!ws->attempt_exec) {
      CUDA_CHECK(cudaStreamBeginCapture(ws->stream, cudaStreamCaptureModeThreadLocal));
      try {
        issue_attempt(ws, a);
      } catch (...) {
        cudaGraph_t partial = nullptr;
        cudaStreamEndCapture(ws->stream, &partial);
        if (partial) cudaGraphDestroy(partial);
        throw;
      }
      CUDA_CHECK(cudaStreamEndCapture(ws->stream, &ws->attempt_graph));
      CUDA_CHECK(cudaGraphInstantiate(&ws->attempt_exec, ws->attempt_graph, 0));
    }
    CUDA_CHECK(cudaGraphLaunch(ws->attempt_exec, ws->stream));
  }
  release_host_tables(ws);
  CUDA_CHECK(cudaStreamSynchronize(ws->stream));
  ws->flush_timing();
  check_column(ws->h_norms, ws->norms.p, ws->stream);
  const bool accepted = decide_attempt(S, pd, ws->h_norms);
  if (accepted) {
    if (S->defer_accept) {
      ws->pending_accept = pd.free_slot;
    } else {
      KernelTimer t(ws, SP_K_ACCEPT);
      CUDA_CHECK(launch_adams_accept(a, pd.free_slot, nullptr, ws->stream));
    }
  }
  return accepted;
}

// The attempt an adaptive march takes next: the landing rule and the equal approach
// (adams_core.py:401-470); returns (dz, end, kink).
struct Next { double dz, end; bool kink; };
static Next adams_next(const sp_session* S, double target);

// stepper/schedule.py:959-1066
struct Stop { double dz; int kind; double target; bool landed; };
static Stop landing(const sp_session* S, double z, double dz, double z_end) {
  const sp_run_desc& R = S->run;
  const double tol = kLandingUlps * ulp(std::max(std::fabs(z), std::fabs(z_end)));
  const auto& e = S->edges;
  int index = (int)(std::upper_bound(e.begin(), e.end(), z) - e.begin()) - 1;
  index = std::min(std::max(index, 0), (int)e.size() - 2);
  const double width = e[index + 1] - e[index];
  // kinds: 0 none, 1 max_step, 2 interval_width, 3 hard_kink, 4 save_plane, 5 end
  struct B { double dz; int kind; double pos; };
  B caps[3] = {{dz, 0, 0}, {R.dz_max, 1, 0}, {width, 2, 0}};
  B cap = caps[0];
  for (auto& c : caps) if (c.dz < cap.dz || (c.dz == cap.dz && c.kind > cap.kind)) cap = c;
  std::vector<B> lands;
  auto add = [&](const std::vector<double>& pos, int kind) {
    auto it = std::lower_bound(pos.begin(), pos.end(), z + tol);
    if (it != pos.end()) lands.push_back({*it - z, kind, *it});
  };
  add(S->kinks, 3);
  add(S->planes, 4);
  add(std::vector<double>{z_end}, 5);
  if (lands.empty())
    throw Failure(SP_ERR_STATE, "the march is already at or past its target (no landing ahead)");
  B best = lands[0];
  for (auto& l : lands) if (l.dz < best.dz || (l.dz == best.dz && l.kind > best.kind)) best = l;
  if (best.dz <= cap.dz) return {best.dz, best.kind, best.pos, true};
  if (best.dz <= std::min(R.stretch * cap.dz, R.dz_max)) return {best.dz, best.kind, best.pos, true};
  return {cap.dz, cap.kind, 0.0, false};
}

static Next adams_next(const sp_session* S, double target) {
  const sp_run_desc& R = S->run;
  Stop stop = landing(S, S->z, S->proposal, target);
  double dz = stop.dz;
  if (!stop.landed && R.equal_approach) {
    const double tol = kLandingUlps * ulp(std::max(std::fabs(S->z), std::fabs(target)));
    double nearest = target;
    for (const auto* pos : {&S->planes, &S->kinks}) {
      auto it = std::upper_bound(pos->begin(), pos->end(), S->z + tol);
      if (it != pos->end()) nearest = std::min(nearest, *it);
    }
    if (nearest > S->z + tol && dz < nearest - S->z && nearest - S->z < 2.0 * dz) {
      double half = 0.5 * (nearest - S->z);
      return {half, S->z + half, false};
    }
  }
  const double end = stop.landed ? stop.target : S->z + dz;
  const double tol = kLandingUlps * ulp(std::max(std::fabs(end), 1.0));
  const bool interior = end < R.z_end - tol;
  bool on_kink = false;
  if (interior) for (double k : S->kinks) on_kink |= std::fabs(k - end) <= tol;
  return {dz, end, stop.kind == 3 || on_kink};
}

static void adams_adaptive_attempt(sp_session* S, double target) {
  if (S->history.empty()) adams_start(S);
  const Next nx = adams_next(S, target);
  adams_attempt(S, nx.dz, nx.end, nx.kink, false);
}

// ---- DOPRI5 (backends/numpy_ref/engines.py:97-181)
static const double kNodes[7] = {0.0, 1.0 / 5, 3.0 / 10, 4.0 / 5, 8.0 / 9, 1.0, 1.0};
static const double kA[7][7] = {
    {0, 0, 0, 0, 0, 0, 0},
    {1.0 / 5, 0, 0, 0, 0, 0, 0},
    {3.0 / 40, 9.0 / 40, 0, 0, 0, 0, 0},
    {44.0 / 45, -56.0 / 15, 32.0 / 9, 0, 0, 0, 0},
    {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729, 0, 0, 0},
    {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656, 0, 0},
    {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84, 0}};
static const double kB[7] = {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84, 0};
static const double kBhat[7] = {5179.0 / 57600, 0, 7571.0 / 16695, 393.0 / 640, -92097.0 / 339200,
                                187.0 / 2100, 1.0 / 40};

static double rk_trial(sp_session* S, double dz) {
  sp_workspace* ws = S->ws;
  const sp_problem& P = *ws->P;
  const sp_run_desc& R = S->run;
  for (int i = 0; i < 7; ++i) fill_stage(ws, i, S->z, S->z + kNodes[i] * dz);
  fill_stage(ws, 7, S->z, S->z + dz);
  upload_stages(ws, 8);
  RkArgs a{};
  a.phi_terms = ws->phi_terms.p;
  a.norm_mask = ws->norm.p;
  a.active_mask = ws->active.p;
  a.n = P.n;
  a.n_omega = P.d.n_omega;
  a.n_phi = P.d.n_phi_terms;
  a.state = ws->state.p;
  a.stages = ws->stages.p;
  a.lab = ws->lab.p;
  a.back = ws->back.p;
  a.advanced = ws->adv.p;
  a.partials = ws->partials.p;
  a.norms = ws->norms.p;
  double e[7];
  for (int i = 0; i < 7; ++i) e[i] = kB[i] - kBhat[i];
  for (int i = 0; i < 7; ++i) {
    a.stage = ws->stage.p + i;
    { KernelTimer t(ws, SP_K_RK_STAGE); CUDA_CHECK(launch_rk_stage_input(a, i, kA[i], dz, ws->stream)); }
    eval_source(ws, ws->lab.p, i, ws->back.p, ws->stages.p + (size_t)i * P.n, false);
  }
  a.stage = ws->stage.p + 7;
  { KernelTimer t(ws, SP_K_RK_FINISH); CUDA_CHECK(launch_rk_finish(a, kB, e, dz, R.rtol, R.atol, ws->stream)); }
  CUDA_CHECK(cudaMemcpyAsync(ws->h_norms, ws->norms.p, (kColumnStatus + 1) * sizeof(double),
                             cudaMemcpyDeviceToHost, ws->stream));
  CUDA_CHECK(cudaStreamSynchronize(ws->stream));
  check_column(ws->h_norms, ws->norms.p, ws->stream);
  S->attempts += 1;
  S->evaluations += 7;
  const double scale = R.rtol * std::max(std::sqrt(ws->h_norms[0]), std::sqrt(ws->h_norms[1])) + R.atol;
  return std::sqrt(ws->h_norms[2]) / scale;
}

static void rk_accept(sp_session* S) {
  sp_workspace* ws = S->ws;
  CUDA_CHECK(launch_mask_copy(ws->state.p, ws->adv.p, ws->active.p, ws->P->n, ws->P->d.n_omega,
                              ws->stream));
}

static double rk_propose_factor(const sp_session* S) {
  const sp_run_desc& R = S->run;
  const int index = (int)S->norms_hist.size() - 1 - R.lag;
  if (index < 0) return 1.0;
  double current = S->norms_hist[index];
  if (!std::isfinite(current)) return R.min_factor;
  if (current <= 0.0) return R.max_factor;
  double previous = index >= 1 ? S->norms_hist[index - 1] : 1.0;
  if (!std::isfinite(previous) || previous <= 0.0) previous = 1.0;
  double f = R.safety * std::pow(1.0 / current, R.beta1) * std::pow(1.0 / previous, R.beta2);
  return std::min(std::max(f, R.min_factor), R.max_factor);
}

static void rk_adaptive_attempt(sp_session* S, double target) {
  const sp_run_desc& R = S->run;
  Stop stop = landing(S, S->z, S->proposal, target);
  const double dz = stop.dz;
  const double norm = rk_trial(S, dz);
  const int q1 = R.estimator_order + 1;
  const double equivalent = std::isfinite(norm) ? norm * std::pow(S->proposal / dz, q1) : norm;
  const bool accepted = std::isfinite(norm) && norm <= 1.0;
  const double end = stop.landed ? stop.target : S->z + dz;
  S->row = {end, dz, norm, accepted};
  if (accepted) {
    rk_accept(S);
    S->z = end;
    S->norms_hist.push_back(equivalent);
    if (R.auto_init && S->norms_hist.size() == 1) {
      // the start-up rule (rk_core.py:67-107, controller.py:528-561): the deadbeat step the
      // first norm implies, capped at start_growth times the first; the history records the
      // norm at that length, or zero where the cap binds
      const double growth = R.start_growth > 0.0 ? R.start_growth : 100.0;
      double factor;
      if (!std::isfinite(equivalent) || equivalent <= 0.0)
        factor = equivalent == 0.0 ? growth : R.min_factor;
      else
        factor = std::min(std::max(R.safety * std::pow(1.0 / equivalent, 1.0 / q1), R.min_factor), growth);
      const double following = limit_step(S->proposal, factor, R.dz_min, R.dz_max);
      S->norms_hist.back() = factor >= growth ? 0.0 : equivalent * std::pow(following / S->proposal, q1);
      S->proposal = following;
    }
    S->proposal = limit_step(S->proposal, rk_propose_factor(S), R.dz_min, R.dz_max);
  } else {
    S->rejected += 1;
    double f;
    if (!std::isfinite(equivalent)) f = R.min_factor;
    else if (equivalent <= 0.0) f = 1.0;
    else f = std::min(std::max(R.safety * std::pow(1.0 / equivalent, 1.0 / q1), R.min_factor), 1.0);
    S->proposal = limit_step(S->proposal, f, R.dz_min, R.dz_max);
  }
}

static void alloc_step_buffers(sp_workspace* ws, int method) {
  const sp_problem& P = *ws->P;
  const size_t n = P.n;
  if (!ws->state.p) ws->state.alloc(n);
  if (!ws->src.p) ws->src.alloc(n);
  if (!ws->adv.p) ws->adv.alloc(n);
  if (method == 0) {
    if (!ws->store.p) ws->store.alloc((size_t)kMaxSlots * n);
    if (!ws->moments.p) ws->moments.alloc((size_t)kMaxWidth * n);
    if (!ws->flow.p) ws->flow.alloc(n);
    if (!ws->exponent.p) ws->exponent.alloc(n);
    if (P.d.phi_expansion) {
      if (!ws->states.p) ws->states.alloc((size_t)kMaxSlots * n);
      if (!ws->rates.p) ws->rates.alloc((size_t)kMaxSlots * n);
      if (!ws->carried.p) ws->carried.alloc((size_t)kMaxWidth * n);
    }
    ws->store.zero(ws->stream);
    if (ws->states.p) ws->states.zero(ws->stream);
    if (ws->rates.p) ws->rates.zero(ws->stream);
  } else {
    if (!ws->stages.p) ws->stages.alloc((size_t)7 * n);
    if (!ws->back.p) ws->back.alloc(n);
  }
}

// ====================================================================== C ABI
extern "C" {

size_t sp_last_error(char* buf, size_t len) {
  if (buf && len) {
    std::strncpy(buf, g_error.c_str(), len - 1);
    buf[len - 1] = '\0';
  }
  return g_error.size();
}

const char* sp_version(void) { return "solprop-b200 0.1 sm_100a fp64"; }

int sp_device_count(void) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    g_error = std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e);
    return -SP_ERR_CUDA;
  }
  return n;
}

sp_status sp_problem_create(const sp_problem_desc* d, sp_problem** out) {
  return guarded([&] {
    if (!out) throw Failure(SP_ERR_ARGUMENT, "out is NULL");
    validate(d);
    auto P = std::make_unique<sp_problem>();
    P->d = *d;
    P->n_cols = d->n_modes * d->n_pol;
    P->n = P->n_cols * d->n_omega;
    P->omega.assign(d->omega, d->omega + d->n_omega);
    P->omega_window.assign(d->omega_window, d->omega_window + d->n_omega);
    P->t_window.assign(d->t_window, d->t_window + d->n_to);
    P->t_window_d.assign(d->t_window_derivative, d->t_window_derivative + d->n_to);
    if (d->absorber_in_stage) P->alpha.assign(d->temporal_absorber_fine, d->temporal_absorber_fine + d->n_to);
    P->crop.assign(d->crop_index, d->crop_index + d->n_omega);
    P->crop_identity = 1;
    for (int j = 0; j < d->n_omega; ++j) P->crop_identity &= (P->crop[j] == j);
    P->active.assign(d->active_mask, d->active_mask + d->n_omega);
    P->norm.assign(d->norm_mask, d->norm_mask + d->n_omega);
    P->phi_terms.assign(d->phi_terms, d->phi_terms + (size_t)2 * d->n_phi_terms * P->n);
    P->pre_terms.assign(d->prefactor_terms, d->prefactor_terms + (size_t)2 * d->n_prefactor_terms * P->n);
    const size_t n_rows = (size_t)d->n_nodes * d->n_pol_transform;
    P->synthesis.assign(d->synthesis, d->synthesis + n_rows * d->n_modes);
    P->projection.assign(d->projection, d->projection + n_rows * d->n_modes);
    if (d->plasma_enabled) {
      P->rate_coeff.assign(d->rate_coefficients, d->rate_coefficients + (size_t)4 * d->rate_intervals);
      P->taps.assign(d->taps, d->taps + d->n_taps);
    }
    P->phi_weights.load(d->phi_weights);
    P->phi_rate.load(d->phi_rate);
    P->pre_weights.load(d->prefactor_weights);
    P->density.load(d->density);
    P->kerr_density.load(d->kerr_density);
    P->plasma_density.load(d->plasma_density);
    P->preion.load(d->preionisation);
    P->taper.load(d->taper_scale);
    if (d->raman_enabled) {
      for (int r = 0; r < d->raman_terms; ++r) P->raman_rates[r].load(d->raman_rates[r]);
      P->raman_density.load(d->raman_density);
      P->raman_undamped.assign(d->raman_undamped, d->raman_undamped + (size_t)d->raman_terms * 2 * d->n_to);
      P->raman_first_row.push_back(d->raman_terms);
      P->raman_fraction.push_back(d->raman_fraction);
      P->raman_densities.push_back(P->raman_density);
      if (d->n_pol_transform == 2)
        P->raman_weights.assign(d->raman_tensor_weights, d->raman_tensor_weights + (size_t)2 * d->raman_terms);
      for (int c = 0; c < d->n_extra_raman; ++c) {  // a mixture's further components
        const sp_raman_component& rc = d->extra_raman[c];
        const int r0 = P->raman_rows();
        for (int r = 0; r < rc.terms; ++r) P->raman_rates[r0 + r].load(rc.rates[r]);
        P->raman_undamped.insert(P->raman_undamped.end(), rc.undamped,
                                 rc.undamped + (size_t)rc.terms * 2 * d->n_to);
        P->raman_first_row.push_back(r0 + rc.terms);
        P->raman_fraction.push_back(rc.fraction);
        P->raman_densities.emplace_back();
        P->raman_densities.back().load(rc.density);
        if (d->n_pol_transform == 2)
          P->raman_weights.insert(P->raman_weights.end(), rc.tensor_weights, rc.tensor_weights + (size_t)2 * rc.terms);
      }
      for (size_t r = 1; r < P->raman_weights.size(); r += 2)
        if (P->raman_weights[r] != 0.0) P->raman_kernels = 2;
    }
    if (d->n_extra_channels) {  // a mixture: every channel, the descriptor's first
      auto add = [&](double qm, double ip, const double* coeff, int n, double lmin, double dl, double fmin,
                     double fmax, double rmax, const sp_table& dens, const sp_table& pre) {
        sp_problem::Channel ch{qm, ip, lmin, dl, fmin, fmax, rmax, {}, {}, {}};
        ch.coefficients.assign(coeff, coeff + (size_t)4 * n);
        ch.density.load(dens);
        ch.preion.load(pre);
        P->channels.push_back(std::move(ch));
      };
      add(d->charge_mass_ratio, d->ionisation_potential, d->rate_coefficients, d->rate_intervals,
          d->log_field_min, d->d_log_field, d->field_min, d->field_max, d->rate_max, d->plasma_density,
          d->preionisation);
      for (int c = 0; c < d->n_extra_channels; ++c) {
        const sp_plasma_channel& e = d->extra_channels[c];
        add(e.charge_mass_ratio, e.ionisation_potential, e.rate_coefficients, e.rate_intervals, e.log_field_min,
            e.d_log_field, e.field_min, e.field_max, e.rate_max, e.plasma_density, e.preionisation);
      }
    }
    P->d.extra_channels = nullptr;  // copied above: nothing keeps the caller's arrays
    P->d.extra_raman = nullptr;
    P->d.raman_tensor_weights = nullptr;
    if (d->phi_expansion && (!P->phi_weights.present() || !P->phi_rate.present()))
      throw Failure(SP_ERR_ARGUMENT, "an expansion of Phi needs its weight and rate tables");
    *out = P.release();
  });
}

sp_status sp_problem_destroy(sp_problem* p) {
  delete p;
  return SP_OK;
}

sp_status sp_workspace_create(const sp_problem* problem, int device, sp_workspace** out) {
  return sp_workspace_create_ex(problem, device, SP_PRECISION_FP64, out);
}

sp_status sp_workspace_create_ex(const sp_problem* problem, int device, int precision,
                                 sp_workspace** out) {
  return sp_workspace_create_ex2(problem, device, precision, SP_MODAL_AUTO, out);
}

sp_status sp_workspace_create_ex2(const sp_problem* problem, int device, int precision, int modal,
                                  sp_workspace** out) {
  return guarded([&] {
    if (!problem || !out) throw Failure(SP_ERR_ARGUMENT, "NULL problem or out");
    if (precision != SP_PRECISION_FP64 && precision != SP_PRECISION_MIXED)
      throw Failure(SP_ERR_ARGUMENT, "unknown precision");
    if (modal != SP_MODAL_AUTO && modal != SP_MODAL_FUSED && modal != SP_MODAL_GEMM)
      throw Failure(SP_ERR_ARGUMENT, "unknown modal transform form");
    const sp_problem_desc& d = problem->d;
    const bool field_raman = d.grid_kind == 0 && d.raman_enabled;
    // the envelope grid's single CTA takes one column on one node without the absorber
    const bool env_products = d.grid_kind == 1 && (problem->n_cols > 1 || d.n_nodes > 1 || d.n_pol_transform > 1 ||
                                                   d.absorber_in_stage || precision == SP_PRECISION_MIXED ||
                                                   d.n_to > kMaxEnvelopeSamples);
    const bool gemm = modal == SP_MODAL_GEMM ||
                      (modal == SP_MODAL_AUTO && (problem->n_cols > kMaxModes || field_raman || env_products));
    if (!gemm && precision == SP_PRECISION_MIXED && d.grid_kind == 1)
      throw Failure(SP_ERR_REFUSED, "the mixed precision of the envelope route takes the modal transform's products");
    if (!gemm && env_products)
      throw Failure(SP_ERR_REFUSED,
                    "the envelope grid's modes, nodes, in-stage absorber and rows above 4096 samples take the modal transform's products");
    if (!gemm && problem->n_cols > kMaxModes)
      throw Failure(SP_ERR_REFUSED, "more than 8 modal columns take the modal transform's products");
    if (!gemm && field_raman)
      throw Failure(SP_ERR_REFUSED, "field-grid Raman takes the modal transform's products (its node field)");
    CUDA_CHECK(cudaSetDevice(device));
    ensure_configured(device);
    auto ws = std::make_unique<sp_workspace>();
    ws->P = problem;
    ws->device = device;
    ws->precision = precision;
    ws->gemm = gemm;
    CUDA_CHECK(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking));
    build_workspace(ws.get());
    *out = ws.release();
  });
}

sp_status sp_workspace_destroy(sp_workspace* ws) {
  delete ws;
  return SP_OK;
}

int sp_workspace_launches_per_source(const sp_workspace* ws) { return ws ? ws->launches : 0; }

sp_status sp_workspace_source_device(sp_workspace* ws, const void* lab, double z, int quiet,
                                     void* out) {
  return guarded([&] {
    if (!ws || !lab || !out) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    CUDA_CHECK(cudaSetDevice(ws->device));
    settle_accept(ws);
    fill_stage(ws, 0, z, z);
    upload_stages(ws, 1);
    eval_source(ws, (const double2*)lab, 0, nullptr, (double2*)out, quiet != 0);
  });
}

sp_status sp_workspace_source(sp_workspace* ws, const double* lab, double z, int quiet, double* out) {
  return guarded([&] {
    if (!ws || !lab || !out) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    CUDA_CHECK(cudaSetDevice(ws->device));
    settle_accept(ws);
    const size_t bytes = (size_t)ws->P->n * sizeof(double2);
    CUDA_CHECK(cudaMemcpyAsync(ws->lab.p, lab, bytes, cudaMemcpyHostToDevice, ws->stream));
    fill_stage(ws, 0, z, z);
    upload_stages(ws, 1);
    eval_source(ws, ws->lab.p, 0, nullptr, ws->out.p, quiet != 0);
    CUDA_CHECK(cudaMemcpyAsync(out, ws->out.p, bytes, cudaMemcpyDeviceToHost, ws->stream));
    CUDA_CHECK(cudaMemcpyAsync(ws->h_norms, ws->norms.p, (kColumnStatus + 1) * sizeof(double),
                               cudaMemcpyDeviceToHost, ws->stream));
    CUDA_CHECK(cudaStreamSynchronize(ws->stream));
    check_column(ws->h_norms, ws->norms.p, ws->stream);
  });
}

sp_status sp_session_start(sp_workspace* ws, const sp_run_desc* run, sp_session** out) {
  return guarded([&] {
    if (!ws || !run || !out || !run->field0) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    if (run->method != 0 && run->method != 1) throw Failure(SP_ERR_ARGUMENT, "unknown method");
    if (run->method == 0 && (run->order < 1 || run->order > 5))
      throw Failure(SP_ERR_ARGUMENT, "Adams order must lie in [1, 5]");
    CUDA_CHECK(cudaSetDevice(ws->device));
    settle_accept(ws);  // a session before this one on the workspace
    auto S = std::make_unique<sp_session>();
    S->ws = ws;
    S->run = *run;
    S->defer_accept = true;
    S->planes.assign(run->save_planes, run->save_planes + run->n_save_planes);
    S->kinks.assign(run->hard_kinks, run->hard_kinks + run->n_hard_kinks);
    S->edges.assign(run->breakpoints, run->breakpoints + run->n_breakpoints);
    if (S->edges.size() < 2) S->edges = {run->z_start, run->z_end};
    if (run->schedule && run->n_schedule > 0) {
      S->schedule.assign(run->schedule, run->schedule + run->n_schedule);
      S->sched_edges.assign(1, run->z_start);
      for (double dz : S->schedule) S->sched_edges.push_back(S->sched_edges.back() + dz);
    }
    S->z = run->z_start;
    S->proposal = run->proposal;
    S->order = run->variable_order ? 1 : run->order;
    alloc_step_buffers(ws, run->method);
    const size_t bytes = (size_t)ws->P->n * sizeof(double2);
    CUDA_CHECK(cudaMemcpyAsync(ws->adv.p, run->field0, bytes, cudaMemcpyHostToDevice, ws->stream));
    CUDA_CHECK(launch_mask_copy(ws->state.p, ws->adv.p, ws->active.p, ws->P->n, ws->P->d.n_omega,
                                ws->stream));
    CUDA_CHECK(cudaStreamSynchronize(ws->stream));
    *out = S.release();
  });
}

static int category_of(sp_status code) {
  switch (code) {
    case SP_ERR_CONVERGENCE: return SP_CATEGORY_CONVERGENCE;
    case SP_ERR_CUDA: return SP_CATEGORY_BACKEND;
    case SP_ERR_REFUSED: return SP_CATEGORY_REFUSED;
    default: return SP_CATEGORY_VALUE;
  }
}

sp_status sp_session_advance(sp_session* S, int32_t work_limit, double deadline, sp_batch* out) {
  return guarded([&] {
    if (!S || !out) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    if (out->rows && out->rows_capacity < 0) throw Failure(SP_ERR_ARGUMENT, "negative rows_capacity");
    if (S->failed) throw Failure(SP_ERR_STATE, "the session failed; close it");
    if (S->stopped) throw Failure(SP_ERR_STATE, "the session was stopped; close it");
    CUDA_CHECK(cudaSetDevice(S->ws->device));
    out->event = SP_EVENT_NONE;
    out->plane_index = -1;
    out->reason = SP_REASON_BOUND;
    out->category = SP_CATEGORY_NONE;
    out->n_rows = 0;
    const sp_run_desc& R = S->run;
    const auto t_call = std::chrono::steady_clock::now();
    const bool timed = std::isfinite(deadline) && deadline > 0.0;
    auto counts = [&] {
      out->z = S->z;
      out->attempts = S->attempts;
      out->rejected = S->rejected;
      out->evaluations = S->evaluations;
    };
    int done = 0;
    try {
      if (!S->finished && reached(S->z, R.z_end)) {
        S->finished = true;
        out->event = SP_EVENT_FINISHED;
        out->reason = SP_REASON_REACHED;
      }
      while (!S->finished && done < work_limit) {
        if (S->stop_requested.load()) {
          S->stopped = true;
          out->event = SP_EVENT_STOPPED;
          out->reason = SP_REASON_STOPPED;
          break;
        }
        // the next stop: a save plane or the end
        double target = R.z_end;
        int plane = -1;
        while (S->plane_cursor < (int)S->planes.size() &&
               reached(S->z, S->planes[S->plane_cursor]))
          ++S->plane_cursor;
        if (S->plane_cursor < (int)S->planes.size()) {
          target = S->planes[S->plane_cursor];
          plane = S->plane_cursor;
        }
        const auto t_attempt = std::chrono::steady_clock::now();
        if (!S->schedule.empty()) {
          if (S->sched_cursor >= (int)S->schedule.size()) {
            S->finished = true;
            out->event = SP_EVENT_FINISHED;
            out->reason = SP_REASON_REACHED;
            break;
          }
          const double dz = S->schedule[S->sched_cursor];
          const double end = S->sched_edges[S->sched_cursor + 1];
          if (R.method == 0) {
            if (S->history.empty()) adams_start(S);
            adams_attempt(S, dz, end, false, true);
          } else {
            double nm = rk_trial(S, dz);
            S->row = {end, dz, nm, true};
            if (!std::isfinite(nm))
              throw Failure(SP_ERR_CONVERGENCE, "a replayed step diverged", SP_REASON_DIVERGED);
            rk_accept(S);
            S->z = end;
          }
          ++S->sched_cursor;
        } else if (R.method == 0) {
          adams_adaptive_attempt(S, target);
        } else {
          rk_adaptive_attempt(S, target);
        }
        ++done;
        const auto t_now = std::chrono::steady_clock::now();
        if (out->rows && out->n_rows < out->rows_capacity) {
          double* r = out->rows + (size_t)5 * out->n_rows++;
          r[0] = S->row.end;
          r[1] = S->row.step;
          r[2] = std::isfinite(S->row.norm) ? S->row.norm : INFINITY;
          r[3] = S->row.accepted ? 1.0 : 0.0;
          r[4] = std::chrono::duration<double>(t_now - t_attempt).count();
        }
        const bool on_plane =
            plane >= 0 && std::fabs(S->z - S->planes[plane]) <=
                              std::max(1e-9 * std::fabs(R.z_end), kLandingUlps * ulp(S->planes[plane]));
        if (on_plane) {
          ++S->plane_cursor;
          out->plane_index = plane;
        }
        if (reached(S->z, R.z_end)) {
          S->finished = true;
          out->event = SP_EVENT_FINISHED;
          out->reason = SP_REASON_REACHED;
          break;
        }
        if (on_plane) {
          out->event = SP_EVENT_PLANE;
          out->reason = SP_REASON_REACHED;
          break;
        }
        if (S->row.accepted && S->snapshot_requested.exchange(false)) {
          out->event = SP_EVENT_HALTED;
          out->reason = SP_REASON_HALTED;
          break;
        }
        if (timed && std::chrono::duration<double>(t_now - t_call).count() >= deadline) break;
      }
    } catch (const Failure& f) {
      S->failed = true;
      out->event = SP_EVENT_FAILED;
      out->reason = f.reason;
      out->category = category_of(f.code);
      counts();
      throw;
    }
    counts();
  });
}

sp_status sp_session_request_stop(sp_session* S) {
  if (!S) return SP_ERR_ARGUMENT;
  S->stop_requested.store(true);
  return SP_OK;
}

sp_status sp_session_request_snapshot(sp_session* S) {
  if (!S) return SP_ERR_ARGUMENT;
  S->snapshot_requested.store(true);
  return SP_OK;
}

sp_status sp_session_march_state(const sp_session* S, sp_march_state* out) {
  return guarded([&] {
    if (!S || !out) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    out->z = S->z;
    out->proposal = S->proposal;
    out->attempts = S->attempts;
    out->rejected = S->rejected;
    out->evaluations = S->evaluations;
    out->order = S->order;
    out->history_rows = (int32_t)S->history.size();
    out->rejections = S->rejections;
    out->plane_index = S->plane_cursor;
    out->outcome = S->failed ? 3 : S->stopped ? 2 : S->finished ? 1 : 0;
  });
}

// ---- plane statistics of a workspace's state, formed on the device; the small results
// alone come back (native statistics.cpp, solprop stats/definitions.py)
static void plane_statistics(sp_workspace* ws, const double* power_weight, sp_statistics* out) {
  const sp_problem& P = *ws->P;
  const sp_problem_desc& d = P.d;
  const bool envelope = d.grid_kind == 1;
  if (envelope ? d.n_omega != d.n_t : d.n_omega != d.n_t / 2 + 1)
    throw Failure(SP_ERR_REFUSED, "statistics need the coarse grid's full spectrum");
  const bool peaks = out->peak_power || out->peak_power_total;
  if (peaks && (d.n_t & (d.n_t - 1)))
    throw Failure(SP_ERR_REFUSED, "peak powers need a power-of-two coarse grid");
  if (d.n_modes > kStatMaxModes) throw Failure(SP_ERR_REFUSED, "statistics of more than 32 modes");
  if (!ws->state.p) throw Failure(SP_ERR_STATE, "the workspace holds no state");
  const size_t n = P.n;
  const int peak_offset = 2 * P.n_cols, spectrum_offset = peak_offset + d.n_modes + 1;
  if (!ws->stat_out.p) {
    ws->stat_out.alloc((size_t)spectrum_offset + d.n_omega);
    ws->stat_power.alloc((size_t)P.n_cols * d.n_t);
  }
  if (power_weight) {
    for (size_t i = 0; i < n; ++i)
      if (!(power_weight[i] > 0.0) || !std::isfinite(power_weight[i]))
        throw Failure(SP_ERR_ARGUMENT, "power weights must be positive and finite");
    if (!ws->stat_weight.p) ws->stat_weight.alloc(n);
    CUDA_CHECK(cudaMemcpyAsync(ws->stat_weight.p, power_weight, n * sizeof(double),
                               cudaMemcpyHostToDevice, ws->stream));
  }
  StatisticsArgs a{};
  a.state = ws->state.p;
  a.power_weight = power_weight ? ws->stat_weight.p : nullptr;
  a.omega = ws->omega.p;
  a.twiddles = ws->twiddles.p;
  a.power = ws->stat_power.p;
  a.out = ws->stat_out.p;
  a.n_modes = d.n_modes;
  a.n_pol = d.n_pol;
  a.n_cols = P.n_cols;
  a.n_omega = d.n_omega;
  a.n_t = d.n_t;
  a.log_m = std::min(ilog2(std::max(d.n_t, 1)), kStatLogRow);
  a.log_table = ws->log_n_to;
  a.envelope = envelope;
  a.dt = d.dt;
  a.peak_offset = peak_offset;
  a.spectrum_offset = spectrum_offset;
  CUDA_CHECK(launch_statistics(a, peaks, ws->stream));
  std::vector<double> h((size_t)spectrum_offset + d.n_omega);
  CUDA_CHECK(cudaMemcpyAsync(h.data(), ws->stat_out.p, h.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, ws->stream));
  CUDA_CHECK(cudaStreamSynchronize(ws->stream));
  if (out->energy) std::copy(h.begin(), h.begin() + P.n_cols, out->energy);
  if (out->omega0) std::copy(h.begin() + P.n_cols, h.begin() + 2 * P.n_cols, out->omega0);
  if (out->peak_power) std::copy(h.begin() + peak_offset, h.begin() + peak_offset + d.n_modes, out->peak_power);
  if (out->peak_power_total) *out->peak_power_total = h[peak_offset + d.n_modes];
  if (out->spectrum) std::copy(h.begin() + spectrum_offset, h.end(), out->spectrum);
}

sp_status sp_session_statistics(sp_session* S, const double* power_weight, sp_statistics* out) {
  return guarded([&] {
    if (!S || !out) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    CUDA_CHECK(cudaSetDevice(S->ws->device));
    settle_accept(S->ws);
    plane_statistics(S->ws, power_weight, out);
  });
}

// ---- snapshots: the march's scalars, its history positions and the device rows a later
// attempt reads (the state, the Adams history rows of sources, and with a varying
// operator the rows of states and rates), as one byte string with a header that names
// the problem's shape, so that a restore on another problem is refused.
namespace {
struct SnapshotHeader {
  char magic[8];
  int32_t version, method, compensated, n_slots;
  int64_t n, n_modes, n_pol, n_omega;
  double z, proposal;
  int64_t attempts, rejected, evaluations;
  int32_t plane_cursor, sched_cursor, finished, rejections, order, last_rejected;
  int64_t n_history, n_norms;
};
constexpr char kSnapshotMagic[8] = {'s', 'p', 's', 'n', 'a', 'p', '\0', '\0'};

struct SnapshotLayout {
  size_t history, norms, state, rows, total;
  int row_buffers;  // device row buffers after the state: 0 (RK), 1 (store) or 3
};

SnapshotLayout snapshot_layout(int method, bool compensated, size_t n, size_t n_history, size_t n_norms) {
  SnapshotLayout L{};
  L.history = sizeof(SnapshotHeader);
  L.norms = L.history + n_history * 2 * sizeof(double);
  L.state = L.norms + n_norms * sizeof(double);
  L.rows = L.state + n * sizeof(double2);
  L.row_buffers = method == 0 ? (compensated ? 3 : 1) : 0;
  L.total = L.rows + (size_t)L.row_buffers * kMaxSlots * n * sizeof(double2);
  return L;
}
}  // namespace

sp_status sp_session_snapshot(sp_session* S, void* buf, size_t capacity, size_t* size) {
  return guarded([&] {
    if (!S || !size) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    if (S->failed) throw Failure(SP_ERR_STATE, "the session failed; there is nothing to resume");
    sp_workspace* ws = S->ws;
    const sp_problem& P = *ws->P;
    const bool comp = S->run.method == 0 && P.d.phi_expansion;
    const SnapshotLayout L =
        snapshot_layout(S->run.method, comp, P.n, S->history.size(), S->norms_hist.size());
    *size = L.total;
    if (!buf) return;
    if (capacity < L.total) throw Failure(SP_ERR_ARGUMENT, "the snapshot buffer is too small");
    CUDA_CHECK(cudaSetDevice(ws->device));
    settle_accept(ws);  // the state and the history rows as accepted
    unsigned char* b = static_cast<unsigned char*>(buf);
    SnapshotHeader h{};
    std::memcpy(h.magic, kSnapshotMagic, sizeof h.magic);
    h.version = 1;
    h.method = S->run.method;
    h.compensated = comp;
    h.n_slots = kMaxSlots;
    h.n = (int64_t)P.n;
    h.n_modes = P.d.n_modes;
    h.n_pol = P.d.n_pol;
    h.n_omega = P.d.n_omega;
    h.z = S->z;
    h.proposal = S->proposal;
    h.attempts = S->attempts;
    h.rejected = S->rejected;
    h.evaluations = S->evaluations;
    h.plane_cursor = S->plane_cursor;
    h.sched_cursor = S->sched_cursor;
    h.finished = S->finished;
    h.rejections = S->rejections;
    h.order = S->order;
    h.last_rejected = S->last_rejected;
    h.n_history = (int64_t)S->history.size();
    h.n_norms = (int64_t)S->norms_hist.size();
    std::memcpy(b, &h, sizeof h);
    double* hist = reinterpret_cast<double*>(b + L.history);
    for (size_t i = 0; i < S->history.size(); ++i) {
      hist[2 * i] = S->history[i].first;
      hist[2 * i + 1] = (double)S->history[i].second;
    }
    if (!S->norms_hist.empty())
      std::memcpy(b + L.norms, S->norms_hist.data(), S->norms_hist.size() * sizeof(double));
    const size_t row = P.n * sizeof(double2);
    CUDA_CHECK(cudaMemcpyAsync(b + L.state, ws->state.p, row, cudaMemcpyDeviceToHost, ws->stream));
    const double2* rows[3] = {ws->store.p, ws->states.p, ws->rates.p};
    for (int k = 0; k < L.row_buffers; ++k)
      CUDA_CHECK(cudaMemcpyAsync(b + L.rows + (size_t)k * kMaxSlots * row, rows[k], kMaxSlots * row,
                                 cudaMemcpyDeviceToHost, ws->stream));
    CUDA_CHECK(cudaStreamSynchronize(ws->stream));
  });
}

sp_status sp_session_restore(sp_workspace* ws, const sp_run_desc* run, const void* snapshot,
                             size_t size, sp_session** out) {
  return guarded([&] {
    if (!ws || !run || !snapshot || !out) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    if (size < sizeof(SnapshotHeader)) throw Failure(SP_ERR_ARGUMENT, "not a snapshot: too short");
    SnapshotHeader h;
    std::memcpy(&h, snapshot, sizeof h);
    if (std::memcmp(h.magic, kSnapshotMagic, sizeof h.magic) != 0 || h.version != 1)
      throw Failure(SP_ERR_ARGUMENT, "not a snapshot of this library");
    const sp_problem& P = *ws->P;
    if (h.method != run->method) throw Failure(SP_ERR_ARGUMENT, "the snapshot is of another method");
    if (h.n != (int64_t)P.n || h.n_modes != P.d.n_modes || h.n_pol != P.d.n_pol ||
        h.n_omega != P.d.n_omega || h.n_slots != kMaxSlots ||
        h.compensated != (run->method == 0 && P.d.phi_expansion))
      throw Failure(SP_ERR_ARGUMENT, "the snapshot is of another problem");
    if (h.n_history < 0 || h.n_norms < 0 || h.n_history > kMaxSlots)
      throw Failure(SP_ERR_ARGUMENT, "a corrupt snapshot");
    const SnapshotLayout L = snapshot_layout(h.method, h.compensated, P.n, (size_t)h.n_history,
                                             (size_t)h.n_norms);
    if (size < L.total) throw Failure(SP_ERR_ARGUMENT, "a truncated snapshot");
    // start the session as sp_session_start does, with the snapshot's state as the field
    const unsigned char* b = static_cast<const unsigned char*>(snapshot);
    sp_run_desc r = *run;
    r.field0 = reinterpret_cast<const double*>(b + L.state);
    sp_session* raw = nullptr;
    const sp_status st = sp_session_start(ws, &r, &raw);
    if (st != SP_OK) throw Failure(st, g_error);
    std::unique_ptr<sp_session> S(raw);
    S->run.field0 = nullptr;  // the caller's pointer is not kept
    // the state exactly as saved (the start masked it: the saved one is already masked)
    const size_t row = P.n * sizeof(double2);
    CUDA_CHECK(cudaMemcpyAsync(ws->state.p, b + L.state, row, cudaMemcpyHostToDevice, ws->stream));
    double2* rows[3] = {ws->store.p, ws->states.p, ws->rates.p};
    for (int k = 0; k < L.row_buffers; ++k)
      CUDA_CHECK(cudaMemcpyAsync(rows[k], b + L.rows + (size_t)k * kMaxSlots * row, kMaxSlots * row,
                                 cudaMemcpyHostToDevice, ws->stream));
    S->z = h.z;
    S->proposal = h.proposal;
    S->attempts = h.attempts;
    S->rejected = h.rejected;
    S->evaluations = h.evaluations;
    S->plane_cursor = h.plane_cursor;
    S->sched_cursor = h.sched_cursor;
    S->finished = h.finished != 0;
    S->rejections = h.rejections;
    S->order = h.order;
    S->last_rejected = h.last_rejected != 0;
    const double* hist = reinterpret_cast<const double*>(b + L.history);
    S->history.clear();
    for (int64_t i = 0; i < h.n_history; ++i) {
      const int slot = (int)hist[2 * i + 1];
      if (slot < 0 || slot >= kMaxSlots) throw Failure(SP_ERR_ARGUMENT, "a corrupt snapshot");
      S->history.push_back({hist[2 * i], slot});
    }
    S->norms_hist.assign(reinterpret_cast<const double*>(b + L.norms),
                         reinterpret_cast<const double*>(b + L.norms) + h.n_norms);
    if (S->sched_cursor < 0 || S->sched_cursor > (int)S->schedule.size() || S->plane_cursor < 0)
      throw Failure(SP_ERR_ARGUMENT, "the snapshot's cursors do not fit the run");
    CUDA_CHECK(cudaStreamSynchronize(ws->stream));
    *out = S.release();
  });
}

sp_status sp_session_export(sp_session* S, double* out) {
  return guarded([&] {
    if (!S || !out) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    CUDA_CHECK(cudaSetDevice(S->ws->device));
    settle_accept(S->ws);
    const size_t bytes = (size_t)S->ws->P->n * sizeof(double2);
    CUDA_CHECK(cudaMemcpyAsync(out, S->ws->state.p, bytes, cudaMemcpyDeviceToHost, S->ws->stream));
    CUDA_CHECK(cudaStreamSynchronize(S->ws->stream));
  });
}

sp_status sp_session_destroy(sp_session* S) {
  delete S;
  return SP_OK;
}

void* sp_workspace_stream(sp_workspace* ws) { return ws ? (void*)ws->stream : nullptr; }

sp_status sp_session_set_timing(sp_session* S, int enable) {
  return guarded([&] {
    if (!S) throw Failure(SP_ERR_ARGUMENT, "NULL session");
    S->ws->flush_timing();
    S->ws->timing = enable != 0;
  });
}

sp_status sp_session_timing(sp_session* S, double* ms, int64_t* launches, int reset) {
  return guarded([&] {
    if (!S || !ms || !launches) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    sp_workspace* ws = S->ws;
    ws->flush_timing();
    for (int k = 0; k < SP_K_COUNT; ++k) {
      ms[k] = ws->t_ms[k];
      launches[k] = ws->t_count[k];
      if (reset) {
        ws->t_ms[k] = 0.0;
        ws->t_count[k] = 0;
      }
    }
  });
}

}  // extern "C"

// ====================================================================== scans
// sp_scan: many independent runs stepped together.  Every batch step gives each
// unfinished run one exponential-Adams attempt: one staging upload of all runs' tables
// and flags, the batched launches (predict, inverse FFT per grid size, the three column
// passes, forward FFT per grid size, stage output, correct and its reductions), one
// read-back of all runs' norms, the host's decisions, and a batched accept.
namespace {

// a transform's forms: one CTA per row (width 0), or a cluster of 2, 4 or 8 CTAs per row
constexpr int kForms = 4;
constexpr int kFormWidth[kForms] = {0, 2, 4, 8};

struct FftClass {
  int n_to = 0;
  int inv_form = 0, fwd_form = 0;  // indices into kFormWidth
  // the autotuner's measurements by form (ms per launch over this class's rows; < 0: not
  // a candidate)
  float inv_ms[kForms] = {-1, -1, -1, -1}, fwd_ms[kForms] = {-1, -1, -1, -1};
  DevBuf<int2> inv_items, fwd_items;
  int n_inv = 0, n_fwd = 0;
};

// the largest transform row (complex samples x element size) one CTA's shared memory
// takes (the single-CTA transforms are configured for 200 KB)
constexpr size_t kBatchedRowBytes = 128 * 1024;

template <class T>
T* pinned(size_t n) {
  T* p = nullptr;
  CUDA_CHECK(cudaMallocHost(&p, sizeof(T) * std::max<size_t>(n, 1)));
  std::memset(p, 0, sizeof(T) * std::max<size_t>(n, 1));
  return p;
}

}  // namespace

struct sp_scan {
  int device = 0;
  cudaStream_t stream = nullptr;
  int R = 0;
  std::vector<std::unique_ptr<sp_workspace>> ws;
  std::vector<std::unique_ptr<sp_session>> ss;
  std::vector<int> done;
  std::vector<Pending> pending;
  int precision = SP_PRECISION_FP64;
  DevBuf<InverseArgs> inv_start, inv_att;
  DevBuf<ColumnTileArgs> col_start, col_att;
  DevBuf<ForwardArgs> fwd;
  DevBuf<ColumnArgsT<float>> col32_start, col32_att;
  DevBuf<ForwardArgsT<float>> fwd32;
  DevBuf<OutputArgs> out_start, out_att;
  DevBuf<StepArgs> step_start, step_att;
  DevBuf<AdamsDev> adams_start, adams_att;
  DevBuf<StageScalarsDev> stages_start, stages_att;
  DevBuf<double> norms;
  DevBuf<int> flag_start, flag_att, flag_accept;
  DevBuf<int2> step_items, out_items;
  DevBuf<int4> col_items, sweep_items;
  int n_step_items = 0, n_out_items = 0, n_col_items = 0, n_sweep_items = 0;
  // the column's form, chosen by tune_column: one CTA per (tile, node group) with the
  // running integrals handed over between CTAs, or one CTA per (run, node group) walking
  // the tiles (ms per launch over all runs; < 0: not timed)
  bool column_sweep = false;
  float column_tile_ms = -1, column_sweep_ms = -1;
  // host copies of the forward records (their n_groups follows the column's form)
  std::vector<ForwardArgs> h_fwd;
  std::vector<ForwardArgsT<float>> h_fwd32;
  std::vector<int> groups;  // node groups per run
  // host threads for the per-run work between the batched launches
  std::unique_ptr<HostPool> pool;
  // the runs' work-list sizes, and the re-planning as runs finish: every batched launch
  // covers the runs still going; when their number has halved since the last plan, the
  // lists are rebuilt and the column's and transforms' forms tuned again
  struct RunWork {
    int n_to, step_blocks, out_blocks, col_blocks, groups, tiles, cols, fwd_rows;
  };
  std::vector<RunWork> work;
  int planned_active = 0, replans = 0;
  // the tail: once no more than kTailRuns runs are going, each goes on as a single run (its
  // own stream, on a host thread of its own), one attempt per batch step
  bool tail = false;
  int64_t tail_from = -1;  // the batch step the tail began at
  // runs gone on alone: a run whose remaining attempts (distance left over its next step)
  // exceed alone_factor x the median of the batch's and alone_min leaves the batch, which
  // it would hold back for many steps, and goes on as a single run on a host thread of its
  // own, side by side with the batched steps (at most alone_max at a time)
  std::vector<int> alone;
  int alone_max = 6, alone_count = 0;
  double alone_min = 2000.0, alone_factor = 4.0;
  std::vector<std::unique_ptr<FftClass>> classes;
  AdamsDev *h_adams_start = nullptr, *h_adams_att = nullptr;
  StageScalarsDev *h_stages_start = nullptr, *h_stages_att = nullptr;
  double* h_norms = nullptr;
  int *h_flag_start = nullptr, *h_flag_att = nullptr, *h_flag_accept = nullptr;
  int64_t batch_steps = 0;
  // host time per batch step, summed over the steps: the runs' preparation before the
  // attempt phase, the wait for it, and the decisions after it (ms)
  double host_prepare_ms = 0, host_wait_ms = 0, host_decide_ms = 0;
  // the attempt phase (uploads, predictor, source, corrector, norms read-back) as one
  // CUDA graph, captured at the first attempt and replayed at every later one
  cudaGraphExec_t attempt_graph = nullptr;
  bool graph_failed = false;
  // per-family device timing (sp_scan_set_timing): events around every batched launch
  // family, the attempt phase launched plainly meanwhile
  bool timing = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
  size_t ev_next = 0;
  double t_ms[SP_K_COUNT] = {};
  int64_t t_count[SP_K_COUNT] = {};
  ~sp_scan() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto e : ev_pool) cudaEventDestroy(e);
    if (attempt_graph) cudaGraphExecDestroy(attempt_graph);
    for (void* p : {(void*)h_adams_start, (void*)h_adams_att, (void*)h_stages_start,
                    (void*)h_stages_att, (void*)h_norms, (void*)h_flag_start, (void*)h_flag_att,
                    (void*)h_flag_accept})
      if (p) cudaFreeHost(p);
    ss.clear();
    ws.clear();
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

template <class T>
void upload_all(DevBuf<T>& dev, const T* host, size_t n, cudaStream_t s) {
  CUDA_CHECK(cudaMemcpyAsync(dev.p, host, n * sizeof(T), cudaMemcpyHostToDevice, s));
}

// One batched launch family, with events around it while the scan's timing is on.
template <class F>
void timed_family(sp_scan* S, int kind, F&& launch) {
  if (!S->timing) {
    launch();
    return;
  }
  auto event = [&] {
    if (S->ev_next == S->ev_pool.size()) {
      cudaEvent_t e;
      CUDA_CHECK(cudaEventCreate(&e));
      S->ev_pool.push_back(e);
    }
    return S->ev_pool[S->ev_next++];
  };
  cudaEvent_t a = event(), b = event();
  CUDA_CHECK(cudaEventRecord(a, S->stream));
  launch();
  CUDA_CHECK(cudaEventRecord(b, S->stream));
  S->ev_pending.push_back({kind, {a, b}});
}

void flush_scan_timing(sp_scan* S) {
  if (S->ev_pending.empty()) return;
  CUDA_CHECK(cudaStreamSynchronize(S->stream));
  for (auto& p : S->ev_pending) {
    float ms = 0.f;
    CUDA_CHECK(cudaEventElapsedTime(&ms, p.second.first, p.second.second));
    S->t_ms[p.first] += ms;
    S->t_count[p.first] += 1;
  }
  S->ev_pending.clear();
  S->ev_next = 0;
}

// Which forms a class's rows may take: one CTA when the row fits its shared memory, a
// cluster of C CTAs when the row is longer than 4096 real samples and a CTA's share fits.
bool inverse_form_ok(int n_to, int form) {
  const int C = kFormWidth[form];
  if (!C) return (size_t)(n_to / 2) * 16 <= kBatchedRowBytes;
  return fft_cluster_size(n_to) > 1 && cluster_transform_smem(n_to, C, 16, false) <= kClusterSmem;
}
bool forward_form_ok(int n_to, int form, size_t elem) {
  const int C = kFormWidth[form];
  if (!C) return (size_t)(n_to / 2) * elem <= kBatchedRowBytes;
  return fft_cluster_size(n_to) > 1 && cluster_transform_smem(n_to, C, elem, true) <= kClusterSmem;
}

cudaError_t launch_inverse_form(const InverseArgs* inv, const FftClass& c, int form, const int* flags,
                                cudaStream_t s) {
  const int C = kFormWidth[form];
  return C ? launch_inverse_cluster_b(inv, c.inv_items.p, flags, c.n_inv, c.n_to, C, s)
           : launch_inverse_b(inv, c.inv_items.p, flags, c.n_inv, c.n_to, s);
}
template <class R>
cudaError_t launch_forward_form(const ForwardArgsT<R>* fwd, const FftClass& c, int form, const int* flags,
                                cudaStream_t s) {
  const int C = kFormWidth[form];
  return C ? launch_forward_cluster_b(fwd, c.fwd_items.p, flags, c.n_fwd, c.n_to, C, s)
           : launch_forward_b(fwd, c.fwd_items.p, flags, c.n_fwd, c.n_to, s);
}

// a work list rewritten in place (the lists only shrink after the first plan)
template <class T>
void refill(DevBuf<T>& dev, const std::vector<T>& host, cudaStream_t s, bool first) {
  if (first) {
    dev.upload(host.data(), host.size(), s);
    return;
  }
  if (host.size() > dev.n) throw Failure(SP_ERR_ARGUMENT, "a scan's work list grew after its first plan");
  if (!host.empty())
    CUDA_CHECK(cudaMemcpyAsync(dev.p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

// The batched launches' work lists for the runs with live[r] set: the stepping and output
// blocks, both forms of the column (the sweep's longest rows first), and every grid
// size's transform rows.
void plan_items(sp_scan* S, const std::vector<int>& live, bool first) {
  std::vector<int2> step, out;
  std::vector<int4> col, sweep;
  for (int r = 0; r < S->R; ++r) {
    if (!live[r]) continue;
    const auto& w = S->work[r];
    for (int b = 0; b < w.step_blocks; ++b) step.push_back(make_int2(r, b));
    for (int b = 0; b < w.out_blocks; ++b) out.push_back(make_int2(r, b));
    for (int b = 0; b < w.col_blocks; ++b) col.push_back(make_int4(r, b, 0, 0));
    for (int g = 0; g < w.groups; ++g) sweep.push_back(make_int4(r, g, 0, 0));
  }
  std::stable_sort(sweep.begin(), sweep.end(), [&](const int4& x, const int4& y) {
    return S->work[x.x].tiles > S->work[y.x].tiles;
  });
  refill(S->step_items, step, S->stream, first);
  refill(S->out_items, out, S->stream, first);
  refill(S->col_items, col, S->stream, first);
  refill(S->sweep_items, sweep, S->stream, first);
  S->n_step_items = (int)step.size();
  S->n_out_items = (int)out.size();
  S->n_col_items = (int)col.size();
  S->n_sweep_items = (int)sweep.size();
  for (auto& c : S->classes) {
    std::vector<int2> inv, fwd;
    for (int r = 0; r < S->R; ++r) {
      if (!live[r] || S->work[r].n_to != c->n_to) continue;
      for (int k = 0; k < S->work[r].cols; ++k) inv.push_back(make_int2(r, k));
      for (int k = 0; k < S->work[r].fwd_rows; ++k) fwd.push_back(make_int2(r, k));
    }
    refill(c->inv_items, inv, S->stream, first);
    refill(c->fwd_items, fwd, S->stream, first);
    c->n_inv = (int)inv.size();
    c->n_fwd = (int)fwd.size();
  }
  int active = 0;
  for (int r = 0; r < S->R; ++r) active += live[r] != 0;
  S->planned_active = active;
}

template <class R>
void scan_transforms(sp_scan* S, const int* flags, const InverseArgs* inv, const ColumnArgsT<R>* col,
                     const ForwardArgsT<R>* fwd) {
  timed_family(S, SP_K_INVERSE, [&] {
    for (auto& c : S->classes)
      if (c->n_inv) CUDA_CHECK(launch_inverse_form(inv, *c, c->inv_form, flags, S->stream));
  });
  timed_family(S, SP_K_COLUMN, [&] {
    if (S->column_sweep)
      CUDA_CHECK(launch_column_sweep_b(col, S->sweep_items.p, flags, S->n_sweep_items, S->stream));
    else
      CUDA_CHECK(launch_column_b(col, S->col_items.p, flags, S->n_col_items, S->stream));
  });
  timed_family(S, SP_K_FORWARD, [&] {
    for (auto& c : S->classes)
      if (c->n_fwd) CUDA_CHECK(launch_forward_form(fwd, *c, c->fwd_form, flags, S->stream));
  });
}

// The scan's transform autotuner: for every grid size, time every form each transform may
// take (one CTA per row; clusters of 2, 4 and 8 CTAs) on this scan's own rows (one warm-up
// and three timed launches each, every run selected) and keep the fastest.  The launches
// write the workspaces' scratch rows only.
template <class R>
void tune_transforms(sp_scan* S, const ForwardArgsT<R>* fwd, const std::vector<int>& live) {
  DevBuf<int> all;
  all.upload(live.data(), live.size(), S->stream);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  auto time = [&](auto&& launch) -> float {
    CUDA_CHECK(launch());
    CUDA_CHECK(cudaEventRecord(e0, S->stream));
    for (int i = 0; i < 3; ++i) CUDA_CHECK(launch());
    CUDA_CHECK(cudaEventRecord(e1, S->stream));
    CUDA_CHECK(cudaEventSynchronize(e1));
    float ms = 0;
    CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    return ms / 3;
  };
  const size_t elem = sizeof(cplx<R>);
  for (auto& c : S->classes) {
    if (!c->n_inv) continue;  // no run of this grid size is going
    int n_inv = 0, n_fwd = 0;
    for (int f = 0; f < kForms; ++f) {
      n_inv += inverse_form_ok(c->n_to, f);
      n_fwd += forward_form_ok(c->n_to, f, elem);
    }
    for (int f = 0; f < kForms && n_inv > 1; ++f) {
      if (!inverse_form_ok(c->n_to, f)) continue;
      c->inv_ms[f] = time([&] { return launch_inverse_form(S->inv_att.p, *c, f, all.p, S->stream); });
      if (c->inv_ms[f] < c->inv_ms[c->inv_form]) c->inv_form = f;
    }
    for (int f = 0; f < kForms && n_fwd > 1; ++f) {
      if (!forward_form_ok(c->n_to, f, elem)) continue;
      c->fwd_ms[f] = time([&] { return launch_forward_form(fwd, *c, f, all.p, S->stream); });
      if (c->fwd_ms[f] < c->fwd_ms[c->fwd_form]) c->fwd_form = f;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CUDA_CHECK(cudaStreamSynchronize(S->stream));
}

// The column's autotuner: time both forms of the response column on this scan's own runs
// at their initial fields (one warm-up and three timed launches each, every run selected)
// and keep the faster.  The sweep has no hand-over between CTAs but one CTA walks a whole
// row, so it wins when the batch holds enough (run, node group) rows to fill the device;
// the tile-parallel form wins for a few long rows.  The stage records are a unit taper
// with zero densities while timing, then put back.
template <class R>
void tune_column(sp_scan* S, const ColumnArgsT<R>* col, const std::vector<int>& live) {
  DevBuf<int> all;
  all.upload(live.data(), live.size(), S->stream);
  std::vector<StageScalarsDev> unit(S->R);
  std::memset(unit.data(), 0, sizeof(StageScalarsDev) * unit.size());
  for (auto& u : unit) u.taper = 1.0;
  upload_all(S->stages_start, unit.data(), S->R, S->stream);
  for (auto& c : S->classes)
    if (c->n_inv) CUDA_CHECK(launch_inverse_form(S->inv_start.p, *c, c->inv_form, all.p, S->stream));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CUDA_CHECK(cudaEventCreate(&e0));
  CUDA_CHECK(cudaEventCreate(&e1));
  auto time = [&](auto&& launch) -> float {
    CUDA_CHECK(launch());
    CUDA_CHECK(cudaEventRecord(e0, S->stream));
    for (int i = 0; i < 3; ++i) CUDA_CHECK(launch());
    CUDA_CHECK(cudaEventRecord(e1, S->stream));
    CUDA_CHECK(cudaEventSynchronize(e1));
    float ms = 0;
    CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    return ms / 3;
  };
  S->column_tile_ms = time([&] { return launch_column_b(col, S->col_items.p, all.p, S->n_col_items, S->stream); });
  S->column_sweep_ms = time([&] { return launch_column_sweep_b(col, S->sweep_items.p, all.p, S->n_sweep_items, S->stream); });
  S->column_sweep = S->column_sweep_ms < S->column_tile_ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  upload_all(S->stages_start, S->h_stages_start, S->R, S->stream);
  S->norms.zero(S->stream);
  CUDA_CHECK(cudaStreamSynchronize(S->stream));
}

// The column's form: both leave every node group's partial rows for the forward transform
// to add (in group order).  A captured attempt graph holds the old launches and is dropped.
void set_column_form(sp_scan* S, bool sweep) {
  S->column_sweep = sweep;
  for (int r = 0; r < S->R; ++r) {
    S->h_fwd[r].n_groups = S->groups[r];
    S->h_fwd32[r].n_groups = S->groups[r];
  }
  upload_all(S->fwd, S->h_fwd.data(), S->R, S->stream);
  if (S->precision == SP_PRECISION_MIXED) upload_all(S->fwd32, S->h_fwd32.data(), S->R, S->stream);
  CUDA_CHECK(cudaStreamSynchronize(S->stream));
  if (S->attempt_graph) {
    CUDA_CHECK(cudaGraphExecDestroy(S->attempt_graph));
    S->attempt_graph = nullptr;
  }
}

void scan_source(sp_scan* S, bool start) {
  const int* flags = start ? S->flag_start.p : S->flag_att.p;
  if (S->precision == SP_PRECISION_MIXED)
    scan_transforms(S, flags, start ? S->inv_start.p : S->inv_att.p,
                    start ? S->col32_start.p : S->col32_att.p, S->fwd32.p);
  else
    scan_transforms(S, flags, start ? S->inv_start.p : S->inv_att.p,
                    start ? S->col_start.p : S->col_att.p, S->fwd.p);
  const DevBuf<OutputArgs>& out = start ? S->out_start : S->out_att;
  timed_family(S, SP_K_OUTPUT, [&] {
    CUDA_CHECK(launch_output_b(out.p, S->out_items.p, flags, S->n_out_items, S->stream));
  });
}

void scan_attempt_launches(sp_scan* S) {
  const int R = S->R;
  upload_all(S->flag_att, S->h_flag_att, R, S->stream);
  upload_all(S->stages_att, S->h_stages_att, 2 * (size_t)R, S->stream);
  upload_all(S->adams_att, S->h_adams_att, R, S->stream);
  timed_family(S, SP_K_PREDICT, [&] {
    CUDA_CHECK(launch_step_b(0, S->step_att.p, S->step_items.p, S->flag_att.p, S->n_step_items, R, S->stream));
  });
  scan_source(S, false);
  timed_family(S, SP_K_CORRECT, [&] {
    CUDA_CHECK(launch_step_b(1, S->step_att.p, S->step_items.p, S->flag_att.p, S->n_step_items, R, S->stream));
  });
  CUDA_CHECK(cudaMemcpyAsync(S->h_norms, S->norms.p, sizeof(double) * 8 * R, cudaMemcpyDeviceToHost,
                             S->stream));
}

constexpr int kTailRuns = 4;

// the runs' host work: on the pool while many runs are going, on this thread for a few
void for_runs(sp_scan* S, const std::function<void(int)>& body) {
  if (S->planned_active >= 16) {
    S->pool->run(S->R, body);
  } else {
    for (int r = 0; r < S->R; ++r) body(r);
  }
}

// The runs still going have halved since the last plan: their work lists only, and the
// column's and transforms' forms tuned again on them (few long rows favour the
// tile-parallel column and wider transform clusters); the next attempt recaptures its graph.
void replan(sp_scan* S) {
  std::vector<int> live(S->R);
  for (int r = 0; r < S->R; ++r) live[r] = !S->done[r] && !S->alone[r];
  CUDA_CHECK(cudaStreamSynchronize(S->stream));
  plan_items(S, live, /*first=*/false);
  if (S->precision == SP_PRECISION_MIXED) tune_column(S, S->col32_start.p, live);
  else tune_column(S, S->col_start.p, live);
  set_column_form(S, S->column_sweep);
  if (S->precision == SP_PRECISION_MIXED) tune_transforms(S, S->fwd32.p, live);
  else tune_transforms(S, S->fwd.p, live);
  if (S->attempt_graph) {
    CUDA_CHECK(cudaGraphExecDestroy(S->attempt_graph));
    S->attempt_graph = nullptr;
  }
  S->replans += 1;
}

// One batch step of the tail: every run still going takes one attempt on the single-run
// path, the runs side by side on the host pool (each on its workspace's stream).  A run
// whose step control falls below its floor stops, as in a batched step; any other failure
// propagates.
void tail_step(sp_scan* S) {
  std::vector<int> live;
  for (int r = 0; r < S->R; ++r)
    if (!S->done[r] && !S->alone[r]) live.push_back(r);
  auto body = [&](int k) {
    const int r = live[k];
    CUDA_CHECK(cudaSetDevice(S->device));
    sp_session* ss = S->ss[r].get();
    try {
      adams_adaptive_attempt(ss, ss->run.z_end);
    } catch (const Failure& f) {
      if (f.code != SP_ERR_CONVERGENCE) throw;
      ss->failed = true;
      S->done[r] = 1;
      return;
    }
    if (reached(ss->z, ss->run.z_end)) {
      ss->finished = true;
      S->done[r] = 1;
    }
  };
  if (live.size() > 1) S->pool->run((int)live.size(), body);
  else if (!live.empty()) body(0);
}

void scan_step(sp_scan* S) {
  if (S->tail) {
    tail_step(S);
    S->batch_steps += 1;
    return;
  }
  const int R = S->R;
  // phase A: runs with an empty history take their startup sample
  int n_start = 0;
  for (int r = 0; r < R; ++r) {
    S->h_flag_start[r] = 0;
    if (S->done[r] || S->alone[r]) continue;
    sp_session* ss = S->ss[r].get();
    if (!ss->history.empty()) continue;
    sp_workspace* w = S->ws[r].get();
    fill_stage(w, 2, ss->z, ss->z);
    S->h_stages_start[r] = w->h_stage[2];
    std::memset(&S->h_adams_start[r], 0, sizeof(AdamsDev));
    if (w->P->d.phi_expansion) w->P->phi_rate.eval(ss->z, S->h_adams_start[r].rate0_w);
    S->h_flag_start[r] = 1;
    ++n_start;
  }
  if (n_start) {
    upload_all(S->flag_start, S->h_flag_start, R, S->stream);
    upload_all(S->stages_start, S->h_stages_start, R, S->stream);
    upload_all(S->adams_start, S->h_adams_start, R, S->stream);
    scan_source(S, true);
    CUDA_CHECK(launch_step_b(3, S->step_start.p, S->step_items.p, S->flag_start.p, S->n_step_items, R, S->stream));
    for (int r = 0; r < R; ++r) {
      if (!S->h_flag_start[r]) continue;
      sp_session* ss = S->ss[r].get();
      ss->evaluations += 1;
      ss->history.assign(1, {ss->z, 0});
      ss->order = ss->run.variable_order ? 1 : ss->run.order;
    }
  }
  // phase B: one attempt for every unfinished run (the runs' host work on the pool)
  using clock = std::chrono::steady_clock;
  const auto t_prepare = clock::now();
  for_runs(S, [&](int r) {
    S->h_flag_att[r] = 0;
    if (S->done[r] || S->alone[r]) return;
    sp_session* ss = S->ss[r].get();
    sp_workspace* w = S->ws[r].get();
    const Next nx = adams_next(ss, ss->run.z_end);
    S->pending[r] = prepare_attempt(ss, nx.dz, nx.end, nx.kink, false);
    S->h_adams_att[r] = *w->h_adams;
    S->h_stages_att[2 * r] = w->h_stage[0];
    S->h_stages_att[2 * r + 1] = w->h_stage[1];
    S->h_flag_att[r] = 1;
  });
  int n_att = 0;
  for (int r = 0; r < R; ++r) n_att += S->h_flag_att[r];
  if (!n_att) return;
  // every operand of the attempt phase lives at a fixed address (pinned host tables, device
  // argument arrays), so its launches are captured once and replayed
  if (!S->attempt_graph && !S->graph_failed && !S->timing) {
    cudaGraph_t graph = nullptr;
    bool ok = cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      try {
        scan_attempt_launches(S);
      } catch (const Failure&) {
        ok = false;
      }
      ok = (cudaStreamEndCapture(S->stream, &graph) == cudaSuccess) && ok;
    }
    if (ok) ok = cudaGraphInstantiate(&S->attempt_graph, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {
      S->attempt_graph = nullptr;
      S->graph_failed = true;  // plain launches from here on
      cudaGetLastError();
    }
  }
  const auto t_launch = clock::now();
  if (S->attempt_graph && !S->timing) CUDA_CHECK(cudaGraphLaunch(S->attempt_graph, S->stream));
  else scan_attempt_launches(S);
  CUDA_CHECK(cudaStreamSynchronize(S->stream));
  const auto t_decide = clock::now();
  for (int r = 0; r < R; ++r)
    if (S->h_flag_att[r]) check_column(S->h_norms + 8 * r, S->norms.p + 8 * r, S->stream);
  for_runs(S, [&](int r) {
    S->h_flag_accept[r] = 0;
    if (!S->h_flag_att[r]) return;
    sp_session* ss = S->ss[r].get();
    try {
      S->h_flag_accept[r] = decide_attempt(ss, S->pending[r], S->h_norms + 8 * r) ? 1 : 0;
    } catch (const Failure&) {
      ss->failed = true;  // below dz_min: this run stops; the others go on
      S->done[r] = 1;
    }
  });
  upload_all(S->flag_accept, S->h_flag_accept, R, S->stream);
  timed_family(S, SP_K_ACCEPT, [&] {
    CUDA_CHECK(launch_step_b(2, S->step_att.p, S->step_items.p, S->flag_accept.p, S->n_step_items, R, S->stream));
  });
  const auto t_end = clock::now();
  auto ms = [](clock::time_point a, clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
  };
  S->host_prepare_ms += ms(t_prepare, t_launch);
  S->host_wait_ms += ms(t_launch, t_decide);
  S->host_decide_ms += ms(t_decide, t_end);
  for (int r = 0; r < R; ++r) {
    sp_session* ss = S->ss[r].get();
    if (!S->done[r] && !S->alone[r] && reached(ss->z, ss->run.z_end)) {
      ss->finished = true;
      S->done[r] = 1;
    }
  }
  S->batch_steps += 1;
  int active = 0;  // runs still in the batch
  for (int r = 0; r < R; ++r) active += !S->done[r] && !S->alone[r];
  if (S->R > kTailRuns && active > 0 && active <= kTailRuns) {
    // the batched launches' fixed costs outweigh their work: the last runs go on alone
    CUDA_CHECK(cudaStreamSynchronize(S->stream));
    S->tail = true;
    S->tail_from = S->batch_steps;
  } else if (active > 0 && 2 * active <= S->planned_active) {
    replan(S);
  }
}

// The runs gone on alone during one sp_scan_advance call: a host thread each, stepping its
// run on the single-run path (its workspace's stream) until the run ends or the call's
// batched steps are done.  The threads are joined before the call returns -- also when it
// throws -- and runs still going resume on fresh threads at the next call.
class LoneRuns {
 public:
  explicit LoneRuns(sp_scan* S) : S_(S) {}
  LoneRuns(const LoneRuns&) = delete;
  LoneRuns& operator=(const LoneRuns&) = delete;
  ~LoneRuns() { join(); }

  // resume the runs already alone, then let the batch's longest runs go
  void start() {
    for (int r = 0; r < S_->R; ++r)
      if (S_->alone[r] && !S_->done[r]) spawn(r);
    release_long_runs();
  }

  // the runs whose remaining attempts stand far above the batch's median leave it
  void release_long_runs() {
    if ((int)lone_.size() >= S_->alone_max) return;
    std::vector<std::pair<double, int>> rem;
    for (int r = 0; r < S_->R; ++r) {
      if (S_->done[r] || S_->alone[r]) continue;
      const sp_session* ss = S_->ss[r].get();
      if (ss->history.empty() || !(ss->proposal > 0.0)) continue;
      rem.push_back({(ss->run.z_end - ss->z) / ss->proposal, r});
    }
    if (rem.size() < 2) return;
    std::vector<double> v;
    for (auto& e : rem) v.push_back(e.first);
    std::nth_element(v.begin(), v.begin() + v.size() / 2, v.end());
    const double median = v[v.size() / 2];
    std::sort(rem.begin(), rem.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    bool synced = false;
    for (auto& e : rem) {
      if ((int)lone_.size() >= S_->alone_max) break;
      if (!(e.first > S_->alone_min && e.first > S_->alone_factor * median)) break;
      if (!synced) {  // the batch's last launches may still touch the run's buffers
        CUDA_CHECK(cudaStreamSynchronize(S_->stream));
        synced = true;
      }
      S_->alone[e.second] = 1;
      S_->alone_count += 1;
      spawn(e.second);
    }
  }

  bool any_running() const {
    for (auto& l : lone_)
      if (l->state.load() == 0) return true;
    return false;
  }

  // with no batch left: until every run alone has ended or taken `steps` more attempts
  void wait(int steps) {
    std::vector<long long> from;
    for (auto& l : lone_) from.push_back(l->attempts.load());
    for (;;) {
      bool waiting = false;
      for (size_t k = 0; k < lone_.size(); ++k)
        waiting |= lone_[k]->state.load() == 0 && lone_[k]->attempts.load() - from[k] < steps;
      if (!waiting) return;
      std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
  }

  // stop and join the threads; ended runs leave the scan, and a thread's unexpected
  // failure is rethrown here
  void join() {
    stop_.store(true);
    std::exception_ptr error;
    for (auto& l : lone_) {
      if (l->thread.joinable()) l->thread.join();
      if (l->state.load() == 1 || l->state.load() == 2) S_->done[l->run] = 1;
      if (l->state.load() == 3 && !error) error = l->error;
    }
    lone_.clear();
    if (error && !std::uncaught_exceptions()) std::rethrow_exception(error);
  }

 private:
  struct Lone {
    int run = 0;
    std::thread thread;
    std::atomic<int> state{0};  // 0 going, 1 finished, 2 failed (step floor), 3 error
    std::atomic<long long> attempts{0};
    std::exception_ptr error;
  };

  void spawn(int r) {
    auto l = std::make_unique<Lone>();
    l->run = r;
    Lone* me = l.get();
    me->thread = std::thread([this, me] {
      sp_session* ss = S_->ss[me->run].get();
      try {
        CUDA_CHECK(cudaSetDevice(S_->device));
        while (!stop_.load()) {
          try {
            adams_adaptive_attempt(ss, ss->run.z_end);
          } catch (const Failure& f) {
            if (f.code != SP_ERR_CONVERGENCE) throw;
            ss->failed = true;
            me->state.store(2);
            return;
          }
          me->attempts.fetch_add(1);
          if (reached(ss->z, ss->run.z_end)) {
            ss->finished = true;
            me->state.store(1);
            return;
          }
        }
      } catch (...) {
        me->error = std::current_exception();
        me->state.store(3);
      }
    });
    lone_.push_back(std::move(l));
  }

  sp_scan* S_;
  std::atomic<bool> stop_{false};
  std::vector<std::unique_ptr<Lone>> lone_;
};

}  // namespace

extern "C" {

sp_status sp_scan_create(int32_t n_runs, const sp_problem* const* problems, const sp_run_desc* runs,
                         int device, sp_scan** out) {
  return sp_scan_create_ex(n_runs, problems, runs, device, SP_PRECISION_FP64, out);
}

sp_status sp_scan_create_ex(int32_t n_runs, const sp_problem* const* problems, const sp_run_desc* runs,
                            int device, int precision, sp_scan** out) {
  return guarded([&] {
    if (n_runs < 1 || !problems || !runs || !out) throw Failure(SP_ERR_ARGUMENT, "bad scan arguments");
    if (precision != SP_PRECISION_FP64 && precision != SP_PRECISION_MIXED)
      throw Failure(SP_ERR_ARGUMENT, "unknown precision");
    for (int r = 0; r < n_runs; ++r) {
      if (problems[r] && (problems[r]->n_cols > kMaxModes ||
                          (problems[r]->d.raman_enabled && problems[r]->d.grid_kind == 0)))
        throw Failure(SP_ERR_REFUSED,
                      "a scan's runs take at most 8 modal columns and no field-grid Raman (the fused transform)");
      if (problems[r] && !problems[r]->channels.empty())
        throw Failure(SP_ERR_REFUSED, "a scan's runs take one plasma channel (no gas mixture)");
    }
    CUDA_CHECK(cudaSetDevice(device));
    ensure_configured(device);
    auto S = std::make_unique<sp_scan>();
    S->device = device;
    S->precision = precision;
    S->R = n_runs;
    CUDA_CHECK(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
    const int R = n_runs;
    for (int r = 0; r < R; ++r) {
      if (runs[r].method != 0 || runs[r].schedule)
        throw Failure(SP_ERR_REFUSED, "a scan steps adaptive exponential-Adams runs only");
      if (problems[r]->d.phi_expansion)
        throw Failure(SP_ERR_REFUSED, "a scan run with a varying operator (Phi expansion)");
      if (problems[r]->d.grid_kind != 0)
        throw Failure(SP_ERR_REFUSED, "a scan run on the envelope grid");
      auto w = std::make_unique<sp_workspace>();
      w->P = problems[r];
      w->device = device;
      w->precision = precision;
      CUDA_CHECK(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking));
      build_workspace(w.get());
      sp_session* raw = nullptr;
      sp_status st = sp_session_start(w.get(), &runs[r], &raw);
      if (st != SP_OK) throw Failure(st, g_error);
      raw->defer_accept = false;  // the scan reads its runs' states between attempts
      S->ss.emplace_back(raw);
      S->ws.push_back(std::move(w));
    }
    S->done.assign(R, 0);
    S->alone.assign(R, 0);
    S->pending.resize(R);
    {
      // up to eight host threads when the batch is large enough to pay for the hand-off
      const int cores = (int)std::thread::hardware_concurrency();
      const int workers = R >= 16 ? std::max(0, std::min(cores, 8) - 1) : 0;
      S->pool = std::make_unique<HostPool>(workers);
    }
    S->h_adams_start = pinned<AdamsDev>(R);
    S->h_adams_att = pinned<AdamsDev>(R);
    S->h_stages_start = pinned<StageScalarsDev>(R);
    S->h_stages_att = pinned<StageScalarsDev>(2 * (size_t)R);
    S->h_norms = pinned<double>(8 * (size_t)R);
    S->h_flag_start = pinned<int>(R);
    S->h_flag_att = pinned<int>(R);
    S->h_flag_accept = pinned<int>(R);
    S->adams_start.alloc(R);
    S->adams_att.alloc(R);
    S->stages_start.alloc(R);
    S->stages_att.alloc(2 * (size_t)R);
    S->norms.alloc(8 * (size_t)R);
    S->norms.zero(S->stream);
    S->flag_start.alloc(R);
    S->flag_att.alloc(R);
    S->flag_accept.alloc(R);
    // per-run argument records and the static work tables
    std::vector<InverseArgs> is(R), ia(R);
    std::vector<ColumnTileArgs> cs(R), ca(R);
    std::vector<ForwardArgs> fa(R);
      std::vector<ColumnArgsT<float>> cs32(R), ca32(R);
    std::vector<ForwardArgsT<float>> fa32(R);
    std::vector<OutputArgs> os(R), oa(R);
    std::vector<StepArgs> ts(R), ta(R);
    std::vector<int> sizes;
    S->work.resize(R);
    for (int r = 0; r < R; ++r) {
      sp_workspace* w = S->ws[r].get();
      const sp_problem& P = *w->P;
      const bool absorber = P.d.absorber_in_stage != 0;
      is[r] = inverse_args(w, w->state.p, absorber);
      ia[r] = inverse_args(w, w->lab.p, absorber);
      cs[r] = column_args(w, S->stages_start.p + r);
      ca[r] = column_args(w, S->stages_att.p + 2 * r + 1);
      cs[r].status = ca[r].status = S->norms.p + 8 * r + kColumnStatus;
      fa[r] = forward_args(w);
      if (precision == SP_PRECISION_MIXED) {
        cs32[r] = column_args<float>(w, S->stages_start.p + r);
        ca32[r] = column_args<float>(w, S->stages_att.p + 2 * r + 1);
        cs32[r].status = ca32[r].status = S->norms.p + 8 * r + kColumnStatus;
        fa32[r] = forward_args<float>(w);
      }
      os[r] = output_args(w, S->stages_start.p + r, nullptr, w->src.p, absorber);
      oa[r] = output_args(w, S->stages_att.p + 2 * r + 1, nullptr, w->src.p, absorber);
      const int nb = std::min(kNormBlocks, (P.n + 255) / 256);
      ts[r] = step_args_of(w, S->adams_start.p + r, S->stages_start.p + r);
      ta[r] = step_args_of(w, S->adams_att.p + r, S->stages_att.p + 2 * r);
      ts[r].n_blocks = ta[r].n_blocks = nb;
      ts[r].norms = ta[r].norms = S->norms.p + 8 * r;
      S->work[r] = {P.d.n_to, nb, (P.n + 255) / 256, cs[r].n_blocks, cs[r].n_groups, cs[r].n_tiles,
                    P.n_cols, forward_rows(w, absorber)};
      if (std::find(sizes.begin(), sizes.end(), P.d.n_to) == sizes.end()) sizes.push_back(P.d.n_to);
    }
    std::sort(sizes.begin(), sizes.end());
    for (int n_to : sizes) {
      auto c = std::make_unique<FftClass>();
      c->n_to = n_to;
      // Until the autotuner (tune_transforms) has timed the forms, a row takes the first
      // that holds it: one CTA, else the narrowest cluster.  (The inverse transform is FP64
      // in both precisions.)
      const size_t elem = precision == SP_PRECISION_MIXED ? 8 : 16;
      while (c->inv_form + 1 < kForms && !inverse_form_ok(n_to, c->inv_form)) ++c->inv_form;
      while (c->fwd_form + 1 < kForms && !forward_form_ok(n_to, c->fwd_form, elem)) ++c->fwd_form;
      S->classes.push_back(std::move(c));
    }
    S->inv_start.upload(is.data(), R, S->stream);
    S->inv_att.upload(ia.data(), R, S->stream);
    S->col_start.upload(cs.data(), R, S->stream);
    S->col_att.upload(ca.data(), R, S->stream);
    S->fwd.upload(fa.data(), R, S->stream);
    if (precision == SP_PRECISION_MIXED) {
      S->col32_start.upload(cs32.data(), R, S->stream);
      S->col32_att.upload(ca32.data(), R, S->stream);
      S->fwd32.upload(fa32.data(), R, S->stream);
    }
    S->out_start.upload(os.data(), R, S->stream);
    S->out_att.upload(oa.data(), R, S->stream);
    S->step_start.upload(ts.data(), R, S->stream);
    S->step_att.upload(ta.data(), R, S->stream);
    const std::vector<int> all(R, 1);
    plan_items(S.get(), all, /*first=*/true);
    CUDA_CHECK(cudaDeviceSynchronize());  // the sessions' initial fields are in place
    if (precision == SP_PRECISION_MIXED) tune_column(S.get(), S->col32_start.p, all);
    else tune_column(S.get(), S->col_start.p, all);
    S->h_fwd = fa;
    S->h_fwd32 = fa32;
    for (int r = 0; r < R; ++r) S->groups.push_back(cs[r].n_groups);
    set_column_form(S.get(), S->column_sweep);
    if (precision == SP_PRECISION_MIXED) tune_transforms(S.get(), S->fwd32.p, all);
    else tune_transforms(S.get(), S->fwd.p, all);
    *out = S.release();
  });
}

sp_status sp_scan_advance(sp_scan* S, int32_t steps, sp_scan_status* out) {
  return guarded([&] {
    if (!S || !out) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    CUDA_CHECK(cudaSetDevice(S->device));
    auto batched = [&] {
      for (int r = 0; r < S->R; ++r)
        if (!S->done[r] && !S->alone[r]) return true;
      return false;
    };
    {
      LoneRuns lone(S);
      if (S->alone_max > 0 && steps > 0) lone.start();
      int i = 0;
      for (; i < steps && batched(); ++i) {
        scan_step(S);
        if (S->alone_max > 0 && (i + 1) % 128 == 0) lone.release_long_runs();
      }
      if (i < steps && lone.any_running()) lone.wait(steps - i);
      lone.join();
    }
    out->active = 0;
    out->attempts = out->rejected = out->evaluations = 0;
    for (int r = 0; r < S->R; ++r) {
      out->active += !S->done[r];
      out->attempts += S->ss[r]->attempts;
      out->rejected += S->ss[r]->rejected;
      out->evaluations += S->ss[r]->evaluations;
    }
    out->batch_steps = S->batch_steps;
  });
}

sp_status sp_scan_run(sp_scan* S, int32_t run, double* state, sp_batch* info) {
  return guarded([&] {
    if (!S || run < 0 || run >= S->R) throw Failure(SP_ERR_ARGUMENT, "run index out of range");
    CUDA_CHECK(cudaSetDevice(S->device));
    CUDA_CHECK(cudaStreamSynchronize(S->stream));
    CUDA_CHECK(cudaStreamSynchronize(S->ws[run]->stream));  // a run that went on alone
    sp_session* ss = S->ss[run].get();
    if (state) {
      const size_t bytes = (size_t)S->ws[run]->P->n * sizeof(double2);
      CUDA_CHECK(cudaMemcpy(state, S->ws[run]->state.p, bytes, cudaMemcpyDeviceToHost));
    }
    if (info) {
      info->event = ss->failed ? 3 : (ss->finished ? 2 : 0);
      info->plane_index = -1;
      info->z = ss->z;
      info->attempts = ss->attempts;
      info->rejected = ss->rejected;
      info->evaluations = ss->evaluations;
      info->reason = ss->failed ? SP_REASON_ERROR : ss->finished ? SP_REASON_REACHED : SP_REASON_BOUND;
      info->category = ss->failed ? SP_CATEGORY_BACKEND : SP_CATEGORY_NONE;
      info->n_rows = 0;
    }
  });
}

void* sp_scan_stream(sp_scan* S) { return S ? (void*)S->stream : nullptr; }

sp_status sp_scan_statistics(sp_scan* S, int32_t run, const double* power_weight, sp_statistics* out) {
  return guarded([&] {
    if (!S || run < 0 || run >= S->R || !out) throw Failure(SP_ERR_ARGUMENT, "bad scan statistics arguments");
    CUDA_CHECK(cudaSetDevice(S->device));
    CUDA_CHECK(cudaStreamSynchronize(S->stream));  // the run's last batched launches
    plane_statistics(S->ws[run].get(), power_weight, out);
  });
}

sp_status sp_scan_set_timing(sp_scan* S, int enable) {
  return guarded([&] {
    if (!S) throw Failure(SP_ERR_ARGUMENT, "NULL scan");
    CUDA_CHECK(cudaSetDevice(S->device));
    flush_scan_timing(S);
    S->timing = enable != 0;
  });
}

sp_status sp_scan_timing(sp_scan* S, double* ms, int64_t* launches, int reset) {
  return guarded([&] {
    if (!S || !ms || !launches) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    CUDA_CHECK(cudaSetDevice(S->device));
    flush_scan_timing(S);
    for (int k = 0; k < SP_K_COUNT; ++k) {
      ms[k] = S->t_ms[k];
      launches[k] = S->t_count[k];
    }
    if (reset) {
      std::fill(S->t_ms, S->t_ms + SP_K_COUNT, 0.0);
      std::fill(S->t_count, S->t_count + SP_K_COUNT, int64_t(0));
    }
  });
}

size_t sp_scan_describe(const sp_scan* S, char* buf, size_t len) {
  std::string text;
  if (S) {
    text += S->attempt_graph ? "attempt phase: one CUDA graph\n"
                             : (S->graph_failed ? "attempt phase: plain launches (capture failed)\n"
                                                : "attempt phase: not yet captured\n");
    char line[512];
    std::snprintf(line, sizeof line, "column: %s (tile-parallel %.4f ms, sweep %.4f ms)\n",
                  S->column_sweep ? "sweep" : "tile-parallel", S->column_tile_ms, S->column_sweep_ms);
    text += line;
    std::snprintf(line, sizeof line,
                  "work lists: planned for %d running runs, re-planned %d times; the last %d runs "
                  "alone from batch step %lld; %d long runs went on alone\n",
                  S->planned_active, S->replans, kTailRuns, (long long)S->tail_from, S->alone_count);
    text += line;
    const double steps = (double)std::max<int64_t>(S->batch_steps, 1);
    std::snprintf(line, sizeof line,
                  "host per batch step: prepare %.4f ms, attempt phase (launch to its end) %.4f ms, "
                  "decide %.4f ms, on %d threads\n",
                  S->host_prepare_ms / steps, S->host_wait_ms / steps, S->host_decide_ms / steps,
                  S->pool ? S->pool->threads() : 1);
    text += line;
    auto form = [](int f) -> std::string {
      return kFormWidth[f] ? "cluster" + std::to_string(kFormWidth[f]) : std::string("single");
    };
    for (const auto& c : S->classes) {
      std::snprintf(line, sizeof line,
                    "n_to %d: inverse %s (single %.4f, cluster2 %.4f, cluster4 %.4f, cluster8 %.4f ms), "
                    "forward %s (single %.4f, cluster2 %.4f, cluster4 %.4f, cluster8 %.4f ms)\n",
                    c->n_to, form(c->inv_form).c_str(), c->inv_ms[0], c->inv_ms[1], c->inv_ms[2],
                    c->inv_ms[3], form(c->fwd_form).c_str(), c->fwd_ms[0], c->fwd_ms[1], c->fwd_ms[2],
                    c->fwd_ms[3]);
      text += line;
    }
  }
  if (buf && len) {
    const size_t n = std::min(len - 1, text.size());
    std::memcpy(buf, text.data(), n);
    buf[n] = 0;
  }
  return text.size();
}

sp_status sp_scan_set_column(sp_scan* S, int32_t form) {
  return guarded([&] {
    if (!S) throw Failure(SP_ERR_ARGUMENT, "NULL scan");
    if (form != SP_SCAN_COLUMN_TILES && form != SP_SCAN_COLUMN_SWEEP)
      throw Failure(SP_ERR_ARGUMENT, "unknown column form");
    CUDA_CHECK(cudaSetDevice(S->device));
    CUDA_CHECK(cudaStreamSynchronize(S->stream));
    set_column_form(S, form == SP_SCAN_COLUMN_SWEEP);
  });
}

sp_status sp_scan_set_alone(sp_scan* S, int32_t max_runs, double min_remaining, double factor) {
  return guarded([&] {
    if (!S) throw Failure(SP_ERR_ARGUMENT, "NULL scan");
    if (max_runs < 0 || !(min_remaining >= 0.0) || !(factor >= 1.0))
      throw Failure(SP_ERR_ARGUMENT, "alone: max_runs >= 0, min_remaining >= 0, factor >= 1");
    S->alone_max = max_runs;
    S->alone_min = min_remaining;
    S->alone_factor = factor;
  });
}

sp_status sp_scan_set_transforms(sp_scan* S, int32_t n_to, int32_t inverse_cluster,
                                 int32_t forward_cluster) {
  return guarded([&] {
    if (!S) throw Failure(SP_ERR_ARGUMENT, "NULL scan");
    auto form_of = [](int32_t width) {
      for (int f = 0; f < kForms; ++f)
        if (kFormWidth[f] == width) return f;
      throw Failure(SP_ERR_ARGUMENT, "a transform's cluster width is 0 (one CTA), 2, 4 or 8");
    };
    const int fi = form_of(inverse_cluster), ff = form_of(forward_cluster);
    const size_t elem = S->precision == SP_PRECISION_MIXED ? 8 : 16;
    for (auto& c : S->classes) {
      if (c->n_to != n_to) continue;
      if (!inverse_form_ok(n_to, fi) || !forward_form_ok(n_to, ff, elem))
        throw Failure(SP_ERR_ARGUMENT, "that transform form does not hold this grid's rows");
      CUDA_CHECK(cudaSetDevice(S->device));
      CUDA_CHECK(cudaStreamSynchronize(S->stream));
      c->inv_form = fi;
      c->fwd_form = ff;
      if (S->attempt_graph) {
        CUDA_CHECK(cudaGraphExecDestroy(S->attempt_graph));
        S->attempt_graph = nullptr;
      }
      return;
    }
    throw Failure(SP_ERR_ARGUMENT, "no run of the scan has that grid size");
  });
}

sp_status sp_scan_destroy(sp_scan* S) {
  delete S;
  return SP_OK;
}

}  // extern "C"

// ====================================================================== no-allocation entry
// sp_source_noalloc: one source evaluation for callers that cannot allocate device
// memory.  Every device buffer it needs -- the problem's tables and the evaluation's
// intermediates -- is carved out of one file-scope array of kNoAllocBytes, which each
// device that loads this library holds until the process exits.
#include <mutex>

namespace {

constexpr size_t kNoAllocBytes = size_t(40) << 20;  // 40 MiB
constexpr int kNoAllocDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_base[kNoAllocDevices];       // device address, per device
StageScalarsDev g_noalloc_stage[kNoAllocDevices][sp_workspace::kStageSlots];

// Bump allocation over the array, 256-byte aligned; throws when the problem does not fit.
struct Carver {
  unsigned char* base;
  size_t used = 0;
  template <class T>
  void take(DevBuf<T>& buf, size_t count) {
    const size_t bytes = ((count * sizeof(T)) + 255) & ~size_t(255);
    if (used + bytes > kNoAllocBytes) {
      char msg[200];
      std::snprintf(msg, sizeof msg,
                    "the problem needs more than the %zu MiB the no-allocation entry point holds",
                    kNoAllocBytes >> 20);
      throw Failure(SP_ERR_ARGUMENT, msg);
    }
    buf.p = reinterpret_cast<T*>(base + used);
    buf.n = count;
    buf.owned = false;
    used += bytes;
  }
};

unsigned char* noalloc_base(int device) {
  if (device < 0 || device >= kNoAllocDevices) throw Failure(SP_ERR_ARGUMENT, "device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_base[device]) {
    // With the device current, resolve the array's device address once; host code
    // cannot use the symbol's name as a device pointer.
    void* ptr = nullptr;
    CUDA_CHECK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    g_noalloc_base[device] = static_cast<unsigned char*>(ptr);
  }
  return g_noalloc_base[device];
}

template <class T>
void put(DevBuf<T>& buf, const void* host, size_t count, cudaStream_t s) {
  if (count) CUDA_CHECK(cudaMemcpyAsync(buf.p, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
}

}  // namespace

extern "C" sp_status sp_source_noalloc(const sp_problem* problem, const void* lab, double z,
                                       int quiet, void* out, void* stream_handle) {
  return guarded([&] {
    if (!problem || !lab || !out) throw Failure(SP_ERR_ARGUMENT, "NULL argument");
    if (problem->d.grid_kind != 0)
      throw Failure(SP_ERR_REFUSED, "the no-allocation entry point takes field-grid problems");
    if (problem->n_cols > kMaxModes || (problem->d.raman_enabled && problem->d.grid_kind == 0))
      throw Failure(SP_ERR_REFUSED,
                    "the no-allocation entry point takes at most 8 modal columns and no field-grid Raman");
    if (!problem->channels.empty())
      throw Failure(SP_ERR_REFUSED, "the no-allocation entry point takes one plasma channel (no gas mixture)");
    int device = 0;
    CUDA_CHECK(cudaGetDevice(&device));
    unsigned char* base = noalloc_base(device);
    cudaStream_t s = static_cast<cudaStream_t>(stream_handle);
    const sp_problem& P = *problem;
    const sp_problem_desc& d = P.d;
    static std::mutex call_mutex;
    std::lock_guard<std::mutex> lock(call_mutex);
    // A view of the workspace whose buffers are regions of the array; it owns nothing.
    static sp_workspace views[kNoAllocDevices];
    sp_workspace& ws = views[device];
    ws.borrowed = true;
    // the caller's stream and the static host scalars are lent for this call only, on
    // every way out of it (a refusal or a failed upload included)
    auto release = on_scope_exit([&ws] {
      ws.stream = nullptr;
      ws.h_stage = nullptr;
      ws.P = nullptr;
    });
    ws.P = problem;
    ws.device = device;
    ws.stream = s;
    ws.h_stage = g_noalloc_stage[device];
    ws.log_m = ilog2(d.n_to / 2);
    ws.log_n_to = ilog2(d.n_to);
    ws.launches = 5;
    Carver carve{base};
    const size_t n = P.n;
    carve.take(ws.phi_terms, (size_t)d.n_phi_terms * n);
    carve.take(ws.pre_terms, (size_t)d.n_prefactor_terms * n);
    carve.take(ws.twiddles, (size_t)d.n_to / 2);
    carve.take(ws.omega, d.n_omega);
    carve.take(ws.omega_window, d.n_omega);
    carve.take(ws.t_window, d.n_to);
    carve.take(ws.t_window_d, d.n_to);
    carve.take(ws.alpha, d.n_to);
    carve.take(ws.synthesis, P.synthesis.size());
    carve.take(ws.projection, P.projection.size());
    carve.take(ws.rate_coeff, std::max<size_t>(P.rate_coeff.size(), 4));
    carve.take(ws.taps, std::max<size_t>(P.taps.size(), 1));
    carve.take(ws.crop, d.n_omega);
    carve.take(ws.fine_to_coarse, (size_t)d.n_to / 2 + 1);
    carve.take(ws.rows, (size_t)6 * P.n_cols);
    carve.take(ws.active, d.n_omega);
    carve.take(ws.norm, d.n_omega);
    carve.take(ws.modal_t, (size_t)P.n_cols * d.n_to);
    const size_t n_tiles = column_tiles(d);
    const size_t n_groups = (d.n_nodes + kGroup - 1) / kGroup;
    carve.take(ws.sums0, (size_t)d.n_nodes * n_tiles);
    carve.take(ws.sums1, (size_t)d.n_nodes * n_tiles);
    carve.take(ws.chain_flags, n_groups * n_tiles);
    carve.take(ws.ticket, 1);
    carve.take(ws.norms, kMaxOrders + 2);
    carve.take(ws.proj, n_groups * 3 * P.n_cols * d.n_to);
    carve.take(ws.streams, (size_t)4 * P.n_cols * d.n_to);
    carve.take(ws.spectra, (size_t)4 * n);
    carve.take(ws.stage, sp_workspace::kStageSlots);
    // the problem's tables, every call: the array keeps the last call's contents, which
    // may be another problem's
    put(ws.phi_terms, P.phi_terms.data(), (size_t)d.n_phi_terms * n, s);
    put(ws.pre_terms, P.pre_terms.data(), (size_t)d.n_prefactor_terms * n, s);
    std::vector<double2> tw(d.n_to / 2);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int m = 0; m < d.n_to / 2; ++m) {
      long double ang = two_pi * (long double)m / (long double)d.n_to;
      tw[m] = make_double2((double)cosl(ang), (double)(-sinl(ang)));
    }
    put(ws.twiddles, tw.data(), tw.size(), s);
    put(ws.omega, P.omega.data(), d.n_omega, s);
    put(ws.omega_window, P.omega_window.data(), d.n_omega, s);
    put(ws.t_window, P.t_window.data(), d.n_to, s);
    put(ws.t_window_d, P.t_window_d.data(), d.n_to, s);
    std::vector<double> alpha(d.n_to, 0.0);
    if (d.absorber_in_stage) alpha = P.alpha;
    put(ws.alpha, alpha.data(), d.n_to, s);
    put(ws.synthesis, P.synthesis.data(), P.synthesis.size(), s);
    put(ws.projection, P.projection.data(), P.projection.size(), s);
    std::vector<double> rc = P.rate_coeff.empty() ? std::vector<double>(4, 0.0) : P.rate_coeff;
    put(ws.rate_coeff, rc.data(), rc.size(), s);
    std::vector<double> taps = P.taps.empty() ? std::vector<double>(1, 1.0) : P.taps;
    put(ws.taps, taps.data(), taps.size(), s);
    put(ws.crop, P.crop.data(), d.n_omega, s);
    std::vector<int> f2c(d.n_to / 2 + 1, -1);  // field grid only (checked above)
    for (int j = 0; j < d.n_omega; ++j) f2c.at(P.crop[j]) = j;
    put(ws.fine_to_coarse, f2c.data(), f2c.size(), s);
    std::vector<int> rows;
    for (int r = 0; r < 4 * P.n_cols; ++r) rows.push_back(r);
    for (int r = 0; r < P.n_cols; ++r) rows.push_back(r);
    for (int r = 0; r < P.n_cols; ++r) rows.push_back(3 * P.n_cols + r);
    put(ws.rows, rows.data(), rows.size(), s);
    put(ws.active, P.active.data(), d.n_omega, s);
    put(ws.norm, P.norm.data(), d.n_omega, s);
    // the buffers the allocating workspace starts at zero
    ws.streams.zero(s);
    ws.spectra.zero(s);
    ws.proj.zero(s);
    ws.chain_flags.zero(s);
    ws.ticket.zero(s);
    ws.norms.zero(s);
    ensure_configured(device);
    fill_stage(&ws, 0, z, z);
    upload_stages(&ws, 1);
    eval_source(&ws, static_cast<const double2*>(lab), 0, nullptr, static_cast<double2*>(out),
                quiet != 0);
    // the response column marks its status slot when a tile gave up waiting: read it with
    // the result (the host copies above also read pageable buffers of this call)
    double status[kColumnStatus + 1] = {};
    CUDA_CHECK(cudaMemcpyAsync(&status[kColumnStatus], ws.norms.p + kColumnStatus, sizeof(double),
                               cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    check_column(status, ws.norms.p, s);
  });
}
