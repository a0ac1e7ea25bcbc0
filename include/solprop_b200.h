/*
 * solprop_b200.h -- the C ABI of the B200 propagation library.
 *
 * The library executes solprop's propagation hot path: the UPPE/GNLSE right-hand side
 * (one "source evaluation") and its exponential-Adams and embedded Runge-Kutta
 * steppers, in FP64, on one CUDA device.  Every entry point takes plain pointers and
 * sizes; complex arrays are interleaved (re, im) doubles in C order, exactly the
 * memory of NumPy's complex128.  Every function returns an sp_status; the message of
 * the last failure on the calling thread is read with sp_last_error().
 *
 * Each entry point names the interface of the reference (LupoLab/solprop, paths inside
 * that repository) whose role it takes:
 *   problem   <- native/src/solprop_native/_core.pyi:51-428       (_core.Problem)
 *   workspace <- native/src/solprop_native/_core.pyi:600-612      (_core.Workspace)
 *   session   <- native/src/solprop_native/_core.pyi:430-470      (_core.Session)
 *   source    <- src/solprop/backends/numpy_ref/workspace.py:819 (lab_source), the
 *                native trial's source evaluation (native/src/general/trial.cpp:697)
 */
#ifndef SOLPROP_B200_H
#define SOLPROP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int sp_status;
enum {
  SP_OK = 0,
  SP_ERR_ARGUMENT = 1,   /* a pointer, size or value the call cannot take */
  SP_ERR_REFUSED = 2,    /* a problem this backend does not execute (BackendRefusal) */
  SP_ERR_CUDA = 3,       /* a CUDA runtime failure; the message names the call */
  SP_ERR_STATE = 4,      /* a lifecycle error: closed object, run not started */
  SP_ERR_CONVERGENCE = 5 /* step control fell below dz_min, or the field diverged */
};

/* Precision of a workspace's source evaluations.  FP64 is the plain form, the reference's
 * arithmetic.  MIXED evaluates the transforms and the response column (synthesis, rate,
 * fraction, currents, Kerr, projection) in FP32; the state, the propagator phase and its
 * exponentials, the Adams history and accumulation, the stage output, the error norms and
 * the plasma running integrals (compensated: FP32 increments summed in FP64) stay FP64.
 * It has no counterpart in the reference. */
enum { SP_PRECISION_FP64 = 0, SP_PRECISION_MIXED = 1 };

/* A piecewise Chebyshev series in z (solprop translate/chebyshev.py:236): interval i
 * holds n_deg coefficients of n_values values, c[(i*n_deg + j)*n_values + v].
 * n_intervals == 0 means "absent". */
typedef struct sp_table {
  int32_t n_intervals, n_deg, n_values;
  const double* breakpoints;  /* n_intervals + 1 */
  const double* coefficients; /* n_intervals * n_deg * n_values */
} sp_table;

/* A further field-plasma channel of a gas mixture (passes/plasma.py:326-485): its own rate
 * table, exposure scan and population; channel 0 is the descriptor's own plasma fields. */
typedef struct sp_plasma_channel {
  double charge_mass_ratio, ionisation_potential; /* ratio x electrons per event */
  int32_t rate_intervals;
  const double* rate_coefficients; /* (4, rate_intervals) */
  double log_field_min, d_log_field, field_min, field_max, rate_max;
  sp_table plasma_density, preionisation;
} sp_plasma_channel;

/* A further Raman-active component of a gas mixture (passes/responses.py:293-334,
 * mixture_raman_spectrum): its rows damped at their own rates, weighted by its fraction and
 * density; component 0 is the descriptor's own Raman fields. */
typedef struct sp_raman_component {
  int32_t terms;
  const double* undamped; /* (terms, 2*n_to) */
  sp_table rates[4];
  double fraction;
  sp_table density;
  const double* tensor_weights; /* (terms, 2): trace, traceless; two field components only */
} sp_raman_component;

/* The lowered problem (solprop_b200.record.ProblemRecord; kernel-contract.md 1-6). */
typedef struct sp_problem_desc {
  int32_t grid_kind; /* 0 field (r2c/c2r), 1 envelope (c2c) */
  int32_t n_modes, n_pol, n_omega, n_t, n_to, n_nodes, n_pol_transform;
  double omega0, dt, dt_fine, z_end;
  const double* omega;               /* n_omega */
  const int64_t* crop_index;         /* n_omega: position in the fine spectrum */
  const uint8_t* active_mask;        /* n_omega */
  const uint8_t* norm_mask;          /* n_omega */
  const double* omega_window;        /* n_omega */
  const double* t_window;            /* n_to */
  const double* t_window_derivative; /* n_to */
  const double* carrier;             /* complex n_to, or NULL */
  /* Phi = sum_j w_j(z) phi_terms[j]; constant: one term, weight z1 - z0. */
  int32_t phi_expansion;
  int32_t n_phi_terms;
  const double* phi_terms; /* complex (n_phi_terms, n_modes, n_pol, n_omega) */
  sp_table phi_weights;    /* expansion: Phi(z) weights, n_values = n_phi_terms */
  sp_table phi_rate;       /* expansion: dPhi/dz weights */
  int32_t n_prefactor_terms;
  const double* prefactor_terms; /* complex (n_prefactor_terms, n_modes, n_pol, n_omega) */
  sp_table prefactor_weights;    /* absent: the one constant term, weight 1 */
  sp_table density, kerr_density, plasma_density, preionisation, taper_scale;
  const double* synthesis;  /* (n_nodes*n_pol_transform, n_modes), pad scale inside */
  const double* projection; /* (n_modes, n_nodes*n_pol_transform), weights inside */
  /* Kerr (translate/responses.py:235-275) */
  int32_t kerr_enabled, kerr_analytic; /* analytic: 1 for the envelope cubic form */
  double kerr_coefficient, kerr_self, kerr_conjugate, kerr_harmonic;
  int32_t kerr_take_real;
  /* field plasma, one channel (translate/ionisation.py:95-323) */
  int32_t plasma_enabled;
  double charge_mass_ratio, ionisation_potential;
  int32_t rate_intervals;
  const double* rate_coefficients; /* (4, rate_intervals) */
  double log_field_min, d_log_field, field_min, field_max, rate_max;
  int32_t band; /* 1: band rule with taps and the exposure floor; 0: trapezoid */
  int32_t n_taps;
  const double* taps; /* centre first */
  /* Raman, scalar (translate/raman.py; kernel-contract.md 5) */
  int32_t raman_enabled, raman_terms, raman_thg;
  const double* raman_undamped; /* (raman_terms, 2*n_to) */
  sp_table raman_rates[4];
  double raman_fraction;
  sp_table raman_density;
  /* the in-stage temporal absorber (stepping.py:286-369) */
  int32_t absorber_in_stage;
  const double* temporal_absorber_fine; /* n_to */
  /* a gas mixture: plasma channels and Raman components after the first (up to 3 each;
   * zero-initialised: none) */
  int32_t n_extra_channels;
  const sp_plasma_channel* extra_channels;
  int32_t n_extra_raman;
  const sp_raman_component* extra_raman;
  /* two Cartesian field components (n_pol_transform 2, envelope grid): the Raman rows'
   * trace and traceless weights, (raman_terms, 2) (passes/responses.py:337-392) */
  const double* raman_tensor_weights;
} sp_problem_desc;

typedef struct sp_problem sp_problem;
typedef struct sp_workspace sp_workspace;
typedef struct sp_session sp_session;

/* A run: the march's policy (backends adams_core MarchPolicy / RungeKuttaPolicy). */
typedef struct sp_run_desc {
  int32_t method;          /* 0 exponential Adams, 1 DOPRI5 */
  const double* field0;    /* complex (n_modes, n_pol, n_omega) */
  double z_start, proposal, rtol, atol;
  double dz_min, dz_max, stretch, z_end;
  const double* save_planes; int32_t n_save_planes;
  const double* hard_kinks; int32_t n_hard_kinks;
  const double* breakpoints; int32_t n_breakpoints;
  const double* schedule; int32_t n_schedule; /* fixed steps, or NULL for adaptive */
  /* Adams */
  int32_t order, variable_order, restart_after, equal_approach;
  double safety, max_growth, min_factor, rejection_growth, hysteresis;
  double collar_stability, collar_rate;
  double real_intervals[8];
  /* Runge-Kutta PI controller */
  double beta1, beta2, max_factor;
  int32_t lag, estimator_order;
  /* Runge-Kutta start-up (rk_core.py:67-107): after the first accepted step, the deadbeat
   * proposal its norm implies, at most start_growth times the first (0: off) */
  int32_t auto_init;
  double start_growth;
} sp_run_desc;

/* Why an advance() returned (the native march's Reason,
 * native/include/solprop_native/march/adams_march.hpp:325-347, same codes). */
enum {
  SP_REASON_REACHED = 0,   /* a save plane or the end was reached */
  SP_REASON_BOUND = 3,     /* the call's attempts or its deadline are spent */
  SP_REASON_FLOOR = 5,     /* a proposal fell below dz_min (a convergence failure) */
  SP_REASON_ERROR = 6,     /* a device or argument failure; earlier steps stand */
  SP_REASON_DIVERGED = 7,  /* a replayed step's norm is not finite */
  SP_REASON_STOPPED = 11,  /* sp_session_request_stop was called */
  SP_REASON_HALTED = 12    /* sp_session_request_snapshot: an accepted endpoint to save */
};
/* What class of solprop error a failure maps to (adams_march.hpp:349-358, same codes):
 * convergence -> solprop's ConvergenceError, backend -> BackendError, value ->
 * ValueError, refused -> BackendRefusal. */
enum {
  SP_CATEGORY_NONE = 0, SP_CATEGORY_CONVERGENCE = 1, SP_CATEGORY_BACKEND = 2,
  SP_CATEGORY_VALUE = 3, SP_CATEGORY_REFUSED = 4
};
/* Events of a batch (_core.SessionEvent's kind and outcome, folded). */
enum {
  SP_EVENT_NONE = 0,     /* the work limit or the deadline ended the call */
  SP_EVENT_PLANE = 1,    /* a save plane was reached */
  SP_EVENT_FINISHED = 2, /* the run reached its end */
  SP_EVENT_FAILED = 3,   /* the run failed; reason and category say how */
  SP_EVENT_STOPPED = 4,  /* the run was stopped on request; it takes no more attempts */
  SP_EVENT_HALTED = 5    /* an accepted endpoint after sp_session_request_snapshot */
};

/* What one advance() returns (the _core.SessionBatch / SessionEvent essentials,
 * native/src/solprop_native/_core.pyi:499-557).  `rows`, when not NULL, is the caller's
 * buffer of `rows_capacity` attempt rows of five doubles -- end, step, norm (infinity when
 * not finite), accepted (1 or 0), wall seconds of the attempt -- filled with the call's
 * attempts in order (`n_rows` of them; an attempt past the capacity is counted in the
 * totals but not written). */
typedef struct sp_batch {
  int32_t event;       /* SP_EVENT_* */
  int32_t plane_index; /* the save plane reached, or -1 */
  double z;            /* position after the batch */
  int64_t attempts, rejected, evaluations; /* cumulative counts of the run */
  int32_t reason;      /* SP_REASON_* */
  int32_t category;    /* SP_CATEGORY_*, on a failure */
  double* rows;        /* caller's buffer of rows_capacity x 5 doubles, or NULL */
  int32_t rows_capacity;
  int32_t n_rows;      /* rows written by this call */
} sp_batch;

/* The march's state between calls (_core.Session.march_state / status,
 * _core.pyi:470-476, 559-587). */
typedef struct sp_march_state {
  double z, proposal;
  int64_t attempts, rejected, evaluations;
  int32_t order;          /* Adams: the order the next attempt takes */
  int32_t history_rows;   /* Adams: accepted rows held (0 right after a restart) */
  int32_t rejections;     /* consecutive rejections */
  int32_t plane_index;    /* the next save plane */
  int32_t outcome;        /* 0 none, 1 completed, 2 stopped, 3 failed */
} sp_march_state;

/* ---- library ---- */
/* Copies the message of the last failure on this thread into buf (NUL-terminated). */
size_t sp_last_error(char* buf, size_t len);
/* Version string of this build, e.g. "solprop-b200 0.1 sm_100a". */
const char* sp_version(void);
/* Number of CUDA devices visible, or a negative sp_status on failure. */
int sp_device_count(void);

/* ---- problem (replaces _core.Problem, native _core.pyi:51-428) ---- */
sp_status sp_problem_create(const sp_problem_desc* desc, sp_problem** out);
sp_status sp_problem_destroy(sp_problem* problem);

/* ---- workspace (replaces _core.Workspace(problem), _core.pyi:600-612) ---- */
sp_status sp_workspace_create(const sp_problem* problem, int device, sp_workspace** out);
/* The same with a precision (SP_PRECISION_*). */
sp_status sp_workspace_create_ex(const sp_problem* problem, int device, int precision,
                                 sp_workspace** out);
/* How a workspace evaluates the modal transform (synthesis of the node field from the
 * modes, projection of the node streams back; numpy_ref passes/transforms.py:87-187):
 *   SP_MODAL_FUSED  inside the response column, on CUDA cores, from a modal window in
 *                   shared memory -- up to 8 modal columns;
 *   SP_MODAL_GEMM   as dense products: FP64 products in the plain form; in the mixed form
 *                   tcgen05 products of three-part BF16 splits of each operand, accumulated
 *                   in FP32 (the reference's synthesis and projection GEMMs,
 *                   native/src/general/trial.cpp:181-315, transforms/gemm.hpp:55-275) --
 *                   up to 1024 modal columns, field grid, one field component;
 *   SP_MODAL_AUTO   FUSED up to 8 columns, GEMM above. */
enum { SP_MODAL_AUTO = 0, SP_MODAL_FUSED = 1, SP_MODAL_GEMM = 2 };
sp_status sp_workspace_create_ex2(const sp_problem* problem, int device, int precision, int modal,
                                  sp_workspace** out);
sp_status sp_workspace_destroy(sp_workspace* ws);
/* One source evaluation F at a lab-frame field, untransported (numpy_ref
 * workspace.py:819 lab_source): lab and out are host complex (n_modes,n_pol,n_omega).
 * quiet != 0 leaves a quiet in-stage collar out (numpy_ref source.py:858-890). */
sp_status sp_workspace_source(sp_workspace* ws, const double* lab, double z, int quiet,
                              double* out);
/* The same on device pointers, on the workspace's stream; for timing.  It returns before
 * the evaluation ends, so a response column that gave up waiting is reported by the next
 * call on the workspace that reads the result back (sp_workspace_source, advance): the
 * column's status mark stays set until a call reports it. */
sp_status sp_workspace_source_device(sp_workspace* ws, const void* lab_device, double z,
                                     int quiet, void* out_device);
/* Kernel launches one source evaluation makes (the evidence of the device path). */
int sp_workspace_launches_per_source(const sp_workspace* ws);

/* The CUDA stream (cudaStream_t) every launch of this workspace goes to; callers that
 * time the device record their events on it. */
void* sp_workspace_stream(sp_workspace* ws);

/* ---- session (replaces _core.Session, _core.pyi:430-470) ---- */
sp_status sp_session_start(sp_workspace* ws, const sp_run_desc* run, sp_session** out);
/* Step until a save plane, the end, work_limit attempts or `deadline` host seconds (the
 * native call's bounds, _core.pyi:469 Session.advance(work_limit, deadline); a deadline
 * <= 0 or not finite means none), a requested stop or snapshot.  A failure returns its
 * status with out->event SP_EVENT_FAILED and its reason and category filled; the
 * attempts before it stand. */
sp_status sp_session_advance(sp_session* s, int32_t work_limit, double deadline, sp_batch* out);
/* Ask a running advance() -- from any thread -- to stop at the next attempt boundary
 * (_core.Session.request_stop, _core.pyi:471): it returns SP_EVENT_STOPPED, and the run
 * takes no more attempts. */
sp_status sp_session_request_stop(sp_session* s);
/* Ask advance() to return at the next accepted endpoint (SP_EVENT_HALTED), where a
 * snapshot holds a consistent history (_core.Session.request_snapshot, _core.pyi:472). */
sp_status sp_session_request_snapshot(sp_session* s);
/* The march's state (_core.Session.march_state / status). */
sp_status sp_session_march_state(const sp_session* s, sp_march_state* out);
/* Copies the current state to out, host complex (n_modes, n_pol, n_omega). */
sp_status sp_session_export(sp_session* s, double* out);
/* A plane's statistics, formed on the device from the run's current state (the native
 * workspace's statistics pass, native/src/general/statistics.cpp:106-450, with solprop's
 * definitions, src/solprop/stats/definitions.py:148-500): only these small arrays come
 * back.  Each pointer is the caller's host buffer, or NULL to skip that statistic.
 *   energy           n_modes*n_pol  J per column: dt / n_t sum_k w_k |a_k|^2 p_k, w_k 1 at a
 *                                   field grid's DC and Nyquist bins, 4 inside, 1 on an
 *                                   envelope grid (fourier.energy_omega)
 *   omega0           n_modes*n_pol  rad/s: the centroid sum omega |a|^2 p / sum |a|^2 p, NaN
 *                                   for an empty column
 *   peak_power       n_modes        W: max over time of sum_pol |E_a(t)|^2, E_a the analytic
 *                                   signal of the column on the coarse grid
 *   peak_power_total 1              W: max over time of the power summed over every column
 *   spectrum         n_omega        J per bin: dt / n_t w_k sum_columns |a_k|^2 p_k
 * p is the caller's power weight (n_modes, n_pol, n_omega) or 1 when power_weight is NULL;
 * the peak powers are the unweighted ones (solprop's saved-field definitions). */
typedef struct sp_statistics {
  double* energy;
  double* omega0;
  double* peak_power;
  double* peak_power_total;
  double* spectrum;
} sp_statistics;
sp_status sp_session_statistics(sp_session* s, const double* power_weight, sp_statistics* out);
/* The run's resumable state as one self-describing byte string (_core.Session.snapshot,
 * _core.pyi:484-494; the Adams history rows of native trial_adams.inc:526-605): the
 * march's scalars and history positions, the state, and the device history rows.  With
 * buf NULL (or capacity too small) it writes the size needed to *size and copies nothing
 * (SP_ERR_ARGUMENT when buf is not NULL). */
sp_status sp_session_snapshot(sp_session* s, void* buf, size_t capacity, size_t* size);
/* A session continuing a snapshot on a workspace of the same problem: the run's policy
 * comes from `run` (its field0 may be NULL), everything else from the snapshot, and the
 * continuation takes the bits the uninterrupted run would. */
sp_status sp_session_restore(sp_workspace* ws, const sp_run_desc* run, const void* snapshot,
                             size_t size, sp_session** out);
sp_status sp_session_destroy(sp_session* s);

/* Per-kernel device timing of a session (replaces the native timing probe and counters,
 * _core.Workspace.probe/counters, _core.pyi:600-612, bindings/module.cpp:832).  While
 * enabled, CUDA events are recorded on the workspace stream around every launch and the
 * elapsed times accumulate per kernel family, in this order: */
enum {
  SP_K_PREDICT = 0, SP_K_INVERSE, SP_K_COLUMN, SP_K_PROJECT, SP_K_FORWARD, SP_K_OUTPUT,
  SP_K_CORRECT, SP_K_ACCEPT, SP_K_START, SP_K_RK_STAGE, SP_K_RK_FINISH, SP_K_COUNT
};
sp_status sp_session_set_timing(sp_session* s, int enable);
/* ms[SP_K_COUNT] accumulated milliseconds, launches[SP_K_COUNT] launch counts; reset=1
 * clears them after reading. */
sp_status sp_session_timing(sp_session* s, double* ms, int64_t* launches, int reset);

/* ---- scans: many independent runs stepped together ---- */
/* The parameter-scan workload (solprop's run_scan, src/solprop/driver/scan.py:30, runs
 * each point as its own process through an executor, driver/executors/*.py; the native
 * backend has no batch, native SEP 36 follow-up).  Each batch step gives every
 * unfinished run one exponential-Adams attempt with batched launches and one host
 * decision pass; runs keep their own grids, mode counts, step sizes and orders. */
typedef struct sp_scan sp_scan;
typedef struct sp_scan_status {
  int32_t active;                          /* runs not yet finished */
  int64_t attempts, rejected, evaluations; /* summed over the runs */
  int64_t batch_steps;
} sp_scan_status;
sp_status sp_scan_create(int32_t n_runs, const sp_problem* const* problems,
                         const sp_run_desc* runs, int device, sp_scan** out);
/* The same with a precision (SP_PRECISION_*) for every run. */
sp_status sp_scan_create_ex(int32_t n_runs, const sp_problem* const* problems,
                            const sp_run_desc* runs, int device, int precision, sp_scan** out);
/* Up to `steps` batch steps (fewer when every run has finished).  A batch step gives every
 * run in the batch one attempt; runs gone on alone (sp_scan_set_alone) step meanwhile, and
 * once no batch is left the call lets them take up to `steps` attempts each. */
sp_status sp_scan_advance(sp_scan* scan, int32_t steps, sp_scan_status* out);
/* One run's state (host complex, may be NULL) and counts (event 2: finished, 3: failed). */
sp_status sp_scan_run(sp_scan* scan, int32_t run, double* state, sp_batch* info);
void* sp_scan_stream(sp_scan* scan);
/* One scan run's statistics at its current state, as sp_session_statistics: a scan
 * reports per-run statistics without exporting the states.  No counterpart in the
 * reference, which has no batch. */
sp_status sp_scan_statistics(sp_scan* scan, int32_t run, const double* power_weight,
                             sp_statistics* out);
/* Per-family device timing of a scan's batch steps (the session's SP_K_* families: the
 * batched predictor, inverse transforms, response column, forward transforms, stage
 * output, corrector and accept).  While enabled, CUDA events are recorded around every
 * batched launch family and the attempt phase runs as plain launches instead of its
 * captured graph.  No counterpart in the reference. */
sp_status sp_scan_set_timing(sp_scan* scan, int enable);
sp_status sp_scan_timing(sp_scan* scan, double* ms, int64_t* launches, int reset);
/* The scan's plan, as text: whether the attempt phase runs as one captured CUDA graph,
 * the response column's form, the host's time per batch step so far, and per grid size
 * whether the inverse and forward transforms run in one CTA per row or over a cluster of
 * 2, 4 or 8 CTAs, with the autotuner's timings (ms per launch; -1 where a form was not a
 * candidate).
 * Returns the text's length. */
size_t sp_scan_describe(const sp_scan* scan, char* buf, size_t len);
/* The response column's form in a scan.  The scan's autotuner times both at creation
 * and keeps the faster; this call fixes one (a later attempt recaptures its graph).
 * SP_SCAN_COLUMN_TILES: one CTA per (tile, node group), the running integrals handed
 * from tile to tile between CTAs; SP_SCAN_COLUMN_SWEEP: one CTA per (run, node group)
 * walking the tiles in order.  Both give the same bits.  No counterpart in the
 * reference, which has no batch. */
#define SP_SCAN_COLUMN_TILES 1
#define SP_SCAN_COLUMN_SWEEP 2
sp_status sp_scan_set_column(sp_scan* scan, int32_t form);
/* Runs that go on alone.  A run whose remaining attempts (the distance left over its next
 * step) exceed `factor` times the median of the batch's runs and `min_remaining` leaves
 * the batch -- which would otherwise give it one attempt per batch step for many steps --
 * and goes on as a single run on a host thread of its own, beside the batched steps, at
 * most `max_runs` at a time (0: none; defaults 6, 2000, 4).  Such a run takes as many
 * attempts per batch step as it manages.  No counterpart in the reference. */
sp_status sp_scan_set_alone(sp_scan* scan, int32_t max_runs, double min_remaining, double factor);
/* The transforms' forms for the runs of one grid size: 0 for one CTA per row, or a
 * cluster of 2, 4 or 8 CTAs per row.  The autotuner's choice stands otherwise; fixing the
 * forms makes two scans of the same runs give the same bits.  SP_ERR_ARGUMENT when no run
 * has that grid size or a row does not fit the form.  No counterpart in the reference. */
sp_status sp_scan_set_transforms(sp_scan* scan, int32_t n_to, int32_t inverse_cluster,
                                 int32_t forward_cluster);
sp_status sp_scan_destroy(sp_scan* scan);

/* ---- the scan surrogate's multilayer perceptron (no counterpart in the reference) ----
 * Device pointers to row-major FP32 tensors; products run in BF16 on the tensor cores
 * with FP32 accumulation.  stream may be NULL (the legacy default stream).
 * sp_mlp_gemm: C[M,N] = op(A) op(B) with op(A)(m,k) = transA ? A[k*lda+m] : A[m*lda+k],
 * op(B)(k,n) = transB ? B[n*ldb+k] : B[k*ldb+n]; epilogue 0: none, 1: + bias[n],
 * 2: GELU(. + bias[n]) with the pre-activation written to pre (ld = ldc) when not NULL. */
sp_status sp_mlp_gemm(const float* A, int lda, int transA, const float* B, int ldb, int transB,
                      float* C, int ldc, int M, int N, int K, const float* bias, int epilogue,
                      float* pre, void* stream);
/* The forward product on the fifth-generation tensor cores (tcgen05, operands brought by
 * TMA): C[M,N] = A[M,K] W[N,K]^T (+ bias) (GELU), A and W BF16 with K contiguous (row
 * pitches lda, ldw elements, multiples of 8; 16-byte aligned), K a multiple of 64, N a
 * multiple of 256; writes FP32 C (pitch ldc) and/or BF16 C16 (pitch ldc16) when not NULL.
 * epilogue 0: none, 1: + bias[n], 2: GELU(. + bias[n]), 3 (training): C the pre-activation
 * . + bias[n], C16 its GELU.  *status (device int) is set to 1 if a wait inside the kernel
 * gave up. */
sp_status sp_mlp_gemm_tc(const void* A, int lda, const void* W, int ldw, float* C, int ldc,
                         void* C16, int ldc16, int M, int N, int K, const float* bias,
                         int epilogue, int* status, void* stream);
/* The same product for `count` (1..8) operand and output sets of one shape in one launch
 * (an ensemble's members through one layer): A[q], W[q], C[q] / C16[q] (NULL arrays or
 * entries where unused), bias[q] (or bias NULL). */
sp_status sp_mlp_gemm_tc_batch(int count, const void* const* A, int lda, const void* const* W, int ldw,
                               float* const* C, int ldc, void* const* C16, int ldc16, int M, int N, int K,
                               const float* const* bias, int epilogue, int* status, void* stream);
/* The transpose of a (rows, cols) FP32 (src_bf16 0) or BF16 (1) matrix as BF16,
 * dst[c * ld_dst + r], zero-padded from rows to rows_pad: the operands of the training's
 * weight and input gradients as products C = A W^T on the tensor cores. */
sp_status sp_mlp_transpose_bf16(const void* src, int src_bf16, int ld_src, int rows, int cols,
                                void* dst, int ld_dst, int rows_pad, void* stream);
/* FP32 rows to BF16 rows, zero-padded from cols to cols_out columns. */
sp_status sp_mlp_to_bf16(const float* src, int ld_src, int rows, int cols, void* dst,
                         int ld_dst, int cols_out, void* stream);
/* dZ = dA * GELU'(pre), elementwise over n values. */
sp_status sp_mlp_gelu_backward(const float* dA, const float* pre, float* dZ, size_t n, void* stream);
/* db[n] = sum over the M rows of dZ[m, n] (rows in order). */
sp_status sp_mlp_bias_grad(const float* dZ, int M, int N, float* db, void* stream);
/* Mean squared error of Y against T (M x N): dY = 2 (Y - T) / (M N), *loss (device) the mean;
 * row_loss is M floats of scratch. */
sp_status sp_mlp_mse(const float* Y, const float* T, int M, int N, float* dY, float* row_loss,
                     float* loss, void* stream);
/* One Adam step (bias-corrected, step >= 1) on n FP32 weights. */
sp_status sp_mlp_adam(float* w, const float* grad, float* m1, float* m2, size_t n, float lr,
                      float beta1, float beta2, float eps, int step, void* stream);
/* Ensemble statistics of Y (members, M, N) of log10 spectral densities: mean (M, N) and,
 * per row, the disagreement: the standard deviation over members of each output weighted
 * by 10^mean (the mean spectrum's energy there), over the summed weights. */
sp_status sp_mlp_ensemble_stats(const float* Y, int members, int M, int N, float* mean,
                                float* spread, void* stream);

/* One source evaluation that allocates no device memory, for callers that cannot call
 * cudaMalloc: code whose device memory belongs to a pool or a framework that owns every
 * allocation, or that runs where an allocation would synchronise the device or fail.
 * It has no counterpart in the reference.  It computes what sp_workspace_source_device
 * computes, from the host-side problem (sp_problem_create allocates host memory only),
 * with lab and out device pointers (complex (n_modes, n_pol, n_omega)) on the caller's
 * stream (NULL: the legacy default stream), and returns once the result is written.
 *
 * Every device buffer it uses -- the problem's tables, uploaded again on every call,
 * and the evaluation's intermediates -- lies in one fixed array of 40 MiB inside the
 * library, which every GPU that loads the library holds until the process exits; a
 * problem needing more is refused with SP_ERR_ARGUMENT.  The first call on a device
 * resolves that array's device address (cudaGetSymbolAddress) with the device current,
 * so make the first call on each device before any stream capture.  All calls share the
 * array: calls that overlap on the GPU -- from several threads or streams at once -- race,
 * so serialise them. */
sp_status sp_source_noalloc(const sp_problem* problem, const void* lab, double z, int quiet,
                            void* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SOLPROP_B200_H */
