/*
 * spinsim_b200.h -- C ABI of the B200 Chebyshev echo engine.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and
 * returns an `int` status (SS_OK == 0).  On failure the thread-local message
 * from ss_last_error() says what went wrong; the C++ host layer turns the
 * status back into the exception type the reference throws (see the table
 * below each status).  Device work is queued on the engine's stream; calls
 * that hand results to host memory synchronise that stream first.
 *
 * Conventions shared with the reference (spinsim, include/spinsim/core):
 *   - spin s owns bit s of a basis index, set bit = up (core/Bits.hpp:15-32);
 *   - amplitudes are interleaved re/im doubles, amplitude k at [2k], [2k+1]
 *     (core/StateVector.hpp:50-55);
 *   - kernels act with Pauli matrices, the physics uses S = sigma/2
 *     (core/SpinOperators.hpp:9-17, src/core/Hamiltonian.cpp:58-60);
 *   - real-time evolution is exp(+iHt) (src/core/Propagator.cpp:14-35).
 */
#ifndef SPINSIM_B200_H
#define SPINSIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---------------------------------------------------------------- status */
enum ss_status {
  SS_OK = 0,
  SS_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument                    */
  SS_ERR_OUT_OF_RANGE = 2,     /* std::out_of_range                        */
  SS_ERR_DOMAIN = 3,           /* std::domain_error (zero norm, bound <= 0) */
  SS_ERR_CONVERGENCE = 4,      /* spinsim::ChebyshevConvergenceError       */
  SS_ERR_CONFIG = 5,           /* spinsim::ConfigError                     */
  SS_ERR_RUNTIME = 6,          /* std::runtime_error (shape mismatch, ...) */
  SS_ERR_OVERFLOW = 7,         /* std::overflow_error (Bessel I, x > 709)  */
  SS_ERR_CUDA = 8,             /* a CUDA call failed                       */
  SS_ERR_NO_DEVICE = 9,        /* no usable sm_100 device                  */
  SS_ERR_TIMEOUT = 10,         /* a bounded device wait gave up            */
  SS_ERR_NUMERIC = 11          /* a norm reduction saw NaN or Inf          */
};

enum ss_axis { SS_AXIS_X = 0, SS_AXIS_Y = 1, SS_AXIS_Z = 2 };
enum ss_time_mode { SS_TIME_REAL = 0, SS_TIME_IMAGINARY = 1 };
enum ss_precision {
  SS_PRECISION_FP64 = 0,  /* everything in FP64                                */
  SS_PRECISION_MIXED = 1  /* FP32 T_n recursion, FP64 series sum and reductions */
};
/* Kernel family of the plain propagator's Chebyshev order. */
enum ss_evolve_kernel {
  SS_KERNEL_AUTO = 0,        /* the faster family for the vector's size          */
  SS_KERNEL_GATHER = 1,      /* one sweep per order; every amplitude gathers its
                                partners through L1                              */
  SS_KERNEL_TILED = 2,       /* a few passes per order over shared-memory tiles
                                of 12 spins (FP64) or 13 (mixed): needs L >= that */
  SS_KERNEL_TILED_SMALL = 3  /* the same with tiles of 8 spins (L >= 8)          */
};

enum ss_initial_state {
  SS_INIT_RANDOM = 0,         /* core: InitialStateKind::Random (Ensemble.hpp:21-26) */
  SS_INIT_UP = 1,
  SS_INIT_DOWN = 2,
  SS_INIT_BASIS = 3,
  SS_INIT_RANDOM_PRODUCT = 4  /* additive: per-spin random Bloch vectors      */
};

enum ss_step_kind {
  SS_STEP_EVOLVE = 0,  /* sequence/Sequence.hpp:28-34 Evolve  */
  SS_STEP_PULSE = 1,   /* sequence/Sequence.hpp:37-39 Pulse   */
  SS_STEP_MEASURE = 2, /* sequence/Sequence.hpp:42 Measure    */
  SS_STEP_REPEAT = 3   /* sequence/Sequence.hpp:47-56 Repeat  */
};

enum ss_observable_kind {
  SS_OBS_CORR = 0,   /* corr:<axis>        (core/Observable.hpp:66-78)   */
  SS_OBS_MAG = 1,    /* mag:<spin>:<axis>  (core/Observable.hpp:80-92)   */
  SS_OBS_NORM = 2,   /* norm               (core/Observable.hpp:94-105)  */
  SS_OBS_ENERGY = 3  /* energy             (core/Observable.hpp:107-118) */
};

/*
 * One node of a pulse program.  The tree of sequence::Step is stored in
 * pre-order: a REPEAT node is followed by the `body_len` nodes of its body
 * (its whole subtree, nested repeats included).
 */
typedef struct ss_step {
  int32_t kind;          /* ss_step_kind                                  */
  int32_t mode;          /* EVOLVE: ss_time_mode                          */
  int32_t autonormalize; /* EVOLVE: rescale to unit norm after each step  */
  int32_t field_table;   /* EVOLVE: -1 keeps the system's fields, else an
                            index into ss_run_config.step_fields          */
  int64_t count;         /* EVOLVE: number of steps; REPEAT: repetitions  */
  int32_t body_len;      /* REPEAT: nodes in the body subtree             */
  int32_t target;        /* PULSE: -1 = every spin, else a 0-based spin   */
  double tau;            /* EVOLVE: step length                           */
  double angle;          /* PULSE: rotation angle in radians              */
  double axis[3];        /* PULSE: rotation axis (normalised by the host) */
  int32_t tau_from_draw; /* EVOLVE (additive): 1 = use the realisation's
                            drawn tau (scaled by `tau`) instead of `tau`   */
  int32_t reserved;
} ss_step;

typedef struct ss_observable {
  int32_t kind; /* ss_observable_kind */
  int32_t axis; /* ss_axis            */
  int32_t spin; /* MAG: 0-based spin  */
  int32_t reserved;
} ss_observable;

/*
 * A whole experiment, the C view of io/Config.hpp:32-58 RunConfig.
 * Fields marked "additive" have no counterpart in the reference schema and
 * default to "off" when zeroed.
 */
typedef struct ss_run_config {
  int32_t nspins;
  int32_t initial_state;     /* ss_initial_state                         */
  uint64_t basis_index;
  uint64_t realizations;
  uint64_t seed;
  int32_t generate_geometry; /* dipolar 2D placement per realisation     */
  int32_t reference_axis;    /* ss_axis                                  */
  double dipolar_scale;
  double field_disorder;     /* sigma of the Gaussian Hz offset          */
  double epsilon;            /* Chebyshev coefficient cutoff             */
  const double* base_fields; /* 3 * nspins: (x, y, z) per spin           */
  int32_t n_observables;
  int32_t n_steps;
  const ss_observable* observables;
  const ss_step* steps;      /* pre-order program                        */
  int32_t n_step_fields;
  int32_t reserved0;
  const double* step_fields; /* n_step_fields tables of 3 * nspins       */
  /* additive: per-realisation draws from a harness stream (seed2, index)
     that leaves the (seed, index) geometry stream untouched */
  uint64_t draw_seed;
  double disorder_range[2];  /* if hi > lo: sigma ~ U[lo, hi)            */
  double tau_range[2];       /* if hi > lo: tau ~ U[lo, hi)              */
  int32_t n_spin_choices;    /* if > 0: L drawn uniformly from the list  */
  int32_t spin_choices[8];
  /* additive: in SS_PRECISION_MIXED, a realisation whose Chebyshev orders
     per state vector exceed this runs in the FP64 kernel of the same batch
     (the FP32 recursion's rounding error grows with the order count and
     shrinks with L); 0 = the measured per-size limits (7400 orders at
     L = 8, 11600 at 10, 38600 at 12, 40000 at 13..15, L = 16 staying mixed),
     > 0 = that limit at every size, negative = never. */
  int64_t mixed_order_limit;
  /* additive: a parameter sweep for the batched engine.  With
     sweep_points = P > 0 a batch of `count` realisations is P consecutive
     blocks of count / P; slot s of point p = s / (count / P) draws its
     geometry, fields and initial state for index first + s % (count / P)
     (every point sees the same realisations) and takes the point's row of
     sweep_params = (dipolar_scale, field_disorder, tau for tau_from_draw
     steps, pulse-angle scale). */
  int32_t sweep_points;
  int32_t reserved1;
  const double* sweep_params; /* 4 * sweep_points */
} ss_run_config;

/* ---------------------------------------------------------------- handles */
typedef struct ss_engine ss_engine;
typedef struct ss_state ss_state;
typedef struct ss_ham ss_ham;
typedef struct ss_batch ss_batch;

/* Thread-local description of the last failure on this thread. */
const char* ss_last_error(void);
/* Library version as 10000*major + 100*minor + patch. */
int ss_version(void);

/* ------------------------------------------------------------------ engine
 * One device, one CUDA stream.  Calls on one engine are not re-entrant. */
int ss_engine_create(int device, ss_engine** out);
int ss_engine_destroy(ss_engine* engine);
int ss_engine_synchronize(ss_engine* engine);
/* The engine's cudaStream_t, for callers that time or order work around it. */
void* ss_engine_stream(ss_engine* engine);
/* Number of kernels this engine has launched since creation. */
int64_t ss_engine_launch_count(const ss_engine* engine);

/* ----------------------------------------------------------- state vector
 * core/StateVector.hpp:82-140.  2^L FP64 complex amplitudes in device
 * memory, interleaved, 256-byte aligned. */
int ss_state_create(ss_engine* engine, int nspins, ss_state** out);
int ss_state_destroy(ss_state* state);
int ss_state_nspins(const ss_state* state);
int ss_state_upload(ss_state* state, const double* interleaved);
int ss_state_download(const ss_state* state, double* interleaved);
int ss_state_copy(ss_state* dst, const ss_state* src);
/* StateVector.cpp:10-33 setZero / scale / negate / addScaled */
int ss_state_set_zero(ss_state* state);
int ss_state_scale(ss_state* state, double factor);
int ss_state_negate(ss_state* state);
int ss_state_add_scaled(ss_state* dst, double cr, double ci,
                        const ss_state* other);
/* StateVector.cpp:35-41 setBasisState */
int ss_state_set_basis(ss_state* state, uint64_t index);
/* StateVector.cpp:43-56 norm / normalize */
int ss_state_norm(const ss_state* state, double* out);
int ss_state_normalize(ss_state* state, double* norm_before);
/* StateVector.cpp:58-70 innerProduct: <other|self> */
int ss_state_inner_product(const ss_state* self, const ss_state* other,
                           double out[2]);
/* StateVector.cpp:72-75 swap (exchanges the device buffers) */
int ss_state_swap(ss_state* a, ss_state* b);

/* ------------------------------------------------------- Pauli kernels
 * core/SpinOperators.hpp:22-58.  `in` and `out` must be distinct. */
int ss_axpy_sigma(double c, const ss_state* in, int spin, int axis,
                  ss_state* out);
int ss_apply_sigma(const ss_state* in, int spin, int axis, ss_state* out);
int ss_axpy_coupling(double jx, double jy, double jz, const ss_state* in,
                     int spin_a, int spin_b, ss_state* out);
/* out += c * diag[k] * in[k] with a host diagonal of 2^L doubles
   (SpinOperators.cpp:211-226 axpyDiagonal). */
int ss_axpy_diagonal(double c, const double* diagonal, const ss_state* in,
                     ss_state* out);
/* out = sum_s sigma_axis(s) in  (src/ensemble/Ensemble.cpp:47-58,
   src/core/Observable.cpp:13-22) */
int ss_apply_total_spin(int axis, const ss_state* in, ss_state* out);

/* ------------------------------------------------------------ Hamiltonian
 * core/Hamiltonian.hpp:32-110. */
int ss_ham_create(ss_engine* engine, int nspins, ss_ham** out);
int ss_ham_destroy(ss_ham* ham);
/* Replaces every term: fields (x,y,z per spin, 3*nspins doubles), npairs
   couplings given as (low, high) spin pairs and (jx, jy, jz) triples.  A
   repeated pair overwrites the earlier one (Hamiltonian.cpp:39-52). */
int ss_ham_set_terms(ss_ham* ham, const double* fields, int npairs,
                     const int32_t* pairs, const double* couplings);
/* Replaces the fields only (Sequence.cpp:17-31 swapFields/restoreFields). */
int ss_ham_set_fields(ss_ham* ham, const double* fields);
/* Hamiltonian.cpp:82-93 spectralBound */
int ss_ham_spectral_bound(const ss_ham* ham, double* out);
/* out (+)= scale * H * in, H the physical spin-1/2 Hamiltonian.
   accumulate = 0 overwrites (applyPhysical, Hamiltonian.cpp:129-132),
   accumulate = 1 adds (accumulate, Hamiltonian.cpp:95-127). */
int ss_ham_apply(const ss_ham* ham, double scale, const ss_state* in,
                 ss_state* out, int accumulate);

/* ------------------------------------------------------------ Bessel
 * core/Bessel.hpp:29-45 besselJ / besselI: kind 0 = J, 1 = I. */
int ss_bessel(int kind, double x, int64_t count, double* values,
              int64_t* nonzero);

/* ------------------------------------------------------------ Chebyshev
 * core/Chebyshev.hpp:56-64 ChebyshevExpansion::build.  Writes order+1
 * coefficients (cap must allow it) and the effective bound. */
int ss_chebyshev_build(int mode, double spectral_bound, double tau,
                       double epsilon, int64_t max_order, double* coeffs,
                       int64_t cap, int64_t* order, double* effective_bound);

/* ------------------------------------------------------------ Propagator
 * src/core/Propagator.cpp:46-100.  ss_evolve applies a ready expansion
 * (coefficients a_0..a_order built against `bound`) `nsteps` times;
 * ss_propagate also builds it, exactly as Propagator::evolve does. */
int ss_evolve(const ss_ham* ham, ss_state* psi, const double* coeffs,
              int64_t ncoeffs, double bound, int mode, int64_t nsteps,
              int autonormalize);
int ss_propagate(const ss_ham* ham, ss_state* psi, int mode, double tau,
                 int64_t nsteps, int autonormalize, double epsilon,
                 int64_t* order_used);
/* The same two calls with a precision (ss_precision) and a kernel family
 * (ss_evolve_kernel).  The reference propagates in FP64 only
 * (src/core/Propagator.cpp:46-100); SS_PRECISION_MIXED keeps psi, the series
 * weights, the diagonal and each T_n's formation in FP64 and stores the
 * Chebyshev vectors T_n and the off-diagonal partial sums in FP32.
 * ss_evolve / ss_propagate are these with SS_PRECISION_FP64, SS_KERNEL_AUTO. */
int ss_evolve_ex(const ss_ham* ham, ss_state* psi, const double* coeffs,
                 int64_t ncoeffs, double bound, int mode, int64_t nsteps,
                 int autonormalize, int precision, int kernel);
int ss_propagate_ex(const ss_ham* ham, ss_state* psi, int mode, double tau,
                    int64_t nsteps, int autonormalize, double epsilon,
                    int precision, int kernel, int64_t* order_used);
/* Host only, no counterpart in the reference: the tile patterns of
 * SS_KERNEL_TILED for an nspins-spin vector and tiles of tile_bits spins
 * that all hold spins 0 .. line_bits-1 (the tiled kernel uses 12 and 3 in
 * FP64, 13 and 4 in mixed precision: whole 128-byte runs), one bit mask per
 * pass (every pair of spins shares a pattern; the last pass forms T_n).
 * *npass receives the count; masks (capacity cap) may be NULL. */
int ss_tile_plan(int nspins, int tile_bits, int line_bits, int32_t* npass,
                 uint32_t* masks, int32_t cap);
/* No counterpart in the reference: the schedule of SS_KERNEL_TILED per
 * precision, as register bits per thread (FP64: 3 or 4, mixed: 4 or 5; 0 =
 * the default, the faster on B200).  Process-wide; results are the same for
 * every choice up to the order of the sums. */
int ss_tiled_select(int precision, int register_bits);

/* ------------------------------------------------------------ gates
 * src/core/Gate.cpp:20-33 Rotation2x2::make; :60-85 SpinRotation::apply;
 * :90-121 TwoSpinGate::apply.  u = (ll, lh, hl, hh) as re,im pairs in the
 * (down, up) basis; m = 4x4 row-major complex in (dd, du, ud, uu) order. */
int ss_rotation_matrix(const double axis[3], double angle, double u[8]);
int ss_rotate(ss_state* psi, const double u[8], const int32_t* targets,
              int32_t ntargets);
int ss_two_spin_gate(ss_state* psi, const double m[32], int spin_a,
                     int spin_b);

/* ------------------------------------------------------------ observables
 * src/core/Observable.cpp:66-120. */
int ss_measure_corr(const ss_state* psi, const ss_state* ref, int axis,
                    double out[2]);
int ss_measure_mag(const ss_state* psi, int spin, int axis, double* out);
int ss_measure_energy(const ss_ham* ham, const ss_state* psi, double* out);

/* No counterpart in the reference: ss_measure_corr over caller-owned device
 * vectors (2*2^nspins doubles each, re/im interleaved, 16-byte aligned, on
 * the current device), allocating nothing.  Its scratch is a fixed ~19 KB
 * array in the library's device memory; nspins outside [1, 30] is rejected
 * with SS_ERR_OUT_OF_RANGE, and a vector whose allocation ends before its
 * 2*2^nspins doubles with SS_ERR_INVALID_ARGUMENT.  `stream` is a
 * cudaStream_t (NULL = the legacy default stream); the call waits for it.
 * The first successful call on each device looks the scratch up (make it
 * before any stream capture; a failed look-up is retried by the next call)
 * and keeps its address for the life of the process, so the device's
 * primary context must not be reset in between.  Calls that overlap on one
 * device race on the scratch: serialise them. */
int ss_measure_corr_noalloc(const double* psi, const double* ref, int nspins,
                            int axis, void* stream, double out[2]);

/* ------------------------------------------------------------ ensemble
 * Host-side, bit-for-bit with the reference's (seed, index) streams:
 * src/ensemble/Rng.cpp:8-23, Ensemble.cpp:20-112, io/Experiment.cpp:10-35.
 * Fills the realisation's fields (3L), couplings (pairs 2*P, J 3*P, P
 * written to *npairs; capacity L(L-1)/2) and initial state (2*2^L). */
int ss_realization_setup(const ss_run_config* config, uint64_t index,
                         int32_t* nspins, double* fields, int32_t* pairs,
                         double* couplings, int32_t* npairs, double* psi0);

/* ------------------------------------------------------ plain FP64 path
 * runRealization (io/Experiment.cpp:10-55) + Sequence::run
 * (src/sequence/Sequence.cpp:69-106) for one realisation: the program is
 * interpreted on the host and every step runs on the device in FP64, with
 * one Propagator::evolve per Evolve step for the state and the reference.
 * times: points; values: points x width (see ss_batch_shape). */
int ss_run_realization(ss_engine* engine, const ss_run_config* config,
                       uint64_t index, double* times, double* values);
/* The same with the propagator's precision (ss_precision) and kernel family
 * (ss_evolve_kernel), as ss_propagate_ex takes them; ss_run_realization is
 * this with SS_PRECISION_FP64 and SS_KERNEL_AUTO. */
int ss_run_realization_ex(ss_engine* engine, const ss_run_config* config,
                          uint64_t index, int precision, int kernel,
                          double* times, double* values);

/* -------------------------------------------------------- batched engine
 * Runs `count` realisations (indices first..first+count-1) of a whole
 * pulse program on the device, state and reference together, and returns
 * their measurement rows in realisation-index order.  This replaces the
 * thread pool of io/Experiment.cpp:57-72 + ensemble/EnsembleRunner.cpp:27-88
 * for one GPU. */
int ss_batch_create(ss_engine* engine, const ss_run_config* config,
                    uint64_t first, int64_t count, int precision,
                    ss_batch** out);
int ss_batch_destroy(ss_batch* batch);
/* Shape: measurement points per realisation, values per point. */
int ss_batch_shape(const ss_batch* batch, int64_t* points, int64_t* width);
/* Uploads the prepared inputs, runs the program and downloads the rows:
   rows is count x points x width, times is points. */
int ss_batch_run(ss_batch* batch, double* rows, double* times);
/* Device-only pieces of ss_batch_run, for timing with inputs resident. */
int ss_batch_upload(ss_batch* batch);
int ss_batch_execute(ss_batch* batch);
int ss_batch_download(ss_batch* batch, double* rows, double* times);
/* Work statistics: total Chebyshev orders applied per run (both vectors,
   all realisations), amplitudes processed per run, kernel launches. */
int ss_batch_stats(const ss_batch* batch, int64_t* orders,
                   double* amplitude_orders, int64_t* launches);
/* Bytes ss_batch_run moves host->device (inputs) and device->host (rows). */
int ss_batch_io_bytes(const ss_batch* batch, int64_t* h2d, int64_t* d2h);
/* Per realisation, in index order (count entries each): the precision it
   runs in (ss_precision; in a mixed batch those past mixed_order_limit are
   FP64) and the amplitudes x orders it applies per run (both vectors).
   Either output may be NULL. */
int ss_batch_precisions(const ss_batch* batch, int32_t* precision,
                        double* amplitude_orders);
/* No counterpart in the reference: per realisation, in index order, the
   coherent error mixed precision would accumulate -- Chebyshev orders (both
   vectors) times the FP32 rounding residuals of the coefficients the kernel
   leaves uncorrected, in the expansion's scaled units -- whatever precision
   it runs in. */
int ss_batch_error_estimates(const ss_batch* batch, double* estimate);

/* ------------------------------------------------------------- autotuner
 * No counterpart in the reference (its CPU kernels have one schedule).
 * Each batched size has candidate schedules -- register bits per thread
 * (the term grouping of the layout passes) and CTAs per state vector.
 * ss_batch_tune times every candidate of every size the config can draw
 * (and, for SS_PRECISION_MIXED, the FP64 kernels of the sizes whose
 * realisations mixed_order_limit can route) on realisations
 * from `first` of the config's own program -- `sample` of them, raised to
 * four waves of the candidate's resident clusters -- installs the
 * fastest in the process-wide schedule table keyed by device name, size and
 * precision, and, if cache_path is not NULL, merges the table into that
 * file (tab-separated text).  Later batches use the table's kernels and,
 * when every size of a batch has been measured, the measured costs for
 * their buckets' shares of the device. */
int ss_batch_tune(ss_engine* engine, const ss_run_config* config, uint64_t first,
                  int64_t sample, int precision, const char* cache_path);
/* Installs the schedules recorded in a cache file written by ss_batch_tune. */
int ss_schedule_load(const char* cache_path);
int ss_schedule_clear(void);
/* The schedule table as text, one "device L precision variant ns" line per
 * entry; *needed receives the buffer size the whole text needs. */
int ss_schedule_describe(char* buf, size_t cap, size_t* needed);
/* Every compiled schedule: "name threads shared_bytes" per line. */
int ss_batch_variants(char* buf, size_t cap, size_t* needed);
/* Split-cluster schedules (names ending ".split") run the state and the
 * reference of a realisation on clusters of their own and keep both vectors
 * at every measurement point; a bucket runs in launches whose snapshots fit
 * `bytes` of device memory (default 16 GiB), or with the paired schedule of
 * its size when fewer than 64 realisations (or the whole bucket) would fit.
 * A size with no paired schedule (FP64 at L = 16) runs at least one
 * realisation per launch.  Process-wide; applies to batches created
 * afterwards.  bytes >= 0. */
int ss_set_snapshot_budget(int64_t bytes);

/* -------------------------------------------------------- echo surrogate
 * No counterpart in the reference (its parameter sweeps always run the
 * exact propagator, io/Experiment.cpp:57-72).  A 6 -> 256 -> 256 -> 256 ->
 * 128 GELU MLP mapping (areal density, field sigma, tau, pulse-angle error,
 * sequence, L), each normalised by the caller, to the disorder-averaged
 * S^x echo at 128 times.  BF16 weights and activations, FP32 accumulation,
 * FP32 master weights under Adam; every product runs on the tcgen05 tensor
 * cores.  Parameters are flat FP32 in the order W0[256][6] b0[256]
 * W1[256][256] b1 W2[256][256] b2 W3[128][256] b3[128] (ss_mlp_param_count
 * values).  `batch` rows go through the device per pass (a multiple of
 * 128); inputs are rows of 6 floats, outputs and targets rows of 128. */
typedef struct ss_mlp ss_mlp;
int64_t ss_mlp_param_count(void);
int ss_mlp_create(ss_engine* engine, int batch, uint64_t seed, ss_mlp** out);
int ss_mlp_destroy(ss_mlp* net);
int ss_mlp_get_params(const ss_mlp* net, float* params);
/* Replaces every parameter and resets the Adam state. */
int ss_mlp_set_params(ss_mlp* net, const float* params);
/* y[rows][128] = net(x[rows][6]); any number of rows. */
int ss_mlp_forward(ss_mlp* net, const float* x, int64_t rows, float* y);
/* Gradient of the mean-squared error over rows (1..batch) of x and target
 * with respect to every parameter (flat order), and the loss; no update. */
int ss_mlp_gradients(ss_mlp* net, const float* x, const float* target,
                     int64_t rows, float* grads, double* loss);
/* Uploads a training set (rows >= batch) that stays on the device. */
int ss_mlp_set_data(ss_mlp* net, const float* x, const float* y, int64_t rows);
/* `steps` Adam steps (beta 0.9 / 0.999) on shuffled batches of the training
 * set, learning rate on a cosine from lr_start to lr_end; losses (steps
 * values, may be NULL) receives each step's batch loss. */
int ss_mlp_train(ss_mlp* net, int64_t steps, float lr_start, float lr_end,
                 uint64_t seed, double* losses);
/* The surrogate's tensor-core product on its own, for verification:
 * c[M][N] = a[M][K] b[N][K]^T with a and b raw BF16 bit patterns, FP32
 * accumulation; M % 128 == 0, K % 64 == 0, N % 16 == 0 and N <= 256. */
int ss_mlp_gemm_test(ss_engine* engine, const uint16_t* a, const uint16_t* b,
                     int M, int N, int K, float* c);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* SPINSIM_B200_H */
