/*
 * pkde_b200 -- C ABI of the B200 (sm_100a) implementation of ParallelKDE.jl's
 * `:gradepro` grid estimator (the `device=:cuda` path).
 *
 * Plain C types only; no CUDA or torch types appear in the signatures.  A `stream`
 * argument is a `cudaStream_t` passed as `void*` (NULL = the legacy default stream).
 *
 * Layout conventions (those of the reference, ParallelKDE.jl):
 *   - samples: N x n, column-major (the N coordinates of one sample are contiguous);
 *   - grid arrays: column-major, grid axis 1 fastest; G = prod(dims);
 *   - bootstrap indices: n x B, column-major, 1-based (like `rand(1:n, n, B)`).
 *
 * Error handling: every entry point returns a pkde_status; on failure the message is
 * available from pkde_last_error(ctx).  PKDE_EINVAL corresponds to the reference's
 * ArgumentError.  Calls on one context are not reentrant (one host thread at a time).
 */
#ifndef PKDE_B200_H
#define PKDE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pkde_status {
  PKDE_OK = 0,
  PKDE_EINVAL = 1,      /* invalid argument; data beyond the grid (ArgumentError) */
  PKDE_ENOMEM = 2,      /* device allocation failed */
  PKDE_ECUDA = 3,       /* CUDA runtime error */
  PKDE_EUNSUPPORTED = 4, /* valid request this build does not handle */
  PKDE_ETIMEDOUT = 5     /* pkde_wait: the request is not done within the timeout */
} pkde_status;

/* flags for the pointer arguments */
#define PKDE_DEVICE_INPUT 1u  /* data / indices / input arrays are device pointers */
#define PKDE_DEVICE_OUTPUT 2u /* output arrays are device pointers */

typedef struct pkde_ctx pkde_ctx;

/* Uniform grid, one entry per axis (axis 1 first).  Mirrors Grid/CuGrid
 * (src/Grids/Grids.jl:67-134): lo/hi are the extrema of the coordinate range
 * (low_bounds/high_bounds, :203-210), h the step (spacings, :189). */
typedef struct pkde_grid {
  int32_t ndim; /* 1..4 */
  int32_t reserved;
  int64_t dims[4];
  double lo[4];
  double hi[4];
  double h[4];
} pkde_grid;

/* Keyword arguments of estimate_density!(est, :gradepro; ...)
 * (docs/src/estimators/gradepro.md:19-28, src/DensityEstimators/GradeProEstimator.jl:700-858).
 * NaN selects the reference default. */
typedef struct pkde_gradepro_params {
  pkde_grid grid;
  int32_t n_bootstraps; /* B >= 2 (default 100, GradeProEstimator.jl:705) */
  int32_t n_steps;      /* > 0: S = n_steps + 1 bandwidths; 0: use bw_step, else 250 */
  double bw_step;       /* bandwidth step (all axes); NaN: unused */
  double bw_final[4];   /* final bandwidth per axis; NaN: Silverman's rule */
  double alpha_s;       /* NaN: 0.0 for 1-D, 0.06 otherwise */
  double alpha_os;      /* NaN: 0.1 */
  double eps;           /* NaN: 2.0 for 1-D, -0.5 otherwise */
} pkde_gradepro_params;

/* Context: owns the device state and scratch of one GPU.
 * Replaces the device set-up of initialize_estimation (src/ParallelKDE.jl:102-158). */
int pkde_create(pkde_ctx **ctx, int device);
int pkde_destroy(pkde_ctx *ctx);
const char *pkde_last_error(const pkde_ctx *ctx);
const char *pkde_version(void);

/* Fill `p` with the reference defaults for an `ndim`-dimensional grid (grid left zeroed). */
int pkde_gradepro_default_params(pkde_gradepro_params *p, int32_t ndim);

/* The hot path: estimate_density!(est, :gradepro; kwargs...) for one sample set.
 * Replaces src/DensityEstimators/DensityEstimators.jl:58-84 (estimate!(::Symbol, kde))
 * -> GradeProEstimator.jl:700-858 (initialize_estimator) -> :968-1051 (estimate!)
 * -> :1053-1072 (replace_nans!) on the CUDA device.
 *   data        : N x n samples (FP64)
 *   boot_idx    : n x B 1-based bootstrap draws, or NULL to draw them from `seed`
 *                 with the counter-based generator documented in pkde_boot_index
 *   density_out : G densities (FP64, column-major grid order)
 *   selected_out: G int32, the 0-based bandwidth step whose means were kept per grid
 *                 point, or S when replace_nans! filled the point (may be NULL)
 * Samples on or beyond the grid bounds give PKDE_EINVAL with the reference's message
 * (DirectSpace.jl:479-512). */
int pkde_gradepro_estimate(pkde_ctx *ctx, const pkde_gradepro_params *p, const double *data,
                           int64_t n, const int32_t *boot_idx, uint64_t seed, double *density_out,
                           int32_t *selected_out, uint32_t flags, void *stream);

/* Several independent estimations in one call (the batched form of
 * pkde_gradepro_estimate; no counterpart in the reference, whose API estimates one
 * sample set per call).  Arrays of `count` entries: params[e], data[e] (N_e x n[e]),
 * boot_idx[e] (or boot_idx == NULL / boot_idx[e] == NULL: seeded draws from seeds[e]),
 * density_out[e] (G_e FP64), selected_out[e] (G_e int32, or selected_out == NULL /
 * selected_out[e] == NULL).  Grids, dimensions (1..4), sample and bootstrap counts may
 * all differ.  Every phase runs for all estimations before the next (one host read-back
 * per phase for the whole call) and the bandwidth steps of all N-D power-of-two
 * estimations share one persistent launch.  Each estimation's results are identical to
 * what pkde_gradepro_estimate gives for it alone.  An invalid estimation fails the call
 * (the message names its index). */
int pkde_gradepro_estimate_batch(pkde_ctx *ctx, int32_t count, const pkde_gradepro_params *params,
                                 const double *const *data, const int64_t *n, const int32_t *const *boot_idx,
                                 const uint64_t *seeds, double *const *density_out, int32_t *const *selected_out,
                                 uint32_t flags, void *stream);

/* The :rot estimator (rule-of-thumb bandwidth), estimate!(::AbstractRoTEstimator, kde)
 * on the CUDA device: RoTEstimator.jl:117-148 (initialize_estimator, initialize_density),
 * :150-201 (estimate!, propagate_kernels!, ifft_density!), :24-49 (the rules).
 *   rule        : PKDE_ROT_SCOTT (n^(-1/(N+4)), the reference's default) or
 *                 PKDE_ROT_SILVERMAN ((n (N+2)/4)^(-1/(N+4))), times the per-axis
 *                 standard deviations; the kernel is propagated by that time - h/2
 *   data        : N x n samples (FP64);  density_out: G FP64 (|inverse FFT|)
 * Same errors as pkde_gradepro_estimate; an unknown rule gives PKDE_EINVAL
 * ("Rule of thumb ... not implemented."). */
#define PKDE_ROT_SCOTT 0
#define PKDE_ROT_SILVERMAN 1
int pkde_rot_estimate(pkde_ctx *ctx, const pkde_grid *grid, int32_t rule, const double *data, int64_t n,
                      double *density_out, uint32_t flags, void *stream);

/* Serving: asynchronous :gradepro requests with continuous batching (no counterpart in
 * the reference, whose estimate_density! blocks).  Submitted requests queue on the
 * context; `lanes` worker threads, each with its own stream and device buffers, take
 * the queued requests in arrival order as a wave (as many as fit the per-lane memory
 * budget, at least one) and run the wave as one pkde_gradepro_estimate_batch call.
 * While one lane's wave is on the GPU, the next arrivals start on another lane, so
 * their work overlaps on the device.  A request's results are identical to what
 * pkde_gradepro_estimate gives for it alone.  Inputs and outputs are host pointers
 * owned by the caller, who keeps them valid until pkde_wait has returned the request.
 * submit/wait are thread-safe; pkde_destroy finishes the queued requests first. */
typedef struct pkde_request {
  pkde_gradepro_params params;
  const double *data;      /* N x n samples (host) */
  int64_t n;
  const int32_t *boot_idx; /* n x B 1-based draws (host), or NULL: seeded draws */
  uint64_t seed;
  double *density_out;     /* G (host) */
  int32_t *selected_out;   /* G (host), or NULL */
} pkde_request;

typedef struct pkde_result {
  int32_t status;          /* pkde_status of this request */
  int32_t batch_size;      /* requests in the wave it ran in */
  double queue_ms;         /* submit -> start of its wave */
  double run_ms;           /* start of its wave -> done */
  double total_ms;         /* submit -> done */
  char message[256];       /* error message when status != PKDE_OK */
} pkde_result;

/* Lanes (1..8, default 2) and per-lane memory budget in bytes (0: 80 % of the free
 * device memory divided by the lanes); only before the first pkde_submit. */
int pkde_serve_config(pkde_ctx *ctx, int32_t lanes, int64_t lane_memory_bytes);
/* Queue one request; returns its ticket.  Parameter errors are reported here (and the
 * request is not queued); data errors (samples beyond the grid) in its result. */
int pkde_submit(pkde_ctx *ctx, const pkde_request *req, uint64_t *ticket);
/* Wait for a request (timeout_ms < 0: no limit).  PKDE_OK: `out` holds its result and
 * the ticket is released; PKDE_ETIMEDOUT: not done yet; PKDE_EINVAL: unknown ticket. */
int pkde_wait(pkde_ctx *ctx, uint64_t ticket, int32_t timeout_ms, pkde_result *out);

/* find_grid (src/Grids/Grids.jl:252-300) from samples that may already be on the
 * device: per-axis extrema reduced on the GPU (no copy of the samples to the host), then
 * the reference's arithmetic: padding = 0.1 |max - min| unless given, bounds extended by
 * the padding, n_i = dims[i] (NULL and steps NULL: 150 per axis) or, with steps,
 * floor((hi - lo)/step) + 1 points of that step; h = (hi - lo)/(n - 1) rounded once
 * (Julia's range(lo, stop=hi, length=n)).  data: N x n; flags PKDE_DEVICE_INPUT. */
int pkde_find_grid(pkde_ctx *ctx, int32_t ndim, const double *data, int64_t n, const int64_t *dims,
                   const double *steps, const double *padding, pkde_grid *out, uint32_t flags, void *stream);

/* get_density(est; normalize=true) (src/ParallelKDE.jl:189-202): density /= sum(density)
 * * dx with the sum in FP64 on the device (dx = prod(spacings(grid)), or the caller's
 * dx).  In place; flags PKDE_DEVICE_INPUT: `density` is a device pointer.  dx <= 0 gives
 * PKDE_EINVAL ("Normalization requires a grid or dx to be specified."). */
int pkde_normalize_density(pkde_ctx *ctx, double *density, int64_t G, double dx, uint32_t flags, void *stream);

/* Dirac-sequence binning of bootstrap resamples onto the grid.
 * Replaces initialize_dirac_sequence(Val(:cuda), ...) (DirectSpace.jl:289-362) and its
 * kernel generate_dirac_cuda! (:364-477), following the CPU arithmetic (:196-287).
 *   means_out : G x B FP64 (sum of corner weights per cell)       (may be NULL)
 *   sq_out    : G x B FP64 (sum of squared corner weights)        (may be NULL)
 *   counts_out: G x B uint32, draws whose lower cell is the cell  (may be NULL)
 * boot_idx NULL with nboot == 0 bins the identity resample (all samples once). */
int pkde_dirac_sequence(pkde_ctx *ctx, const pkde_grid *grid, const double *data, int64_t n,
                        const int32_t *boot_idx, int32_t nboot, uint64_t seed, double *means_out,
                        double *sq_out, uint32_t *counts_out, uint32_t flags, void *stream);

/* pkde_dirac_sequence without any device allocation.  No counterpart in the reference.
 * For callers that cannot allocate device memory: a host framework whose caching
 * allocator owns the GPU's memory, or a caller that must not make cudaMalloc/cudaFree
 * calls, which synchronise the whole device and so stall every other stream.  The call
 * does not allocate, but it is not asynchronous: it synchronises `stream` twice (once
 * to read back the error flags and the largest cell count, once at its end), so the
 * calling host thread blocks until the binning has finished.  All pointers are device
 * pointers (means_out required; sq_out, counts_out optional).  Scratch is one fixed
 * array inside the library (about 9 MB, held by every GPU that loads the library until
 * exit): at most 16384 samples per call, and when counts_out is NULL at most 2^20
 * resample x grid-point counters.  Larger requests return PKDE_EINVAL.  The work runs
 * on the device that owns `stream` (for the legacy default stream, NULL: the calling
 * thread's current device); the pointers must belong to that device.  The first call on
 * a device looks up the array's device address (once per device).  Calls share the
 * array: calls whose work overlaps on the GPU race; order them on one stream.  ctx may
 * be NULL: the error message is then kept for pkde_last_error(NULL) (per thread). */
int pkde_dirac_sequence_noalloc(pkde_ctx *ctx, const pkde_grid *grid, const double *data, int64_t n,
                                const int32_t *boot_idx, int32_t nboot, uint64_t seed, double *means_out,
                                double *sq_out, uint32_t *counts_out, void *stream);

/* N-D complex FFT of `batch` arrays of G complex values (interleaved re, im FP64).
 * direction -1: forward, unnormalised (fourier_statistics!, FourierSpace.jl:25-104);
 * direction +1: inverse scaled by 1/G (ifourier_statistics!, FourierSpace.jl:445-524). */
int pkde_fft(pkde_ctx *ctx, int32_t ndim, const int64_t *dims, double *data, int32_t batch,
             int32_t direction, uint32_t flags, void *stream);

/* Scaled variance-to-mean ratio of B bootstrap means/second-moment arrays
 * (complex, G x B): calculate_scaled_vmr! (DirectSpace.jl:526-740).
 * vmr_out: G values log(prod(t^2+t0^2)^(3/2) n^3 var_b(vmr)) or NaN. */
int pkde_scaled_vmr(pkde_ctx *ctx, int64_t G, int32_t nboot, const double *means,
                    const double *sq, int32_t ndim, const double *t, const double *t0,
                    int64_t n_samples, double *vmr_out, uint32_t flags, void *stream);

/* One convergence update per grid point: identify_convergence! / find_stability
 * (DirectSpace.jl:829-1100).  All arrays have G entries and are updated in place;
 * `flags` bit PKDE_DEVICE_INPUT says they are device pointers. */
int pkde_identify_convergence(pkde_ctx *ctx, int64_t G, double *density, const double *means,
                              const double *vmr_current, const double *vmr_prev1,
                              const double *vmr_prev2, double dlogt, double eps, int64_t steps_low,
                              int64_t steps_over, double *minima, uint16_t *counters_low,
                              uint16_t *counters_over, uint8_t *low_density_flags, uint32_t flags,
                              void *stream);

/* How the bandwidth steps of an estimation are executed (a context setting).
 *   PKDE_STEPS_AUTO          : the persistent step engine for N-D grids with axes of
 *                              2..2048 points, one CTA per bandwidth step for 1-D
 *                              power-of-two grids of 256..4096 points, else per-step
 *                              kernel launches;
 *   PKDE_STEPS_PER_STEP_LAUNCH: every estimation on the plain form -- per bandwidth step
 *                              and pair group, one kernel launch per FFT axis, then the
 *                              VMR and the means/convergence launches, estimations one
 *                              after another.  This mirrors the reference's CUDA path
 *                              (GradeProEstimator.jl:968-1051: propagate, ifft, VMR,
 *                              means, convergence per step) and is the comparator of the
 *                              batched form; results agree with AUTO to FP64 round-off.
 * No counterpart in the reference. */
#define PKDE_STEPS_AUTO 0
#define PKDE_STEPS_PER_STEP_LAUNCH 1
int pkde_set_step_path(pkde_ctx *ctx, int path);

/* Autotuning of the step engine's schedule per shape (grid dimensions and bootstrap
 * pairs): the first estimation of a new shape times trial runs over its first 16
 * bandwidth steps for ring-slot sizes 8..64 MB, slots holding half or all of the
 * bootstrap pairs where those are larger (while the ring stays within an eighth of the
 * free device memory; the context keeps the largest ring it tried), 1..8 tiles per
 * work item and pipeline delays 2..4, and keeps the fastest for the context (and, when
 * the environment variable PKDE_TUNE_CACHE names a file, appends it there and reads it
 * back in later processes).  A batch whose tuned rings together would not fit in half
 * of the free memory runs with slots of at most 64 MB.  The schedule never changes
 * results, only time.  On by default; 0 uses the fixed defaults (32 MB, 2 or 8 tiles,
 * delay 2).  No counterpart in the reference. */
int pkde_set_autotune(pkde_ctx *ctx, int enable);

/* Failure detection of the step engine.  Every dependency wait of the persistent
 * step engine (a work item waiting for the items it reads from) polls a counter at most
 * `polls` times (about 0.1 us each) before it gives up: it then sets the launch's error
 * flag, every CTA leaves, and the call returns PKDE_ECUDA ("step engine: a dependency
 * wait timed out").  The context stays usable.  Default 20,000,000 (about 1-2 s);
 * polls >= 0 (0: give up at the first check that finds the dependency not ready).
 * No counterpart in the reference, which has no waits that can time out (its
 * failures are ArgumentErrors, DirectSpace.jl:479-512). */
int pkde_set_wait_limit(pkde_ctx *ctx, int64_t polls);

/* Host-side fault injection, for tests of the error paths (no device fault is ever
 * made).  The next call that reaches the armed point throws a host error there and
 * returns PKDE_ECUDA ("injected host fault"); the point then disarms itself.
 *   PKDE_FAULT_AFTER_BINNING: in pkde_gradepro_estimate(_batch), after the binning
 *   of every estimation and the copy of its error flags have been queued, before the
 *   forward transforms -- the call fails with device work in flight and flags
 *   outstanding, which the context's next call must wait for and discard.
 * No counterpart in the reference. */
#define PKDE_FAULT_NONE 0
#define PKDE_FAULT_AFTER_BINNING 1
int pkde_set_fault(pkde_ctx *ctx, int32_t point);

/* Diagnostic: out[i] = num[i] / den[i] with the quotient the step engine uses for the
 * variance-to-mean ratio (a refined hardware reciprocal estimate instead of the IEEE
 * division subroutine), so that tests can compare it with IEEE division.  Device
 * pointers with PKDE_DEVICE_INPUT, else host pointers.  No counterpart in the reference
 * (whose quotient is the IEEE one, DirectSpace.jl:550-552). */
int pkde_diag_divide(pkde_ctx *ctx, const double *num, const double *den, double *out, int64_t n, uint32_t flags,
                     void *stream);

/* Launch accounting and per-phase device time, for tracing and the roofline report.
 * No counterpart in the reference, which has no tracing.
 * pkde_set_profiling levels: PKDE_PROFILE_ALL brackets every kernel the context
 * launches with CUDA events on its stream and adds its elapsed time to its phase when
 * the call synchronises; PKDE_PROFILE_STEPS brackets only the bandwidth-step phases
 * (2..4), two events per step-engine launch, so that timing a whole call is not
 * slowed by events between short launches; PKDE_PROFILE_OFF brackets nothing.  Launch
 * counts are kept at every level.  Other levels return PKDE_EINVAL. */
#define PKDE_PROFILE_OFF 0
#define PKDE_PROFILE_ALL 1
#define PKDE_PROFILE_STEPS 2
#define PKDE_NPHASES 6
typedef enum pkde_phase {
  PKDE_PHASE_BINNING = 0,      /* binning + fixed-point conversion */
  PKDE_PHASE_FORWARD_FFT = 1,  /* forward transforms, once per estimation */
  PKDE_PHASE_STEP_FFT = 2,     /* per-bandwidth-step inverse FFT passes (axes N..2) */
  PKDE_PHASE_STEP_VMR = 3,     /* per-step fused axis-1 inverse FFT + VMR + bootstrap variance */
  PKDE_PHASE_STEP_MEANS = 4,   /* per-step means + convergence update */
  PKDE_PHASE_OTHER = 5         /* moments, state init, replace_nans */
} pkde_phase;

typedef struct pkde_stats {
  uint64_t launches;                  /* kernels launched since the last reset */
  uint64_t phase_launches[PKDE_NPHASES];
  double phase_ms[PKDE_NPHASES];      /* device time per phase (profiling enabled only) */
} pkde_stats;

int pkde_set_profiling(pkde_ctx *ctx, int enable);
int pkde_get_stats(pkde_ctx *ctx, pkde_stats *out, int reset);

/* Counter-based bootstrap draw used when boot_idx is NULL (0-based result):
 *   x = seed + (b*n + j + 1) * 0x9E3779B97F4A7C15 (mod 2^64), z = splitmix64(x),
 *   idx = ((z >> 32) * n) >> 32.
 * No counterpart in the reference, whose Julia RNG streams are not reproducible
 * outside Julia (src/KDEs/KDEs.jl:182-206). */
int64_t pkde_boot_index(uint64_t seed, int64_t n, int64_t b, int64_t j);

#ifdef __cplusplus
}
#endif

#endif /* PKDE_B200_H */
