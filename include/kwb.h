/*
 * kwb.h -- C ABI of libkwb, the B200 (sm_100a) implementation of KWave.jl's fluid k-space
 * time-stepping path.
 *
 * The reference has no FFI on this path: its boundary is the Julia generic function
 *
 *   kspace_first_order(kgrid::KWaveGrid{1,2,3}D, medium::KWaveMedium, source::KWaveSource,
 *                      sensor::KWaveSensor; pml_size, pml_alpha, smooth_p0, data_cast, ...)
 *       -> SimulationOutput                      (KWave.jl/src/solver/first_order.jl:92-111,
 *                                                 287-306, 505-524; sensor.jl:76-82)
 *
 * A Julia shim (ccall) or any other host builds one kwb_problem from those four structs and
 * the keyword arguments and calls kwb_solve().  The same problem struct also carries the
 * axisymmetric solver (kspace_first_order_as, solver/axisymmetric.jl:26-227; the axisymmetric
 * flag) and the elastic solvers (pstd_elastic_2d / pstd_elastic_3d, solver/elastic.jl:133-588;
 * the elastic flag and fields).  Everything here is plain C: host pointers,
 * 64-bit sizes, FP64 inputs and outputs, negative status codes instead of exceptions.
 *
 * Array convention: every grid-shaped input is FP64 in the reference's column-major order
 * (x fastest), i.e. Julia's linear indexing; every mask is given as the sorted 0-based linear
 * indices that Julia's findall(mask) returns (minus one).
 */
#ifndef KWB_H
#define KWB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KWB_VERSION 10000 /* 1.0.0 */

/* Status codes.  The reference raises ErrorException (first_order.jl:117, 312, 530;
 * sensor.jl:55); here every such error is a negative code plus kwb_last_error(). */
enum kwb_status {
  KWB_OK = 0,
  KWB_E_INVALID = -1,     /* malformed problem (the reference's error(...) / BoundsError cases) */
  KWB_E_UNSUPPORTED = -2, /* valid for the reference but outside this library (a grid side above 4096, or
                             above 2048 with a prime factor > 7) */
  KWB_E_NOMEM = -3,       /* device memory admission failed */
  KWB_E_DEVICE = -4,      /* CUDA error or a device-side bounded wait that gave up */
  KWB_E_TIMEOUT = -5,     /* kwb_wait() deadline passed */
  KWB_E_CANCELLED = -6,   /* request cancelled by kwb_cancel() */
  KWB_E_BUSY = -7,        /* request still running */
  KWB_E_NOTFOUND = -8     /* unknown ticket */
};

/* medium.jl:62-66 alpha_mode */
enum kwb_alpha_mode { KWB_NO_ABSORPTION = 0, KWB_NO_DISPERSION = 1, KWB_STOKES = 2 };

/* types.jl:11 SourceMode */
enum kwb_source_mode { KWB_DIRICHLET = 0, KWB_ADDITIVE = 1, KWB_ADDITIVE_NO_CORRECTION = 2 };

/* sensor.jl:41-45 VALID_RECORD_FIELDS, one bit each */
enum kwb_record {
  KWB_REC_P = 0, KWB_REC_P_MAX = 1, KWB_REC_P_MIN = 2, KWB_REC_P_RMS = 3, KWB_REC_P_FINAL = 4,
  KWB_REC_UX = 5, KWB_REC_UY = 6, KWB_REC_UZ = 7, KWB_REC_U_MAX = 8, KWB_REC_U_RMS = 9,
  KWB_REC_U_FINAL = 10, KWB_REC_I_AVG = 11, KWB_REC_I_MAX = 12, KWB_REC_COUNT = 13
};

/* A medium property: count 0 = absent (`nothing`), 1 = scalar, N = per voxel (column-major). */
typedef struct kwb_field {
  const double *data;
  int64_t count;
} kwb_field;

/* A time-varying source signal, column-major n_rows x n_cols: element (j, t) at j + n_rows*t.
 * Column t_index (1-based) is min(t_index, n_cols), so a short signal holds its last column
 * (first_order_steps.jl:548, 567, 593, 625, 698). */
typedef struct kwb_signal {
  const double *data; /* NULL = this component is `nothing` */
  int64_t n_rows;     /* must be >= the number of mask points */
  int64_t n_cols;
} kwb_signal;

/* One set of sensor points with the fields recorded on them.  A reference KWaveSensor maps to
 * exactly one group; more groups let one solve record different fields on different masks. */
typedef struct kwb_sensor_group {
  const int64_t *index;  /* sorted 0-based column-major linear indices (findall(mask) - 1) */
  int64_t n_index;       /* number of points (for a Cartesian mask: its number of columns) */
  int32_t dense;         /* 1: every voxel in linear order; index may be NULL */
  int32_t cartesian;     /* 1: Cartesian (Float64 matrix) mask -- outputs are allocated but never
                            filled, as in first_order.jl:417-421 */
  uint32_t record_mask;  /* OR of (1u << kwb_record) */
  uint8_t record_count[KWB_REC_COUNT]; /* times each field appears in sensor.record; the running
                            sums of p_rms, u_rms and I_avg are added that many times per step
                            (record_sensor_data! loops over the record list) */
  /* Post-loop filters of this group's pressure series, the reference's
   * apply_sensor_directivity! and apply_frequency_response! (first_order_steps.jl:836-910),
   * applied on the device before read-back (fluid solvers; the elastic solvers have none).
   * Each replaces p_j by real(ifft(fft(p_j) .* H)) along time, directivity first:
   *   directivity_angle != NULL: H = sinc(2 pi |f| / d_min * directivity_size * sin(theta_j) / 2),
   *     theta_j = directivity_angle[0] for every point (n_directivity_angle == 1) or
   *     directivity_angle[j] (n_directivity_angle >= the number of points); points whose angle
   *     is exactly 0 are not filtered by it; d_min = dx (1-D) or the smallest grid spacing;
   *   has_frequency_response != 0: H = exp(-(|f| - frequency_center)^2 / (2 frequency_bandwidth^2)).
   * f = fftfreq(Nt, 1/dt).  Only the "p" series is filtered, as in the reference. */
  const double *directivity_angle;
  int64_t n_directivity_angle;
  double directivity_size;
  int32_t has_frequency_response;
  double frequency_center;
  double frequency_bandwidth;
} kwb_sensor_group;

/* Optional per-step callback, the reference's progress_callback(t_index, Nt, p)
 * (first_order.jl:479-481): p is the full FP32 pressure field in column-major order.  Setting
 * it copies p to the host every step (slow path). */
typedef void (*kwb_progress_fn)(int64_t t_index, int64_t Nt, const float *p, void *user);

typedef struct kwb_problem {
  int32_t ndim;          /* 1, 2 or 3 */
  int64_t N[3];          /* Nx, Ny, Nz (unused entries 1) */
  double d[3];           /* dx, dy, dz [m] */
  double dt;             /* kgrid.dt[] */
  int64_t Nt;            /* kgrid.Nt[] */
  int64_t pml_size[3];   /* per axis, pml_size normalised as first_order.jl:322, 540 */
  double pml_alpha[3];

  kwb_field c0;          /* medium.sound_speed (scalar or array) */
  kwb_field rho0;        /* medium.density     (scalar or array) */
  kwb_field BonA;        /* medium.BonA        (absent, scalar or array) */
  int32_t alpha_mode;    /* kwb_alpha_mode; KWB_NO_ABSORPTION when alpha_coeff is nothing */
  double alpha_coeff;    /* dB/(MHz^y cm), scalar only (an array raises in the reference) */
  double alpha_power;    /* y */

  kwb_field p0;          /* initial pressure, already smoothed by the caller when smooth_p0
                            (filter/filters.jl:20-60); count 0 = no p0 */

  const int64_t *p_index; int64_t n_p_index; int32_t p_mode; kwb_signal p_signal;
  const int64_t *u_index; int64_t n_u_index; int32_t u_mode; kwb_signal u_signal[3];

  /* time reversal: sensor.time_reversal_boundary_data, n_rows x n_cols column-major; injected
   * at sensor group 0's points (first_order.jl:428-460, 654-689).  data NULL = off. */
  kwb_signal tr;

  int32_t n_groups;
  const kwb_sensor_group *groups;

  kwb_progress_fn progress; void *progress_user;

  /* Memory order of the grid-shaped arrays (c0, rho0, BonA, p0): 0 = column-major, the
   * reference's Julia order (x fastest); 1 = row-major, NumPy's default (the last axis
   * fastest).  Row-major arrays are uploaded as they are and reordered on the device.  Index
   * lists (p_index, u_index, sensor indices) are column-major linear indices either way. */
  int32_t row_major;

  /* 1: the axisymmetric solver, kspace_first_order_as (solver/axisymmetric.jl:26-227): ndim 2,
   * x axial, y radial; the radial density update adds u_r / r to the divergence, r = |y_vec|
   * with r = 0 replaced by dy/2.  Time-reversal data is not accepted with it. */
  int32_t axisymmetric;

  /* 1: the elastic stress-velocity solver, pstd_elastic_2d / pstd_elastic_3d
   * (solver/elastic.jl:133-366, 386-588); ndim 2 or 3.  c0 holds sound_speed_compression, cs
   * sound_speed_shear and rho0 the density (an array density when either speed is an array:
   * with a scalar density the reference squares an array speed as a matrix, elastic.jl:169).
   * alpha_mode != KWB_NO_ABSORPTION carries alpha_coeff_compression in alpha_coeff (with
   * alpha_power); has_alpha_shear / alpha_coeff_shear the shear coefficient.  p0 sets every normal
   * stress to -p0 (not smoothed); the velocity source is u_*; s_* are the stress sources.  BonA,
   * pressure sources, time reversal and the axisymmetric flag are not part of it. */
  int32_t elastic;
  kwb_field cs;
  int32_t has_alpha_shear;
  double alpha_coeff_shear;
  const int64_t *s_index; int64_t n_s_index; int32_t s_mode;
  kwb_signal s_signal[6]; /* sxx, syy, szz, sxy, sxz, syz (2D: sxx, syy, sxy; szz/sxz/syz unused) */
} kwb_problem;

/* Output sizes of one group: rows x cols per field, 0 x 0 when the field is not recorded. */
typedef struct kwb_group_sizes {
  int64_t rows[KWB_REC_COUNT];
  int64_t cols[KWB_REC_COUNT];
} kwb_group_sizes;

/* Caller-allocated FP64 output buffers, column-major like the reference's Dict values
 * (sensor.jl:109-133).  NULL skips a field. */
typedef struct kwb_group_outputs {
  double *field[KWB_REC_COUNT];
} kwb_group_outputs;

typedef struct kwb_outputs {
  kwb_group_outputs *groups;  /* n_groups entries */
  double *p_final_full;       /* time-reversal mode: full-field p_final (N voxels), first_order.jl:491-494 */
} kwb_outputs;

typedef struct kwb_ctx kwb_ctx;
typedef struct kwb_sim kwb_sim;

/* ---- library / context ------------------------------------------------------------------ */
int kwb_version(void);
/* Create a context bound to CUDA device `device` (one host thread at a time per context). */
int kwb_context_create(int device, kwb_ctx **out);
void kwb_context_destroy(kwb_ctx *ctx);
/* Message of the last error on this context (or of the last failed kwb_context_create when
 * ctx is NULL).  Valid until the next call on the context. */
const char *kwb_last_error(const kwb_ctx *ctx);

/* ---- blocking solve: the kspace_first_order replacement --------------------------------- */
/* Sizes of every output of `problem` (n_groups entries in `sizes`); *p_final_full_len is N in
 * time-reversal mode and 0 otherwise. */
int kwb_query_outputs(kwb_ctx *ctx, const kwb_problem *problem, kwb_group_sizes *sizes,
                      int64_t *p_final_full_len);
/* Run the whole simulation (first_order.jl:92-728) and fill `outputs`. */
int kwb_solve(kwb_ctx *ctx, const kwb_problem *problem, kwb_outputs *outputs);

/* ---- resident simulation: the same solve split into phases ------------------------------ */
/* Validate, admit by free device memory, upload the medium/sources, build the FP64 operator
 * tables on the device and apply the p0 initialisation.  Nothing is stepped yet. */
int kwb_sim_create(kwb_ctx *ctx, const kwb_problem *problem, kwb_sim **out);
/* Enqueue `steps` time steps (clamped to the remaining Nt) on the simulation's stream;
 * returns without waiting. */
int kwb_sim_advance(kwb_sim *sim, int64_t steps);
/* Enqueue `steps` steps and time them with CUDA events on the simulation's stream; blocks and
 * writes the device time in milliseconds. */
int kwb_sim_advance_timed(kwb_sim *sim, int64_t steps, double *device_ms);
/* Steps done so far. */
int64_t kwb_sim_steps_done(const kwb_sim *sim);
/* Block until the simulation's queued work is complete. */
int kwb_sim_sync(kwb_sim *sim);
/* Finalize (p_rms/u_rms square roots, directivity-free outputs) and copy all recorded outputs
 * to the caller's FP64 buffers.  Blocks. */
int kwb_sim_read_outputs(kwb_sim *sim, kwb_outputs *outputs);
/* Run the remaining steps and read all outputs (kwb_sim_advance to Nt, then
 * kwb_sim_read_outputs), copying the recorded time series to the caller's buffers block by
 * block while later steps run, so that only the last block's rows and the aggregates are read
 * after the loop.  kwb_solve is kwb_sim_create + kwb_sim_finish + kwb_sim_destroy.  Blocks.
 * (No reference counterpart of its own: the reference's loop returns its outputs at the end,
 * KWave.jl/src/solver/first_order.jl:448-484.) */
int kwb_sim_finish(kwb_sim *sim, kwb_outputs *outputs);
/* Copy the current FP32 pressure field (N voxels, column-major) to host memory.  Blocks. */
int kwb_sim_read_pressure(kwb_sim *sim, float *p_host);
void kwb_sim_destroy(kwb_sim *sim);

/* Per-kernel device time of `steps` eagerly launched steps, each launch bracketed by CUDA
 * events on the simulation's stream (a profiling aid; slower than kwb_sim_advance). */
typedef struct kwb_kernel_times {
  int32_t n;                 /* number of kernel kinds filled */
  char name[16][32];
  double total_ms[16];
  int64_t launches[16];
  double bytes_per_launch[16];  /* algorithmic bytes one launch moves (operand reads + writes) */
} kwb_kernel_times;
int kwb_sim_profile(kwb_sim *sim, int64_t steps, kwb_kernel_times *out);

/* The FFT schedule the simulation's time step runs with, as text: where it came from ("tuned"
 * on first use of the grid shape, "cache" from an earlier measurement of it, or "heuristic"
 * when tuning is off), then the per-pass choices.  Measured schedules play the role of the
 * reference's FFTW.MEASURE plans (fft_utils.jl:59-60); they are cached per device and shape in
 * memory and in the file KWB_TUNE_CACHE (default $HOME/.cache/kwb/fft_schedules.txt; "none"
 * keeps no file).  KWB_TUNE=0 keeps the size heuristic. */
int kwb_sim_schedule(const kwb_sim *sim, char *buf, int64_t len);

/* Device bytes the simulation holds and kernels launched per time step. */
int kwb_sim_info(const kwb_sim *sim, int64_t *device_bytes, int32_t *launches_per_step);

/* Device bytes a simulation of `problem` would hold (what admission compares with free memory). */
int kwb_estimate_device_bytes(kwb_ctx *ctx, const kwb_problem *problem, int64_t *bytes);

/* ---- continuous batching: many independent simulations on one GPU ----------------------
 * No counterpart in the reference (its solver runs one simulation per call on the host).
 * Requests are admitted in submission order as slots and device memory allow, each admitted
 * simulation keeps its fields resident and advances in CUDA-graph chunks on its own stream, so
 * requests that arrive while others run overlap with them on the device.  `problem` (and every
 * array it points to) and `outputs` must stay valid until kwb_wait() has returned for the ticket.
 * The results are the same as kwb_solve's for the same problem. */
typedef struct kwb_request_info {
  int32_t status;                 /* the request's final status (KWB_OK, ...) */
  int64_t submit_ns, start_ns, end_ns; /* steady-clock times: submitted, admitted, completed */
  char error[256];
} kwb_request_info;

typedef struct kwb_serving_stats {
  int64_t submitted, admitted, completed, failed, cancelled, chunks, peak_running;
  int64_t queued, running, running_bytes;
} kwb_serving_stats;

/* Scheduler limits: at most `max_running` admitted simulations (default 64), `chunk_steps` time
 * steps per launch (default 32), and (if > 0) at most `mem_cap_bytes` of modelled device memory
 * in use. */
int kwb_serving_config(kwb_ctx *ctx, int32_t max_running, int32_t chunk_steps, int64_t mem_cap_bytes);
/* Admission by size: a queued request starts while the running simulations hold at most
 * `voxels` grid points in total (default 4 Mi), or when none is running; 0 removes the limit.
 * No counterpart in the reference (scheduling of many kspace_first_order calls). */
int kwb_serving_voxel_budget(kwb_ctx *ctx, int64_t voxels);
int kwb_submit(kwb_ctx *ctx, const kwb_problem *problem, kwb_outputs *outputs, uint64_t *ticket);
/* *done = 1 once the request has completed (successfully or not). */
int kwb_poll(kwb_ctx *ctx, uint64_t ticket, int32_t *done);
/* Wait up to timeout_ns (< 0: forever); returns the request's status or KWB_E_TIMEOUT.  After a
 * completed wait the ticket is released. */
int kwb_wait(kwb_ctx *ctx, uint64_t ticket, int64_t timeout_ns, kwb_request_info *info);
/* Ask a queued or running request to stop; it completes with KWB_E_CANCELLED. */
int kwb_cancel(kwb_ctx *ctx, uint64_t ticket);
int kwb_serving_stats_get(kwb_ctx *ctx, kwb_serving_stats *out);
/* Submit n problems together and wait for all; status[i] per problem, returns the first error. */
int kwb_solve_batch(kwb_ctx *ctx, int32_t n, const kwb_problem *const *problems,
                    kwb_outputs *const *outputs, int32_t *status);

/* ---- equation of state without device allocation ----------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc -- hosts that own
 * all device memory through their own pool and forbid hidden allocations, real-time loops that
 * must not allocate after start-up -- this computes one equation-of-state step,
 *   p = irfftn( M .* rfftn( [c0^2] rho_eff ) ),  rho_eff = rho (1 + Q rho),  rho = sum_d rho_d,
 *   M = [c0^2] kappa (1 + tau |k|^y) / (Nx Ny Nz)          (first_order_steps.jl:214-290 without
 *                                                           the :stokes dispersion branch)
 * with the same kernels as kwb_solve, from caller-owned device arrays (FP32, column-major):
 * rho[0..ndim-1], optional c0sq (c0^2 per voxel; NULL = scalar c0sq_scalar), optional nlq
 * (Q = BonA/(2 rho0) per voxel; NULL = nlq_scalar, used when nonlinear != 0), output p.
 * Its scratch (descriptor, twiddles, multiplier, half spectrum) is one static device array of
 * KWB_NOALLOC_SCRATCH_MIB MiB that every GPU loading libkwb holds until exit.  Limits: the half
 * spectrum (Nx/2+1)*Ny*Nz must not exceed KWB_NOALLOC_MAX_SPECTRUM (else KWB_E_UNSUPPORTED);
 * alpha_mode KWB_STOKES with scalar c0 (the dispersion branch) is rejected.  The work is queued on
 * `stream` (a cudaStream_t; NULL = legacy default stream) and the call returns without waiting.
 * The first call on a device looks up the array's device address; make that first call before
 * any stream capture.  All calls share the array: calls whose GPU work overlaps race on it and
 * must be serialised by the caller.  Errors: kwb_noalloc_last_error(). */
#define KWB_NOALLOC_SCRATCH_MIB 32
#define KWB_NOALLOC_MAX_SPECTRUM 2621440
int kwb_eos_pressure_noalloc(int device, int32_t ndim, const int64_t N[3], const double d[3],
                             double dt, double c_ref, int32_t alpha_mode, double alpha_coeff,
                             double alpha_power, const float *const rho[3], const float *c0sq,
                             float c0sq_scalar, const float *nlq, float nlq_scalar,
                             int32_t nonlinear, float *p, void *stream);
const char *kwb_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* KWB_H */
