// Internal device/host structures of libkwb (not part of the C ABI).
//
// Data layout in HBM (one simulation):
//   * real fields p, u_d, rho_d (FP32): [Nz][Ny][Nx], x fastest -- the reference's column-major
//     order, so a Julia linear index is a direct offset;
//   * EOS half spectrum (complex FP32): [Nz][Ny][n1], n1 = Nx/2 + 1 -- the shape of the
//     reference's rfft scratch (fft_utils.jl:178);
//   * medium (FP32): rho0, c0^2, Q = BonA/(2 rho0), each present only when it varies per voxel;
//   * operator tables (built in FP64 on the device, stored FP32): per-axis twiddles, gradient
//     multipliers i k e^{+-i k d/2}/N, PML deficits 1 - pml, and the EOS multiplier
//     M = [c^2] kappa (1 + nabla1) / (Nx Ny Nz) in the half-spectrum shape.
#pragma once
#include <string>
#include <utility>
#include <cuda.h>  // CUtensorMap (the tensor-map type only; the encoder is fetched at run time)
#include <cuda_runtime.h>
#include <stdint.h>

#define KWB_MAX_STAGES 16
#define KWB_THREADS 256
#define KWB_PASS_THREADS_MAX 1024  // Stockham passes on grids with few tiles (pass_threads)
#define KWB_MAX_N 4096
#define KWB_BLUESTEIN_MAX_N 2048  // Bluestein inner length 4096 at most: one line fits shared memory
#define KWB_CHUNK_STEPS 32  // time steps per replayed CUDA graph

// Programmatic dependent launch between the kernels of a time step.  Each step kernel is
// launched with kwb_launch, so its blocks may be dispatched while its predecessor finishes; its
// first statement waits for the predecessor to complete (every block, before any early return,
// so completion stays ordered along the stream), and it then lets its own successor be
// dispatched (which needs every block of this kernel to be resident already, so it never holds
// back this kernel's blocks).
#define KWB_STEP_KERNEL_PROLOGUE()                                  \
  do {                                                              \
    asm volatile("griddepcontrol.wait;\n" ::: "memory");            \
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); \
  } while (0)

// Stockham plan of a line of n points.  A length with a prime factor above 7 is transformed by
// Bluestein's algorithm (chirp z-transform): m > 0 is the power-of-two length of the inner
// transforms (m >= 2n - 1), the stages are m's, chirp[j] = exp(-i pi j^2 / n) (j < n) and
// chirp_ft = FFT_m(conj chirp, wrapped) / m; m == 0 for a direct transform.
// Division by a run-time constant d as a multiply and shift: n / d == (umulhi(n, mul) + n) >> shift
// for 0 <= n < 2^31 (mul = floor(2^32 (2^shift - d) / d) + 1, shift = ceil(log2 d)).
struct FastDiv {
  unsigned mul;
  unsigned shift;
};
inline FastDiv make_fastdiv(unsigned d) {
  unsigned s = 0;
  while ((1ull << s) < d) ++s;
  return FastDiv{(unsigned)(((1ull << 32) * ((1ull << s) - d)) / d + 1), s};
}
struct FftPlan {
  int n;
  int nstages;
  int radix[KWB_MAX_STAGES];
  int m;
  const float2 *chirp;
  const float2 *chirp_ft;
  // per stage: division by the butterflies per line (len / radix) and by the sub-transform
  // length so far (the product of the earlier radices)
  FastDiv div_nr[KWB_MAX_STAGES];
  FastDiv div_ns[KWB_MAX_STAGES];
};
// Length of the transforms a plan runs (the buffers and twiddle table of a line are this long).
__host__ __device__ inline int fft_len(const FftPlan &p) { return p.m > 0 ? p.m : p.n; }

// Pass slots of the FFT schedule: line passes per axis, the x equation-of-state passes, the
// y/z spectrum passes.
enum { KWB_SLOT_LINE0 = 0, KWB_SLOT_LINE1 = 1, KWB_SLOT_LINE2 = 2, KWB_SLOT_EOS_FWD = 3, KWB_SLOT_EOS_INV = 4,
       KWB_SLOT_SPEC1 = 5, KWB_SLOT_SPEC2 = 6, KWB_SLOT_PLANE = 7, KWB_NSLOTS = 8 };

// Line-pass modes.
enum { KWB_MODE_STEP = 0, KWB_MODE_INIT = 1 };
// Spectrum-pass operations.
enum { KWB_SPEC_FWD = 0, KWB_SPEC_FWD_MUL_INV = 1, KWB_SPEC_INV = 2 };

// One point source that lies on a line of an axis pass: line id, position along the line,
// source row j.
struct SrcEntry {
  int line;
  int pos;
  int j;
  int pad;
};

struct SimDev {
  int ndim;
  int N[3];
  int n1;
  long long nvox;
  long long nspec;
  float dt;
  float dt_over_rho0_s;  // dt / rho0 for scalar density
  float dt_rho0_s;       // dt * rho0 for scalar density
  int D;                 // number of split density components (= ndim)

  float *p;
  float *u[3];
  float *rho[3];
  float *rho_prev;  // dispersion only
  float2 *spec;
  float2 *spec2;    // dispersion only

  const float *rho0;  // nullptr: scalar density
  const float *c0sq;  // nullptr: scalar sound speed
  float c0sq_s;
  const float *nlq;   // nullptr: scalar Q (nlq_s)
  float nlq_s;
  int nonlinear;
  int dispersion;     // scalar c0 with :stokes absorption -> second spectrum
  int scalar_c;       // c^2 folded into M (scalar c0) vs applied per voxel
  const float *M;     // [Nz][Ny][n1]; plane pass: [n1][Nz][slot] or slot-major [n1][slot][z]
  const float *M2;    // dispersion multiplier, [Nz][Ny][n1]

  const float *pml_def[3];
  const float *pml_sg_def[3];
  const float2 *gpos[3];
  const float2 *gneg[3];
  const float2 *tw[3];
  FftPlan plan[3];

  // tile shapes: complex lines per tile for line passes (per axis), x-direction EOS passes and
  // spectrum passes (per axis); tiles per plane for each
  int L_line[3];
  int L_eosx;
  int L_spec[3];

  // sources
  int p_mode;
  int n_p;
  int p_cols;
  const float *p_sig;  // [col][j], already divided by D c^2 at the source point
  const int *p_line_ptr[3];
  const SrcEntry *p_entry[3];
  int u_mode;
  int n_u;
  int u_cols[3];
  const float *u_sig[3];  // [col][j], nullptr when the component is absent
  const int *u_line_ptr[3];
  const SrcEntry *u_entry[3];

  // time reversal
  int n_tr;
  const long long *tr_idx;
  const float *tr_sig;  // [col][j] already divided by D c^2

  long long Nt;
  const long long *t0;  // device step base (CUDA graph replays advance it)

  int fast;  // register-FFT kernels (kwb_fast.cu) for power-of-two lines: bit 0 line passes, bit 1 EOS passes

  // axisymmetric solver: 1/r along the radial (y) axis, added as u_r / r to the y divergence;
  // nullptr otherwise
  const float *inv_r;
  // 3-D equation of state with the y/z transforms in one cluster pass per kx plane: the half
  // spectrum is then [z][kx][y] and M is [kx][k_z][slot] (slot: register order of the pass's y
  // transform, fast_plane_slot_ky)
  int plane;
  // the x line pass ends with the equation of state's x R2C (no separate EOS forward pass)
  int fuse_xeos;

  // A dense (every-voxel) sensor group recording only pressure fields, updated by the x C2R
  // pass as it writes p (no separate gather); nullptr when there is none.
  const struct GroupDev *dense_p;
  // A sparse pressure-only sensor group also recorded by that pass (per-x-line index in
  // GroupDev::line_ptr / line_ent); nullptr when there is none.
  const struct GroupDev *sparse_p;

  // Device error word: kernels set bit 0 when a bounded wait gave up (a tile copy that did not
  // complete); the host reads it after synchronising and reports KWB_E_DEVICE.
  int *err;
  int test_drop_copy;  // test hook: the first CTA of a contiguous line pass drops its p-tile copy
  // Register line passes: tiles staged by TMA copies (1: bulk copies of contiguous rows, tiled
  // tensor copies of strided columns) or by 16-byte cp.async (0); tma_line[axis] is the measured
  // choice of each pass (-1: tile_tma, the default).
  int tile_tma;
  signed char tma_line[3];
  int eos_prefetch;    // the fused x pass prefetches its equation-of-state operands into L2
  int num_sms;        // multiprocessors of the device (tile sizing)
  int tile_override;  // register-FFT tile variant forced for every pass (-1: chosen per pass)
  // Measured FFT schedule (kwb_tune.cu): register-FFT tile variant per pass slot (KWB_SLOT_*;
  // -1: the size heuristic) and Stockham line-pass threads per CTA per axis (0: heuristic).
  // Lines per tile (L_*) and the Stockham radix order (plan) are the other tuned choices.
  signed char tile_var[8];
  short thr_line[3];
  signed char plan_order[3];  // make_plan_order's order of each axis's Stockham plan
  int grid_fill;      // Stockham passes of small grids: narrower tiles and larger CTAs to fill the GPU

  // Elastic solver (pstd_elastic_2d/3d).  u[d] are the velocities, p the recorded pressure
  // -trace(sigma)/D.  el_s: stresses in the slots xx, yy, zz, xy, xz, yz (2-D: 0, 1, 3).  el_w:
  // derivative scratch in the same slots -- first the velocity right-hand sides
  // sum_d d/dx_d sigma_dj in 0..D-1, then dv_d/dx_d in 0..2 and the shear sums
  // dv_i/dx_j + dv_j/dx_i in 3..5.
  int elastic;
  float *el_s[6];
  float *el_w[6];
  const float *el_lam, *el_mu;  // Lame parameters per voxel; nullptr: scalar (el_lam_s, el_mu_s)
  float el_lam_s, el_mu_s;
  float el_chi_p, el_chi_s;     // Kelvin-Voigt factors (2-D homogeneous medium only, else 0)
  int s_mode;
  int n_s;
  int s_cols[6];
  const float *s_sig[6];        // stress source tables [col][j]; nullptr when a component is absent
  const long long *s_idx;       // stress source points (column-major linear indices)
  const long long *u_idx;       // velocity source points (elastic solver)

  // Strided (y / z) register line passes: tensor maps of the staged fields (0 p, 1 rho0, 2 u_d,
  // 3 rho_d), each box 2L columns x tile_box_rows positions along the line, encoded by the host
  // for the launch that uses them (fast_line_pass); tile_tma_s = 0 stages by 16-byte cp.async.
  int tile_tma_s;
  int tile_box_rows;
  alignas(64) CUtensorMap tile_map[4];
};

// Stress slot of sigma_{dj}: the diagonal in 0..2, the pair {d, j} in 3..5 (xy, xz, yz).
__host__ __device__ inline int kwb_stress_slot(int d, int j) { return d == j ? d : 2 + d + j; }

// Launch a step kernel with programmatic stream serialization (see KWB_STEP_KERNEL_PROLOGUE).
template <typename... K, typename... A>
inline cudaError_t kwb_launch(void (*kern)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              A &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

// Sensor group on the device.
struct GroupDev {
  const long long *idx;  // nullptr when dense
  long long n;
  int dense;
  unsigned mask;
  int cnt_prms, cnt_urms, cnt_iavg;
  float *ser_p;
  float *ser_u[3];
  long long nt_alloc;
  float *pmax, *pmin, *pfinal;
  double *prms;
  double *umax, *urms, *ufinal, *iavg, *imax;
  // sparse groups recorded by the x C2R pass: points of x-line (y + Ny z) are entries
  // line_ptr[line] .. line_ptr[line+1]-1 of line_ent = {x, j}, sorted by x
  const int *line_ptr;
  const int2 *line_ent;
};

// Kernel launchers (kwb_kernels.cu).
namespace kwb {
// Let kernel fn take `bytes` of dynamic shared memory: raises its limit to the device's opt-in
// maximum less the kernel's own static shared memory (cudaErrorInvalidValue if bytes exceed it).
cudaError_t raise_dynamic_smem(const void *fn, size_t bytes);
// Stockham plan of a line of N points (false: a prime factor above 7 or too many stages), and
// the complex lines per tile of a line pass (spec = false) or spectrum pass (spec = true) that
// fit the shared-memory budget, at most cap_lines (kwb_api.cu).
bool make_plan(int N, FftPlan &pl);
// The same stages in another order: 0 as make_plan (8s first, then 4 or 2, then 3, 5, 7),
// 1 radix-4 stages instead of 8s, 2 the odd radices first.
bool make_plan_order(int N, FftPlan &pl, int order);
// The plan of a line of N points: direct Stockham stages when N is 2/3/5/7-smooth, else
// Bluestein with a power-of-two inner length (N <= KWB_BLUESTEIN_MAX_N); keeps pl's chirp tables.
bool plan_line(int N, FftPlan &pl, int order);
int choose_L(int N, int want, int cap_lines, int dispersion, bool spec);
size_t line_pass_smem(int N, int L);
size_t spec_pass_smem(int N, int L, int dispersion);
// threads per CTA of a Stockham line pass along `axis` (-1: not a line pass)
int pass_threads(const SimDev &h, long long tiles, long long elems_per_tile, int axis = -1);
cudaError_t launch_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode,
                             long long step_s, cudaStream_t st);
cudaError_t launch_eos_x_fwd(const SimDev *d_sim, const SimDev &h, long long step_s,
                             cudaStream_t st);
cudaError_t launch_spec_pass(const SimDev *d_sim, const SimDev &h, int axis, int op,
                             long long step_s, cudaStream_t st);
cudaError_t launch_eos_x_inv(const SimDev *d_sim, const SimDev &h, long long step_s,
                             cudaStream_t st);
cudaError_t launch_tr_inject(const SimDev *d_sim, const SimDev &h, long long step_s,
                             cudaStream_t st);
cudaError_t launch_sensor_gather(const SimDev *d_sim, const SimDev &h, const GroupDev *d_group,
                                 long long n, long long step_s, cudaStream_t st);
cudaError_t launch_advance_t0(long long *t0, long long k, cudaStream_t st);
// Raise the dynamic shared-memory limit of every time-step kernel for this simulation's tiles.
cudaError_t prime_attributes(const SimDev &h);

// Register-FFT kernels (kwb_fast.cu) for line lengths 64, 128, 256, 512, 1024, and (through
// kwb_fast_mixed.cu) the mixed-radix lengths 96, 160, 192, 320
struct ElGrad;
bool fast_size(int N);
bool fast_mixed_size(int N);
cudaError_t fast_mixed_prime(int N);
cudaError_t fast_mixed_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                                 cudaStream_t st);
cudaError_t fast_mixed_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st);
cudaError_t fast_mixed_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s,
                            cudaStream_t st);
cudaError_t fast_mixed_el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st);
// ... and (kwb_fast_mixed2.cu) 80, 384, 640, 768.
bool fast_mixed2_size(int N);
cudaError_t fast_mixed2_prime(int N);
cudaError_t fast_mixed2_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                                  cudaStream_t st);
cudaError_t fast_mixed2_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st);
cudaError_t fast_mixed2_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s,
                             cudaStream_t st);
cudaError_t fast_mixed2_el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st);
// ... (kwb_fast_mixed3.cu) 144, 288, 432.
bool fast_mixed3_size(int N);
cudaError_t fast_mixed3_prime(int N);
cudaError_t fast_mixed3_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                                  cudaStream_t st);
cudaError_t fast_mixed3_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st);
cudaError_t fast_mixed3_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s,
                             cudaStream_t st);
cudaError_t fast_mixed3_el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st);
// ... (kwb_fast_mixed4.cu) 576, 864, 400.
bool fast_mixed4_size(int N);
cudaError_t fast_mixed4_prime(int N);
cudaError_t fast_mixed4_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                                  cudaStream_t st);
cudaError_t fast_mixed4_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st);
cudaError_t fast_mixed4_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s,
                             cudaStream_t st);
cudaError_t fast_mixed4_el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st);
// ... (kwb_fast_mixed5.cu) 500, 800, 1000.
bool fast_mixed5_size(int N);
cudaError_t fast_mixed5_prime(int N);
cudaError_t fast_mixed5_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                                  cudaStream_t st);
cudaError_t fast_mixed5_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st);
cudaError_t fast_mixed5_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s,
                             cudaStream_t st);
cudaError_t fast_mixed5_el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st);
cudaError_t fast_prime(int N);
cudaError_t fast_line_pass(const SimDev *d_sim, const SimDev &h, int axis, int mode, long long s,
                           cudaStream_t st);
cudaError_t fast_eos(const SimDev *d_sim, const SimDev &h, bool fwd, long long s, cudaStream_t st);
cudaError_t fast_spec(const SimDev *d_sim, const SimDev &h, int axis, int op, long long s,
                      cudaStream_t st);
bool fast_plane_size(int Ny, int Nz);
bool fast_plane_available();
#define KWB_PLANE_VARIANTS 6  // cluster plane-pass variants (kwb_fast_impl.cuh PlaneVariant)
int fast_plane_variants(int *ids = nullptr);
// The chosen plane-pass variant wants its multiplier slot-major ([kx][slot][j], k_z of j from
// fast_plane_slot_kz).
bool fast_plane_slot_major(const SimDev &h);
void fast_plane_slot_kz(int Nz, int *kz);
cudaError_t fast_plane_prime();
// Tensor maps of the fields a strided register line pass stages (p, rho0, u_d, rho_d), boxes of
// `cols` columns x N / k positions along `axis` (the smallest k with N / k <= 256 dividing N);
// false when the driver's encoder is unavailable or rejects a map (the pass then stages by
// 16-byte cp.async).
bool encode_strided_maps(SimDev &h, int axis, int cols);
void fast_plane_slot_ky(int Ny, int *ky);
cudaError_t fast_plane(const SimDev *d_sim, const SimDev &h, long long s, cudaStream_t st);

// Elastic solver kernels (kwb_elastic.cu).  One gradient pass along `axis` transforms up to
// three fields and writes (or, per bit of acc, adds) each derivative into its destination.
struct ElGrad {
  const float *src[3];
  float *dst[3];
  int nf;
  int acc;  // bit f: dst[f] += d/dx_axis src[f]; else dst[f] = d/dx_axis src[f]
  int neg;  // 1: staggered - (velocity gradients), 0: staggered + (stress gradients)
};
cudaError_t el_prime(const SimDev &h);
cudaError_t el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st);
cudaError_t el_velocity(const SimDev &h, long long s, cudaStream_t st);
cudaError_t el_stress(const SimDev &h, long long s, cudaStream_t st);
// which 0: velocity sources, 1: stress sources (and p at their points)
cudaError_t el_inject(const SimDev &h, int which, long long s, cudaStream_t st);
cudaError_t el_init(const SimDev &h, cudaStream_t st);
// Register-FFT gradient pass (kwb_fast.cu) for line lengths 64 ... 1024.
cudaError_t fast_el_grad(const SimDev &h, int axis, const ElGrad &g, long long s, cudaStream_t st);

// Post-loop sensor filters (kwb_postfilter.cu): build the FP32 convolution kernels h[nf][Nt] of
// nf filters (sin_th[f]: sin(theta) of filter f's directivity, NaN for none; freq != 0 adds the
// Gaussian frequency response), using the FP64 scratch H[nf][Nt] and cosT[Nt]; then filter the
// series in[t][j] of n_pts points into out with filter fid[j].
cudaError_t filter_build_kernels(float *h, double *H, double *cosT, int Nt, int nf, const double *sin_th,
                                 double dir_size, double d_min, double dt, int freq, double fc, double bw,
                                 cudaStream_t st);
cudaError_t filter_apply(float *out, const float *in, const float *h, const int *fid, int Nt, long long n_pts,
                         cudaStream_t st);

// FFT schedule (kwb_tune.cu): the tuned fields of a SimDev.
struct Schedule {
  signed char tile_var[8];
  signed char tma_line[3];
  short thr_line[3];
  int L_line[3], L_eosx, L_spec[3];
  signed char plan_order[3];
};
void schedule_of(const SimDev &h, Schedule &s);
void schedule_apply(SimDev &h, const Schedule &s);  // also rebuilds the plans
std::string schedule_str(const Schedule &s);
bool schedule_parse(const char *txt, Schedule &s);
// Measure every pass of h's time step under its candidate schedules (pick >= 0: take candidate
// `pick` of every pass instead) and store the fastest in h.  Runs on h's own field and spectrum
// buffers, which the caller must reset afterwards; d_scratch holds the timing descriptor.
// explore_order adds the Stockham radix orders (not bit-identical to the default order).
cudaError_t tune_schedule(SimDev &h, SimDev *d_scratch, cudaStream_t st, int pick, bool explore_order,
                          std::string *log);

// FP64 table builders.
cudaError_t build_twiddles(float2 *out, int N, cudaStream_t st);
cudaError_t build_gradient(float2 *pos, float2 *neg, int N, double d, cudaStream_t st);
cudaError_t build_pml_deficit(float *out, int N, int pml_size, double alpha, double dt,
                              int staggered, cudaStream_t st);
cudaError_t build_eos_multiplier(float *M, float *M2, const int N[3], const double d[3],
                                 double c_ref, double dt, double c_sq_fold, int absorbing,
                                 double tau, double eta, double y, const int *slot_ky,
                                 const int *slot_kz, cudaStream_t st);
// Reorder a row-major grid array (NumPy order) into column-major (x fastest); ndim 2 or 3.
cudaError_t transpose_to_column_major(double *out, const double *in, int ndim, const int N[3],
                                      cudaStream_t st);
cudaError_t convert_f64_to_f32(float *out, const double *in, long long n, int op,
                               cudaStream_t st);
cudaError_t build_nlq(float *out, const double *bona, int bona_array, double bona_s,
                      const double *rho0, int rho0_array, double rho0_s, long long n,
                      cudaStream_t st);
cudaError_t build_source_table(float *out, const double *sig, long long n_rows, long long n_pts,
                               long long n_cols, const double *c_at_pts, double c_s,
                               int c_array, double divisor, int apply_c, cudaStream_t st);
}  // namespace kwb
