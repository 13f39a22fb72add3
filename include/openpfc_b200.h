/*
 * openpfc_b200.h -- C ABI of the B200-native spectral PFC time step.
 *
 * One handle = one periodic 3D field on one GPU.  The state is kept resident
 * in k-space; every call returns an int status (0 = OK, negative = error) and
 * never throws.  opfc_last_error() returns a message for the last failure on a
 * handle.  Handles are not thread-safe; all work of a handle is issued on one
 * CUDA stream.
 *
 * Layout at the boundary (identical to the reference):
 *   real field  : N0*N1*N2 values, x fastest, idx = i + N0*(j + N1*k)
 *                 (include/openpfc/kernel/field/operations.hpp:96-103)
 *   half spectrum: (N0/2+1)*N1*N2 complex values, interleaved (re, im), same
 *                 order (src/openpfc/runtime/cpu/fft.cpp:58-70)
 *   forward transform unnormalised, backward scaled by 1/(N0*N1*N2)
 *                 (include/openpfc/kernel/fft/detail/fft_heffte_backend.hpp:216,243)
 */
#ifndef OPENPFC_B200_H
#define OPENPFC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define OPFC_OK 0
#define OPFC_ERR_ARG (-1)         /* bad argument (null pointer, bad enum)      */
#define OPFC_ERR_SIZE (-2)        /* size contract violated / unsupported size  */
#define OPFC_ERR_CUDA (-3)        /* CUDA runtime error                         */
#define OPFC_ERR_NONFINITE (-4)   /* NaN/Inf detected in the field              */
#define OPFC_ERR_TIMEOUT (-5)     /* bounded device wait expired                */
#define OPFC_ERR_OOM (-6)         /* device allocation failed                   */
#define OPFC_ERR_STATE (-7)       /* call out of order (e.g. step before init)  */
#define OPFC_ERR_IO (-8)          /* file could not be opened / written         */

/* precision of the bulk arithmetic */
#define OPFC_FP32 0
#define OPFC_FP64 1

/* model kinds */
#define OPFC_MODEL_PLAIN 0     /* conserved PFC, docs/api/examples/10_complete_pfc_model.cpp:121-213 */
#define OPFC_MODEL_TUNGSTEN 1  /* Tungsten ETD, apps/tungsten/include/tungsten/cpu/tungsten_model.hpp:306-366 */
#define OPFC_MODEL_FILTERED 2  /* Gaussian mean-field filter + polynomial of psi_MF */
#define OPFC_MODEL_ALUMINUM 3  /* Aluminum PFC variant, apps/aluminumNew/Aluminum.hpp */
#define OPFC_MODEL_USER_ETD 4  /* caller-supplied ETD1 operators (opfc_set_operators) */

/* where a user pointer lives */
#define OPFC_HOST 0
#define OPFC_DEVICE 1

/* element type of a user buffer */
#define OPFC_F32 0
#define OPFC_F64 1

/* Tungsten base parameters, same names and defaults as
 * apps/tungsten/include/tungsten/common/tungsten_params.hpp:33-57. */
typedef struct opfc_tungsten_params {
  double n0, n_sol, n_vap, T, T0, Bx, alpha, alpha_farTol;
  int alpha_highOrd;
  double lambda, stabP, shift_u, shift_s, p2, p3, p4, q20, q21, q30, q31, q40;
} opfc_tungsten_params;

/* Aluminum PFC parameters: the fields of Aluminum::params
 * (apps/aluminumNew/Aluminum.hpp:29-82), same names; the reference leaves
 * unset fields at 0 (opfc_desc_default: all 0, T0 = 1).  With G_grid != 0 the
 * step carries the moving temperature T_var(x, t) and a third field
 * P*psi = F^-1[P_F psi_hat] (direct-load kernels); its time comes from
 * opfc_set_time. */
typedef struct opfc_aluminum_params {
  double n0, n_sol, n_vap, T, T0, Bx, T_const, T_max, T_min, G_grid, V_grid, x_initial, m_xpos, alpha,
      alpha_farTol;
  int alpha_highOrd;
  double tau_const, lambda, stabP, shift_u, shift_s, p2, p3, p4, p2_bar, p3_bar, p4_bar, q20, q21, q30, q31,
      q40, q20_bar, q21_bar, q30_bar, q31_bar, q40_bar, q2_bar, q3_bar, q4_bar, q2_bar_L;
} opfc_aluminum_params;

typedef struct opfc_desc {
  int n[3];            /* N0 (x, fastest), N1, N2 */
  double dx[3];        /* grid spacing */
  double origin[3];    /* physical coordinate of cell (0,0,0) */
  int precision;       /* OPFC_FP32 / OPFC_FP64 */
  int model;           /* OPFC_MODEL_* */
  double r;            /* PLAIN/FILTERED: L(k) = -k^2 (r + (1-k^2)^2) */
  double filter_alpha; /* FILTERED: chi = exp(-k^2 / (2 alpha^2)) */
  double p2, p3, p4;   /* FILTERED: N = p2 v^2/2 + p3 v^3/3 + p4 v^4/4, v = psi_MF */
  opfc_tungsten_params tungsten; /* TUNGSTEN */
  void *stream;        /* cudaStream_t to use, or NULL for a private stream */
  int device;          /* CUDA device ordinal */
  opfc_aluminum_params aluminum; /* ALUMINUM */
  /* Slab of a grid shared by several handles (sharded step, opfc_pass):
   * n_global = the whole grid (0 = the handle's own n), kx0 = first global kx
   * of the handle's half-spectrum columns.  The handle's operators use the
   * global wave numbers (kx0 + kx) 2 pi / (dx n_global) and its C2R scales by
   * 1 / (N0 N1 N2 of n_global).  PLAIN and FILTERED. */
  int n_global[3];
  int kx0;
} opfc_desc;

typedef struct opfc_handle opfc_handle;

/* Fill a descriptor with defaults: TungstenParams defaults, dx = 1,
 * origin = 0, FP32, PLAIN, r = -0.25.  Replaces the default-constructed
 * parameter block of tungsten_params.hpp:33-57. */
void opfc_desc_default(opfc_desc *desc);

/* Lifetime.  opfc_create replaces the GPU model ctor + FFT plan
 * (apps/tungsten/include/tungsten/cuda/tungsten_model.hpp:132-178). */
int opfc_create(const opfc_desc *desc, opfc_handle **out);
int opfc_destroy(opfc_handle *h);
const char *opfc_last_error(const opfc_handle *h);
const char *opfc_status_string(int status);

/* Operator tables in FP64 on the host, rounded to the handle precision and
 * uploaded.  Replaces Model::initialize(dt) / prepare_operators
 * (cpu/tungsten_model.hpp:223-292; 10_complete_pfc_model.cpp:94-115,166-213). */
int opfc_initialize(opfc_handle *h, double dt);

/* Field access.  count must be N0*N1*N2 (real) or (N0/2+1)*N1*N2 (complex);
 * dtype OPFC_F32/OPFC_F64; where OPFC_HOST/OPFC_DEVICE (device pointers must
 * hold the handle's own precision).  set_psi replaces writing the registered
 * "psi" field + finalize_after_field_modifiers (model.hpp:272); get_psi
 * replaces prepare_for_field_modifiers (model.hpp:265) + reading "psi". */
int opfc_set_psi(opfc_handle *h, const void *psi, size_t count, int dtype, int where);
int opfc_get_psi(opfc_handle *h, void *psi, size_t count, int dtype, int where);
int opfc_get_psi_hat(opfc_handle *h, void *psi_hat, size_t count, int dtype, int where);
/* The mean-field filtered density psi_MF (Tungsten "psiMF" field,
 * cpu/tungsten_model.hpp:200), computed from the current state. */
int opfc_get_psi_mf(opfc_handle *h, void *psi_mf, size_t count, int dtype, int where);

/* Advance n_steps time steps (Model::step, cpu/tungsten_model.hpp:306;
 * 10_complete_pfc_model.cpp:121).  Asynchronous on the handle's stream; the
 * step sequence is captured in a CUDA graph on first use. */
int opfc_step(opfc_handle *h, int n_steps);
/* Wait for the handle's stream; reports OPFC_ERR_NONFINITE if any step
 * produced NaN/Inf since the last check. */
int opfc_sync(opfc_handle *h);

/* One pass of the step, or of a transform, on the handle's own arrays, queued
 * on its stream (no counterpart in the reference, whose GPU model runs whole
 * 3D transforms; these are the pieces a sharded step is built from -- a field
 * split over ranks in z slabs for the x and y passes and in kx slabs for the z
 * update, with all-to-all transposes between them, the decomposition of the
 * reference's HeFFTe plans, src/openpfc/runtime/cpu/fft.cpp:72-81).  PLAIN,
 * FILTERED and USER_ETD.  Arrays (opfc_array): WORK = A, the half spectrum in
 * the split layout (main part (N0/2) x N1 x N2 complex, kx fastest, then the
 * kx = N0/2 plane N1 x N2); STATE = psi_hat, same layout; REAL = N0 N1 N2 reals,
 * x fastest.  Passes (`mean`: the mean density the x passes add; `flags`):
 *   Y_INVERSE, Y_FORWARD       A along y, in place
 *   X_FUSED                    A: per x row C2R, nonlinearity (+ mean), R2C
 *   Z_UPDATE                   A -> psi_hat (ETD update) and A = F_z^-1 of the
 *                              new state; then the Hermitian projection of the
 *                              kx = 0 plane (flags bit 0) and of the kx = N0/2
 *                              plane (bit 1) -- give only the planes the handle
 *                              holds of the whole grid
 *   XY_FORWARD                 REAL -> A: x R2C, y forward
 *   XY_BACKWARD                A -> REAL: y inverse, x C2R scaled by 1/(N0 N1 N2
 *                              of n_global), + mean
 *   Z_FORWARD                  A -> psi_hat (flags bit 2: zero the k = 0 slot)
 *   Z_INVERSE                  psi_hat -> A as a step starts from it (chi psi_hat
 *                              for FILTERED)
 *   Z_INVERSE_STATE            psi_hat -> A
 * opfc_array returns a device pointer (REAL is allocated on first use), NULL
 * for a bad argument. */
#define OPFC_PASS_Y_INVERSE 0
#define OPFC_PASS_X_FUSED 1
#define OPFC_PASS_Y_FORWARD 2
#define OPFC_PASS_Z_UPDATE 3
#define OPFC_PASS_XY_FORWARD 4
#define OPFC_PASS_XY_BACKWARD 5
#define OPFC_PASS_Z_FORWARD 6
#define OPFC_PASS_Z_INVERSE 7
#define OPFC_PASS_Z_INVERSE_STATE 8
#define OPFC_ARRAY_WORK 0
#define OPFC_ARRAY_STATE 1
#define OPFC_ARRAY_REAL 2
int opfc_pass(opfc_handle *h, int pass, double mean, int flags);
void *opfc_array(opfc_handle *h, int which);

/* Failure-path check (no reference counterpart; the reference's GPU model
 * blocks in cudaDeviceSynchronize without a limit): runs the bounded mbarrier
 * wait that every pipelined pass kernel uses on a barrier that nothing
 * completes, with a limit of limit_ms (0.1 .. 1000, the passes use 4 s).  The
 * wait expires, the kernel records the timeout in the handle's status flag and
 * returns, and the next opfc_sync reports OPFC_ERR_TIMEOUT; the handle stays
 * usable.  No fault is raised and no copy is left in flight. */
int opfc_check_bounded_wait(opfc_handle *h, double limit_ms);

/* Stand-alone transforms with the reference's IFFT contract
 * (include/openpfc/kernel/fft/fft_interface.hpp:51,61): forward R2C
 * unnormalised, backward C2R scaled by 1/(N0 N1 N2).  Buffers as above. */
int opfc_fft_forward(opfc_handle *h, const void *in_real, void *out_complex, int dtype, int where);
int opfc_fft_backward(opfc_handle *h, const void *in_complex, void *out_real, int dtype, int where);

/* Diagnostics.  mass = mean density (sum psi / N0 N1 N2), carried in FP64.
 * free energy (plain / filtered models; project-defined, the reference has
 * none): F = sum dV [1/2 psi F^-1{(r + (1-k^2)^2) psi_hat} + 1/4 psi^4],
 * reduced in FP64. */
int opfc_mass(opfc_handle *h, double *mean_density);
int opfc_free_energy(opfc_handle *h, double *energy);

/* Introspection (IFFT::size_inbox/size_outbox/get_allocated_memory_bytes,
 * fft_interface.hpp:68-72). */
size_t opfc_size_inbox(const opfc_handle *h);
size_t opfc_size_outbox(const opfc_handle *h);
size_t opfc_allocated_bytes(const opfc_handle *h);
void *opfc_get_stream(const opfc_handle *h);
/* Number of kernels one opfc_step(1) launches (for launch accounting). */
int opfc_kernels_per_step(const opfc_handle *h);
/* Measurement hook (no reference counterpart; the reference times FFT calls
 * with MPI_Wtime, fft_heffte_backend.hpp:158-164): times each kernel of the
 * step alone, `reps` launches each, with CUDA events on the handle's stream;
 * ms[k] = mean milliseconds per launch.  Returns the number of kernels timed
 * (>= 0) or an error.  The repeated in-place passes leave the field undefined:
 * call opfc_set_psi before stepping again. */
int opfc_profile_step(opfc_handle *h, int reps, double *ms, int max_kernels);
/* Name of kernel k of the step ("y_inverse", "x_fused", ...). */
const char *opfc_step_kernel_name(int k);
/* NVTX range name of kernel k: the reference's profiling regions whose work the
 * kernel does (OPENPFC_PROFILE "gradient/mean_field/...", "gradient/evolve/...",
 * apps/tungsten/include/tungsten/cpu/tungsten_model.hpp:313-362), pass in
 * brackets.  opfc_profile_step times each kernel inside its range; with
 * OPFC_NVTX=1 in the environment at opfc_create, opfc_step runs eagerly (no
 * CUDA graph) and encloses every kernel in its range and every step in "step",
 * so an NVTX-aware profiler groups the work by the reference's regions. */
const char *opfc_step_kernel_region(int k);

/* Autotuner (replaces pfc::gpu::AutoTuner::tune_kernel,
 * include/openpfc/runtime/common/gpu_autotune.hpp:295-333, same environment
 * variables OPENPFC_GPU_AUTOTUNE_{DISABLE,MODE,CACHE_DIR}): times the kernel
 * variants of each pass of the step (y: 0 pipelined | 1 direct | 2 pipelined
 * with half-width tiles, two CTAs per SM | 3 pipelined with ping-pong FFT
 * exchange buffers | 4 direct with 32 values per thread (N = 512, 1024); x: 0
 * pipelined (warp-square kernel
 * where M = R^2 or 2 R^2) | 1 direct | 2 pipelined without it | 3 warp-square
 * with rows loaded straight into registers (PLAIN, FILTERED) | 4 as 3, loading
 * the next row into registers while the current one is transformed; z update:
 * 0 pipelined with streamed tables | 1 pipelined with radial tables (isotropic
 * grids) | 2 direct with streamed tables | 3 pipelined with operators computed
 * from k^2 | 4 direct with computed operators | 5 as 3 with ping-pong exchange
 * buffers (3-5: PLAIN and FILTERED) | 6 pipelined with the folded tables and
 * ping-pong exchange buffers | 7 direct with the folded tables | 8 pipelined
 * with the folded tables | 9 pipelined with the folded tables and 128-byte
 * tile rows, the tiles streamed in 256-row boxes through a two-slot ring (z
 * length 1024, PLAIN and FILTERED; otherwise as 7) (6-9: every model but the
 * moving-gradient Aluminum and caller-supplied operators);
 * 3 warm-up + 10 timed launches each), keeps the fastest and caches it per
 * device; opfc_initialize applies cached choices.  Every table variant holds
 * operators built in FP64 on the host and rounded once to the compute
 * precision (the folded tables hold the per-mode values of the modes
 * (kx, |ky|, |kz|), k^2 being even in ky and kz); the computed variants 3-5
 * evaluate them per mode in the compute precision, so FP32 handles consider
 * them only with OPFC_FP32_COMPUTED_OPERATORS=1 in the environment.
 * ms (OPFC_AUTOTUNE_SLOTS doubles, may be NULL) receives the mean
 * milliseconds per launch of y0 .. y4 x0 .. x4 z0 .. z9 (-1 if not applicable).
 * Call after opfc_initialize; the passes run in place, so set the field
 * afterwards.  opfc_variants reports the chosen (y, x, z) variants. */
#define OPFC_AUTOTUNE_SLOTS 20
int opfc_autotune(opfc_handle *h, double *ms);
int opfc_variants(const opfc_handle *h, int *var);

/* Adjoint of the step (no counterpart in the reference, which has no
 * differentiation) for the plain, filtered, Tungsten and Aluminum (G_grid = 0)
 * models and caller-supplied operators.  opfc_set_r changes r
 * (PLAIN/FILTERED) and rebuilds the tables.  opfc_forward_checkpointed advances
 * n_steps from the current state, keeping a device snapshot of psi_hat every K
 * steps.  opfc_adjoint then takes dLoss/dpsi_T (real field, count N0*N1*N2)
 * and returns dLoss/dpsi_0 (same dtype/location), dLoss/dr (NaN for the
 * models without r) and dLoss/dn0 = sum(dLoss/dpsi_0), re-running each K-step
 * segment from its snapshot and stepping the adjoint
 *   lambda_n = A lambda + dN/du (B lambda) + C[dN/dv (B lambda)]
 * backwards, A = F^-1 opL F, B = F^-1 opN F, C = F^-1 chi F (the mean-field
 * filter; u = psi, v = C psi; N the model's nonlinearity); the handle is left
 * at the forward run's final state. */
/* Uneven-size ensembles (no counterpart in the reference, which runs one field
 * per MPI job): `count` independent plain-PFC fields, each with its own size
 * (N0/2 in {16,24,32,40,48,64}, N1, N2 in {16,32,48,64,80,96,128}), dx and r,
 * one precision.  Every stage of a step is one persistent kernel over all
 * members; opfc_ensemble_step(n) captures the n-step loop as one CUDA graph.
 * Fields are host FP64 arrays (x fastest).  opfc_ensemble_autotune times the
 * variants (tile width 16 / 8 lines x 4 / 8 / 16 CTAs per SM, which also sets
 * the kernel's register budget) of the y, x and z-update stages separately,
 * reports 6 milliseconds per stage, caches the fastest (see
 * OPENPFC_GPU_AUTOTUNE_* in the library notes) and invalidates the states. */
typedef struct opfc_ensemble opfc_ensemble;
int opfc_ensemble_create(int count, const opfc_desc *descs, opfc_ensemble **out);
int opfc_ensemble_destroy(opfc_ensemble *e);
const char *opfc_ensemble_last_error(const opfc_ensemble *e);
int opfc_ensemble_initialize(opfc_ensemble *e, double dt);
int opfc_ensemble_set_psi(opfc_ensemble *e, int member, const double *psi, size_t count);
int opfc_ensemble_get_psi(opfc_ensemble *e, int member, double *psi, size_t count);
int opfc_ensemble_step(opfc_ensemble *e, int n_steps);
int opfc_ensemble_sync(opfc_ensemble *e);
int opfc_ensemble_autotune(opfc_ensemble *e, double *ms_col, double *ms_x, double *ms_upd);
int opfc_ensemble_variants(const opfc_ensemble *e, int *var_col, int *var_x, int *var_upd);
size_t opfc_ensemble_cells(const opfc_ensemble *e);
void *opfc_ensemble_stream(const opfc_ensemble *e);

int opfc_set_r(opfc_handle *h, double r);
/* Time of the next step for models whose step depends on it (Aluminum with a
 * moving temperature gradient: the t of Aluminum::step(t)); each step then
 * advances it by dt_per_step on the device (opfc_initialize sets the time to 0
 * and the increment to dt).  Other models ignore it. */
int opfc_set_time(opfc_handle *h, double t, double dt_per_step);
/* OPFC_MODEL_USER_ETD: the GPU backend of the reference's generic ETD1 stepper
 * (Etd1Stepper::set_coefficients / attempt_step,
 * include/openpfc/kernel/simulation/steppers/etd1.hpp, with the spectral
 * coefficients of spectral_exp_coefficients.hpp): per-mode tables in the
 * reference's half-spectrum layout ((N0/2+1) x N1 x N2, count entries):
 * psi_hat <- exp_Ldt psi_hat + n_weight N_hat with N = p2 v^2/2 + p3 v^3/3 +
 * p4 v^4/4 (opfc_desc p2, p3, p4) of v = F^-1[chi psi_hat] (chi NULL = 1).
 * The fused passes carry the mean exactly, so the k = 0 entries must be
 * exp_Ldt = 1, n_weight = 0, chi = 1 (conserved dynamics), else OPFC_ERR_ARG.
 * Call before opfc_initialize (whose dt is then only recorded). */
int opfc_set_operators(opfc_handle *h, const double *exp_Ldt, const double *n_weight, const double *chi,
                       size_t count);
int opfc_forward_checkpointed(opfc_handle *h, int n_steps, int K);
int opfc_adjoint(opfc_handle *h, const void *grad_psi_T, int dtype, int where, void *grad_psi0,
                 double *grad_r, double *grad_n0);

/* Initial conditions, host-side (set-up only), x-fastest cell order.
 * Random numbers: one draw of std::mt19937_64(seed) per number, mapped to
 * [0,1) as (draw >> 11) * 2^-53.
 * opfc_ic_noise: psi = n0 + U(-amp, amp) per cell.
 * opfc_ic_seed: one-mode BCC seed, u = rho + sum_q 2 amp cos(q.(x - center)) over
 *   the six <110>/sqrt(2) vectors inside |x - center| < radius, x = origin + i dx
 *   (include/openpfc/kernel/simulation/initial_conditions/single_seed.hpp; with
 *   outside_zero = 1 the outside is zeroed like SingleSeed::apply, with 0 it is
 *   left as is like apps/tungsten/tests/test_tungsten.cpp:262-280).
 * opfc_ic_seeds: noisy liquid n0 + U(-noise, noise), then nseeds spheres of
 *   radius_cells at centres (u0 N0, u1 N1, u2 N2) drawn from the same stream,
 *   filled with n0 + amp sum_q cos(q.(x - c)) (periodic minimum image). */
int opfc_ic_noise(double *psi, size_t count, double n0, double amp, uint64_t seed);
int opfc_ic_seed(double *psi, const int n[3], const double dx[3], const double origin[3],
                 const double center[3], double radius, double rho, double amp, int outside_zero);
int opfc_ic_seeds(double *psi, const int n[3], const double dx[3], double n0, double noise,
                  int nseeds, double radius_cells, double amp, uint64_t seed);
/* opfc_ic_seed_grid_fcc: the Aluminum app's SeedGridFCC (apps/aluminumNew/
 * SeedGridFCC.hpp, SeedFCC.hpp) on a pre-filled field: Ny x Nz FCC seeds at
 * x = X0 (+ jitter), rotated at random; positions and angles from
 * std::mt19937_64(rseed) through std::uniform_real_distribution in the
 * reference's order (the standard library's mapping, as in the reference). */
int opfc_ic_seed_grid_fcc(double *psi, const int n[3], const double dx[3], const double origin[3], int Nx, int Ny,
                          int Nz, double X0, double radius, double amplitude, double rho, double rseed);
/* opfc_ic_random_seeds: the reference's RandomSeeds initial condition
 * (include/openpfc/kernel/simulation/initial_conditions/random_seeds.hpp:54-101,
 * with Seed of seed.hpp): 150 seeds of radius 20 placed in the reference's
 * fixed box (x in [-108, -68), y, z in [-128, 128)) and rotated at random, from
 * std::mt19937_64(42) through std::uniform_real_distribution in the
 * reference's order; a cell inside a seed takes density + sum_q 2 amplitude
 * cos(q.x) over the six rotated <110>/sqrt(2) vectors (the first seed that
 * contains it wins), every other cell 0.  The whole field is written. */
int opfc_ic_random_seeds(double *psi, const int n[3], const double dx[3], const double origin[3], double density,
                         double amplitude);

/* On-disk formats of the reference's writers and readers (one process owns
 * the whole grid; no MPI).
 * opfc_format_filename: pfc::utils::format_with_number
 *   (include/openpfc/frontend/utils/utils.hpp:96-139): a pattern without '%' is
 *   returned as is; otherwise exactly one "%[-+ 0][*][width]d" and no other '%'
 *   (else OPFC_ERR_ARG); out_len too small -> OPFC_ERR_SIZE.
 * opfc_write_binary: psi as raw native FP64, x fastest, no header, file named
 *   format_with_number(pattern, increment) and truncated first
 *   (BinaryWriter::write(increment, RealField),
 *   include/openpfc/frontend/io/binary_writer.hpp).
 * opfc_write_binary_hat: psi_hat in the reference layout ((N0/2+1) x N1 x N2,
 *   interleaved re, im FP64), BinaryWriter::write(increment, ComplexField).
 * opfc_read_binary: such a raw FP64 psi file -> the state, as opfc_set_psi
 *   (FileReader::apply, include/openpfc/kernel/simulation/initial_conditions/
 *   file_reader.hpp, via BinaryReader::read); a short file -> OPFC_ERR_SIZE.
 * opfc_write_vti: psi as VTK XML ImageData, one Float64 point array appended
 *   raw with a UInt64 length prefix, Origin / Spacing from the descriptor,
 *   array name field_name (NULL: "Field") (VTKWriter::write,
 *   src/openpfc/frontend/io/vtk_writer.cpp:70-108,166-225).
 * File errors -> OPFC_ERR_IO with the message in opfc_last_error. */
int opfc_format_filename(const char *pattern, int increment, char *out, size_t out_len);
int opfc_write_binary(opfc_handle *h, const char *pattern, int increment);
int opfc_write_binary_hat(opfc_handle *h, const char *pattern, int increment);
int opfc_read_binary(opfc_handle *h, const char *filename);
int opfc_write_vti(opfc_handle *h, const char *pattern, int increment, const char *field_name);
/* The same formats for host arrays and one process's box of a global grid
 * (x fastest; box = local extent at offset, as set_domain(global, local,
 * offset) of the reference's writers): opfc_write_raw writes the box of
 * `ncomp` (1 real, 2 complex) doubles per point at its place in the global
 * array -- a box covering the whole grid truncates `filename` first, a smaller
 * box is written in place (the file is created if missing, never truncated), so
 * that several writers can each fill their own box of one file;
 * opfc_prepare_raw truncates `filename` and sizes it to the whole grid, the
 * one-time step before such writers (the reference's collective
 * MPI_File_set_size(fh, 0), binary_writer.hpp); opfc_read_raw reads a box
 * (short file -> OPFC_ERR_SIZE); opfc_write_vti_raw writes one .vti piece.  A
 * box outside the grid -> OPFC_ERR_ARG. */
int opfc_write_raw(const char *filename, const int global[3], const int local[3], const int offset[3],
                   const double *data, int ncomp);
int opfc_prepare_raw(const char *filename, const int global[3], int ncomp);
int opfc_read_raw(const char *filename, const int global[3], const int local[3], const int offset[3],
                  double *data, int ncomp);
int opfc_write_vti_raw(const char *filename, const int global[3], const int local[3], const int offset[3],
                       const double origin[3], const double spacing[3], const char *name, const double *data);

/* Forward R2C transform that allocates nothing (no counterpart in the
 * reference; it is opfc_fft_forward without a handle).  For callers that cannot
 * call cudaMalloc: latency-bound loops, where cudaMalloc's implicit device-wide
 * synchronisation and unbounded run time are not acceptable, and host
 * applications whose own memory manager owns every device allocation and does
 * not let a library allocate.  in_real and out_complex are device pointers of
 * the given precision (OPFC_FP32/OPFC_FP64) in the boundary layout above; the
 * work is queued on `stream` (NULL = legacy default stream) and the call does
 * not wait for it.
 * The intermediate half spectrum lives in a fixed 16 MiB device array inside
 * the library (held by every GPU that loads it until exit):
 * (N0/2+1)*N1*N2 * (8 bytes FP32 | 16 bytes FP64) must be <= 16 MiB and every
 * axis <= 1024, else OPFC_ERR_SIZE.  The first call on a device looks up that
 * array's device address (cudaGetSymbolAddress) with the device current; make
 * that first call before any stream capture.  All calls share the array and the
 * twiddle tables next to it: calls that overlap on the GPU race. */
int opfc_fft_forward_noalloc(const void *in_real, void *out_complex, const int n[3], int precision,
                             void *stream);

#ifdef __cplusplus
}
#endif
#endif /* OPENPFC_B200_H */
