/*
 * tcgpu — B200 (sm_100a) implementation of SimpleTCSolver's RK3 time step
 * behind the reference's own C entry points.
 *
 * Drop-in boundary: the structs below are layout-compatible with the
 * reference's domain_t / array_t / fluid_t / tdm_t, and every function in the
 * "reference entry points" section keeps the reference's name, signature,
 * argument meaning and 0 / non-zero return convention (errors are also printed
 * to stderr). A C host that links libtcgpu.so instead of the reference's
 * src/integrate.c, src/decide_dt.c, src/fluid/{predict,correct,boundary}/,
 * src/fluid/compute_potential.c, src/fluid/update_pressure.c, src/tdm.c,
 * src/linear_system.c and src/halo.c runs its time step on the GPU.
 *
 * One GPU owns the whole domain: mysizes must equal glsizes and offsets be 0
 * (a single rank). The solver state (device copies of the fields, RK source
 * terms, spectral buffers) lives in a context created on the first call for a
 * given fluid_t and released by tcgpu_release().
 *
 * Coherence: by default each reference entry point reads the fields it needs
 * from the caller's host arrays and writes back the fields it changes, so the
 * caller sees exactly the reference's side effects ("coherent" mode). The
 * tcgpu_* extensions at the end let a caller keep the state on the GPU across
 * many steps and copy only when it wants to.
 */
#if !defined(TCGPU_H)
#define TCGPU_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#if defined(__cplusplus)
extern "C" {
#endif

#if !defined(NDIMS)
#define NDIMS 3
#endif

/* ---------------------------------------------------------------- types */

/* opaque: the reference's SimpleDecomp handle; this library never reads it */
typedef struct sdecomp_info_t_ sdecomp_info_t;

/* include/array.h:9-23 */
typedef struct {
  size_t size;
  int (* nadds)[2];
  size_t datasize;
  void * data;
} array_t;

/* include/domain.h:23-37 */
typedef struct {
  sdecomp_info_t * info;
  bool is_curved;
  size_t glsizes[NDIMS];
  size_t mysizes[NDIMS];
  size_t offsets[NDIMS];
  double lengths[NDIMS];
  double * xf, * xc;
  double * jdxf, * jdxc;
  double * hxxf, * hxxc;
  double * hyxf, * hyxc;
  double hz;
} domain_t;

/* include/fluid.h:18-36 */
typedef struct {
  array_t ux;
  array_t uy;
  array_t uz;
  array_t p;
  array_t psi;
  array_t t;
  array_t srcux[3];
  array_t srcuy[3];
  array_t srcuz[3];
  array_t srct[3];
  array_t lxx;
  array_t lyx0, lyx1, lxy;
  array_t lzx, lxz;
  array_t lyy0, lyy1;
  array_t lzy, lyz;
  array_t lzz;
  double Re, Pr;
} fluid_t;

typedef struct tdm_info_t_ tdm_info_t;

/* include/tdm.h:8-42 */
typedef struct {
  int (* const construct)(const int size, const int nrhs, const bool is_periodic, const bool is_complex, tdm_info_t ** info);
  int (* const get_l)(const tdm_info_t * info, double ** l);
  int (* const get_c)(const tdm_info_t * info, double ** c);
  int (* const get_u)(const tdm_info_t * info, double ** u);
  int (* const get_size)(const tdm_info_t * info, int * size);
  int (* const get_nrhs)(const tdm_info_t * info, int * nrhs);
  int (* const solve)(const tdm_info_t * info, void * data);
  int (* const destruct)(tdm_info_t * info);
} tdm_t;

/* include/runge_kutta.h:8-15 */
typedef double rkcoef_t[3];

/* ---------------------------------------------------- reference entry points */

/* include/integrate.h:5-9, src/integrate.c:9-35: decide_dt, then three RK
 * substeps of predict / compute_potential / correct / update_pressure */
int integrate(const domain_t * domain, fluid_t * fluid, double * dt);

/* include/decide_dt.h:5-9, src/decide_dt.c:125-160; reads coef_dt_adv and
 * coef_dt_dif from the environment on first use, as the reference does */
int decide_dt(const domain_t * domain, const fluid_t * fluid, double * dt);

/* include/fluid_solver.h:31-36, src/fluid/predict/main.c:35-110 */
int fluid_predict_field(const domain_t * domain, const size_t rkstep, const double dt, fluid_t * fluid);

/* include/fluid_solver.h:39-44, src/fluid/compute_potential.c:499-583.
 * The singular zero-wavenumber mode is pinned by setting its last radial
 * unknown to zero, so psi (and p) can differ from the reference's by an
 * additive constant; the reference leaves that constant to round-off. */
int fluid_compute_potential(const domain_t * domain, const size_t rkstep, const double dt, fluid_t * fluid);

/* include/fluid_solver.h:47-52, src/fluid/correct/main.c:15-28 */
int fluid_correct_velocity(const domain_t * domain, const size_t rkstep, const double dt, fluid_t * fluid);

/* include/fluid_solver.h:55-60, src/fluid/update_pressure.c:146-173 */
int fluid_update_pressure(const domain_t * domain, const size_t rkstep, const double dt, fluid_t * fluid);

/* include/fluid_solver.h:64-92, src/fluid/boundary/*.c + src/halo.c:
 * wall values / Neumann copies, then periodic y and z images */
int fluid_update_boundaries_ux(const domain_t * domain, array_t * array);
int fluid_update_boundaries_uy(const domain_t * domain, array_t * array);
int fluid_update_boundaries_uz(const domain_t * domain, array_t * array);
int fluid_update_boundaries_p(const domain_t * domain, array_t * array);
int fluid_update_boundaries_psi(const domain_t * domain, array_t * array);
int fluid_update_boundaries_t(const domain_t * domain, array_t * array);

/* include/fluid_solver.h:22-28, src/fluid/compute_diffusivity.c */
double fluid_compute_momentum_diffusivity(const fluid_t * fluid);
double fluid_compute_scalar_diffusivity(const fluid_t * fluid);

/* include/fluid_solver.h:9-19, src/fluid/init.c:98-122, src/fluid/save.c:8-28:
 * NPY load/save in the reference layout; Re and Pr come from the environment */
int fluid_init(const char dirname_ic[], const domain_t * domain, fluid_t * fluid);
int fluid_save(const char dirname[], const domain_t * domain, const fluid_t * fluid);

/* include/domain.h:40-47, src/domain.c:63-86, 389-432 (single rank) */
int domain_init(const char dirname_ic[], domain_t * domain);
int domain_save(const char dirname[], const domain_t * domain);

/* include/tdm.h:44 + src/tdm.c:255-325: batched tri-diagonal solver; solve()
 * accepts host or device memory and runs on the GPU */
extern const tdm_t tdm;

/* include/runge_kutta.h:8-15, src/runge_kutta.c:3-15 */
extern const uint_fast8_t rk_a;
extern const uint_fast8_t rk_b;
extern const uint_fast8_t rk_g;
extern const rkcoef_t rkcoefs[3];

/* ------------------------------------------------------------- extensions */
/* No counterparts in the reference: run-time replacements for its
 * compile-time constants, explicit residency control and diagnostics. */

/* replaces src/param/boundary-condition.c and src/param/implicit.c; the
 * defaults are the reference's shipped values (uy walls 1 / 0, scalar walls
 * +0.5 / -0.5, implicit diffusion in x only). coef_dt_* < 0 keeps the value
 * taken from the environment. Applies to contexts created afterwards. */
typedef struct {
  double uy_xm, uy_xp;
  double t_xm, t_xp;
  int implicit_x, implicit_y, implicit_z;
  double coef_dt_adv, coef_dt_dif;
} tcgpu_params_t;

int tcgpu_set_params(const tcgpu_params_t * params);
int tcgpu_get_params(tcgpu_params_t * params);

/* what the reference entry points copy back to the host besides the fields
 * they change (bit mask, per context) */
#define TCGPU_SYNC_SRCS    1u  /* RK source terms after fluid_predict_field */
#define TCGPU_SYNC_TENSORS 2u  /* velocity-gradient tensors after fluid_predict_field
                                  and integrate (those of the substep-3 input, as the
                                  reference leaves them) */
#define TCGPU_NO_COHERENCE 4u  /* copy nothing: the caller uses tcgpu_push/pull */
#define TCGPU_PIN_HOST     8u  /* page-lock the caller's six field arrays until
                                  tcgpu_release (faster host<->device copies) */
/* A host that cannot call tcgpu_set_coherence (the reference's unmodified
 * main.c) sets the environment variable TCGPU_SYNC_TENSORS=1 (and/or
 * TCGPU_SYNC_SRCS=1): contexts created afterwards start with that flag. */
int tcgpu_set_coherence(const domain_t * domain, fluid_t * fluid, unsigned flags);

/* field masks for tcgpu_push / tcgpu_pull */
#define TCGPU_UX  1u
#define TCGPU_UY  2u
#define TCGPU_UZ  4u
#define TCGPU_P   8u
#define TCGPU_PSI 16u
#define TCGPU_T   32u
#define TCGPU_FIELDS 63u
#define TCGPU_SRCS 64u
#define TCGPU_TENSORS 128u
int tcgpu_push(const domain_t * domain, fluid_t * fluid, unsigned fields);
int tcgpu_pull(const domain_t * domain, fluid_t * fluid, unsigned fields);

/* run nsteps full time steps on the device without host copies; dts (may be
 * NULL) receives each step's dt */
int tcgpu_run(const domain_t * domain, fluid_t * fluid, int nsteps, double * dts);

/* kernels of one time step, for tcgpu_run_timed's per-kernel accounting */
typedef enum {
  TCGPU_K_DTMIN = 0,     /* CFL reduction (decide_dt_adv) */
  TCGPU_K_DTFINAL,       /* dt from the reduction and the diffusive limits */
  TCGPU_K_FACTORS,       /* implicit-solve elimination factors for the step */
  TCGPU_K_PREDICT,       /* fused predict: right-hand sides, RK increment,
                            radial implicit solve, update, boundaries */
  TCGPU_K_APPLY,         /* update after the y / z solves (planar case) */
  TCGPU_K_YZSOLVE,       /* implicit line solves outside the predict: periodic y
                            and z, and x when nx > 256 */
  TCGPU_K_DIV_FFTY,      /* divergence + forward y transform */
  TCGPU_K_FFTZ_FWD,      /* forward z transform */
  TCGPU_K_TDM,           /* radial Poisson solve per wavenumber pair */
  TCGPU_K_FFTZ_INV,      /* backward z transform */
  TCGPU_K_IFFTY,         /* backward y transform -> psi */
  TCGPU_K_CORRECT,       /* velocity correction + pressure update */
  TCGPU_K_COUNT
} tcgpu_kernel_t;

/* tcgpu_run, timed with CUDA events recorded on the library's own stream.
 * elapsed_ms: device time of the nsteps steps. With instrument != 0 the steps
 * run as individual launches with an event after each kernel, and
 * kernel_ms[TCGPU_K_COUNT] / kernel_launches[TCGPU_K_COUNT] receive the summed
 * device time and launch count per kernel kind (otherwise the captured CUDA
 * graph runs and only the launch counts are filled). Any output may be NULL. */
int tcgpu_run_timed(const domain_t * domain, fluid_t * fluid, int nsteps, int instrument, double * dts,
                    float * elapsed_ms, double * kernel_ms, int * kernel_launches);

/* select the CUDA device used by contexts created afterwards in this thread */
int tcgpu_set_device(int device);

/* FP32-storage mode. No counterpart in the reference. bytes = 8 (default:
 * everything in FP64) or 4: contexts created afterwards store ux, uy, uz, t,
 * the RK source terms and the Poisson spectra in 4-byte floats (in a padded
 * device layout; host arrays stay the reference's doubles and are converted on
 * every copy), while p, psi and every coefficient table stay FP64; the
 * predict forms its explicit right-hand sides and the power-of-two y/z
 * transforms run in FP32 arithmetic, and the implicit solves, the radial
 * Poisson eliminations, the correction and the reductions stay FP64. An existing context keeps its storage until tcgpu_release(). Returns 0, or
 * non-zero for other byte counts. */
int tcgpu_set_storage(int bytes);
/* bytes per stored value of this fluid's context (the default for new ones
 * when it has none) */
int tcgpu_get_storage(const fluid_t * fluid);

/* logging quantities of src/logging/*.c from the device state:
 * out[0] max |div u|, out[1..2] energy injection (momentum, scalar),
 * out[3..4] dissipation (momentum, scalar), out[5..8] total energy
 * (ux, uy, uz, scalar). Injection and dissipation use the velocity-gradient
 * tensors of the current fields. */
int tcgpu_diagnostics(const domain_t * domain, fluid_t * fluid, double out[9]);

/* The same nine quantities with the reference's logging semantics
 * (src/logging/main.c after integrate()): momentum injection and dissipation
 * use the velocity-gradient tensors of the last predict's input fields, which
 * is what src/fluid/predict/main.c:56-82 leaves in fluid_t for
 * src/logging/injection.c:49-51 and dissipation.c; the wall velocity, the
 * scalar terms, the divergence and the energies use the current fields.
 * Before any predict, the tensors of the current fields. */
int tcgpu_log_quantities(const domain_t * domain, fluid_t * fluid, double out[9]);

/* Statistics of src/statistics.c:124-240 accumulated on the device (no
 * counterpart entry points in the reference, which accumulates on the host).
 * collect: adds one sample from the current fields (ux1, ux2, uy1, uy2, uz1,
 * uz2, adv) and, for dif = lyx0 + lyx1 + lxy, from the fields the reference's
 * tensors belong to (those of tcgpu_log_quantities); the accumulators are
 * allocated on the first call. reset: zero them and the sample count. get:
 * *num = samples so far, out[s] (host arrays, NULL to skip) = accumulator s in
 * the order ux1 ux2 uy1 uy2 uz1 uz2 adv dif, laid out [k][j][i] over the
 * interior j, k with i = 1..nx+1 (ux1, ux2, adv, dif: nx+1 values per row) or
 * i = 0..nx+1 (uy1, uy2, uz1, uz2: nx+2). save: the reference's statistics
 * directory (src/statistics.c:250-300): num.npy, the domain, and the eight
 * arrays with those shapes (nothing is written when no sample was collected).
 * mean_uy: profile[i], i = 0..nx+1, = mean of uy over j, k and the samples. */
/* A seeded initial field generated on the device, in place of fluid_init for
 * grids whose NPY files would be large (no counterpart in the reference, whose
 * initial_condition/main.py writes NPY files). Allocates the fluid_t arrays as
 * fluid_init does (Re and Pr from the environment), creates the device context
 * and fills it: uy the laminar profile (circular Couette A r + B / r between
 * the wall speeds of tcgpu_set_params when the domain is curved, linear when
 * planar), t linear between its wall values, p = 0, plus uniform noise in
 * [-noise_u, noise_u) on ux (interior faces), uy and uz and in
 * [-noise_t, noise_t) on t; each value's noise depends only on the seed, the
 * field and the cell. Boundary values and periodic images as after fluid_init;
 * the caller's host arrays receive the same field. */
typedef struct {
  uint64_t seed;
  double noise_u, noise_t;
} tcgpu_ic_t;
int tcgpu_fluid_init_generated(const domain_t * domain, fluid_t * fluid, const tcgpu_ic_t * ic);

/* Values of one field (TCGPU_UX ... TCGPU_T) at the radial indices i0 ..
 * i0 + count - 1 of the reference's index space (ux: faces 1 .. nx+1, the
 * others 0 .. nx+1) over the interior j, k of the current device state, into
 * the host array out[((k - 1) ny + j - 1) count + c]. No counterpart in the
 * reference; for wall-layer diagnostics that need a few radial planes without
 * copying the whole field. */
int tcgpu_radial_slab(const domain_t * domain, fluid_t * fluid, unsigned field, int i0, int count, double * out);

int tcgpu_statistics_collect(const domain_t * domain, fluid_t * fluid);
int tcgpu_statistics_reset(const domain_t * domain, fluid_t * fluid);
int tcgpu_statistics_get(const domain_t * domain, fluid_t * fluid, size_t * num, double * const out[8]);
int tcgpu_statistics_save(const char dirname[], const domain_t * domain, fluid_t * fluid);
int tcgpu_statistics_mean_uy(const domain_t * domain, fluid_t * fluid, double * profile);

/* Allocation-free variant of tdm.solve(). No counterpart in the reference.
 * For callers that cannot allocate device memory or let a library do it: a
 * framework that owns the whole device memory pool and forbids other
 * allocators, a real-time host that reserves all device memory at start-up and
 * may not allocate afterwards, or a plugin whose allocations belong to someone
 * else. The elimination factors go to a fixed static device array of
 * 4 * TCGPU_TDM_NOALLOC_MAX_SIZE doubles (256 KiB) that every GPU which loads
 * this library holds until the process exits; nothing is cudaMalloc'd or freed.
 * l, c, u: host arrays of length size (lower, centre, upper diagonals as in
 * tdm.get_l/get_c/get_u); data: device memory of the current device with nrhs
 * right-hand sides of length size, contiguous (interleaved re/im when
 * is_complex), solved in place with the same arithmetic as tdm.solve(). size
 * must lie in [1, TCGPU_TDM_NOALLOC_MAX_SIZE] ([3, ...] when periodic); larger
 * systems, host memory and memory of another device are rejected with a
 * non-zero return. The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current. The work runs on the
 * legacy default stream and the call returns only once it has finished, so data
 * must be complete before the call: synchronise the stream that wrote it when
 * that stream does not synchronise with the legacy default stream (a
 * non-blocking stream, or per-thread default streams). All calls share the one
 * array and each rewrites every entry it reads; calls whose kernels could
 * overlap on the GPU (other threads, other streams) would race on it, so this
 * library serialises its own calls and synchronises before returning. */
#define TCGPU_TDM_NOALLOC_MAX_SIZE 8192
int tcgpu_tdm_solve_noalloc(int size, int nrhs, bool is_periodic, bool is_complex, const double * l,
                            const double * c, const double * u, double * data);

/* Self-test of the bounded waits inside the kernels. No counterpart in the
 * reference. Runs one block whose mbarrier wait can never complete (it expects
 * bytes no copy delivers): the wait must give up after its limit (about two
 * seconds of SM clock), the kernel report it and return, and the device stay
 * usable. Returns 0 when that happened; *seconds (if not NULL) = elapsed time. */
int tcgpu_selftest_wait(double * seconds);

/* free the device state that belongs to this fluid_t */
int tcgpu_release(fluid_t * fluid);

/* ---- learned closure: grid side --------------------------------------------
 * No counterpart in the reference. A coarse solver (its own fluid_t, a grid 4x
 * coarser in every direction whose radial faces are every 4th fine face)
 * takes a forcing, predicted by a 3x3x3 convolutional network from its own
 * state, that is added to the explicit terms of ux, uy, uz in every predict.
 * All coarse contexts need 8-byte storage. */
/* the CUDA stream of this fluid's device context (network kernels launched on
 * it stay ordered with the solver's own work) */
void * tcgpu_stream(const domain_t * domain, fluid_t * fluid);
/* restrict the fine device state to the coarse one: face fluxes summed (the
 * restriction keeps a divergence-free field divergence-free), t and p volume
 * means; walls and periodic images applied. Synchronous. */
int tcgpu_coarsen(const domain_t * fine_domain, fluid_t * fine, const domain_t * coarse_domain, fluid_t * coarse);
/* network input of this fluid's device state, asynchronous on its stream:
 * BF16 [cell][cp] (cp a multiple of 16), channels ux at the centre / scale[0],
 * uy / scale[1], uz / scale[2], radial index coordinate in [-1, 1], zeros */
int tcgpu_closure_input(const domain_t * domain, fluid_t * fluid, const double scale[3], int cp, void * out);
/* training target of one sample, synchronous: out[cell][3] =
 * (reference - predicted) / tau for ux (channel 0 of cell i = face i + 1 of
 * the reference's numbering), uy, uz; both fluids on the same coarse grid */
int tcgpu_closure_target(const domain_t * domain, fluid_t * predicted, fluid_t * reference, double tau, float * out);
/* f (FP32 [cell][nc], device) times scale becomes the forcing of every
 * following predict of this fluid (asynchronous on its stream); f = NULL turns
 * the forcing off */
int tcgpu_set_forcing(const domain_t * domain, fluid_t * fluid, const float * f, int nc, const double scale[3]);

/* ---- learned closure: network kernels --------------------------------------
 * No counterpart in the reference. Device pointers, asynchronous on the given
 * CUDA stream (NULL: the legacy default stream). Activations are channels-last
 * BF16 over the interior cells of a grid (nx, ny, nz), act[((k ny + j) nx + i)
 * C + c], C in {16, 32}; x is zero-padded, y and z periodic. All buffers
 * 16-byte aligned; nx a multiple of 8, ny of 16.
 *
 * Weights: FP32 master copy w[t][co][ci] (t = 9 (dz+1) + 3 (dy+1) + (dx+1),
 * real channel counts) packed into BF16 images for the forward convolution
 * (fwd, 27 cinp coutp values) and, if bwd != NULL, for the input-gradient
 * convolution (taps mirrored, channels swapped). */
int tcgpu_nn_pack_weights(const float * w, int cin, int cout, int cinp, int coutp, void * fwd, void * bwd,
                          void * stream);
/* 3x3x3 convolution on the tensor cores (BF16 operands, FP32 accumulation).
 * mode 0: out = GELU(conv(in) + bias) (BF16, cout channels), pre = conv(in) +
 *         bias (BF16, optional, kept for the backward pass);
 * mode 1: outf[cell][c] = conv(in) + bias for c < nout (FP32);
 * mode 2: out = conv(in) * GELU'(zsave) (input gradient through the layer
 *         below; in = the gradient of this layer's pre-activation, wpacked =
 *         the bwd image, cin/cout = this layer's cout/cin). */
int tcgpu_nn_conv3(int mode, int cin, int cout, int nx, int ny, int nz, const void * in, const void * wpacked,
                   const float * bias, const void * zsave, void * out, void * pre, float * outf, int nout,
                   void * stream);
/* weight gradient of a convolution: dw[t][co][ci] (real counts cin x cout,
 * FP32) = sum over cells of x[cell + tap t][ci] dy[cell][co], db[co] = sum of
 * dy[cell][co]; beta 0 overwrites dw/db, 1 accumulates. x has cinp channels,
 * dy coutp (padded counts, 16 or 32). workspace: device scratch of at least
 * tcgpu_nn_wgrad_workspace() bytes. */
size_t tcgpu_nn_wgrad_workspace(int nx, int ny, int nz, int coutp);
int tcgpu_nn_conv3_wgrad(int cinp, int coutp, int cin, int cout, int nx, int ny, int nz, const void * x,
                         const void * dy, float * dw, float * db, float beta, void * workspace, size_t ws_bytes,
                         void * stream);
/* mean squared error of f against t (FP32 [cell][nc], optional per-cell
 * weight w): *loss += mean w (f - t)^2; grad (BF16 [cell][cp]) = its
 * gradient with respect to f, zero in channels nc .. cp-1 */
int tcgpu_nn_mse(const float * f, const float * t, const float * w, size_t ncell, int nc, int cp, void * grad,
                 double * loss, void * stream);
/* one Adam step on n FP32 parameters p with gradients g and moments m, v;
 * step = 1, 2, ... (bias correction) */
int tcgpu_nn_adam(float * p, const float * g, float * m, float * v, size_t n, float lr, float beta1, float beta2,
                  float eps, int step, void * stream);
/* error bits raised by the network kernels since the last clear (4: a wait
 * gave up); synchronises the device; -1 on a CUDA error */
int tcgpu_nn_status(int clear);
/* last error message of the network entry points of this thread */
const char * tcgpu_nn_last_error(void);

/* last error message of this thread ("" when none) */
const char * tcgpu_last_error(void);

#if defined(__cplusplus)
}
#endif

#endif // TCGPU_H
