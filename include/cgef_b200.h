/*
 * cgef_b200.h -- C ABI of the B200 coarse-graining library (libcgef_b200.so).
 *
 * Drop-in replacement for the real-space hot path of jbphyswx/CoarseGrainingEnergyFluxes.jl:
 * the footprint filter behind `Filtering.plan_filter` / `filter_apply!` / `filter_apply_batch!`,
 * the strain stencils of `Derivatives.ddx!`/`ddy!`, the flux `Diagnostics.compute_Π!`, the
 * area-weighted `cumulative_energy!`, and the scale-by-slice sweep of `Pipeline.coarse_grain!` /
 * `coarse_grain_batch!` / `coarse_grain_slices!`.  Every entry point below names the reference
 * interface it replaces (file:line in the reference repository).
 *
 * Conventions
 *  - Fields are the reference's column-major (Nx, Ny[, batch...]) arrays, i.e. C row-major
 *    [batch][ny][nx] with the x (longitude) index fastest.
 *  - Host-buffer entry points (`cgef_filter`, `cgef_compute_pi`, ...) are synchronous and copy
 *    through device memory owned by the plan; `*_device` entry points take device pointers and a
 *    cudaStream_t (passed as void*) and return without synchronising.
 *  - All calls return CGEF_OK (0) or a negative status; `cgef_last_error()` gives the message of
 *    the calling thread's last failure.
 *  - A plan is used by one host thread at a time (the reference's "one plan per task",
 *    Derivatives.jl:74-77); different plans may run concurrently.  A plan's device work is ordered
 *    on one stream at a time: its scratch and the work queue of its direct gather are the plan's
 *    own, so `*_device` calls of one plan on two streams must not overlap on the GPU.
 *  - Arithmetic is FP64 on the device: footprint sums accumulate with double-precision FMA and
 *    the subtraction tau = (uu)bar - ubar ubar, the normalisation and the energy reductions are
 *    FP64.  `dtype` selects only the storage type of inputs and outputs.
 */
#ifndef CGEF_B200_H
#define CGEF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CGEF_ABI_VERSION 1

/* Status codes. */
enum {
  CGEF_OK = 0,
  CGEF_EINVAL = -1,       /* bad shape / argument: ArgumentError, DimensionMismatch in the reference */
  CGEF_ENOMEM = -2,       /* device or host allocation failed */
  CGEF_ECUDA = -3,        /* a CUDA runtime call failed */
  CGEF_ESTRATEGY = -4,    /* plan built for another mask strategy (Filtering.jl:952-965, 1484-1503) */
  CGEF_EUNSUPPORTED = -5, /* combination outside the supported path */
  CGEF_ENODEVICE = -6,    /* no CUDA device visible */
  CGEF_ETIMEOUT = -7      /* a bounded device-side wait ran out (the call's results are not valid) */
};

/* Geometry (FlowGeometries.Geometry.CartesianGeometry / SphericalGeometry). */
enum { CGEF_CARTESIAN = 0, CGEF_SPHERICAL = 1 };
/* Kernels (Kernels.jl:28 TopHatKernel, :59-62 GaussianKernel). */
enum { CGEF_TOPHAT = 0, CGEF_GAUSSIAN = 1 };
/* Mask strategies (Filtering.jl:36-48 ZeroFill, :50-57 Deformable). */
enum { CGEF_ZEROFILL = 0, CGEF_DEFORMABLE = 1 };
/* Engines: AUTO dispatches as the reference does (Filtering.jl:636-749, 1121-1141, 1533-1561):
 * Gaussian on Cartesian -> SEPARABLE, top-hat -> PREFIXSUM, otherwise BANDED.
 * SPECTRAL is the reference's `method = Spectral()` (plan_filter, Filtering.jl:2944-2946, with the FFTW
 * extension's plan, ext/CoarseGrainingEnergyFluxesFFTWExt.jl:121-206): a periodic convolution by the
 * kernel's isotropic transfer function, so only on a Cartesian grid periodic along both axes
 * (CGEF_EINVAL otherwise, Filtering.jl:2998-3004).  A field f filters to
 *     IDFT2(Ghat(|k|, l) * DFT2(mask * f)),  Ghat = exp(-k^2 l^2 / (4 alpha)) (Gaussian),
 *                                            2 J1(k l / 2) / (k l / 2) (top-hat, 1 at k = 0),
 * with kx = 2 pi m / (nx dx), ky = 2 pi m' / (ny dy) on the rfft / fft frequency grids (Kernels.jl:394-406).
 * ZeroFill stops there; Deformable multiplies by 1 / filter(mask) where |filter(mask)| >= 0.01 and by 0
 * elsewhere (FFTWExt.jl:163-173), on a grid with masked cells.  Unlike the real-space engines the output
 * is defined on every cell, masked ones too (FFTWExt.jl:184-206).  CGEF_EUNSUPPORTED unless nx is even,
 * nx / 2 and ny have no prime factor above 5, and both are at most 4096. */
enum { CGEF_ENGINE_AUTO = 0, CGEF_ENGINE_BANDED = 1, CGEF_ENGINE_SEPARABLE = 2, CGEF_ENGINE_PREFIXSUM = 3,
       CGEF_ENGINE_SPECTRAL = 4 };
/* Storage types of caller buffers. */
enum { CGEF_F64 = 0, CGEF_F32 = 1 };

/* A uniform 2-D structured grid (FlowGeometries.Grids.StructuredGrid over two ranges).
 * Coordinates: x_i = x0 + i*dx, y_j = y0 + j*dy, evaluated as fma(i, dx, x0); radians on the
 * sphere (x = longitude, y = latitude).  `mask` is host memory, ny*nx bytes, nonzero = active
 * (NULL = every cell active); it is copied at plan creation. */
typedef struct cgef_grid_desc {
  int32_t geometry;
  int32_t periodic_x;
  int32_t periodic_y;
  int32_t reserved;
  int64_t nx;
  int64_t ny;
  double x0, dx, y0, dy;
  double radius; /* sphere radius in metres (ignored on the plane) */
  const uint8_t* mask;
} cgef_grid_desc;

typedef struct cgef_plan cgef_plan;

typedef struct cgef_plan_info {
  int32_t engine;     /* CGEF_ENGINE_* actually built */
  int32_t nbands;     /* banded: 1 (Cartesian) or ny (sphere); 0 otherwise */
  int64_t nentries;   /* banded: footprint entries summed over bands */
  int32_t dj_lim;     /* row half-width of the footprint */
  int32_t di_max;     /* widest column half-width over all bands (banded/separable) */
  double kernel_radius;
  double active_area; /* sum of active-cell areas of the plan's grid mask */
} cgef_plan_info;

/* Optional outputs of the flux computation; every non-NULL buffer holds nbatch*ny*nx values of
 * the call's dtype, except `energy` (nbatch doubles).  Local-frame components on the sphere
 * (east/north), Diagnostics.jl:596-650. */
typedef struct cgef_pi_outputs {
  void* pi;      /* -(Sxx tau_xx + 2 Sxy tau_xy + Syy tau_yy) on active cells, else 0 (no rho0) */
  void* ubar;
  void* vbar;
  void* tau_xx;
  void* tau_xy;
  void* tau_yy;
  void* s_xx;
  void* s_xy;
  void* s_yy;
  double* energy; /* E = 1/2 <|ubar|^2>, area weighted over active cells (Diagnostics.jl:1086-1134) */
} cgef_pi_outputs;

/* Library/ABI version (CGEF_ABI_VERSION). */
int32_t cgef_version(void);

/* Message of the calling thread's last failed call ("" if none). */
const char* cgef_last_error(void);

/* Number of visible CUDA devices (0 when none; never fails). */
int32_t cgef_device_count(void);

/* The device architecture the library's kernels are compiled for, in __CUDA_ARCH__ form: 1000 for
 * sm_100a (the build refuses any other target).  No device needed. */
int32_t cgef_build_arch(void);

/* Filtering.plan_filter (Filtering.jl:2931-2954) plus the GPU extension's prepare_workspace
 * upload (Filtering.jl:2910-2912; ext/CoarseGrainingEnergyFluxesKernelAbstractionsExt.jl:474-571):
 * builds the engine's tables on the host once and keeps them resident on the current device.
 * scale must be finite and positive (Filtering.jl:2917-2922). */
int32_t cgef_plan_create(cgef_plan** out, const cgef_grid_desc* grid, int32_t kernel, double alpha, double scale,
                         int32_t mask_strategy, int32_t engine);

/* Releases the plan's device and host memory. */
int32_t cgef_plan_destroy(cgef_plan* plan);

/* Zeroes the work queue of the plan's direct gather, synchronously (no counterpart in the reference,
 * whose loops have no queue).  Each gather launch takes its work items from this queue and the last
 * warp to leave zeroes it; a launch that stopped part-way would leave it mid-count, so every launch
 * also zeroes it first (stream-ordered) and a stale queue never reaches a later launch.  This call is
 * for a host that wants the queue clean at once. */
int32_t cgef_plan_reset_queue(cgef_plan* plan);

/* Plan statistics. */
int32_t cgef_plan_get_info(const cgef_plan* plan, cgef_plan_info* info);

/* Where the banded engine builds a spherical footprint on a periodic longitude axis (no counterpart in
 * the reference, which builds on the CPU, Filtering.jl:675-731).  The host always decides the entry
 * set with its libm, as the reference's loop does: per (band, row offset) the great-circle distance
 * grows with |di|, so it bisects for the last included offset and tests the four either side of it
 * (a row where rounding breaks that order is built entirely on the host).  With the device build, the
 * weights of those entries (one exp per |di|, from the host's row constants) and the ZeroFill
 * denominators are computed on the GPU: the same entries as a host build, weights within a few ulps
 * of it, denominators summed in another order.  CGEF_BUILD_AUTO (the default) takes the device build
 * once a footprint holds about 2e6 half-row weights.  Applies to plans created afterwards, from any
 * thread. */
enum { CGEF_BUILD_AUTO = 0, CGEF_BUILD_HOST = 1, CGEF_BUILD_DEVICE = 2 };
int32_t cgef_set_footprint_build(int32_t where);
/* CGEF_BUILD_DEVICE if the plan's footprint weights were computed on the device, else CGEF_BUILD_HOST. */
int32_t cgef_plan_get_build(const cgef_plan* plan, int32_t* where);

/* Schedule autotuner of the banded engine (no counterpart in the reference, whose loops have no
 * schedule).  Times the flux's footprint sums on this plan's grid and mask (zero-valued inputs; their
 * cost depends on the footprint and the mask, not on the values): first the row-spectral evaluation
 * (where the plan has it) and the direct gather at its current granularity.  When the direct gather is
 * more than twice slower the spectral evaluation is kept and nothing else is timed.  Otherwise each
 * candidate split granularity of the direct gather -- the work-item schedule cut into about 2, 4, 8 or
 * 16 rounds of resident warps per SM -- is timed and the fastest kept (`chosen`, may be NULL, receives
 * it); a three-field filter pass is timed with 4- and 8-row tiles and the faster kept for the filter
 * passes; and the faster of the two evaluations is kept.  A no-op for the separable and prefix engines.
 * Results stay within FP64 rounding of each other across schedules: only the order in which a split
 * tile's partial sums are added changes. */
int32_t cgef_plan_autotune(cgef_plan* plan, int32_t nbatch, double* chosen);
/* Sets the split granularity directly (rounds of resident warps per SM, > 0; the default is 4). */
int32_t cgef_plan_set_split_waves(cgef_plan* plan, double waves);
/* Tile height of the banded engine's filter passes (cgef_filter*, cumulative energy, the closure's and
 * the decompositions' gathers): 4 or 8 target rows per thread (the flux always uses 4).  The autotuner
 * also chooses it, timing a three-field pass.  Results are identical either way up to FP64 rounding of
 * split tiles' partial sums. */
int32_t cgef_plan_set_filter_rows(cgef_plan* plan, int32_t rows);
/* The plan's current schedule: split granularity of the flux gather and the filters' tile height
 * (both 0 off the banded engine). */
int32_t cgef_plan_get_schedule(const cgef_plan* plan, double* waves, int32_t* filter_rows);

/* Row-spectral evaluation of the banded engine's sums (no counterpart in the reference, which sums
 * the footprint directly, Filtering.jl:1569-1744, 2536-2598).  For a target row and a row offset the
 * footprint weights depend only on the column offset, so each such term is a correlation along x;
 * with an FFT along x of every source row's accumulated quantities, the band's kernel spectra
 * applied and summed per target row, and an inverse FFT, the plan computes the same sums at a cost
 * linear, not quadratic, in the footprint's reach.  Results equal the direct sums up to FP64
 * rounding of the transforms, and each quantity is transformed on its own, so batched applies stay
 * bit-identical to per-field ones.  Available on a periodic x axis (FFT length Nx) or with symmetric
 * rows on a bounded one (a zero-padded length >= Nx + the widest half-width), when the length is even
 * and its half has no prime factor above 5, and when the device has room for the plan's kernel spectra
 * (8 bytes per band row and bin; 1.5 GB at 2000 km on the 0.25° sphere); built with the plan and enabled
 * by default when available;
 * cgef_plan_autotune keeps whichever evaluation times faster for the flux.  Work-item subsets (the
 * closure's judge) and cgef_filter_device_noalloc always sum directly. */
int32_t cgef_plan_set_row_spectral(cgef_plan* plan, int32_t enable);
/* available: the plan can use it; enabled: full-grid launches use it; fft_length: its FFT length
 * along x (0 when unavailable).  Any pointer may be NULL. */
int32_t cgef_plan_get_row_spectral(const cgef_plan* plan, int32_t* available, int32_t* enabled,
                                   int32_t* fft_length);

/* A spectral-method plan's transfer function Ghat(|k|, l) on the rfft grid, the FFTW plan's `transfer`
 * array (FFTWExt.jl:146): transfer[ky * (nx/2 + 1) + kx], ny * (nx/2 + 1) values, ky in fftfreq order.
 * CGEF_EINVAL for a real-space plan. */
int32_t cgef_plan_get_transfer(const cgef_plan* plan, double* transfer);

/* Banded footprint of the plan in the reference's CSR form (FilterFootprint, Filtering.jl:327-336):
 * di/dj/w have nentries entries, ptr has nbands+1 (0-based offsets).  Any pointer may be NULL. */
int32_t cgef_plan_get_footprint(const cgef_plan* plan, int32_t* di, int32_t* dj, double* w, int64_t* ptr);

/* Filtering.filter_apply! (Filtering.jl:3242-3256) and filter_apply_batched! over a trailing
 * batch axis (Filtering.jl:3286-3305), replacing gpu_filter_field! / gpu_filter_field_batched!
 * (Filtering.jl:195-197, 3342-3344).  field/out: nbatch*ny*nx host values of dtype. */
int32_t cgef_filter(cgef_plan* plan, int32_t dtype, const void* field, void* out, int64_t nbatch);

/* Filtering.filter_apply_batch! (Filtering.jl:3360-3375): k separate fields through one
 * footprint traversal.  fields[m]/outs[m]: ny*nx host values of dtype. */
int32_t cgef_filter_batch(cgef_plan* plan, int32_t dtype, const void* const* fields, void* const* outs, int32_t k);

/* Diagnostics.compute_Π! for a 2-D StructuredGrid (Diagnostics.jl:389-416, 472-702), batched over
 * nbatch slices sharing the grid (the batch-native driver, Pipeline.jl:519-563).  slice_masks is
 * NULL (use the plan's grid mask) or nbatch*ny*nx host bytes, one mask per slice
 * (coarse_grain_slices!, Pipeline.jl:866-904). */
int32_t cgef_compute_pi(cgef_plan* plan, int32_t dtype, const void* u, const void* v, int64_t nbatch,
                        const uint8_t* slice_masks, const cgef_pi_outputs* out);

/* Diagnostics.compute_Π! with the vertical velocity w (the 2.5-D path: `w::AbstractArray` in
 * Diagnostics.jl:389-416, its terms at 254-260 and 483-681).  u, v, w: nbatch*ny*nx values of dtype.
 * The plane filters u, v, w and the products uu, uv, vv, uw, vw, ww; the sphere takes w along the local
 * up vector into the planetary velocity (vector_to_cartesian), filters its 3 components and 6
 * products, and rotates back to east/north/up in full.  tau gains its xz, yz, zz (east-up, north-up,
 * up-up) components; the strain S_xz = 1/2 dwbar/dx, S_yz = 1/2 dwbar/dy and S_zz = 0 (layers flat in
 * the vertical, no curvature terms); Pi = -(Sxx txx + 2 Sxy txy + Syy tyy + 2 Sxz txz + 2 Syz tyz +
 * Szz tzz) on active cells.  E = 1/2 <ubar^2 + vbar^2 + wbar^2>.  Every non-NULL output holds
 * nbatch*ny*nx values of dtype (energy: nbatch doubles).  slice_masks as in cgef_compute_pi. */
typedef struct cgef_pi_w_outputs {
  void* pi;
  void* ubar;
  void* vbar;
  void* wbar;
  void* tau_xx;
  void* tau_xy;
  void* tau_yy;
  void* tau_xz;
  void* tau_yz;
  void* tau_zz;
  void* s_xx;
  void* s_xy;
  void* s_yy;
  void* s_xz;
  void* s_yz;
  double* energy;
} cgef_pi_w_outputs;
int32_t cgef_compute_pi_w(cgef_plan* plan, int32_t dtype, const void* u, const void* v, const void* w, int64_t nbatch,
                          const uint8_t* slice_masks, const cgef_pi_w_outputs* out);
int32_t cgef_compute_pi_w_device(cgef_plan* plan, int32_t dtype, const void* u, const void* v, const void* w,
                                 int64_t nbatch, const uint8_t* slice_masks, const cgef_pi_w_outputs* out,
                                 void* stream);

/* Diagnostics.cumulative_energy! (Diagnostics.jl:1144-1217): u, v (ny*nx, dtype) filtered as
 * scalars at every plan's scale; spectrum[s] = 1/2 <|ubar|^2>.  All plans share one grid. */
int32_t cgef_cumulative_energy(cgef_plan* const* plans, int32_t nscales, int32_t dtype, const void* u,
                               const void* v, double* spectrum);

/* Pipeline.coarse_grain! / coarse_grain_batch! / coarse_grain_profile! (Pipeline.jl:412-468,
 * 686-717, 991-1007): Pi and E(l) for every (slice, scale).  pi: NULL or
 * nbatch*nscales*ny*nx values of dtype ([slice][scale][ny][nx], the reference's trailing
 * (Nscales, batch) axes); energy: NULL or nbatch*nscales doubles ([slice][scale]). */
int32_t cgef_sweep(cgef_plan* const* plans, int32_t nscales, int32_t dtype, const void* u, const void* v,
                   int64_t nbatch, const uint8_t* slice_masks, void* pi, double* energy);

/* Derivatives.ddx! / ddy! (Derivatives.jl:42-51, 141-142): 3-node first derivative with the
 * ReduceInRun mask policy and the sphere's metric division; f/out: ny*nx host values of dtype. */
int32_t cgef_ddx(cgef_plan* plan, int32_t dtype, const void* f, void* out);
int32_t cgef_ddy(cgef_plan* plan, int32_t dtype, const void* f, void* out);

/* Device-pointer forms of the calls above: same semantics, buffers in device memory of the
 * plan's device, work queued on `stream` (a cudaStream_t; NULL = legacy default stream). */
int32_t cgef_filter_device(cgef_plan* plan, int32_t dtype, const void* field, void* out, int64_t nbatch,
                           void* stream);
int32_t cgef_compute_pi_device(cgef_plan* plan, int32_t dtype, const void* u, const void* v, int64_t nbatch,
                               const uint8_t* slice_masks, const cgef_pi_outputs* out, void* stream);
int32_t cgef_sweep_device(cgef_plan* const* plans, int32_t nscales, int32_t dtype, const void* u, const void* v,
                          int64_t nbatch, const uint8_t* slice_masks, void* pi, double* energy, void* stream);

/* A captured sweep: one cgef_sweep_device call recorded as a CUDA graph and replayed.  No
 * counterpart in the reference (its GPU driver launches per scale).  `create` runs the sweep once on
 * `stream` (sizing every workspace), then captures the same call; each `launch` replays it on the
 * given stream, reading u, v and the masks and writing pi and energy at the captured addresses.  The
 * plans' device tables and workspaces are baked into the graph: keep the plans alive, unchanged
 * (no autotune or other calls on them in between) and unused by other streams while the graph is
 * replayed. */
typedef struct cgef_graph cgef_graph;
int32_t cgef_sweep_graph_create(cgef_graph** out, cgef_plan* const* plans, int32_t nscales, int32_t dtype,
                                const void* u, const void* v, int64_t nbatch, const uint8_t* slice_masks, void* pi,
                                double* energy, void* stream);
int32_t cgef_graph_launch(cgef_graph* graph, void* stream);
int32_t cgef_graph_destroy(cgef_graph* graph);

/* Streaming sweep: the snapshots of a time series submitted one after another from host memory,
 * each copied in, swept over the plans (as cgef_sweep) and its Pi and E copied out, with a
 * snapshot's copies overlapping its neighbours' sweeps (double-buffered device memory, three
 * streams).  The synchronous reference driver loops over snapshots one call at a time
 * (Pipeline.jl:519-563, 686-717); this is that loop with the transfers off the critical path.
 * `submit` returns once the step is queued: u, v (nbatch*ny*nx of dtype), pi (nbatch*nscales*ny*nx,
 * required when the pipeline was created with want_pi) and energy (nbatch*nscales doubles, may be
 * NULL) must stay valid and untouched until `drain` returns; they overlap the GPU's work only when
 * they are pinned host memory.  slice_masks (host, copied at create) as in cgef_sweep.  The plans
 * are used by the pipeline's streams: make no other call on them before `drain`. */
typedef struct cgef_pipeline cgef_pipeline;
int32_t cgef_pipeline_create(cgef_pipeline** out, cgef_plan* const* plans, int32_t nscales, int32_t dtype,
                             int64_t nbatch, const uint8_t* slice_masks, int32_t want_pi);
int32_t cgef_pipeline_submit(cgef_pipeline* pipeline, const void* u, const void* v, void* pi, double* energy);
int32_t cgef_pipeline_drain(cgef_pipeline* pipeline);
int32_t cgef_pipeline_destroy(cgef_pipeline* pipeline);

/* cgef_filter_device without any device allocation.  No counterpart in the reference.
 * For callers that cannot let a library allocate device memory during a call: a host whose device
 * memory is owned by its own pool allocator (a Julia or PyTorch caching allocator, which a library
 * cudaMalloc would bypass and which can leave no memory for it), or a loop with a fixed memory
 * budget.  The scratch is one 64 MiB array compiled into the library, which every GPU that loads
 * the library holds until the process exits; a grid and batch needing more is rejected with
 * CGEF_EINVAL.  The CUDA driver reserves the array on a device, and the library resolves its device
 * address there, when the first plan is created on that device (cgef_plan_create, with that device
 * current), so a call of this entry point never makes the driver reserve memory; create plans before
 * any stream capture.  All calls share the array and it keeps the last call's contents, so calls that
 * overlap on the GPU race: serialise them.  Same arguments and results as cgef_filter_device. */
int32_t cgef_filter_device_noalloc(cgef_plan* plan, int32_t dtype, const void* field, void* out, int64_t nbatch,
                                   void* stream);

/* Diagnostics.tau_decomposition (Diagnostics.jl:1350-1527): tau = Leonard + Cross + Reynolds with
 * generalized central moments M(f, g) = (fg)bar - fbar gbar of ubar and u' = u - ubar (Germano 1992);
 * on the sphere the moments are formed from planetary Cartesian components and each part is rotated
 * to east/north.  One (ny, nx) field pair; each part has xx, xy, yy outputs (ny*nx values of dtype;
 * NULL skips one).  Masked cells give 0. */
typedef struct cgef_tau_parts {
  void* leonard[3];
  void* cross[3];
  void* reynolds[3];
} cgef_tau_parts;
int32_t cgef_tau_decomposition(cgef_plan* plan, int32_t dtype, const void* u, const void* v,
                               const cgef_tau_parts* out);
int32_t cgef_tau_decomposition_device(cgef_plan* plan, int32_t dtype, const void* u, const void* v,
                                      const cgef_tau_parts* out, void* stream);

/* Diagnostics.compute_Π_strain_convergence! (Diagnostics.jl:1724-1852; Srinivasan, Barkan &
 * McWilliams 2023, eq. 10), Cartesian grids: with delta = u_x + v_y, sigma_n = u_x - v_y,
 * sigma_s = u_y + v_x of the filtered velocity, Pi_alpha = (tau_vv - tau_uu) sigma_n / 2 - tau_uv sigma_s,
 * Pi_delta = (tau_vv + tau_uu) delta / 2, total = Pi_alpha - Pi_delta (= compute_Π!'s Pi),
 * strain_magnitude = sqrt(sigma_n^2 + sigma_s^2).  Batched like cgef_compute_pi; NULL skips an
 * output.  CGEF_EUNSUPPORTED on the sphere (the reference defines it on the plane only). */
typedef struct cgef_strain_conv_outputs {
  void* total;
  void* strain;
  void* convergence;
  void* divergence;
  void* strain_magnitude;
} cgef_strain_conv_outputs;
int32_t cgef_pi_strain_convergence(cgef_plan* plan, int32_t dtype, const void* u, const void* v, int64_t nbatch,
                                   const cgef_strain_conv_outputs* out);
int32_t cgef_pi_strain_convergence_device(cgef_plan* plan, int32_t dtype, const void* u, const void* v,
                                          int64_t nbatch, const uint8_t* slice_masks,
                                          const cgef_strain_conv_outputs* out, void* stream);

/* ---- Learned closure.  No counterpart in the reference. ----
 * A pointwise MLP (5 -> 64 -> 64 -> 64 -> 3, GELU) maps the filtered velocity-gradient tensor,
 * scaled by ell^2, and log ell to the subfilter stress tau; the flux is then -S:tau with S from the
 * same gradients.  Weights are BF16 operands of tcgen05 tensor-core MMAs with FP32 accumulation
 * (FP32 master copy, AdamW).  The exact flux path (cgef_compute_pi) generates the training pairs,
 * judges a seeded fraction of every closure result tile by tile and replaces a slice whose judged
 * error exceeds the tolerance.
 *
 * Per grid point at scale ell (g = ell^2 * (S_ee, du/dy, dv/dx + u t, S_nn) in the local frame, n^2 =
 * mean over the slice's active points of |g|^2):
 *   features x = (g / n, (ln ell - ln 223607 m) / 1.4979)         (5 floats)
 *   targets  y = (tau_ee, tau_en, tau_nn) * ell^2 / n^2            (3 floats)
 *   closure  tau = MLP(x) * n^2 / ell^2,  Pi = -(S_ee tau_ee + 2 S_en tau_en + S_nn tau_nn).
 * Parameters (float, CGEF_CLOSURE_NPARAM): W1[64][5] b1[64] W2[64][64] b2[64] W3[64][64] b3[64]
 * W4[3][64] b4[3]. */
typedef struct cgef_closure cgef_closure;
enum { CGEF_CLOSURE_NIN = 5, CGEF_CLOSURE_NHIDDEN = 64, CGEF_CLOSURE_NOUT = 3, CGEF_CLOSURE_NPARAM = 8899 };

typedef struct {
  double lr, beta1, beta2, eps, weight_decay; /* AdamW; weight decay on the weight matrices only */
} cgef_adamw;

typedef struct {
  int64_t judged_tiles; /* 32 x 32 tiles recomputed exactly, summed over slices */
  int64_t failed_tiles; /* judged tiles whose own Pi error exceeded the tolerance */
  double est_rel_l2;    /* largest per-slice Pi rel-L2 error of the closure on its judged tiles */
  int32_t fallbacks;    /* slices recomputed by the exact path */
  int32_t reserved;
} cgef_closure_report;

/* Creates a closure on the current device with uniform(+-1/sqrt(fan_in)) weights from `seed`. */
int32_t cgef_closure_create(cgef_closure** out, uint64_t seed);
int32_t cgef_closure_destroy(cgef_closure* c);
/* Host copies of the FP32 master parameters (CGEF_CLOSURE_NPARAM floats). */
int32_t cgef_closure_get_params(const cgef_closure* c, float* params);
int32_t cgef_closure_set_params(cgef_closure* c, const float* params);

/* Training pairs from the exact flux path on device buffers: features[nbatch][5][ny*nx] and
 * targets[nbatch][3][ny*nx] (FP32, planar); masked points hold zeros. */
int32_t cgef_closure_pairs_device(cgef_plan* plan, int32_t dtype, const void* u, const void* v, int64_t nbatch,
                                  const uint8_t* slice_masks, float* features, float* targets, void* stream);

/* `nsteps` AdamW steps on device pairs x[npoints][5], t[npoints][3]; step k uses the `batch` points
 * from (k * batch) mod npoints (shuffle beforehand).  Loss L = sum_o (y_o - t_o)^2 averaged over the
 * batch; losses[k] receives step k's loss (device buffer, may be NULL). */
int32_t cgef_closure_train_device(cgef_closure* c, const float* x, const float* t, int64_t npoints, int64_t batch,
                                  int32_t nsteps, const cgef_adamw* opt, float* losses, void* stream);

/* Network outputs y[npoints][3] for features x[npoints][5] (device). */
int32_t cgef_closure_forward_device(cgef_closure* c, const float* x, int64_t npoints, float* y, void* stream);

/* Gradient of L over all npoints as one batch, no update: grads[CGEF_CLOSURE_NPARAM] and loss[1]
 * (device). */
int32_t cgef_closure_grad_device(cgef_closure* c, const float* x, const float* t, int64_t npoints, float* grads,
                                 float* loss, void* stream);

/* The flux by the closure at the plan's scale for nbatch slices (device buffers, like
 * cgef_compute_pi_device's pi output).  A seeded `judge_fraction` of the 32 x 32 tiles (at least one)
 * is recomputed by the exact path and written exactly; a slice whose closure error on its judged
 * tiles exceeds `tol` (relative L2) is recomputed entirely by the exact path.  Synchronises
 * `stream` once to read the judge's sums.  `report` may be NULL. */
int32_t cgef_closure_pi_device(cgef_closure* c, cgef_plan* plan, int32_t dtype, const void* u, const void* v,
                               int64_t nbatch, const uint8_t* slice_masks, double judge_fraction,
                               uint64_t judge_seed, double tol, void* pi, cgef_closure_report* report, void* stream);

/* Failure injection for the tests of the failure paths (no counterpart in the reference).  Host side
 * only: it writes one device word with a synchronous copy and never makes a kernel fault or wait.
 * CGEF_INJECT_CLOSURE_TIMEOUT: `object` is a cgef_closure*; its device error word is set as a bounded
 * tensor-core wait that ran out sets it, so its next call returns CGEF_ETIMEOUT (and clears it).
 * CGEF_INJECT_STALE_QUEUE: `object` is a cgef_plan*; its direct gather's work queue is left as a launch
 * that stopped part-way would leave it. */
enum { CGEF_INJECT_CLOSURE_TIMEOUT = 1, CGEF_INJECT_STALE_QUEUE = 2 };
int32_t cgef_debug_inject(void* object, int32_t what);

/* Tracing (no counterpart in the reference, which has none).  Kernel launches made by this
 * thread's calls since the last reset. */
int64_t cgef_launch_count(void);
void cgef_reset_launch_count(void);

/* Per-kernel device timing: while enabled, this thread's calls bracket every launch of the kinds
 * below with CUDA events on the launch's own stream.  `cgef_profile_read` waits for the recorded
 * events and returns the summed duration (ms) and launch count of one kind since the last reset. */
enum { CGEF_KERNEL_STAGE = 0, CGEF_KERNEL_BANDED = 1, CGEF_KERNEL_SEPARABLE = 2, CGEF_KERNEL_PREFIX = 3,
       CGEF_KERNEL_STRAIN = 4, CGEF_KERNEL_CLOSURE = 5, CGEF_KERNEL_ROWSPEC = 6, CGEF_KERNEL_KINDS = 7 };
void cgef_profile_enable(int32_t enable);
int32_t cgef_profile_read(int32_t kind, double* total_ms, int64_t* launches);
void cgef_profile_reset(void);

#ifdef __cplusplus
}
#endif

#endif /* CGEF_B200_H */
