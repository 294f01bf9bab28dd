// Internal declarations shared by the host plan builder, the kernels and the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "cgef_b200.h"

// Every kernel of the library is written for sm_100a (tcgen05, its shared-memory and register
// budgets); cgef_build_arch() reports 1000 on the strength of this guard.
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ != 1000 || !defined(__CUDA_ARCH_FEAT_SM100_ALL))
#error "libcgef_b200 device code is built for sm_100a only"
#endif

namespace cgef {

// Filtering.jl:1633 and every apply path: denominators at or below this give 0.
constexpr double kNormEps = 1e-15;
// Kernels.jl:307: relative weight at which a Gaussian footprint is truncated.
constexpr double kGaussianTruncationTol = 1e-10;

#ifndef CGEF_ROWS
#define CGEF_ROWS 4
#endif
#ifndef CGEF_WARPS
#define CGEF_WARPS 4
#endif
// Target rows carried by one thread of the banded gather (register tile height): the flux's, and
// the taller tile the schedule autotuner may choose for filters of up to four fields.
constexpr int kRows = CGEF_ROWS;
constexpr int kRowsTall = 2 * CGEF_ROWS;
// Warps per CTA of the banded gather; every warp works on its own item.
constexpr int kWarps = CGEF_WARPS;
// Width of the staged planes' column tiling (the pitch is padded to a multiple of this).
constexpr int kTileCols = 160;
// Most slices one launch takes (the grid's z extent of the per-slice kernels).
constexpr int kMaxSlices = 65535;

// One (target band j, source row offset dj) of the banded footprint: weights for longitude
// offsets di in [-a, hi] live at w[woff + |di|] (the sphere's weight is even in di).  a < 0
// means the row holds no entries.  hi is a or, where the band closes the ring on an even
// ring, a - 1 (Filtering.jl:711-713).
struct BandRow {
  int32_t woff;
  int32_t a;
  int32_t hi;
  int32_t pad;
};

// A warp's work item of the banded gather: 32 target columns from x0, kRows target rows from
// j0, and the source rows [jr0, jr1) (raw, possibly outside the grid on a periodic axis).  slot
// is -1 when the item covers every source row and finishes the targets itself; otherwise the
// item writes its partial sums to partial slot `slot` and a combine pass adds the slots of the
// group in order (the heavy polar bands are split this way).
struct WorkItem {
  int32_t x0;
  int32_t j0;
  int32_t jr0;
  int32_t jr1;
  int32_t slot;
  int32_t cost;
};

// A split target tile: its partial slots are [slot0, slot0 + nslots).
struct SplitGroup {
  int32_t x0;
  int32_t j0;
  int32_t slot0;
  int32_t nslots;
};

// A work-item schedule of the banded gather for one tile height `rows` (rows == 0: not built).
struct Schedule {
  int rows = 0;
  std::vector<std::vector<double>> rowcost;  // per target group, per source row (cost model)
  double waves = 4.0;                        // split granularity (rounds of resident warps)
  std::vector<WorkItem> h_items;
  WorkItem* d_items = nullptr;
  std::vector<SplitGroup> h_groups;
  SplitGroup* d_groups = nullptr;
  int nslots = 0;
};

// Per (target row j, source row slot b) of the prefix-sum top-hat sweep (Filtering.jl:974-1097).
struct PrefixRow {
  int32_t jj;    // source row, or -1 when skipped
  int32_t mode;  // 0 skip, 1 whole ring, 2 uniform window +-w, 3 general interval search
  int32_t w;     // half-window in cells (mode 2)
  int32_t pad;
  double hw;     // half-width in axis-1 coordinate units (mode 3)
  double wy;     // row measure factor
};

enum Mode { kModeFields = 0, kModePiCart = 1, kModePiSphere = 2 };

struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace cgef

struct cgef_plan {
  int device = 0;
  // grid
  int geometry = 0, nx = 0, ny = 0, periodic_x = 0, periodic_y = 0;
  double x0 = 0, dx = 0, y0 = 0, dy = 0, R = 0;
  std::vector<uint8_t> h_mask;  // empty = all active
  bool masked = false;
  double active_area = 0;
  // filter
  int kernel = 0, strategy = 0, engine = 0;
  double alpha = 0, scale = 0, rad = 0;
  // host tables kept for introspection
  std::vector<double> h_x, h_y;
  std::vector<cgef::BandRow> h_rows;  // banded: per (band, row offset) intervals
  std::vector<double> h_whalf;        // banded: weights by |di| (empty when built on the device)
  int64_t nwhalf = 0;                 // banded: half-row weights (d_w's length)
  bool built_on_device = false;       // banded: weights and denominators computed by device_band_tables
  std::vector<int64_t> h_ptr;         // banded: CSR band offsets of the reference's layout
  int64_t nentries = 0;
  int dj_lim = 0, di_max = 0;
  // device geometry tables
  uint8_t* d_mask = nullptr;
  double* d_x = nullptr;       // nx coordinates
  double* d_sinlam = nullptr;  // nx
  double* d_coslam = nullptr;  // nx
  double* d_sinphi = nullptr;  // ny
  double* d_cosphi = nullptr;  // ny
  double* d_area = nullptr;    // ny: cell measure of row j
  double* d_xscale = nullptr;  // ny: d/dx metric factor (1/(R cos phi) on the sphere, 0 at the pole guard)
  double* d_tanfac = nullptr;  // ny: sin(phi)/(R cos phi) curvature factor (0 where |cos phi| <= 1e-12)
  // banded engine
  int D = 0;           // row half-width
  int H = 0;           // column halo of the padded planes
  int Amax = 0;        // widest column half-width over all rows
  cgef::BandRow* d_rows = nullptr;  // ny * (2D+1)
  double* d_w = nullptr;            // weights, half rows
  double* d_den_zf = nullptr;       // ZeroFill denominator: ny (periodic x) or ny*nx
  int den_zf_2d = 0;
  cgef::Schedule sched[2];  // [0]: kRows-row tiles (every mode), [1]: kRowsTall rows (filters, when built)
  int filter_rows = CGEF_ROWS;  // tile height of the filter passes (kModeFields)
  bool paired = false;          // the gather adds mirrored columns first (weights even in the offset)
  // row-spectral evaluation of the same sums: each (target row, row offset) term is a correlation
  // along x, done as a product of ring spectra
  int rs_L = 0;                 // FFT length along x; 0 = not available for this plan
  int rs_nk = 0;                // spectrum bins kept, rs_L / 2 + 1
  int rs_nkp = 0;               // row stride of the spectra in bins: rs_nk rounded up to 32
  int rs_nrad = 0;              // Stockham passes
  int rs_rad[16] = {};          // their radices (2, 3, 4 or 5)
  double* d_rs_tw = nullptr;    // rs_L twiddles exp(-2 pi i n / rs_L), (re, im) pairs
  double* d_rs_k = nullptr;     // kernel spectra / rs_L: [band][row offset][bin < rs_nkp], zero past rs_nk
  double* d_rs_ptw = nullptr;   // per-pass twiddles, pass p at rs_poff[p] (complex), [r - 1][jm]
  int rs_poff[16] = {};
  bool rs_on = false;           // full-grid banded launches use the row-spectral evaluation
  // spectral method (CGEF_ENGINE_SPECTRAL): the x transforms are the row-spectral ones above with
  // rs_L = nx (no kernel spectra); the y transforms are complex FFTs of length ny over the bins
  int sp_nrad = 0;
  int sp_rad[16] = {};
  int sp_poff[16] = {};
  double* d_sp_ptw = nullptr;   // per-pass twiddles of the length-ny FFT, pass p at sp_poff[p]
  double* d_sp_T = nullptr;     // transfer function / (nx ny): [ky row][rs_nkp bins], zero past rs_nk
  std::vector<double> h_sp_T;   // the transfer function itself, [ky row][rs_nk bins]
  // separable engine
  int di_lim = 0, sep_dj_lim = 0;
  double* d_gx = nullptr;
  double* d_gy = nullptr;
  double* d_px = nullptr;
  double* d_py = nullptr;
  // prefix-sum engine
  int pre_nrep = 1, pre_ne = 0, pre_nb = 0;
  double x_period = 0, y_period = 0;
  double* d_xe = nullptr;         // ne extended coordinates
  double* d_prefix_wx = nullptr;  // ne + 1
  cgef::PrefixRow* d_prows = nullptr;  // ny * nb
  // execution
  cudaStream_t stream = nullptr;
  cgef::DeviceBuffer ws[13];  // workspace slots (cgef::WsSlot), grown on demand
  unsigned long long* d_queue = nullptr;  // banded work queue: [next unit, warps finished], zero between launches
};

namespace cgef {

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

double kernel_weight(int kernel, double alpha, double d, double ell);
double kernel_radius(int kernel, double alpha, double ell);

// Host plan construction (plan_build.cpp).
int build_plan_tables(cgef_plan* p);
// Where later plans build large spherical footprints (CGEF_BUILD_*; process-wide).
int set_footprint_build(int where);

// Device part of a large spherical footprint build (plan_device.cu): with the plan's rows (a, hi, woff)
// decided and uploaded (d_rows), computes the half-row weights into d_w (nweights) from the host's row
// constants -- sdp = sin((phi' - phi) / 2), cc = cos(phi) cos(phi'), area = the row's cell measure, per
// row -- and sdl[k] = sin(k dlambda / 2); copies the rows the host built itself (woff, weights) over
// them; then the ZeroFill denominators per band into d_den_zf (periodic x).
int device_band_tables(cgef_plan* p, const std::vector<double>& sdp, const std::vector<double>& cc,
                       const std::vector<double>& area, const std::vector<double>& sdl, size_t nweights,
                       const std::vector<std::pair<int64_t, std::vector<double>>>& host_rows);

// Sets the closure's device error word from the host, as a bounded wait that ran out sets it
// (cgef_debug_inject; closure.cu).
int closure_inject_timeout(cgef_closure* c);

// Resolves, on `device` (current), the device address of the allocation-free filter's fixed scratch
// array (noalloc.cu); resolving it is what makes the driver reserve the array on that device.
int noalloc_prepare(int device);

// Banded schedule pieces.  Source-row costs of the R-row target group starting at j0: for each
// source row in [j0 - D, j0 + R - 1 + D], the width of the union of the group's intervals plus a
// per-row overhead (0 where the row is outside a bounded grid or holds no entries).
std::vector<double> group_row_costs(const cgef_plan* p, int j0, int R = kRows);
// Appends the work items of target group (x0, j0): one item when its cost is within `target`,
// otherwise contiguous source-row parts of about `target` cost plus their split group (slots
// numbered from `slots`, which advances).
void emit_group_items(int x0, int j0, int D, const std::vector<double>& rc, double target,
                      std::vector<WorkItem>& items, std::vector<SplitGroup>& groups, int& slots);
// Builds (or rebuilds) and uploads schedule `which` of the plan (0: kRows rows, 1: kRowsTall rows),
// split so that the banded gather runs in about `waves` rounds of 16 resident warps per SM.
int rebuild_schedule(cgef_plan* p, double waves, int which = 0);
// Accumulated quantities up to which the taller tile keeps its accumulators in registers.
constexpr int kTallMaxQuantities = 3;
// The schedule a launch of `mode` with `na` accumulated quantities uses: the flux modes always the
// kRows one; a filter pass of at most kTallMaxQuantities quantities the taller one when the plan
// chose it and it is built.
inline const Schedule& schedule_for(const cgef_plan* p, int mode, int na);
// A schedule for the 32 x 32 tiles (tx, ty) only, split so that it fills `sms` SMs in one wave;
// slots are numbered from 0.
void subset_schedule(const cgef_plan* p, const std::vector<std::pair<int, int>>& tiles, int sms,
                     std::vector<WorkItem>& items, std::vector<SplitGroup>& groups, int& slots);

// Visits band b's footprint entries in the reference's CSR order (row offset ascending, then
// column offset ascending): f(ddi, ddj, w).  `whalf`: the half-row weights (default: the host copy).
template <typename F>
void for_each_entry(const cgef_plan* p, int b, F f, const double* whalf = nullptr) {
  const double* wh = whalf ? whalf : p->h_whalf.data();
  const int W = 2 * p->D + 1;
  for (int r = 0; r < W; ++r) {
    const BandRow& br = p->h_rows[static_cast<size_t>(b) * W + r];
    if (br.a < 0) continue;
    for (int di = -br.a; di <= br.hi; ++di) {
      const double w = wh[br.woff + (di < 0 ? -di : di)];
      if (w != 0.0) f(di, r - p->D, w);
    }
  }
}

// Workspace slot of at least `bytes` bytes.
int ensure_ws(cgef_plan* p, int slot, size_t bytes, void** out);

void count_launch(int64_t n = 1);

// Tracing: events around one launch of `kind` on stream `st` (no-ops unless enabled).
void prof_begin(int kind, cudaStream_t st);
void prof_end(int kind, cudaStream_t st);
// Suspends tracing on this thread (the allocation-free entry point creates no events).
void prof_suspend(bool suspend);

// ---- launchers (kernels.cu) ----
struct StageArgs {
  const void* a;  // field 0 (u) or nullptr
  const void* b;  // field 1 (v) or nullptr
  const void* const* fields;  // kModeFields: nf fields (each nbatch*ny*nx)
  int nf;
  int dtype;
  const uint8_t* mask;  // device mask (ny*nx) or nullptr
  int64_t mask_slice_stride;  // 0 = shared mask
  int nbatch;
};

// The staged planes [nbatch][np][ny][pitch] (FP64) are followed, 256-byte aligned, by nbatch + 1 int
// flags: flag s is set when an active source cell of slice s holds a non-finite value (or, in the
// flux modes, a non-finite product of two), the last flag when any slice's is.  The banded engine
// sums a flagged slice with a gather that never multiplies a zero weight by a staged value, so a NaN
// or Inf reaches exactly the targets whose footprint holds its cell, as in the reference's per-entry
// loop (Filtering.jl:2575-2585).
inline size_t stage_planes_bytes(const cgef_plan* p, int np, int pitch, int nbatch) {
  return (sizeof(double) * static_cast<size_t>(np) * p->ny * pitch * nbatch + 255) / 256 * 256;
}
inline size_t stage_bytes(const cgef_plan* p, int np, int pitch, int nbatch) {
  return stage_planes_bytes(p, np, pitch, nbatch) + sizeof(int) * (static_cast<size_t>(nbatch) + 1);
}
inline int* stage_flags(const cgef_plan* p, const double* planes, int np, int pitch, int nbatch) {
  return reinterpret_cast<int*>(reinterpret_cast<char*>(const_cast<double*>(planes)) +
                                stage_planes_bytes(p, np, pitch, nbatch));
}

// Writes padded FP64 planes [nbatch][np][ny][pitch] with halo H (wrapped or zero), masked
// values, planetary components on the sphere for kModePiSphere, and a mask plane when
// `with_mask_plane`; then the non-finite flags after them (stage_flags).  The planes buffer holds
// stage_bytes().
int launch_stage(const cgef_plan* p, int mode, const StageArgs& s, double* planes, int pitch, int halo, int np,
                 bool with_mask_plane, cudaStream_t st);

struct GatherOut {
  double* o[9];  // kModeFields: one plane per field; Pi modes: ubar, vbar, txx, txy, tyy
  int64_t slice_stride;
};

// `partials` holds banded_scratch_bytes() of scratch (the direct gather's split tiles, or the
// row-spectral evaluation's spectra when the plan uses it); `direct_only` keeps the direct gather,
// whose scratch is banded_partials_bytes().
int launch_banded(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                  const uint8_t* mask, int64_t mask_slice_stride, double* partials, const GatherOut& out,
                  cudaStream_t st, bool direct_only = false);

// The row-spectral evaluation of a full-grid banded launch: x-direction FFTs of the accumulated
// quantities of every source row, the band's kernel spectra applied and summed per target row,
// inverse FFTs, and the same epilogue as the direct gather.  `scratch` holds rowspec_bytes().
// Source spectra shared by the plans of one sweep (they depend on the staged fields and the FFT
// length, not on the scale): `keep` = transform into this buffer and leave it there, `in` = use the
// spectra an earlier plan left there (no forward transform).  Either way the launch's own scratch holds
// only the summed spectra and the unnormalised sums.
struct RsShare {
  double* keep = nullptr;
  const double* in = nullptr;
};
// `leave_raw` (flux modes): stop before the epilogue and leave the unnormalised sums [slice][NA][ny][nx]
// at the start of `scratch`, for the strain pass to finish (StrainArgs::raw).
int launch_rowspec(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                   const uint8_t* mask, int64_t mask_slice_stride, double* scratch, const GatherOut& out,
                   cudaStream_t st, const RsShare& share = RsShare{}, bool leave_raw = false);

// The spectral method (CGEF_ENGINE_SPECTRAL) over staged planes: the row transforms of the row-spectral
// evaluation (L = nx), a column pass per bin that transforms along y, multiplies by the transfer
// function and transforms back, the inverse row transforms, and an epilogue that applies Deformable's
// renormalisation (`renorm`) and forms tau in the flux mode.  Every cell gets a value.  `scratch`
// holds spectral_scratch_bytes().
int launch_spectral(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                    bool renorm, double* scratch, const GatherOut& out, cudaStream_t st);
inline size_t spectral_scratch_bytes(const cgef_plan* p, int na, int nbatch) {
  return 2 * 2 * sizeof(double) * static_cast<size_t>(nbatch) * p->ny * na * p->rs_nkp;
}
// Builds the spectral method's transforms and transfer function (CGEF_EUNSUPPORTED for lengths the
// transforms do not cover).
int build_spectral(cgef_plan* p);

// Bytes of one sweep's shared source spectra: `na` quantities over `nbatch` slices.
inline size_t rowspec_spectra_bytes(const cgef_plan* p, int na, int nbatch) {
  return 2 * sizeof(double) * static_cast<size_t>(nbatch) * p->ny * na * p->rs_nkp;
}

// Decides whether the plan's banded sums can be evaluated through ring spectra and, if so, builds
// the twiddles and the kernel spectra on the device (called once the band tables are uploaded).
int build_row_spectra(cgef_plan* p);

// The same over a caller-given device schedule: work items and the split groups they belong to
// (e.g. from subset_schedule); `partials` holds the slots that schedule numbers.
// Slices the stage flagged as holding a non-finite value are skipped by the fast gather and summed by
// a second launch that skips zero weights (it returns at once when no slice is flagged).
int launch_banded_items(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                        const uint8_t* mask, int64_t mask_slice_stride, double* partials, const WorkItem* items,
                        int nitems, const SplitGroup* groups, int ngroups, const GatherOut& out, cudaStream_t st);

// Only the flagged slices, by that second gather, over the full schedule, with their unnormalised sums
// written to `raw` in the row-spectral layout [slice][NA][ny][nx] (the row-spectral evaluation's
// non-finite fallback; its epilogue then finishes them).
int launch_banded_nonfinite(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                            const uint8_t* mask, int64_t mask_slice_stride, double* partials, const GatherOut& out,
                            cudaStream_t st, double* raw);

// Bytes of partial-sum scratch a banded launch of `mode` with `na` accumulated quantities over
// `nbatch` slices needs (its own schedule's, or the kRows schedule's that the non-finite pass uses).
inline size_t banded_partials_bytes(const cgef_plan* p, int na, int nbatch, int mode) {
  const Schedule& s = schedule_for(p, mode, na);
  const size_t own = sizeof(double) * static_cast<size_t>(s.nslots) * nbatch * s.rows * na * 32;
  const size_t safe = sizeof(double) * static_cast<size_t>(p->sched[0].nslots) * nbatch * kRows * na * 32;
  return std::max(own, safe);
}

// Bytes of the row-spectral evaluation's scratch: the spectra of the source rows and the summed
// spectra of the target rows, `na` quantities over `nbatch` slices.
inline size_t rowspec_bytes(const cgef_plan* p, int na, int nbatch) {
  return 2 * 2 * sizeof(double) * static_cast<size_t>(nbatch) * p->ny * na * p->rs_nkp;
}

// Scratch of a full-grid banded launch, whichever evaluation the plan uses: the row-spectral
// evaluation's spectra, then the direct gather's split-tile partials (its non-finite fallback runs
// while the spectral evaluation's unnormalised sums are still live).
inline size_t banded_scratch_bytes(const cgef_plan* p, int na, int nbatch, int mode) {
  const size_t d = banded_partials_bytes(p, na, nbatch, mode);
  return p->rs_on ? rowspec_bytes(p, na, nbatch) + d : d;
}

int launch_separable(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                     const uint8_t* mask, int64_t mask_slice_stride, double* rowbuf, const GatherOut& out,
                     cudaStream_t st);

int launch_prefix(const cgef_plan* p, int mode, int nf, const double* planes, int pitch, int np, int nbatch,
                  const uint8_t* mask, int64_t mask_slice_stride, double* prefix, const GatherOut& out,
                  cudaStream_t st);

struct StrainArgs {
  const double* ubar;
  const double* vbar;
  const double* txx;
  const double* txy;
  const double* tyy;
  int64_t in_slice_stride;
  const uint8_t* mask;
  int64_t mask_slice_stride;
  int nbatch;
  int dtype;
  // outputs (dtype), each with out_slice_stride between slices; nullptr = skip
  void* pi;
  void* ubar_o;
  void* vbar_o;
  void* txx_o;
  void* txy_o;
  void* tyy_o;
  void* sxx_o;
  void* sxy_o;
  void* syy_o;
  int64_t out_slice_stride;
  // energy: per-slice numerator and active area partials, reduced into energy[slice*estride]
  double* partials;  // nbatch * nblocks * 2, or nullptr
  double* energy;    // nullptr = skip
  int64_t energy_stride;
  // closure features: grad[slice][4][ny*nx] (FP32) = grad_scale * (S_ee, du/dy, dv/dx + u t, S_nn),
  // and grad_mean[slice] = mean over active cells of their squared norm (grad_partials: scratch of
  // nbatch * nblocks * 2 doubles).  nullptr = skip.  txx/txy/tyy may be nullptr (read as 0).
  float* grad;
  int64_t grad_slice_stride;
  double grad_scale;
  double* grad_partials;
  double* grad_mean;
  // strain / convergence split (plane; outputs of dtype, out_slice_stride): total, strain,
  // convergence, divergence, strain magnitude.  nullptr = skip.
  void* sc[5];
  // The row-spectral evaluation's unnormalised sums [slice][NA][ny][nx] (pi_gather's raw output):
  // finished here instead of reading ubar, vbar and tau.  nullptr = the finished planes.
  const double* raw = nullptr;
};

int launch_strain(const cgef_plan* p, const StrainArgs& a, cudaStream_t st);

// Plain derivative of one field (ddx / ddy).
int launch_derivative(const cgef_plan* p, int axis, int dtype, const void* f, void* out, cudaStream_t st);

// Converts FP64 planes to the caller's dtype: dst[s*dst_stride + k] = src[s*src_stride + k].
int launch_convert(const double* src, int64_t src_stride, void* dst, int64_t dst_stride, int dtype, int64_t n,
                   int nbatch, cudaStream_t st);

// Energy of `fields` (ubar, vbar planes) per slice.
// energy[s * energy_stride] = factor * sum_k partials[s][k][0] / sum_k partials[s][k][1] (0 when the
// weight is 0), one block per slice, the partials summed in a fixed order: the energies' last step.
// Target tiles of the strain pass (and of the energy partials) over one slice: the partials buffers
// hold two doubles per tile and slice.
int64_t strain_tiles(const cgef_plan* p);
int launch_energy_finish(const double* partials, int64_t nblk, int nbatch, double* energy, int64_t energy_stride,
                         double factor, cudaStream_t st);
int launch_energy(const cgef_plan* p, const double* ubar, const double* vbar, int64_t slice_stride,
                  const uint8_t* mask, int64_t mask_slice_stride, int nbatch, double* partials, double* energy,
                  int64_t energy_stride, cudaStream_t st);


// ---- shared host helpers (cgef_api.cu) ----
// Workspace slots of a plan (cgef_plan::ws).
enum WsSlot {
  kSlotPlanes = 0,
  kSlotGather = 1,
  kSlotPartials = 2,
  kSlotIn = 3,
  kSlotOut = 4,
  kSlotAux = 5,
  kSlotMask = 6,
  kSlotDeriv = 7,
  kSlotSplit = 8,
  kSlotVel = 9,
  kSlotDecomp = 10,
  kSlotSpectra = 11,  // a sweep's shared source spectra (row-spectral evaluation)
  kSlotW = 12,        // the 2.5-D flux: the velocities and products before and after filtering
  kNumSlots = 13,
};

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

size_t dsize(int dtype);
int check_plan(const cgef_plan* p);
int check_dtype(int dtype);
// Row pitch (doubles) of the staged planes for a halo of `halo` columns.
int pitch_for(const cgef_plan* p, int halo);
// kModePiSphere or kModePiCart.
int mode_for(const cgef_plan* p);
// Stages u, v (planetary components on the sphere) into padded planes in slot kSlotPlanes.
int stage_pi(cgef_plan* p, int dtype, const void* u, const void* v, int nbatch, const uint8_t* mask, int64_t mstride,
             int halo, double** planes_out, int* pitch_out, int* np_out, cudaStream_t st);
// Runs the plan's engine in a flux mode: 5 FP64 planes (ubar, vbar, txx, txy, tyy) per slice.  With
// `raw_out`, a plan on the row-spectral evaluation instead leaves its unnormalised sums and points
// *raw_out at them (nullptr otherwise), for a strain pass that finishes them itself.
int pi_gather(cgef_plan* p, const double* planes, int pitch, int halo, int np, int nbatch, const uint8_t* mask,
              int64_t mstride, double* gather, cudaStream_t st, const RsShare& share = RsShare{},
              const double** raw_out = nullptr);
int compute_pi_device(cgef_plan* p, int dtype, const void* u, const void* v, int64_t nbatch64,
                      const uint8_t* slice_masks, const cgef_pi_outputs* out, cudaStream_t st);
// The 2.5-D flux (pi_w.cu): u, v, w device buffers of dtype.
int compute_pi_w_device(cgef_plan* p, int dtype, const void* u, const void* v, const void* w, int64_t nbatch64,
                        const uint8_t* slice_masks, const cgef_pi_w_outputs* out, cudaStream_t st);
// The sweep over plans (one grid) for nbatch slices on stream st: Pi [nbatch][nscales][N] (dtype) and
// E [nbatch][nscales], either may be nullptr.
int sweep_device(cgef_plan* const* plans, int nscales, int dtype, const void* u, const void* v, int64_t nbatch64,
                 const uint8_t* slice_masks, void* pi, double* energy, cudaStream_t st);
// Filters nf (<= 4) fields of dtype through the plan's engine into FP64 planes outs[m] (slice stride
// `ostride`).
int filter_fields_device(cgef_plan* p, int dtype, const void* const* fields, int nf, double* const* outs,
                         int64_t ostride, int nbatch, const uint8_t* mask, int64_t mstride, cudaStream_t st);

inline const Schedule& schedule_for(const cgef_plan* p, int mode, int na) {
  if (mode == kModeFields && na <= kTallMaxQuantities && p->filter_rows == kRowsTall && p->sched[1].rows == kRowsTall)
    return p->sched[1];
  return p->sched[0];
}

}  // namespace cgef
