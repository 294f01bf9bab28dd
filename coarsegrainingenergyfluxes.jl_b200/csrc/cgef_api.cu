// C ABI of libcgef_b200.so (declared in include/cgef_b200.h): plan lifecycle, workspaces and
// the host- and device-buffer entry points that orchestrate the kernels of kernels.cu.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "cgef_internal.h"

namespace cgef {

namespace {
thread_local std::string g_err;
thread_local int64_t g_launches = 0;

struct ProfRec {
  int kind;
  cudaEvent_t a, b;
};
thread_local bool g_prof = false;
thread_local bool g_prof_suspended = false;
thread_local std::vector<ProfRec> g_recs;
thread_local cudaEvent_t g_open = nullptr;
thread_local int g_open_kind = -1;
thread_local double g_prof_ms[CGEF_KERNEL_KINDS] = {};
thread_local int64_t g_prof_n[CGEF_KERNEL_KINDS] = {};

void drain_profile() {
  for (auto& r : g_recs) {
    float ms = 0.f;
    if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      g_prof_ms[r.kind] += ms;
      g_prof_n[r.kind] += 1;
    }
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  g_recs.clear();
  cudaGetLastError();
}
}  // namespace

void prof_suspend(bool suspend) { g_prof_suspended = suspend; }

void prof_begin(int kind, cudaStream_t st) {
  if (!g_prof || g_prof_suspended) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, st);
  g_open = e;
  g_open_kind = kind;
}

void prof_end(int kind, cudaStream_t st) {
  if (!g_prof || g_prof_suspended || g_open == nullptr || g_open_kind != kind) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, st);
  g_recs.push_back(ProfRec{kind, g_open, e});
  g_open = nullptr;
  g_open_kind = -1;
  if (g_recs.size() > 4096) drain_profile();
}

void set_error(const std::string& msg) { g_err = msg; }

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return CGEF_ECUDA;
}

void count_launch(int64_t n) { g_launches += n; }

int ensure_ws(cgef_plan* p, int slot, size_t bytes, void** out) {
  DeviceBuffer& b = p->ws[slot];
  if (b.bytes < bytes) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMalloc(&b.ptr, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(CGEF_ENOMEM, "workspace allocation of " + std::to_string(bytes) + " bytes failed: " +
                                   cudaGetErrorString(e));
    }
    b.bytes = bytes;
  }
  *out = b.ptr;
  return CGEF_OK;
}

}  // namespace cgef

using namespace cgef;

namespace cgef {

size_t dsize(int dtype) { return dtype == CGEF_F32 ? sizeof(float) : sizeof(double); }

int check_plan(const cgef_plan* p) {
  if (!p) return fail(CGEF_EINVAL, "plan is NULL");
  if (p->device < 0) return fail(CGEF_ENODEVICE, "no CUDA device was visible when the plan was created");
  return CGEF_OK;
}

int check_dtype(int dtype) {
  return (dtype == CGEF_F64 || dtype == CGEF_F32) ? CGEF_OK : fail(CGEF_EINVAL, "dtype must be CGEF_F64 or CGEF_F32");
}

int pitch_for(const cgef_plan* p, int halo) {
  const int wide = kTileCols;
  int nxr = ((p->nx + wide - 1) / wide) * wide;
  int pitch = halo + nxr + halo + 32;
  return ((pitch + 31) / 32) * 32;
}

int mode_for(const cgef_plan* p) { return p->geometry == CGEF_SPHERICAL ? kModePiSphere : kModePiCart; }

// Stages the inputs and runs one plan's engine for a flux computation; leaves the 5 FP64
// gather planes (ubar, vbar, txx, txy, tyy) at `gather` with slice stride 5*N.
int pi_gather(cgef_plan* p, const double* planes, int pitch, int halo, int np, int nbatch, const uint8_t* mask,
              int64_t mstride, double* gather, cudaStream_t st, const RsShare& share, const double** raw_out) {
  if (raw_out) *raw_out = nullptr;
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  GatherOut go{};
  for (int m = 0; m < 5; ++m) go.o[m] = gather + m * N;
  go.slice_stride = 5 * N;
  const int mode = mode_for(p);
  (void)halo;
  if (p->engine == CGEF_ENGINE_BANDED) {
    const int na = (mode == kModePiSphere ? 9 : 5) + (p->strategy == CGEF_DEFORMABLE ? 1 : 0);
    void* part = nullptr;
    const size_t pb = banded_scratch_bytes(p, na, nbatch, mode);
    if (pb > 0) {
      int rc = ensure_ws(p, kSlotSplit, pb, &part);
      if (rc) return rc;
    }
    if (p->rs_on) {
      int rc = launch_rowspec(p, mode, 0, planes, pitch, np, nbatch, mask, mstride, static_cast<double*>(part), go, st,
                              share, raw_out != nullptr);
      if (rc == CGEF_OK && raw_out) *raw_out = static_cast<const double*>(part);
      return rc;
    }
    return launch_banded(p, mode, 0, planes, pitch, np, nbatch, mask, mstride, static_cast<double*>(part), go, st,
                         true);
  }
  if (p->engine == CGEF_ENGINE_SPECTRAL) {
    const int na = 5 + (p->strategy == CGEF_DEFORMABLE ? 1 : 0);
    void* sc = nullptr;
    int rc = ensure_ws(p, kSlotSplit, spectral_scratch_bytes(p, na, nbatch), &sc);
    if (rc) return rc;
    return launch_spectral(p, mode, 0, planes, pitch, np, nbatch, mstride != 0 || p->masked, static_cast<double*>(sc),
                           go, st);
  }
  if (p->engine == CGEF_ENGINE_SEPARABLE) {
    const int na = 5 + (p->strategy == CGEF_DEFORMABLE ? 1 : 0);
    void* rb = nullptr;
    int rc = ensure_ws(p, kSlotAux, sizeof(double) * na * N * nbatch, &rb);
    if (rc) return rc;
    return launch_separable(p, mode, 0, planes, pitch, np, nbatch, mask, mstride, static_cast<double*>(rb), go, st);
  }
  const int na = (mode == kModePiSphere ? 9 : 5) + (p->strategy == CGEF_DEFORMABLE ? 1 : 0);
  void* pre = nullptr;
  int rc = ensure_ws(p, kSlotAux, sizeof(double) * na * static_cast<int64_t>(p->ny) * (p->pre_ne + 1) * nbatch, &pre);
  if (rc) return rc;
  return launch_prefix(p, mode, 0, planes, pitch, np, nbatch, mask, mstride, static_cast<double*>(pre), go, st);
}

// Column halo the flux's staged planes need for plan q: the direct gather reads up to H columns past either
// end of a row, while the row-spectral evaluation reads the row alone (its non-finite re-sum wraps or zeroes
// its own columns), so it is staged without one -- half the stage pass's writes on the 0.25-degree sphere.
int stage_halo(const cgef_plan* q) { return q->engine == CGEF_ENGINE_BANDED && q->rs_on ? 0 : q->H; }

int stage_pi(cgef_plan* p, int dtype, const void* u, const void* v, int nbatch, const uint8_t* mask, int64_t mstride,
             int halo, double** planes_out, int* pitch_out, int* np_out, cudaStream_t st) {
  const bool def = p->strategy == CGEF_DEFORMABLE;
  const int mode = mode_for(p);
  const int np = (mode == kModePiSphere ? 3 : 2) + (def ? 1 : 0);
  const int pitch = pitch_for(p, halo);
  void* planes = nullptr;
  int rc = ensure_ws(p, kSlotPlanes, stage_bytes(p, np, pitch, nbatch), &planes);
  if (rc) return rc;
  StageArgs sa{};
  sa.a = u;
  sa.b = v;
  sa.nf = 2;
  sa.dtype = dtype;
  sa.mask = mask;
  sa.mask_slice_stride = mstride;
  sa.nbatch = nbatch;
  rc = launch_stage(p, mode, sa, static_cast<double*>(planes), pitch, halo, np, def, st);
  if (rc) return rc;
  *planes_out = static_cast<double*>(planes);
  *pitch_out = pitch;
  *np_out = np;
  return CGEF_OK;
}

int compute_pi_device(cgef_plan* p, int dtype, const void* u, const void* v, int64_t nbatch64,
                      const uint8_t* slice_masks, const cgef_pi_outputs* out, cudaStream_t st) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!u || !v) return fail(CGEF_EINVAL, "u and v must be non-NULL");
  if (nbatch64 < 1 || nbatch64 > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  const int nbatch = static_cast<int>(nbatch64);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const uint8_t* mask = slice_masks ? slice_masks : p->d_mask;
  const int64_t mstride = slice_masks ? N : 0;
  double* planes = nullptr;
  int pitch = 0, np = 0;
  const int halo = stage_halo(p);
  if ((rc = stage_pi(p, dtype, u, v, nbatch, mask, mstride, halo, &planes, &pitch, &np, st))) return rc;
  void* gather = nullptr;
  if ((rc = ensure_ws(p, kSlotGather, sizeof(double) * 5 * N * nbatch, &gather))) return rc;
  double* g = static_cast<double*>(gather);
  const double* raw = nullptr;
  // the engine reads the planes with the halo they were staged with
  const int saveH = p->H;
  p->H = halo;
  rc = pi_gather(p, planes, pitch, halo, np, nbatch, mask, mstride, g, st, RsShare{}, &raw);
  p->H = saveH;
  if (rc) return rc;
  StrainArgs sa{};
  sa.raw = raw;
  sa.ubar = g;
  sa.vbar = g + N;
  sa.txx = g + 2 * N;
  sa.txy = g + 3 * N;
  sa.tyy = g + 4 * N;
  sa.in_slice_stride = 5 * N;
  sa.mask = mask;
  sa.mask_slice_stride = mstride;
  sa.nbatch = nbatch;
  sa.dtype = dtype;
  cgef_pi_outputs none{};
  const cgef_pi_outputs* o = out ? out : &none;
  sa.pi = o->pi;
  sa.ubar_o = o->ubar;
  sa.vbar_o = o->vbar;
  sa.txx_o = o->tau_xx;
  sa.txy_o = o->tau_xy;
  sa.tyy_o = o->tau_yy;
  sa.sxx_o = o->s_xx;
  sa.sxy_o = o->s_xy;
  sa.syy_o = o->s_yy;
  sa.out_slice_stride = N;
  if (o->energy) {
    void* part = nullptr;
    const int64_t nblk = strain_tiles(p);
    if ((rc = ensure_ws(p, kSlotPartials, sizeof(double) * 2 * nblk * nbatch, &part))) return rc;
    sa.partials = static_cast<double*>(part);
    sa.energy = o->energy;
    sa.energy_stride = 1;
  }
  return launch_strain(p, sa, st);
}

// Filters nf (<= 4 per pass) fields; outputs FP64 planes (slice stride `ostride`).
int filter_fields_device(cgef_plan* p, int dtype, const void* const* fields, int nf, double* const* outs,
                         int64_t ostride, int nbatch, const uint8_t* mask, int64_t mstride, cudaStream_t st) {
  const bool def = p->strategy == CGEF_DEFORMABLE;
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const int np = nf + (def ? 1 : 0);
  const int pitch = pitch_for(p, p->H);
  void* planes = nullptr;
  int rc = ensure_ws(p, kSlotPlanes, stage_bytes(p, np, pitch, nbatch), &planes);
  if (rc) return rc;
  StageArgs sa{};
  sa.fields = fields;
  sa.nf = nf;
  sa.dtype = dtype;
  sa.mask = mask;
  sa.mask_slice_stride = mstride;
  sa.nbatch = nbatch;
  if ((rc = launch_stage(p, kModeFields, sa, static_cast<double*>(planes), pitch, p->H, np, def, st))) return rc;
  GatherOut go{};
  for (int m = 0; m < nf; ++m) go.o[m] = outs[m];
  go.slice_stride = ostride;
  double* pl = static_cast<double*>(planes);
  if (p->engine == CGEF_ENGINE_BANDED) {
    void* part = nullptr;
    const size_t pb = banded_scratch_bytes(p, nf + (def ? 1 : 0), nbatch, kModeFields);
    if (pb > 0 && (rc = ensure_ws(p, kSlotSplit, pb, &part))) return rc;
    return launch_banded(p, kModeFields, nf, pl, pitch, np, nbatch, mask, mstride, static_cast<double*>(part), go, st);
  }
  if (p->engine == CGEF_ENGINE_SEPARABLE) {
    void* rb = nullptr;
    if ((rc = ensure_ws(p, kSlotAux, sizeof(double) * (nf + 1) * N * nbatch, &rb))) return rc;
    return launch_separable(p, kModeFields, nf, pl, pitch, np, nbatch, mask, mstride, static_cast<double*>(rb), go, st);
  }
  if (p->engine == CGEF_ENGINE_SPECTRAL) {
    void* sc = nullptr;
    if ((rc = ensure_ws(p, kSlotSplit, spectral_scratch_bytes(p, np, nbatch), &sc))) return rc;
    return launch_spectral(p, kModeFields, nf, pl, pitch, np, nbatch, mstride != 0 || p->masked,
                           static_cast<double*>(sc), go, st);
  }
  void* pre = nullptr;
  if ((rc = ensure_ws(p, kSlotAux, sizeof(double) * (nf + 1) * static_cast<int64_t>(p->ny) * (p->pre_ne + 1) * nbatch,
                      &pre)))
    return rc;
  return launch_prefix(p, kModeFields, nf, pl, pitch, np, nbatch, mask, mstride, static_cast<double*>(pre), go, st);
}

}  // namespace cgef

namespace {

// One field with a trailing batch axis: device in/out of the caller's dtype.
int filter_device(cgef_plan* p, int dtype, const void* field, void* out, int64_t nbatch64, cudaStream_t st) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!field || !out) return fail(CGEF_EINVAL, "field and out must be non-NULL");
  if (nbatch64 < 1 || nbatch64 > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  const int nbatch = static_cast<int>(nbatch64);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  double* dst = nullptr;
  if (dtype == CGEF_F64) {
    dst = static_cast<double*>(out);
  } else {
    void* t = nullptr;
    if ((rc = ensure_ws(p, kSlotGather, sizeof(double) * N * nbatch, &t))) return rc;
    dst = static_cast<double*>(t);
  }
  const void* fl[1] = {field};
  double* ol[1] = {dst};
  if ((rc = filter_fields_device(p, dtype, fl, 1, ol, N, nbatch, p->d_mask, 0, st))) return rc;
  if (dtype != CGEF_F64) return launch_convert(dst, N, out, N, dtype, N, nbatch, st);
  return CGEF_OK;
}

}  // namespace

namespace cgef {

int sweep_device(cgef_plan* const* plans, int nscales, int dtype, const void* u, const void* v, int64_t nbatch64,
                 const uint8_t* slice_masks, void* pi, double* energy, cudaStream_t st) {
  int rc;
  if (!plans || nscales < 1) return fail(CGEF_EINVAL, "need at least one plan");
  cgef_plan* p0 = plans[0];
  if ((rc = check_plan(p0)) || (rc = check_dtype(dtype))) return rc;
  if (nbatch64 < 1 || nbatch64 > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  int halo = 0;
  for (int s = 0; s < nscales; ++s) {
    const cgef_plan* q = plans[s];
    if ((rc = check_plan(q))) return rc;
    if (q->nx != p0->nx || q->ny != p0->ny || q->geometry != p0->geometry || q->engine != p0->engine ||
        q->strategy != p0->strategy || q->periodic_x != p0->periodic_x || q->periodic_y != p0->periodic_y ||
        q->dx != p0->dx || q->dy != p0->dy || q->x0 != p0->x0 || q->y0 != p0->y0 || q->h_mask != p0->h_mask)
      return fail(CGEF_EINVAL, "all plans of a sweep must share one grid, engine and mask strategy");
    halo = std::max(halo, stage_halo(q));
  }
  const int nbatch = static_cast<int>(nbatch64);
  const int64_t N = static_cast<int64_t>(p0->nx) * p0->ny;
  const uint8_t* mask = slice_masks ? slice_masks : p0->d_mask;
  const int64_t mstride = slice_masks ? N : 0;
  double* planes = nullptr;
  int pitch = 0, np = 0;
  if ((rc = stage_pi(p0, dtype, u, v, nbatch, mask, mstride, halo, &planes, &pitch, &np, st))) return rc;
  void* gather = nullptr;
  if ((rc = ensure_ws(p0, kSlotGather, sizeof(double) * 5 * N * nbatch, &gather))) return rc;
  double* g = static_cast<double*>(gather);
  void* part = nullptr;
  const int64_t nblk = strain_tiles(p0);
  if ((rc = ensure_ws(p0, kSlotPartials, sizeof(double) * 2 * nblk * nbatch, &part))) return rc;
  // The row-spectral plans of one FFT length share the source spectra: they depend on the staged fields,
  // not on the scale, so the first such plan transforms them and the others start from its spectra.
  int share_L = 0, nshare = 0;
  for (int s = 0; s < nscales; ++s) {
    const cgef_plan* q = plans[s];
    if (q->engine != CGEF_ENGINE_BANDED || !q->rs_on) continue;
    if (share_L == 0) share_L = q->rs_L;
    if (q->rs_L == share_L) ++nshare;
  }
  double* spectra = nullptr;
  if (nshare > 1) {
    const int na = (mode_for(p0) == kModePiSphere ? 9 : 5) + (p0->strategy == CGEF_DEFORMABLE ? 1 : 0);
    const cgef_plan* qs = nullptr;
    for (int s = 0; s < nscales && !qs; ++s)
      if (plans[s]->engine == CGEF_ENGINE_BANDED && plans[s]->rs_on) qs = plans[s];
    void* buf = nullptr;
    if ((rc = ensure_ws(p0, kSlotSpectra, rowspec_spectra_bytes(qs, na, nbatch), &buf))) return rc;
    spectra = static_cast<double*>(buf);
  }
  bool transformed = false;
  for (int s = 0; s < nscales; ++s) {
    cgef_plan* q = plans[s];
    // the sweep's planes carry the widest halo; run each plan against them
    const int saveH = q->H;
    q->H = halo;
    RsShare share;
    if (spectra && q->engine == CGEF_ENGINE_BANDED && q->rs_on && q->rs_L == share_L) {
      if (transformed)
        share.in = spectra;
      else
        share.keep = spectra;
      transformed = true;
    }
    // each plan runs its engine with its own scratch (split partials, separable rows, prefix sums, spectra)
    const double* raw = nullptr;
    rc = pi_gather(q, planes, pitch, halo, np, nbatch, mask, mstride, g, st, share, &raw);
    q->H = saveH;
    if (rc) return rc;
    StrainArgs sa{};
    sa.raw = raw;
    sa.ubar = g;
    sa.vbar = g + N;
    sa.txx = g + 2 * N;
    sa.txy = g + 3 * N;
    sa.tyy = g + 4 * N;
    sa.in_slice_stride = 5 * N;
    sa.mask = mask;
    sa.mask_slice_stride = mstride;
    sa.nbatch = nbatch;
    sa.dtype = dtype;
    if (pi) sa.pi = static_cast<char*>(pi) + dsize(dtype) * static_cast<size_t>(s) * N;
    sa.out_slice_stride = static_cast<int64_t>(nscales) * N;
    if (energy) {
      sa.partials = static_cast<double*>(part);
      sa.energy = energy + s;
      sa.energy_stride = nscales;
    }
    if ((rc = launch_strain(q, sa, st))) return rc;
  }
  return CGEF_OK;
}

}  // namespace cgef

namespace {

int h2d(cgef_plan* p, int slot, const void* src, size_t bytes, void** dst) {
  int rc = ensure_ws(p, slot, bytes, dst);
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, p->stream);
  return e == cudaSuccess ? CGEF_OK : cuda_fail(e, "cudaMemcpyAsync(H2D)");
}

int d2h(cgef_plan* p, void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, p->stream);
  return e == cudaSuccess ? CGEF_OK : cuda_fail(e, "cudaMemcpyAsync(D2H)");
}

int sync(cgef_plan* p) {
  cudaError_t e = cudaStreamSynchronize(p->stream);
  return e == cudaSuccess ? CGEF_OK : cuda_fail(e, "cudaStreamSynchronize");
}

}  // namespace

extern "C" {

int32_t cgef_version(void) { return CGEF_ABI_VERSION; }

int32_t cgef_build_arch(void) { return 1000; }  // every .cu file refuses any other device target

int32_t cgef_set_footprint_build(int32_t where) { return set_footprint_build(where); }

int32_t cgef_plan_get_build(const cgef_plan* p, int32_t* where) {
  if (!p) return fail(CGEF_EINVAL, "plan is NULL");
  if (where) *where = p->built_on_device ? CGEF_BUILD_DEVICE : CGEF_BUILD_HOST;
  return CGEF_OK;
}

int32_t cgef_plan_reset_queue(cgef_plan* p) {
  int rc = check_plan(p);
  if (rc) return rc;
  if (p->d_queue == nullptr) return CGEF_OK;
  DeviceGuard dg(p->device);
  cudaError_t e = cudaMemsetAsync(p->d_queue, 0, 2 * sizeof(unsigned long long), p->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
  return e == cudaSuccess ? CGEF_OK : cuda_fail(e, "cgef_plan_reset_queue");
}

int32_t cgef_debug_inject(void* object, int32_t what) {
  if (!object) return fail(CGEF_EINVAL, "object is NULL");
  if (what == CGEF_INJECT_CLOSURE_TIMEOUT) return closure_inject_timeout(static_cast<cgef_closure*>(object));
  if (what != CGEF_INJECT_STALE_QUEUE) return fail(CGEF_EINVAL, "unknown injection");
  cgef_plan* p = static_cast<cgef_plan*>(object);
  int rc = check_plan(p);
  if (rc) return rc;
  if (p->d_queue == nullptr) return fail(CGEF_EINVAL, "the plan has no work queue (not the banded engine)");
  DeviceGuard dg(p->device);
  // a launch that handed out 7 units and saw 3 warps leave
  const unsigned long long stale[2] = {7ull, 3ull};
  cudaError_t e = cudaMemcpy(p->d_queue, stale, sizeof(stale), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? CGEF_OK : cuda_fail(e, "work queue");
}

const char* cgef_last_error(void) { return g_err.c_str(); }

int32_t cgef_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int64_t cgef_launch_count(void) { return g_launches; }
void cgef_reset_launch_count(void) { g_launches = 0; }

void cgef_profile_enable(int32_t enable) { g_prof = enable != 0; }

int32_t cgef_profile_read(int32_t kind, double* total_ms, int64_t* launches) {
  if (kind < 0 || kind >= CGEF_KERNEL_KINDS) return fail(CGEF_EINVAL, "unknown kernel kind");
  drain_profile();
  if (total_ms) *total_ms = g_prof_ms[kind];
  if (launches) *launches = g_prof_n[kind];
  return CGEF_OK;
}

void cgef_profile_reset(void) {
  drain_profile();
  for (int k = 0; k < CGEF_KERNEL_KINDS; ++k) {
    g_prof_ms[k] = 0;
    g_prof_n[k] = 0;
  }
}

int32_t cgef_plan_create(cgef_plan** out, const cgef_grid_desc* g, int32_t kernel, double alpha, double scale,
                         int32_t mask_strategy, int32_t engine) {
  if (!out) return fail(CGEF_EINVAL, "out is NULL");
  *out = nullptr;
  if (!g) return fail(CGEF_EINVAL, "grid descriptor is NULL");
  if (g->geometry != CGEF_CARTESIAN && g->geometry != CGEF_SPHERICAL) return fail(CGEF_EINVAL, "unknown geometry");
  if (g->nx < 1 || g->ny < 1 || g->nx > (1 << 24) || g->ny > (1 << 24)) return fail(CGEF_EINVAL, "grid size out of range");
  if (!(g->dx > 0) || !(g->dy > 0) || !std::isfinite(g->dx) || !std::isfinite(g->dy))
    return fail(CGEF_EINVAL, "grid spacing must be finite and positive");
  if (g->geometry == CGEF_SPHERICAL && !(g->radius > 0)) return fail(CGEF_EINVAL, "sphere radius must be positive");
  if (kernel != CGEF_TOPHAT && kernel != CGEF_GAUSSIAN) return fail(CGEF_EINVAL, "unknown kernel");
  if (kernel == CGEF_GAUSSIAN && !(alpha > 0 && std::isfinite(alpha))) return fail(CGEF_EINVAL, "Gaussian alpha must be positive");
  // Filtering.jl:2917-2922
  if (!(std::isfinite(scale) && scale > 0)) return fail(CGEF_EINVAL, "filter scale must be finite and positive");
  if (mask_strategy != CGEF_ZEROFILL && mask_strategy != CGEF_DEFORMABLE) return fail(CGEF_EINVAL, "unknown mask strategy");
  int eng = engine;
  if (eng == CGEF_ENGINE_AUTO)
    eng = kernel == CGEF_TOPHAT ? CGEF_ENGINE_PREFIXSUM
                                : (g->geometry == CGEF_CARTESIAN ? CGEF_ENGINE_SEPARABLE : CGEF_ENGINE_BANDED);
  if (eng == CGEF_ENGINE_SEPARABLE && (kernel != CGEF_GAUSSIAN || g->geometry != CGEF_CARTESIAN))
    return fail(CGEF_EUNSUPPORTED, "the separable engine needs a Gaussian kernel on a Cartesian grid");
  if (eng == CGEF_ENGINE_PREFIXSUM && kernel != CGEF_TOPHAT)
    return fail(CGEF_EUNSUPPORTED, "the prefix-sum engine needs the top-hat kernel");
  // FFTWExt.jl:130-135 and Filtering.jl:2998-3004: a periodic transform is the filter only on a
  // Cartesian grid that wraps along both axes
  if (eng == CGEF_ENGINE_SPECTRAL && (g->geometry != CGEF_CARTESIAN || !g->periodic_x || !g->periodic_y))
    return fail(CGEF_EINVAL, "spectral FFT filtering requires a doubly-periodic Cartesian grid");
  if (eng < CGEF_ENGINE_BANDED || eng > CGEF_ENGINE_SPECTRAL) return fail(CGEF_EINVAL, "unknown engine");

  cgef_plan* p = new (std::nothrow) cgef_plan();
  if (!p) return fail(CGEF_ENOMEM, "host allocation failed");
  p->geometry = g->geometry;
  p->nx = static_cast<int>(g->nx);
  p->ny = static_cast<int>(g->ny);
  p->periodic_x = g->periodic_x ? 1 : 0;
  p->periodic_y = g->periodic_y ? 1 : 0;
  p->x0 = g->x0;
  p->dx = g->dx;
  p->y0 = g->y0;
  p->dy = g->dy;
  p->R = g->geometry == CGEF_SPHERICAL ? g->radius : 0.0;
  if (g->mask) {
    const size_t n = static_cast<size_t>(p->nx) * p->ny;
    p->h_mask.resize(n);
    for (size_t k = 0; k < n; ++k) p->h_mask[k] = g->mask[k] ? 1 : 0;
    p->masked = std::find(p->h_mask.begin(), p->h_mask.end(), 0) != p->h_mask.end();
  }
  p->kernel = kernel;
  p->alpha = kernel == CGEF_GAUSSIAN ? alpha : 0.0;
  p->scale = scale;
  p->strategy = mask_strategy;
  p->engine = eng;
  int ndev = cgef_device_count();
  if (ndev > 0) {
    if (cudaGetDevice(&p->device) != cudaSuccess) p->device = 0;
  } else {
    p->device = -1;
  }
  int rc = build_plan_tables(p);
  if (rc == CGEF_OK && p->device >= 0) {
    cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaStreamCreate");
  }
  // The allocation-free filter's fixed array is reserved on this device now, by resolving its
  // address, so that entry point's first call on the device does not reserve it itself.
  if (rc == CGEF_OK && p->device >= 0) rc = noalloc_prepare(p->device);
  if (rc != CGEF_OK) {
    std::string msg = g_err;
    cgef_plan_destroy(p);
    g_err = msg;
    return rc;
  }
  *out = p;
  return CGEF_OK;
}

int32_t cgef_plan_destroy(cgef_plan* p) {
  if (!p) return CGEF_OK;
  if (p->device >= 0) {
    DeviceGuard dg(p->device);
    void* ptrs[] = {p->d_mask, p->d_x, p->d_sinlam, p->d_coslam, p->d_sinphi, p->d_cosphi, p->d_area, p->d_xscale,
                    p->d_tanfac, p->d_rows, p->d_w, p->d_den_zf, p->sched[0].d_items, p->sched[0].d_groups,
                    p->sched[1].d_items, p->sched[1].d_groups, p->d_gx, p->d_gy, p->d_px, p->d_py, p->d_xe,
                    p->d_prefix_wx, p->d_prows, p->d_queue, p->d_rs_tw, p->d_rs_k, p->d_rs_ptw,
                    p->d_sp_ptw, p->d_sp_T};
    for (void* q : ptrs)
      if (q) cudaFree(q);
    for (auto& b : p->ws)
      if (b.ptr) cudaFree(b.ptr);
    if (p->stream) cudaStreamDestroy(p->stream);
  }
  delete p;
  return CGEF_OK;
}

int32_t cgef_plan_get_info(const cgef_plan* p, cgef_plan_info* info) {
  if (!p || !info) return fail(CGEF_EINVAL, "plan and info must be non-NULL");
  info->engine = p->engine;
  info->nbands = p->engine == CGEF_ENGINE_BANDED ? (p->geometry == CGEF_SPHERICAL ? p->ny : 1) : 0;
  info->nentries = p->nentries;
  info->dj_lim = p->dj_lim;
  info->di_max = p->di_max;
  info->kernel_radius = p->rad;
  info->active_area = p->active_area;
  return CGEF_OK;
}

int32_t cgef_plan_set_split_waves(cgef_plan* p, double waves) {
  int rc = check_plan(p);
  if (rc) return rc;
  if (!(waves > 0.0 && waves <= 1024.0)) return fail(CGEF_EINVAL, "waves must be in (0, 1024]");
  if (p->engine != CGEF_ENGINE_BANDED) return CGEF_OK;
  DeviceGuard dg(p->device);
  int rc2 = rebuild_schedule(p, waves, 0);
  if (rc2 == CGEF_OK && p->sched[1].rows) rc2 = rebuild_schedule(p, waves, 1);
  return rc2;
}

int32_t cgef_plan_set_filter_rows(cgef_plan* p, int32_t rows) {
  int rc = check_plan(p);
  if (rc) return rc;
  if (rows != kRows && rows != kRowsTall) return fail(CGEF_EINVAL, "filter tile height must be 4 or 8 rows");
  if (p->engine != CGEF_ENGINE_BANDED) return CGEF_OK;
  DeviceGuard dg(p->device);
  if (rows == kRowsTall && p->sched[1].rows == 0 && (rc = rebuild_schedule(p, p->sched[0].waves, 1))) return rc;
  p->filter_rows = rows;
  return CGEF_OK;
}

int32_t cgef_plan_set_row_spectral(cgef_plan* p, int32_t enable) {
  int rc = check_plan(p);
  if (rc) return rc;
  if (enable && (p->rs_L == 0 || p->engine != CGEF_ENGINE_BANDED))
    return fail(CGEF_EINVAL, "row-spectral evaluation is not available for this plan (banded engine on a periodic "
                             "x axis or with symmetric rows, and an even FFT length whose half has factors 2, 3, 5 "
                             "only)");
  p->rs_on = enable != 0;
  return CGEF_OK;
}

int32_t cgef_plan_get_row_spectral(const cgef_plan* p, int32_t* available, int32_t* enabled, int32_t* fft_length) {
  if (!p) return fail(CGEF_EINVAL, "plan is NULL");
  const bool banded = p->engine == CGEF_ENGINE_BANDED;
  if (available) *available = banded && p->rs_L > 0;
  if (enabled) *enabled = banded && p->rs_on;
  if (fft_length) *fft_length = banded ? p->rs_L : 0;
  return CGEF_OK;
}

int32_t cgef_plan_get_transfer(const cgef_plan* p, double* transfer) {
  if (!p || !transfer) return fail(CGEF_EINVAL, "plan and transfer must be non-NULL");
  if (p->engine != CGEF_ENGINE_SPECTRAL) return fail(CGEF_EINVAL, "plan is not a spectral-method plan");
  std::copy(p->h_sp_T.begin(), p->h_sp_T.end(), transfer);
  return CGEF_OK;
}

int32_t cgef_plan_get_schedule(const cgef_plan* p, double* waves, int32_t* filter_rows) {
  if (!p) return fail(CGEF_EINVAL, "plan is NULL");
  if (waves) *waves = p->engine == CGEF_ENGINE_BANDED ? p->sched[0].waves : 0.0;
  if (filter_rows) *filter_rows = p->engine == CGEF_ENGINE_BANDED ? p->filter_rows : 0;
  return CGEF_OK;
}

int32_t cgef_plan_autotune(cgef_plan* p, int32_t nbatch, double* chosen) {
  int rc = check_plan(p);
  if (rc) return rc;
  if (nbatch < 1 || nbatch > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  if (p->engine != CGEF_ENGINE_BANDED) {
    if (chosen) *chosen = 0.0;
    return CGEF_OK;
  }
  DeviceGuard dg(p->device);
  cudaStream_t st = p->stream;
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  void* zin = nullptr;
  if ((rc = ensure_ws(p, kSlotIn, sizeof(double) * 2 * N * nbatch, &zin))) return rc;
  cudaError_t e = cudaMemsetAsync(zin, 0, sizeof(double) * 2 * N * nbatch, st);
  if (e != cudaSuccess) return cuda_fail(e, "autotune inputs");
  double* planes = nullptr;
  int pitch = 0, np = 0;
  if ((rc = stage_pi(p, CGEF_F64, zin, static_cast<double*>(zin) + N * nbatch, nbatch, p->d_mask, 0, p->H, &planes,
                     &pitch, &np, st)))
    return rc;
  void* gather = nullptr;
  if ((rc = ensure_ws(p, kSlotGather, sizeof(double) * 5 * N * nbatch, &gather))) return rc;
  cudaEvent_t e0, e1;
  if ((e = cudaEventCreate(&e0)) != cudaSuccess) return cuda_fail(e, "autotune events");
  if ((e = cudaEventCreate(&e1)) != cudaSuccess) {
    cudaEventDestroy(e0);
    return cuda_fail(e, "autotune events");
  }
  // mean device time of `pass`: one untimed pass (workspaces, caches), then three timed ones, or one
  // when a pass takes more than 20 ms
  auto time_pass = [&](auto pass, double* ms_out) -> int {
    int r = pass();
    if (r) return r;
    double ms = 0.0;
    int done = 0;
    while (done < 3) {
      cudaEventRecord(e0, st);
      if ((r = pass())) return r;
      cudaEventRecord(e1, st);
      float one = 0.f;
      cudaError_t ee;
      if ((ee = cudaEventSynchronize(e1)) != cudaSuccess || (ee = cudaEventElapsedTime(&one, e0, e1)) != cudaSuccess)
        return cuda_fail(ee, "autotune timing");
      ms += one;
      ++done;
      if (one > 20.0f) break;
    }
    *ms_out = ms / done;
    return CGEF_OK;
  };
  auto flux_pass = [&] {
    return pi_gather(p, planes, pitch, p->H, np, nbatch, p->d_mask, 0, static_cast<double*>(gather), st);
  };
  // 0. the row-spectral evaluation of the flux's sums, where the plan has it, and the direct gather at
  // the default granularity: when the direct gather is more than twice slower, the spectral evaluation
  // is kept without tuning the direct gather's schedule (at large scales that tuning would cost seconds
  // of gathers that the plan will never run)
  const bool rs_avail = p->rs_L > 0;
  double ms_rs = 1e300;
  if (rs_avail) {
    p->rs_on = true;
    rc = time_pass(flux_pass, &ms_rs);
  }
  p->rs_on = false;
  double best = p->sched[0].waves, best_ms = 1e300;
  // a lower bound on the direct gather's time: its multiply-adds (one per quantity and entry pair of
  // each active target: mirrored columns are paired) at 22.5e12 a second, above the B200's FP64 peak.
  // Where even that is twice the spectral evaluation's time, the direct gather is not timed at all.
  // Only where every target has its band's full entry count: on the sphere (bands hold in-domain rows
  // only, x periodic) and on doubly periodic planes.
  bool direct_hopeless = false;
  if (rc == CGEF_OK && rs_avail && p->periodic_x && (p->geometry == CGEF_SPHERICAL || p->periodic_y)) {
    const int na = (p->geometry == CGEF_SPHERICAL ? 9 : 5) + (p->strategy == CGEF_DEFORMABLE ? 1 : 0);
    double fma = 0.0;
    for (int j = 0; j < p->ny; ++j) {
      const size_t band = p->geometry == CGEF_SPHERICAL ? static_cast<size_t>(j) : 0;
      if (band + 1 >= p->h_ptr.size()) break;
      int64_t act = p->nx;
      if (!p->h_mask.empty()) {
        act = 0;
        for (int i = 0; i < p->nx; ++i) act += p->h_mask[static_cast<size_t>(j) * p->nx + i] != 0;
      }
      fma += static_cast<double>(p->h_ptr[band + 1] - p->h_ptr[band]) * static_cast<double>(act);
    }
    const double lb_ms = 1e3 * fma * nbatch * na * 0.5 / 22.5e12;
    direct_hopeless = lb_ms > 2.0 * ms_rs;
  }
  if (rc == CGEF_OK && !direct_hopeless) rc = time_pass(flux_pass, &best_ms);
  const bool spectral_clear = rc == CGEF_OK && rs_avail && best_ms > 2.0 * ms_rs;
  // 1. split granularity of the direct flux gather's schedule
  const double cand[4] = {2.0, 4.0, 8.0, 16.0};
  for (double w : cand) {
    if (rc != CGEF_OK || spectral_clear) break;
    if (w == best) continue;
    double ms = 0.0;
    if ((rc = rebuild_schedule(p, w, 0))) break;
    if ((rc = time_pass(flux_pass, &ms))) break;
    if (ms < best_ms) {
      best_ms = ms;
      best = w;
    }
  }
  if (rc == CGEF_OK) rc = rebuild_schedule(p, best, 0);
  // 2. tile height of the filter passes (timed on a three-field pass: the velocity gather); the
  // spectral evaluation serves the filter passes too where it is kept
  if (rc == CGEF_OK) rc = rebuild_schedule(p, best, 1);
  if (rc == CGEF_OK && !spectral_clear) {
    const void* f[3] = {zin, zin, zin};
    double* G = static_cast<double*>(gather);
    double* o[3] = {G, G + N, G + 2 * N};
    double ms_r[2] = {0.0, 0.0};
    const int heights[2] = {kRows, kRowsTall};
    for (int k = 0; k < 2 && rc == CGEF_OK; ++k) {
      p->filter_rows = heights[k];
      rc = time_pass([&] { return filter_fields_device(p, CGEF_F64, f, 3, o, 5 * N, nbatch, p->d_mask, 0, st); },
                     &ms_r[k]);
    }
    p->filter_rows = (rc == CGEF_OK && ms_r[1] < ms_r[0]) ? kRowsTall : kRows;
  }
  // 3. direct gather or row-spectral evaluation of the flux's sums, whichever is faster here
  p->rs_on = rc == CGEF_OK && rs_avail && ms_rs < best_ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (chosen) *chosen = best;
  return CGEF_OK;
}

int32_t cgef_plan_get_footprint(const cgef_plan* p, int32_t* di, int32_t* dj, double* w, int64_t* ptr) {
  if (!p) return fail(CGEF_EINVAL, "plan is NULL");
  if (p->engine != CGEF_ENGINE_BANDED) return fail(CGEF_EINVAL, "plan has no banded footprint");
  if (ptr) std::memcpy(ptr, p->h_ptr.data(), p->h_ptr.size() * sizeof(int64_t));
  if (di || dj || w) {
    // a footprint built on the device keeps its weights there only: fetch them for this call
    std::vector<double> fetched;
    if (p->built_on_device) {
      fetched.resize(static_cast<size_t>(std::max<int64_t>(p->nwhalf, 1)));
      DeviceGuard dg(p->device);
      cudaError_t e = cudaMemcpy(fetched.data(), p->d_w, sizeof(double) * p->nwhalf, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) return cuda_fail(e, "footprint weights");
    }
    const int nb = static_cast<int>(p->h_ptr.size()) - 1;
    int64_t k = 0;
    for (int b = 0; b < nb; ++b)
      for_each_entry(
          p, b,
          [&](int ddi, int ddj, double wv) {
            if (di) di[k] = ddi;
            if (dj) dj[k] = ddj;
            if (w) w[k] = wv;
            ++k;
          },
          p->built_on_device ? fetched.data() : nullptr);
  }
  return CGEF_OK;
}

int32_t cgef_filter_device(cgef_plan* p, int32_t dtype, const void* field, void* out, int64_t nbatch, void* stream) {
  int rc = check_plan(p);
  if (rc) return rc;
  DeviceGuard dg(p->device);
  return filter_device(p, dtype, field, out, nbatch, static_cast<cudaStream_t>(stream));
}

int32_t cgef_filter(cgef_plan* p, int32_t dtype, const void* field, void* out, int64_t nbatch) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!field || !out) return fail(CGEF_EINVAL, "field and out must be non-NULL");
  if (nbatch < 1 || nbatch > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  DeviceGuard dg(p->device);
  const size_t bytes = dsize(dtype) * static_cast<size_t>(p->nx) * p->ny * nbatch;
  void *din = nullptr, *dout = nullptr;
  if ((rc = h2d(p, kSlotIn, field, bytes, &din))) return rc;
  if ((rc = ensure_ws(p, kSlotOut, bytes, &dout))) return rc;
  if ((rc = filter_device(p, dtype, din, dout, nbatch, p->stream))) return rc;
  if ((rc = d2h(p, out, dout, bytes))) return rc;
  return sync(p);
}

int32_t cgef_filter_batch(cgef_plan* p, int32_t dtype, const void* const* fields, void* const* outs, int32_t k) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!fields || !outs || k < 1) return fail(CGEF_EINVAL, "need k >= 1 fields and outputs");
  for (int m = 0; m < k; ++m)
    if (!fields[m] || !outs[m]) return fail(CGEF_EINVAL, "field/output pointer is NULL");
  DeviceGuard dg(p->device);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const size_t fb = dsize(dtype) * N;
  void* din = nullptr;
  if ((rc = ensure_ws(p, kSlotIn, fb * k, &din))) return rc;
  for (int m = 0; m < k; ++m) {
    cudaError_t e = cudaMemcpyAsync(static_cast<char*>(din) + fb * m, fields[m], fb, cudaMemcpyHostToDevice, p->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(H2D)");
  }
  void* dout = nullptr;
  if ((rc = ensure_ws(p, kSlotOut, sizeof(double) * N * k, &dout))) return rc;
  void* conv = nullptr;
  if (dtype != CGEF_F64 && (rc = ensure_ws(p, kSlotMask, fb * k, &conv))) return rc;
  for (int m0 = 0; m0 < k; m0 += 4) {
    const int nf = std::min(4, k - m0);
    const void* fl[4];
    double* ol[4];
    for (int m = 0; m < nf; ++m) {
      fl[m] = static_cast<char*>(din) + fb * (m0 + m);
      ol[m] = static_cast<double*>(dout) + N * (m0 + m);
    }
    if ((rc = filter_fields_device(p, dtype, fl, nf, ol, N, 1, p->d_mask, 0, p->stream))) return rc;
  }
  for (int m = 0; m < k; ++m) {
    const void* src = static_cast<double*>(dout) + N * m;
    if (dtype != CGEF_F64) {
      void* c = static_cast<char*>(conv) + fb * m;
      if ((rc = launch_convert(static_cast<const double*>(src), N, c, N, dtype, N, 1, p->stream))) return rc;
      src = c;
    }
    if ((rc = d2h(p, outs[m], src, fb))) return rc;
  }
  return sync(p);
}

int32_t cgef_compute_pi_device(cgef_plan* p, int32_t dtype, const void* u, const void* v, int64_t nbatch,
                               const uint8_t* slice_masks, const cgef_pi_outputs* out, void* stream) {
  int rc = check_plan(p);
  if (rc) return rc;
  DeviceGuard dg(p->device);
  return compute_pi_device(p, dtype, u, v, nbatch, slice_masks, out, static_cast<cudaStream_t>(stream));
}

int32_t cgef_compute_pi_w_device(cgef_plan* p, int32_t dtype, const void* u, const void* v, const void* w,
                                 int64_t nbatch, const uint8_t* slice_masks, const cgef_pi_w_outputs* out,
                                 void* stream) {
  int rc = check_plan(p);
  if (rc) return rc;
  DeviceGuard dg(p->device);
  return compute_pi_w_device(p, dtype, u, v, w, nbatch, slice_masks, out, static_cast<cudaStream_t>(stream));
}

int32_t cgef_compute_pi_w(cgef_plan* p, int32_t dtype, const void* u, const void* v, const void* w, int64_t nbatch,
                          const uint8_t* slice_masks, const cgef_pi_w_outputs* out) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!u || !v || !w) return fail(CGEF_EINVAL, "u, v and w must be non-NULL");
  if (nbatch < 1 || nbatch > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  DeviceGuard dg(p->device);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const size_t fb = dsize(dtype) * N * nbatch;
  void* din = nullptr;
  if ((rc = ensure_ws(p, kSlotIn, 3 * fb, &din))) return rc;
  cudaError_t e = cudaMemcpyAsync(din, u, fb, cudaMemcpyHostToDevice, p->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(static_cast<char*>(din) + fb, v, fb, cudaMemcpyHostToDevice, p->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(static_cast<char*>(din) + 2 * fb, w, fb, cudaMemcpyHostToDevice, p->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(H2D)");
  const uint8_t* dmask = nullptr;
  if (slice_masks) {
    void* dm = nullptr;
    if ((rc = h2d(p, kSlotMask, slice_masks, static_cast<size_t>(N) * nbatch, &dm))) return rc;
    dmask = static_cast<const uint8_t*>(dm);
  }
  cgef_pi_w_outputs none{};
  const cgef_pi_w_outputs* o = out ? out : &none;
  void* const hosts[15] = {o->pi,     o->ubar,   o->vbar,   o->wbar, o->tau_xx, o->tau_xy, o->tau_yy, o->tau_xz,
                           o->tau_yz, o->tau_zz, o->s_xx,   o->s_xy, o->s_yy,   o->s_xz,   o->s_yz};
  int nreq = 0;
  for (void* h : hosts)
    if (h) ++nreq;
  void* dout = nullptr;
  const size_t fba = (fb + 255) / 256 * 256;
  if ((rc = ensure_ws(p, kSlotOut, fba * (nreq > 0 ? nreq : 1) + sizeof(double) * nbatch, &dout))) return rc;
  cgef_pi_w_outputs dev{};
  void** devs[15] = {&dev.pi,     &dev.ubar,   &dev.vbar, &dev.wbar, &dev.tau_xx, &dev.tau_xy, &dev.tau_yy, &dev.tau_xz,
                     &dev.tau_yz, &dev.tau_zz, &dev.s_xx, &dev.s_xy, &dev.s_yy,   &dev.s_xz,   &dev.s_yz};
  int slot = 0;
  for (int m = 0; m < 15; ++m)
    if (hosts[m]) *devs[m] = static_cast<char*>(dout) + fba * slot++;
  double* denergy = reinterpret_cast<double*>(static_cast<char*>(dout) + fba * (nreq > 0 ? nreq : 1));
  if (o->energy) dev.energy = denergy;
  if ((rc = compute_pi_w_device(p, dtype, din, static_cast<char*>(din) + fb, static_cast<char*>(din) + 2 * fb, nbatch,
                                dmask, &dev, p->stream)))
    return rc;
  for (int m = 0; m < 15; ++m)
    if (hosts[m] && (rc = d2h(p, hosts[m], *devs[m], fb))) return rc;
  if (o->energy && (rc = d2h(p, o->energy, denergy, sizeof(double) * nbatch))) return rc;
  return sync(p);
}

int32_t cgef_compute_pi(cgef_plan* p, int32_t dtype, const void* u, const void* v, int64_t nbatch,
                        const uint8_t* slice_masks, const cgef_pi_outputs* out) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!u || !v) return fail(CGEF_EINVAL, "u and v must be non-NULL");
  if (nbatch < 1 || nbatch > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  DeviceGuard dg(p->device);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const size_t fb = dsize(dtype) * N * nbatch;
  void* din = nullptr;
  if ((rc = ensure_ws(p, kSlotIn, 2 * fb, &din))) return rc;
  cudaError_t e = cudaMemcpyAsync(din, u, fb, cudaMemcpyHostToDevice, p->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(static_cast<char*>(din) + fb, v, fb, cudaMemcpyHostToDevice, p->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(H2D)");
  const uint8_t* dmask = nullptr;
  if (slice_masks) {
    void* dm = nullptr;
    if ((rc = h2d(p, kSlotMask, slice_masks, static_cast<size_t>(N) * nbatch, &dm))) return rc;
    dmask = static_cast<const uint8_t*>(dm);
  }
  cgef_pi_outputs none{};
  const cgef_pi_outputs* o = out ? out : &none;
  // device mirrors of the requested outputs
  void* const hosts[9] = {o->pi, o->ubar, o->vbar, o->tau_xx, o->tau_xy, o->tau_yy, o->s_xx, o->s_xy, o->s_yy};
  int nreq = 0;
  for (void* h : hosts)
    if (h) ++nreq;
  void* dout = nullptr;
  const size_t fba = (fb + 255) / 256 * 256;
  if ((rc = ensure_ws(p, kSlotOut, fba * (nreq > 0 ? nreq : 1) + sizeof(double) * nbatch, &dout))) return rc;
  cgef_pi_outputs dev{};
  void** devs[9] = {&dev.pi, &dev.ubar, &dev.vbar, &dev.tau_xx, &dev.tau_xy, &dev.tau_yy, &dev.s_xx, &dev.s_xy, &dev.s_yy};
  int slot = 0;
  for (int m = 0; m < 9; ++m)
    if (hosts[m]) *devs[m] = static_cast<char*>(dout) + fba * slot++;
  double* denergy = reinterpret_cast<double*>(static_cast<char*>(dout) + fba * (nreq > 0 ? nreq : 1));
  if (o->energy) dev.energy = denergy;
  if ((rc = compute_pi_device(p, dtype, din, static_cast<char*>(din) + fb, nbatch, dmask, &dev, p->stream))) return rc;
  for (int m = 0; m < 9; ++m)
    if (hosts[m] && (rc = d2h(p, hosts[m], *devs[m], fb))) return rc;
  if (o->energy && (rc = d2h(p, o->energy, denergy, sizeof(double) * nbatch))) return rc;
  return sync(p);
}

int32_t cgef_sweep_device(cgef_plan* const* plans, int32_t nscales, int32_t dtype, const void* u, const void* v,
                          int64_t nbatch, const uint8_t* slice_masks, void* pi, double* energy, void* stream) {
  if (!plans || nscales < 1 || !plans[0]) return fail(CGEF_EINVAL, "need at least one plan");
  int rc = check_plan(plans[0]);
  if (rc) return rc;
  DeviceGuard dg(plans[0]->device);
  return sweep_device(plans, nscales, dtype, u, v, nbatch, slice_masks, pi, energy, static_cast<cudaStream_t>(stream));
}

}  // extern "C"

struct cgef_graph {
  int device = -1;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t kernels = 0;
};

extern "C" {

int32_t cgef_sweep_graph_create(cgef_graph** out, cgef_plan* const* plans, int32_t nscales, int32_t dtype,
                                const void* u, const void* v, int64_t nbatch, const uint8_t* slice_masks, void* pi,
                                double* energy, void* stream) {
  if (!out) return fail(CGEF_EINVAL, "out is NULL");
  *out = nullptr;
  if (!plans || nscales < 1 || !plans[0]) return fail(CGEF_EINVAL, "need at least one plan");
  int rc = check_plan(plans[0]);
  if (rc) return rc;
  DeviceGuard dg(plans[0]->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (st == nullptr) return fail(CGEF_EINVAL, "capture needs a created stream, not the legacy default stream");
  // a first run sizes every workspace, so the captured call allocates nothing
  if ((rc = sweep_device(plans, nscales, dtype, u, v, nbatch, slice_masks, pi, energy, st))) return rc;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "sweep before capture");
  cgef_graph* g = new (std::nothrow) cgef_graph();
  if (!g) return fail(CGEF_ENOMEM, "graph allocation failed");
  g->device = plans[0]->device;
  prof_suspend(true);
  const int64_t before = g_launches;
  e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rc = sweep_device(plans, nscales, dtype, u, v, nbatch, slice_masks, pi, energy, st);
    cudaError_t e2 = cudaStreamEndCapture(st, &g->graph);
    if (rc == CGEF_OK && e2 != cudaSuccess) rc = cuda_fail(e2, "cudaStreamEndCapture");
  } else {
    rc = cuda_fail(e, "cudaStreamBeginCapture");
  }
  prof_suspend(false);
  g->kernels = g_launches - before;
  g_launches = before;
  if (rc == CGEF_OK && (e = cudaGraphInstantiate(&g->exec, g->graph, 0)) != cudaSuccess)
    rc = cuda_fail(e, "cudaGraphInstantiate");
  if (rc) {
    cgef_graph_destroy(g);
    return rc;
  }
  *out = g;
  return CGEF_OK;
}

int32_t cgef_graph_launch(cgef_graph* g, void* stream) {
  if (!g || !g->exec) return fail(CGEF_EINVAL, "graph is NULL");
  DeviceGuard dg(g->device);
  cudaError_t e = cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
  count_launch(g->kernels);
  return CGEF_OK;
}

int32_t cgef_graph_destroy(cgef_graph* g) {
  if (!g) return CGEF_OK;
  DeviceGuard dg(g->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return CGEF_OK;
}

int32_t cgef_sweep(cgef_plan* const* plans, int32_t nscales, int32_t dtype, const void* u, const void* v,
                   int64_t nbatch, const uint8_t* slice_masks, void* pi, double* energy) {
  if (!plans || nscales < 1 || !plans[0]) return fail(CGEF_EINVAL, "need at least one plan");
  cgef_plan* p = plans[0];
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!u || !v) return fail(CGEF_EINVAL, "u and v must be non-NULL");
  if (nbatch < 1 || nbatch > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  DeviceGuard dg(p->device);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const size_t fb = dsize(dtype) * N * nbatch;
  void* din = nullptr;
  if ((rc = ensure_ws(p, kSlotIn, 2 * fb, &din))) return rc;
  cudaError_t e = cudaMemcpyAsync(din, u, fb, cudaMemcpyHostToDevice, p->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(static_cast<char*>(din) + fb, v, fb, cudaMemcpyHostToDevice, p->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(H2D)");
  const uint8_t* dmask = nullptr;
  if (slice_masks) {
    void* dm = nullptr;
    if ((rc = h2d(p, kSlotMask, slice_masks, static_cast<size_t>(N) * nbatch, &dm))) return rc;
    dmask = static_cast<const uint8_t*>(dm);
  }
  const size_t pib = (fb * nscales + 255) / 256 * 256;
  void* dout = nullptr;
  if ((rc = ensure_ws(p, kSlotOut, (pi ? pib : 0) + sizeof(double) * nscales * nbatch, &dout))) return rc;
  void* dpi = pi ? dout : nullptr;
  double* den = reinterpret_cast<double*>(static_cast<char*>(dout) + (pi ? pib : 0));
  if ((rc = sweep_device(plans, nscales, dtype, din, static_cast<char*>(din) + fb, nbatch, dmask, dpi,
                         energy ? den : nullptr, p->stream)))
    return rc;
  if (pi && (rc = d2h(p, pi, dpi, fb * nscales))) return rc;
  if (energy && (rc = d2h(p, energy, den, sizeof(double) * nscales * nbatch))) return rc;
  return sync(p);
}

int32_t cgef_cumulative_energy(cgef_plan* const* plans, int32_t nscales, int32_t dtype, const void* u, const void* v,
                               double* spectrum) {
  if (!plans || nscales < 1 || !plans[0]) return fail(CGEF_EINVAL, "need at least one plan");
  cgef_plan* p = plans[0];
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!u || !v || !spectrum) return fail(CGEF_EINVAL, "u, v and spectrum must be non-NULL");
  DeviceGuard dg(p->device);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const size_t fb = dsize(dtype) * N;
  void* din = nullptr;
  if ((rc = ensure_ws(p, kSlotIn, 2 * fb, &din))) return rc;
  cudaError_t e = cudaMemcpyAsync(din, u, fb, cudaMemcpyHostToDevice, p->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(static_cast<char*>(din) + fb, v, fb, cudaMemcpyHostToDevice, p->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(H2D)");
  void* dout = nullptr;
  if ((rc = ensure_ws(p, kSlotOut, sizeof(double) * (2 * N + nscales), &dout))) return rc;
  double* uf = static_cast<double*>(dout);
  double* vf = uf + N;
  double* dE = vf + N;
  void* part = nullptr;
  const int64_t nblk = strain_tiles(p);
  if ((rc = ensure_ws(p, kSlotPartials, sizeof(double) * 2 * nblk, &part))) return rc;
  for (int s = 0; s < nscales; ++s) {
    cgef_plan* q = plans[s];
    if ((rc = check_plan(q))) return rc;
    if (q->nx != p->nx || q->ny != p->ny) return fail(CGEF_EINVAL, "all plans must share one grid");
    const void* fl[2] = {din, static_cast<char*>(din) + fb};
    double* ol[2] = {uf, vf};
    // q's own workspace holds its staging; the stream is the first plan's
    if ((rc = filter_fields_device(q, dtype, fl, 2, ol, N, 1, q->d_mask, 0, p->stream))) return rc;
    if ((rc = launch_energy(q, uf, vf, N, q->d_mask, 0, 1, static_cast<double*>(part), dE + s, 1, p->stream))) return rc;
  }
  if ((rc = d2h(p, spectrum, dE, sizeof(double) * nscales))) return rc;
  return sync(p);
}

static int32_t deriv_host(cgef_plan* p, int axis, int32_t dtype, const void* f, void* out) {
  int rc;
  if ((rc = check_plan(p)) || (rc = check_dtype(dtype))) return rc;
  if (!f || !out) return fail(CGEF_EINVAL, "f and out must be non-NULL");
  DeviceGuard dg(p->device);
  const size_t fb = dsize(dtype) * static_cast<size_t>(p->nx) * p->ny;
  void *din = nullptr, *dout = nullptr;
  if ((rc = h2d(p, kSlotIn, f, fb, &din))) return rc;
  if ((rc = ensure_ws(p, kSlotOut, fb, &dout))) return rc;
  if ((rc = launch_derivative(p, axis, dtype, din, dout, p->stream))) return rc;
  if ((rc = d2h(p, out, dout, fb))) return rc;
  return sync(p);
}

int32_t cgef_ddx(cgef_plan* p, int32_t dtype, const void* f, void* out) { return deriv_host(p, 0, dtype, f, out); }
int32_t cgef_ddy(cgef_plan* p, int32_t dtype, const void* f, void* out) { return deriv_host(p, 1, dtype, f, out); }

}  // extern "C"
