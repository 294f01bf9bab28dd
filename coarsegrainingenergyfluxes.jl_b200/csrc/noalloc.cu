// cgef_filter_device_noalloc: the footprint filter with its scratch in a fixed array compiled
// into the library, for callers that cannot let the library allocate device memory.
//
// The scratch is g_noalloc_scratch below: kNoallocScratchBytes of device memory that every GPU
// which loads the library holds until the process exits.  Host code cannot use the array's name
// as a device address (in host code it names a host-side stand-in), so the address is resolved with
// cudaGetSymbolAddress once per device, with that device current, and kept.  The CUDA driver loads
// this file's module -- and so reserves the array -- only when something first asks for it, and
// resolving the address is that request.  cgef_plan_create therefore resolves it on the plan's
// device (noalloc_prepare), so the allocation-free entry point itself never makes the driver
// reserve memory; should a plan reach it on a device where that did not happen, its call resolves
// the address then.
//
// Every call shares the one array and the array keeps the previous call's contents.  The non-finite
// flags after the staged planes are zeroed by the call (cudaMemsetAsync, which allocates nothing)
// and the staging kernel writes every other element the filter then reads, halos included.  Calls
// whose work overlaps on the GPU (different streams, or different host threads) race on the array and
// must be serialised by the caller.
#include <mutex>

#include "cgef_internal.h"

namespace {

constexpr size_t kNoallocScratchBytes = size_t(64) << 20;  // 64 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device (resolved once per device).
int noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return cgef::fail(CGEF_EINVAL, "device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_ptr[device] == nullptr) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return cgef::cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
    if (ptr == nullptr) return cgef::fail(CGEF_ECUDA, "cudaGetSymbolAddress returned a null address");
    g_noalloc_ptr[device] = ptr;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[device]);
  return CGEF_OK;
}

size_t round256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

int cgef::noalloc_prepare(int device) {
  unsigned char* ptr = nullptr;
  return noalloc_scratch(device, &ptr);
}

extern "C" int32_t cgef_filter_device_noalloc(cgef_plan* p, int32_t dtype, const void* field, void* out,
                                              int64_t nbatch64, void* stream) {
  using namespace cgef;
  if (!p) return fail(CGEF_EINVAL, "plan is NULL");
  if (p->device < 0) return fail(CGEF_ENODEVICE, "no CUDA device was visible when the plan was created");
  if (dtype != CGEF_F64 && dtype != CGEF_F32) return fail(CGEF_EINVAL, "dtype must be CGEF_F64 or CGEF_F32");
  if (!field || !out) return fail(CGEF_EINVAL, "field and out must be non-NULL");
  if (nbatch64 < 1 || nbatch64 > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  const int nbatch = static_cast<int>(nbatch64);
  const int64_t N = static_cast<int64_t>(p->nx) * p->ny;
  const bool def = p->strategy == CGEF_DEFORMABLE;
  const int np = 1 + (def ? 1 : 0);
  const int wide = kTileCols;
  const int nxr = ((p->nx + wide - 1) / wide) * wide;
  const int pitch = ((p->H + nxr + p->H + 32 + 31) / 32) * 32;

  // Scratch layout: staged planes, then the engine's intermediate, then (FP32 callers) the FP64
  // result before conversion.
  const size_t planes_b = round256(stage_bytes(p, np, pitch, nbatch));
  size_t engine_b = 0;
  if (p->engine == CGEF_ENGINE_SEPARABLE) engine_b = round256(sizeof(double) * 2 * static_cast<size_t>(N) * nbatch);
  if (p->engine == CGEF_ENGINE_PREFIXSUM)
    engine_b = round256(sizeof(double) * 2 * static_cast<size_t>(p->ny) * (p->pre_ne + 1) * nbatch);
  if (p->engine == CGEF_ENGINE_BANDED) engine_b = round256(banded_partials_bytes(p, np, nbatch, kModeFields));
  if (p->engine == CGEF_ENGINE_SPECTRAL) engine_b = round256(spectral_scratch_bytes(p, np, nbatch));
  const size_t result_b = dtype == CGEF_F64 ? 0 : round256(sizeof(double) * static_cast<size_t>(N) * nbatch);
  const size_t need = planes_b + engine_b + result_b;
  if (need > kNoallocScratchBytes)
    return fail(CGEF_EINVAL, "cgef_filter_device_noalloc needs " + std::to_string(need) +
                                 " bytes of scratch for this grid and batch, more than its fixed " +
                                 std::to_string(kNoallocScratchBytes) + "-byte array; use cgef_filter_device");

  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (prev != p->device && cudaSetDevice(p->device) != cudaSuccess)
    return fail(CGEF_ECUDA, "cudaSetDevice failed");
  int rc = CGEF_OK;
  unsigned char* base = nullptr;
  prof_suspend(true);
  if ((rc = noalloc_scratch(p->device, &base)) == CGEF_OK) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* planes = reinterpret_cast<double*>(base);
    double* aux = reinterpret_cast<double*>(base + planes_b);
    double* dst = dtype == CGEF_F64 ? static_cast<double*>(out) : reinterpret_cast<double*>(base + planes_b + engine_b);
    StageArgs sa{};
    const void* fl[1] = {field};
    sa.fields = fl;
    sa.nf = 1;
    sa.dtype = dtype;
    sa.mask = p->d_mask;
    sa.mask_slice_stride = 0;
    sa.nbatch = nbatch;
    rc = launch_stage(p, kModeFields, sa, planes, pitch, p->H, np, def, st);
    GatherOut go{};
    go.o[0] = dst;
    go.slice_stride = N;
    if (rc == CGEF_OK) {
      if (p->engine == CGEF_ENGINE_BANDED)
        rc = launch_banded(p, kModeFields, 1, planes, pitch, np, nbatch, p->d_mask, 0, engine_b ? aux : nullptr, go, st,
                          true);
      else if (p->engine == CGEF_ENGINE_SEPARABLE)
        rc = launch_separable(p, kModeFields, 1, planes, pitch, np, nbatch, p->d_mask, 0, aux, go, st);
      else if (p->engine == CGEF_ENGINE_SPECTRAL)
        rc = launch_spectral(p, kModeFields, 1, planes, pitch, np, nbatch, p->masked, aux, go, st);
      else
        rc = launch_prefix(p, kModeFields, 1, planes, pitch, np, nbatch, p->d_mask, 0, aux, go, st);
    }
    if (rc == CGEF_OK && dtype != CGEF_F64) rc = launch_convert(dst, N, out, N, dtype, N, nbatch, st);
  }
  prof_suspend(false);
  if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
  return rc;
}
