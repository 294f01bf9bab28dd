// Streaming sweep: snapshots submitted from host memory one after another, each copied in, swept
// and copied out, with the copies of one snapshot overlapping the sweep of its neighbours.  The
// host side of the reference's batch driver loops over snapshots synchronously
// (Pipeline.jl:519-563, 686-717); this is that loop with the transfers taken off the critical path.
//
// Three streams and two device buffer sets: snapshot k copies into input set k % 2 on the H2D
// stream, is swept on the compute stream into output set k % 2, and is copied out on the D2H
// stream.  Events keep each set from being overwritten while the step two back still reads it.
// Each set's sweep runs call by call on its first submit (which sizes every workspace) and is then
// captured as a CUDA graph that the later submits replay, so the host issues one launch per sweep.
// The graphs hold the plans as they were at that first submit.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "cgef_internal.h"

using namespace cgef;

struct cgef_pipeline {
  int device = -1;
  std::vector<cgef_plan*> plans;
  int nscales = 0, dtype = 0, nbatch = 0;
  bool want_pi = true;
  size_t in_bytes = 0, pi_bytes = 0, e_bytes = 0;
  cudaStream_t h2d = nullptr, comp = nullptr, d2h = nullptr;
  void* d_in[2] = {nullptr, nullptr};
  void* d_pi[2] = {nullptr, nullptr};
  double* d_e[2] = {nullptr, nullptr};
  uint8_t* d_mask = nullptr;
  cudaEvent_t in_ready[2] = {}, in_free[2] = {}, out_ready[2] = {}, out_free[2] = {};
  cudaGraph_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  int64_t graph_kernels[2] = {0, 0};
  bool no_graph[2] = {false, false};  // a capture failed: this set keeps launching call by call
  int64_t submitted = 0;
};

namespace {

void release(cgef_pipeline* p) {
  for (int b = 0; b < 2; ++b) {
    if (p->exec[b]) cudaGraphExecDestroy(p->exec[b]);
    if (p->graph[b]) cudaGraphDestroy(p->graph[b]);
    if (p->d_in[b]) cudaFree(p->d_in[b]);
    if (p->d_pi[b]) cudaFree(p->d_pi[b]);
    if (p->d_e[b]) cudaFree(p->d_e[b]);
    for (cudaEvent_t e : {p->in_ready[b], p->in_free[b], p->out_ready[b], p->out_free[b]})
      if (e) cudaEventDestroy(e);
  }
  if (p->d_mask) cudaFree(p->d_mask);
  for (cudaStream_t s : {p->h2d, p->comp, p->d2h})
    if (s) cudaStreamDestroy(s);
}

int sweep_set(cgef_pipeline* p, int b) {
  const char* din = static_cast<const char*>(p->d_in[b]);
  return sweep_device(p->plans.data(), p->nscales, p->dtype, din, din + p->in_bytes, p->nbatch, p->d_mask,
                      p->want_pi ? p->d_pi[b] : nullptr, p->d_e[b], p->comp);
}

// Captures set b's sweep on the compute stream (nothing runs; the workspaces are sized already).
void capture_set(cgef_pipeline* p, int b) {
  prof_suspend(true);
  const int64_t before = cgef_launch_count();
  cudaError_t e = cudaStreamBeginCapture(p->comp, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const int rc = sweep_set(p, b);
    e = cudaStreamEndCapture(p->comp, &p->graph[b]);
    if (rc != CGEF_OK && e == cudaSuccess) e = cudaErrorUnknown;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec[b], p->graph[b], 0);
  prof_suspend(false);
  p->graph_kernels[b] = cgef_launch_count() - before;
  count_launch(-p->graph_kernels[b]);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (p->exec[b]) cudaGraphExecDestroy(p->exec[b]);
    if (p->graph[b]) cudaGraphDestroy(p->graph[b]);
    p->exec[b] = nullptr;
    p->graph[b] = nullptr;
    p->no_graph[b] = true;
  }
}

}  // namespace

extern "C" {

int32_t cgef_pipeline_create(cgef_pipeline** out, cgef_plan* const* plans, int32_t nscales, int32_t dtype,
                             int64_t nbatch, const uint8_t* slice_masks, int32_t want_pi) {
  if (!out) return fail(CGEF_EINVAL, "out is NULL");
  *out = nullptr;
  if (!plans || nscales < 1 || !plans[0]) return fail(CGEF_EINVAL, "need at least one plan");
  int rc;
  if ((rc = check_plan(plans[0])) || (rc = check_dtype(dtype))) return rc;
  if (nbatch < 1 || nbatch > 65535) return fail(CGEF_EINVAL, "nbatch must be in 1..65535");
  for (int s = 0; s < nscales; ++s)
    if ((rc = check_plan(plans[s]))) return rc;
  DeviceGuard dg(plans[0]->device);
  cgef_pipeline* p = new (std::nothrow) cgef_pipeline();
  if (!p) return fail(CGEF_ENOMEM, "pipeline allocation failed");
  p->device = plans[0]->device;
  p->plans.assign(plans, plans + nscales);
  p->nscales = nscales;
  p->dtype = dtype;
  p->nbatch = static_cast<int>(nbatch);
  p->want_pi = want_pi != 0;
  const size_t N = static_cast<size_t>(plans[0]->nx) * plans[0]->ny;
  p->in_bytes = dsize(dtype) * N * p->nbatch;
  p->pi_bytes = p->want_pi ? dsize(dtype) * N * p->nbatch * nscales : 0;
  p->e_bytes = sizeof(double) * p->nbatch * nscales;
  cudaError_t e = cudaSuccess;
  for (cudaStream_t* s : {&p->h2d, &p->comp, &p->d2h})
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
    e = cudaMalloc(&p->d_in[b], 2 * p->in_bytes);
    if (e == cudaSuccess && p->want_pi) e = cudaMalloc(&p->d_pi[b], p->pi_bytes);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&p->d_e[b]), p->e_bytes);
    for (cudaEvent_t* ev : {&p->in_ready[b], &p->in_free[b], &p->out_ready[b], &p->out_free[b]})
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  }
  if (e == cudaSuccess && slice_masks) {
    e = cudaMalloc(reinterpret_cast<void**>(&p->d_mask), N * p->nbatch);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_mask, slice_masks, N * p->nbatch, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    release(p);
    delete p;
    return cuda_fail(e, "pipeline setup");
  }
  *out = p;
  return CGEF_OK;
}

int32_t cgef_pipeline_submit(cgef_pipeline* p, const void* u, const void* v, void* pi, double* energy) {
  if (!p) return fail(CGEF_EINVAL, "pipeline is NULL");
  if (!u || !v) return fail(CGEF_EINVAL, "u and v must be non-NULL");
  if (p->want_pi && !pi) return fail(CGEF_EINVAL, "this pipeline returns Pi: pi must be non-NULL");
  DeviceGuard dg(p->device);
  const int b = static_cast<int>(p->submitted & 1);
  char* din = static_cast<char*>(p->d_in[b]);
  cudaError_t e;
  // copy in, once the sweep two steps back has finished reading this input set
  if ((e = cudaStreamWaitEvent(p->h2d, p->in_free[b], 0)) != cudaSuccess) return cuda_fail(e, "pipeline wait");
  if ((e = cudaMemcpyAsync(din, u, p->in_bytes, cudaMemcpyHostToDevice, p->h2d)) != cudaSuccess ||
      (e = cudaMemcpyAsync(din + p->in_bytes, v, p->in_bytes, cudaMemcpyHostToDevice, p->h2d)) != cudaSuccess)
    return cuda_fail(e, "pipeline H2D");
  if ((e = cudaEventRecord(p->in_ready[b], p->h2d)) != cudaSuccess) return cuda_fail(e, "pipeline event");
  // sweep, once the inputs are in and the copy-out two steps back has released this output set
  if ((e = cudaStreamWaitEvent(p->comp, p->in_ready[b], 0)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(p->comp, p->out_free[b], 0)) != cudaSuccess)
    return cuda_fail(e, "pipeline wait");
  if (p->exec[b]) {
    if ((e = cudaGraphLaunch(p->exec[b], p->comp)) != cudaSuccess) return cuda_fail(e, "pipeline graph launch");
    count_launch(p->graph_kernels[b]);
  } else {
    const int rc = sweep_set(p, b);
    if (rc) return rc;
    if (!p->no_graph[b]) capture_set(p, b);
  }
  if ((e = cudaEventRecord(p->in_free[b], p->comp)) != cudaSuccess ||
      (e = cudaEventRecord(p->out_ready[b], p->comp)) != cudaSuccess)
    return cuda_fail(e, "pipeline event");
  // copy out
  if ((e = cudaStreamWaitEvent(p->d2h, p->out_ready[b], 0)) != cudaSuccess) return cuda_fail(e, "pipeline wait");
  if (p->want_pi && (e = cudaMemcpyAsync(pi, p->d_pi[b], p->pi_bytes, cudaMemcpyDeviceToHost, p->d2h)) != cudaSuccess)
    return cuda_fail(e, "pipeline D2H");
  if (energy && (e = cudaMemcpyAsync(energy, p->d_e[b], p->e_bytes, cudaMemcpyDeviceToHost, p->d2h)) != cudaSuccess)
    return cuda_fail(e, "pipeline D2H");
  if ((e = cudaEventRecord(p->out_free[b], p->d2h)) != cudaSuccess) return cuda_fail(e, "pipeline event");
  ++p->submitted;
  return CGEF_OK;
}

int32_t cgef_pipeline_drain(cgef_pipeline* p) {
  if (!p) return fail(CGEF_EINVAL, "pipeline is NULL");
  DeviceGuard dg(p->device);
  cudaError_t e = cudaStreamSynchronize(p->d2h);
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->comp);
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->h2d);
  return e == cudaSuccess ? CGEF_OK : cuda_fail(e, "pipeline drain");
}

int32_t cgef_pipeline_destroy(cgef_pipeline* p) {
  if (!p) return CGEF_OK;
  DeviceGuard dg(p->device);
  cudaStreamSynchronize(p->d2h);
  cudaStreamSynchronize(p->comp);
  cudaStreamSynchronize(p->h2d);
  release(p);
  delete p;
  return CGEF_OK;
}

}  // extern "C"
