// Allocation-free variant of the tracer step: tracer_advect_device_noalloc.
//
// Some callers cannot allocate device memory when they advance a tracer: a
// coupled model whose runtime reserves the GPU's memory for its own pool up
// front (an OpenACC or CUDA host that owns every byte it did not hand out),
// or a time loop that must not stall or fail on an allocation in the middle
// of a run.  They keep their tracer fields in their own device buffers and
// call this entry point, which runs the same four kernels as
// tracer_advect_step for one tracer but takes every work array (edge volume
// fluxes, antidiffusive fluxes, low-order solution, limiter ratios) from a
// fixed array that is part of the library image.
//
// The array is a file-scope __device__ variable of kScratchBytes (64 MiB):
// every GPU that loads the library holds it until the process exits.  Host
// code cannot use its name as a device address, so the first call on a device
// looks the address up with cudaGetSymbolAddress (with that device current)
// and keeps it; that first call should therefore come before any stream
// capture.  Every call shares the array and overwrites it: calls that overlap
// on the same GPU (for example from two host threads) race; each device has
// its own copy.  No part of it needs to start at zero: each step writes every
// work element before it reads it.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/fesom_tracer.h"
#include "engine.hpp"

namespace fesom {
Engine *capi_engine();
int capi_num_tracers();
bool capi_initialized();
int capi_fail(const std::string &msg);
}  // namespace fesom

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;
constexpr size_t kScratchDoubles = kScratchBytes / sizeof(double);
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_mu;
double *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device.
int scratch_on_current_device(double **out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fesom::capi_fail("tracer_advect_device_noalloc: no current CUDA device");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fesom::capi_fail(std::string("tracer_advect_device_noalloc: cudaGetSymbolAddress failed: ") +
                              cudaGetErrorString(e));
    g_scratch_ptr[dev] = (double *)p;
  }
  *out = g_scratch_ptr[dev];
  return 0;
}

}  // namespace

extern "C" long long tracer_noalloc_scratch_bytes(void) { return (long long)kScratchBytes; }

extern "C" int tracer_advect_device_noalloc(int tracer_id, const double *T_dev, const double *TAB_dev,
                                            double *T_out_dev, double dt) {
  try {
    if (!fesom::capi_initialized()) return fesom::capi_fail("tracer not initialized. Call tracer_init first.");
    fesom::Engine *eng = fesom::capi_engine();
    if (!eng)
      return fesom::capi_fail("tracer_advect_device_noalloc: the device state does not exist yet "
                              "(call tracer_init_for_advection once before)");
    if (tracer_id < 1 || tracer_id > fesom::capi_num_tracers())
      return fesom::capi_fail("invalid tracer_id " + std::to_string(tracer_id));
    if (!T_dev || !TAB_dev || !T_out_dev) return fesom::capi_fail("tracer_advect_device_noalloc: null buffer");
    if (T_out_dev == T_dev || T_out_dev == TAB_dev)
      return fesom::capi_fail("tracer_advect_device_noalloc: T_out must not alias T or TAB");
    if (!(dt > 0.0)) return fesom::capi_fail("dt must be positive");
    const size_t need = eng->step_scratch_doubles();
    if (need > kScratchDoubles)
      return fesom::capi_fail("tracer_advect_device_noalloc: this mesh needs " +
                              std::to_string(need * sizeof(double)) + " bytes of work space, more than the " +
                              std::to_string(kScratchBytes) + "-byte static array");
    double *scratch = nullptr;
    if (scratch_on_current_device(&scratch)) return -1;
    eng->step_with_scratch(tracer_id - 1, T_dev, TAB_dev, T_out_dev, dt, scratch, kScratchDoubles);
    return 0;
  } catch (const std::exception &e) {
    return fesom::capi_fail(e.what());
  }
}
