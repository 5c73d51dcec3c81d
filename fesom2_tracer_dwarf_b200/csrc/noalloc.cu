// Allocation-free variant of the tracer step: tracer_advect_device_noalloc.
//
// Some callers cannot allocate device memory when they advance a tracer: a
// coupled model whose runtime reserves the GPU's memory for its own pool up
// front (an OpenACC or CUDA host that owns every byte it did not hand out),
// or a time loop that must not stall or fail on an allocation in the middle
// of a run.  They keep their tracer fields in their own device buffers and
// call this entry point, which runs the same kernels as tracer_advect_step
// for one tracer but takes every work array (edge volume fluxes,
// antidiffusive fluxes, low-order solution, limiter ratios) from a fixed
// array that is part of the library image.
//
// The array is a file-scope __device__ variable of kScratchBytes (64 MiB).
// CUDA loads a module's device variables lazily, on first use, so the memory
// behind it is committed on a device when its address is first looked up
// there and then stays until the process exits.  Host code cannot use the
// array's name as a device address: the set-up looks the address up with
// cudaGetSymbolAddress, once per device, with that device current.  That
// set-up runs inside tracer_init_for_advection, on the engine's device, so a
// host that reserves its memory pool after that call does not starve the
// entry point; an engine created another way gets the set-up on its first
// call here, which should then come before the host reserves its pool and
// before any stream capture.
//
// Every call shares the array and overwrites it: calls that overlap on the
// same GPU (for example from two host threads) race; each device has its own
// copy.  No part of it needs to start at zero: each step writes every work
// element before it reads it.
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
void set_last_error(const std::string &s);
}  // namespace fesom

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;
constexpr size_t kScratchDoubles = kScratchBytes / sizeof(double);
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_mu;
double *g_scratch_ptr[kMaxDevices] = {};

// Makes `device` current for the lifetime of the guard and restores the
// caller's current device afterwards.
struct DeviceGuard {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceGuard(int device) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != device) err = cudaSetDevice(device);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Device address of the scratch array on `device` (the current device),
// looked up once per device.  Returns an error message, empty on success.
std::string lookup_scratch(int device, double **out) {
  if (device < 0 || device >= kMaxDevices) return "device index " + std::to_string(device) + " out of range";
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
    g_scratch_ptr[device] = (double *)p;
  }
  *out = g_scratch_ptr[device];
  return "";
}

}  // namespace

namespace fesom {
// Set-up of the static work array on `device`: commits it there and records
// its device address.  Called by tracer_init_for_advection on the engine's
// device.  Returns an error message, empty on success.
std::string noalloc_prepare(int device) {
  DeviceGuard dg(device);
  if (dg.err != cudaSuccess) return std::string("cudaSetDevice failed: ") + cudaGetErrorString(dg.err);
  double *p = nullptr;
  return lookup_scratch(device, &p);
}
}  // namespace fesom

extern "C" long long tracer_noalloc_scratch_bytes(void) { return (long long)kScratchBytes; }

extern "C" int tracer_advect_device_noalloc(int tracer_id, const double *T_dev, const double *TAB_dev,
                                            double *T_out_dev, double dt) {
  try {
    fesom::set_last_error("");
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
    // run on the engine's device whatever the calling thread's current device
    DeviceGuard dg(eng->device());
    if (dg.err != cudaSuccess)
      return fesom::capi_fail(std::string("tracer_advect_device_noalloc: cannot make the engine's device current: ") +
                              cudaGetErrorString(dg.err));
    double *scratch = nullptr;
    const std::string err = lookup_scratch(eng->device(), &scratch);
    if (!err.empty()) return fesom::capi_fail("tracer_advect_device_noalloc: " + err);
    // The step runs on the engine's own stream, which does not wait for the
    // caller's streams: wait here for every piece of work already queued on
    // the device (for example an asynchronous copy that fills T_dev).
    const cudaError_t se = cudaDeviceSynchronize();
    if (se != cudaSuccess)
      return fesom::capi_fail(std::string("tracer_advect_device_noalloc: ") + cudaGetErrorString(se));
    eng->step_with_scratch(tracer_id - 1, T_dev, TAB_dev, T_out_dev, dt, scratch, kScratchDoubles);
    return 0;
  } catch (const std::exception &e) {
    return fesom::capi_fail(e.what());
  }
}
