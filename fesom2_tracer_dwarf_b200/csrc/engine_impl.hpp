// Engine internals shared by the host engine (engine.cu) and the
// per-precision kernel translation units (step_f64.cu, step_f32.cu).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "dmesh.hpp"
#include "engine.hpp"
#include "tile.hpp"

namespace fesom {

#define CK(x)                                                                                          \
  do {                                                                                                 \
    cudaError_t e_ = (x);                                                                              \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr int kBatchMax = 4;  // tracers per batch (NTMAX of the kernels)

// Device pointers of one batch of tracers, untyped (the element types follow
// the engine's precision mode).
struct BatchPtrs {
  const void *T[kBatchMax] = {};
  const void *TAB[kBatchMax] = {};
  void *T_out[kBatchMax] = {};
  void *adf_h[kBatchMax] = {};
  void *adf_v[kBatchMax] = {};
  void *lo[kBatchMax] = {};
  void *rpm[kBatchMax] = {};  // (2, S, node): R+ and R- side by side
  void *vflux = nullptr;
  int vflux_mode = 0;             // edge volume fluxes (FusedArgs::vflux_mode)
  void *gradn[kBatchMax] = {};
  void *feat[kBatchMax] = {};     // learned flux: features (BF16 x 16) per edge cell
  void *fscale[kBatchMax] = {};   // learned flux: correction scale per edge cell
  double off[kBatchMax] = {};     // storage offsets (16-bit storage)
  uint32_t seed[kBatchMax] = {};  // stochastic-rounding streams
  int sround = 0;
};

struct LearnedState;  // mlp.cu

struct EngineImpl {
  MeshHost mesh;
  LearnedState *learn = nullptr;  // learned antidiffusive flux (FP32 engines)
  std::vector<int> slot_edge;  // edge stored in each slot
  int cells_per_block = 512;   // schedule tile
  int S = 0;
  Precision prec = Precision::FP64;
  bool fma64 = false;    // FP64 mode with FMA-contracted kernels (step_f64fma.cu)
  size_t ts_bytes = 8;  // tracer storage element
  size_t r_bytes = 8;   // compute / geometry / work element
  cudaStream_t stream = nullptr;
  int device = 0;  // current CUDA device when the engine was created
  std::vector<void *> allocs;
  size_t bytes = 0;
  DMeshT<double> dm64{};
  DMeshT<float> dm32{};
  void *vel = nullptr, *W = nullptr;
  struct Tracer {
    void *T = nullptr, *Tout = nullptr, *TAB = nullptr;
    TracerScheme sch;
    double off = 0.0;    // 16-bit storage holds T - off on wet cells
    uint32_t nstep = 0;  // steps taken (stochastic-rounding stream)
  };
  int sround = 0;        // 1: stochastic rounding of 16-bit stores
  uint32_t sround_seed = 0x2545f491u;
  // transfers (transfer.cu): device staging of one tracer in the user's
  // (nl-1, nod2D) FP64 layout, and a ring of pinned host slots
  static constexpr int kRing = 4;
  double *stage_d = nullptr;
  double *stats_d = nullptr;  // per-block partial statistics (tracer_stats)
  // pipelined host-I/O step (Engine::step_io): per-tracer device buffers of
  // the host layout, the two copy streams and their events
  std::vector<double *> io_in, io_out;
  cudaStream_t io_h2d = nullptr, io_d2h = nullptr;
  std::vector<cudaEvent_t> io_ev_in, io_ev_out;
  unsigned long long *nonfinite_d = nullptr;  // non-finite new values written by the steps
  void *ring[kRing] = {};
  cudaEvent_t ring_ev[kRing] = {};
  std::vector<Tracer> tr;
  int slots = 0;
  void *vflux = nullptr;
  bool vflux_valid = false;  // vflux holds the edge volume fluxes of the current velocity
  // fused patch kernel (tile.cuh): the plan's maxima (host lists released
  // after upload) and its device copy; step_path 0 runs it wherever the
  // scheme allows, 1 (the default, faster on B200) the five-kernel path
  TilePlanHost tplan;
  DTiles tiles{};
  int step_path = 1;
  void *adfh[kBatchMax] = {}, *adfv[kBatchMax] = {}, *lo[kBatchMax] = {}, *rpm[kBatchMax] = {};
  void *gradn[kBatchMax] = {};

  // launch profiling: when prof is set, every launch is bracketed by events
  struct ProfRec {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<ProfRec> *prof = nullptr;
  void mark_begin(int kind) {
    if (!prof) return;
    ProfRec r{kind, nullptr, nullptr};
    CK(cudaEventCreate(&r.a));
    CK(cudaEventCreate(&r.b));
    CK(cudaEventRecord(r.a, stream));
    prof->push_back(r);
  }
  void mark_end() {
    if (!prof) return;
    CK(cudaEventRecord(prof->back().b, stream));
  }

  void *dalloc_bytes(size_t n) {
    void *p = nullptr;
    if (n == 0) n = 8;
    CK(cudaMalloc(&p, n));
    CK(cudaMemsetAsync(p, 0, n, stream));
    allocs.push_back(p);
    bytes += n;
    return p;
  }
  template <typename T>
  T *dalloc(size_t n) {
    return (T *)dalloc_bytes(n * sizeof(T));
  }
  void dfree(void *p) {
    if (!p) return;
    auto it = std::find(allocs.begin(), allocs.end(), p);
    if (it == allocs.end()) return;  // not ours
    allocs.erase(it);
    cudaFree(p);
  }
  // Every transfer is ordered on the engine's stream (which does not
  // synchronise with the legacy default stream) and completes before the call
  // returns, so host staging buffers may be released right after.
  void h2d(void *d, const void *h, size_t n) {
    if (!n) return;
    CK(cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
  }
  void d2h(void *h, const void *d, size_t n) {
    if (!n) return;
    CK(cudaMemcpyAsync(h, d, n, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
  }
  void d2d(void *dst, const void *src, size_t n) {
    if (!n) return;
    CK(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToDevice, stream));
    CK(cudaStreamSynchronize(stream));
  }
  template <typename T>
  T *upload(const std::vector<T> &h) {
    T *d = dalloc<T>(h.size());
    h2d(d, h.data(), h.size() * sizeof(T));
    return d;
  }
};

// Kernel kinds reported by profile_steps.
enum { KK_EDGE = 0, KK_COL1, KK_COL2, KK_COL3, KK_GRAD, KK_TILE, KK_VFLUX, KK_COUNT };

// Launch one batch of nt tracers (kernels in step_f64.cu / step_f32.cu).
void launch_batch_f64(EngineImpl &P, const TracerScheme &sc, int nt, const BatchPtrs &b, double dt);
void launch_batch_f32(EngineImpl &P, const TracerScheme &sc, int nt, const BatchPtrs &b, double dt);
// The FP64 kernels built with FMA contraction (step_f64fma.cu).
void launch_batch_f64fma(EngineImpl &P, const TracerScheme &sc, int nt, const BatchPtrs &b, double dt);
// Whether the fused patch kernel runs a batch of this scheme (precision,
// storage type, vertical scheme, learned flux and plan permitting).
bool fused_step(const EngineImpl &P, const TracerScheme &sc, bool learned);
// Geometry reciprocals of k_col3 (step_f64.cu / step_f32.cu).
void build_rcp_f64(EngineImpl &P);
void build_rcp_f32(EngineImpl &P);
// Compensated FP64 sums of T and of T * areasvol * hnode_new over the wet
// cells of one tracer.
void volume_sum_f64(EngineImpl &P, const void *T, double out[2]);
void volume_sum_f32(EngineImpl &P, const void *T, double off, double out[2]);

// Transfers of one tracer field (transfer.cu).  stage_upload / stage_download
// move a host (nl-1, nod2D) FP64 array to / from the device staging array
// (one DMA for ranges registered with host_register, a pinned ring
// otherwise); stage_pack converts the staging array into up to three storage
// arrays (wet cells minus off), stage_unpack the reverse (plus off).
void stage_upload(EngineImpl &P, const double *host);
void stage_download(EngineImpl &P, double *host);
double stage_wet_mean(EngineImpl &P);
void stage_pack(EngineImpl &P, double off, void *d0, void *d1, void *d2);
void stage_unpack(EngineImpl &P, const void *s, double off);
void storage_reoffset(EngineImpl &P, void *s, double off_old, double off_new);
// Host-I/O step helpers (FP64 / FP32 storage): whether a host range lies in
// page-locked memory; (nl-1, nod2D) doubles -> storage arrays and back, on a
// given stream with explicit device buffers.
bool host_range_pinned(const void *p, size_t bytes);
void pack_from(EngineImpl &P, const double *src, cudaStream_t st, void *d0, void *d1, void *d2);
void unpack_to(EngineImpl &P, const void *s, double *dst, cudaStream_t st);
// min, max, sum and NaN count of a tracer over the (nl-1, nod2D) values the
// host reads back, reduced on the device (transfer.cu)
void tracer_stats(EngineImpl &P, const void *s, double off, double out[4]);
void release_ring(EngineImpl &P);

// Learned flux (mlp.cu): after the edge kernel wrote features and scales,
// adds scale x MLP(features) to the antidiffusive edge fluxes of nt tracers.
template <typename R, typename TS>
struct FusedArgs;
void learned_correct_f32(EngineImpl &P, int nt, const FusedArgs<float, float> &a);
void learned_release(EngineImpl &P);
bool learned_active(const EngineImpl &P);
void learned_slot_buffers(EngineImpl &P, int t, void **feat, void **scale);

}  // namespace fesom
