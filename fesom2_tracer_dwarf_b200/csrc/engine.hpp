// Tracer advection engine: owns the device copy of one mesh, its velocity
// and any number of tracers, and advances them with the CUDA kernels.
//
// Host arrays cross this interface in the reference's Fortran layouts
// (column-major, level fastest): tracers (nl-1, nod2D), uv (2, nl-1, elem2D),
// w (nl, nod2D).  On the device every column is padded to a level stride S.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "mesh.hpp"

namespace fesom {

struct TracerScheme {
  int hor = 0;      // 0 UPW1, 1 MUSCL, 2 MFCT
  int ver = 0;      // 0 UPW1, 1 PPM, 2 QR4C, 3 CDIFF
  int lim = 0;      // 0 NONE, 1 FCT
  double ph = 1.0;  // tra_adv_ph
  double pv = 1.0;  // tra_adv_pv
};

// Arithmetic / storage modes.  FP64: the bit-exact drop-in.  FP32: FP32
// tracers, geometry and arithmetic.  BF16 / FP16: 16-bit tracer storage with
// FP32 arithmetic and accumulation.  In the FP32-based modes the FCT ratio
// denominators are formed in FP64.
enum class Precision { FP64 = 0, FP32 = 1, BF16 = 2, FP16 = 3 };

struct EngineImpl;

// Storage slot of every edge in the engine's edge arrays (edges sorted by
// their smaller node id, stable in edge id).
std::vector<int> edge_slot_order(const MeshHost &m);

// Page-lock a host range for single-DMA tracer transfers (transfer.cu);
// 0 on success.
int host_register(void *p, size_t bytes);
int host_unregister(void *p);

class Engine {
 public:
  explicit Engine(const MeshHost &mesh, Precision prec = Precision::FP64);
  Precision precision() const;
  // Compensated FP64 sums over the wet cells of tracer id: out[0] = Sum T,
  // out[1] = Sum T * areasvol * hnode_new (the conserved tracer content).
  void volume_sum(int id, double out[2]) const;
  // 16-bit storage: 0 rounds new values to nearest, 1 rounds them
  // stochastically (a reproducible per-step, per-tracer, per-cell stream)
  void set_rounding(int mode);
  int rounding() const;
  // offset subtracted from a tracer's wet cells in 16-bit storage (0 otherwise)
  double storage_offset(int id) const;
  ~Engine();
  Engine(const Engine &) = delete;
  Engine &operator=(const Engine &) = delete;

  const MeshHost &mesh() const;
  int level_stride() const;
  // Schedule tile: the most wet cells a block of the step kernels takes
  // (32..576, default 512: two per thread of a 256-thread block).
  static constexpr int kDefaultCellsPerBlock = 512;
  void set_cells_per_block(int cells);
  int cells_per_block() const;
  // Internal state, for the multi-member batch runner (batch.cu).
  EngineImpl *impl();

  // Learned antidiffusive flux (FP32 engines, MUSCL tracers): the edge kernel
  // writes 16 features per edge cell and the MLP's output, times a local
  // scale, is added to the antidiffusive flux before the vertical and FCT
  // kernels.  params (packed MLP parameters) = nullptr keeps the current ones.
  void set_learned(const float *params, bool on);
  bool learned() const;
  void get_learned(float *params) const;
  // gradient of the loss of the last updating learn_step (before its update)
  void get_learned_grad(float *grad) const;
  // One training step on tracer 0: values := T_in, one MUSCL+PPM step (with
  // the FCT limiter when fct) and the learned correction, loss =
  // volume-weighted mean squared difference to T_target; with update, one
  // Adam step of rate lr on the MLP.  With the limiter the gradient goes
  // through its ratios R+/- (fct_grad) or holds its factors at their forward
  // values.  Returns the loss before the update.  Both arrays (nl-1, nod2D).
  double learn_step(const double *T_in, const double *T_target, double dt, double lr, bool update, bool fct = false,
                    bool fct_grad = true);

  void set_velocity(const double *uv, const double *w);
  void set_velocity_zero();
  // (Re)allocate ntr tracers, all zero, default scheme UPW1/UPW1/NONE.
  // with_ab = false: no separate valuesAB arrays (valuesAB := values only).
  void allocate_tracers(int ntr, bool with_ab = true);
  // Frees the per-batch work arrays (reallocated by the next step).
  void release_work();
  int num_tracers() const;
  // values -> tracer id (0-based); valuesAB follows when also_ab.
  void set_values(int id, const double *v, bool also_ab);
  void set_values_ab(int id, const double *v);
  void get_values(int id, double *out) const;
  // valuesAB of tracer id (its own array, or the values when it has none)
  void get_values_ab(int id, double *out) const;
  void set_scheme(int id, const TracerScheme &s);
  TracerScheme scheme(int id) const;
  // Advance every tracer one step.  refresh_ab: valuesAB := values first.
  void step(double dt, bool refresh_ab);
  // One step with host I/O, pipelined per tracer: in[t] (nullable) becomes
  // tracer t's values (and valuesAB), every tracer is advanced, out[t]
  // (nullable) receives its new values.  Each tracer's upload, step and
  // download run on their own streams so that tracer t+1's upload and
  // tracer t-1's download overlap tracer t's step.  Needs page-locked host
  // arrays (tracer_host_register) and FP64 or FP32 storage; returns false
  // (nothing done) otherwise.
  bool step_io(double dt, bool refresh_ab, const double *const *in, double *const *out);
  // Advance one tracer one step (the reference's tracer_advect_step on id).
  void step_tracer(int id, double dt, bool refresh_ab);
  // Device pointers / stream for benchmarking and tests.
  void *stream() const;
  // CUDA device the engine was created on (current device at construction)
  int device() const;
  // FP64 engines: true runs the kernels built with FMA contraction (about
  // 1e-13 relative to the bit-exact ones, fewer FP64 instructions)
  void set_fma64(bool on);
  bool fma64() const;
  // Non-finite new values the steps have written since the last reset
  // (counted on the device by the update kernels); reset = true zeroes it.
  long long nonfinite_values(bool reset);
  // Step kernels: 0 = the fused patch kernel wherever the scheme allows it
  // (FP64 or FP32 storage, PPM or UPW1 vertical, no learned flux), else the
  // five-kernel path; 1 (default) = always the five-kernel path.  Both give
  // the same bits in FP64.
  void set_step_path(int path);
  int step_path() const;
  bool fused(int id) const;      // whether tracer id's steps run the fused kernel
  int tile_count() const;        // patches of the fused kernel's plan (0: none)
  // Rebuilds the fused kernel's plan with patches of about `owned` owned
  // nodes (default kTileOwned); any size gives the same results.
  void set_patch_size(int owned);
  double tile_node_ratio() const;  // LO-solution nodes computed per node (halo redundancy)
  void synchronize() const;
  // Kernel launches issued by one step() of every tracer.
  int launches_per_step() const;
  // min, max, sum and NaN count of tracer id over (nl-1, nod2D) incl. dry
  // cells, in the reference's sequential order (src/fesom_analytic.F90:441-446).
  void stats(int id, double out4[4]) const;
  size_t device_bytes() const;
  // Per-kernel device time: run nsteps steps of every tracer with a CUDA
  // event pair around each launch and add the milliseconds of each kernel
  // kind into ms[kind] (kinds: kernel_kind_names()).  Returns launches done.
  int profile_steps(int nsteps, double dt, bool refresh_ab, double *ms, int nkinds);
  static const char *const *kernel_kind_names(int *n);
  // Doubles of work space one tracer step needs (edge volume fluxes,
  // antidiffusive fluxes, LO solution, limiter ratios).
  size_t step_scratch_doubles() const;
  // One step of tracer id's scheme on caller-owned device buffers in the
  // engine's layout (nod2D columns of level stride S): T and TAB in, T_out
  // out, with every work array carved from `scratch` (step_scratch_doubles()
  // doubles, 256-byte aligned).  Allocates nothing; returns when the step is
  // done.
  void step_with_scratch(int id, const double *T, const double *TAB, double *T_out, double dt, double *scratch,
                         size_t scratch_doubles);

 private:
  EngineImpl *p_;
};

// Last CUDA / engine error message of this thread ("" if none).
const char *last_error();
void set_last_error(const std::string &s);

}  // namespace fesom
