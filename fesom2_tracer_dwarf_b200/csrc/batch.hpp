// Multi-member batched stepping (many tracers of many ensemble members on
// meshes of different sizes, advanced together).
//
// Every member is an FP32 Engine that owns its mesh, velocity and tracers.
// Two step paths walk the same work list of (member, 4-tracer batch, block
// of wet cells) items phase by phase -- ring-mean gradients, edge fluxes,
// vertical fluxes and low-order solution, FCT bounds and ratios, limiting and
// update.  Path 0: ONE persistent cooperative launch per step, a grid-wide
// barrier between phases; the kernel swaps the new and old tracer buffers in
// its device-side task table at the end, so the same launch, captured once in
// a CUDA graph, advances the batch step after step.  Path 1: one persistent
// launch per phase and wave over all members (kernel boundaries order the
// phases), each phase kernel with its own register budget and the wave's task
// descriptors passed by value in parameter space, the tasks of each
// work-array slot on their own stream (so that different phase kernels of
// independent slots share the SMs); two steps are captured as one CUDA
// graph.  Tracer batches run in waves of a bounded number per member
// so the work arrays stay small; every member's edge volume fluxes are
// computed once per velocity.  An autotuner picks the path and the tile (wet
// cells per block, i.e. nodes per block x levels), the threads per block and
// persistent grid size of path 0, and the number of tracer batches in
// flight.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "engine.hpp"

namespace fesom {

struct BatchTile {
  int cells_per_block = 512;  // schedule tile (wet cells per block)
  int threads = 256;          // threads per block
  int blocks_per_sm = 2;      // persistent grid = SMs x this
  int wave = 3;               // 4-tracer batches in flight per member
};

struct BatchImpl;

class Batch {
 public:
  Batch();
  ~Batch();
  Batch(const Batch &) = delete;
  Batch &operator=(const Batch &) = delete;

  // Members: FP32 engines on their own meshes; ntracers must be a multiple of 4.
  int add_member(const MeshHost &mesh, int ntracers);
  int num_members() const;
  Engine &member(int i);

  // Scheme (one for every tracer), per-member time steps and valuesAB
  // refresh; then device work arrays and the task table for a tile.
  void configure(const TracerScheme &sch, const std::vector<double> &dt, bool refresh_ab);
  void set_tile(const BatchTile &tile);
  BatchTile tile() const;

  // Step path: 0 = one persistent cooperative launch per step (phases
  // separated by a bounded-wait grid barrier); 1 (default) = one persistent
  // launch per phase and wave over every member's blocks, each phase with the
  // register budget of its standalone kernel and the task descriptors in
  // kernel parameter space.
  void set_path(int path);
  int path() const;

  // Learned antidiffusive flux (MUSCL tracers) on every member with these
  // parameters (nullptr: keep each member's); while on, the batch runs path
  // 2, whose member engines evaluate the MLP between their edge and column
  // kernels, and set_path refuses the persistent paths.
  void set_learned(const float *params, bool on);
  bool learned() const;

  // nsteps steps of the selected path (replayed from a CUDA graph when use_graph).
  void step(int nsteps, bool use_graph);
  // Device time of nsteps (CUDA events on the batch stream), milliseconds;
  // path 2 returns time_separate's host time (one more, untimed step first).
  double time_steps(int nsteps, bool use_graph);
  // The same steps as separate per-member, per-batch kernel launches on the
  // members' streams; with use_graph those launches are replayed from a CUDA
  // graph (two steps per graph).  The timed variant runs one untimed step
  // first and returns the host time of nsteps between device syncs.
  void step_separate(int nsteps, bool use_graph = false);
  double time_separate(int nsteps, bool use_graph = false);

  // Times candidate tiles (steps_per_candidate steps each, from copies of the
  // current tracer state, which is restored afterwards) and keeps the
  // fastest.  Returns a description of every candidate and its time.
  std::string autotune(int steps_per_candidate);

  bool graph_captured() const;
  long long work_bytes() const;
  long long wet_cells() const;  // sum over members of wet cells x tracers

 private:
  BatchImpl *p_;
};

}  // namespace fesom
