// Domain-decomposed tracer step: one engine per mesh part (partition.hpp),
// the parts of this process on its GPU, halo values exchanged after every
// step.  Within a process the exchange is a device copy between the parts'
// engines; between processes the caller moves the packed halo buffers (one
// per peer, (nl-1) levels x nodes, FP64) with NCCL and unpacks them.
#pragma once
#include <memory>
#include <vector>

#include "engine.hpp"
#include "partition.hpp"

namespace fesom {

class Decomposition {
 public:
  // Parts `local_parts` of the node -> part map `node_part` (nparts parts)
  // of the global mesh g, each with `rings` halo rings, as FP64 or FP32
  // engines.
  Decomposition(const MeshHost &g, const std::vector<int> &node_part, int nparts, const std::vector<int> &local_parts,
                int rings, Precision prec);
  ~Decomposition();
  Decomposition(const Decomposition &) = delete;
  Decomposition &operator=(const Decomposition &) = delete;

  int nparts() const;
  int num_local() const;
  const MeshPart &part(int i) const;
  Engine &engine(int i);

  // Global-layout inputs and outputs (the whole mesh's arrays): every local
  // part takes its local rows; get_values writes the owned rows only.
  void allocate_tracers(int ntr);
  void set_scheme(int id, const TracerScheme &s);
  void set_velocity(const double *uv, const double *w);
  void set_values(int id, const double *v);
  void get_values(int id, double *out) const;

  // One step of every tracer on every local part (no exchange).
  void step(double dt, bool refresh_ab);
  // Halo values of every tracer between the parts held here.
  void exchange_local();
  // Nodes of the transfer from local part i to part `peer` (send) or from
  // `peer` to local part i (receive).
  int transfer_nodes(int i, int peer, bool send) const;
  // Owned values of local part i that `peer` needs, as (nl-1) x n FP64 on
  // the device (node-major, level fastest); and the reverse.
  void pack(int i, int id, int peer, double *dev_out);
  void unpack(int i, int id, int peer, const double *dev_in);
  void synchronize() const;

 private:
  struct Impl;
  std::unique_ptr<Impl> p_;
};

}  // namespace fesom
