// Raw binary mesh and tracer output for the reference's plotting scripts
// (output.cpp).
#pragma once
#include <cstdio>
#include <string>
#include <vector>

#include "mesh.hpp"

namespace fesom {

// mesh_info.txt, coord_nod2D.bin, elem2D_nodes.bin, zbar.bin, depth.bin
void write_mesh_files(const MeshHost &m, const std::string &dir);

// File name of tracer n (1-based): temperature, salinity, tracer3, ...
std::string scalar_name(int n);

// scalar_info.txt plus one stream file per tracer, one (nz, nod2D) FP64
// frame appended per write
class ScalarOutput {
 public:
  ~ScalarOutput() { close(); }
  void open(const std::string &dir, int nod2D, int nz, int nsteps, int ntracers, int wp);
  void write(int tracer, const double *values);  // tracer 0-based
  void close();
  bool is_open() const { return !files_.empty(); }
  int tracers() const { return (int)files_.size(); }

 private:
  std::vector<std::FILE *> files_;
  int nod2D_ = 0, nz_ = 0, frames_ = 0;
};

}  // namespace fesom
