// Mesh and per-step tracer output as raw binary files for the reference's
// Python plotting scripts (visualization/plot_mesh.py, plot_scalars.py), in
// the layout of lib/mesh_output.F90:19-161 of suvarchal/fesom2_tracer_dwarf:
//
//   mesh_info.txt     nod2D=, elem2D=, nl=
//   coord_nod2D.bin   float64 (2, nod2D) column-major, metres
//   elem2D_nodes.bin  int32 (3, elem2D) column-major, 0-based
//   zbar.bin          float64 (nl)
//   depth.bin         float64 (nod2D), negative down
//   scalar_info.txt   nod2D=, nz=, nsteps=, num_tracers=, wp=, tracer_<n>=<name>
//   <name>.bin        float64 frames of (nz, nod2D) column-major, one per write
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "output.hpp"

namespace fesom {

namespace {

void make_dir(const std::string &dir) {
  std::error_code ec;
  std::filesystem::create_directories(dir, ec);
  if (!std::filesystem::is_directory(dir)) throw std::runtime_error("cannot create directory " + dir);
}

void write_raw(const std::string &path, const void *data, size_t bytes) {
  std::FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot open " + path);
  const size_t n = bytes ? std::fwrite(data, 1, bytes, f) : 0;
  std::fclose(f);
  if (n != bytes) throw std::runtime_error("short write to " + path);
}

}  // namespace

void write_mesh_files(const MeshHost &m, const std::string &dir) {
  make_dir(dir);
  {
    std::ofstream info(dir + "/mesh_info.txt");
    info << "nod2D=" << m.nod2D << "\n" << "elem2D=" << m.elem2D << "\n" << "nl=" << m.nl << "\n";
    if (!info) throw std::runtime_error("cannot write " + dir + "/mesh_info.txt");
  }
  std::vector<double> xy((size_t)2 * m.nod2D);
  for (size_t i = 0; i < xy.size(); i++) xy[i] = m.coord[i] * kREarth;
  write_raw(dir + "/coord_nod2D.bin", xy.data(), xy.size() * sizeof(double));
  std::vector<int> en(m.elem_nodes.begin(), m.elem_nodes.end());  // already 0-based
  write_raw(dir + "/elem2D_nodes.bin", en.data(), en.size() * sizeof(int));
  write_raw(dir + "/zbar.bin", m.zbar.data(), m.zbar.size() * sizeof(double));
  // the bottom of each node's column (the reference's flat analytic mesh has
  // -max_depth everywhere, which this reproduces)
  std::vector<double> depth(m.nod2D);
  for (int n = 0; n < m.nod2D; n++) depth[n] = m.zbar[m.nlev_node[n] - 1];
  write_raw(dir + "/depth.bin", depth.data(), depth.size() * sizeof(double));
}

std::string scalar_name(int n) {
  if (n == 1) return "temperature";
  if (n == 2) return "salinity";
  return "tracer" + std::to_string(n);
}

void ScalarOutput::open(const std::string &dir, int nod2D, int nz, int nsteps, int ntracers, int wp) {
  close();
  make_dir(dir);
  {
    std::ofstream info(dir + "/scalar_info.txt");
    info << "nod2D=" << nod2D << "\n" << "nz=" << nz << "\n" << "nsteps=" << nsteps << "\n"
         << "num_tracers=" << ntracers << "\n" << "wp=" << wp << "\n";
    for (int n = 1; n <= ntracers; n++) info << "tracer_" << n << "=" << scalar_name(n) << "\n";
    if (!info) throw std::runtime_error("cannot write " + dir + "/scalar_info.txt");
  }
  for (int n = 1; n <= ntracers; n++) {
    std::FILE *f = std::fopen((dir + "/" + scalar_name(n) + ".bin").c_str(), "wb");
    if (!f) {
      close();
      throw std::runtime_error("cannot open " + dir + "/" + scalar_name(n) + ".bin");
    }
    files_.push_back(f);
  }
  nod2D_ = nod2D;
  nz_ = nz;
  frames_ = 0;
}

void ScalarOutput::write(int tracer, const double *values) {
  if (tracer < 0 || tracer >= (int)files_.size()) throw std::out_of_range("scalar output: no such tracer file");
  const size_t n = (size_t)nz_ * nod2D_;
  if (std::fwrite(values, sizeof(double), n, files_[tracer]) != n) throw std::runtime_error("scalar output: short write");
}

void ScalarOutput::close() {
  for (std::FILE *f : files_) std::fclose(f);
  files_.clear();
}

}  // namespace fesom
