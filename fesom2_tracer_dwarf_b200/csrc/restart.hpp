// Binary restarts in the reference's derived-type format
// (lib/io_restart_derivedtype.F90:33-199): per rank r of npes, the files
//   <dir>/np<npes>/t_mesh.<r>, t_partit.<r>, t_tracer.<r>, t_dynamics.<r>
// each holding one Fortran unformatted sequential record written by the
// type's user-defined WRITE(UNFORMATTED) procedure (lib/MOD_MESH.F90:185-279,
// lib/MOD_PARTIT.F90 WRITE_T_PARTIT, lib/MOD_TRACER.F90:104-206,
// lib/MOD_DYN.F90:256-312), plus the metadata file <dir>/meta.time.
//
// Record framing is gfortran's: a 4-byte length before and after the
// payload; payloads longer than 2^31 - 9 bytes are split into subrecords whose
// leading marker is negative on every subrecord but the last and whose
// trailing marker is negative on every subrecord but the first.  Inside a
// record, every child WRITE adds its items back to back (no markers):
// default integers and logicals are 4 bytes, reals (WP = MP = 8) 8 bytes,
// character(20) 20 bytes; an allocatable array is its extents (4 bytes each,
// all zero when unallocated) followed by its elements in column-major order;
// a static array is its size followed by its elements.
#pragma once
#include <string>
#include <vector>

#include "engine.hpp"
#include "mesh.hpp"

namespace fesom {

struct RestartData {
  MeshHost mesh;                              // connectivity, geometry, MUSCL tables
  std::vector<std::vector<double>> values;    // per tracer (nl-1, nod2D)
  std::vector<std::vector<double>> values_ab; // per tracer (nl-1, nod2D)
  std::vector<TracerScheme> schemes;
  std::vector<int> ids;                       // tracer IDs
  std::vector<double> uv;                     // (2, nl-1, elem2D); empty: none stored
  std::vector<double> w;                      // (nl, nod2D)
};

// Writes the four record files of rank 0 of one process into
// <dir>/np1/ (created) and <dir>/meta.time.  Throws std::runtime_error.
void write_restart(const std::string &dir, const RestartData &r);

// Reads <dir>/np1/*.0 (one process).  The mesh comes back with its MUSCL
// tables from the tracer record and no node coordinates (the mesh record
// holds none).  Throws std::runtime_error naming the file and the field.
RestartData read_restart(const std::string &dir, bool want_tracers, bool want_dynamics);

}  // namespace fesom
