// Domain decomposition of a mesh into parts with halos.
//
// A part owns a set of nodes and holds, as its local mesh, those nodes plus
// `rings` rings of neighbouring nodes (halo), the elements whose three nodes
// are all local, and the edges between local nodes whose first element is
// local.  Local nodes, elements and edges keep the global order within their
// class (owned nodes first, then halo nodes; elements and edges in ascending
// global id), so every gather of the step walks the same edges and elements
// in the same order as on the whole mesh.
//
// The new value of an owned node depends on values within three rings: its
// own edges' high-order fluxes read valuesAB and gradients within two rings,
// and the FCT ratios of its neighbours read their bounds (low-order solution
// within two rings, itself reading values within three) and their edges'
// fluxes.  With rings = 3 every quantity an owned node reads is computed on
// the part exactly as on the whole mesh (edges and elements cut by the halo
// boundary only touch third-ring nodes), so one exchange of the halo values
// after each step replaces the reference's three exchanges (low-order
// solution, FCT ratios, new values: lib/oce_adv_tra_driver.F90:234,
// lib/oce_adv_tra_fct.F90:383) at the price of computing the halo redundantly.
#pragma once
#include <string>
#include <vector>

#include "mesh.hpp"

namespace fesom {

struct MeshPart {
  int part = 0;
  int owned = 0;                  // local nodes [0, owned) are owned
  MeshHost mesh;                  // local mesh
  std::vector<int> node_global;   // local -> global node
  std::vector<int> elem_global;   // local -> global element
  std::vector<int> edge_global;   // local -> global edge
};

// Nodes of part `part` and their `rings` rings of neighbours that other parts
// own (the halo), ascending global id.
std::vector<int> halo_nodes(const MeshHost &g, const std::vector<int> &node_part, int part, int rings);

MeshPart build_mesh_part(const MeshHost &g, const std::vector<int> &node_part, int part, int rings);

// Halo exchange lists between two parts: global ids of the nodes `from`
// owns that lie in the halo of `to`, ascending.
std::vector<int> halo_transfer(const MeshHost &g, const std::vector<int> &node_part, int from, int to, int rings);

// Simple partitions: contiguous strips of ascending node id
// (each part a band of rows on the analytic mesh).
std::vector<int> partition_by_index(int nod2D, int parts);

// Node -> part map of a FESOM2 partition directory dist_<n>
// (lib/oce_mesh.F90:150-200): rpart.out gives the part count and the owned
// node count of each part, my_list<part>.out the part id, myDim_nod2D,
// eDim_nod2D and the owned then halo nodes (1-based) of that part.  Every
// node must be owned by exactly one part.
std::vector<int> read_dist_partition(const std::string &dist_dir, int nod2D, int *parts);

}  // namespace fesom
