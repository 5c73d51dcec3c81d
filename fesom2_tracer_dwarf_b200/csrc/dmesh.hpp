// Device-resident mesh tables and work schedules.
//
// Edge arrays are stored in "slot" order -- edges sorted by their first node,
// so the edges of neighbouring nodes sit next to each other -- while every
// node-side gather still walks its edges in ascending edge id, the order of
// the reference's serial scatters.
//
// HBM layout: every 3D field is column-major per node (or element, or edge)
// with the level index fastest and a padded level stride S (multiple of 4
// levels, so every column starts on a 32-byte sector for FP64).  A cell
// (column c, level k, 0-based) lives at c*S + k.  The 2D tables are
// structure-of-arrays in int2/double2/double4 records so one vector load
// fetches an edge's nodes, elements or cross distances.
//
// Work is scheduled over wet cells only: a schedule lists, for groups of
// consecutive columns, the prefix sums of their wet-level counts, so a block
// walks a dense range of wet cells and every lane has work even where the
// bathymetry leaves most of a column dry.
#pragma once
#include <cuda_runtime.h>

namespace fesom {

// Schedule over "items" (nodes or edges) with a variable number of levels.
struct DSched {
  const int *cell_off;  // (n_items + 1) prefix sums of wet levels
  const int *blk;       // (nblk + 1) first item of each block
  int nblk;
  int max_items;        // largest item count in one block
};

template <typename R>
struct DMeshT {
  int N, T, E, nl, S;
  // 2D tables
  const int2 *edge_nodes;   // (n1, n2)
  const int2 *edge_tri;     // (el1, el2), el2 = -1 on boundary edges
  const int2 *edge_lev;     // (shared levels = min(nl1, nl2), edge levels = max(nl1, nl2))
  const R *edge_cross;      // (4, E): dX1, dY1, dX2, dY2
  const R *edge_dxdy;       // (2, E)
  const R *edge_a;          // (E)
  const int2 *up_dn;        // (up, dn) triangles, -1 = none
  const int *nlev_elem;     // nlevels(elem)
  const int *nlev_node;     // nlevels_nod2D
  const int *nlev_node_min; // nlevels_nod2D_min
  const int *nbl;           // nboundary_lay
  const int *elem_nodes;    // (3, T)
  const R *grad_sca;        // (6, T)
  const R *elem_area;       // (T)
  const int *ring_ptr;      // (N+1)
  const int *ring_elem;
  const unsigned char *ring_full;  // (N) 1: the ring holds every element of the node
  const int *ne_ptr;        // (N+1)
  const int4 *ne4;          // per incidence, in ascending edge id:
                            // (slot << 1 | node is the edge's 2nd node, other node, edge levels,
                            //  other node x S: its column base)
  const R *zbar;            // (nl)
  const R *Z;               // (nl-1)
  // 3D geometry, stride S
  const R *area;            // node, nl levels
  const R *areasvol;        // node
  const R *hnode;           // node
  const R *hnode_new;       // node
  const R *helem;           // element
  // reciprocals 1/areasvol (plane 0) and 1/hnode_new (plane 1) of the wet
  // cells, S x N each, computed once per mesh (k_rcp_planes)
  const R *rcp;
  size_t rcp_plane;         // S * N
  DSched node_sched;        // items = nodes, levels = nlev_node - 1
  DSched edge_sched;        // items = edges, levels = edge levels
  // node-levels whose MUSCL gradient is the ring mean for some incident edge
  // (levels grad_lev0[n] .. nlev_node[n]-2 of node n)
  const int *grad_lev0;
  DSched grad_sched;        // items = nodes, levels = nlev_node - 1 - grad_lev0
};

}  // namespace fesom
