// Patch plan of the fused step kernel (tile.cuh).
//
// The fused kernel advances the owned nodes of one patch per thread block.
// An owned node's new value depends on data within three rings of it (its
// edges' MUSCL fluxes read valuesAB within two rings; the FCT ratios of its
// neighbours read low-order solutions within two rings, which read values
// within three), so a block that holds its patch plus three halo rings in
// shared memory needs nothing from other blocks: it recomputes the halo's
// intermediates itself and writes only the owned new values.
//
// Local numbering of a patch (every list in ascending global id):
//   nodes  [ owned O | ring R1 | ring R2 | ring R3 ]   N1 = O+R1, N2 = N1+R2
//   edges  [ E1: an end in N1 | E2 \ E1: an end in N2 ]
//   elements EL: a node in N2 (every up/down triangle of an E1 edge and every
//            ring element of an N2 node)
// Per N2 node: its incident edges in ascending global edge id (the
// reference's serial scatter order) and its element ring in ring order.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "mesh.hpp"

namespace fesom {

constexpr int kTileThreads = 384;       // threads per patch block
constexpr int kTileOwned = 225;         // target owned nodes per patch
constexpr int kTileSmemMax = 227 * 1024;  // dynamic shared memory of a block
constexpr int kTileMaxN3 = 2 * kTileThreads;  // nodes of a patch region (owned + 3 rings)
constexpr int kTileMaxEdges = 2048;     // local edge index bits (11)
constexpr int kTileMaxLevels = 255;     // nlevels fits in 8 bits
constexpr int kTileAH = 3;              // levels of antidiffusive fluxes kept in shared memory
constexpr int kTileR = 3;               // levels of limiter ratios kept in shared memory

// per-patch counts (cumulative node and edge counts)
struct TileCounts {
  int n0, n1, n2, n3;  // |O|, |N1|, |N2|, |N3|
  int e1, e2, nel, jmax;  // |E1|, |E2|, |EL|, deepest wet layer count over N3
  int node_off, inc_off, edge_off, elem_off;  // offsets of the patch's lists
  int ring_off, ptr_off, pad1, pad2;  // ptr_off: first of the patch's n2 + 1 inc_ptr / ring_ptr entries
};

struct TilePlanHost {
  int np = 0;
  int max_n1 = 0, max_n2 = 0, max_n3 = 0, max_e1 = 0, max_e2 = 0, max_el = 0, max_inc = 0;
  std::vector<TileCounts> cnt;
  std::vector<int> node_gid;        // per patch, n3 entries
  std::vector<uint32_t> node_info;  // nlev | nlev_min << 8 | nboundary_lay << 16 | ring_full << 24
  std::vector<int> inc_ptr;         // per patch, n2 + 1 entries from ptr_off
  std::vector<uint32_t> inc;        // local edge | second << 11 | other local node << 12 | edge levels << 22
  std::vector<int> edge_slot;       // per local edge: slot of the edge in the engine's edge order
  std::vector<uint32_t> edge_nn;    // local n1 | local n2 << 10 | edge levels << 20
  std::vector<uint32_t> edge_ud;    // local up element | local down element << 16 (0xffff: none)
  std::vector<int> elem_gid;        // per local element
  std::vector<uint32_t> elem_nn;    // local nodes a | b << 10 | c << 20
  std::vector<int> ring_ptr;        // per patch, n2 + 1 entries from ptr_off
  std::vector<uint16_t> ring;       // local element ids of each N2 node's ring, in ring order
  // redundancy of the plan: region nodes / owned nodes, edges / owned edges
  double node_ratio = 0, edge_ratio = 0;
};

// Device copy of a plan (the same lists, in device memory).
struct DTiles {
  const TileCounts *cnt;
  const int *node_gid;
  const uint32_t *node_info;
  const int *inc_ptr;
  const uint32_t *inc;
  const int *edge_slot;
  const uint32_t *edge_nn;
  const uint32_t *edge_ud;
  const int *elem_gid;
  const uint32_t *elem_nn;
  const int *ring_ptr;
  const uint16_t *ring;
  int np;
};

// Shared-memory layout of a patch block (byte offsets), the same for every
// block of a launch (sized by the plan's maxima).
struct TileLayout {
  unsigned info, incp, inc, eslot, enn, eud, elnn, elg, elv;
  unsigned sT, sA, sG, sVF, sLF, sAH, sLO, sRp, sRm;
  unsigned bytes;
  int n3s, e2s, e1s, n1s;  // strides of the level-buffered arrays (the plan's maxima)
};

inline unsigned tile_align(unsigned x) { return (x + 15u) & ~15u; }

inline TileLayout tile_layout(const TilePlanHost &p, unsigned rsz, bool ab, bool grad, bool fct) {
  TileLayout L{};
  unsigned o = 0;
  auto put = [&](unsigned &f, size_t bytes) {
    f = o;
    o = tile_align(o + (unsigned)bytes);
  };
  put(L.info, 4u * p.max_n3);
  put(L.incp, 4u * (p.max_n2 + 1));
  put(L.inc, 4u * p.max_inc);
  put(L.eslot, 4u * p.max_e2);
  put(L.enn, 4u * p.max_e2);
  put(L.eud, grad ? 4u * p.max_e1 : 0u);
  put(L.elnn, grad ? 4u * p.max_el : 0u);
  put(L.elg, grad ? 4u * p.max_el : 0u);
  put(L.elv, grad ? 1u * p.max_el : 0u);
  put(L.sT, 2u * rsz * p.max_n3);
  put(L.sA, ab ? 0u : 2u * rsz * p.max_n3);
  put(L.sG, grad ? 2u * rsz * p.max_el : 0u);
  put(L.sVF, 2u * rsz * p.max_e2);
  put(L.sLF, fct ? rsz * p.max_e2 : 0u);
  put(L.sAH, (unsigned)kTileAH * rsz * p.max_e1);
  put(L.sLO, fct ? rsz * p.max_n2 : 0u);
  put(L.sRp, fct ? (unsigned)kTileR * rsz * p.max_n1 : 0u);
  put(L.sRm, fct ? (unsigned)kTileR * rsz * p.max_n1 : 0u);
  L.bytes = o;
  L.n3s = p.max_n3;
  L.e2s = p.max_e2;
  L.e1s = p.max_e1;
  L.n1s = p.max_n1;
  return L;
}

// Patches from recursive coordinate bisection of the nodes into parts of
// about max_owned owned nodes (at most max_owned), split further until every
// region fits the block; edge_slot[e] is the engine's storage slot of edge e.  Throws
// std::runtime_error when a single node's region cannot fit (a mesh with
// nl > 255 levels or extreme valence).
TilePlanHost build_tile_plan(const MeshHost &m, const std::vector<int> &edge_slot, int max_owned);

// Checks a plan (host lists still present) against the mesh: every node owned
// by exactly one patch, the three rings, the incidence lists (every incident
// edge in ascending edge id, with the right flags, far node and levels), E1
// membership, up/down triangles, rings, element nodes and the deepest layer.
// Returns "" when consistent, else what failed.
std::string check_tile_plan(const MeshHost &m, const TilePlanHost &plan, const std::vector<int> &edge_slot);

}  // namespace fesom
