// Host-side mesh for the FESOM2 tracer advection step.
//
// MeshHost holds the reference's mesh arrays (lib/MOD_MESH.F90:24-166) that
// the advection step reads, 0-based and level-major per column exactly as the
// Fortran arrays (level index fastest), plus the tables the GPU path is built
// on:
//   * node -> incident-edge lists sorted by edge id, each entry carrying the
//     sign the edge's flux enters the node with; a gather over this list
//     reproduces the reference's serial edge-scatter order bit for bit
//     (lib/oce_adv_tra_driver.F90:122-181, :379-437; lib/oce_adv_tra_fct.F90:281-346);
//   * node -> element rings (nod_in_elem2D);
//   * up/down-wind triangles and nboundary_lay for MUSCL
//     (lib/oce_muscl_adv.F90:96-357).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace fesom {

// Zero-filled host array backed by an anonymous mapping advised as
// transparent huge pages: first-touch faults of multi-GB inputs cost 512x
// fewer page faults than with 4 KB pages (glibc's malloc does not advise).
template <typename T>
class HugeArray {
 public:
  HugeArray() = default;
  explicit HugeArray(size_t n);
  ~HugeArray();
  HugeArray(const HugeArray &) = delete;
  HugeArray &operator=(const HugeArray &) = delete;
  T *data() { return p_; }
  const T *data() const { return p_; }
  T &operator[](size_t i) { return p_[i]; }
  const T &operator[](size_t i) const { return p_[i]; }
  size_t size() const { return n_; }

 private:
  T *p_ = nullptr;
  size_t n_ = 0, bytes_ = 0;
};

constexpr double kREarth = 6367500.0;          // lib/oce_modules.F90:24
constexpr double kPiRef = 3.14159265358979;     // lib/oce_modules.F90:19
constexpr double kCyclicLength = 360.0;         // lib/gen_modules_config.F90:83

struct MeshHost {
  int nl = 0;             // number of levels (interfaces); layers = nl-1
  int nod2D = 0, elem2D = 0, edge2D = 0;
  bool periodic = false;
  bool full_rings = true;
  double Lx = 0, Ly = 0, max_depth = 0;
  // cyclic_length in the units of coord (the reference keeps 360 while its
  // coordinates are radians, so its trim never fires)
  double cyclic_length = kCyclicLength;

  std::vector<double> coord;        // (2, nod2D) radians
  std::vector<int> elem_nodes;      // (3, elem2D)
  std::vector<int> edge_nodes;      // (2, edge2D)
  std::vector<int> edge_tri;        // (2, edge2D), -1 = no element
  std::vector<int> nlev_elem;       // nlevels(elem)
  std::vector<int> nlev_node;       // nlevels_nod2D(node)
  std::vector<int> nlev_node_min;   // nlevels_nod2D_min(node)
  std::vector<int> ring_ptr, ring_elem;  // nod_in_elem2D as CSR
  std::vector<double> elem_area;    // (elem2D) m^2
  std::vector<double> area;         // (nl, nod2D) m^2
  std::vector<double> areasvol;     // (nl, nod2D) m^2
  std::vector<double> edge_dxdy;    // (2, edge2D) radians
  std::vector<double> edge_cross;   // (4, edge2D) m
  std::vector<double> grad_sca;     // (6, elem2D)
  std::vector<double> elem_cos;     // (elem2D)
  std::vector<double> edge_a;       // (edge2D) r_earth * mean elem_cos (MUSCL "a")
  std::vector<double> zbar, Z;      // (nl), (nl-1)
  std::vector<double> hnode, hnode_new;  // (nl-1, nod2D)
  std::vector<double> helem;        // (nl-1, elem2D)
  std::vector<int> up_dn_tri;       // (2, edge2D), -1 = not found
  std::vector<int> nboundary_lay;   // (nod2D)
  std::vector<int> node_edge_ptr;   // CSR over nodes
  std::vector<int> node_edge;       // (edge << 1) | (node is the edge's 2nd node)

  int layers() const { return nl - 1; }
  // Levels an edge carries fluxes on: max(nlevels(el1), nlevels(el2)) - 1.
  int edge_levels(int e) const;
  // Shared levels of an edge: min(...) - 1 (0 on boundary edges).
  int edge_shared_levels(int e) const;
  // Number of wet (node, layer) cells.
  long long wet_cells() const;
  // Finish the derived tables (rings must exist): nlev_node_min, edge_a,
  // up/down triangles, nboundary_lay, node->edge lists.  muscl_tables =
  // false keeps up_dn_tri and nboundary_lay as given (read from a restart).
  void finalize_tables();
  void finalize_tables(bool muscl_tables);
  void build_muscl_tables();  // up/down triangles (from coord) and nboundary_lay
  void build_nboundary_lay();
  std::string validate() const;  // "" when consistent
};

// Analytic rectangular mesh of lib/analytic_mesh.F90:114-829 (doubly periodic
// or closed wall), flat or with a per-node bottom level index node_K
// (length nod2D, values in [3, nl]); full_rings = false keeps the reference's
// incomplete periodic nod_in_elem2D lists; left_oriented = true reverses the
// horizontal and vertical edges so that edge_tri(1) lies left of
// edges(1)->edges(2) on every edge (the reference mesh has it on the right of
// those two families and on the left of the diagonals).
MeshHost build_analytic_mesh(int nx, int ny, int nl, double Lx, double Ly, double max_depth,
                             bool periodic, bool full_rings, const int *node_K, bool left_oriented = false);

// Number of 2D nodes of the analytic mesh.
int analytic_nodes(int nx, int ny, bool periodic);

// Mesh read from the ASCII mesh files of a FESOM2 mesh directory (nod2d.out,
// elem2d.out, aux3d.out, edgenum.out, edges.out, edge_tri.out, elvls.out,
// nlvls.out) as mesh_setup does on one process (lib/oce_mesh.F90:49-94),
// followed by the thicknesses of tracer_init_ale_arrays
// (lib/tracer_c_interface.F90:875-929).  The defaults are the reference's:
// coordinates rotated with the Euler angles (50, 15, -90) passed to cos/sin
// as they are (lib/gen_modules_rotate_grid.F90:42-44) and cyclic_length 360
// against coordinates in radians; angle_scale = pi/180 and cyclic_length =
// 2 pi give FESOM2's conventions.  Throws std::runtime_error naming the file
// on malformed input.
struct MeshFileOptions {
  bool rotate = true;
  double alpha = 50.0, beta = 15.0, gamma = -90.0;
  double angle_scale = 1.0;
  double cyclic_length = kCyclicLength;
};
MeshHost load_mesh_files(const std::string &dir, const MeshFileOptions &opt);

// Seeded per-node bottom level index, uniform in [3, nl] (std::mt19937_64).
std::vector<int> synth_bathymetry(int nnodes, int nl, uint64_t seed);
// Seeded smooth bottom level index of the analytic grid's nodes: a Gaussian
// random field (correlation length about corr_cells grid cells) mapped to a
// uniform marginal on [3, nl].
std::vector<int> synth_bathymetry_smooth(int nx, int ny, bool periodic, int nl, double corr_cells, uint64_t seed);

// Seeded synthetic flow: element velocity u(k) = f1 a1(k) U1 + f2 a2(k) U2 with
// U1 = curl(psi1), U2 = curl(psi2) + grad(chi) smooth periodic patterns and
// a1, a2 the first two cosine modes of the element's own water column (zero
// column mean), scaled to |u| <= umax.  Every edge flux then integrates to
// zero over the column, so W, obtained from the discrete continuity of the
// edge volume fluxes upward from W = 0 at the bottom, closes with W = 0 at the
// surface (to round-off) whatever the orientation convention of edge_tri.
// baro_frac != 0 adds a depth-independent part baro_frac curl(psi0), psi0
// zeroed at nodes next to an element dry at the level and on walls: its edge
// fluxes sum to zero around every node only on a mesh whose edges all carry
// edge_tri(1) on their left (build_analytic_mesh(left_oriented = true)).
// uv: (2, nl-1, elem2D); W: (nl, nod2D).
void synth_velocity(const MeshHost &m, uint64_t seed, double umax, double mode1_frac, double mode2_frac,
                    double baro_frac, double *uv, double *W);

// Seeded tracer fields: kind 0 = temperature-like U[0,20] plus Gaussian blobs,
// kind 1 = salinity-like 35 + N(0, 0.5), kind 2 = smooth blobs and periodic
// tanh fronts (a function of position only: the same field on any
// resolution).  (nl-1, nod2D); dry cells are 0.  In synth_velocity, umax < 0
// takes -umax as the amplitude itself instead of normalising the maximum.
void synth_tracer(const MeshHost &m, uint64_t seed, int kind, double *T);

// Initial fields of the analytic driver (src/fesom_analytic.F90:251-256,306-331).
void analytic_driver_fields(const MeshHost &m, std::vector<double> &T, std::vector<double> &S,
                            std::vector<double> &uv, std::vector<double> &W);

}  // namespace fesom
