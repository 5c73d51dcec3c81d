// FESOM2 ASCII mesh directory -> MeshHost, for one process.
//
// Follows mesh_setup (lib/oce_mesh.F90:49-94): read_mesh (nod2d.out with the
// grid rotation, elem2d.out, aux3d.out), test_tri, load_edges, find_neighbors
// (element rings in ascending element order), find_levels (elvls.out,
// nlvls.out), find_levels_min_e2n, mesh_areas and the part of
// mesh_auxiliary_arrays the advection reads; then the uniform thicknesses of
// tracer_init_ale_arrays (lib/tracer_c_interface.F90:875-929).  Every sum and
// product is formed in the reference's order so the geometry is bit-identical
// to a serial evaluation of those routines.
#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "mesh.hpp"

namespace fesom {

namespace {

// Whitespace-separated numbers of one mesh file.
class MeshFile {
 public:
  MeshFile(const std::string &dir, const std::string &name) : name_(name), in_(dir + "/" + name) {
    if (!in_) throw std::runtime_error("mesh: cannot open " + dir + "/" + name);
  }
  template <typename T>
  T next(const char *what) {
    T v{};
    if (!(in_ >> v)) throw std::runtime_error("mesh: " + name_ + ": cannot read " + what);
    return v;
  }
  template <typename T>
  std::vector<T> many(size_t n, const char *what) {
    std::vector<T> v(n);
    for (size_t i = 0; i < n; i++) v[i] = next<T>(what);
    return v;
  }

 private:
  std::string name_;
  std::ifstream in_;
};

// Grid rotation (lib/gen_modules_rotate_grid.F90:33-106); r[i][j] holds
// r2g_matrix(i+1, j+1).
struct Rotation {
  double r[3][3];
  Rotation(double al, double be, double ga) {
    r[0][0] = std::cos(ga) * std::cos(al) - std::sin(ga) * std::cos(be) * std::sin(al);
    r[0][1] = std::cos(ga) * std::sin(al) + std::sin(ga) * std::cos(be) * std::cos(al);
    r[0][2] = std::sin(ga) * std::sin(be);
    r[1][0] = -std::sin(ga) * std::cos(al) - std::cos(ga) * std::cos(be) * std::sin(al);
    r[1][1] = -std::sin(ga) * std::sin(al) + std::cos(ga) * std::cos(be) * std::cos(al);
    r[1][2] = std::cos(ga) * std::sin(be);
    r[2][0] = std::sin(be) * std::sin(al);
    r[2][1] = -std::sin(be) * std::cos(al);
    r[2][2] = std::cos(be);
  }
  // rotated -> geographical (transposed matrix)
  void to_geo(double rlon, double rlat, double &glon, double &glat) const {
    const double x = std::cos(rlat) * std::cos(rlon), y = std::cos(rlat) * std::sin(rlon), z = std::sin(rlat);
    const double gx = r[0][0] * x + r[1][0] * y + r[2][0] * z;
    const double gy = r[0][1] * x + r[1][1] * y + r[2][1] * z;
    const double gz = r[0][2] * x + r[1][2] * y + r[2][2] * z;
    glat = std::asin(gz);
    glon = (gy == 0.0 && gx == 0.0) ? 0.0 : std::atan2(gy, gx);
  }
  // geographical -> rotated
  void to_rot(double glon, double glat, double &rlon, double &rlat) const {
    const double x = std::cos(glat) * std::cos(glon), y = std::cos(glat) * std::sin(glon), z = std::sin(glat);
    const double rx = r[0][0] * x + r[0][1] * y + r[0][2] * z;
    const double ry = r[1][0] * x + r[1][1] * y + r[1][2] * z;
    const double rz = r[2][0] * x + r[2][1] * y + r[2][2] * z;
    rlat = std::asin(rz);
    rlon = (ry == 0.0 && rx == 0.0) ? 0.0 : std::atan2(ry, rx);
  }
};

inline void trim(double &b, double L) {  // trim_cyclic
  if (b > L / 2.0) b = b - L;
  if (b < -L / 2.0) b = b + L;
}

}  // namespace

MeshHost load_mesh_files(const std::string &dir, const MeshFileOptions &opt) {
  MeshHost m;
  const double L = opt.cyclic_length;
  const double rad = kPiRef / 180.0;  // lib/oce_modules.F90:20
  m.cyclic_length = L;
  m.periodic = false;
  m.full_rings = true;
  const Rotation rot(opt.alpha * opt.angle_scale, opt.beta * opt.angle_scale, opt.gamma * opt.angle_scale);

  // nodes, degrees -> radians, rotated; the reference refuses a mesh that
  // already has ocean next to the rotated pole when asked to rotate it, and
  // one without ocean there when not (lib/oce_mesh.F90:245-330)
  {
    MeshFile f(dir, "nod2d.out");
    const int N = f.next<int>("the node count");
    if (N < 3) throw std::runtime_error("mesh: nod2d.out: fewer than 3 nodes");
    m.nod2D = N;
    m.coord.resize(2 * (size_t)N);
    double xp, yp;
    rot.to_geo(0.0 * rad, 90.0 * rad, xp, yp);
    xp = xp / rad;
    yp = yp / rad;
    const double box = 2.5;
    bool near_pole = false;
    for (int n = 0; n < N; n++) {
      f.next<long>("a node id");
      const double lon = f.next<double>("a longitude"), lat = f.next<double>("a latitude");
      f.next<long>("a node flag");
      const double shift = lon > 180.0 ? -360.0 : (lon < -180.0 ? 360.0 : 0.0);
      if (lon + shift >= xp - box && lon + shift <= xp + box && lat >= yp - box && lat <= yp + box) near_pole = true;
      double x = lon * rad, y = lat * rad;
      if (opt.rotate) {
        const double gx = x, gy = y;
        rot.to_rot(gx, gy, x, y);
      }
      m.coord[2 * n] = x;
      m.coord[2 * n + 1] = y;
    }
    if (opt.rotate && near_pole)
      throw std::runtime_error("mesh: the nodes seem to be rotated already (ocean next to the rotated pole)");
    if (!opt.rotate && !near_pole)
      throw std::runtime_error("mesh: the nodes seem to be unrotated (no ocean next to the rotated pole)");
  }
  const int N = m.nod2D;

  // elements, 1-based in the file; clockwise order fixed as test_tri does
  {
    MeshFile f(dir, "elem2d.out");
    const int T = f.next<int>("the element count");
    if (T < 1) throw std::runtime_error("mesh: elem2d.out: no elements");
    m.elem2D = T;
    m.elem_nodes = f.many<int>(3 * (size_t)T, "element nodes");
    for (int &v : m.elem_nodes) {
      if (v < 1 || v > N) throw std::runtime_error("mesh: elem2d.out: node index out of range");
      v -= 1;
    }
    for (int e = 0; e < T; e++) {
      int *el = &m.elem_nodes[3 * (size_t)e];
      const double ax = m.coord[2 * el[0]], ay = m.coord[2 * el[0] + 1];
      double bx = m.coord[2 * el[1]] - ax, by = m.coord[2 * el[1] + 1] - ay;
      double cx = m.coord[2 * el[2]] - ax, cy = m.coord[2 * el[2] + 1] - ay;
      trim(bx, L);
      trim(cx, L);
      if (bx * cy - by * cx > 0.0) std::swap(el[1], el[2]);
    }
  }
  const int T = m.elem2D;

  // standard levels (depths are read for completeness; the step uses the
  // level counts of elvls/nlvls)
  {
    MeshFile f(dir, "aux3d.out");
    const int nl = f.next<int>("the level count");
    if (nl < 3) throw std::runtime_error("mesh: aux3d.out: fewer than 3 levels");
    m.nl = nl;
    m.zbar = f.many<double>((size_t)nl, "a level depth");
    if (m.zbar[1] > 0.0)
      for (double &z : m.zbar) z = -z;
    m.Z.resize(nl - 1);
    for (int k = 0; k < nl - 1; k++) m.Z[k] = 0.5 * (m.zbar[k] + m.zbar[k + 1]);
    f.many<double>((size_t)N, "a node depth");
    m.max_depth = -m.zbar[nl - 1];
  }
  const int nl = m.nl;

  // edges (load_edges); a missing second element is stored as -1
  {
    MeshFile fn(dir, "edgenum.out");
    const int E = fn.next<int>("the edge count");
    fn.next<int>("the inner edge count");
    if (E < 1) throw std::runtime_error("mesh: edgenum.out: no edges");
    m.edge2D = E;
    MeshFile fe(dir, "edges.out"), ft(dir, "edge_tri.out");
    m.edge_nodes = fe.many<int>(2 * (size_t)E, "edge nodes");
    m.edge_tri = ft.many<int>(2 * (size_t)E, "edge elements");
    for (int &v : m.edge_nodes) {
      if (v < 1 || v > N) throw std::runtime_error("mesh: edges.out: node index out of range");
      v -= 1;
    }
    for (int &v : m.edge_tri) {
      if (v > T) throw std::runtime_error("mesh: edge_tri.out: element index out of range");
      v = v > 0 ? v - 1 : -1;
    }
    for (int e = 0; e < E; e++)
      if (m.edge_tri[2 * (size_t)e] < 0) throw std::runtime_error("mesh: edge_tri.out: an edge without a first element");
  }
  const int E = m.edge2D;

  // rings (nod_in_elem2D) and the neighbour check of find_neighbors
  m.ring_ptr.assign(N + 1, 0);
  for (int v : m.elem_nodes) m.ring_ptr[v + 1]++;
  for (int n = 0; n < N; n++) m.ring_ptr[n + 1] += m.ring_ptr[n];
  m.ring_elem.resize(m.ring_ptr[N]);
  {
    std::vector<int> fill(m.ring_ptr.begin(), m.ring_ptr.end() - 1);
    for (int e = 0; e < T; e++)
      for (int q = 0; q < 3; q++) m.ring_elem[fill[m.elem_nodes[3 * (size_t)e + q]]++] = e;
    std::vector<int> sides(T, 0), neighbours(T, 0);
    for (int e = 0; e < E; e++) {
      const int t1 = m.edge_tri[2 * (size_t)e], t2 = m.edge_tri[2 * (size_t)e + 1];
      sides[t1]++;
      if (t2 >= 0) {
        sides[t2]++;
        neighbours[t1]++;
        neighbours[t2]++;
      }
    }
    for (int t = 0; t < T; t++)
      if (sides[t] != 3 || neighbours[t] < 2)
        throw std::runtime_error("mesh: element " + std::to_string(t + 1) + " has not three edges or fewer than two neighbours");
  }

  // levels
  {
    MeshFile fe(dir, "elvls.out"), fn(dir, "nlvls.out");
    m.nlev_elem = fe.many<int>((size_t)T, "an element level count");
    m.nlev_node = fn.many<int>((size_t)N, "a node level count");
    for (int v : m.nlev_elem)
      if (v < 3 || v > nl) throw std::runtime_error("mesh: elvls.out: level count outside [3, nl]");
    for (int v : m.nlev_node)
      if (v < 3 || v > nl) throw std::runtime_error("mesh: nlvls.out: level count outside [3, nl]");
  }

  // mesh_areas: element areas on the sphere, nodal areas from the rings
  m.elem_area.resize(T);
  for (int e = 0; e < T; e++) {
    const int *el = &m.elem_nodes[3 * (size_t)e];
    double ay = (m.coord[2 * el[0] + 1] + m.coord[2 * el[1] + 1] + m.coord[2 * el[2] + 1]) / 3.0;
    ay = std::cos(ay);
    double ax_ = m.coord[2 * el[1]] - m.coord[2 * el[0]], ay_ = m.coord[2 * el[1] + 1] - m.coord[2 * el[0] + 1];
    double bx_ = m.coord[2 * el[2]] - m.coord[2 * el[0]], by_ = m.coord[2 * el[2] + 1] - m.coord[2 * el[0] + 1];
    trim(ax_, L);
    trim(bx_, L);
    ax_ = ax_ * ay;
    bx_ = bx_ * ay;
    m.elem_area[e] = 0.5 * std::fabs(ax_ * by_ - bx_ * ay_);
  }
  m.area.assign((size_t)nl * N, 0.0);
  m.areasvol.assign((size_t)nl * N, 0.0);
  for (int n = 0; n < N; n++) {
    double *a = &m.area[(size_t)n * nl];
    for (int p = m.ring_ptr[n]; p < m.ring_ptr[n + 1]; p++) {
      const int t = m.ring_elem[p];
      for (int k = 0; k < m.nlev_elem[t] - 1; k++) a[k] = a[k] + m.elem_area[t] / 3.0;
    }
    for (int k = 0; k < m.nlev_node[n] - 1; k++) m.areasvol[(size_t)n * nl + k] = a[k];
  }
  for (double &v : m.elem_area) v = v * kREarth * kREarth;
  for (size_t i = 0; i < m.area.size(); i++) {
    m.area[i] = m.area[i] * kREarth * kREarth;
    m.areasvol[i] = m.areasvol[i] * kREarth * kREarth;
  }

  // mesh_auxiliary_arrays: element centres and cosines, edge vectors, the
  // edge-centre -> element-centre cross vectors, P1 gradients
  std::vector<double> cx(T), cy(T);
  m.elem_cos.resize(T);
  for (int e = 0; e < T; e++) {
    const int *el = &m.elem_nodes[3 * (size_t)e];
    double ax[3] = {m.coord[2 * el[0]], m.coord[2 * el[1]], m.coord[2 * el[2]]};
    const double amin = std::min(std::min(ax[0], ax[1]), ax[2]);
    for (double &x : ax) {
      if (x - amin >= L / 2.0) x = x - L;
      if (x - amin < -L / 2.0) x = x + L;
    }
    cx[e] = (ax[0] + ax[1] + ax[2]) / 3.0;
    cy[e] = (m.coord[2 * el[0] + 1] + m.coord[2 * el[1] + 1] + m.coord[2 * el[2] + 1]) / 3.0;
    m.elem_cos[e] = std::cos(cy[e]);
  }
  m.edge_dxdy.resize(2 * (size_t)E);
  m.edge_cross.resize(4 * (size_t)E);
  for (int e = 0; e < E; e++) {
    const int a = m.edge_nodes[2 * (size_t)e], b = m.edge_nodes[2 * (size_t)e + 1];
    double dx = m.coord[2 * b] - m.coord[2 * a];
    trim(dx, L);
    m.edge_dxdy[2 * (size_t)e] = dx;
    m.edge_dxdy[2 * (size_t)e + 1] = m.coord[2 * b + 1] - m.coord[2 * a + 1];
    double ax = m.coord[2 * a], bx = m.coord[2 * b];
    if (ax - bx > L / 2.0) ax = ax - L;
    if (ax - bx < -L / 2.0) bx = bx - L;
    const double mx = 0.5 * (ax + bx), my = 0.5 * (m.coord[2 * a + 1] + m.coord[2 * b + 1]);
    for (int s = 0; s < 2; s++) {
      const int t = m.edge_tri[2 * (size_t)e + s];
      double *c = &m.edge_cross[4 * (size_t)e + 2 * s];
      if (t < 0) {
        c[0] = c[1] = 0.0;
        continue;
      }
      double qx = cx[t] - mx, qy = cy[t] - my;
      trim(qx, L);
      qx = qx * m.elem_cos[t];
      c[0] = qx * kREarth;
      c[1] = qy * kREarth;
    }
  }
  m.grad_sca.resize(6 * (size_t)T);
  for (int e = 0; e < T; e++) {
    const int *el = &m.elem_nodes[3 * (size_t)e];
    double dX31 = m.coord[2 * el[2]] - m.coord[2 * el[0]];
    trim(dX31, L);
    dX31 = m.elem_cos[e] * dX31;
    double dX21 = m.coord[2 * el[1]] - m.coord[2 * el[0]];
    trim(dX21, L);
    dX21 = m.elem_cos[e] * dX21;
    const double dY31 = m.coord[2 * el[2] + 1] - m.coord[2 * el[0] + 1];
    const double dY21 = m.coord[2 * el[1] + 1] - m.coord[2 * el[0] + 1];
    const double f = -(0.5 * kREarth / m.elem_area[e]);
    double *gs = &m.grad_sca[6 * (size_t)e];
    gs[0] = (-dY31 + dY21) * f;
    gs[1] = dY31 * f;
    gs[2] = -(dY21 * f);
    gs[3] = (dX31 - dX21) * f;
    gs[4] = -(dX31 * f);
    gs[5] = dX21 * f;
  }

  // the coordinate box (domain of the seeded synthetic fields), metres
  {
    double x0 = m.coord[0], x1 = x0, y0 = m.coord[1], y1 = y0;
    for (int n = 1; n < N; n++) {
      x0 = std::min(x0, m.coord[2 * n]);
      x1 = std::max(x1, m.coord[2 * n]);
      y0 = std::min(y0, m.coord[2 * n + 1]);
      y1 = std::max(y1, m.coord[2 * n + 1]);
    }
    m.Lx = (x1 - x0) * kREarth;
    m.Ly = (y1 - y0) * kREarth;
  }

  // uniform layer thicknesses (tracer_init_ale_arrays)
  m.hnode.resize((size_t)(nl - 1) * N);
  m.helem.resize((size_t)(nl - 1) * T);
  for (int n = 0; n < N; n++)
    for (int k = 0; k < nl - 1; k++) m.hnode[(size_t)n * (nl - 1) + k] = m.zbar[k] - m.zbar[k + 1];
  for (int e = 0; e < T; e++)
    for (int k = 0; k < nl - 1; k++) m.helem[(size_t)e * (nl - 1) + k] = m.zbar[k] - m.zbar[k + 1];
  m.hnode_new = m.hnode;

  m.finalize_tables();
  const std::string bad = m.validate();
  if (!bad.empty()) throw std::runtime_error("mesh: " + bad);
  return m;
}

}  // namespace fesom
