// Analytic mesh construction and derived tables (host, C++17).
//
// The geometry follows the reference's formulas operation for operation, so
// the arrays come out bit-identical to what lib/analytic_mesh.F90 and
// lib/oce_mesh.F90 compute: coordinates (lib/analytic_mesh.F90:268-305),
// areas (lib/oce_mesh.F90:2043-2309), edge and cross distances and P1
// gradient coefficients (lib/oce_mesh.F90:2313-2534), the periodic
// minimum-image fix and halo-area merge (lib/analytic_mesh.F90:756-782).
// Build it on the host once; the device only ever sees the finished tables.
#include "mesh.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <sstream>
#include <stdexcept>

namespace fesom {

namespace {

inline void trim_cyclic(double &b, double L = kCyclicLength) {  // lib/gen_modules_rotate_grid.F90:216-223
  if (b > L / 2.0) b = b - L;
  if (b < -L / 2.0) b = b + L;
}
inline void trim_period(double &v, double P) {
  if (v > 0.5 * P) v = v - P;
  if (v < -0.5 * P) v = v + P;
}

// Grid description shared by the steps of the builder.  "Extended" node ids
// include the periodic halo copies (right column, top row, corner) that carry
// shifted coordinates until the geometry is done.
struct Grid {
  int nx, ny;
  bool periodic;
  int nreal, next;  // real nodes, real + halo
  int ext(int i, int j) const {  // 1-based grid point -> 0-based extended id
    if (!periodic) return (j - 1) * nx + (i - 1);
    if (i <= nx - 1 && j <= ny - 1) return (j - 1) * (nx - 1) + (i - 1);
    if (i == nx && j <= ny - 1) return nreal + (j - 1);
    if (i <= nx - 1 && j == ny) return nreal + (ny - 1) + (i - 1);
    return next - 1;
  }
  int real_of(int x) const {
    if (x < nreal) return x;
    int h = x - nreal;  // 0-based halo id
    if (h < ny - 1) return h * (nx - 1);         // right halo j=h+1 -> (1, j)
    if (h < (ny - 1) + (nx - 1)) return h - (ny - 1);  // top halo i -> (i, 1)
    return 0;                                     // corner -> (1, 1)
  }
};

}  // namespace

int analytic_nodes(int nx, int ny, bool periodic) {
  return periodic ? (nx - 1) * (ny - 1) : nx * ny;
}

int MeshHost::edge_levels(int e) const {
  int a = nlev_elem[edge_tri[2 * e]] - 1;
  int b = edge_tri[2 * e + 1] >= 0 ? nlev_elem[edge_tri[2 * e + 1]] - 1 : 0;
  return std::max(a, b);
}
int MeshHost::edge_shared_levels(int e) const {
  int a = nlev_elem[edge_tri[2 * e]] - 1;
  int b = edge_tri[2 * e + 1] >= 0 ? nlev_elem[edge_tri[2 * e + 1]] - 1 : 0;
  return std::min(a, b);
}
long long MeshHost::wet_cells() const {
  long long c = 0;
  for (int n = 0; n < nod2D; n++) c += nlev_node[n] - 1;
  return c;
}

MeshHost build_analytic_mesh(int nx, int ny, int nl, double Lx, double Ly, double max_depth,
                             bool periodic, bool full_rings, const int *node_K, bool left_oriented) {
  if (nx < 2 || ny < 2 || nl < 3) throw std::invalid_argument("analytic mesh needs nx, ny >= 2 and nl >= 3");
  if (periodic && (nx < 4 || ny < 4)) throw std::invalid_argument("periodic analytic mesh needs nx, ny >= 4");
  MeshHost m;
  m.nl = nl;
  m.periodic = periodic;
  m.full_rings = full_rings;
  m.Lx = Lx;
  m.Ly = Ly;
  m.max_depth = max_depth;
  Grid g{nx, ny, periodic, 0, 0};
  g.nreal = analytic_nodes(nx, ny, periodic);
  g.next = periodic ? g.nreal + (nx - 1) + (ny - 1) + 1 : g.nreal;
  const int N = g.nreal, NX = g.next;
  const int T = 2 * (nx - 1) * (ny - 1);
  m.nod2D = N;
  m.elem2D = T;

  // coordinates of every extended node
  const double dx = Lx / (double)(nx - 1), dy = Ly / (double)(ny - 1);
  std::vector<double> xc(NX), yc(NX);
  const int imax = periodic ? nx - 1 : nx, jmax = periodic ? ny - 1 : ny;
  for (int j = 1; j <= jmax; j++)
    for (int i = 1; i <= imax; i++) {
      int n = g.ext(i, j);
      xc[n] = (double)(i - 1) * dx / kREarth;
      yc[n] = (double)(j - 1) * dy / kREarth;
    }
  if (periodic) {
    for (int j = 1; j <= ny - 1; j++) { xc[g.ext(nx, j)] = Lx / kREarth; yc[g.ext(nx, j)] = (double)(j - 1) * dy / kREarth; }
    for (int i = 1; i <= nx - 1; i++) { xc[g.ext(i, ny)] = (double)(i - 1) * dx / kREarth; yc[g.ext(i, ny)] = Ly / kREarth; }
    xc[NX - 1] = Lx / kREarth;
    yc[NX - 1] = Ly / kREarth;
  }

  // elements over extended ids, clockwise, then the orientation check of
  // lib/oce_mesh.F90:1565-1615
  std::vector<int> en(3 * T);
  for (int j = 1, e = 0; j <= ny - 1; j++)
    for (int i = 1; i <= nx - 1; i++) {
      int n1 = g.ext(i, j), n2 = g.ext(i + 1, j), n3 = g.ext(i + 1, j + 1), n4 = g.ext(i, j + 1);
      en[3 * e + 0] = n1; en[3 * e + 1] = n3; en[3 * e + 2] = n2; e++;
      en[3 * e + 0] = n1; en[3 * e + 1] = n4; en[3 * e + 2] = n3; e++;
    }
  for (int e = 0; e < T; e++) {
    int *el = &en[3 * e];
    double b1 = xc[el[1]] - xc[el[0]], b2 = yc[el[1]] - yc[el[0]];
    double c1 = xc[el[2]] - xc[el[0]], c2 = yc[el[2]] - yc[el[0]];
    trim_cyclic(b1);
    trim_cyclic(c1);
    if (b1 * c2 - b2 * c1 > 0.0) std::swap(el[1], el[2]);
  }

  // edges over extended ids with their two elements
  std::vector<int> ednx, etri;
  auto quad = [&](int i, int j) { return (j - 1) * (nx - 1) + (i - 1); };  // 0-based quad
  auto lower = [&](int i, int j) { return 2 * quad(i, j); };
  auto upper = [&](int i, int j) { return 2 * quad(i, j) + 1; };
  auto push = [&](int a, int b, int t1, int t2) {
    ednx.push_back(a); ednx.push_back(b); etri.push_back(t1); etri.push_back(t2);
  };
  // horizontal and vertical edges, optionally reversed (see left_oriented)
  auto ab = [&](int a, int b, int &x, int &y) {
    x = left_oriented ? b : a;
    y = left_oriented ? a : b;
  };
  if (periodic) {
    int x, y;
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        ab(g.ext(i, j), g.ext(i + 1, j), x, y);
        push(x, y, j >= 2 ? upper(i, j - 1) : upper(i, ny - 1), lower(i, j));
      }
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) {
        ab(g.ext(i, j), g.ext(i, j + 1), x, y);
        push(x, y, upper(i, j), i >= 2 ? lower(i - 1, j) : lower(nx - 1, j));
      }
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) push(g.ext(i, j), g.ext(i + 1, j + 1), upper(i, j), lower(i, j));
  } else {
    std::vector<int> rn, rt;
    auto rpush = [&](int a, int b, int t1, int t2) {
      if (t1 < 0 && t2 >= 0) { t1 = t2; t2 = -1; }  // valid element first
      rn.push_back(a); rn.push_back(b); rt.push_back(t1); rt.push_back(t2);
    };
    int x, y;
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx - 1; i++) {
        ab(g.ext(i, j), g.ext(i + 1, j), x, y);
        rpush(x, y, j >= 2 ? upper(i, j - 1) : -1, j <= ny - 1 ? lower(i, j) : -1);
      }
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx; i++) {
        ab(g.ext(i, j), g.ext(i, j + 1), x, y);
        rpush(x, y, i <= nx - 1 ? upper(i, j) : -1, i >= 2 ? lower(i - 1, j) : -1);
      }
    for (int j = 1; j <= ny - 1; j++)
      for (int i = 1; i <= nx - 1; i++) rpush(g.ext(i, j), g.ext(i + 1, j + 1), upper(i, j), lower(i, j));
    // internal edges first, boundary edges after, each in generation order
    for (int pass = 0; pass < 2; pass++)
      for (size_t e = 0; e < rt.size() / 2; e++) {
        bool bnd = rt[2 * e + 1] < 0;
        if ((int)bnd != pass) continue;
        push(rn[2 * e], rn[2 * e + 1], rt[2 * e], rt[2 * e + 1]);
      }
  }
  const int E = (int)etri.size() / 2;
  m.edge2D = E;

  // levels
  m.nlev_elem.assign(T, nl);
  m.nlev_node.assign(N, nl);
  if (node_K) {
    for (int e = 0; e < T; e++) {
      int k = nl;
      for (int q = 0; q < 3; q++) k = std::min(k, node_K[g.real_of(en[3 * e + q])]);
      m.nlev_elem[e] = k;
    }
    std::fill(m.nlev_node.begin(), m.nlev_node.end(), 0);
    for (int e = 0; e < T; e++)
      for (int q = 0; q < 3; q++) {
        int r = g.real_of(en[3 * e + q]);
        m.nlev_node[r] = std::max(m.nlev_node[r], m.nlev_elem[e]);
      }
  }
  auto node_levels_ext = [&](int x) { return m.nlev_node[g.real_of(x)]; };

  // element rings over extended ids (ascending element ids)
  std::vector<int> xr_ptr(NX + 1, 0), xr(3 * T);
  for (int e = 0; e < T; e++)
    for (int q = 0; q < 3; q++) xr_ptr[en[3 * e + q] + 1]++;
  std::partial_sum(xr_ptr.begin(), xr_ptr.end(), xr_ptr.begin());
  {
    std::vector<int> fill(xr_ptr.begin(), xr_ptr.end() - 1);
    for (int e = 0; e < T; e++)
      for (int q = 0; q < 3; q++) xr[fill[en[3 * e + q]]++] = e;
  }

  // areas: triangle areas, per-level scalar-cell areas over the extended
  // rings, scaled to m^2 (lib/oce_mesh.F90:2088-2204)
  m.elem_area.resize(T);
  for (int e = 0; e < T; e++) {
    const int *el = &en[3 * e];
    double a1 = xc[el[1]] - xc[el[0]], a2 = yc[el[1]] - yc[el[0]];
    double b1 = xc[el[2]] - xc[el[0]], b2 = yc[el[2]] - yc[el[0]];
    trim_cyclic(a1);
    trim_cyclic(b1);
    a1 = a1 * 1.0;
    b1 = b1 * 1.0;
    m.elem_area[e] = 0.5 * std::fabs(a1 * b2 - b1 * a2);
  }
  std::vector<double> xarea((size_t)nl * NX, 0.0), xvol((size_t)nl * NX, 0.0);
  for (int n = 0; n < NX; n++) {
    for (int p = xr_ptr[n]; p < xr_ptr[n + 1]; p++) {
      int e = xr[p];
      for (int k = 1; k <= m.nlev_elem[e] - 1; k++) xarea[(size_t)n * nl + k - 1] = xarea[(size_t)n * nl + k - 1] + m.elem_area[e] / 3.0;
    }
    for (int k = 1; k <= node_levels_ext(n) - 1; k++) xvol[(size_t)n * nl + k - 1] = xarea[(size_t)n * nl + k - 1];
  }
  for (int e = 0; e < T; e++) m.elem_area[e] = m.elem_area[e] * kREarth * kREarth;
  for (size_t i = 0; i < xarea.size(); i++) {
    xarea[i] = xarea[i] * kREarth * kREarth;
    xvol[i] = xvol[i] * kREarth * kREarth;
  }

  // geometry over extended coordinates (lib/oce_mesh.F90:2402-2534)
  m.elem_cos.assign(T, 1.0);  // cartesian
  std::vector<double> cx(T), cy(T);
  for (int e = 0; e < T; e++) {
    const int *el = &en[3 * e];
    double ax[3] = {xc[el[0]], xc[el[1]], xc[el[2]]};
    double amin = std::min(std::min(ax[0], ax[1]), ax[2]);
    for (int q = 0; q < 3; q++) {
      if (ax[q] - amin >= kCyclicLength / 2.0) ax[q] = ax[q] - kCyclicLength;
      if (ax[q] - amin < -kCyclicLength / 2.0) ax[q] = ax[q] + kCyclicLength;
    }
    cx[e] = ((ax[0] + ax[1]) + ax[2]) / 3.0;
    cy[e] = ((yc[el[0]] + yc[el[1]]) + yc[el[2]]) / 3.0;
  }
  m.edge_dxdy.resize(2 * E);
  m.edge_cross.resize(4 * E);
  for (int e = 0; e < E; e++) {
    int a = ednx[2 * e], b = ednx[2 * e + 1];
    double d1 = xc[b] - xc[a], d2 = yc[b] - yc[a];
    trim_cyclic(d1);
    m.edge_dxdy[2 * e] = d1;
    m.edge_dxdy[2 * e + 1] = d2;
    double a1 = xc[a], b1 = xc[b];
    if (a1 - b1 > kCyclicLength / 2.0) a1 = a1 - kCyclicLength;
    if (a1 - b1 < -kCyclicLength / 2.0) b1 = b1 - kCyclicLength;
    double mx = 0.5 * (a1 + b1), my = 0.5 * (yc[a] + yc[b]);
    for (int s = 0; s < 2; s++) {
      int t = etri[2 * e + s];
      if (t < 0) { m.edge_cross[4 * e + 2 * s] = 0.0; m.edge_cross[4 * e + 2 * s + 1] = 0.0; continue; }
      double q1 = cx[t] - mx, q2 = cy[t] - my;
      trim_cyclic(q1);
      q1 = q1 * m.elem_cos[t];
      q1 = q1 * kREarth;
      q2 = q2 * kREarth;
      m.edge_cross[4 * e + 2 * s] = q1;
      m.edge_cross[4 * e + 2 * s + 1] = q2;
    }
  }
  m.grad_sca.resize(6 * T);
  for (int e = 0; e < T; e++) {
    const int *el = &en[3 * e];
    double dX31 = xc[el[2]] - xc[el[0]];
    trim_cyclic(dX31);
    dX31 = m.elem_cos[e] * dX31;
    double dX21 = xc[el[1]] - xc[el[0]];
    trim_cyclic(dX21);
    dX21 = m.elem_cos[e] * dX21;
    double dY31 = yc[el[2]] - yc[el[0]], dY21 = yc[el[1]] - yc[el[0]];
    double f = -(0.5 * kREarth / m.elem_area[e]);
    double *gs = &m.grad_sca[6 * e];
    gs[0] = (-dY31 + dY21) * f;
    gs[1] = dY31 * f;
    gs[2] = -(dY21 * f);
    gs[3] = (dX31 - dX21) * f;
    gs[4] = -(dX31 * f);
    gs[5] = dX21 * f;
  }

  // periodic post-remap (lib/analytic_mesh.F90:756-819)
  if (periodic) {
    const double hx = 0.5 * Lx, hy = 0.5 * Ly;
    for (int e = 0; e < E; e++)
      for (int s = 0; s < 2; s++) {
        double &vx = m.edge_cross[4 * e + 2 * s], &vy = m.edge_cross[4 * e + 2 * s + 1];
        if (std::fabs(vx) > hx) vx = vx - std::copysign(Lx, vx);
        if (std::fabs(vy) > hy) vy = vy - std::copysign(Ly, vy);
      }
    for (int x = N; x < NX; x++) {
      int r = g.real_of(x);
      for (int k = 0; k < nl - 1; k++) {
        xarea[(size_t)r * nl + k] = xarea[(size_t)r * nl + k] + xarea[(size_t)x * nl + k];
        xvol[(size_t)r * nl + k] = xvol[(size_t)r * nl + k] + xvol[(size_t)x * nl + k];
      }
    }
  }
  m.area.assign(xarea.begin(), xarea.begin() + (size_t)nl * N);
  m.areasvol.assign(xvol.begin(), xvol.begin() + (size_t)nl * N);

  m.coord.resize(2 * N);
  for (int n = 0; n < N; n++) { m.coord[2 * n] = xc[n]; m.coord[2 * n + 1] = yc[n]; }
  m.elem_nodes.resize(3 * T);
  for (int i = 0; i < 3 * T; i++) m.elem_nodes[i] = g.real_of(en[i]);
  m.edge_nodes.resize(2 * E);
  for (int i = 0; i < 2 * E; i++) m.edge_nodes[i] = g.real_of(ednx[i]);
  m.edge_tri = etri;

  // rings of the real nodes: the pre-remap lists, or rebuilt after the remap
  m.ring_ptr.assign(N + 1, 0);
  if (!periodic || !full_rings) {
    for (int n = 0; n < N; n++) m.ring_ptr[n + 1] = m.ring_ptr[n] + (xr_ptr[n + 1] - xr_ptr[n]);
    m.ring_elem.assign(xr.begin(), xr.begin() + xr_ptr[N]);
  } else {
    for (int e = 0; e < T; e++)
      for (int q = 0; q < 3; q++) m.ring_ptr[m.elem_nodes[3 * e + q] + 1]++;
    std::partial_sum(m.ring_ptr.begin(), m.ring_ptr.end(), m.ring_ptr.begin());
    m.ring_elem.resize(m.ring_ptr[N]);
    std::vector<int> fill(m.ring_ptr.begin(), m.ring_ptr.end() - 1);
    for (int e = 0; e < T; e++)
      for (int q = 0; q < 3; q++) m.ring_elem[fill[m.elem_nodes[3 * e + q]]++] = e;
  }

  // vertical grid and ALE thicknesses (lib/analytic_mesh.F90:361-369,
  // src/fesom_analytic.F90:206-244)
  m.zbar.resize(nl);
  m.Z.resize(nl - 1);
  for (int k = 1; k <= nl; k++) m.zbar[k - 1] = -((double)(k - 1) * max_depth / (double)(nl - 1));
  for (int k = 1; k <= nl - 1; k++) m.Z[k - 1] = 0.5 * (m.zbar[k - 1] + m.zbar[k]);
  m.hnode.resize((size_t)(nl - 1) * N);
  m.helem.resize((size_t)(nl - 1) * T);
  for (int n = 0; n < N; n++)
    for (int k = 0; k < nl - 1; k++) m.hnode[(size_t)n * (nl - 1) + k] = m.zbar[k] - m.zbar[k + 1];
  for (int e = 0; e < T; e++)
    for (int k = 0; k < nl - 1; k++) m.helem[(size_t)e * (nl - 1) + k] = m.zbar[k] - m.zbar[k + 1];
  m.hnode_new = m.hnode;

  m.finalize_tables();
  return m;
}

void MeshHost::finalize_tables() { finalize_tables(true); }

void MeshHost::finalize_tables(bool muscl_tables) {
  const int N = nod2D, E = edge2D;
  // nlevels_nod2D_min over the rings (lib/oce_mesh.F90:1522-1560)
  nlev_node_min.assign(N, 0);
  for (int n = 0; n < N; n++) {
    int mn = 1 << 30;
    for (int p = ring_ptr[n]; p < ring_ptr[n + 1]; p++) mn = std::min(mn, nlev_elem[ring_elem[p]]);
    nlev_node_min[n] = mn;
  }
  // MUSCL "a" per edge (lib/oce_adv_tra_hor.F90:333,346)
  edge_a.resize(E);
  for (int e = 0; e < E; e++) {
    double a = kREarth * elem_cos[edge_tri[2 * e]];
    if (edge_tri[2 * e + 1] >= 0) a = 0.5 * (a + kREarth * elem_cos[edge_tri[2 * e + 1]]);
    edge_a[e] = a;
  }
  if (muscl_tables) build_muscl_tables();
  // node -> incident edges, ascending edge id
  node_edge_ptr.assign(N + 1, 0);
  for (int e = 0; e < E; e++) { node_edge_ptr[edge_nodes[2 * e] + 1]++; node_edge_ptr[edge_nodes[2 * e + 1] + 1]++; }
  std::partial_sum(node_edge_ptr.begin(), node_edge_ptr.end(), node_edge_ptr.begin());
  node_edge.resize(node_edge_ptr[N]);
  std::vector<int> fill(node_edge_ptr.begin(), node_edge_ptr.end() - 1);
  for (int e = 0; e < E; e++) {
    node_edge[fill[edge_nodes[2 * e]]++] = (e << 1);
    node_edge[fill[edge_nodes[2 * e + 1]]++] = (e << 1) | 1;
  }
}

void MeshHost::build_muscl_tables() {
  const int E = edge2D;
  // up/down-wind triangles (lib/oce_muscl_adv.F90:245-338) with a
  // minimum-image wrap on periodic meshes; the last matching ring element wins
  up_dn_tri.assign(2 * E, -1);
  const double Px = Lx / kREarth, Py = Ly / kREarth;
  for (int e = 0; e < E; e++) {
    int a = edge_nodes[2 * e], b = edge_nodes[2 * e + 1];
    for (int side = 0; side < 2; side++) {
      int node = side == 0 ? a : b;
      double x0 = coord[2 * b] - coord[2 * a], x1 = coord[2 * b + 1] - coord[2 * a + 1];
      trim_cyclic(x0, cyclic_length);
      if (periodic) { trim_period(x0, Px); trim_period(x1, Py); }
      if (side == 0) { x0 = -x0; x1 = -x1; }
      for (int p = ring_ptr[node]; p < ring_ptr[node + 1]; p++) {
        int t = ring_elem[p];
        const int *el = &elem_nodes[3 * t];
        int i0 = el[0] == node ? 0 : (el[1] == node ? 1 : 2);
        int i1 = i0 == 0 ? 1 : 0;
        int i2 = i0 == 2 ? 1 : 2;
        double b0 = coord[2 * el[i1]] - coord[2 * el[i0]], b1 = coord[2 * el[i1] + 1] - coord[2 * el[i0] + 1];
        double c0 = coord[2 * el[i2]] - coord[2 * el[i0]], c1 = coord[2 * el[i2] + 1] - coord[2 * el[i0] + 1];
        trim_cyclic(b0, cyclic_length);
        trim_cyclic(c0, cyclic_length);
        if (periodic) { trim_period(b0, Px); trim_period(b1, Py); trim_period(c0, Px); trim_period(c1, Py); }
        double cr = c0 * c0 + c1 * c1;
        double bx = (b0 * c0 + b1 * c1) / cr;
        double by = (-b0 * c1 + b1 * c0) / cr;
        double xx = (x0 * c0 + x1 * c1) / cr;
        double xy = (-x0 * c1 + x1 * c0) / cr;
        double ab = std::atan2(by, bx), ax = std::atan2(xy, xx);
        if ((ab > 0.0 && ax > 0.0 && ax < ab) || (ab < 0.0 && ax < 0.0 && ax > ab) || (ab == ax) || (ax == 0.0))
          up_dn_tri[2 * e + side] = t;
      }
    }
  }
  build_nboundary_lay();
}

void MeshHost::build_nboundary_lay() {
  const int N = nod2D, E = edge2D;
  // nboundary_lay (lib/oce_muscl_adv.F90:96-161)
  nboundary_lay.assign(N, nl - 1);
  for (int e = 0; e < E; e++) {
    int n1 = edge_nodes[2 * e], n2 = edge_nodes[2 * e + 1];
    int t1 = edge_tri[2 * e], t2 = edge_tri[2 * e + 1];
    if (t1 < 0 || t2 < 0) {
      nboundary_lay[n1] = 0;
      nboundary_lay[n2] = 0;
    } else {
      int mn = std::min(nlev_elem[t1], nlev_elem[t2]) - 1;
      nboundary_lay[n1] = std::min(nboundary_lay[n1], mn);
      nboundary_lay[n2] = std::min(nboundary_lay[n2], mn);
    }
  }
}

std::string MeshHost::validate() const {
  std::ostringstream err;
  const int N = nod2D, T = elem2D, E = edge2D;
  if (nl < 3) err << "nl < 3; ";
  for (int i = 0; i < 3 * T; i++)
    if (elem_nodes[i] < 0 || elem_nodes[i] >= N) { err << "elem node out of range; "; break; }
  for (int i = 0; i < 2 * E; i++)
    if (edge_nodes[i] < 0 || edge_nodes[i] >= N) { err << "edge node out of range; "; break; }
  for (int e = 0; e < E; e++)
    if (edge_tri[2 * e] < 0 || edge_tri[2 * e] >= T || edge_tri[2 * e + 1] >= T) { err << "edge_tri out of range; "; break; }
  for (int e = 0; e < T; e++)
    if (nlev_elem[e] < 3 || nlev_elem[e] > nl) { err << "element nlevels outside [3, nl]; "; break; }
  for (int n = 0; n < N; n++)
    if (nlev_node[n] < 3 || nlev_node[n] > nl) { err << "node nlevels outside [3, nl]; "; break; }
  for (int e = 0; e < T; e++)
    for (int q = 0; q < 3; q++)
      if (nlev_elem[e] > nlev_node[elem_nodes[3 * e + q]]) { err << "element deeper than one of its nodes; "; e = T; break; }
  return err.str();
}

}  // namespace fesom
