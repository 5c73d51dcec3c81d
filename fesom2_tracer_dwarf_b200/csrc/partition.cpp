// Mesh parts with halos for the domain-decomposed step (see partition.hpp).
#include "partition.hpp"

#include <algorithm>
#include <cstdio>
#include <fstream>
#include <stdexcept>

namespace fesom {

namespace {

// node -> neighbouring nodes over the edges (CSR)
void node_neighbours(const MeshHost &g, std::vector<int> &ptr, std::vector<int> &nb) {
  const int N = g.nod2D, E = g.edge2D;
  ptr.assign(N + 1, 0);
  for (int e = 0; e < E; e++) {
    ptr[g.edge_nodes[2 * (size_t)e] + 1]++;
    ptr[g.edge_nodes[2 * (size_t)e + 1] + 1]++;
  }
  for (int n = 0; n < N; n++) ptr[n + 1] += ptr[n];
  nb.resize(ptr[N]);
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int e = 0; e < E; e++) {
    const int a = g.edge_nodes[2 * (size_t)e], b = g.edge_nodes[2 * (size_t)e + 1];
    nb[fill[a]++] = b;
    nb[fill[b]++] = a;
  }
}

void check_part_map(const MeshHost &g, const std::vector<int> &node_part, int part) {
  if ((int)node_part.size() != g.nod2D) throw std::invalid_argument("partition: one part per node expected");
  if (part < 0) throw std::invalid_argument("partition: negative part");
}

}  // namespace

std::vector<int> halo_nodes(const MeshHost &g, const std::vector<int> &node_part, int part, int rings) {
  check_part_map(g, node_part, part);
  std::vector<int> ptr, nb;
  node_neighbours(g, ptr, nb);
  const int N = g.nod2D;
  std::vector<char> seen(N, 0);
  std::vector<int> front, halo;
  for (int n = 0; n < N; n++)
    if (node_part[n] == part) {
      seen[n] = 1;
      front.push_back(n);
    }
  for (int r = 0; r < rings; r++) {
    std::vector<int> next;
    for (int n : front)
      for (int p = ptr[n]; p < ptr[n + 1]; p++)
        if (!seen[nb[p]]) {
          seen[nb[p]] = 1;
          next.push_back(nb[p]);
        }
    halo.insert(halo.end(), next.begin(), next.end());
    front.swap(next);
  }
  std::sort(halo.begin(), halo.end());
  return halo;
}

std::vector<int> halo_transfer(const MeshHost &g, const std::vector<int> &node_part, int from, int to, int rings) {
  std::vector<int> out;
  for (int n : halo_nodes(g, node_part, to, rings))
    if (node_part[n] == from) out.push_back(n);
  return out;
}

MeshPart build_mesh_part(const MeshHost &g, const std::vector<int> &node_part, int part, int rings) {
  MeshPart P;
  P.part = part;
  const int N = g.nod2D, T = g.elem2D, E = g.edge2D, nl = g.nl, L = nl - 1;
  for (int n = 0; n < N; n++)
    if (node_part[n] == part) P.node_global.push_back(n);
  P.owned = (int)P.node_global.size();
  if (P.owned == 0) throw std::invalid_argument("partition: part " + std::to_string(part) + " owns no node");
  const std::vector<int> halo = halo_nodes(g, node_part, part, rings);
  P.node_global.insert(P.node_global.end(), halo.begin(), halo.end());
  std::vector<int> nmap(N, -1), tmap(T, -1), emap(E, -1);
  for (int i = 0; i < (int)P.node_global.size(); i++) nmap[P.node_global[i]] = i;
  for (int t = 0; t < T; t++) {
    const int *en = &g.elem_nodes[3 * (size_t)t];
    if (nmap[en[0]] >= 0 && nmap[en[1]] >= 0 && nmap[en[2]] >= 0) {
      tmap[t] = (int)P.elem_global.size();
      P.elem_global.push_back(t);
    }
  }
  for (int e = 0; e < E; e++) {
    const int a = g.edge_nodes[2 * (size_t)e], b = g.edge_nodes[2 * (size_t)e + 1];
    if (nmap[a] >= 0 && nmap[b] >= 0 && tmap[g.edge_tri[2 * (size_t)e]] >= 0) {
      emap[e] = (int)P.edge_global.size();
      P.edge_global.push_back(e);
    }
  }
  const int n_loc = (int)P.node_global.size(), t_loc = (int)P.elem_global.size(), e_loc = (int)P.edge_global.size();

  MeshHost &m = P.mesh;
  m.nl = nl;
  m.nod2D = n_loc;
  m.elem2D = t_loc;
  m.edge2D = e_loc;
  m.periodic = g.periodic;
  m.full_rings = g.full_rings;
  m.Lx = g.Lx;
  m.Ly = g.Ly;
  m.max_depth = g.max_depth;
  m.cyclic_length = g.cyclic_length;
  m.zbar = g.zbar;
  m.Z = g.Z;

  m.coord.resize(2 * (size_t)n_loc);
  m.nlev_node.resize(n_loc);
  m.area.resize((size_t)nl * n_loc);
  m.areasvol.resize((size_t)nl * n_loc);
  m.hnode.resize((size_t)L * n_loc);
  m.hnode_new.resize((size_t)L * n_loc);
  for (int i = 0; i < n_loc; i++) {
    const int n = P.node_global[i];
    m.coord[2 * (size_t)i] = g.coord[2 * (size_t)n];
    m.coord[2 * (size_t)i + 1] = g.coord[2 * (size_t)n + 1];
    m.nlev_node[i] = g.nlev_node[n];
    std::copy_n(&g.area[(size_t)n * nl], nl, &m.area[(size_t)i * nl]);
    std::copy_n(&g.areasvol[(size_t)n * nl], nl, &m.areasvol[(size_t)i * nl]);
    std::copy_n(&g.hnode[(size_t)n * L], L, &m.hnode[(size_t)i * L]);
    std::copy_n(&g.hnode_new[(size_t)n * L], L, &m.hnode_new[(size_t)i * L]);
  }
  m.elem_nodes.resize(3 * (size_t)t_loc);
  m.nlev_elem.resize(t_loc);
  m.elem_area.resize(t_loc);
  m.elem_cos.resize(t_loc);
  m.grad_sca.resize(6 * (size_t)t_loc);
  m.helem.resize((size_t)L * t_loc);
  for (int i = 0; i < t_loc; i++) {
    const int t = P.elem_global[i];
    for (int q = 0; q < 3; q++) m.elem_nodes[3 * (size_t)i + q] = nmap[g.elem_nodes[3 * (size_t)t + q]];
    m.nlev_elem[i] = g.nlev_elem[t];
    m.elem_area[i] = g.elem_area[t];
    m.elem_cos[i] = g.elem_cos[t];
    std::copy_n(&g.grad_sca[6 * (size_t)t], 6, &m.grad_sca[6 * (size_t)i]);
    std::copy_n(&g.helem[(size_t)t * L], L, &m.helem[(size_t)i * L]);
  }
  m.edge_nodes.resize(2 * (size_t)e_loc);
  m.edge_tri.resize(2 * (size_t)e_loc);
  m.edge_dxdy.resize(2 * (size_t)e_loc);
  m.edge_cross.resize(4 * (size_t)e_loc);
  for (int i = 0; i < e_loc; i++) {
    const int e = P.edge_global[i];
    m.edge_nodes[2 * (size_t)i] = nmap[g.edge_nodes[2 * (size_t)e]];
    m.edge_nodes[2 * (size_t)i + 1] = nmap[g.edge_nodes[2 * (size_t)e + 1]];
    m.edge_tri[2 * (size_t)i] = tmap[g.edge_tri[2 * (size_t)e]];
    const int t2 = g.edge_tri[2 * (size_t)e + 1];
    m.edge_tri[2 * (size_t)i + 1] = t2 >= 0 ? tmap[t2] : -1;
    std::copy_n(&g.edge_dxdy[2 * (size_t)e], 2, &m.edge_dxdy[2 * (size_t)i]);
    std::copy_n(&g.edge_cross[4 * (size_t)e], 4, &m.edge_cross[4 * (size_t)i]);
    if (m.edge_tri[2 * (size_t)i + 1] < 0) {  // the cut-off element's segment carries no flux
      m.edge_cross[4 * (size_t)i + 2] = 0.0;
      m.edge_cross[4 * (size_t)i + 3] = 0.0;
    }
  }
  // element rings: the global lists (which may be the reference's incomplete
  // periodic ones) restricted to local elements, in their global order
  m.ring_ptr.assign(n_loc + 1, 0);
  for (int i = 0; i < n_loc; i++) {
    const int n = P.node_global[i];
    for (int p = g.ring_ptr[n]; p < g.ring_ptr[n + 1]; p++)
      if (tmap[g.ring_elem[p]] >= 0) m.ring_elem.push_back(tmap[g.ring_elem[p]]);
    m.ring_ptr[i + 1] = (int)m.ring_elem.size();
  }
  m.finalize_tables();  // node -> edge lists
  // derived tables as on the whole mesh (exact for every node and edge the
  // owned nodes read)
  for (int i = 0; i < n_loc; i++) {
    m.nlev_node_min[i] = g.nlev_node_min[P.node_global[i]];
    m.nboundary_lay[i] = g.nboundary_lay[P.node_global[i]];
  }
  for (int i = 0; i < e_loc; i++) {
    const int e = P.edge_global[i];
    m.edge_a[i] = g.edge_a[e];
    for (int s = 0; s < 2; s++) {
      const int t = g.up_dn_tri[2 * (size_t)e + s];
      m.up_dn_tri[2 * (size_t)i + s] = t >= 0 ? tmap[t] : -1;
    }
  }
  return P;
}

std::vector<int> partition_by_index(int nod2D, int parts) {
  if (parts < 1 || parts > nod2D) throw std::invalid_argument("partition: 1 <= parts <= nod2D expected");
  std::vector<int> p(nod2D);
  for (int n = 0; n < nod2D; n++) p[n] = (int)((long long)n * parts / nod2D);
  return p;
}

std::vector<int> read_dist_partition(const std::string &dist_dir, int nod2D, int *parts) {
  const std::string rpart = dist_dir + "/rpart.out";
  std::ifstream in(rpart);
  if (!in) throw std::runtime_error("partition: cannot open " + rpart);
  int np = 0;
  if (!(in >> np) || np < 1) throw std::runtime_error("partition: " + rpart + ": bad part count");
  std::vector<long> count(np);
  for (auto &c : count)
    if (!(in >> c)) throw std::runtime_error("partition: " + rpart + ": short count list");
  std::vector<int> p(nod2D, -1);
  for (int q = 0; q < np; q++) {
    char name[32];
    std::snprintf(name, sizeof name, "/my_list%05d.out", q);
    const std::string path = dist_dir + name;
    std::ifstream f(path);
    if (!f) throw std::runtime_error("partition: cannot open " + path);
    long rank = -1, my = -1, halo = -1;
    if (!(f >> rank >> my >> halo) || rank != q || my < 0 || halo < 0)
      throw std::runtime_error("partition: " + path + ": bad header");
    if (my != count[q]) throw std::runtime_error("partition: " + path + ": owned count disagrees with rpart.out");
    for (long i = 0; i < my; i++) {
      long n = 0;
      if (!(f >> n)) throw std::runtime_error("partition: " + path + ": short node list");
      if (n < 1 || n > nod2D) throw std::runtime_error("partition: " + path + ": node out of range");
      if (p[n - 1] >= 0) throw std::runtime_error("partition: " + path + ": node owned twice");
      p[n - 1] = q;
    }
  }
  for (int n = 0; n < nod2D; n++)
    if (p[n] < 0) throw std::runtime_error("partition: " + dist_dir + ": node " + std::to_string(n + 1) + " has no owner");
  *parts = np;
  return p;
}

}  // namespace fesom
