// Patch plan of the fused step kernel: recursive coordinate bisection of the
// nodes, three halo rings per patch, and the local tables the kernel stages
// in shared memory (tile.hpp).
#include "tile.hpp"

#include <algorithm>
#include <numeric>
#include <stdexcept>

namespace fesom {

namespace {

// Split ids[lo, hi) into nparts parts of (nearly) equal counts, each cut
// across the larger coordinate extent of its node set.
void bisect(const MeshHost &m, std::vector<int> &ids, int lo, int hi, int nparts,
            std::vector<std::pair<int, int>> &parts) {
  if (nparts <= 1 || hi - lo <= 1) {
    parts.push_back({lo, hi});
    return;
  }
  double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
  for (int i = lo; i < hi; i++) {
    const double x = m.coord[2 * ids[i]], y = m.coord[2 * ids[i] + 1];
    x0 = std::min(x0, x); x1 = std::max(x1, x);
    y0 = std::min(y0, y); y1 = std::max(y1, y);
  }
  const int ax = (x1 - x0 >= y1 - y0) ? 0 : 1;
  const int k1 = nparts / 2;
  const int mid = lo + (int)((long long)(hi - lo) * k1 / nparts);
  std::nth_element(ids.begin() + lo, ids.begin() + mid, ids.begin() + hi, [&](int a, int b) {
    const double ca = m.coord[2 * a + ax], cb = m.coord[2 * b + ax];
    return ca < cb || (ca == cb && a < b);
  });
  bisect(m, ids, lo, mid, k1, parts);
  bisect(m, ids, mid, hi, nparts - k1, parts);
}

struct Region {
  std::vector<int> nodes;  // O, R1, R2, R3
  int n0 = 0, n1 = 0, n2 = 0, n3 = 0;
};

// Owned nodes plus three rings, each ring ascending.  Two nodes are
// neighbours when an edge or an element joins them (the same on a whole
// mesh; on the local mesh of a domain-decomposition part an element may be
// kept while one of its edges is not).
Region grow(const MeshHost &m, const std::vector<int> &nel_ptr, const std::vector<int> &nel,
            std::vector<int> owned, std::vector<int> &mark, int stamp) {
  Region r;
  std::sort(owned.begin(), owned.end());
  r.nodes = owned;
  for (int n : owned) mark[n] = stamp;
  r.n0 = (int)owned.size();
  int begin = 0;
  std::vector<int> ring;
  for (int q = 1; q <= 3; q++) {
    ring.clear();
    const int end = (int)r.nodes.size();
    for (int i = begin; i < end; i++) {
      const int n = r.nodes[i];
      for (int p = m.node_edge_ptr[n]; p < m.node_edge_ptr[n + 1]; p++) {
        const int e = m.node_edge[p] >> 1;
        const int o = m.edge_nodes[2 * e] == n ? m.edge_nodes[2 * e + 1] : m.edge_nodes[2 * e];
        if (mark[o] != stamp) {
          mark[o] = stamp;
          ring.push_back(o);
        }
      }
      for (int p = nel_ptr[n]; p < nel_ptr[n + 1]; p++)
        for (int q = 0; q < 3; q++) {
          const int o = m.elem_nodes[3 * nel[p] + q];
          if (mark[o] != stamp) {
            mark[o] = stamp;
            ring.push_back(o);
          }
        }
    }
    std::sort(ring.begin(), ring.end());
    r.nodes.insert(r.nodes.end(), ring.begin(), ring.end());
    begin = end;
    if (q == 1) r.n1 = (int)r.nodes.size();
    if (q == 2) r.n2 = (int)r.nodes.size();
  }
  r.n3 = (int)r.nodes.size();
  return r;
}

}  // namespace

TilePlanHost build_tile_plan(const MeshHost &m, const std::vector<int> &edge_slot, int max_owned) {
  const int N = m.nod2D, E = m.edge2D, T = m.elem2D;
  if (m.nl > kTileMaxLevels) throw std::runtime_error("fused step: more than 255 levels");
  TilePlanHost P;
  std::vector<int> ids(N);
  std::iota(ids.begin(), ids.end(), 0);
  std::vector<std::pair<int, int>> parts;
  const int target = std::max(1, max_owned);
  bool flat = true;  // no coordinates (a mesh read from a restart record)
  for (int n = 1; n < N && flat; n++)
    flat = m.coord[2 * n] == m.coord[0] && m.coord[2 * n + 1] == m.coord[1];
  if (flat && N > 1) {
    // breadth-first parts: from the lowest unassigned node, collect target
    // nodes over the edge graph
    std::vector<char> used(N, 0);
    std::vector<int> order, queue;
    order.reserve(N);
    for (int s = 0; s < N; s++) {
      if (used[s]) continue;
      size_t head = 0;
      queue.assign(1, s);
      used[s] = 1;
      const int begin = (int)order.size();
      while (head < queue.size() && (int)order.size() - begin < target) {
        const int n = queue[head++];
        order.push_back(n);
        for (int p = m.node_edge_ptr[n]; p < m.node_edge_ptr[n + 1]; p++) {
          const int e = m.node_edge[p] >> 1;
          const int o = m.edge_nodes[2 * e] == n ? m.edge_nodes[2 * e + 1] : m.edge_nodes[2 * e];
          if (!used[o]) {
            used[o] = 1;
            queue.push_back(o);
          }
        }
      }
      for (size_t q = head; q < queue.size(); q++) used[queue[q]] = 0;  // not taken
      parts.push_back({begin, (int)order.size()});
    }
    ids = order;
  } else {
    bisect(m, ids, 0, N, (N + target - 1) / target, parts);
  }

  // which elements hold every node (the ring lists may be incomplete)
  std::vector<int> holds(N, 0);
  for (int e = 0; e < T; e++)
    for (int q = 0; q < 3; q++) holds[m.elem_nodes[3 * e + q]]++;

  std::vector<int> mark(N, -1), loc(N, -1), eloc(E, -1), tloc(T, -1);
  std::vector<int> node_elems_ptr(N + 1, 0), node_elems;  // elements holding each node
  for (int e = 0; e < T; e++)
    for (int q = 0; q < 3; q++) node_elems_ptr[m.elem_nodes[3 * e + q] + 1]++;
  for (int n = 0; n < N; n++) node_elems_ptr[n + 1] += node_elems_ptr[n];
  node_elems.resize(node_elems_ptr[N]);
  {
    std::vector<int> fill(node_elems_ptr.begin(), node_elems_ptr.end() - 1);
    for (int e = 0; e < T; e++)
      for (int q = 0; q < 3; q++) node_elems[fill[m.elem_nodes[3 * e + q]]++] = e;
  }

  int stamp = 0;
  long long owned_edges = 0, region_edges = 0;
  // a work list of owned sets; a set whose region does not fit is bisected
  std::vector<std::vector<int>> todo;
  for (auto &pr : parts) todo.emplace_back(ids.begin() + pr.first, ids.begin() + pr.second);
  while (!todo.empty()) {
    std::vector<int> owned = std::move(todo.back());
    todo.pop_back();
    Region r = grow(m, node_elems_ptr, node_elems, owned, mark, stamp++);
    // edges: E1 (an end in N1), then E2 \ E1 (an end in N2)
    std::vector<int> e1, e2;
    for (int i = 0; i < r.n2; i++) loc[r.nodes[i]] = i;
    for (int i = r.n2; i < r.n3; i++) loc[r.nodes[i]] = i;
    for (int i = 0; i < r.n2; i++) {
      const int n = r.nodes[i];
      for (int p = m.node_edge_ptr[n]; p < m.node_edge_ptr[n + 1]; p++) {
        const int e = m.node_edge[p] >> 1;
        if (eloc[e] == -2) continue;
        eloc[e] = -2;
        const int a = loc[m.edge_nodes[2 * e]], b = loc[m.edge_nodes[2 * e + 1]];
        if (a < r.n1 || b < r.n1) e1.push_back(e);
        else e2.push_back(e);
      }
    }
    std::sort(e1.begin(), e1.end());
    std::sort(e2.begin(), e2.end());
    const int ne1 = (int)e1.size();
    std::vector<int> edges = e1;
    edges.insert(edges.end(), e2.begin(), e2.end());
    // elements with a node in N2
    std::vector<int> els;
    for (int i = 0; i < r.n2; i++) {
      const int n = r.nodes[i];
      for (int p = node_elems_ptr[n]; p < node_elems_ptr[n + 1]; p++) {
        const int t = node_elems[p];
        if (tloc[t] == -2) continue;
        tloc[t] = -2;
        els.push_back(t);
      }
    }
    std::sort(els.begin(), els.end());
    const bool fits = r.n2 <= kTileThreads && r.n3 - r.n2 <= kTileThreads && (int)edges.size() <= kTileMaxEdges &&
                      (int)els.size() < 0xffff;
    if (!fits) {
      for (int n : r.nodes) loc[n] = -1;
      for (int e : edges) eloc[e] = -1;
      for (int t : els) tloc[t] = -1;
      if ((int)owned.size() <= 1) throw std::runtime_error("fused step: a node's three-ring region does not fit a block");
      std::vector<int> sub = owned;
      std::vector<std::pair<int, int>> halves;
      bisect(m, sub, 0, (int)sub.size(), 2, halves);
      for (auto &h : halves) todo.emplace_back(sub.begin() + h.first, sub.begin() + h.second);
      continue;
    }
    for (int i = 0; i < (int)edges.size(); i++) eloc[edges[i]] = i;
    for (int i = 0; i < (int)els.size(); i++) tloc[els[i]] = i;

    TileCounts c{};
    c.n0 = r.n0; c.n1 = r.n1; c.n2 = r.n2; c.n3 = r.n3;
    c.e1 = ne1; c.e2 = (int)edges.size(); c.nel = (int)els.size();
    c.node_off = (int)P.node_gid.size();
    c.inc_off = (int)P.inc.size();
    c.edge_off = (int)P.edge_slot.size();
    c.elem_off = (int)P.elem_gid.size();
    c.ring_off = (int)P.ring.size();
    int jmax = 0;
    for (int i = 0; i < r.n3; i++) {
      const int n = r.nodes[i];
      jmax = std::max(jmax, m.nlev_node[n] - 1);
      P.node_gid.push_back(n);
      const uint32_t full = (m.ring_ptr[n + 1] - m.ring_ptr[n]) == holds[n] ? 1u : 0u;
      P.node_info.push_back((uint32_t)m.nlev_node[n] | (uint32_t)m.nlev_node_min[n] << 8 |
                            (uint32_t)m.nboundary_lay[n] << 16 | full << 24);
    }
    c.jmax = jmax;
    // incidence and rings of N2 nodes (n2 + 1 pointers each from ptr_off)
    c.ptr_off = (int)P.inc_ptr.size();
    int ninc = 0, nring = 0;
    P.inc_ptr.push_back(0);
    P.ring_ptr.push_back(0);
    for (int i = 0; i < r.n2; i++) {
      const int n = r.nodes[i];
      for (int p = m.node_edge_ptr[n]; p < m.node_edge_ptr[n + 1]; p++) {
        const int code = m.node_edge[p], e = code >> 1, second = code & 1;
        const int o = m.edge_nodes[2 * e + (second ? 0 : 1)];
        const int le = eloc[e], lo = loc[o];
        if (le < 0 || lo < 0) throw std::logic_error("fused step plan: incidence outside the region");
        P.inc.push_back((uint32_t)le | (uint32_t)second << 11 | (uint32_t)lo << 12 |
                        (uint32_t)m.edge_levels(e) << 22);
        ninc++;
      }
      P.inc_ptr.push_back(ninc);
      for (int p = m.ring_ptr[n]; p < m.ring_ptr[n + 1]; p++) {
        const int t = tloc[m.ring_elem[p]];
        if (t < 0) throw std::logic_error("fused step plan: ring element outside the region");
        P.ring.push_back((uint16_t)t);
        nring++;
      }
      P.ring_ptr.push_back(nring);
    }
    for (int i = 0; i < (int)edges.size(); i++) {
      const int e = edges[i];
      const int a = loc[m.edge_nodes[2 * e]], b = loc[m.edge_nodes[2 * e + 1]];
      P.edge_slot.push_back(edge_slot[e]);
      P.edge_nn.push_back((uint32_t)a | (uint32_t)b << 10 | (uint32_t)m.edge_levels(e) << 20);
      uint32_t ud = 0xffffffffu;
      if (i < ne1) {
        const int up = m.up_dn_tri[2 * e], dn = m.up_dn_tri[2 * e + 1];
        const uint32_t lu = up >= 0 ? (uint32_t)tloc[up] : 0xffffu, ld = dn >= 0 ? (uint32_t)tloc[dn] : 0xffffu;
        if ((up >= 0 && tloc[up] < 0) || (dn >= 0 && tloc[dn] < 0))
          throw std::logic_error("fused step plan: up/down triangle outside the region");
        ud = lu | ld << 16;
      }
      P.edge_ud.push_back(ud);
    }
    for (int t : els) {
      P.elem_gid.push_back(t);
      uint32_t nn = 0;
      for (int q = 0; q < 3; q++) {
        const int l = loc[m.elem_nodes[3 * t + q]];
        if (l < 0) throw std::logic_error("fused step plan: element node outside the region");
        nn |= (uint32_t)l << (10 * q);
      }
      P.elem_nn.push_back(nn);
    }
    P.cnt.push_back(c);
    P.max_n1 = std::max(P.max_n1, c.n1);
    P.max_n2 = std::max(P.max_n2, c.n2);
    P.max_n3 = std::max(P.max_n3, c.n3);
    P.max_e1 = std::max(P.max_e1, c.e1);
    P.max_e2 = std::max(P.max_e2, c.e2);
    P.max_el = std::max(P.max_el, c.nel);
    P.max_inc = std::max(P.max_inc, ninc);
    for (int i = 0; i < r.n0; i++) owned_edges += m.node_edge_ptr[r.nodes[i] + 1] - m.node_edge_ptr[r.nodes[i]];
    region_edges += c.e1;
    for (int n : r.nodes) loc[n] = -1;
    for (int e : edges) eloc[e] = -1;
    for (int t : els) tloc[t] = -1;
  }
  P.np = (int)P.cnt.size();
  long long region_nodes = 0;
  for (auto &c : P.cnt) region_nodes += c.n2;
  P.node_ratio = N ? (double)region_nodes / N : 0.0;
  P.edge_ratio = E ? (double)region_edges / E : 0.0;
  (void)owned_edges;
  return P;
}

std::string check_tile_plan(const MeshHost &m, const TilePlanHost &P, const std::vector<int> &edge_slot) {
  const int N = m.nod2D;
  std::vector<int> owner(N, -1);
  std::vector<int> slot_edge(edge_slot.size());
  for (size_t e = 0; e < edge_slot.size(); e++) slot_edge[edge_slot[e]] = (int)e;
  auto err = [](int p, const std::string &what) { return "patch " + std::to_string(p) + ": " + what; };
  for (int p = 0; p < P.np; p++) {
    const TileCounts &c = P.cnt[p];
    if (!(0 < c.n0 && c.n0 <= c.n1 && c.n1 <= c.n2 && c.n2 <= c.n3)) return err(p, "node counts");
    if (c.n2 > kTileThreads || c.n3 - c.n2 > kTileThreads) return err(p, "region larger than the block");
    const int *g = &P.node_gid[c.node_off];
    std::vector<int> ring(N, -1);  // ring index of each region node
    for (int i = 0; i < c.n3; i++) {
      const int q = i < c.n0 ? 0 : i < c.n1 ? 1 : i < c.n2 ? 2 : 3;
      if (ring[g[i]] != -1) return err(p, "node listed twice");
      ring[g[i]] = q;
      if (q == 0) {
        if (owner[g[i]] != -1) return err(p, "node owned twice");
        owner[g[i]] = p;
      }
    }
    // ring q + 1 is exactly the set of new neighbours of rings <= q
    for (int i = 0; i < c.n3; i++) {
      const int n = g[i], q = ring[n];
      for (int e = m.node_edge_ptr[n]; e < m.node_edge_ptr[n + 1]; e++) {
        const int ed = m.node_edge[e] >> 1;
        const int o = m.edge_nodes[2 * ed] == n ? m.edge_nodes[2 * ed + 1] : m.edge_nodes[2 * ed];
        if (q < 3 && (ring[o] == -1 || ring[o] > q + 1)) return err(p, "ring structure");
      }
    }
    // incidence lists of N2 nodes: every incident edge, ascending, consistent
    int pos = 0;
    for (int i = 0; i < c.n2; i++) {
      const int n = g[i];
      const int b = P.inc_ptr[c.ptr_off + i], e = P.inc_ptr[c.ptr_off + i + 1];
      if (b != pos || e - b != m.node_edge_ptr[n + 1] - m.node_edge_ptr[n]) return err(p, "incidence count");
      for (int k = b; k < e; k++) {
        const uint32_t q = P.inc[c.inc_off + k];
        const int le = q & 2047u, second = (q >> 11) & 1u, oth = (q >> 12) & 1023u, lev = (int)(q >> 22);
        const int code = m.node_edge[m.node_edge_ptr[n] + (k - b)], ed = code >> 1;
        if (le >= c.e2 || slot_edge[P.edge_slot[c.edge_off + le]] != ed) return err(p, "incidence edge");
        if (second != (code & 1) || lev != m.edge_levels(ed)) return err(p, "incidence flags");
        if (oth >= c.n3 || g[oth] != m.edge_nodes[2 * ed + (second ? 0 : 1)]) return err(p, "incidence other node");
        if (i < c.n1 && le >= c.e1) return err(p, "an N1 node's edge outside E1");
      }
      pos = e;
    }
    for (int le = 0; le < c.e2; le++) {
      const int ed = slot_edge[P.edge_slot[c.edge_off + le]];
      const uint32_t nn = P.edge_nn[c.edge_off + le];
      const int a = nn & 1023u, bb = (nn >> 10) & 1023u;
      if (g[a] != m.edge_nodes[2 * ed] || g[bb] != m.edge_nodes[2 * ed + 1]) return err(p, "edge nodes");
      if ((le < c.e1) != (a < c.n1 || bb < c.n1)) return err(p, "E1 membership");
      if (a >= c.n2 && bb >= c.n2) return err(p, "edge without an end in N2");
      if (le < c.e1) {
        const uint32_t ud = P.edge_ud[c.edge_off + le];
        const int up = ud & 0xffffu, dn = ud >> 16;
        const int gu = m.up_dn_tri[2 * ed], gd = m.up_dn_tri[2 * ed + 1];
        if ((gu < 0) != (up == 0xffff) || (gd < 0) != (dn == 0xffff)) return err(p, "up/down presence");
        if (gu >= 0 && P.elem_gid[c.elem_off + up] != gu) return err(p, "up triangle");
        if (gd >= 0 && P.elem_gid[c.elem_off + dn] != gd) return err(p, "down triangle");
      }
    }
    for (int i = 0; i < c.n2; i++) {
      const int n = g[i];
      const int b = P.ring_ptr[c.ptr_off + i], e = P.ring_ptr[c.ptr_off + i + 1];
      if (e - b != m.ring_ptr[n + 1] - m.ring_ptr[n]) return err(p, "ring count");
      for (int k = b; k < e; k++)
        if (P.elem_gid[c.elem_off + P.ring[c.ring_off + k]] != m.ring_elem[m.ring_ptr[n] + (k - b)])
          return err(p, "ring element");
    }
    for (int t = 0; t < c.nel; t++) {
      const int gt = P.elem_gid[c.elem_off + t];
      const uint32_t nn = P.elem_nn[c.elem_off + t];
      for (int q = 0; q < 3; q++)
        if (g[(nn >> (10 * q)) & 1023u] != m.elem_nodes[3 * gt + q]) return err(p, "element nodes");
    }
    int jmax = 0;
    for (int i = 0; i < c.n3; i++) jmax = std::max(jmax, m.nlev_node[g[i]] - 1);
    if (jmax != c.jmax) return err(p, "deepest layer");
  }
  for (int n = 0; n < N; n++)
    if (owner[n] < 0) return "node " + std::to_string(n) + " owned by no patch";
  return "";
}

}  // namespace fesom
