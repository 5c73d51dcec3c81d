// C ABI of libfesom_tracer.so (declarations and reference citations in
// include/fesom_tracer.h).  One global instance, like the module state of the
// reference's lib/tracer_c_interface.F90.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fesom_tracer.h"
#include "batch.hpp"
#include "dd.hpp"
#include "engine.hpp"
#include "output.hpp"
#include "partition.hpp"
#include "restart.hpp"
#include "tile.hpp"

using namespace fesom;

namespace {

struct State {
  bool initialized = false;     // tracer_initialized of the reference
  bool ab_refresh = false;
  int nl = 0, nod2D = 0, edge2D = 0, elem2D = 0;  // tracer_set_mesh_dims
  int myDim = 0, eDim = 0;
  std::vector<int> nlevels_nod2D;
  std::vector<double> hnode_new;
  std::unique_ptr<MeshHost> mesh;  // connectivity (analytic or from arrays)
  std::unique_ptr<Engine> eng;
  int ntr = 0;
  std::vector<TracerScheme> schemes;
  // host copies kept until the engine exists
  std::vector<std::vector<double>> pend_values, pend_ab;
  std::vector<double> pend_uv, pend_w;  // uv in (2, nl-1, elem2D)
  bool pend_vel = false;
  Precision prec = Precision::FP64;
  int sround = 0;  // rounding of 16-bit stores (tracer_set_rounding)
  int step_path = 1;  // tracer_set_step_path (1: five kernels, the default)
  bool fma64 = false;  // precision mode 4: FP64 with FMA-contracted kernels
  bool nan_check = false;  // tracer_set_nan_check
  int patch_size = 0;  // tracer_set_patch_size (0: the default)
  int cells_per_block = 0;  // tracer_set_cells_per_block (0: the default)
  std::vector<int> ids;  // tracer IDs read from a restart
};
State g;
std::unique_ptr<Decomposition> g_dd;  // domain-decomposed runner (tracer_dd_*)
// global ids of the part installed by tracer_partition_install_part
std::vector<int> g_part_nodes, g_part_elems;

int fail(const std::string &msg) {
  set_last_error(msg);
  std::fprintf(stderr, "### error: %s\n", msg.c_str());
  return -1;
}

template <class F>
int guarded(F &&f) {
  try {
    set_last_error("");
    return f();
  } catch (const std::exception &e) {
    return fail(e.what());
  }
}

// Create the engine once a mesh with connectivity exists, then push any
// values that were set before.
void ensure_engine() {
  if (g.eng) return;
  if (!g.mesh) throw std::runtime_error("no mesh connectivity: use tracer_init_analytic or tracer_set_mesh_arrays");
  g.eng.reset(new Engine(*g.mesh, g.prec));
  g.eng->set_rounding(g.sround);
  g.eng->set_step_path(g.step_path);
  g.eng->set_fma64(g.fma64);
  if (g.patch_size > 0) g.eng->set_patch_size(g.patch_size);
  if (g.cells_per_block > 0) g.eng->set_cells_per_block(g.cells_per_block);
  if (g.ntr > 0) {
    g.eng->allocate_tracers(g.ntr);
    for (int i = 0; i < g.ntr; i++) {
      g.eng->set_scheme(i, g.schemes[i]);
      if (!g.pend_values[i].empty()) g.eng->set_values(i, g.pend_values[i].data(), true);
      if (!g.pend_ab[i].empty()) g.eng->set_values_ab(i, g.pend_ab[i].data());
    }
  }
  if (g.pend_vel) g.eng->set_velocity(g.pend_uv.data(), g.pend_w.data());
}

void install_mesh(MeshHost &&m) {
  g.eng.reset();
  g.mesh.reset(new MeshHost(std::move(m)));
  g.nl = g.mesh->nl;
  g.nod2D = g.mesh->nod2D;
  g.edge2D = g.mesh->edge2D;
  g.elem2D = g.mesh->elem2D;
  g.myDim = g.nod2D;
  g.eDim = 0;
  g.nlevels_nod2D = g.mesh->nlev_node;
  g.hnode_new = g.mesh->hnode_new;
  g.pend_vel = false;
}

TracerScheme parse_scheme(const char *hor, const char *ver, const char *lim, double ph, double pv) {
  TracerScheme s;
  std::string h = hor ? hor : "", v = ver ? ver : "", l = lim ? lim : "";
  auto trim = [](std::string &x) { while (!x.empty() && (x.back() == ' ' || x.back() == '\0')) x.pop_back(); };
  trim(h); trim(v); trim(l);
  if (h == "UPW1") s.hor = 0; else if (h == "MUSCL") s.hor = 1; else if (h == "MFCT") s.hor = 2;
  else throw std::invalid_argument("Unknown horizontal advection type " + h);
  if (v == "UPW1") s.ver = 0; else if (v == "PPM") s.ver = 1; else if (v == "QR4C") s.ver = 2; else if (v == "CDIFF") s.ver = 3;
  else throw std::invalid_argument("Unknown vertical advection type " + v);
  if (l == "NONE") s.lim = 0; else if (l == "FCT") s.lim = 1;
  else throw std::invalid_argument("Unknown limiter type " + l);
  s.ph = ph;
  s.pv = pv;
  return s;
}

int check_ready() {
  if (!g.initialized) return fail("tracer not initialized. Call tracer_init first.");
  return 0;
}

}  // namespace

namespace fesom {
// The engine of the C ABI's global instance (nullptr before the first step or
// tracer_init_for_advection) and its tracer count, for the allocation-free
// entry point in noalloc.cu.
Engine *capi_engine() { return g.eng.get(); }
int capi_num_tracers() { return g.ntr; }
bool capi_initialized() { return g.initialized; }
int capi_fail(const std::string &msg) { return fail(msg); }
std::string noalloc_prepare(int device);  // noalloc.cu
}  // namespace fesom

extern "C" {

int tracer_init_mpi(int) { return 0; }
int tracer_finalize_mpi(void) { return 0; }

// Installs a restart's mesh, and its tracers and flow when read.
static void install_restart(RestartData &&d) {
  install_mesh(std::move(d.mesh));
  g.ntr = (int)d.values.size();
  g.schemes = d.schemes;
  g.pend_values = std::move(d.values);
  g.pend_ab = std::move(d.values_ab);
  g.ids = d.ids;
  if (!d.uv.empty()) {
    g.pend_uv = std::move(d.uv);
    g.pend_w = std::move(d.w);
    g.pend_vel = true;
  }
  g.ab_refresh = false;  // valuesAB as stored, like the reference's drivers
  g.initialized = true;
}

int tracer_init(const char *restart_dir) {
  return guarded([&] {
    if (!restart_dir) return fail("tracer_init: null restart_dir");
    install_restart(read_restart(restart_dir, true, true));
    std::printf("Tracer initialized from: %s/np1\n", restart_dir);
    return 0;
  });
}

int tracer_finalize(const char *output_dir) {
  return guarded([&] {
    if (!g.initialized) return fail("tracer not initialized.");
    if (!output_dir) return fail("tracer_finalize: null output_dir");
    if (!g.mesh) return fail("tracer_finalize: no mesh connectivity to write");
    RestartData d;
    d.mesh = *g.mesh;
    const size_t LN = (size_t)(g.nl - 1) * g.nod2D;
    for (int t = 0; t < g.ntr; t++) {
      std::vector<double> v(LN), ab(LN);
      if (g.eng) {
        g.eng->get_values(t, v.data());
        if (g.ab_refresh) ab = v;
        else g.eng->get_values_ab(t, ab.data());
      } else {
        v = g.pend_values[t].empty() ? std::vector<double>(LN, 0.0) : g.pend_values[t];
        ab = (g.ab_refresh || g.pend_ab[t].empty()) ? v : g.pend_ab[t];
      }
      d.values.push_back(std::move(v));
      d.values_ab.push_back(std::move(ab));
      d.schemes.push_back(g.schemes[t]);
      d.ids.push_back(t < (int)g.ids.size() ? g.ids[t] : t + 1);
    }
    if (g.pend_vel) {
      d.uv = g.pend_uv;
      d.w = g.pend_w;
    }
    write_restart(output_dir, d);
    std::printf("Restart files written to: %s/np1\n", output_dir);
    g.initialized = false;  // as the reference's tracer_finalize
    return 0;
  });
}

int tracer_run_workflow(const char *restart_dir, int nsteps, double dt) {
  int status = tracer_init(restart_dir);
  if (status) return status;
  for (int step = 1; step <= nsteps; step++) {
    if ((status = tracer_advect_step(dt))) return status;
    double mn = 0, mx = 0, sm = 0;
    if ((status = tracer_get_stats(&mn, &mx, &sm))) return status;
    std::printf("Step %3d: min/max/sum = %15.6E%15.6E%15.6E\n", step, mn, mx, sm);
  }
  return tracer_finalize(restart_dir);
}

int tracer_load_mesh_partition(const char *restart_dir) {
  return guarded([&] {
    if (!restart_dir) return fail("tracer_load_mesh_partition: null restart_dir");
    RestartData d = read_restart(restart_dir, false, true);
    const int nl = d.mesh.nl, N = d.mesh.nod2D, E = d.mesh.edge2D;
    install_restart(std::move(d));
    std::printf("Loaded mesh partition from: %s/np1\n  Mesh: nl=%8d, nod2D=%8d, edge2D=%8d\n", restart_dir, nl, N, E);
    return 0;
  });
}
int tracer_load_mesh_from_files_opts(const char *mesh_path, int rotate, double alpha, double beta, double gamma,
                                     double angle_scale, double cyclic_length) {
  return guarded([&] {
    if (!mesh_path) return fail("tracer_load_mesh_from_files: null path");
    if (!(cyclic_length > 0.0)) return fail("tracer_load_mesh_from_files: cyclic_length must be positive");
    MeshFileOptions o;
    o.rotate = rotate != 0;
    o.alpha = alpha;
    o.beta = beta;
    o.gamma = gamma;
    o.angle_scale = angle_scale;
    o.cyclic_length = cyclic_length;
    install_mesh(load_mesh_files(mesh_path, o));
    g.initialized = true;
    return 0;
  });
}
int tracer_load_mesh_from_files(const char *mesh_path) {
  const MeshFileOptions o;
  return tracer_load_mesh_from_files_opts(mesh_path, o.rotate ? 1 : 0, o.alpha, o.beta, o.gamma, o.angle_scale,
                                          o.cyclic_length);
}

int tracer_cleanup(void) {
  return guarded([&] {
    g_dd.reset();
    g.eng.reset();
    g = State();
    return 0;
  });
}

int tracer_set_mesh_dims(int nl, int nod2D, int edge2D, int elem2D) {
  if (nl < 3 || nod2D < 1 || edge2D < 0 || elem2D < 0) return fail("invalid mesh dimensions");
  if (g.mesh && (g.mesh->nl != nl || g.mesh->nod2D != nod2D || g.mesh->edge2D != edge2D || g.mesh->elem2D != elem2D))
    return fail("mesh dimensions differ from the loaded mesh");
  g.nl = nl; g.nod2D = nod2D; g.edge2D = edge2D; g.elem2D = elem2D;
  return 0;
}

int tracer_set_levels(const int *nlevels, const int *ulevels, int nod2D) {
  if (!nlevels || !ulevels) return fail("null level array");
  if (nod2D != g.nod2D) return fail("tracer_set_levels: nod2D does not match the mesh dimensions");
  for (int i = 0; i < nod2D; i++) {
    if (ulevels[i] != 1) return fail("ulevels /= 1 (cavities) is not supported");
    if (nlevels[i] < 2 || nlevels[i] > g.nl) return fail("nlevels outside [2, nl]");
  }
  if (g.mesh)
    for (int i = 0; i < nod2D; i++)
      if (nlevels[i] != g.mesh->nlev_node[i]) return fail("nlevels differ from the loaded mesh");
  g.nlevels_nod2D.assign(nlevels, nlevels + nod2D);
  return 0;
}

int tracer_set_thickness(const double *hnode, int nl, int nod2D) {
  if (!hnode) return fail("null thickness array");
  if (nl != g.nl || nod2D != g.nod2D) return fail("tracer_set_thickness: dimensions do not match");
  g.hnode_new.assign(hnode, hnode + (size_t)(nl - 1) * nod2D);
  if (g.mesh) {
    g.mesh->hnode_new = g.hnode_new;
    g.eng.reset();  // geometry changed: rebuild the device copy lazily
  }
  return 0;
}

int tracer_set_partition(int myDim_nod2D, int eDim_nod2D) {
  if (eDim_nod2D != 0) return fail("halo nodes (eDim_nod2D > 0) are not supported on one GPU");
  if (myDim_nod2D != g.nod2D) return fail("myDim_nod2D does not match nod2D");
  g.myDim = myDim_nod2D;
  g.eDim = 0;
  return 0;
}

int tracer_allocate_tracers(int num_tracers, int nl, int nod2D, int AB_order) {
  return guarded([&] {
    if (num_tracers < 1) return fail("num_tracers < 1");
    if (nl != g.nl || nod2D != g.nod2D) return fail("tracer_allocate_tracers: dimensions do not match");
    if (AB_order < 1) return fail("AB_order < 1");
    g.ntr = num_tracers;
    g.ids.clear();
    g.schemes.assign(num_tracers, TracerScheme());
    g.pend_values.assign(num_tracers, std::vector<double>((size_t)(nl - 1) * nod2D, 0.0));
    g.pend_ab.assign(num_tracers, std::vector<double>());
    if (g.eng) {
      g.eng->allocate_tracers(num_tracers);
      for (int i = 0; i < num_tracers; i++) {
        g.eng->set_values(i, g.pend_values[i].data(), true);
        std::vector<double>().swap(g.pend_values[i]);
      }
    }
    return 0;
  });
}

int tracer_set_values(int tracer_id, const double *values, int nl, int nod2D) {
  return guarded([&] {
    if (tracer_id < 1 || tracer_id > g.ntr)
      return fail("invalid tracer_id " + std::to_string(tracer_id) + ", num_tracers=" + std::to_string(g.ntr));
    if (!values) return fail("null values");
    if (nl != g.nl || nod2D != g.nod2D) return fail("tracer_set_values: dimensions do not match");
    g.pend_ab[tracer_id - 1].clear();
    if (g.eng) {
      // the engine holds the values; host copies are only kept until it exists
      std::vector<double>().swap(g.pend_values[tracer_id - 1]);
      g.eng->set_values(tracer_id - 1, values, true);
    } else {
      g.pend_values[tracer_id - 1].assign(values, values + (size_t)(nl - 1) * nod2D);
    }
    return 0;
  });
}

int tracer_set_values_ab(int tracer_id, const double *values, int nl, int nod2D) {
  return guarded([&] {
    if (tracer_id < 1 || tracer_id > g.ntr) return fail("invalid tracer_id " + std::to_string(tracer_id));
    if (!values) return fail("null values");
    if (nl != g.nl || nod2D != g.nod2D) return fail("tracer_set_values_ab: dimensions do not match");
    if (g.eng) {
      std::vector<double>().swap(g.pend_ab[tracer_id - 1]);
      g.eng->set_values_ab(tracer_id - 1, values);
    } else {
      g.pend_ab[tracer_id - 1].assign(values, values + (size_t)(nl - 1) * nod2D);
    }
    return 0;
  });
}

int tracer_set_velocity_zero(int nl, int nod2D, int) {
  return guarded([&] {
    if (nl != g.nl || nod2D != g.nod2D) return fail("tracer_set_velocity_zero: dimensions do not match");
    g.pend_uv.assign((size_t)2 * (nl - 1) * g.elem2D, 0.0);
    g.pend_w.assign((size_t)nl * nod2D, 0.0);
    g.pend_vel = true;
    if (g.eng) g.eng->set_velocity_zero();
    return 0;
  });
}

int tracer_set_velocity_elem(const double *uv, const double *w, int nl, int nod2D, int elem2D) {
  return guarded([&] {
    if (!uv || !w) return fail("null velocity");
    if (nl != g.nl || nod2D != g.nod2D || elem2D != g.elem2D) return fail("tracer_set_velocity_elem: dimensions do not match");
    g.pend_uv.assign(uv, uv + (size_t)2 * (nl - 1) * elem2D);
    g.pend_w.assign(w, w + (size_t)nl * nod2D);
    g.pend_vel = true;
    if (g.eng) g.eng->set_velocity(uv, w);
    return 0;
  });
}

int tracer_set_velocity(const double *uv, const double *w, int nl, int nod2D, int nelem) {
  return guarded([&] {
    if (!uv || !w) return fail("null velocity");
    if (nelem != g.elem2D)
      return fail("tracer_set_velocity: uv must be (nl-1, elem2D, 2); got " + std::to_string(nelem) +
                  " columns for " + std::to_string(g.elem2D) + " elements");
    const int L = nl - 1;
    std::vector<double> t((size_t)2 * L * nelem);
    for (int c = 0; c < 2; c++)
      for (int e = 0; e < nelem; e++)
        for (int k = 0; k < L; k++) t[2 * ((size_t)e * L + k) + c] = uv[((size_t)c * nelem + e) * L + k];
    return tracer_set_velocity_elem(t.data(), w, nl, nod2D, nelem);
  });
}

int tracer_init_complete(void) {
  g.initialized = true;
  return 0;
}

int tracer_init_ale_arrays(void) {
  if (!g.initialized) return fail("tracer_init_ale_arrays called before initialization");
  if (!g.mesh) return fail("tracer_init_ale_arrays: no vertical grid (zbar) loaded");
  g.mesh->hnode_new = g.mesh->hnode;
  g.hnode_new = g.mesh->hnode_new;
  g.eng.reset();
  return 0;
}

int tracer_init_for_advection(void) {
  return guarded([&] {
    if (!g.initialized) return fail("tracer_init_for_advection called before mesh loaded");
    ensure_engine();
    // commit the allocation-free entry point's static work array now, before
    // a host that reserves the GPU's memory pool takes it
    const std::string err = noalloc_prepare(g.eng->device());
    if (!err.empty()) return fail("tracer_init_for_advection: static work array: " + err);
    return 0;
  });
}

int tracer_init_analytic(int nx, int ny, int nl, double Lx, double Ly, double max_depth, int periodic,
                         int options, const int *node_K) {
  return guarded([&] {
    if (node_K) {
      int nn = analytic_nodes(nx, ny, periodic != 0);
      for (int i = 0; i < nn; i++)
        if (node_K[i] < 3 || node_K[i] > nl) return fail("node_K outside [3, nl]");
    }
    install_mesh(build_analytic_mesh(nx, ny, nl, Lx, Ly, max_depth, periodic != 0, (options & 1) != 0, node_K,
                                     (options & 2) != 0));
    g.initialized = true;
    return 0;
  });
}

int tracer_analytic_nodes(int nx, int ny, int periodic) { return analytic_nodes(nx, ny, periodic != 0); }

int tracer_set_mesh_arrays(int nl, int nod2D, int elem2D, int edge2D, int max_ring, const int *elem2D_nodes,
                           const int *edges, const int *edge_tri, const int *nlevels, const int *nlevels_nod2D,
                           const int *ring_num, const int *ring, const double *elem_area, const double *area,
                           const double *areasvol, const double *edge_dxdy, const double *edge_cross_dxdy,
                           const double *gradient_sca, const double *elem_cos, const double *zbar,
                           const double *hnode, const double *hnode_new, const double *helem,
                           const double *coord_nod2D, double Lx, double Ly) {
  return guarded([&] {
    if (nl < 3 || nod2D < 1 || elem2D < 1 || edge2D < 1 || max_ring < 1) return fail("invalid mesh dimensions");
    const void *ptrs[] = {elem2D_nodes, edges, edge_tri, nlevels, nlevels_nod2D, ring_num, ring, elem_area, area,
                          areasvol, edge_dxdy, edge_cross_dxdy, gradient_sca, elem_cos, zbar, hnode, hnode_new,
                          helem, coord_nod2D};
    for (const void *p : ptrs)
      if (!p) return fail("null mesh array");
    MeshHost m;
    m.nl = nl; m.nod2D = nod2D; m.elem2D = elem2D; m.edge2D = edge2D;
    m.periodic = Lx > 0.0 && Ly > 0.0;
    m.Lx = Lx; m.Ly = Ly;
    m.coord.assign(coord_nod2D, coord_nod2D + 2 * (size_t)nod2D);
    m.elem_nodes.resize(3 * (size_t)elem2D);
    for (size_t i = 0; i < m.elem_nodes.size(); i++) m.elem_nodes[i] = elem2D_nodes[i] - 1;
    m.edge_nodes.resize(2 * (size_t)edge2D);
    m.edge_tri.resize(2 * (size_t)edge2D);
    for (size_t i = 0; i < m.edge_nodes.size(); i++) {
      m.edge_nodes[i] = edges[i] - 1;
      m.edge_tri[i] = edge_tri[i] > 0 ? edge_tri[i] - 1 : -1;
    }
    for (int e = 0; e < edge2D; e++)
      if (m.edge_tri[2 * e] < 0) return fail("edge_tri(1, e) must be a valid element");
    m.nlev_elem.assign(nlevels, nlevels + elem2D);
    m.nlev_node.assign(nlevels_nod2D, nlevels_nod2D + nod2D);
    m.ring_ptr.assign(nod2D + 1, 0);
    for (int n = 0; n < nod2D; n++) {
      if (ring_num[n] < 1 || ring_num[n] > max_ring) return fail("ring_num outside [1, max_ring]");
      m.ring_ptr[n + 1] = m.ring_ptr[n] + ring_num[n];
    }
    m.ring_elem.resize(m.ring_ptr[nod2D]);
    for (int n = 0; n < nod2D; n++)
      for (int j = 0; j < ring_num[n]; j++) m.ring_elem[m.ring_ptr[n] + j] = ring[(size_t)n * max_ring + j] - 1;
    m.elem_area.assign(elem_area, elem_area + elem2D);
    m.area.assign(area, area + (size_t)nl * nod2D);
    m.areasvol.assign(areasvol, areasvol + (size_t)nl * nod2D);
    m.edge_dxdy.assign(edge_dxdy, edge_dxdy + 2 * (size_t)edge2D);
    m.edge_cross.assign(edge_cross_dxdy, edge_cross_dxdy + 4 * (size_t)edge2D);
    m.grad_sca.assign(gradient_sca, gradient_sca + 6 * (size_t)elem2D);
    m.elem_cos.assign(elem_cos, elem_cos + elem2D);
    m.zbar.assign(zbar, zbar + nl);
    m.Z.resize(nl - 1);
    for (int k = 0; k < nl - 1; k++) m.Z[k] = 0.5 * (m.zbar[k] + m.zbar[k + 1]);
    m.hnode.assign(hnode, hnode + (size_t)(nl - 1) * nod2D);
    m.hnode_new.assign(hnode_new, hnode_new + (size_t)(nl - 1) * nod2D);
    m.helem.assign(helem, helem + (size_t)(nl - 1) * elem2D);
    for (int i = 0; i < 3 * elem2D; i++)
      if (m.elem_nodes[i] < 0 || m.elem_nodes[i] >= nod2D) return fail("elem2D_nodes out of range");
    for (int i = 0; i < 2 * edge2D; i++)
      if (m.edge_nodes[i] < 0 || m.edge_nodes[i] >= nod2D || m.edge_tri[i] >= elem2D) return fail("edges / edge_tri out of range");
    for (int r : m.ring_elem)
      if (r < 0 || r >= elem2D) return fail("nod_in_elem2D out of range");
    m.finalize_tables();
    std::string bad = m.validate();
    if (!bad.empty()) return fail("mesh: " + bad);
    install_mesh(std::move(m));
    g.initialized = true;
    return 0;
  });
}

int tracer_set_scheme(int tracer_id, const char *hor, const char *ver, const char *lim, double ph, double pv) {
  return guarded([&] {
    if (tracer_id < 1 || tracer_id > g.ntr) return fail("invalid tracer_id " + std::to_string(tracer_id));
    g.schemes[tracer_id - 1] = parse_scheme(hor, ver, lim, ph, pv);
    if (g.eng) g.eng->set_scheme(tracer_id - 1, g.schemes[tracer_id - 1]);
    return 0;
  });
}

int tracer_set_precision(int mode) {
  if (mode < 0 || mode > 4)
    return fail("precision mode must be 0 (FP64), 1 (FP32), 2 (BF16 storage), 3 (FP16 storage) or 4 (FP64 with FMA)");
  const Precision p = mode == 4 ? Precision::FP64 : (Precision)mode;
  g.fma64 = mode == 4;
  if (g.eng && g.eng->precision() == p) g.eng->set_fma64(g.fma64);
  if (g.eng && g.eng->precision() != p) {
    // rebuild the device state in the new mode, keeping the tracer values
    std::vector<std::vector<double>> keep(g.ntr);
    for (int i = 0; i < g.ntr; i++) {
      keep[i].resize((size_t)(g.nl - 1) * g.nod2D);
      g.eng->get_values(i, keep[i].data());
    }
    g.eng.reset();
    g.pend_values = keep;
    for (auto &ab : g.pend_ab) ab.clear();
  }
  g.prec = p;
  return 0;
}

int tracer_host_register(void *ptr, long long bytes) {
  if (!ptr || bytes <= 0) return fail("tracer_host_register: null pointer or empty range");
  if (host_register(ptr, (size_t)bytes) != 0) return fail("tracer_host_register: cudaHostRegister failed");
  return 0;
}

int tracer_host_unregister(void *ptr) {
  if (host_unregister(ptr) != 0) return fail("tracer_host_unregister: range was not registered");
  return 0;
}

int tracer_set_rounding(int mode) {
  if (mode < 0 || mode > 1) return fail("rounding mode must be 0 (nearest) or 1 (stochastic)");
  g.sround = mode;
  if (g.eng) g.eng->set_rounding(mode);
  return 0;
}

int tracer_set_step_path(int path) {
  return guarded([&] {
    if (path < 0 || path > 1) return fail("step path must be 0 (fused where possible) or 1 (five kernels)");
    g.step_path = path;
    if (g.eng) g.eng->set_step_path(path);
    return 0;
  });
}

int tracer_tile_plan_check(int max_owned, double *out8) {
  return guarded([&] {
    if (!out8) return fail("null output");
    if (!g.mesh) return fail("no mesh");
    if (max_owned < 1) return fail("max_owned must be positive");
    const std::vector<int> slot = edge_slot_order(*g.mesh);
    const TilePlanHost P = build_tile_plan(*g.mesh, slot, max_owned);
    const std::string bad = check_tile_plan(*g.mesh, P, slot);
    if (!bad.empty()) return fail("tile plan: " + bad);
    int mn = 1 << 30;
    for (const TileCounts &c : P.cnt) mn = std::min(mn, c.n0);
    out8[0] = P.np; out8[1] = mn; out8[2] = P.max_n2; out8[3] = P.max_n3;
    out8[4] = P.max_e2; out8[5] = P.max_el; out8[6] = P.node_ratio; out8[7] = P.edge_ratio;
    return 0;
  });
}

int tracer_set_patch_size(int owned) {
  return guarded([&] {
    if (owned < 0) return fail("patch size must be >= 0 (0: the default)");
    g.patch_size = owned;
    if (g.eng) g.eng->set_patch_size(owned > 0 ? owned : kTileOwned);
    return 0;
  });
}

int tracer_set_cells_per_block(int cells) {
  return guarded([&] {
    if (cells != 0 && (cells < 32 || cells > 576)) return fail("cells per block must be 0 (the default) or in [32, 576]");
    g.cells_per_block = cells;
    if (g.eng) g.eng->set_cells_per_block(cells > 0 ? cells : Engine::kDefaultCellsPerBlock);
    return 0;
  });
}

int tracer_set_nan_check(int on) {
  g.nan_check = on != 0;
  return 0;
}

int tracer_step_status(long long *nonfinite) {
  return guarded([&] {
    if (!nonfinite) return fail("null output");
    *nonfinite = g.eng ? g.eng->nonfinite_values(true) : 0;
    return 0;
  });
}

int tracer_step_info(double *out4) {
  return guarded([&] {
    if (!out4) return fail("null output");
    if (check_ready()) return -1;
    ensure_engine();
    out4[0] = g.eng->step_path();
    out4[1] = (g.ntr > 0 && g.eng->num_tracers() > 0) ? (g.eng->fused(0) ? 1.0 : 0.0) : 0.0;
    out4[2] = g.eng->tile_count();
    out4[3] = g.eng->tile_node_ratio();
    return 0;
  });
}

int tracer_storage_offset(int tracer_id, double *off) {
  return guarded([&] {
    if (check_ready()) return -1;
    if (tracer_id < 1 || tracer_id > g.ntr) return fail("invalid tracer_id " + std::to_string(tracer_id));
    if (!off) return fail("null output");
    ensure_engine();
    *off = g.eng->storage_offset(tracer_id - 1);
    return 0;
  });
}

int tracer_volume_sum(int tracer_id, double *out2) {
  return guarded([&] {
    if (check_ready()) return -1;
    if (tracer_id < 1 || tracer_id > g.ntr) return fail("invalid tracer_id " + std::to_string(tracer_id));
    if (!out2) return fail("null output");
    ensure_engine();
    g.eng->volume_sum(tracer_id - 1, out2);
    return 0;
  });
}

int tracer_set_ab_refresh(int on) {
  g.ab_refresh = on != 0;
  return 0;
}

int tracer_advect_steps(int nsteps, double dt) {
  return guarded([&] {
    if (check_ready()) return -1;
    if (g.ntr < 1) return fail("no tracers allocated");
    if (!(dt > 0.0)) return fail("dt must be positive");
    ensure_engine();
    for (int s = 0; s < nsteps; s++) g.eng->step(dt, g.ab_refresh);
    g.eng->synchronize();
    if (g.nan_check) {
      const long long bad = g.eng->nonfinite_values(true);
      if (bad) return fail("tracer_advect_step: " + std::to_string(bad) + " non-finite new values");
    }
    return 0;
  });
}

int tracer_advect_step(double dt) { return tracer_advect_steps(1, dt); }

int tracer_advect_step_io(double dt, const double *const *values_in, double *const *values_out, int ntracers) {
  return guarded([&] {
    if (check_ready()) return -1;
    if (g.ntr < 1) return fail("no tracers allocated");
    if (ntracers != g.ntr) return fail("tracer_advect_step_io: ntracers must equal the allocated tracers");
    if (!(dt > 0.0)) return fail("dt must be positive");
    ensure_engine();
    if (g.eng->step_io(dt, g.ab_refresh, values_in, values_out)) return 0;
    // not page-locked (or 16-bit storage): the same operations one by one
    const size_t LN = (size_t)(g.nl - 1) * g.nod2D;
    (void)LN;
    for (int t = 0; t < g.ntr; t++)
      if (values_in && values_in[t]) g.eng->set_values(t, values_in[t], true);
    g.eng->step(dt, g.ab_refresh);
    for (int t = 0; t < g.ntr; t++)
      if (values_out && values_out[t]) g.eng->get_values(t, values_out[t]);
    return 0;
  });
}

int tracer_get_values_id(int tracer_id, double *values, int nz, int nn) {
  return guarded([&] {
    if (check_ready()) return -1;
    if (tracer_id < 1 || tracer_id > g.ntr) return fail("invalid tracer_id " + std::to_string(tracer_id));
    if (!values) return fail("null values");
    if (nz != g.nl - 1 || nn != g.nod2D) return fail("tracer_get_values: expected (" + std::to_string(g.nl - 1) + ", " + std::to_string(g.nod2D) + ")");
    if (g.eng) g.eng->get_values(tracer_id - 1, values);
    else if (g.pend_values[tracer_id - 1].empty()) std::memset(values, 0, sizeof(double) * (size_t)nz * nn);
    else std::memcpy(values, g.pend_values[tracer_id - 1].data(), sizeof(double) * (size_t)nz * nn);
    return 0;
  });
}

int tracer_get_values(double *values, int nz, int nn) { return tracer_get_values_id(1, values, nz, nn); }

int tracer_get_stats_id(int tracer_id, double *s4) {
  return guarded([&] {
    if (check_ready()) return -1;
    if (tracer_id < 1 || tracer_id > g.ntr) return fail("invalid tracer_id " + std::to_string(tracer_id));
    if (g.eng) {
      g.eng->stats(tracer_id - 1, s4);
    } else {
      const std::vector<double> &v = g.pend_values[tracer_id - 1];
      double mn = v.empty() ? 0.0 : v[0], mx = mn, sm = 0.0, nan = 0.0;
      for (double x : v) { mn = x < mn ? x : mn; mx = x > mx ? x : mx; sm += x; nan += (x != x); }
      s4[0] = mn; s4[1] = mx; s4[2] = sm; s4[3] = nan;
    }
    return 0;
  });
}

int tracer_get_stats(double *tmin, double *tmax, double *tsum) {
  if (!g.initialized) {
    if (tmin) *tmin = 0.0;
    if (tmax) *tmax = 0.0;
    if (tsum) *tsum = 0.0;
    return fail("tracer not initialized.");
  }
  double s4[4];
  int rc = tracer_get_stats_id(1, s4);
  if (rc) return rc;
  *tmin = s4[0]; *tmax = s4[1]; *tsum = s4[2];
  return 0;
}

int tracer_get_size(int *nz, int *nn) {
  if (!g.initialized) {
    if (nz) *nz = 0;
    if (nn) *nn = 0;
    return fail("tracer not initialized.");
  }
  *nz = g.nl - 1;
  *nn = g.nod2D;
  return 0;
}

int tracer_analytic_fields(double *T, double *S, double *uv, double *w) {
  return guarded([&] {
    if (!g.mesh) return fail("no analytic mesh");
    std::vector<double> t, s, u, ww;
    analytic_driver_fields(*g.mesh, t, s, u, ww);
    if (T) std::memcpy(T, t.data(), t.size() * 8);
    if (S) std::memcpy(S, s.data(), s.size() * 8);
    if (uv) std::memcpy(uv, u.data(), u.size() * 8);
    if (w) std::memcpy(w, ww.data(), ww.size() * 8);
    return 0;
  });
}

int tracer_synth_bathymetry(int nnodes, int nl, uint64_t seed, int *K) {
  return guarded([&] {
    if (!K || nnodes < 0 || nl < 3) return fail("invalid bathymetry request");
    std::vector<int> k = synth_bathymetry(nnodes, nl, seed);
    std::memcpy(K, k.data(), sizeof(int) * (size_t)nnodes);
    return 0;
  });
}

int tracer_synth_bathymetry_smooth(int nx, int ny, int periodic, int nl, double corr_cells, uint64_t seed, int *K) {
  return guarded([&] {
    if (!K || nx < 2 || ny < 2 || nl < 3) return fail("invalid bathymetry request");
    std::vector<int> k = synth_bathymetry_smooth(nx, ny, periodic != 0, nl, corr_cells, seed);
    std::memcpy(K, k.data(), sizeof(int) * k.size());
    return 0;
  });
}

int tracer_synth_velocity(uint64_t seed, double umax, double mode1, double frac, double baro, double *uv,
                          double *w) {
  return guarded([&] {
    if (!g.mesh) return fail("no mesh");
    const MeshHost &m = *g.mesh;
    HugeArray<double> u(uv ? 0 : (size_t)2 * (m.nl - 1) * m.elem2D), ww(w ? 0 : (size_t)m.nl * m.nod2D);
    synth_velocity(m, seed, umax, mode1, frac, baro, uv ? uv : u.data(), w ? w : ww.data());
    return 0;
  });
}

int tracer_synth_tracer(uint64_t seed, int kind, double *values) {
  return guarded([&] {
    if (!g.mesh) return fail("no mesh");
    if (!values) return fail("values is NULL");
    synth_tracer(*g.mesh, seed, kind, values);
    return 0;
  });
}

int tracer_mesh_dims(int *d) {
  if (!g.mesh) return fail("no mesh");
  d[0] = g.mesh->nl; d[1] = g.mesh->nod2D; d[2] = g.mesh->elem2D; d[3] = g.mesh->edge2D;
  long long wc = g.mesh->wet_cells();
  d[4] = (int)(wc & 0x7fffffff);
  d[5] = (g.mesh->nl + 3) / 4 * 4;
  return 0;
}

static bool mesh_field(const char *name, const std::vector<int> **vi, const std::vector<double> **vd) {
  const MeshHost &m = *g.mesh;
  *vi = nullptr;
  *vd = nullptr;
  std::string s = name ? name : "";
  if (s == "coord") *vd = &m.coord;
  else if (s == "elem_area") *vd = &m.elem_area;
  else if (s == "area") *vd = &m.area;
  else if (s == "areasvol") *vd = &m.areasvol;
  else if (s == "edge_dxdy") *vd = &m.edge_dxdy;
  else if (s == "edge_cross_dxdy") *vd = &m.edge_cross;
  else if (s == "gradient_sca") *vd = &m.grad_sca;
  else if (s == "elem_cos") *vd = &m.elem_cos;
  else if (s == "hnode") *vd = &m.hnode;
  else if (s == "hnode_new") *vd = &m.hnode_new;
  else if (s == "helem") *vd = &m.helem;
  else if (s == "zbar") *vd = &m.zbar;
  else if (s == "elem2D_nodes") *vi = &m.elem_nodes;
  else if (s == "edges") *vi = &m.edge_nodes;
  else if (s == "edge_tri") *vi = &m.edge_tri;
  else if (s == "nlevels") *vi = &m.nlev_elem;
  else if (s == "nlevels_nod2D") *vi = &m.nlev_node;
  else if (s == "nlevels_nod2D_min") *vi = &m.nlev_node_min;
  else if (s == "edge_up_dn_tri") *vi = &m.up_dn_tri;
  else if (s == "nboundary_lay") *vi = &m.nboundary_lay;
  else if (s == "ring_num") *vi = &m.ring_ptr;
  else if (s == "ring_elem") *vi = &m.ring_elem;
  else if (s == "Z") *vd = &m.Z;
  else return false;
  return true;
}

long tracer_mesh_len(const char *name) {
  if (!g.mesh) return -1;
  const std::vector<int> *vi;
  const std::vector<double> *vd;
  if (!mesh_field(name, &vi, &vd)) return -1;
  if (std::string(name) == "ring_num") return g.mesh->nod2D;
  return vi ? (long)vi->size() : (long)vd->size();
}

int tracer_mesh_get_int(const char *name, int *out) {
  if (!g.mesh) return fail("no mesh");
  const std::vector<int> *vi;
  const std::vector<double> *vd;
  if (!mesh_field(name, &vi, &vd) || !vi) return fail(std::string("unknown integer mesh array ") + (name ? name : ""));
  const std::string s(name);
  if (s == "ring_num") {
    for (int n = 0; n < g.mesh->nod2D; n++) out[n] = g.mesh->ring_ptr[n + 1] - g.mesh->ring_ptr[n];
    return 0;
  }
  const bool index = (s == "elem2D_nodes" || s == "edges" || s == "edge_tri" || s == "edge_up_dn_tri" ||
                       s == "ring_elem");
  for (size_t i = 0; i < vi->size(); i++) out[i] = index ? ((*vi)[i] >= 0 ? (*vi)[i] + 1 : 0) : (*vi)[i];
  return 0;
}

int tracer_mesh_get_dbl(const char *name, double *out) {
  if (!g.mesh) return fail("no mesh");
  const std::vector<int> *vi;
  const std::vector<double> *vd;
  if (!mesh_field(name, &vi, &vd) || !vd) return fail(std::string("unknown real mesh array ") + (name ? name : ""));
  std::memcpy(out, vd->data(), vd->size() * sizeof(double));
  return 0;
}

int tracer_time_steps(int nsteps, double dt, float *ms) {
  return guarded([&] {
    if (check_ready()) return -1;
    if (g.ntr < 1) return fail("no tracers allocated");
    ensure_engine();
    cudaStream_t s = (cudaStream_t)g.eng->stream();
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    g.eng->synchronize();
    cudaEventRecord(a, s);
    for (int i = 0; i < nsteps; i++) g.eng->step(dt, g.ab_refresh);
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(cudaGetErrorString(e));
    return 0;
  });
}

int tracer_profile_steps(int nsteps, double dt, double *ms, const char **names, int nkinds, int *launches) {
  return guarded([&] {
    if (check_ready()) return -1;
    if (g.ntr < 1) return fail("no tracers allocated");
    ensure_engine();
    int nk = 0;
    const char *const *nm = Engine::kernel_kind_names(&nk);
    if (names)
      for (int k = 0; k < nkinds && k < nk; k++) names[k] = nm[k];
    int l = g.eng->profile_steps(nsteps, dt, g.ab_refresh, ms, nkinds);
    if (launches) *launches = l;
    return 0;
  });
}

int tracer_set_device(int device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n)
    return fail("invalid CUDA device " + std::to_string(device));
  if (g.eng) return fail("tracer_set_device must come before the engine is created");
  if (cudaSetDevice(device) != cudaSuccess) return fail("cudaSetDevice failed");
  return 0;
}

int tracer_launches_per_step(void) {
  if (!g.eng) return 0;
  return g.eng->launches_per_step();
}

long long tracer_device_bytes(void) { return g.eng ? (long long)g.eng->device_bytes() : 0; }

const char *tracer_last_error(void) { return last_error(); }

}  // extern "C"

// ---------------------------------------------------------------------------
// multi-member batch (batch.hpp)
// ---------------------------------------------------------------------------
namespace fesom {
int batch_selftest_barrier_timeout(long long limit);
}

namespace {
std::unique_ptr<Batch> g_batch;

Batch &batch() {
  if (!g_batch) throw std::runtime_error("no batch: call tracer_batch_create");
  return *g_batch;
}
Engine &batch_member(int m) { return batch().member(m); }
}  // namespace

int tracer_batch_create(void) {
  return guarded([&] {
    g_batch.reset();
    g_batch.reset(new Batch());
    return 0;
  });
}

int tracer_batch_destroy(void) {
  return guarded([&] {
    g_batch.reset();
    return 0;
  });
}

int tracer_batch_add_member(int nx, int ny, int nl, double Lx, double Ly, double max_depth, int periodic,
                            int options, const int *node_K, int ntracers) {
  return guarded([&] {
    if (node_K) {
      const int nn = analytic_nodes(nx, ny, periodic != 0);
      for (int i = 0; i < nn; i++)
        if (node_K[i] < 3 || node_K[i] > nl) return fail("node_K outside [3, nl]");
    }
    MeshHost m = build_analytic_mesh(nx, ny, nl, Lx, Ly, max_depth, periodic != 0, (options & 1) != 0, node_K,
                                     (options & 2) != 0);
    return batch().add_member(m, ntracers);
  });
}

int tracer_batch_member_dims(int member, int *dims4) {
  return guarded([&] {
    const MeshHost &m = batch_member(member).mesh();
    dims4[0] = m.nl; dims4[1] = m.nod2D; dims4[2] = m.elem2D; dims4[3] = m.edge2D;
    return 0;
  });
}

int tracer_batch_set_velocity(int member, const double *uv, const double *w) {
  return guarded([&] {
    if (!uv || !w) return fail("null velocity");
    batch_member(member).set_velocity(uv, w);
    return 0;
  });
}

int tracer_batch_set_values(int member, int tracer_id, const double *values) {
  return guarded([&] {
    if (!values) return fail("null values");
    Engine &e = batch_member(member);
    if (tracer_id < 1 || tracer_id > e.num_tracers()) return fail("invalid tracer_id " + std::to_string(tracer_id));
    e.set_values(tracer_id - 1, values, true);
    return 0;
  });
}

int tracer_batch_get_values(int member, int tracer_id, double *values) {
  return guarded([&] {
    if (!values) return fail("null values");
    Engine &e = batch_member(member);
    if (tracer_id < 1 || tracer_id > e.num_tracers()) return fail("invalid tracer_id " + std::to_string(tracer_id));
    e.get_values(tracer_id - 1, values);
    return 0;
  });
}

int tracer_batch_configure(const char *hor, const char *ver, const char *lim, double ph, double pv, const double *dt,
                           int refresh_ab) {
  return guarded([&] {
    if (!dt) return fail("null dt");
    Batch &b = batch();
    std::vector<double> d(dt, dt + b.num_members());
    b.configure(parse_scheme(hor, ver, lim, ph, pv), d, refresh_ab != 0);
    return 0;
  });
}

int tracer_batch_set_tile(int cells_per_block, int threads, int blocks_per_sm, int wave) {
  return guarded([&] {
    BatchTile t;
    t.cells_per_block = cells_per_block;
    t.threads = threads;
    t.blocks_per_sm = blocks_per_sm;
    t.wave = wave;
    batch().set_tile(t);
    return 0;
  });
}

int tracer_batch_get_tile(int *tile4) {
  return guarded([&] {
    const BatchTile t = batch().tile();
    tile4[0] = t.cells_per_block; tile4[1] = t.threads; tile4[2] = t.blocks_per_sm; tile4[3] = t.wave;
    return 0;
  });
}

int tracer_batch_set_path(int path) {
  return guarded([&] {
    batch().set_path(path);
    return 0;
  });
}

int tracer_batch_get_path(void) {
  return guarded([&] { return batch().path(); });
}

int tracer_batch_learn_set(const float *params, int on) {
  return guarded([&] {
    if (batch().num_members() == 0) return fail("the batch has no members");
    batch().set_learned(params, on != 0);
    return 0;
  });
}

int tracer_batch_steps(int nsteps, int use_graph) {
  return guarded([&] {
    if (nsteps < 0) return fail("nsteps < 0");
    batch().step(nsteps, use_graph != 0);
    return 0;
  });
}

int tracer_batch_time_steps(int nsteps, int use_graph, double *ms) {
  return guarded([&] {
    if (nsteps < 1 || !ms) return fail("nsteps < 1 or null output");
    *ms = batch().time_steps(nsteps, use_graph != 0);
    return 0;
  });
}

int tracer_batch_steps_separate(int nsteps, int use_graph) {
  return guarded([&] {
    if (nsteps < 0) return fail("nsteps < 0");
    batch().step_separate(nsteps, use_graph != 0);
    return 0;
  });
}

int tracer_batch_time_separate(int nsteps, int use_graph, double *ms) {
  return guarded([&] {
    if (nsteps < 1 || !ms) return fail("nsteps < 1 or null output");
    *ms = batch().time_separate(nsteps, use_graph != 0);
    return 0;
  });
}

int tracer_batch_autotune(int steps_per_candidate, char *log, int log_capacity) {
  return guarded([&] {
    const std::string s = batch().autotune(std::max(1, steps_per_candidate));
    if (log && log_capacity > 0) {
      const size_t n = std::min(s.size(), (size_t)log_capacity - 1);
      std::memcpy(log, s.data(), n);
      log[n] = 0;
    }
    return 0;
  });
}

int tracer_batch_info(long long *info4) {
  return guarded([&] {
    Batch &b = batch();
    info4[0] = b.num_members();
    info4[1] = b.wet_cells();
    info4[2] = b.work_bytes();
    info4[3] = b.graph_captured() ? 1 : 0;
    return 0;
  });
}

int tracer_selftest_barrier_timeout(long long limit) {
  return guarded([&] { return batch_selftest_barrier_timeout(limit); });
}

// ---------------------------------------------------------------------------
// learned antidiffusive flux (Engine::set_learned / learn_step)
// ---------------------------------------------------------------------------
int tracer_learn_set(const float *params, int on) {
  return guarded([&] {
    if (check_ready()) return -1;
    ensure_engine();
    g.eng->set_learned(params, on != 0);
    return 0;
  });
}

int tracer_learn_get(float *params) {
  return guarded([&] {
    if (!params) return fail("null output");
    if (!g.eng) return fail("no engine");
    g.eng->get_learned(params);
    return 0;
  });
}

int tracer_learn_grad(float *grad) {
  return guarded([&] {
    if (!grad) return fail("null output");
    if (!g.eng) return fail("no engine");
    g.eng->get_learned_grad(grad);
    return 0;
  });
}

int tracer_learn_step(const double *T_in, const double *T_target, double dt, double lr, int update, int fct,
                      double *loss) {
  return guarded([&] {
    if (!T_in || !T_target || !loss) return fail("null argument");
    if (check_ready()) return -1;
    ensure_engine();
    // fct: 0 no limiter; 1 limiter, gradient through its ratios; 2 limiter,
    // its factors held fixed in the gradient
    *loss = g.eng->learn_step(T_in, T_target, dt, lr, update != 0, fct != 0, fct != 2);
    return 0;
  });
}

// ---------------------------------------------------------------------------
// raw binary output for the reference's plotting scripts (output.hpp)
// ---------------------------------------------------------------------------
namespace {
ScalarOutput g_scalars;
}

int tracer_partition_read_dist(const char *dist_dir, int *node_part, int *nparts) {
  return guarded([&] {
    if (!g.mesh) return fail("tracer_partition_read_dist: no mesh");
    if (!dist_dir || !node_part || !nparts) return fail("tracer_partition_read_dist: null argument");
    int np = 0;
    std::vector<int> p = read_dist_partition(dist_dir, g.mesh->nod2D, &np);
    std::memcpy(node_part, p.data(), p.size() * sizeof(int));
    *nparts = np;
    return 0;
  });
}

static std::vector<int> part_map(const int *node_part, int nparts) {
  if (!g.mesh) throw std::runtime_error("no mesh");
  if (!node_part) throw std::invalid_argument("null node_part");
  std::vector<int> p(node_part, node_part + g.mesh->nod2D);
  for (int q : p)
    if (q < 0 || q >= nparts) throw std::invalid_argument("node part outside [0, nparts)");
  return p;
}

int tracer_partition_halo(const int *node_part, int nparts, int from, int to, int rings, int *out, int capacity) {
  return guarded([&] {
    const std::vector<int> v = halo_transfer(*g.mesh, part_map(node_part, nparts), from, to, rings);
    if ((int)v.size() > capacity) return fail("tracer_partition_halo: capacity too small");
    for (size_t i = 0; i < v.size(); i++) out[i] = v[i] + 1;
    return (int)v.size();
  });
}

int tracer_partition_part_dims(const int *node_part, int nparts, int part, int rings, int *dims4) {
  return guarded([&] {
    const MeshPart mp = build_mesh_part(*g.mesh, part_map(node_part, nparts), part, rings);
    dims4[0] = mp.owned;
    dims4[1] = mp.mesh.nod2D;
    dims4[2] = mp.mesh.elem2D;
    dims4[3] = mp.mesh.edge2D;
    return 0;
  });
}

int tracer_partition_install_part(const int *node_part, int nparts, int part, int rings, int *dims4) {
  return guarded([&] {
    MeshPart mp = build_mesh_part(*g.mesh, part_map(node_part, nparts), part, rings);
    dims4[0] = mp.owned;
    dims4[1] = mp.mesh.nod2D;
    dims4[2] = mp.mesh.elem2D;
    dims4[3] = mp.mesh.edge2D;
    g_part_nodes = mp.node_global;
    g_part_elems = mp.elem_global;
    install_mesh(std::move(mp.mesh));
    g.initialized = true;
    return 0;
  });
}

int tracer_partition_part_ids(int *nodes, int *elems) {
  if (g_part_nodes.empty()) return fail("tracer_partition_part_ids: no part installed");
  for (size_t i = 0; i < g_part_nodes.size(); i++) nodes[i] = g_part_nodes[i] + 1;
  for (size_t i = 0; i < g_part_elems.size(); i++) elems[i] = g_part_elems[i] + 1;
  return 0;
}

int tracer_dd_setup(const int *node_part, int nparts, const int *local_parts, int nlocal, int rings) {
  return guarded([&] {
    if (!local_parts || nlocal < 1) return fail("tracer_dd_setup: no local part");
    g_dd.reset();
    g_dd.reset(new Decomposition(*g.mesh, part_map(node_part, nparts), nparts,
                                 std::vector<int>(local_parts, local_parts + nlocal), rings, g.prec));
    return 0;
  });
}

static Decomposition &dd() {
  if (!g_dd) throw std::runtime_error("no domain decomposition: call tracer_dd_setup");
  return *g_dd;
}

int tracer_dd_destroy(void) {
  return guarded([&] {
    g_dd.reset();
    return 0;
  });
}

int tracer_dd_part_info(int i, int *info5) {
  return guarded([&] {
    const MeshPart &mp = dd().part(i);
    info5[0] = mp.part;
    info5[1] = mp.owned;
    info5[2] = mp.mesh.nod2D;
    info5[3] = mp.mesh.elem2D;
    info5[4] = mp.mesh.edge2D;
    return 0;
  });
}

int tracer_dd_allocate_tracers(int ntr) {
  return guarded([&] {
    if (ntr < 1) return fail("tracer_dd_allocate_tracers: ntr < 1");
    dd().allocate_tracers(ntr);
    return 0;
  });
}

int tracer_dd_set_scheme(int tracer_id, const char *hor, const char *ver, const char *lim, double ph, double pv) {
  return guarded([&] {
    dd().set_scheme(tracer_id - 1, parse_scheme(hor, ver, lim, ph, pv));
    return 0;
  });
}

int tracer_dd_set_velocity(const double *uv, const double *w) {
  return guarded([&] {
    if (!uv || !w) return fail("tracer_dd_set_velocity: null array");
    dd().set_velocity(uv, w);
    return 0;
  });
}

int tracer_dd_set_values(int tracer_id, const double *values) {
  return guarded([&] {
    if (!values) return fail("tracer_dd_set_values: null array");
    dd().set_values(tracer_id - 1, values);
    return 0;
  });
}

int tracer_dd_get_values(int tracer_id, double *values) {
  return guarded([&] {
    if (!values) return fail("tracer_dd_get_values: null array");
    dd().get_values(tracer_id - 1, values);
    return 0;
  });
}

int tracer_dd_steps(int nsteps, double dt, int refresh_ab, int exchange) {
  return guarded([&] {
    Decomposition &d = dd();
    for (int s = 0; s < nsteps; s++) {
      d.step(dt, refresh_ab != 0);
      if (exchange) d.exchange_local();
    }
    d.synchronize();
    return 0;
  });
}

int tracer_dd_transfer_nodes(int i, int peer, int send) {
  return guarded([&] { return dd().transfer_nodes(i, peer, send != 0); });
}

int tracer_dd_pack(int i, int tracer_id, int peer, double *dev_out) {
  return guarded([&] {
    dd().pack(i, tracer_id - 1, peer, dev_out);
    return 0;
  });
}

int tracer_dd_unpack(int i, int tracer_id, int peer, const double *dev_in) {
  return guarded([&] {
    dd().unpack(i, tracer_id - 1, peer, dev_in);
    return 0;
  });
}

int tracer_write_mesh(const char *output_dir) {
  return guarded([&] {
    if (!output_dir) return fail("null output directory");
    if (!g.mesh) return fail("no mesh");
    write_mesh_files(*g.mesh, output_dir);
    return 0;
  });
}

int tracer_scalar_output_open(const char *output_dir, int nsteps) {
  return guarded([&] {
    if (!output_dir) return fail("null output directory");
    if (check_ready()) return -1;
    if (g.ntr < 1) return fail("no tracers allocated");
    const int wp = g.prec == Precision::FP64 ? 8 : (g.prec == Precision::FP32 ? 4 : 2);
    g_scalars.open(output_dir, g.nod2D, g.nl - 1, nsteps, g.ntr, wp);
    return 0;
  });
}

int tracer_scalar_output_write(void) {
  return guarded([&] {
    if (!g_scalars.is_open()) return fail("scalar output is not open");
    std::vector<double> v((size_t)(g.nl - 1) * g.nod2D);
    for (int t = 0; t < g_scalars.tracers(); t++) {
      if (tracer_get_values_id(t + 1, v.data(), g.nl - 1, g.nod2D) != 0) return -1;
      g_scalars.write(t, v.data());
    }
    return 0;
  });
}

int tracer_scalar_output_close(void) {
  return guarded([&] {
    g_scalars.close();
    return 0;
  });
}

