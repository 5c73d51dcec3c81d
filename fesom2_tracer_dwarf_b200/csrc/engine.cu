// Engine: device memory, layout conversion, schedules and kernel dispatch.
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>

#include "advect_kernels.cuh"
#include "engine.hpp"

namespace fesom {

namespace {
thread_local std::string g_err;
}
const char *last_error() { return g_err.c_str(); }
void set_last_error(const std::string &s) { g_err = s; }

#define CK(x)                                                                                 \
  do {                                                                                        \
    cudaError_t e_ = (x);                                                                     \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

constexpr int kBlock = 256;
constexpr int kCellsPerBlock = 1024;
constexpr int kMaxItemsPerBlock = 1024;

void build_sched(const std::vector<int> &counts, std::vector<int> &off, std::vector<int> &blk, int &max_items) {
  const int n = (int)counts.size();
  off.assign(n + 1, 0);
  for (int i = 0; i < n; i++) off[i + 1] = off[i] + counts[i];
  blk.clear();
  blk.push_back(0);
  max_items = 1;
  int start = 0;
  for (int i = 0; i < n; i++) {
    const int items = i + 1 - start, cells = off[i + 1] - off[start];
    if (cells >= kCellsPerBlock || items >= kMaxItemsPerBlock || i == n - 1) {
      blk.push_back(i + 1);
      max_items = std::max(max_items, items);
      start = i + 1;
    }
  }
  if (n == 0) blk.push_back(0);
}

}  // namespace

struct EngineImpl {
  MeshHost mesh;
  int S = 0;
  cudaStream_t stream = nullptr;
  std::vector<void *> allocs;
  size_t bytes = 0;
  DMeshT<double> dm{};
  double *vel = nullptr, *W = nullptr;
  struct Tracer {
    double *T = nullptr, *Tout = nullptr, *TAB = nullptr;
    TracerScheme sch;
  };
  std::vector<Tracer> tr;
  double *flo = nullptr, *adfh = nullptr, *adfv = nullptr, *lo = nullptr;
  double *tmax = nullptr, *tmin = nullptr, *rp = nullptr, *rm = nullptr;
  // launch profiling: when prof is set, every launch is bracketed by events
  struct ProfRec { int kind; cudaEvent_t a, b; };
  std::vector<ProfRec> *prof = nullptr;
  void mark_begin(int kind) {
    if (!prof) return;
    ProfRec r{kind, nullptr, nullptr};
    CK(cudaEventCreate(&r.a));
    CK(cudaEventCreate(&r.b));
    CK(cudaEventRecord(r.a, stream));
    prof->push_back(r);
  }
  void mark_end() {
    if (!prof) return;
    CK(cudaEventRecord(prof->back().b, stream));
  }

  template <typename T>
  T *dalloc(size_t n) {
    void *p = nullptr;
    if (n == 0) n = 1;
    CK(cudaMalloc(&p, n * sizeof(T)));
    CK(cudaMemsetAsync(p, 0, n * sizeof(T), stream));
    allocs.push_back(p);
    bytes += n * sizeof(T);
    return (T *)p;
  }
  void dfree(void *p) {
    if (!p) return;
    auto it = std::find(allocs.begin(), allocs.end(), p);
    if (it != allocs.end()) allocs.erase(it);
    cudaFree(p);
  }
  template <typename T>
  T *upload(const std::vector<T> &h) {
    T *d = dalloc<T>(h.size());
    if (!h.empty()) CK(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
  }
  // (ld, ncol) column-major host array -> device columns of stride S
  double *upload_cols(const double *h, int ld, int ncol, int nvalid) {
    std::vector<double> st((size_t)ncol * S, 0.0);
    for (int c = 0; c < ncol; c++) std::memcpy(&st[(size_t)c * S], h + (size_t)c * ld, sizeof(double) * nvalid);
    return upload(st);
  }
  void copy_cols_to(double *d, const double *h, int ld, int ncol) {
    std::vector<double> st((size_t)ncol * S, 0.0);
    for (int c = 0; c < ncol; c++) std::memcpy(&st[(size_t)c * S], h + (size_t)c * ld, sizeof(double) * ld);
    CK(cudaMemcpy(d, st.data(), st.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
};

Engine::Engine(const MeshHost &mesh) : p_(new EngineImpl) {
  EngineImpl &P = *p_;
  P.mesh = mesh;
  const std::string bad = mesh.validate();
  if (!bad.empty()) throw std::invalid_argument("mesh: " + bad);
  const MeshHost &M = P.mesh;
  const int N = M.nod2D, T = M.elem2D, E = M.edge2D, nl = M.nl, L = nl - 1;
  P.S = (nl + 3) / 4 * 4;
  CK(cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking));
  DMeshT<double> &d = P.dm;
  d.N = N; d.T = T; d.E = E; d.nl = nl; d.S = P.S;

  std::vector<int2> en(E), et(E), el(E), ud(E);
  for (int e = 0; e < E; e++) {
    en[e] = make_int2(M.edge_nodes[2 * e], M.edge_nodes[2 * e + 1]);
    et[e] = make_int2(M.edge_tri[2 * e], M.edge_tri[2 * e + 1]);
    el[e] = make_int2(M.edge_shared_levels(e), M.edge_levels(e));
    ud[e] = make_int2(M.up_dn_tri[2 * e], M.up_dn_tri[2 * e + 1]);
  }
  d.edge_nodes = P.upload(en);
  d.edge_tri = P.upload(et);
  d.edge_lev = P.upload(el);
  d.up_dn = P.upload(ud);
  d.edge_cross = P.upload(M.edge_cross);
  d.edge_dxdy = P.upload(M.edge_dxdy);
  d.edge_a = P.upload(M.edge_a);
  d.nlev_elem = P.upload(M.nlev_elem);
  d.nlev_node = P.upload(M.nlev_node);
  d.nlev_node_min = P.upload(M.nlev_node_min);
  d.nbl = P.upload(M.nboundary_lay);
  d.elem_nodes = P.upload(M.elem_nodes);
  d.grad_sca = P.upload(M.grad_sca);
  d.elem_area = P.upload(M.elem_area);
  d.ring_ptr = P.upload(M.ring_ptr);
  d.ring_elem = P.upload(M.ring_elem);
  d.ne_ptr = P.upload(M.node_edge_ptr);
  d.ne = P.upload(M.node_edge);
  d.zbar = P.upload(M.zbar);
  d.Z = P.upload(M.Z);
  d.area = P.upload_cols(M.area.data(), nl, N, nl);
  d.areasvol = P.upload_cols(M.areasvol.data(), nl, N, nl);
  d.hnode = P.upload_cols(M.hnode.data(), L, N, L);
  d.hnode_new = P.upload_cols(M.hnode_new.data(), L, N, L);
  d.helem = P.upload_cols(M.helem.data(), L, T, L);

  std::vector<int> cnt(N), off, blk;
  for (int n = 0; n < N; n++) cnt[n] = M.nlev_node[n] - 1;
  build_sched(cnt, off, blk, d.node_sched.max_items);
  d.node_sched.cell_off = P.upload(off);
  d.node_sched.blk = P.upload(blk);
  d.node_sched.nblk = (int)blk.size() - 1;
  cnt.assign(E, 0);
  for (int e = 0; e < E; e++) cnt[e] = M.edge_levels(e);
  build_sched(cnt, off, blk, d.edge_sched.max_items);
  d.edge_sched.cell_off = P.upload(off);
  d.edge_sched.blk = P.upload(blk);
  d.edge_sched.nblk = (int)blk.size() - 1;

  P.vel = P.dalloc<double>((size_t)2 * T * P.S);
  P.W = P.dalloc<double>((size_t)N * P.S);
  P.flo = P.dalloc<double>((size_t)E * P.S);
  P.adfh = P.dalloc<double>((size_t)E * P.S);
  P.adfv = P.dalloc<double>((size_t)N * P.S);
  P.lo = P.dalloc<double>((size_t)N * P.S);
  P.tmax = P.dalloc<double>((size_t)N * P.S);
  P.tmin = P.dalloc<double>((size_t)N * P.S);
  P.rp = P.dalloc<double>((size_t)N * P.S);
  P.rm = P.dalloc<double>((size_t)N * P.S);
  CK(cudaStreamSynchronize(P.stream));
}

Engine::~Engine() {
  if (!p_) return;
  cudaStreamSynchronize(p_->stream);
  for (void *a : p_->allocs) cudaFree(a);
  cudaStreamDestroy(p_->stream);
  delete p_;
}

const MeshHost &Engine::mesh() const { return p_->mesh; }
int Engine::level_stride() const { return p_->S; }
void *Engine::stream() const { return (void *)p_->stream; }
void Engine::synchronize() const { CK(cudaStreamSynchronize(p_->stream)); }
size_t Engine::device_bytes() const { return p_->bytes; }
int Engine::num_tracers() const { return (int)p_->tr.size(); }

void Engine::set_velocity(const double *uv, const double *w) {
  EngineImpl &P = *p_;
  const MeshHost &M = P.mesh;
  const int L = M.nl - 1, T = M.elem2D, N = M.nod2D;
  std::vector<double> st((size_t)2 * T * P.S, 0.0);
  for (int e = 0; e < T; e++)
    for (int k = 0; k < L; k++) {
      st[2 * ((size_t)e * P.S + k)] = uv[2 * ((size_t)e * L + k)];
      st[2 * ((size_t)e * P.S + k) + 1] = uv[2 * ((size_t)e * L + k) + 1];
    }
  CK(cudaMemcpy(P.vel, st.data(), st.size() * sizeof(double), cudaMemcpyHostToDevice));
  P.copy_cols_to(P.W, w, M.nl, N);
}

void Engine::set_velocity_zero() {
  EngineImpl &P = *p_;
  CK(cudaMemset(P.vel, 0, sizeof(double) * 2 * P.mesh.elem2D * P.S));
  CK(cudaMemset(P.W, 0, sizeof(double) * P.mesh.nod2D * P.S));
}

void Engine::allocate_tracers(int ntr) {
  EngineImpl &P = *p_;
  CK(cudaStreamSynchronize(P.stream));
  for (auto &t : P.tr) { P.dfree(t.T); P.dfree(t.Tout); P.dfree(t.TAB); }
  P.tr.assign(ntr, EngineImpl::Tracer{});
  const size_t n = (size_t)P.mesh.nod2D * P.S;
  for (auto &t : P.tr) {
    t.T = P.dalloc<double>(n);
    t.Tout = P.dalloc<double>(n);
    t.TAB = P.dalloc<double>(n);
  }
  CK(cudaStreamSynchronize(P.stream));
}

static void check_id(const EngineImpl &P, int id) {
  if (id < 0 || id >= (int)P.tr.size()) throw std::out_of_range("invalid tracer id " + std::to_string(id + 1));
}

void Engine::set_values(int id, const double *v, bool also_ab) {
  EngineImpl &P = *p_;
  check_id(P, id);
  const int L = P.mesh.nl - 1;
  CK(cudaStreamSynchronize(P.stream));
  P.copy_cols_to(P.tr[id].T, v, L, P.mesh.nod2D);
  CK(cudaMemcpy(P.tr[id].Tout, P.tr[id].T, sizeof(double) * P.mesh.nod2D * P.S, cudaMemcpyDeviceToDevice));
  if (also_ab) CK(cudaMemcpy(P.tr[id].TAB, P.tr[id].T, sizeof(double) * P.mesh.nod2D * P.S, cudaMemcpyDeviceToDevice));
}

void Engine::set_values_ab(int id, const double *v) {
  EngineImpl &P = *p_;
  check_id(P, id);
  CK(cudaStreamSynchronize(P.stream));
  P.copy_cols_to(P.tr[id].TAB, v, P.mesh.nl - 1, P.mesh.nod2D);
}

void Engine::get_values(int id, double *out) const {
  EngineImpl &P = *p_;
  check_id(P, id);
  const int L = P.mesh.nl - 1, N = P.mesh.nod2D;
  std::vector<double> st((size_t)N * P.S);
  CK(cudaStreamSynchronize(P.stream));
  CK(cudaMemcpy(st.data(), P.tr[id].T, st.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int n = 0; n < N; n++) std::memcpy(out + (size_t)n * L, &st[(size_t)n * P.S], sizeof(double) * L);
}

void Engine::set_scheme(int id, const TracerScheme &s) {
  check_id(*p_, id);
  if (s.hor < 0 || s.hor > 2 || s.ver < 0 || s.ver > 3 || s.lim < 0 || s.lim > 1)
    throw std::invalid_argument("unknown advection scheme");
  p_->tr[id].sch = s;
}
TracerScheme Engine::scheme(int id) const {
  check_id(*p_, id);
  return p_->tr[id].sch;
}

int Engine::launches_per_tracer_step(int id) const {
  check_id(*p_, id);
  return p_->tr[id].sch.lim == 1 ? 6 : 3;
}

namespace {

enum { KK_EDGE = 0, KK_LO, KK_VERT, KK_BOUNDS, KK_RATIO, KK_APPLY, KK_COUNT };
const char *const kKindNames[KK_COUNT] = {"edge_flux", "node_lo", "node_vert", "node_bounds", "node_ratio",
                                          "node_apply"};

template <int HOR, int LIM>
void launch_edge(EngineImpl &P, const StepArgs<double> &a) {
  const DSched &s = P.dm.edge_sched;
  if (s.nblk <= 0) return;
  P.mark_begin(KK_EDGE);
  k_edge_flux<double, HOR, LIM><<<s.nblk, kBlock, (s.max_items + 1) * sizeof(int), P.stream>>>(P.dm, a);
  P.mark_end();
}
template <int VER, int LIM>
void launch_vert(EngineImpl &P, const StepArgs<double> &a) {
  const DSched &s = P.dm.node_sched;
  P.mark_begin(KK_VERT);
  k_node_vert<double, VER, LIM><<<s.nblk, kBlock, (s.max_items + 1) * sizeof(int), P.stream>>>(P.dm, a);
  P.mark_end();
}

template <int LIM>
void run_step(EngineImpl &P, const TracerScheme &sc, const StepArgs<double> &a) {
  switch (sc.hor) {
    case 1: launch_edge<HOR_MUSCL, LIM>(P, a); break;
    case 2: launch_edge<HOR_MFCT, LIM>(P, a); break;
    default: launch_edge<HOR_UPW1, LIM>(P, a); break;
  }
  const DSched &s = P.dm.node_sched;
  const size_t sm = (s.max_items + 1) * sizeof(int);
  if (LIM == LIM_FCT) {
    P.mark_begin(KK_LO);
    k_node_lo<double><<<s.nblk, kBlock, sm, P.stream>>>(P.dm, a);
    P.mark_end();
  }
  switch (sc.ver) {
    case 1: launch_vert<VER_PPM, LIM>(P, a); break;
    case 2: launch_vert<VER_QR4C, LIM>(P, a); break;
    case 3: launch_vert<VER_CDIFF, LIM>(P, a); break;
    default: launch_vert<VER_UPW1, LIM>(P, a); break;
  }
  if (LIM == LIM_FCT) {
    P.mark_begin(KK_BOUNDS);
    k_node_bounds<double><<<s.nblk, kBlock, sm, P.stream>>>(P.dm, a);
    P.mark_end();
    P.mark_begin(KK_RATIO);
    k_node_ratio<double><<<s.nblk, kBlock, sm, P.stream>>>(P.dm, a);
    P.mark_end();
  }
  P.mark_begin(KK_APPLY);
  k_node_apply<double, LIM><<<s.nblk, kBlock, sm, P.stream>>>(P.dm, a);
  P.mark_end();
}

}  // namespace

void Engine::step_tracer(int id, double dt, bool refresh_ab) {
  EngineImpl &P = *p_;
  check_id(P, id);
  auto &t = P.tr[id];
  StepArgs<double> a;
  a.T = t.T;
  a.TAB = refresh_ab ? t.T : t.TAB;
  a.vel = P.vel;
  a.W = P.W;
  a.dt = dt;
  a.ph = t.sch.ph;
  a.pv = t.sch.pv;
  a.flo = P.flo; a.adf_h = P.adfh; a.adf_v = P.adfv; a.lo = P.lo;
  a.tmax = P.tmax; a.tmin = P.tmin; a.rp = P.rp; a.rm = P.rm;
  a.T_out = t.Tout;
  if (P.mesh.nod2D > 0) {
    if (t.sch.lim == 1) run_step<LIM_FCT>(P, t.sch, a);
    else run_step<LIM_NONE>(P, t.sch, a);
    CK(cudaGetLastError());
  }
  std::swap(t.T, t.Tout);
}

void Engine::step(double dt, bool refresh_ab) {
  for (int i = 0; i < (int)p_->tr.size(); i++) step_tracer(i, dt, refresh_ab);
}

const char *const *Engine::kernel_kind_names(int *n) {
  *n = KK_COUNT;
  return kKindNames;
}

int Engine::profile_steps(int nsteps, double dt, bool refresh_ab, double *ms, int nkinds) {
  EngineImpl &P = *p_;
  std::vector<EngineImpl::ProfRec> recs;
  P.prof = &recs;
  try {
    for (int s = 0; s < nsteps; s++) step(dt, refresh_ab);
  } catch (...) {
    P.prof = nullptr;
    throw;
  }
  P.prof = nullptr;
  CK(cudaStreamSynchronize(P.stream));
  for (int k = 0; k < nkinds; k++) ms[k] = 0.0;
  for (auto &r : recs) {
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, r.a, r.b));
    if (r.kind < nkinds) ms[r.kind] += t;
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  return (int)recs.size();
}

void Engine::stats(int id, double out[4]) const {
  const int L = p_->mesh.nl - 1, N = p_->mesh.nod2D;
  std::vector<double> v((size_t)L * N);
  get_values(id, v.data());
  double mn = v.empty() ? 0.0 : v[0], mx = mn, sm = 0.0, nan = 0.0;
  for (double x : v) {
    if (x < mn) mn = x;
    if (x > mx) mx = x;
    sm += x;
    if (x != x) nan += 1.0;
  }
  out[0] = mn; out[1] = mx; out[2] = sm; out[3] = nan;
}

}  // namespace fesom
