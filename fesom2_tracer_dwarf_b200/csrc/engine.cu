// Engine: device memory, layout conversion, schedules and kernel dispatch.
#include <algorithm>
#include <mutex>
#include <unordered_map>
#include <cstring>
#include <stdexcept>
#include <string>

#include "advect_fused.cuh"
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
  for (size_t b = 0; b + 1 < blk.size(); b++)
    if (off[blk[b + 1]] - off[blk[b]] > kMaxCellsPerBlock)
      throw std::runtime_error("schedule block exceeds the per-block cell capacity");
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
  // work arrays, one slot per tracer of a batch
  int slots = 0;
  double *vflux = nullptr;
  double *adfh[NTMAX] = {}, *adfv[NTMAX] = {}, *lo[NTMAX] = {}, *rp[NTMAX] = {}, *rm[NTMAX] = {};
  void ensure_slots(int n) {
    if (n <= slots) return;
    const size_t ns = (size_t)mesh.nod2D * S, es = (size_t)mesh.edge2D * S;
    if (!vflux) vflux = dalloc<double>(es);
    for (int t = slots; t < n; t++) {
      adfh[t] = dalloc<double>(es);
      adfv[t] = dalloc<double>(ns);
      lo[t] = dalloc<double>(ns);
      rp[t] = dalloc<double>(ns);
      rm[t] = dalloc<double>(ns);
    }
    slots = n;
  }
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
  // Every transfer is ordered on the engine's stream (which does not
  // synchronise with the legacy default stream) and completes before the call
  // returns, so host staging buffers may be released right after.
  void h2d(void *d, const void *h, size_t bytes) {
    if (!bytes) return;
    CK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
  }
  void d2h(void *h, const void *d, size_t bytes) {
    if (!bytes) return;
    CK(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
  }
  void d2d(void *dst, const void *src, size_t bytes) {
    if (!bytes) return;
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream));
    CK(cudaStreamSynchronize(stream));
  }
  template <typename T>
  T *upload(const std::vector<T> &h) {
    T *d = dalloc<T>(h.size());
    h2d(d, h.data(), h.size() * sizeof(T));
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
    h2d(d, st.data(), st.size() * sizeof(double));
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

  // slot order: edges sorted by their smaller node id (stable in edge id)
  std::vector<int> slot_edge(E), edge_slot(E);
  for (int e = 0; e < E; e++) slot_edge[e] = e;
  std::stable_sort(slot_edge.begin(), slot_edge.end(), [&](int a, int b) {
    return std::min(M.edge_nodes[2 * a], M.edge_nodes[2 * a + 1]) <
           std::min(M.edge_nodes[2 * b], M.edge_nodes[2 * b + 1]);
  });
  for (int s = 0; s < E; s++) edge_slot[slot_edge[s]] = s;
  std::vector<int2> en(E), et(E), el(E), ud(E);
  std::vector<double> ecross(4 * (size_t)E), edxdy(2 * (size_t)E), ea(E);
  for (int s = 0; s < E; s++) {
    const int e = slot_edge[s];
    en[s] = make_int2(M.edge_nodes[2 * e], M.edge_nodes[2 * e + 1]);
    et[s] = make_int2(M.edge_tri[2 * e], M.edge_tri[2 * e + 1]);
    el[s] = make_int2(M.edge_shared_levels(e), M.edge_levels(e));
    ud[s] = make_int2(M.up_dn_tri[2 * e], M.up_dn_tri[2 * e + 1]);
    for (int q = 0; q < 4; q++) ecross[4 * (size_t)s + q] = M.edge_cross[4 * (size_t)e + q];
    for (int q = 0; q < 2; q++) edxdy[2 * (size_t)s + q] = M.edge_dxdy[2 * (size_t)e + q];
    ea[s] = M.edge_a[e];
  }
  d.edge_nodes = P.upload(en);
  d.edge_tri = P.upload(et);
  d.edge_lev = P.upload(el);
  d.up_dn = P.upload(ud);
  d.edge_cross = P.upload(ecross);
  d.edge_dxdy = P.upload(edxdy);
  d.edge_a = P.upload(ea);
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
  {
    std::vector<int4> ne4(M.node_edge.size());
    for (int n = 0; n < N; n++)
      for (int p = M.node_edge_ptr[n]; p < M.node_edge_ptr[n + 1]; p++) {
        const int code = M.node_edge[p], e = code >> 1, second = code & 1;
        const int other = M.edge_nodes[2 * e + (second ? 0 : 1)];
        ne4[p] = make_int4((edge_slot[e] << 1) | second, other, M.edge_levels(e), 0);
      }
    d.ne4 = P.upload(ne4);
  }
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
  for (int s = 0; s < E; s++) cnt[s] = M.edge_levels(slot_edge[s]);
  build_sched(cnt, off, blk, d.edge_sched.max_items);
  d.edge_sched.cell_off = P.upload(off);
  d.edge_sched.blk = P.upload(blk);
  d.edge_sched.nblk = (int)blk.size() - 1;

  P.vel = P.dalloc<double>((size_t)2 * T * P.S);
  P.W = P.dalloc<double>((size_t)N * P.S);
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
  P.h2d(P.vel, st.data(), st.size() * sizeof(double));
  P.copy_cols_to(P.W, w, M.nl, N);
}

void Engine::set_velocity_zero() {
  EngineImpl &P = *p_;
  CK(cudaMemsetAsync(P.vel, 0, sizeof(double) * 2 * P.mesh.elem2D * P.S, P.stream));
  CK(cudaMemsetAsync(P.W, 0, sizeof(double) * P.mesh.nod2D * P.S, P.stream));
  CK(cudaStreamSynchronize(P.stream));
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
  P.d2d(P.tr[id].Tout, P.tr[id].T, sizeof(double) * P.mesh.nod2D * P.S);
  if (also_ab) P.d2d(P.tr[id].TAB, P.tr[id].T, sizeof(double) * P.mesh.nod2D * P.S);
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
  P.d2h(st.data(), P.tr[id].T, st.size() * sizeof(double));
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

namespace {

enum { KK_EDGE = 0, KK_COL1, KK_COL2, KK_COL3, KK_COUNT };
const char *const kKindNames[KK_COUNT] = {"k_edge", "k_col1", "k_col2", "k_col3"};

// Raise the dynamic shared-memory limit of a kernel once (per kernel
// function; all kernels share one C++ function-pointer type).
template <typename K>
void set_smem(K kernel, size_t bytes) {
  static std::mutex mu;
  static std::unordered_map<const void *, size_t> done;
  std::lock_guard<std::mutex> lock(mu);
  auto it = done.find((const void *)kernel);
  if (it != done.end() && it->second >= bytes) return;
  CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  done[(const void *)kernel] = bytes;
}

template <int NT, int HOR, int LIM>
void launch_edge(EngineImpl &P, const FusedArgs<double> &a) {
  const DSched &s = P.dm.edge_sched;
  if (s.nblk <= 0) return;
  const size_t sm = smem_edge<double>();
  P.mark_begin(KK_EDGE);
  k_edge<double, NT, HOR, LIM><<<s.nblk, kThreads, sm, P.stream>>>(P.dm, a);
  P.mark_end();
}

template <int NT, int VER, int LIM>
void launch_col1(EngineImpl &P, const FusedArgs<double> &a) {
  const DSched &s = P.dm.node_sched;
  const size_t sm = smem_col<double>(NT, 4);
  set_smem(k_col1<double, NT, VER, LIM>, sm);
  P.mark_begin(KK_COL1);
  k_col1<double, NT, VER, LIM><<<s.nblk, kThreads, sm, P.stream>>>(P.dm, a);
  P.mark_end();
}

template <int NT, int LIM>
void run_group(EngineImpl &P, const TracerScheme &sc, const FusedArgs<double> &a) {
  switch (sc.hor) {
    case 1: launch_edge<NT, HOR_MUSCL, LIM>(P, a); break;
    case 2: launch_edge<NT, HOR_MFCT, LIM>(P, a); break;
    default: launch_edge<NT, HOR_UPW1, LIM>(P, a); break;
  }
  switch (sc.ver) {
    case 1: launch_col1<NT, VER_PPM, LIM>(P, a); break;
    case 2: launch_col1<NT, VER_QR4C, LIM>(P, a); break;
    case 3: launch_col1<NT, VER_CDIFF, LIM>(P, a); break;
    default: launch_col1<NT, VER_UPW1, LIM>(P, a); break;
  }
  const DSched &s = P.dm.node_sched;
  if (LIM == LIM_FCT) {
    const size_t sm2 = smem_col<double>(NT, 2);
    set_smem(k_col2<double, NT>, sm2);
    P.mark_begin(KK_COL2);
    k_col2<double, NT><<<s.nblk, kThreads, sm2, P.stream>>>(P.dm, a);
    P.mark_end();
  }
  const size_t sm3 = smem_col<double>(NT, 0);
  P.mark_begin(KK_COL3);
  k_col3<double, NT, LIM><<<s.nblk, kThreads, sm3, P.stream>>>(P.dm, a);
  P.mark_end();
}

template <int NT>
void run_group_nt(EngineImpl &P, const TracerScheme &sc, const FusedArgs<double> &a) {
  if (sc.lim == 1) run_group<NT, LIM_FCT>(P, sc, a);
  else run_group<NT, LIM_NONE>(P, sc, a);
}

}  // namespace

// Tracers are advanced in batches of up to NTMAX consecutive tracers with
// the same scheme; a batch shares the edge volume fluxes, the geometry loads
// and every geometry-only division.
static void run_batch(EngineImpl &P, int first, int nt, double dt, bool refresh_ab) {
  P.ensure_slots(nt);
  FusedArgs<double> a{};
  const TracerScheme &sc = P.tr[first].sch;
  for (int t = 0; t < nt; t++) {
    auto &tr = P.tr[first + t];
    a.T[t] = tr.T;
    a.TAB[t] = refresh_ab ? tr.T : tr.TAB;
    a.T_out[t] = tr.Tout;
    a.adf_h[t] = P.adfh[t];
    a.adf_v[t] = P.adfv[t];
    a.lo[t] = P.lo[t];
    a.rp[t] = P.rp[t];
    a.rm[t] = P.rm[t];
  }
  a.vflux = P.vflux;
  a.vel = P.vel;
  a.W = P.W;
  a.dt = dt;
  a.ph = sc.ph;
  a.pv = sc.pv;
  if (P.mesh.nod2D > 0) {
    if (nt == 4) run_group_nt<4>(P, sc, a);
    else if (nt == 2) run_group_nt<2>(P, sc, a);
    else run_group_nt<1>(P, sc, a);
    CK(cudaGetLastError());
  }
  for (int t = 0; t < nt; t++) std::swap(P.tr[first + t].T, P.tr[first + t].Tout);
}

static bool same_scheme(const TracerScheme &a, const TracerScheme &b) {
  return a.hor == b.hor && a.ver == b.ver && a.lim == b.lim && a.ph == b.ph && a.pv == b.pv;
}

// batch sizes the engine launches: 4, 2 or 1 tracers
static int batch_size(const EngineImpl &P, int first) {
  int run = 1;
  while (first + run < (int)P.tr.size() && run < NTMAX && same_scheme(P.tr[first].sch, P.tr[first + run].sch)) run++;
  return run >= 4 ? 4 : (run >= 2 ? 2 : 1);
}

int Engine::launches_per_step() const {
  const EngineImpl &P = *p_;
  int n = 0;
  for (int i = 0; i < (int)P.tr.size();) {
    const int nt = batch_size(P, i);
    n += P.tr[i].sch.lim == 1 ? 4 : 3;
    i += nt;
  }
  return n;
}

void Engine::step_tracer(int id, double dt, bool refresh_ab) {
  check_id(*p_, id);
  run_batch(*p_, id, 1, dt, refresh_ab);
}

size_t Engine::step_scratch_doubles() const {
  const EngineImpl &P = *p_;
  auto up = [](size_t n) { return (n + 31) / 32 * 32; };  // 256-byte pieces
  const size_t es = up((size_t)P.mesh.edge2D * P.S), ns = up((size_t)P.mesh.nod2D * P.S);
  return 2 * es + 4 * ns;
}

void Engine::step_with_scratch(int id, const double *T, const double *TAB, double *T_out, double dt,
                               double *scratch, size_t scratch_doubles) {
  EngineImpl &P = *p_;
  check_id(P, id);
  if (scratch_doubles < step_scratch_doubles()) throw std::length_error("scratch too small for this mesh");
  auto up = [](size_t n) { return (n + 31) / 32 * 32; };
  const size_t es = up((size_t)P.mesh.edge2D * P.S), ns = up((size_t)P.mesh.nod2D * P.S);
  const TracerScheme &sc = P.tr[id].sch;
  FusedArgs<double> a{};
  a.T[0] = T;
  a.TAB[0] = TAB;
  a.T_out[0] = T_out;
  a.vflux = scratch;
  a.adf_h[0] = scratch + es;
  a.adf_v[0] = scratch + 2 * es;
  a.lo[0] = scratch + 2 * es + ns;
  a.rp[0] = scratch + 2 * es + 2 * ns;
  a.rm[0] = scratch + 2 * es + 3 * ns;
  a.vel = P.vel;
  a.W = P.W;
  a.dt = dt;
  a.ph = sc.ph;
  a.pv = sc.pv;
  if (P.mesh.nod2D > 0) {
    run_group_nt<1>(P, sc, a);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(P.stream));
}

void Engine::step(double dt, bool refresh_ab) {
  for (int i = 0; i < (int)p_->tr.size();) {
    const int nt = batch_size(*p_, i);
    run_batch(*p_, i, nt, dt, refresh_ab);
    i += nt;
  }
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
