// Engine: device memory, layout conversion, schedules, batching and
// dispatch to the per-precision kernel units (step_f64.cu, step_f32.cu).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>

#include "advect_fused.cuh"
#include "engine_impl.hpp"

namespace fesom {

namespace {
thread_local std::string g_err;
}
const char *last_error() { return g_err.c_str(); }
void set_last_error(const std::string &s) { g_err = s; }

namespace {

void build_sched(const std::vector<int> &counts, std::vector<int> &off, std::vector<int> &blk, int &max_items,
                 int cells_per_block) {
  const int n = (int)counts.size();
  off.assign(n + 1, 0);
  for (int i = 0; i < n; i++) off[i + 1] = off[i] + counts[i];
  blk.clear();
  blk.push_back(0);
  max_items = 1;
  // cells_per_block is a cap: a block takes whole items while its wet cells
  // stay within it, so that the 256 threads of a block walk its cells in at
  // most cap / 256 rounds (with a target instead, blocks overshooting 512
  // cells by a column gave a third round to a few threads, and the block's
  // time followed them: measured at 1000x1000x64, a 448 target was 6 %
  // faster than a 512 one).  A single item larger than the cap gets a block
  // of its own.
  const int cap = std::min(cells_per_block, kMaxCellsPerBlock);
  int start = 0, cells = 0;
  for (int i = 0; i < n; i++) {
    // close the block before an item that would overflow its capacity
    if (i > start && (cells + counts[i] > cap || i - start >= kMaxItemsPerBlock)) {
      blk.push_back(i);
      max_items = std::max(max_items, i - start);
      start = i;
      cells = 0;
    }
    cells += counts[i];
  }
  if (start < n || n == 0) {
    blk.push_back(n);
    max_items = std::max(max_items, n - start);
  }
  for (size_t b = 0; b + 1 < blk.size(); b++)
    if (off[blk[b + 1]] - off[blk[b]] > kMaxCellsPerBlock)
      throw std::runtime_error("a column or edge has more levels than a block holds");
}

// (ld, ncol) column-major host doubles -> device columns of stride S, type R
template <typename R>
R *upload_cols(EngineImpl &P, const double *h, int ld, int ncol, int nvalid) {
  std::vector<R> st((size_t)ncol * P.S, R(0));
  for (int c = 0; c < ncol; c++)
    for (int k = 0; k < nvalid; k++) st[(size_t)c * P.S + k] = (R)h[(size_t)c * ld + k];
  return P.upload(st);
}
template <typename R>
R *upload_conv(EngineImpl &P, const std::vector<double> &h) {
  std::vector<R> st(h.size());
  for (size_t i = 0; i < h.size(); i++) st[i] = (R)h[i];
  return P.upload(st);
}

// Work schedules (node, edge and gradient cells) for a cap on the wet
// cells per block; the arrays of a previous tiling are released.
template <typename R>
void build_schedules(EngineImpl &P, DMeshT<R> &d, int cells_per_block) {
  const MeshHost &M = P.mesh;
  const int N = M.nod2D, E = M.edge2D;
  const std::vector<int> &slot_edge = P.slot_edge;
  for (const void *q : {(const void *)d.node_sched.cell_off, (const void *)d.node_sched.blk,
                        (const void *)d.edge_sched.cell_off, (const void *)d.edge_sched.blk,
                        (const void *)d.grad_sched.cell_off, (const void *)d.grad_sched.blk,
                        (const void *)d.grad_lev0})
    P.dfree(const_cast<void *>(q));
  std::vector<int> cnt(N), off, blk;
  for (int n = 0; n < N; n++) cnt[n] = M.nlev_node[n] - 1;
  build_sched(cnt, off, blk, d.node_sched.max_items, cells_per_block);
  d.node_sched.cell_off = P.upload(off);
  d.node_sched.blk = P.upload(blk);
  d.node_sched.nblk = (int)blk.size() - 1;
  cnt.assign(E, 0);
  for (int s = 0; s < E; s++) cnt[s] = M.edge_levels(slot_edge[s]);
  build_sched(cnt, off, blk, d.edge_sched.max_items, cells_per_block);
  d.edge_sched.cell_off = P.upload(off);
  d.edge_sched.blk = P.upload(blk);
  d.edge_sched.nblk = (int)blk.size() - 1;

  // ring-mean gradient levels: an edge uses the node ring means from level
  // k = min(nlevels_nod2D_min(n1), nlevels_nod2D_min(n2)) - 1 down (from the
  // surface when it lacks an up or down triangle)
  std::vector<int> lev0(N);
  for (int n = 0; n < N; n++) lev0[n] = std::max(0, M.nlev_node[n] - 1);
  for (int e = 0; e < E; e++) {
    const int n1 = M.edge_nodes[2 * e], n2 = M.edge_nodes[2 * e + 1];
    const bool pair = M.up_dn_tri[2 * e] >= 0 && M.up_dn_tri[2 * e + 1] >= 0;
    const int thr = pair ? std::max(0, std::min(M.nlev_node_min[n1], M.nlev_node_min[n2]) - 1) : 0;
    lev0[n1] = std::min(lev0[n1], thr);
    lev0[n2] = std::min(lev0[n2], thr);
  }
  d.grad_lev0 = P.upload(lev0);
  for (int n = 0; n < N; n++) cnt[n] = std::max(0, M.nlev_node[n] - 1 - lev0[n]);
  cnt.resize(N);
  build_sched(cnt, off, blk, d.grad_sched.max_items, cells_per_block);
  d.grad_sched.cell_off = P.upload(off);
  d.grad_sched.blk = P.upload(blk);
  d.grad_sched.nblk = (int)blk.size() - 1;
}

template <typename R>
void build_dmesh(EngineImpl &P, DMeshT<R> &d, const std::vector<int> &slot_edge, const std::vector<int> &edge_slot) {
  const MeshHost &M = P.mesh;
  const int N = M.nod2D, T = M.elem2D, E = M.edge2D, nl = M.nl, L = nl - 1;
  d.N = N; d.T = T; d.E = E; d.nl = nl; d.S = P.S;
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
  d.edge_cross = upload_conv<R>(P, ecross);
  d.edge_dxdy = upload_conv<R>(P, edxdy);
  d.edge_a = upload_conv<R>(P, ea);
  d.nlev_elem = P.upload(M.nlev_elem);
  d.nlev_node = P.upload(M.nlev_node);
  d.nlev_node_min = P.upload(M.nlev_node_min);
  d.nbl = P.upload(M.nboundary_lay);
  d.elem_nodes = P.upload(M.elem_nodes);
  d.grad_sca = upload_conv<R>(P, M.grad_sca);
  d.elem_area = upload_conv<R>(P, M.elem_area);
  d.ring_ptr = P.upload(M.ring_ptr);
  d.ring_elem = P.upload(M.ring_elem);
  {
    // complete rings: every element holding the node is listed (the
    // reference's periodic compat lists are not, on the wrap rows)
    std::vector<int> holds(N, 0);
    for (int e = 0; e < T; e++)
      for (int q = 0; q < 3; q++) holds[M.elem_nodes[3 * e + q]]++;
    std::vector<unsigned char> full(N);
    for (int n = 0; n < N; n++) full[n] = (M.ring_ptr[n + 1] - M.ring_ptr[n]) == holds[n];
    d.ring_full = P.upload(full);
  }
  d.ne_ptr = P.upload(M.node_edge_ptr);
  {
    std::vector<int4> ne4(M.node_edge.size());
    for (int n = 0; n < N; n++)
      for (int p = M.node_edge_ptr[n]; p < M.node_edge_ptr[n + 1]; p++) {
        const int code = M.node_edge[p], e = code >> 1, second = code & 1;
        const int other = M.edge_nodes[2 * e + (second ? 0 : 1)];
        ne4[p] = make_int4((edge_slot[e] << 1) | second, other, M.edge_levels(e), other * P.S);
      }
    d.ne4 = P.upload(ne4);
  }
  d.zbar = upload_conv<R>(P, M.zbar);
  d.Z = upload_conv<R>(P, M.Z);
  d.area = upload_cols<R>(P, M.area.data(), nl, N, nl);
  d.areasvol = upload_cols<R>(P, M.areasvol.data(), nl, N, nl);
  d.hnode = upload_cols<R>(P, M.hnode.data(), L, N, L);
  d.hnode_new = upload_cols<R>(P, M.hnode_new.data(), L, N, L);
  d.helem = upload_cols<R>(P, M.helem.data(), L, T, L);

  build_schedules(P, d, kCellsPerBlock);
}

// Patch plan of the fused step kernel: built on the host, uploaded, host
// lists released (the maxima stay for the shared-memory layout).
void build_tiles(EngineImpl &P, const std::vector<int> &edge_slot, int owned) {
  for (const void *q : {(const void *)P.tiles.cnt, (const void *)P.tiles.node_gid, (const void *)P.tiles.node_info,
                        (const void *)P.tiles.inc_ptr, (const void *)P.tiles.inc, (const void *)P.tiles.edge_slot,
                        (const void *)P.tiles.edge_nn, (const void *)P.tiles.edge_ud, (const void *)P.tiles.elem_gid,
                        (const void *)P.tiles.elem_nn, (const void *)P.tiles.ring_ptr, (const void *)P.tiles.ring})
    P.dfree(const_cast<void *>(q));
  P.tiles = DTiles{};
  P.tplan = TilePlanHost();
  if (P.mesh.nod2D <= 0 || P.mesh.nl > kTileMaxLevels) return;
  TilePlanHost &t = P.tplan;
  try {
    t = build_tile_plan(P.mesh, edge_slot, owned);
  } catch (const std::exception &) {
    t = TilePlanHost();  // no plan: the five-kernel path runs every scheme
    return;
  }
  DTiles &d = P.tiles;
  d.cnt = P.upload(t.cnt);
  d.node_gid = P.upload(t.node_gid);
  d.node_info = P.upload(t.node_info);
  d.inc_ptr = P.upload(t.inc_ptr);
  d.inc = P.upload(t.inc);
  d.edge_slot = P.upload(t.edge_slot);
  d.edge_nn = P.upload(t.edge_nn);
  d.edge_ud = P.upload(t.edge_ud);
  d.elem_gid = P.upload(t.elem_gid);
  d.elem_nn = P.upload(t.elem_nn);
  d.ring_ptr = P.upload(t.ring_ptr);
  d.ring = P.upload(t.ring);
  d.np = t.np;
  for (auto *v : {&t.node_gid, &t.inc_ptr, &t.edge_slot, &t.elem_gid, &t.ring_ptr}) std::vector<int>().swap(*v);
  for (auto *v : {&t.node_info, &t.inc, &t.edge_nn, &t.edge_ud, &t.elem_nn}) std::vector<uint32_t>().swap(*v);
  std::vector<uint16_t>().swap(t.ring);
  std::vector<TileCounts>().swap(t.cnt);
}

}  // namespace

static_assert(Engine::kDefaultCellsPerBlock == kCellsPerBlock, "one default schedule tile");

std::vector<int> edge_slot_order(const MeshHost &M) {
  // slot order: edges sorted by their smaller node id (stable in edge id)
  const int E = M.edge2D;
  std::vector<int> slot_edge(E), edge_slot(E);
  for (int e = 0; e < E; e++) slot_edge[e] = e;
  std::stable_sort(slot_edge.begin(), slot_edge.end(), [&](int a, int b) {
    return std::min(M.edge_nodes[2 * a], M.edge_nodes[2 * a + 1]) < std::min(M.edge_nodes[2 * b], M.edge_nodes[2 * b + 1]);
  });
  for (int s = 0; s < E; s++) edge_slot[slot_edge[s]] = s;
  return edge_slot;
}

Engine::Engine(const MeshHost &mesh, Precision prec) : p_(new EngineImpl) {
  EngineImpl &P = *p_;
  P.mesh = mesh;
  P.prec = prec;
  P.r_bytes = prec == Precision::FP64 ? 8 : 4;
  P.ts_bytes = prec == Precision::FP64 ? 8 : (prec == Precision::FP32 ? 4 : 2);
  const std::string bad = mesh.validate();
  if (!bad.empty()) throw std::invalid_argument("mesh: " + bad);
  const MeshHost &M = P.mesh;
  const int E = M.edge2D;
  // level stride: 32-byte aligned columns for FP64, 16-byte aligned ones (or
  // better) for the 4- and 2-byte types
  P.S = prec == Precision::FP64 ? (M.nl + 3) / 4 * 4 : (M.nl + 7) / 8 * 8;
  // the kernels index cells with 32-bit offsets (node column bases as int)
  if ((long long)M.nod2D * P.S >= (1ll << 31) || (long long)M.edge2D * P.S >= (1ll << 32))
    throw std::invalid_argument("mesh too large: nodes x level stride must stay below 2^31 and edges x level stride "
                                "below 2^32");
  CK(cudaGetDevice(&P.device));
  CK(cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking));
  const std::vector<int> edge_slot = edge_slot_order(M);
  std::vector<int> slot_edge(E);
  for (int e = 0; e < E; e++) slot_edge[edge_slot[e]] = e;
  P.slot_edge = slot_edge;
  if (prec == Precision::FP64) {
    build_dmesh<double>(P, P.dm64, slot_edge, edge_slot);
    build_rcp_f64(P);
  } else {
    build_dmesh<float>(P, P.dm32, slot_edge, edge_slot);
    build_rcp_f32(P);
  }
  build_tiles(P, edge_slot, kTileOwned);
  P.nonfinite_d = P.dalloc<unsigned long long>(1);
  P.vel = P.dalloc_bytes((size_t)2 * M.elem2D * P.S * P.r_bytes);
  P.W = P.dalloc_bytes((size_t)M.nod2D * P.S * P.r_bytes);
  CK(cudaStreamSynchronize(P.stream));
}

Engine::~Engine() {
  if (!p_) return;
  cudaStreamSynchronize(p_->stream);
  if (p_->io_h2d) {
    cudaStreamSynchronize(p_->io_h2d);
    cudaStreamSynchronize(p_->io_d2h);
    cudaStreamDestroy(p_->io_h2d);
    cudaStreamDestroy(p_->io_d2h);
  }
  for (cudaEvent_t e : p_->io_ev_in) cudaEventDestroy(e);
  for (cudaEvent_t e : p_->io_ev_out) cudaEventDestroy(e);
  release_ring(*p_);
  learned_release(*p_);
  for (void *a : p_->allocs) cudaFree(a);
  cudaStreamDestroy(p_->stream);
  delete p_;
}

const MeshHost &Engine::mesh() const { return p_->mesh; }
EngineImpl *Engine::impl() { return p_; }

void Engine::set_cells_per_block(int cells) {
  EngineImpl &P = *p_;
  if (cells < 32 || cells > kMaxCellsPerBlock) throw std::invalid_argument("cells per block must be in [32, 576]");
  CK(cudaStreamSynchronize(P.stream));
  if (P.prec == Precision::FP64) build_schedules(P, P.dm64, cells);
  else build_schedules(P, P.dm32, cells);
  P.cells_per_block = cells;
  CK(cudaStreamSynchronize(P.stream));
}
int Engine::cells_per_block() const { return p_->cells_per_block; }
int Engine::level_stride() const { return p_->S; }
Precision Engine::precision() const { return p_->prec; }
void *Engine::stream() const { return (void *)p_->stream; }
int Engine::device() const { return p_->device; }
void Engine::set_fma64(bool on) { p_->fma64 = on; }
long long Engine::nonfinite_values(bool reset) {
  EngineImpl &P = *p_;
  unsigned long long n = 0;
  P.d2h(&n, P.nonfinite_d, sizeof(n));
  if (reset && n) {
    CK(cudaMemsetAsync(P.nonfinite_d, 0, sizeof(n), P.stream));
    CK(cudaStreamSynchronize(P.stream));
  }
  return (long long)n;
}
bool Engine::fma64() const { return p_->fma64; }
void Engine::synchronize() const { CK(cudaStreamSynchronize(p_->stream)); }
size_t Engine::device_bytes() const { return p_->bytes; }
int Engine::num_tracers() const { return (int)p_->tr.size(); }

void Engine::set_velocity(const double *uv, const double *w) {
  EngineImpl &P = *p_;
  P.vflux_valid = false;
  const MeshHost &M = P.mesh;
  const int L = M.nl - 1, T = M.elem2D, N = M.nod2D;
  std::vector<double> st((size_t)2 * T * P.S, 0.0), wst((size_t)N * P.S, 0.0);
  for (int e = 0; e < T; e++)
    for (int k = 0; k < L; k++) {
      st[2 * ((size_t)e * P.S + k)] = uv[2 * ((size_t)e * L + k)];
      st[2 * ((size_t)e * P.S + k) + 1] = uv[2 * ((size_t)e * L + k) + 1];
    }
  for (int n = 0; n < N; n++) std::memcpy(&wst[(size_t)n * P.S], w + (size_t)n * M.nl, sizeof(double) * M.nl);
  if (P.prec == Precision::FP64) {
    P.h2d(P.vel, st.data(), st.size() * sizeof(double));
    P.h2d(P.W, wst.data(), wst.size() * sizeof(double));
  } else {
    std::vector<float> f(st.begin(), st.end()), fw(wst.begin(), wst.end());
    P.h2d(P.vel, f.data(), f.size() * sizeof(float));
    P.h2d(P.W, fw.data(), fw.size() * sizeof(float));
  }
}

void Engine::set_velocity_zero() {
  EngineImpl &P = *p_;
  P.vflux_valid = false;
  CK(cudaMemsetAsync(P.vel, 0, P.r_bytes * 2 * P.mesh.elem2D * P.S, P.stream));
  CK(cudaMemsetAsync(P.W, 0, P.r_bytes * P.mesh.nod2D * P.S, P.stream));
  CK(cudaStreamSynchronize(P.stream));
}

void Engine::allocate_tracers(int ntr, bool with_ab) {
  EngineImpl &P = *p_;
  CK(cudaStreamSynchronize(P.stream));
  for (auto &t : P.tr) { P.dfree(t.T); P.dfree(t.Tout); P.dfree(t.TAB); }
  P.tr.assign(ntr, EngineImpl::Tracer{});
  const size_t n = (size_t)P.mesh.nod2D * P.S * P.ts_bytes;
  for (auto &t : P.tr) {
    t.T = P.dalloc_bytes(n);
    t.Tout = P.dalloc_bytes(n);
    t.TAB = with_ab ? P.dalloc_bytes(n) : nullptr;
  }
  CK(cudaStreamSynchronize(P.stream));
}

void Engine::release_work() {
  EngineImpl &P = *p_;
  CK(cudaStreamSynchronize(P.stream));
  P.dfree(P.adfh[0]);  // the interleaved arrays: one allocation each
  P.dfree(P.lo[0]);
  P.dfree(P.adfv[0]);
  for (int t = 0; t < P.slots; t++) {
    P.adfh[t] = P.lo[t] = P.adfv[t] = nullptr;
    for (void **q : {&P.rpm[t], &P.gradn[t]}) {
      P.dfree(*q);
      *q = nullptr;
    }
  }
  P.dfree(P.vflux);
  P.vflux = nullptr;
  P.vflux_valid = false;
  P.slots = 0;
}

static void check_id(const EngineImpl &P, int id) {
  if (id < 0 || id >= (int)P.tr.size()) throw std::out_of_range("invalid tracer id " + std::to_string(id + 1));
}

static bool storage16(const EngineImpl &P) { return P.prec == Precision::BF16 || P.prec == Precision::FP16; }

void Engine::set_values(int id, const double *v, bool also_ab) {
  EngineImpl &P = *p_;
  check_id(P, id);
  CK(cudaStreamSynchronize(P.stream));
  auto &tr = P.tr[id];
  stage_upload(P, v);
  // 16-bit storage offset: the wet-cell mean of this upload, rounded to FP32
  double off = 0.0;
  if (storage16(P)) {
    off = (double)(float)stage_wet_mean(P);
    if (!std::isfinite(off)) off = 0.0;
  }
  if (!also_ab && off != tr.off) storage_reoffset(P, tr.TAB, tr.off, off);  // valuesAB stays
  tr.off = off;
  stage_pack(P, off, tr.T, also_ab ? tr.TAB : nullptr, tr.Tout);
  CK(cudaStreamSynchronize(P.stream));
}

void Engine::set_values_ab(int id, const double *v) {
  EngineImpl &P = *p_;
  check_id(P, id);
  CK(cudaStreamSynchronize(P.stream));
  if (!P.tr[id].TAB) throw std::invalid_argument("tracer has no valuesAB array (valuesAB := values each step)");
  stage_upload(P, v);
  stage_pack(P, P.tr[id].off, P.tr[id].TAB, nullptr, nullptr);
  CK(cudaStreamSynchronize(P.stream));
}

void Engine::get_values(int id, double *out) const {
  EngineImpl &P = *p_;
  check_id(P, id);
  CK(cudaStreamSynchronize(P.stream));
  stage_unpack(P, P.tr[id].T, P.tr[id].off);
  stage_download(P, out);
}

void Engine::get_values_ab(int id, double *out) const {
  EngineImpl &P = *p_;
  check_id(P, id);
  CK(cudaStreamSynchronize(P.stream));
  stage_unpack(P, P.tr[id].TAB ? P.tr[id].TAB : P.tr[id].T, P.tr[id].off);
  stage_download(P, out);
}

void Engine::set_rounding(int mode) {
  if (mode < 0 || mode > 1) throw std::invalid_argument("rounding mode must be 0 (nearest) or 1 (stochastic)");
  p_->sround = mode;
}
int Engine::rounding() const { return p_->sround; }
double Engine::storage_offset(int id) const {
  check_id(*p_, id);
  return p_->tr[id].off;
}

// host copy of the kernels' mix32 (lowbias32)
static uint32_t mix32_host(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
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

static void ensure_slots(EngineImpl &P, int n) {
  if (n <= P.slots) return;
  const size_t ns = (size_t)P.mesh.nod2D * P.S * P.r_bytes, es = (size_t)P.mesh.edge2D * P.S * P.r_bytes;
  if (!P.vflux) P.vflux = P.dalloc_bytes(es);
  // adf_h, lo and adf_v are interleaved by tracer (a batch of NT tracers uses stride
  // NT): one array each, reallocated for the larger batch
  CK(cudaStreamSynchronize(P.stream));
  P.dfree(P.adfh[0]);
  P.dfree(P.lo[0]);
  P.dfree(P.adfv[0]);
  char *ah = (char *)P.dalloc_bytes(n * es), *lo = (char *)P.dalloc_bytes(n * ns), *av = (char *)P.dalloc_bytes(n * ns);
  for (int t = 0; t < n; t++) {
    P.adfh[t] = ah + t * P.r_bytes;
    P.lo[t] = lo + t * P.r_bytes;
    P.adfv[t] = av + t * P.r_bytes;
  }
  for (int t = P.slots; t < n; t++) {
    P.rpm[t] = P.dalloc_bytes(2 * ns);
    P.gradn[t] = P.dalloc_bytes(2 * ns);
  }
  P.slots = n;
}

bool fused_step(const EngineImpl &P, const TracerScheme &sc, bool learned) {
  if (P.step_path != 0 || P.tiles.np <= 0 || learned) return false;
  if (P.prec != Precision::FP64 && P.prec != Precision::FP32) return false;
  if (sc.ver != 0 && sc.ver != 1) return false;  // QR4C and CDIFF: five-kernel path
  const TileLayout L = tile_layout(P.tplan, (unsigned)P.r_bytes, false, sc.hor != 0, sc.lim == 1);
  return L.bytes <= (unsigned)kTileSmemMax;
}

static void dispatch(EngineImpl &P, const TracerScheme &sc, int nt, const BatchPtrs &b, double dt) {
  if (P.mesh.nod2D <= 0) return;
  if (P.prec == Precision::FP64) (P.fma64 ? launch_batch_f64fma : launch_batch_f64)(P, sc, nt, b, dt);
  else launch_batch_f32(P, sc, nt, b, dt);
  CK(cudaGetLastError());
}

// Tracers are advanced in batches of up to kBatchMax consecutive tracers with
// the same scheme; a batch shares the edge volume fluxes, the geometry loads
// and every geometry-only division.
static void run_batch(EngineImpl &P, int first, int nt, double dt, bool refresh_ab) {
  ensure_slots(P, nt);
  BatchPtrs b;
  for (int t = 0; t < nt; t++) {
    auto &tr = P.tr[first + t];
    b.T[t] = tr.T;
    if (!refresh_ab && !tr.TAB) throw std::invalid_argument("tracer has no valuesAB array: advance with valuesAB := values");
    b.TAB[t] = refresh_ab ? tr.T : tr.TAB;
    b.T_out[t] = tr.Tout;
    b.adf_h[t] = P.adfh[t];
    b.adf_v[t] = P.adfv[t];
    b.lo[t] = P.lo[t];
    b.rpm[t] = P.rpm[t];
    b.gradn[t] = P.gradn[t];
    if (learned_active(P) && tr.sch.hor == 1) learned_slot_buffers(P, t, &b.feat[t], &b.fscale[t]);
    b.off[t] = tr.off;
    b.seed[t] = mix32_host(P.sround_seed ^ mix32_host((uint32_t)(first + t) * 0x9e3779b9u + tr.nstep));
    tr.nstep++;
  }
  b.sround = storage16(P) ? P.sround : 0;
  // the velocity only changes through set_velocity: the first launch after it
  // stores the edge volume fluxes, later ones load them
  b.vflux = P.vflux;
  b.vflux_mode = P.vflux_valid ? 2 : 1;
  dispatch(P, P.tr[first].sch, nt, b, dt);
  P.vflux_valid = true;
  for (int t = 0; t < nt; t++) std::swap(P.tr[first + t].T, P.tr[first + t].Tout);
}

static bool same_scheme(const TracerScheme &a, const TracerScheme &b) {
  return a.hor == b.hor && a.ver == b.ver && a.lim == b.lim && a.ph == b.ph && a.pv == b.pv;
}

// batch sizes the engine launches: 4, 2 or 1 tracers
static int batch_size(const EngineImpl &P, int first) {
  int run = 1;
  while (first + run < (int)P.tr.size() && run < kBatchMax && same_scheme(P.tr[first].sch, P.tr[first + run].sch)) run++;
  return run >= 4 ? 4 : (run >= 2 ? 2 : 1);
}

int Engine::launches_per_step() const {
  const EngineImpl &P = *p_;
  int n = 0;
  for (int i = 0; i < (int)P.tr.size();) {
    const int nt = batch_size(P, i);
    if (fused_step(P, P.tr[i].sch, learned_active(P) && P.tr[i].sch.hor == 1)) n += nt;
    else n += (P.tr[i].sch.lim == 1 ? 4 : 3) + (P.tr[i].sch.hor != 0 ? 1 : 0);
    i += nt;
  }
  return n;
}

void Engine::set_step_path(int path) {
  if (path < 0 || path > 1) throw std::invalid_argument("step path must be 0 (fused where possible) or 1 (five kernels)");
  p_->step_path = path;
}
int Engine::step_path() const { return p_->step_path; }
bool Engine::fused(int id) const {
  check_id(*p_, id);
  return fused_step(*p_, p_->tr[id].sch, learned_active(*p_) && p_->tr[id].sch.hor == 1);
}
int Engine::tile_count() const { return p_->tiles.np; }
void Engine::set_patch_size(int owned) {
  if (owned < 1) throw std::invalid_argument("patch size must be at least one owned node");
  CK(cudaStreamSynchronize(p_->stream));
  build_tiles(*p_, edge_slot_order(p_->mesh), owned);
  CK(cudaStreamSynchronize(p_->stream));
}
double Engine::tile_node_ratio() const { return p_->tplan.node_ratio; }

bool Engine::step_io(double dt, bool refresh_ab, const double *const *in, double *const *out) {
  EngineImpl &P = *p_;
  const int ntr = (int)P.tr.size();
  const size_t bytes = sizeof(double) * (size_t)(P.mesh.nl - 1) * P.mesh.nod2D;
  if (P.prec != Precision::FP64 && P.prec != Precision::FP32) return false;
  for (int t = 0; t < ntr; t++) {
    if (in && in[t] && !host_range_pinned(in[t], bytes)) return false;
    if (out && out[t] && !host_range_pinned(out[t], bytes)) return false;
    if (!refresh_ab && !P.tr[t].TAB) return false;
  }
  CK(cudaStreamSynchronize(P.stream));
  if (!P.io_h2d) {
    CK(cudaStreamCreateWithFlags(&P.io_h2d, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&P.io_d2h, cudaStreamNonBlocking));
  }
  while ((int)P.io_in.size() < ntr) {
    P.io_in.push_back(P.dalloc<double>(bytes / sizeof(double)));
    P.io_out.push_back(P.dalloc<double>(bytes / sizeof(double)));
    cudaEvent_t a, b;
    CK(cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
    P.io_ev_in.push_back(a);
    P.io_ev_out.push_back(b);
  }
  // every input copy is queued at once on the H2D stream; the compute stream
  // takes each tracer as soon as its copy lands, and the D2H stream takes
  // each new field as soon as its step is done
  for (int t = 0; t < ntr; t++)
    if (in && in[t]) {
      CK(cudaMemcpyAsync(P.io_in[t], in[t], bytes, cudaMemcpyHostToDevice, P.io_h2d));
      CK(cudaEventRecord(P.io_ev_in[t], P.io_h2d));
    }
  for (int t = 0; t < ntr; t++) {
    auto &tr = P.tr[t];
    if (in && in[t]) {
      CK(cudaStreamWaitEvent(P.stream, P.io_ev_in[t], 0));
      pack_from(P, P.io_in[t], P.stream, tr.T, tr.TAB, tr.Tout);
    }
    run_batch(P, t, 1, dt, refresh_ab);
    if (out && out[t]) {
      unpack_to(P, tr.T, P.io_out[t], P.stream);
      CK(cudaEventRecord(P.io_ev_out[t], P.stream));
      CK(cudaStreamWaitEvent(P.io_d2h, P.io_ev_out[t], 0));
      CK(cudaMemcpyAsync(out[t], P.io_out[t], bytes, cudaMemcpyDeviceToHost, P.io_d2h));
    }
  }
  CK(cudaStreamSynchronize(P.stream));
  CK(cudaStreamSynchronize(P.io_d2h));
  CK(cudaStreamSynchronize(P.io_h2d));
  return true;
}

void Engine::step_tracer(int id, double dt, bool refresh_ab) {
  check_id(*p_, id);
  run_batch(*p_, id, 1, dt, refresh_ab);
}

void Engine::step(double dt, bool refresh_ab) {
  for (int i = 0; i < (int)p_->tr.size();) {
    const int nt = batch_size(*p_, i);
    run_batch(*p_, i, nt, dt, refresh_ab);
    i += nt;
  }
}

size_t Engine::step_scratch_doubles() const {
  const EngineImpl &P = *p_;
  auto up = [](size_t n) { return (n + 31) / 32 * 32; };  // 256-byte pieces
  const size_t es = up((size_t)P.mesh.edge2D * P.S), ns = up((size_t)P.mesh.nod2D * P.S);
  return 2 * es + 6 * ns;
}

void Engine::step_with_scratch(int id, const double *T, const double *TAB, double *T_out, double dt, double *scratch,
                               size_t scratch_doubles) {
  EngineImpl &P = *p_;
  check_id(P, id);
  if (P.prec != Precision::FP64) throw std::invalid_argument("the allocation-free step runs the FP64 engine only");
  if (scratch_doubles < step_scratch_doubles()) throw std::length_error("scratch too small for this mesh");
  auto up = [](size_t n) { return (n + 31) / 32 * 32; };
  const size_t es = up((size_t)P.mesh.edge2D * P.S), ns = up((size_t)P.mesh.nod2D * P.S);
  BatchPtrs b;
  b.T[0] = T;
  b.TAB[0] = TAB;
  b.T_out[0] = T_out;
  b.vflux = scratch;
  b.adf_h[0] = scratch + es;
  b.adf_v[0] = scratch + 2 * es;
  b.lo[0] = scratch + 2 * es + ns;
  b.rpm[0] = scratch + 2 * es + 2 * ns;  // 2 ns
  b.gradn[0] = scratch + 2 * es + 4 * ns;
  dispatch(P, P.tr[id].sch, 1, b, dt);
  CK(cudaStreamSynchronize(P.stream));
}

const char *const *Engine::kernel_kind_names(int *n) {
  static const char *const names[KK_COUNT] = {"k_edge", "k_col1", "k_col2", "k_col3", "k_grad", "k_tile", "k_vflux"};
  *n = KK_COUNT;
  return names;
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

void Engine::volume_sum(int id, double out[2]) const {
  EngineImpl &P = *p_;
  check_id(P, id);
  CK(cudaStreamSynchronize(P.stream));
  if (P.prec == Precision::FP64) volume_sum_f64(P, P.tr[id].T, out);
  else volume_sum_f32(P, P.tr[id].T, P.tr[id].off, out);
}

void Engine::stats(int id, double out[4]) const {
  EngineImpl &P = *p_;
  check_id(P, id);
  CK(cudaStreamSynchronize(P.stream));
  tracer_stats(P, P.tr[id].T, P.tr[id].off, out);
}

}  // namespace fesom
