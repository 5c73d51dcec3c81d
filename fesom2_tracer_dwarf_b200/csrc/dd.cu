// Domain-decomposed tracer step (see dd.hpp).
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>

#include "dd.hpp"
#include "engine_impl.hpp"

namespace fesom {

namespace {

template <typename TS>
__global__ void k_halo_pack(const TS *__restrict__ T, const int *__restrict__ nodes, int n, int L, int S,
                            double *__restrict__ out) {
  const long long total = (long long)n * L;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / L), k = (int)(q - (long long)i * L);
    out[q] = (double)T[(size_t)nodes[i] * S + k];
  }
}

template <typename TS>
__global__ void k_halo_unpack(TS *__restrict__ T, const int *__restrict__ nodes, int n, int L, int S,
                              const double *__restrict__ in) {
  const long long total = (long long)n * L;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / L), k = (int)(q - (long long)i * L);
    T[(size_t)nodes[i] * S + k] = (TS)in[q];
  }
}

int grid_for(long long items) {
  return (int)std::max<long long>(1, std::min<long long>((items + 255) / 256, 148LL * 16));
}

}  // namespace

struct Decomposition::Impl {
  int nparts = 0, rings = 0, L = 0, nod2D = 0, elem2D = 0;
  Precision prec = Precision::FP64;
  std::vector<MeshPart> parts;
  std::vector<std::unique_ptr<Engine>> eng;
  // per local part and peer part: device lists of local node ids
  std::vector<std::vector<int *>> send_d, recv_d;
  std::vector<std::vector<int>> send_n, recv_n;
  double *stage = nullptr;
  size_t stage_cap = 0;

  ~Impl() {
    for (auto &v : send_d)
      for (int *p : v) cudaFree(p);
    for (auto &v : recv_d)
      for (int *p : v) cudaFree(p);
    cudaFree(stage);
  }
  void *values_ptr(int i, int id) {
    EngineImpl &E = *eng[i]->impl();
    if (id < 0 || id >= (int)E.tr.size()) throw std::out_of_range("decomposition: invalid tracer id");
    return E.tr[id].T;
  }
  int level_stride(int i) { return eng[i]->level_stride(); }
  double *staging(size_t doubles) {
    if (doubles > stage_cap) {
      CK(cudaFree(stage));
      stage = nullptr;
      CK(cudaMalloc(&stage, doubles * sizeof(double)));
      stage_cap = doubles;
    }
    return stage;
  }
};

Decomposition::Decomposition(const MeshHost &g, const std::vector<int> &node_part, int nparts,
                             const std::vector<int> &local_parts, int rings, Precision prec)
    : p_(new Impl) {
  if (prec != Precision::FP64 && prec != Precision::FP32)
    throw std::invalid_argument("domain decomposition runs the FP64 and FP32 engines");
  if (rings < 3) throw std::invalid_argument("domain decomposition needs at least 3 halo rings");
  if ((int)node_part.size() != g.nod2D) throw std::invalid_argument("one part per node expected");
  for (int q : node_part)
    if (q < 0 || q >= nparts) throw std::invalid_argument("node part outside [0, nparts)");
  {
    std::vector<int> seen(local_parts);
    std::sort(seen.begin(), seen.end());
    if (std::adjacent_find(seen.begin(), seen.end()) != seen.end())
      throw std::invalid_argument("a part is listed twice among the local parts");
  }
  Impl &P = *p_;
  P.nparts = nparts;
  P.rings = rings;
  P.L = g.nl - 1;
  P.nod2D = g.nod2D;
  P.elem2D = g.elem2D;
  P.prec = prec;
  // halos of every part (the exchange lists of a local part need its peers')
  std::vector<std::vector<int>> halo(nparts);
  for (int q = 0; q < nparts; q++) halo[q] = halo_nodes(g, node_part, q, rings);
  for (int p : local_parts) {
    if (p < 0 || p >= nparts) throw std::invalid_argument("local part outside [0, nparts)");
    P.parts.push_back(build_mesh_part(g, node_part, p, rings));
    const MeshPart &mp = P.parts.back();
    P.eng.push_back(std::make_unique<Engine>(mp.mesh, prec));
    std::vector<int> g2l(g.nod2D, -1);
    for (int i = 0; i < (int)mp.node_global.size(); i++) g2l[mp.node_global[i]] = i;
    std::vector<int *> sd(nparts, nullptr), rd(nparts, nullptr);
    std::vector<int> sn(nparts, 0), rn(nparts, 0);
    for (int q = 0; q < nparts; q++) {
      if (q == p) continue;
      std::vector<int> snd, rcv;
      for (int n : halo[q])
        if (node_part[n] == p) snd.push_back(g2l[n]);  // owned here, in q's halo
      for (int n : halo[p])
        if (node_part[n] == q) rcv.push_back(g2l[n]);  // in the halo here, owned by q
      for (int v : snd)
        if (v < 0 || v >= mp.owned) throw std::logic_error("decomposition: send node not owned");
      for (int v : rcv)
        if (v < mp.owned) throw std::logic_error("decomposition: receive node not in the halo");
      sn[q] = (int)snd.size();
      rn[q] = (int)rcv.size();
      if (!snd.empty()) {
        CK(cudaMalloc(&sd[q], snd.size() * sizeof(int)));
        CK(cudaMemcpy(sd[q], snd.data(), snd.size() * sizeof(int), cudaMemcpyHostToDevice));
      }
      if (!rcv.empty()) {
        CK(cudaMalloc(&rd[q], rcv.size() * sizeof(int)));
        CK(cudaMemcpy(rd[q], rcv.data(), rcv.size() * sizeof(int), cudaMemcpyHostToDevice));
      }
    }
    P.send_d.push_back(sd);
    P.recv_d.push_back(rd);
    P.send_n.push_back(sn);
    P.recv_n.push_back(rn);
  }
}

Decomposition::~Decomposition() = default;

int Decomposition::nparts() const { return p_->nparts; }
int Decomposition::num_local() const { return (int)p_->parts.size(); }
const MeshPart &Decomposition::part(int i) const { return p_->parts.at(i); }
Engine &Decomposition::engine(int i) { return *p_->eng.at(i); }

void Decomposition::allocate_tracers(int ntr) {
  for (auto &e : p_->eng) e->allocate_tracers(ntr, true);
}

void Decomposition::set_scheme(int id, const TracerScheme &s) {
  for (auto &e : p_->eng) e->set_scheme(id, s);
}

void Decomposition::set_velocity(const double *uv, const double *w) {
  Impl &P = *p_;
  const int L = P.L, nl = L + 1;
  for (size_t i = 0; i < P.parts.size(); i++) {
    const MeshPart &mp = P.parts[i];
    std::vector<double> luv((size_t)2 * L * mp.elem_global.size()), lw((size_t)nl * mp.node_global.size());
    for (size_t t = 0; t < mp.elem_global.size(); t++)
      std::copy_n(uv + (size_t)2 * L * mp.elem_global[t], 2 * L, &luv[(size_t)2 * L * t]);
    for (size_t n = 0; n < mp.node_global.size(); n++)
      std::copy_n(w + (size_t)nl * mp.node_global[n], nl, &lw[(size_t)nl * n]);
    P.eng[i]->set_velocity(luv.data(), lw.data());
  }
}

void Decomposition::set_values(int id, const double *v) {
  Impl &P = *p_;
  const int L = P.L;
  for (size_t i = 0; i < P.parts.size(); i++) {
    const MeshPart &mp = P.parts[i];
    std::vector<double> lv((size_t)L * mp.node_global.size());
    for (size_t n = 0; n < mp.node_global.size(); n++)
      std::copy_n(v + (size_t)L * mp.node_global[n], L, &lv[(size_t)L * n]);
    P.eng[i]->set_values(id, lv.data(), true);
  }
}

void Decomposition::get_values(int id, double *out) const {
  const Impl &P = *p_;
  const int L = P.L;
  for (size_t i = 0; i < P.parts.size(); i++) {
    const MeshPart &mp = P.parts[i];
    std::vector<double> lv((size_t)L * mp.node_global.size());
    P.eng[i]->get_values(id, lv.data());
    for (int n = 0; n < mp.owned; n++) std::copy_n(&lv[(size_t)L * n], L, out + (size_t)L * mp.node_global[n]);
  }
}

void Decomposition::step(double dt, bool refresh_ab) {
  for (auto &e : p_->eng) e->step(dt, refresh_ab);
}

void Decomposition::synchronize() const {
  for (auto &e : p_->eng) e->synchronize();
}

int Decomposition::transfer_nodes(int i, int peer, bool send) const {
  const Impl &P = *p_;
  if (i < 0 || i >= (int)P.parts.size() || peer < 0 || peer >= P.nparts) throw std::out_of_range("decomposition: part");
  return send ? P.send_n[i][peer] : P.recv_n[i][peer];
}

void Decomposition::pack(int i, int id, int peer, double *dev_out) {
  Impl &P = *p_;
  const int n = transfer_nodes(i, peer, true);
  if (n == 0) return;
  P.eng[i]->synchronize();
  const int S = P.level_stride(i);
  const long long items = (long long)n * P.L;
  if (P.prec == Precision::FP64)
    k_halo_pack<double><<<grid_for(items), 256>>>((const double *)P.values_ptr(i, id), P.send_d[i][peer], n, P.L, S, dev_out);
  else
    k_halo_pack<float><<<grid_for(items), 256>>>((const float *)P.values_ptr(i, id), P.send_d[i][peer], n, P.L, S, dev_out);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
}

void Decomposition::unpack(int i, int id, int peer, const double *dev_in) {
  Impl &P = *p_;
  const int n = transfer_nodes(i, peer, false);
  if (n == 0) return;
  P.eng[i]->synchronize();
  const int S = P.level_stride(i);
  const long long items = (long long)n * P.L;
  if (P.prec == Precision::FP64)
    k_halo_unpack<double><<<grid_for(items), 256>>>((double *)P.values_ptr(i, id), P.recv_d[i][peer], n, P.L, S, dev_in);
  else
    k_halo_unpack<float><<<grid_for(items), 256>>>((float *)P.values_ptr(i, id), P.recv_d[i][peer], n, P.L, S, dev_in);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
}

void Decomposition::exchange_local() {
  Impl &P = *p_;
  synchronize();
  std::vector<int> where(P.nparts, -1);
  for (int i = 0; i < (int)P.parts.size(); i++) where[P.parts[i].part] = i;
  const int ntr = P.eng.empty() ? 0 : P.eng[0]->num_tracers();
  for (int i = 0; i < (int)P.parts.size(); i++)
    for (int j = 0; j < (int)P.parts.size(); j++) {
      if (i == j) continue;
      const int from = P.parts[j].part, to = P.parts[i].part;
      const int n = P.send_n[j][to];
      if (n != P.recv_n[i][from]) throw std::logic_error("decomposition: transfer sizes disagree");
      if (n == 0) continue;
      double *buf = P.staging((size_t)n * P.L);
      for (int id = 0; id < ntr; id++) {
        pack(j, id, to, buf);
        unpack(i, id, from, buf);
      }
    }
}

}  // namespace fesom
