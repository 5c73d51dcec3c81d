// Multi-member batched stepping: one persistent cooperative launch per step
// (see batch.hpp).  FP32 tracers, geometry and arithmetic.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <sstream>
#include <stdexcept>

#include "advect_fused.cuh"
#include "batch.hpp"
#include "engine_impl.hpp"

namespace fesom {

namespace {

constexpr int kNT = 4;  // tracers per batch task

struct BatchTask {
  DMeshT<float> m;
  FusedArgs<float, float> a;
};

// Grid-wide barrier with a bounded wait: a block that waits longer than
// `limit` polls sets err and every block leaves the kernel.
struct GridBarrier {
  unsigned count;
  unsigned gen;
  int err;
  int pad;
};

__device__ __forceinline__ bool grid_sync(GridBarrier *b, unsigned nblocks, long long limit) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *vgen = &b->gen;
    volatile int *verr = &b->err;
    const unsigned g = *vgen;
    __threadfence();
    if (atomicAdd(&b->count, 1u) == nblocks - 1) {
      atomicExch(&b->count, 0u);
      __threadfence();
      atomicAdd(&b->gen, 1u);
    } else {
      long long it = 0;
      while (*vgen == g && *verr == 0) {
        if (++it > limit) {
          atomicExch(&b->err, 1);
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile int *)&b->err == 0;
}

enum { PH_GRAD = 0, PH_EDGE, PH_COL1, PH_COL2, PH_COL3, PH_COUNT };

constexpr size_t kTaskSmem = (sizeof(BatchTask) + 15) / 16 * 16;
size_t batch_smem() {
  return kTaskSmem + std::max(smem_col_staged<float>(kNT, 2), smem_col_staged<float>(kNT, 0));
}

// prefix: PH_COUNT rows of (ntasks + 1) running totals of each task's blocks;
// wave_first: (nwaves + 1) first task of each wave (tasks are wave-major).
// MINB: resident 256-thread blocks per SM the register budget is cut for
template <int HOR, int VER, int LIM, int MINB>
__global__ void __launch_bounds__(256, MINB)
    k_batch_step(BatchTask *tasks, const int *prefix, int ntasks, const int *wave_first, int nwaves, GridBarrier *bar,
                 long long spin_limit, int refresh_ab) {
  extern __shared__ __align__(16) int smem[];
  BatchTask &st = *reinterpret_cast<BatchTask *>(smem);
  int *work = smem + kTaskSmem / sizeof(int);
  const unsigned nb = gridDim.x;
  for (int w = 0; w < nwaves; w++) {
    const int t0 = wave_first[w], t1 = wave_first[w + 1];
    for (int ph = 0; ph < PH_COUNT; ph++) {
      if (ph == PH_GRAD && HOR == HOR_UPW1) continue;
      if (ph == PH_COL2 && LIM != LIM_FCT) continue;
      const int *pre = prefix + ph * (ntasks + 1);
      const int base = pre[t0], total = pre[t1] - base;
      int task = t0, loaded = -1;
      for (int it = blockIdx.x; it < total; it += nb) {
        const int g = base + it;
        while (pre[task + 1] <= g) task++;
        __syncthreads();  // the previous item is done with shared memory
        if (task != loaded) {
          for (int q = threadIdx.x; q < (int)(sizeof(BatchTask) / sizeof(int)); q += blockDim.x)
            reinterpret_cast<int *>(&st)[q] = reinterpret_cast<const int *>(&tasks[task])[q];
          loaded = task;
          __syncthreads();
        }
        const int vblk = g - pre[task];
        switch (ph) {
          case PH_GRAD: grad_block<float, float, kNT>(st.m, st.a, vblk, work); break;
          case PH_EDGE: edge_block<float, float, kNT, HOR, LIM>(st.m, st.a, vblk, work); break;
          case PH_COL1: col1_block<float, float, kNT, VER, LIM>(st.m, st.a, vblk, work); break;
          case PH_COL2: col2_block<float, float, kNT>(st.m, st.a, vblk, work); break;
          default: col3_block<float, float, kNT, LIM>(st.m, st.a, vblk, work); break;
        }
      }
      if (!grid_sync(bar, nb, spin_limit)) return;
    }
  }
  // the new values become the current ones for the next launch
  if (blockIdx.x == 0) {
    for (int t = threadIdx.x; t < ntasks * kNT; t += blockDim.x) {
      FusedArgs<float, float> &a = tasks[t / kNT].a;
      const int q = t % kNT;
      float *old = const_cast<float *>(a.T[q]);
      a.T[q] = a.T_out[q];
      a.T_out[q] = old;
      if (refresh_ab) a.TAB[q] = a.T[q];
    }
  }
}

using BatchKernel = void (*)(BatchTask *, const int *, int, const int *, int, GridBarrier *, long long, int);

template <int MINB>
BatchKernel pick_kernel_b(const TracerScheme &s) {
  if (s.hor == HOR_MUSCL && s.ver == VER_PPM && s.lim == LIM_FCT) return k_batch_step<HOR_MUSCL, VER_PPM, LIM_FCT, MINB>;
  if (s.hor == HOR_MUSCL && s.ver == VER_PPM && s.lim == LIM_NONE) return k_batch_step<HOR_MUSCL, VER_PPM, LIM_NONE, MINB>;
  if (s.hor == HOR_UPW1 && s.ver == VER_UPW1 && s.lim == LIM_FCT) return k_batch_step<HOR_UPW1, VER_UPW1, LIM_FCT, MINB>;
  if (s.hor == HOR_UPW1 && s.ver == VER_UPW1 && s.lim == LIM_NONE) return k_batch_step<HOR_UPW1, VER_UPW1, LIM_NONE, MINB>;
  return nullptr;
}

// the register budget follows the resident threads per SM the tile asks for
BatchKernel pick_kernel(const TracerScheme &s, int threads = 256, int blocks_per_sm = 2) {
  const int minb = std::max(2, std::min(7, (threads * blocks_per_sm + 255) / 256));
  if (minb == 7) return pick_kernel_b<7>(s);
  if (minb == 6) return pick_kernel_b<6>(s);
  if (minb == 5) return pick_kernel_b<5>(s);
  if (minb == 4) return pick_kernel_b<4>(s);
  if (minb == 3) return pick_kernel_b<3>(s);
  return pick_kernel_b<2>(s);
}

// One persistent launch per phase: the launch walks the blocks of every task
// of a wave for one phase (grid = SMs x resident blocks of that kernel), so
// each phase keeps the register budget of its standalone kernel and the task
// descriptors sit in the kernel's parameter space (constant bank) instead of
// shared memory.  Kernel boundaries order the phases.
constexpr int kPackTasks = 16;
struct PhasePack {
  int ntasks;
  int prefix[kPackTasks + 1];  // running totals of the tasks' blocks of this phase
  BatchTask t[kPackTasks];
};
static_assert(sizeof(PhasePack) <= 32000, "phase pack must fit the kernel parameter space");

// resident 256-thread blocks per SM each phase kernel's register budget is
// cut for (build-time knobs).  One block fewer than the standalone FP32
// kernels: the task lookup and the descriptor loads from parameter space
// need registers of their own.  Measured on the 48-tracer x 8-member
// ensemble: 424 ms per step against 456 with the standalone budgets.
// (Copying the descriptor into shared memory instead was slower still:
// 491-525 ms, the pointers then occupy registers.)
#ifndef FESOM_PHASE_MINB_GRAD
#define FESOM_PHASE_MINB_GRAD FESOM_MINB32_GRAD
#endif
#ifndef FESOM_PHASE_MINB_EDGE
#define FESOM_PHASE_MINB_EDGE 5
#endif
#ifndef FESOM_PHASE_MINB_COL1
#define FESOM_PHASE_MINB_COL1 6
#endif
#ifndef FESOM_PHASE_MINB_COL2
#define FESOM_PHASE_MINB_COL2 6
#endif
#ifndef FESOM_PHASE_MINB_COL3
#define FESOM_PHASE_MINB_COL3 6
#endif
template <int PH>
struct PhaseBudget {
  static constexpr int v = PH == PH_GRAD   ? FESOM_PHASE_MINB_GRAD
                           : PH == PH_EDGE ? FESOM_PHASE_MINB_EDGE
                           : PH == PH_COL1 ? FESOM_PHASE_MINB_COL1
                           : PH == PH_COL2 ? FESOM_PHASE_MINB_COL2
                                           : FESOM_PHASE_MINB_COL3;
};

template <int PH, int HOR, int VER, int LIM>
__global__ void __launch_bounds__(kThreads, PhaseBudget<PH>::v) k_batch_phase(const __grid_constant__ PhasePack p) {
  extern __shared__ __align__(16) int smem[];
  const int total = p.prefix[p.ntasks];
  int task = 0;
  for (int g = blockIdx.x; g < total; g += gridDim.x) {
    while (p.prefix[task + 1] <= g) task++;
    if (g != (int)blockIdx.x) __syncthreads();  // the previous item is done with shared memory
    const int vblk = g - p.prefix[task];
    const BatchTask &st = p.t[task];
    if (PH == PH_GRAD) grad_block<float, float, kNT>(st.m, st.a, vblk, smem);
    else if (PH == PH_EDGE) edge_block<float, float, kNT, HOR, LIM>(st.m, st.a, vblk, smem);
    else if (PH == PH_COL1) col1_block<float, float, kNT, VER, LIM>(st.m, st.a, vblk, smem);
    else if (PH == PH_COL2) col2_block<float, float, kNT>(st.m, st.a, vblk, smem);
    else col3_block<float, float, kNT, LIM>(st.m, st.a, vblk, smem);
  }
}

// dynamic shared memory of each phase: that of its standalone kernel
size_t phase_smem(int ph) {
  switch (ph) {
    case PH_GRAD:
    case PH_EDGE: return smem_edge();
    case PH_COL1: return StageIncidence<float>::col1 ? smem_col_staged<float>(kNT, 2) : smem_col<float>(kNT, 2);
    case PH_COL2: return StageIncidence<float>::col2 ? smem_col_staged<float>(kNT, 2) : smem_col<float>(kNT, 2);
    default: return StageIncidence<float>::col3 ? smem_col_staged<float>(kNT, 0) : smem_col<float>(kNT, 0);
  }
}

struct PhaseKernel {
  const void *fn = nullptr;
  void (*launch)(const PhasePack &, int, size_t, cudaStream_t) = nullptr;
};

template <int PH, int HOR, int VER, int LIM>
void launch_phase(const PhasePack &p, int grid, size_t smem, cudaStream_t st) {
  k_batch_phase<PH, HOR, VER, LIM><<<grid, kThreads, smem, st>>>(p);
}

template <int HOR, int VER, int LIM>
void phase_kernels_t(PhaseKernel *k) {
  k[PH_GRAD] = {(const void *)k_batch_phase<PH_GRAD, HOR, VER, LIM>, launch_phase<PH_GRAD, HOR, VER, LIM>};
  k[PH_EDGE] = {(const void *)k_batch_phase<PH_EDGE, HOR, VER, LIM>, launch_phase<PH_EDGE, HOR, VER, LIM>};
  k[PH_COL1] = {(const void *)k_batch_phase<PH_COL1, HOR, VER, LIM>, launch_phase<PH_COL1, HOR, VER, LIM>};
  if (LIM == LIM_FCT)
    k[PH_COL2] = {(const void *)k_batch_phase<PH_COL2, HOR, VER, LIM>, launch_phase<PH_COL2, HOR, VER, LIM>};
  k[PH_COL3] = {(const void *)k_batch_phase<PH_COL3, HOR, VER, LIM>, launch_phase<PH_COL3, HOR, VER, LIM>};
}

bool phase_kernels(const TracerScheme &s, PhaseKernel *k) {
  for (int ph = 0; ph < PH_COUNT; ph++) k[ph] = PhaseKernel{};
  if (s.hor == HOR_MUSCL && s.ver == VER_PPM && s.lim == LIM_FCT) phase_kernels_t<HOR_MUSCL, VER_PPM, LIM_FCT>(k);
  else if (s.hor == HOR_MUSCL && s.ver == VER_PPM && s.lim == LIM_NONE) phase_kernels_t<HOR_MUSCL, VER_PPM, LIM_NONE>(k);
  else if (s.hor == HOR_UPW1 && s.ver == VER_UPW1 && s.lim == LIM_FCT) phase_kernels_t<HOR_UPW1, VER_UPW1, LIM_FCT>(k);
  else if (s.hor == HOR_UPW1 && s.ver == VER_UPW1 && s.lim == LIM_NONE) phase_kernels_t<HOR_UPW1, VER_UPW1, LIM_NONE>(k);
  else return false;
  return true;
}

// Edge volume fluxes of a member's velocity (the values k_edge computes), so
// that every batch task loads them (vflux_mode 2) instead of recomputing them.
__global__ void __launch_bounds__(256) k_batch_vflux(DMeshT<float> m, const float *vel, float *vflux) {
  const size_t n = (size_t)m.E * m.S;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(q / m.S), k = (int)(q - (size_t)s * m.S);
    if (k >= m.edge_lev[s].y) continue;
    vflux[q] = edge_vflux(m, edge_ctx(m, s), vel, k);
  }
}

// test kernel: a barrier that waits for one block more than the grid has,
// so it must give up after `limit` polls and report it
__global__ void k_barrier_timeout(GridBarrier *bar, long long limit, int *status) {
  const bool ok = grid_sync(bar, gridDim.x + 1, limit);
  if (blockIdx.x == 0 && threadIdx.x == 0) *status = ok ? 0 : 1;
}

}  // namespace

struct BatchImpl {
  std::vector<std::unique_ptr<Engine>> members;
  std::vector<int> ntr;
  std::vector<double> dt;
  TracerScheme sch;
  bool refresh_ab = true;
  bool configured = false;
  BatchTile tile;
  cudaStream_t stream = nullptr;
  int sms = 0;

  // device state
  BatchTask *d_tasks = nullptr;
  int *d_prefix = nullptr, *d_wave_first = nullptr;
  GridBarrier *d_bar = nullptr;
  int ntasks = 0, nwaves = 0;
  std::vector<void *> work;  // work arrays of every (member, wave slot)
  long long work_bytes = 0;
  BatchKernel kernel = nullptr;
  int grid = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  long long spin_limit = 1ll << 24;
  // separate per-member launches captured as one graph of two steps
  cudaGraph_t sep_graph = nullptr;
  cudaGraphExec_t sep_exec = nullptr;
  std::vector<cudaEvent_t> sep_events;

  // step path: 0 one cooperative launch per step, 1 one persistent launch
  // per phase and wave, 2 the members' own launches
  int mode = 1;
  // learned antidiffusive flux on every member (path 2 only: the member
  // engines run the MLP between their edge and column kernels; the
  // persistent paths' phase kernels have no MLP phase)
  bool learned = false;
  // work-array slots, host task table (wave-major) and blocks per phase
  struct Slot {
    void *adfh[kNT], *adfv[kNT], *lo[kNT], *rpm[kNT], *gradn[kNT];
  };
  std::vector<std::vector<Slot>> slots;
  std::vector<BatchTask> tasks;
  std::vector<int> task_slot;  // work-array slot of each task
  std::vector<int> wave_first;
  std::vector<std::vector<int>> nblk;
  PhaseKernel phk[PH_COUNT];
  int phgrid[PH_COUNT] = {0, 0, 0, 0, 0};
  // phase launches of two steps captured as a graph; valid while the first
  // tracer's current buffer is the one seen at capture
  cudaGraph_t ph_graph = nullptr;
  cudaGraphExec_t ph_exec = nullptr;
  const void *ph_key = nullptr;
  // the phase path runs the tasks of each work-array slot on its own stream
  // (slots are independent), so that different phase kernels share the SMs
  static constexpr int kPhaseStreams = 4;
  cudaStream_t ph_streams[kPhaseStreams] = {};
  cudaEvent_t ph_fork = nullptr, ph_join[kPhaseStreams] = {};

  ~BatchImpl() {
    release();
    release_sep();
    if (stream) cudaStreamDestroy(stream);
    for (int i = 0; i < kPhaseStreams; i++) {
      if (ph_streams[i]) cudaStreamDestroy(ph_streams[i]);
      if (ph_join[i]) cudaEventDestroy(ph_join[i]);
    }
    if (ph_fork) cudaEventDestroy(ph_fork);
  }
  void release_sep() {
    if (sep_exec) cudaGraphExecDestroy(sep_exec);
    if (sep_graph) cudaGraphDestroy(sep_graph);
    sep_exec = nullptr;
    sep_graph = nullptr;
    for (auto e : sep_events) cudaEventDestroy(e);
    sep_events.clear();
  }

  void release_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
    if (ph_exec) cudaGraphExecDestroy(ph_exec);
    if (ph_graph) cudaGraphDestroy(ph_graph);
    ph_exec = nullptr;
    ph_graph = nullptr;
    ph_key = nullptr;
  }
  void release() {
    release_graph();
    for (void *w : work) cudaFree(w);
    work.clear();
    work_bytes = 0;
    slots.clear();
    tasks.clear();
    if (d_tasks) cudaFree(d_tasks);
    if (d_prefix) cudaFree(d_prefix);
    if (d_wave_first) cudaFree(d_wave_first);
    if (d_bar) cudaFree(d_bar);
    d_tasks = nullptr;
    d_prefix = d_wave_first = nullptr;
    d_bar = nullptr;
  }
  void *walloc(size_t bytes) {
    void *p = nullptr;
    CK(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
    work.push_back(p);
    work_bytes += (long long)bytes;
    return p;
  }
};

namespace {

// Every member's edge volume fluxes, computed once per velocity (the member
// engine's own cache: a new velocity invalidates it).
void refresh_vflux(BatchImpl &B) {
  for (auto &mem : B.members) {
    EngineImpl &P = *mem->impl();
    if (P.vflux && P.vflux_valid) continue;
    if (!P.vflux) P.vflux = P.dalloc_bytes((size_t)P.mesh.edge2D * P.S * P.r_bytes);
    const size_t n = (size_t)P.dm32.E * P.dm32.S;
    const int grid = (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)B.sms * 16));
    mem->synchronize();
    k_batch_vflux<<<grid, 256, 0, B.stream>>>(P.dm32, (const float *)P.vel, (float *)P.vflux);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(B.stream));
    P.vflux_valid = true;
  }
}

// The task table (wave-major) from the members' current tracer buffers and
// the batch's work-array slots.
void make_tasks(BatchImpl &B) {
  const int M = (int)B.members.size(), W = B.tile.wave;
  B.tasks.clear();
  B.task_slot.clear();
  B.wave_first.clear();
  B.nblk.assign(PH_COUNT, std::vector<int>());
  for (int w = 0; w < B.nwaves; w++) {
    B.wave_first.push_back((int)B.tasks.size());
    for (int m = 0; m < M; m++) {
      EngineImpl &P = *B.members[m]->impl();
      for (int b = w * W; b < std::min((w + 1) * W, B.ntr[m] / kNT); b++) {
        const BatchImpl::Slot &sl = B.slots[m][b % W];
        BatchTask T{};
        T.m = P.dm32;
        FusedArgs<float, float> &a = T.a;
        for (int t = 0; t < kNT; t++) {
          auto &tr = P.tr[b * kNT + t];
          a.T[t] = (const float *)tr.T;
          a.TAB[t] = (const float *)(B.refresh_ab ? tr.T : tr.TAB);
          a.T_out[t] = (float *)tr.Tout;
          a.adf_h[t] = (float *)sl.adfh[t];
          a.adf_v[t] = (float *)sl.adfv[t];
          a.lo[t] = (float *)sl.lo[t];
          a.rpm[t] = (float *)sl.rpm[t];
          a.gradn[t] = (float *)sl.gradn[t];
        }
        a.vflux = (float *)P.vflux;
        a.vflux_mode = 2;
        a.vel = (const float *)P.vel;
        a.W = (const float *)P.W;
        a.dt = (float)B.dt[m];
        a.ph = (float)B.sch.ph;
        a.pv = (float)B.sch.pv;
        B.tasks.push_back(T);
        B.task_slot.push_back(b % W);
        B.nblk[PH_GRAD].push_back(B.sch.hor == HOR_UPW1 ? 0 : P.dm32.grad_sched.nblk);
        B.nblk[PH_EDGE].push_back(P.dm32.edge_sched.nblk);
        B.nblk[PH_COL1].push_back(P.dm32.node_sched.nblk);
        B.nblk[PH_COL2].push_back(B.sch.lim == LIM_FCT ? P.dm32.node_sched.nblk : 0);
        B.nblk[PH_COL3].push_back(P.dm32.node_sched.nblk);
      }
    }
  }
  B.wave_first.push_back((int)B.tasks.size());
  B.ntasks = (int)B.tasks.size();
}

}  // namespace

Batch::Batch() : p_(new BatchImpl) {
  CK(cudaStreamCreateWithFlags(&p_->stream, cudaStreamNonBlocking));
  for (int i = 0; i < BatchImpl::kPhaseStreams; i++) {
    CK(cudaStreamCreateWithFlags(&p_->ph_streams[i], cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&p_->ph_join[i], cudaEventDisableTiming));
  }
  CK(cudaEventCreateWithFlags(&p_->ph_fork, cudaEventDisableTiming));
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&p_->sms, cudaDevAttrMultiProcessorCount, dev));
}
Batch::~Batch() { delete p_; }

int Batch::add_member(const MeshHost &mesh, int ntracers) {
  if (ntracers < kNT || ntracers % kNT) throw std::invalid_argument("batch members need a multiple of 4 tracers");
  if (p_->learned)
    throw std::logic_error("batch: switch the learned flux off (tracer_batch_learn_set) before adding members");
  p_->members.emplace_back(new Engine(mesh, Precision::FP32));
  p_->members.back()->allocate_tracers(ntracers, false);  // valuesAB := values
  p_->ntr.push_back(ntracers);
  p_->configured = false;
  return (int)p_->members.size() - 1;
}
int Batch::num_members() const { return (int)p_->members.size(); }
Engine &Batch::member(int i) {
  if (i < 0 || i >= num_members()) throw std::out_of_range("invalid member " + std::to_string(i));
  return *p_->members[i];
}

void Batch::configure(const TracerScheme &sch, const std::vector<double> &dt, bool refresh_ab) {
  BatchImpl &B = *p_;
  if ((int)dt.size() != num_members()) throw std::invalid_argument("one dt per member");
  if (!pick_kernel(sch)) throw std::invalid_argument("the batched step supports MUSCL+PPM and UPW1+UPW1, with or without FCT");
  if (!refresh_ab) throw std::invalid_argument("the batched step advances with valuesAB := values");
  B.sch = sch;
  B.dt = dt;
  B.refresh_ab = refresh_ab;
  for (int m = 0; m < num_members(); m++)
    for (int t = 0; t < B.ntr[m]; t++) B.members[m]->set_scheme(t, sch);
  B.configured = true;
  set_tile(B.tile);
}

BatchTile Batch::tile() const { return p_->tile; }
long long Batch::work_bytes() const { return p_->work_bytes; }
bool Batch::graph_captured() const {
  if (p_->mode == 2) return p_->sep_exec != nullptr;
  return p_->mode == 1 ? p_->ph_exec != nullptr : p_->graph_exec != nullptr;
}

long long Batch::wet_cells() const {
  long long c = 0;
  for (int m = 0; m < num_members(); m++) c += p_->members[m]->mesh().wet_cells() * p_->ntr[m];
  return c;
}

void Batch::set_tile(const BatchTile &tile) {
  BatchImpl &B = *p_;
  if (!B.configured) throw std::runtime_error("configure the batch first");
  if (tile.threads < 64 || tile.threads > 256 || tile.threads % 32) throw std::invalid_argument("threads per block in {64..256}");
  if (tile.wave < 1) throw std::invalid_argument("wave must be >= 1");
  for (auto &m : B.members) m->synchronize();
  CK(cudaStreamSynchronize(B.stream));
  B.release();
  B.tile = tile;
  B.kernel = pick_kernel(B.sch, tile.threads, tile.blocks_per_sm);
  phase_kernels(B.sch, B.phk);
  const size_t smem = batch_smem();
  CK(cudaFuncSetAttribute(B.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, B.kernel, tile.threads, smem));
  if (occ < 1) throw std::runtime_error("batched step kernel cannot be resident");
  B.tile.blocks_per_sm = std::min(tile.blocks_per_sm, occ);
  B.grid = B.sms * B.tile.blocks_per_sm;

  const int M = num_members();
  for (int m = 0; m < M; m++) B.members[m]->set_cells_per_block(tile.cells_per_block);

  // work arrays per (member, wave slot) and the task table, wave-major
  int max_batches = 0;
  for (int m = 0; m < M; m++) max_batches = std::max(max_batches, B.ntr[m] / kNT);
  const int W = std::min(tile.wave, max_batches);
  {
    size_t need = 0, free_b = 0, total_b = 0;
    for (int m = 0; m < M; m++) {
      const EngineImpl &P = *B.members[m]->impl();
      const size_t ns = (size_t)P.mesh.nod2D * P.S * sizeof(float), es = (size_t)P.mesh.edge2D * P.S * sizeof(float);
      need += (size_t)std::min(W, B.ntr[m] / kNT) * kNT * (es + 6 * ns);
    }
    CK(cudaMemGetInfo(&free_b, &total_b));
    if (need > free_b / 10 * 9)
      throw std::runtime_error("not enough device memory for " + std::to_string(W) + " tracer batches in flight");
  }
  B.tile.wave = W;
  B.nwaves = (max_batches + W - 1) / W;
  B.slots.assign(M, std::vector<BatchImpl::Slot>(W));
  for (int m = 0; m < M; m++) {
    EngineImpl &P = *B.members[m]->impl();
    const size_t ns = (size_t)P.mesh.nod2D * P.S * sizeof(float), es = (size_t)P.mesh.edge2D * P.S * sizeof(float);
    const int used = std::min(W, B.ntr[m] / kNT);
    for (int j = 0; j < used; j++) {
      BatchImpl::Slot &sl = B.slots[m][j];
      // adf_h, lo and adf_v interleaved by tracer (stride kNT)
      char *ah = (char *)B.walloc(kNT * es), *lo = (char *)B.walloc(kNT * ns), *av = (char *)B.walloc(kNT * ns);
      for (int t = 0; t < kNT; t++) {
        sl.adfh[t] = ah + t * sizeof(float);
        sl.adfv[t] = av + t * sizeof(float);
        sl.lo[t] = lo + t * sizeof(float);
        sl.rpm[t] = B.walloc(2 * ns);
        sl.gradn[t] = B.walloc(2 * ns);
      }
    }
  }
  refresh_vflux(B);
  make_tasks(B);
  std::vector<int> prefix((size_t)PH_COUNT * (B.ntasks + 1), 0);
  for (int ph = 0; ph < PH_COUNT; ph++)
    for (int i = 0; i < B.ntasks; i++)
      prefix[(size_t)ph * (B.ntasks + 1) + i + 1] = prefix[(size_t)ph * (B.ntasks + 1) + i] + B.nblk[ph][i];
  CK(cudaMalloc(&B.d_tasks, sizeof(BatchTask) * std::max(1, B.ntasks)));
  CK(cudaMalloc(&B.d_prefix, sizeof(int) * prefix.size()));
  CK(cudaMalloc(&B.d_wave_first, sizeof(int) * B.wave_first.size()));
  CK(cudaMalloc(&B.d_bar, sizeof(GridBarrier)));
  CK(cudaMemcpyAsync(B.d_tasks, B.tasks.data(), sizeof(BatchTask) * B.tasks.size(), cudaMemcpyHostToDevice, B.stream));
  CK(cudaMemcpyAsync(B.d_prefix, prefix.data(), sizeof(int) * prefix.size(), cudaMemcpyHostToDevice, B.stream));
  CK(cudaMemcpyAsync(B.d_wave_first, B.wave_first.data(), sizeof(int) * B.wave_first.size(), cudaMemcpyHostToDevice,
                     B.stream));
  CK(cudaMemsetAsync(B.d_bar, 0, sizeof(GridBarrier), B.stream));
  // persistent grid of every phase kernel
  for (int ph = 0; ph < PH_COUNT; ph++) {
    B.phgrid[ph] = 0;
    if (!B.phk[ph].fn) continue;
    const size_t sm = phase_smem(ph);
    CK(cudaFuncSetAttribute(B.phk[ph].fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int pocc = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pocc, B.phk[ph].fn, kThreads, sm));
    if (pocc < 1) throw std::runtime_error("batched phase kernel cannot be resident");
    B.phgrid[ph] = B.sms * pocc;
  }
  CK(cudaStreamSynchronize(B.stream));
}

namespace {

void launch_once(BatchImpl &B) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(B.grid);
  cfg.blockDim = dim3(B.tile.threads);
  cfg.dynamicSmemBytes = batch_smem();
  cfg.stream = B.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, B.kernel, B.d_tasks, (const int *)B.d_prefix, B.ntasks, (const int *)B.d_wave_first,
                        B.nwaves, B.d_bar, B.spin_limit, (int)B.refresh_ab));
}

// host copies of the device-side ping-pong
void swap_host(BatchImpl &B, int nsteps) {
  if (nsteps % 2 == 0) return;
  for (auto &m : B.members)
    for (auto &tr : m->impl()->tr) std::swap(tr.T, tr.Tout);
}

void check_barrier(BatchImpl &B) {
  GridBarrier h{};
  CK(cudaMemcpyAsync(&h, B.d_bar, sizeof(h), cudaMemcpyDeviceToHost, B.stream));
  CK(cudaStreamSynchronize(B.stream));
  if (h.err) {
    CK(cudaMemsetAsync(B.d_bar, 0, sizeof(GridBarrier), B.stream));
    CK(cudaStreamSynchronize(B.stream));
    throw std::runtime_error("batched step: a grid barrier timed out");
  }
}

void capture(BatchImpl &B) {
  if (B.graph_exec) return;
  CK(cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeThreadLocal));
  launch_once(B);
  cudaGraph_t g = nullptr;
  CK(cudaStreamEndCapture(B.stream, &g));
  B.graph = g;
  CK(cudaGraphInstantiate(&B.graph_exec, g, 0));
}

}  // namespace

namespace {

// the host task table after one step: new and old buffers swap
void swap_tasks(BatchImpl &B) {
  for (auto &T : B.tasks) {
    FusedArgs<float, float> &a = T.a;
    for (int q = 0; q < kNT; q++) {
      float *old = const_cast<float *>(a.T[q]);
      a.T[q] = a.T_out[q];
      a.T_out[q] = old;
      if (B.refresh_ab) a.TAB[q] = a.T[q];
    }
  }
}

// one step as persistent phase launches (one per phase, wave and slot
// stream) from the host task table, which then swaps.  The tasks of one
// work-array slot run in order on that slot's stream; slots are independent,
// so up to kPhaseStreams phase kernels of different slots run side by side.
void phase_step(BatchImpl &B) {
  const int K = std::max(1, std::min(B.tile.wave, BatchImpl::kPhaseStreams));
  if (K > 1) {
    CK(cudaEventRecord(B.ph_fork, B.stream));
    for (int k = 0; k < K; k++) CK(cudaStreamWaitEvent(B.ph_streams[k], B.ph_fork, 0));
  }
  PhasePack p{};
  std::vector<int> sel;
  for (int w = 0; w < B.nwaves; w++) {
    const int t0 = B.wave_first[w], t1 = B.wave_first[w + 1];
    for (int k = 0; k < K; k++) {
      sel.clear();
      for (int t = t0; t < t1; t++)
        if (B.task_slot[t] % K == k) sel.push_back(t);
      cudaStream_t st = K > 1 ? B.ph_streams[k] : B.stream;
      for (int ph = 0; ph < PH_COUNT; ph++) {
        if (!B.phk[ph].fn) continue;
        for (size_t c0 = 0; c0 < sel.size(); c0 += kPackTasks) {
          p.ntasks = 0;
          p.prefix[0] = 0;
          for (size_t i = c0; i < std::min(sel.size(), c0 + kPackTasks); i++) {
            p.t[p.ntasks] = B.tasks[sel[i]];
            p.prefix[p.ntasks + 1] = p.prefix[p.ntasks] + B.nblk[ph][sel[i]];
            p.ntasks++;
          }
          const int total = p.prefix[p.ntasks];
          if (total == 0) continue;
          B.phk[ph].launch(p, std::min(total, B.phgrid[ph]), phase_smem(ph), st);
        }
      }
    }
  }
  if (K > 1) {
    for (int k = 0; k < K; k++) {
      CK(cudaEventRecord(B.ph_join[k], B.ph_streams[k]));
      CK(cudaStreamWaitEvent(B.stream, B.ph_join[k], 0));
    }
  }
  swap_tasks(B);
}

void capture_phases(BatchImpl &B) {
  const void *key = B.tasks.empty() ? nullptr : (const void *)B.tasks[0].a.T[0];
  if (B.ph_exec && B.ph_key == key) return;
  if (B.ph_exec) cudaGraphExecDestroy(B.ph_exec);
  if (B.ph_graph) cudaGraphDestroy(B.ph_graph);
  B.ph_exec = nullptr;
  B.ph_graph = nullptr;
  CK(cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeThreadLocal));
  phase_step(B);
  phase_step(B);  // two steps: the task table is back where it started
  cudaGraph_t g = nullptr;
  CK(cudaStreamEndCapture(B.stream, &g));
  B.ph_graph = g;
  CK(cudaGraphInstantiate(&B.ph_exec, g, 0));
  B.ph_key = key;
}

// nsteps of the selected path on the batch stream
void run_steps(BatchImpl &B, int nsteps, bool use_graph, bool upload = true) {
  if (B.mode == 1) {
    if (use_graph && nsteps >= 2) {
      capture_phases(B);
      for (int s = 0; s + 1 < nsteps; s += 2) CK(cudaGraphLaunch(B.ph_exec, B.stream));
      if (nsteps % 2) phase_step(B);
    } else {
      for (int s = 0; s < nsteps; s++) phase_step(B);
    }
    return;
  }
  // the cooperative kernel swaps its device-side table itself; the host copy follows
  if (upload)
    CK(cudaMemcpyAsync(B.d_tasks, B.tasks.data(), sizeof(BatchTask) * B.tasks.size(), cudaMemcpyHostToDevice, B.stream));
  if (use_graph) capture(B);
  for (int s = 0; s < nsteps; s++) {
    if (use_graph) CK(cudaGraphLaunch(B.graph_exec, B.stream));
    else launch_once(B);
  }
  if (nsteps % 2) swap_tasks(B);
}

void begin_steps(BatchImpl &B) {
  if (!B.configured || !B.d_tasks) throw std::runtime_error("configure the batch first");
  for (auto &m : B.members) m->synchronize();
  bool stale = false;
  for (auto &m : B.members) stale = stale || !m->impl()->vflux_valid || !m->impl()->vflux;
  if (stale) {
    refresh_vflux(B);
    make_tasks(B);
    B.release_graph();
  }
}

}  // namespace

void Batch::set_path(int path) {
  if (path < 0 || path > 2)
    throw std::invalid_argument("batch path: 0 (one cooperative launch per step), 1 (one launch per phase) or 2 "
                                "(per-member launches)");
  if (p_->learned && path != 2)
    throw std::invalid_argument("batch path: with the learned flux only path 2 (per-member launches) runs");
  p_->mode = path;
}
int Batch::path() const { return p_->mode; }

void Batch::set_learned(const float *params, bool on) {
  BatchImpl &B = *p_;
  CK(cudaStreamSynchronize(B.stream));
  for (auto &m : B.members) m->set_learned(params, on);
  B.learned = on;
  if (on) B.mode = 2;
}
bool Batch::learned() const { return p_->learned; }

void Batch::step(int nsteps, bool use_graph) {
  BatchImpl &B = *p_;
  if (B.learned && B.mode != 2) throw std::logic_error("batch: the learned flux runs on path 2 only");
  if (B.mode == 2) {
    step_separate(nsteps, use_graph);
    return;
  }
  begin_steps(B);
  run_steps(B, nsteps, use_graph);
  CK(cudaGetLastError());
  if (B.mode == 0) check_barrier(B);
  else CK(cudaStreamSynchronize(B.stream));
  swap_host(B, nsteps);
}

double Batch::time_steps(int nsteps, bool use_graph) {
  BatchImpl &B = *p_;
  if (B.learned && B.mode != 2) throw std::logic_error("batch: the learned flux runs on path 2 only");
  if (B.mode == 2) return time_separate(nsteps, use_graph);
  begin_steps(B);
  // capture (and the device table upload) outside the timed region
  if (use_graph && B.mode == 1 && nsteps >= 2) capture_phases(B);
  if (B.mode == 0) {
    CK(cudaMemcpyAsync(B.d_tasks, B.tasks.data(), sizeof(BatchTask) * B.tasks.size(), cudaMemcpyHostToDevice, B.stream));
    if (use_graph) capture(B);
  }
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a, B.stream));
  run_steps(B, nsteps, use_graph, false);
  CK(cudaEventRecord(b, B.stream));
  CK(cudaEventSynchronize(b));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  CK(cudaGetLastError());
  if (B.mode == 0) check_barrier(B);
  swap_host(B, nsteps);
  return ms;
}

// The separate path uses the member engines' own work arrays; the batch's are
// released meanwhile (device memory) and rebuilt with the task table after.
// Members launch on their own streams; with use_graph the launches of two
// steps (so that every engine's buffer ping-pong returns to where it started)
// are captured once as a graph forked from and joined into the batch stream.
namespace {
void separate_steps_direct(BatchImpl &B, int nsteps) {
  for (int s = 0; s < nsteps; s++)
    for (size_t m = 0; m < B.members.size(); m++) B.members[m]->step(B.dt[m], B.refresh_ab);
}

void capture_separate(BatchImpl &B) {
  if (B.sep_exec) return;
  const size_t M = B.members.size();
  B.sep_events.resize(M + 1);
  for (auto &e : B.sep_events) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  CK(cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeRelaxed));
  CK(cudaEventRecord(B.sep_events[M], B.stream));
  for (size_t m = 0; m < M; m++) CK(cudaStreamWaitEvent((cudaStream_t)B.members[m]->stream(), B.sep_events[M], 0));
  separate_steps_direct(B, 2);
  for (size_t m = 0; m < M; m++) {
    CK(cudaEventRecord(B.sep_events[m], (cudaStream_t)B.members[m]->stream()));
    CK(cudaStreamWaitEvent(B.stream, B.sep_events[m], 0));
  }
  cudaGraph_t g = nullptr;
  CK(cudaStreamEndCapture(B.stream, &g));
  B.sep_graph = g;
  CK(cudaGraphInstantiate(&B.sep_exec, g, 0));
}

// nsteps separate steps (graph-replayed in pairs when use_graph)
void separate_steps(BatchImpl &B, int nsteps, bool use_graph) {
  if (!use_graph) {
    separate_steps_direct(B, nsteps);
    return;
  }
  for (int s = 0; s + 1 < nsteps; s += 2) CK(cudaGraphLaunch(B.sep_exec, B.stream));
  if (nsteps % 2) {
    CK(cudaStreamSynchronize(B.stream));
    separate_steps_direct(B, 1);
  }
}
}  // namespace

void Batch::step_separate(int nsteps, bool use_graph) {
  BatchImpl &B = *p_;
  CK(cudaStreamSynchronize(B.stream));
  B.release();
  // one direct step allocates the engines' work arrays and kernel attributes
  // before any capture
  const int first = nsteps > 0 ? 1 : 0;
  separate_steps_direct(B, first);
  CK(cudaDeviceSynchronize());
  if (use_graph) capture_separate(B);
  separate_steps(B, nsteps - first, use_graph);
  CK(cudaDeviceSynchronize());
  B.release_sep();
  for (auto &m : B.members) m->release_work();
  set_tile(B.tile);
}

double Batch::time_separate(int nsteps, bool use_graph) {
  BatchImpl &B = *p_;
  CK(cudaStreamSynchronize(B.stream));
  B.release();
  // one untimed step allocates the engines' work arrays
  separate_steps_direct(B, 1);
  CK(cudaDeviceSynchronize());
  if (use_graph) capture_separate(B);
  const auto t0 = std::chrono::steady_clock::now();
  separate_steps(B, nsteps, use_graph);
  CK(cudaDeviceSynchronize());
  const auto t1 = std::chrono::steady_clock::now();
  B.release_sep();
  for (auto &m : B.members) m->release_work();
  set_tile(B.tile);
  return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

std::string Batch::autotune(int steps_per_candidate) {
  BatchImpl &B = *p_;
  if (!B.configured) throw std::runtime_error("configure the batch first");
  // save the current tracer state
  std::vector<void *> saved;
  std::vector<void *> where;
  for (auto &m : B.members) {
    EngineImpl &P = *m->impl();
    const size_t bytes = (size_t)P.mesh.nod2D * P.S * P.ts_bytes;
    for (auto &tr : P.tr) {
      void *s = nullptr;
      CK(cudaMalloc(&s, bytes));
      CK(cudaMemcpy(s, tr.T, bytes, cudaMemcpyDeviceToDevice));
      saved.push_back(s);
      where.push_back(tr.T);
    }
  }
  std::ostringstream log;
  BatchTile best = B.tile;
  double best_ms = 1e30;
  int max_batches = 0;
  for (int m = 0; m < num_members(); m++) max_batches = std::max(max_batches, B.ntr[m] / kNT);
  int best_mode = B.mode;
  for (int cells : {256, 384, 512}) {
    {
      // per-member launches: only the cells per block of the members apply
      BatchTile t;
      t.cells_per_block = cells;
      t.wave = 1;
      set_tile(t);
      B.mode = 2;
      const double ms = time_steps(steps_per_candidate, false) / steps_per_candidate;
      log << "path=separate cells=" << cells << " ms_per_step=" << ms << "\n";
      if (ms < best_ms) {
        best_ms = ms;
        best = B.tile;
        best_mode = 2;
      }
    }
    for (int wave : {1, 2, 4}) {
      if (B.learned) break;  // the persistent paths have no MLP phase
      if (wave > max_batches && wave != 1) continue;
      // one launch per phase: the tile's threads and blocks per SM do not apply
      {
        BatchTile t;
        t.cells_per_block = cells;
        t.wave = wave;
        bool ok = true;
        try {
          set_tile(t);
        } catch (const std::exception &e) {
          cudaGetLastError();
          log << "path=phases cells=" << cells << " wave=" << wave << " skipped: " << e.what() << "\n";
          ok = false;
        }
        if (ok) {
          B.mode = 1;
          time_steps(1, false);  // warm-up
          const double ms = time_steps(steps_per_candidate, false) / steps_per_candidate;
          log << "path=phases cells=" << cells << " wave=" << B.tile.wave << " ms_per_step=" << ms << "\n";
          if (ms < best_ms) {
            best_ms = ms;
            best = B.tile;
            best_mode = 1;
          }
        }
      }
      for (int threads : {128, 256}) {
        for (int bps : {2, 3, 4, 5, 6, 8, 10}) {
          BatchTile t;
          t.cells_per_block = cells;
          t.wave = wave;
          t.threads = threads;
          t.blocks_per_sm = bps;
          try {
            set_tile(t);
          } catch (const std::exception &e) {
            cudaGetLastError();
            log << "path=cooperative cells=" << cells << " wave=" << wave << " threads=" << threads << " bps=" << bps
                << " skipped: " << e.what() << "\n";
            continue;
          }
          if (B.tile.blocks_per_sm != bps) continue;  // occupancy cap: same as a smaller candidate
          B.mode = 0;
          time_steps(1, false);  // warm-up
          const double ms = time_steps(steps_per_candidate, false) / steps_per_candidate;
          log << "path=cooperative cells=" << cells << " wave=" << B.tile.wave << " threads=" << threads
              << " bps=" << bps << " ms_per_step=" << ms << "\n";
          if (ms < best_ms) {
            best_ms = ms;
            best = B.tile;
            best_mode = 0;
          }
        }
      }
    }
  }
  // restore the state and keep the best tile
  size_t i = 0;
  for (auto &m : B.members) {
    EngineImpl &P = *m->impl();
    const size_t bytes = (size_t)P.mesh.nod2D * P.S * P.ts_bytes;
    for (auto &tr : P.tr) {
      if (tr.T != where[i]) std::swap(tr.T, tr.Tout);
      CK(cudaMemcpy(tr.T, saved[i], bytes, cudaMemcpyDeviceToDevice));
      cudaFree(saved[i]);
      i++;
    }
  }
  set_tile(best);
  B.mode = best_mode;
  log << "best: path=" << (best_mode == 2 ? "separate" : best_mode == 1 ? "phases" : "cooperative")
      << " cells=" << best.cells_per_block
      << " wave=" << best.wave << " threads=" << best.threads << " bps=" << best.blocks_per_sm
      << " ms_per_step=" << best_ms << "\n";
  return log.str();
}

int batch_selftest_barrier_timeout(long long limit) {
  GridBarrier *bar = nullptr;
  int *st = nullptr;
  if (cudaMalloc(&bar, sizeof(GridBarrier)) != cudaSuccess) return -1;
  if (cudaMalloc(&st, sizeof(int)) != cudaSuccess) { cudaFree(bar); return -1; }
  cudaMemset(bar, 0, sizeof(GridBarrier));
  cudaMemset(st, 0xff, sizeof(int));
  k_barrier_timeout<<<2, 64>>>(bar, limit, st);
  int h = -1;
  const cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) cudaMemcpy(&h, st, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(bar);
  cudaFree(st);
  return e == cudaSuccess ? h : -1;
}

}  // namespace fesom
