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

  ~BatchImpl() {
    release();
    release_sep();
    if (stream) cudaStreamDestroy(stream);
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
  }
  void release() {
    release_graph();
    for (void *w : work) cudaFree(w);
    work.clear();
    work_bytes = 0;
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

Batch::Batch() : p_(new BatchImpl) {
  CK(cudaStreamCreateWithFlags(&p_->stream, cudaStreamNonBlocking));
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&p_->sms, cudaDevAttrMultiProcessorCount, dev));
}
Batch::~Batch() { delete p_; }

int Batch::add_member(const MeshHost &mesh, int ntracers) {
  if (ntracers < kNT || ntracers % kNT) throw std::invalid_argument("batch members need a multiple of 4 tracers");
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
bool Batch::graph_captured() const { return p_->graph_exec != nullptr; }

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
      need += (size_t)std::min(W, B.ntr[m] / kNT) * (es + kNT * (es + 6 * ns));
    }
    CK(cudaMemGetInfo(&free_b, &total_b));
    if (need > free_b / 10 * 9)
      throw std::runtime_error("not enough device memory for " + std::to_string(W) + " tracer batches in flight");
  }
  B.tile.wave = W;
  B.nwaves = (max_batches + W - 1) / W;
  struct Slot { void *adfh[kNT], *adfv[kNT], *lo[kNT], *rp[kNT], *rm[kNT], *gradn[kNT], *vflux; };
  std::vector<std::vector<Slot>> slots(M, std::vector<Slot>(W));
  for (int m = 0; m < M; m++) {
    EngineImpl &P = *B.members[m]->impl();
    const size_t ns = (size_t)P.mesh.nod2D * P.S * sizeof(float), es = (size_t)P.mesh.edge2D * P.S * sizeof(float);
    const int used = std::min(W, B.ntr[m] / kNT);
    for (int j = 0; j < used; j++) {
      Slot &s = slots[m][j];
      s.vflux = B.walloc(es);
      for (int t = 0; t < kNT; t++) {
        s.adfh[t] = B.walloc(es);
        s.adfv[t] = B.walloc(ns);
        s.lo[t] = B.walloc(ns);
        s.rp[t] = B.walloc(ns);
        s.rm[t] = B.walloc(ns);
        s.gradn[t] = B.walloc(2 * ns);
      }
    }
  }
  std::vector<BatchTask> tasks;
  std::vector<int> wave_first;
  std::vector<std::vector<int>> nblk(PH_COUNT);
  for (int w = 0; w < B.nwaves; w++) {
    wave_first.push_back((int)tasks.size());
    for (int m = 0; m < M; m++) {
      EngineImpl &P = *B.members[m]->impl();
      for (int b = w * W; b < std::min((w + 1) * W, B.ntr[m] / kNT); b++) {
        const Slot &s = slots[m][b % W];
        BatchTask T{};
        T.m = P.dm32;
        FusedArgs<float, float> &a = T.a;
        for (int t = 0; t < kNT; t++) {
          auto &tr = P.tr[b * kNT + t];
          a.T[t] = (const float *)tr.T;
          a.TAB[t] = (const float *)(B.refresh_ab ? tr.T : tr.TAB);
          a.T_out[t] = (float *)tr.Tout;
          a.adf_h[t] = (float *)s.adfh[t];
          a.adf_v[t] = (float *)s.adfv[t];
          a.lo[t] = (float *)s.lo[t];
          a.rp[t] = (float *)s.rp[t];
          a.rm[t] = (float *)s.rm[t];
          a.gradn[t] = (float *)s.gradn[t];
        }
        a.vflux = (float *)s.vflux;
        a.vel = (const float *)P.vel;
        a.W = (const float *)P.W;
        a.dt = (float)B.dt[m];
        a.ph = (float)B.sch.ph;
        a.pv = (float)B.sch.pv;
        tasks.push_back(T);
        nblk[PH_GRAD].push_back(P.dm32.grad_sched.nblk);
        nblk[PH_EDGE].push_back(P.dm32.edge_sched.nblk);
        for (int ph : {PH_COL1, PH_COL2, PH_COL3}) nblk[ph].push_back(P.dm32.node_sched.nblk);
      }
    }
  }
  wave_first.push_back((int)tasks.size());
  B.ntasks = (int)tasks.size();
  std::vector<int> prefix((size_t)PH_COUNT * (B.ntasks + 1), 0);
  for (int ph = 0; ph < PH_COUNT; ph++)
    for (int i = 0; i < B.ntasks; i++) prefix[(size_t)ph * (B.ntasks + 1) + i + 1] = prefix[(size_t)ph * (B.ntasks + 1) + i] + nblk[ph][i];
  CK(cudaMalloc(&B.d_tasks, sizeof(BatchTask) * std::max(1, B.ntasks)));
  CK(cudaMalloc(&B.d_prefix, sizeof(int) * prefix.size()));
  CK(cudaMalloc(&B.d_wave_first, sizeof(int) * wave_first.size()));
  CK(cudaMalloc(&B.d_bar, sizeof(GridBarrier)));
  CK(cudaMemcpyAsync(B.d_tasks, tasks.data(), sizeof(BatchTask) * tasks.size(), cudaMemcpyHostToDevice, B.stream));
  CK(cudaMemcpyAsync(B.d_prefix, prefix.data(), sizeof(int) * prefix.size(), cudaMemcpyHostToDevice, B.stream));
  CK(cudaMemcpyAsync(B.d_wave_first, wave_first.data(), sizeof(int) * wave_first.size(), cudaMemcpyHostToDevice, B.stream));
  CK(cudaMemsetAsync(B.d_bar, 0, sizeof(GridBarrier), B.stream));
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

void Batch::step(int nsteps, bool use_graph) {
  BatchImpl &B = *p_;
  if (!B.configured || !B.d_tasks) throw std::runtime_error("configure the batch first");
  for (auto &m : B.members) m->synchronize();
  if (use_graph) capture(B);
  for (int s = 0; s < nsteps; s++) {
    if (use_graph) CK(cudaGraphLaunch(B.graph_exec, B.stream));
    else launch_once(B);
  }
  CK(cudaGetLastError());
  check_barrier(B);
  swap_host(B, nsteps);
}

double Batch::time_steps(int nsteps, bool use_graph) {
  BatchImpl &B = *p_;
  if (!B.configured || !B.d_tasks) throw std::runtime_error("configure the batch first");
  for (auto &m : B.members) m->synchronize();
  if (use_graph) capture(B);
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a, B.stream));
  for (int s = 0; s < nsteps; s++) {
    if (use_graph) CK(cudaGraphLaunch(B.graph_exec, B.stream));
    else launch_once(B);
  }
  CK(cudaEventRecord(b, B.stream));
  CK(cudaEventSynchronize(b));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  check_barrier(B);
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
  for (int cells : {256, 384, 512}) {
    for (int wave : {1, 2, 4}) {
      if (wave > max_batches && wave != 1) continue;
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
            log << "cells=" << cells << " wave=" << wave << " threads=" << threads << " bps=" << bps
                << " skipped: " << e.what() << "\n";
            continue;
          }
          if (B.tile.blocks_per_sm != bps) continue;  // occupancy cap: same as a smaller candidate
          time_steps(1, false);  // warm-up
          const double ms = time_steps(steps_per_candidate, false) / steps_per_candidate;
          log << "cells=" << cells << " wave=" << B.tile.wave << " threads=" << threads << " bps=" << bps
              << " ms_per_step=" << ms << "\n";
          if (ms < best_ms) {
            best_ms = ms;
            best = B.tile;
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
  log << "best: cells=" << best.cells_per_block << " wave=" << best.wave << " threads=" << best.threads
      << " bps=" << best.blocks_per_sm << " ms_per_step=" << best_ms << "\n";
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
