// FP64 step kernels, compiled without FMA contraction (--fmad=false) so the
// results are bit-identical to the CPU oracle.
#include "launch.cuh"

namespace fesom {

void launch_batch_f64(EngineImpl &P, const TracerScheme &sc, int nt, const BatchPtrs &b, double dt) {
  launch_batch_t<double, double>(P, sc, nt, b, dt);
}

void build_rcp_f64(EngineImpl &P) { build_rcp_planes_t<double>(P, P.dm64); }

void volume_sum_f64(EngineImpl &P, const void *T, double out[2]) { volume_sum_t<double, double>(P, T, 0.0, out); }

}  // namespace fesom
