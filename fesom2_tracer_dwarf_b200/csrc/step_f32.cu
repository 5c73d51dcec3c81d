// FP32 step kernels (FMA contraction allowed): FP32 tracers, or BF16 / FP16
// tracer storage with FP32 arithmetic and accumulation; the FCT ratio
// denominators are formed in FP64 inside k_col2.
#include "launch.cuh"

namespace fesom {

void launch_batch_f32(EngineImpl &P, const TracerScheme &sc, int nt, const BatchPtrs &b, double dt) {
  switch (P.prec) {
    case Precision::BF16: launch_batch_t<float, __nv_bfloat16>(P, sc, nt, b, dt); break;
    case Precision::FP16: launch_batch_t<float, __half>(P, sc, nt, b, dt); break;
    default: launch_batch_t<float, float>(P, sc, nt, b, dt); break;
  }
}

void build_rcp_f32(EngineImpl &P) { build_rcp_planes_t<float>(P, P.dm32); }

void volume_sum_f32(EngineImpl &P, const void *T, double off, double out[2]) {
  switch (P.prec) {
    case Precision::BF16: volume_sum_t<float, __nv_bfloat16>(P, T, off, out); break;
    case Precision::FP16: volume_sum_t<float, __half>(P, T, off, out); break;
    default: volume_sum_t<float, float>(P, T, off, out); break;
  }
}

}  // namespace fesom
