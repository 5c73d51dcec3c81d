// FP64 step kernels compiled WITH FMA contraction (--fmad=true): the same
// operations as step_f64.cu in the same order, each a*b+c pair fused where
// the compiler contracts it.  Results agree with the reference's arithmetic
// to about 1e-13 relative instead of bit for bit, for fewer FP64
// instructions per cell.  The kernels live in the inline namespace fma64.
#define FESOM_KERNEL_VARIANT fma64
#include "launch.cuh"

namespace fesom {

void launch_batch_f64fma(EngineImpl &P, const TracerScheme &sc, int nt, const BatchPtrs &b, double dt) {
  launch_batch_t<double, double>(P, sc, nt, b, dt);
}

}  // namespace fesom
