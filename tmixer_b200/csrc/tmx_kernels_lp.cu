// tmx_kernels_lp.cu -- sm_100a kernels of the reduced-precision forms: FP32
// arithmetic with FP32 storage, and FP32 arithmetic with populations stored in
// FP16 as f_q - feq_q of the node that wrote them.  Both keep the four fields
// of a (direction, node) pair side by side, one vector access each.  Compiled
// with multiply-add contraction (the default); results are compared with the
// FP64 form within stated tolerances, not bit for bit.
#include "tmx_engine.cuh"

namespace tmx {

TMX_DEFINE_STEP_KERNELS(F32, f32)
TMX_DEFINE_BOUNDARY_KERNELS(F32, f32)
TMX_DEFINE_BATCH_KERNELS(F32, f32)
TMX_DEFINE_STEP_KERNELS(F16, f16)
TMX_DEFINE_BOUNDARY_KERNELS(F16, f16)
TMX_DEFINE_BATCH_KERNELS(F16, f16)
TMX_DEFINE_SWEEP_KERNELS(F16, f16)

}  // namespace tmx
