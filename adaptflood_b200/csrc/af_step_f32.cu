// af_step_f32.cu -- FP32 instantiation of the fused step (FP32 state and
// arithmetic; FP64 time, dt, hydrograph interpolation and volume sums).
#include "af_step.cuh"

namespace af {
const void* step_kernel_f32(int wx) {
  switch (wx) {
    case 1: return (const void*)&k_step<float, 1>;
    case 2: return (const void*)&k_step<float, 2>;
    default: return (const void*)&k_step<float, 4>;
  }
}
}  // namespace af
