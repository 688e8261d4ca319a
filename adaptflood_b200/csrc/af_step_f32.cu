// af_step_f32.cu -- FP32 instantiation of the fused step (FP32 state and
// arithmetic; FP64 time, dt, hydrograph interpolation and volume sums).
#include "af_step.cuh"

namespace af {
// Indices follow kStepVariant in af_step.cuh.
const void* step_kernel_f32(int variant, bool tma) {
  if (!tma) {
    switch (variant) {
      case 1: return (const void*)&k_step<float, 1, 12, false, false>;
      case 2: return (const void*)&k_step<float, 1, 20, false, false>;
      case 3: return (const void*)&k_step<float, 4, 4, false, false>;
      case 4: return (const void*)&k_step<float, 2, 8, false, false>;
      default: return (const void*)&k_step<float, 1, 16, false, false>;
    }
  }
  switch (variant) {
    case 1: return (const void*)&k_step<float, 1, 12>;
    case 2: return (const void*)&k_step<float, 1, 20>;
    case 3: return (const void*)&k_step<float, 4, 4>;
    case 4: return (const void*)&k_step<float, 2, 8>;
    default: return (const void*)&k_step<float, 1, 16>;
  }
}
const void* batch_kernel_f32(int variant) {
  switch (variant) {
    case 1: return (const void*)&k_batch_step<float, 1, 12>;
    case 2: return (const void*)&k_batch_step<float, 1, 20>;
    case 3: return (const void*)&k_batch_step<float, 4, 4>;
    case 4: return (const void*)&k_batch_step<float, 2, 8>;
    default: return (const void*)&k_batch_step<float, 1, 16>;
  }
}
const void* batch_begin_f32() { return (const void*)&k_batch_begin<float>; }
const void* batch_fold_f32() { return (const void*)&k_batch_fold<float>; }
}  // namespace af
