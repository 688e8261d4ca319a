// af_step_f64.cu -- FP64 instantiation of the fused step.  Compiled with
// -fmad=false so each expression rounds as the reference's C++ does.
#include "af_step.cuh"

namespace af {
// Indices follow kStepVariant in af_step.cuh.
const void* step_kernel_f64(int variant, bool face_call, bool tma) {
  if (!tma) {  // large grids: the face law inline, bulk copies
    switch (variant) {
      case 1: return (const void*)&k_step<double, 1, 12, false, false>;
      case 2: return (const void*)&k_step<double, 1, 20, false, false>;
      case 3: return (const void*)&k_step<double, 4, 4, false, false>;
      case 4: return (const void*)&k_step<double, 2, 8, false, false>;
      default: return (const void*)&k_step<double, 1, 16, false, false>;
    }
  }
  if (face_call) {
    switch (variant) {
      case 1: return (const void*)&k_step<double, 1, 12, true>;
      case 2: return (const void*)&k_step<double, 1, 20, true>;
      case 3: return (const void*)&k_step<double, 4, 4, true>;
      case 4: return (const void*)&k_step<double, 2, 8, true>;
      default: return (const void*)&k_step<double, 1, 16, true>;
    }
  }
  switch (variant) {
    case 1: return (const void*)&k_step<double, 1, 12>;
    case 2: return (const void*)&k_step<double, 1, 20>;
    case 3: return (const void*)&k_step<double, 4, 4>;
    case 4: return (const void*)&k_step<double, 2, 8>;
    default: return (const void*)&k_step<double, 1, 16>;
  }
}
const void* batch_kernel_f64(int variant) {
  switch (variant) {
    case 1: return (const void*)&k_batch_step<double, 1, 12>;
    case 2: return (const void*)&k_batch_step<double, 1, 20>;
    case 3: return (const void*)&k_batch_step<double, 4, 4>;
    case 4: return (const void*)&k_batch_step<double, 2, 8>;
    default: return (const void*)&k_batch_step<double, 1, 16>;
  }
}
const void* batch_begin_f64() { return (const void*)&k_batch_begin<double>; }
const void* batch_fold_f64() { return (const void*)&k_batch_fold<double>; }
}  // namespace af
