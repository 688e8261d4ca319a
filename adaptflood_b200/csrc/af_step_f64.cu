// af_step_f64.cu -- FP64 instantiation of the fused step.  Compiled with
// -fmad=false so each expression rounds as the reference's C++ does.
#include "af_step.cuh"

namespace af {
const void* step_kernel_f64(int wx) {
  switch (wx) {
    case 1: return (const void*)&k_step<double, 1>;
    case 2: return (const void*)&k_step<double, 2>;
    default: return (const void*)&k_step<double, 4>;
  }
}
}  // namespace af
