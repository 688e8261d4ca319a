// af_xfer.h -- host<->device copies of row blocks (the fields a caller hands
// in or reads back) at the link's rate whether or not the host memory is
// pinned.
//
// Pinned (page-locked) host memory, and any copy under 1 MB, is copied by
// cudaMemcpy2DAsync straight away.  Larger copies of pageable memory, which
// the driver would move through its own small staging buffers at a fraction
// of the link's rate, go through two 16 MB pinned buffers of this library
// instead: host threads fill one (or drain it) while the DMA of the other
// runs.  Such a copy returns when the host side is done with the caller's
// memory (for a copy to the device: when the data has left this library's
// buffers too).  Copies through the buffers run one at a time per process.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace af {

// Same arguments as cudaMemcpy2DAsync (pitches and width in bytes).
cudaError_t copy2d_h2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                       size_t rows, cudaStream_t st);
cudaError_t copy2d_d2h(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                       size_t rows, cudaStream_t st);

}  // namespace af
