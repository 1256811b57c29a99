// fl_launch.cuh -- host-side launch of the sweep kernel for one dtype.
#pragma once

#include <cuda_runtime.h>

#include "fl_internal.cuh"

namespace fl {

// Launches one dimensional sweep; dtype fixed by the translation unit.
cudaError_t launch_sweep_f64(const SweepParams& p, int dims, int dim, int flux,
                             cudaStream_t stream);
cudaError_t launch_sweep_f32(const SweepParams& p, int dims, int dim, int flux,
                             cudaStream_t stream);

}  // namespace fl
