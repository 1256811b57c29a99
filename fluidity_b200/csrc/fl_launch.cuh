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

// Whether the device-resident 2-D loop alternates layouts (each sweep reads
// the state with its own dimension slowest and writes it transposed) for
// this sweep configuration; p carries the loop's buffers and extents.
bool loop_transposes_f64(const SweepParams& p, int flux);
bool loop_transposes_f32(const SweepParams& p, int flux);

}  // namespace fl
