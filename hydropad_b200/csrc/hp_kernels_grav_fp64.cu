// hp_kernels_grav_fp64.cu -- FP64 sweep instantiations with the static
// gravity source (a box attached with gforce): the g parabola in the
// characteristic tracing and the source terms of integrate.  Same flags as
// the gravity-free FP64 sweeps (--fmad=false).
#include <cuda_runtime.h>

#include "hp_launch.h"
#include "hp_sweep.cuh"
#include "hp_sweep_launch.cuh"

namespace hp {

int launch_sweep_grav_fp64(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st) {
    return launch_sweep_policy<PolicyFP64, true>(b, axis, tile, bslot, flags, st);
}

}  // namespace hp
