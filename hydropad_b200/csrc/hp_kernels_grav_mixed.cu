// hp_kernels_grav_mixed.cu -- mixed-precision sweep instantiations with the
// static gravity source.  Same flags as the gravity-free mixed sweeps
// (-use_fast_math --fmad=false).
#include <cuda_runtime.h>

#include "hp_launch.h"
#include "hp_sweep.cuh"
#include "hp_sweep_launch.cuh"

namespace hp {

int launch_sweep_grav_mixed(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st) {
    return launch_sweep_policy<PolicyMixed, true>(b, axis, tile, bslot, flags, st);
}

}  // namespace hp
