// hp_batch_mixed.cu -- mixed-precision instantiations of the persistent
// batched sweep (many boxes per launch).  Same flags as the single-box mixed
// sweeps (-use_fast_math --fmad=false).
#include <cuda_runtime.h>

#include "hp_launch.h"
#include "hp_sweep.cuh"
#include "hp_sweep_launch.cuh"

namespace hp {

int launch_sweep_batch_mixed(const BatchLaunch& bl, int axis, int tile, cudaStream_t st) {
    return launch_sweep_batch_policy<PolicyMixed>(bl, axis, tile, st);
}

}  // namespace hp
