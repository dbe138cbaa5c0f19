// hp_batch_fp64.cu -- FP64 instantiations of the persistent batched sweep
// (many boxes per launch).  Same flags as the single-box FP64 sweeps
// (--fmad=false), so a box swept in a batch is bitwise identical to the same
// box swept alone with the same tile.
#include <cuda_runtime.h>

#include "hp_launch.h"
#include "hp_sweep.cuh"
#include "hp_sweep_launch.cuh"

namespace hp {

int launch_sweep_batch_fp64(const BatchLaunch& bl, int axis, int tile, cudaStream_t st) {
    return launch_sweep_batch_policy<PolicyFP64>(bl, axis, tile, st);
}

}  // namespace hp
