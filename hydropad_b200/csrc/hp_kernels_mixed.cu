// hp_kernels_mixed.cu -- mixed-precision sweep instantiations.
//
// Reconstruction, flattening, characteristic tracing, the traced face
// states, the closed-form Riemann solutions and the Newton iteration of
// weak faces run in FP32; the Newton iteration for p*, u* across strong
// shocks and near-vacuum states, the conservative update (fluxes formed in
// FP64) and the total-minus-kinetic energy of the dual-energy switch stay
// FP64, and the state in HBM stays FP64.
#include <cuda_runtime.h>

#include "hp_device.cuh"
#include "hp_launch.h"
#include "hp_physics.cuh"
#include "hp_sweep.cuh"
#include "hp_sweep_launch.cuh"

namespace hp {

int launch_sweep_grav_mixed(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st);

int launch_sweep_mixed(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st) {
    if (b.g[0]) return launch_sweep_grav_mixed(b, axis, tile, bslot, flags, st);
    return launch_sweep_policy<PolicyMixed>(b, axis, tile, bslot, flags, st);
}

}  // namespace hp
