// hp_kernels_mixed.cu -- mixed-precision sweep instantiations.
//
// Reconstruction, flattening, characteristic tracing and the traced face
// states run in FP32; the Riemann solver (Newton for p*, u*), the
// conservative update and the total-minus-kinetic energy of the dual-energy
// switch stay FP64, and the state in HBM stays FP64.
#include <cuda_runtime.h>

#include "hp_device.cuh"
#include "hp_launch.h"
#include "hp_physics.cuh"
#include "hp_sweep.cuh"
#include "hp_sweep_launch.cuh"

namespace hp {

struct PolicyMixed {
    using R = float;             // reconstruction, flattening, tracing
    using Pow = PowRootShort;    // FP64 Newton for p*, u* (patterns 1, 2) and vacuum
    using CT = float;            // wave-pattern classification
    using PowC = PowF32m;
    using RareT = float;         // closed two-rarefaction form: no iteration
    using PowRare = PowRareF32;
};

int launch_sweep_mixed(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st) {
    return launch_sweep_policy<PolicyMixed>(b, axis, tile, bslot, flags, st);
}

}  // namespace hp
