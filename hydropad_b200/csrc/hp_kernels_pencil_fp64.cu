// hp_kernels_pencil_fp64.cu -- FP64 instantiations of the non-STENCIL
// build's full-pencil solver (hydro/ppm.F90, called per pencil by the
// #else branches of ppmsolver.F90): the STENCIL sweep's fused kernel with
// the four differences of ppm() (sound speed of the next cell in the
// characteristic speeds, the peak window along the sweep, cho at density
// peaks, the 3-cell dual-energy switch) and no gravity source.  Same flags
// as the other FP64 sweeps (--fmad=false).
#include <cuda_runtime.h>

#include "hp_launch.h"
#include "hp_sweep.cuh"
#include "hp_sweep_launch.cuh"

namespace hp {

int launch_sweep_pencil_fp64(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st) {
    return launch_sweep_policy<PolicyFP64, false, true>(b, axis, tile, bslot, flags, st);
}

}  // namespace hp
