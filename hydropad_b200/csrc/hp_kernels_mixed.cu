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

namespace hp {

struct PolicyMixed {
    using R = float;
    using Pow = PowRoot;
};

constexpr int kPx = 8, kTx = 32, kRingX = 64;
constexpr int kPyz = 32, kTyz = 8, kRingYZ = 16;

template <int AXIS, int P, int T, int RING>
static int launch_mixed_t(const Box& b, int bslot, int flags, cudaStream_t st) {
    SweepArgs a;
    a.f[0] = b.f[0];
    a.f[1] = b.f[1];
    if (AXIS == 0) { a.f[2] = b.f[2]; a.f[3] = b.f[3]; a.f[4] = b.f[4]; }
    if (AXIS == 1) { a.f[2] = b.f[3]; a.f[3] = b.f[2]; a.f[4] = b.f[4]; }
    if (AXIS == 2) { a.f[2] = b.f[4]; a.f[3] = b.f[3]; a.f[4] = b.f[2]; }
    for (int q = 0; q < 4; ++q) a.snap[q] = b.snap[q];
    a.peak = b.peak;
    a.ctl = b.ctl;
    a.k = b.k;
    a.nx = b.nx; a.ny = b.ny; a.nz = b.nz;
    a.nsweep = AXIS == 0 ? b.nx : (AXIS == 1 ? b.ny : b.nz);
    a.npencil = AXIS == 0 ? (long long)b.ny * b.nz : (AXIS == 1 ? (long long)b.nx * b.nz : (long long)b.nx * b.ny);
    a.bslot = bslot;
    a.flags = flags;
    const size_t smem = sizeof(SweepSmem<AXIS, P, T, RING, PolicyMixed>);
    auto kern = ppm_sweep_kernel<AXIS, P, T, RING, PolicyMixed>;
    static bool attr_set = false;
    if (!attr_set) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return -1;
        attr_set = true;
    }
    const long long grid = (a.npencil + P - 1) / P;
    kern<<<(unsigned)grid, P * T, smem, st>>>(a);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

int launch_sweep_mixed(const Box& b, int axis, int bslot, int flags, cudaStream_t st) {
    switch (axis) {
        case 0: return launch_mixed_t<0, kPx, kTx, kRingX>(b, bslot, flags, st);
        case 1: return launch_mixed_t<1, kPyz, kTyz, kRingYZ>(b, bslot, flags, st);
        case 2: return launch_mixed_t<2, kPyz, kTyz, kRingYZ>(b, bslot, flags, st);
    }
    return -1;
}

size_t sweep_smem_bytes_mixed(int axis) {
    if (axis == 0) return sizeof(SweepSmem<0, kPx, kTx, kRingX, PolicyMixed>);
    return sizeof(SweepSmem<1, kPyz, kTyz, kRingYZ, PolicyMixed>);
}

}  // namespace hp
