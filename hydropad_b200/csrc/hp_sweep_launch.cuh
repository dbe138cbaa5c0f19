// hp_sweep_launch.cuh -- tile table and launcher of the fused sweep, shared
// by the FP64 and mixed-precision translation units.
//
// A tile is (P pencils per CTA, T cells per window step, RING slots).  Along
// x a warp covers 32/T pencils x T consecutive cells; along y/z a warp
// covers 32 consecutive pencils (x) x 1 cell.  The best tile depends on the
// grid and the precision; hp_autotune measures them.
#pragma once
#include <cuda_runtime.h>

#include "hp_launch.h"
#include "hp_sweep.cuh"

namespace hp {

constexpr int kTilesX = 8, kTilesYZ = 8;

template <int AXIS, int P, int T, int RING, class Policy, int MINB = 1>
static int launch_sweep_t(const Box& b, int bslot, int flags, cudaStream_t st) {
    SweepArgs a;
    // permute velocities into (normal, transverse1, transverse2) of this
    // sweep (ppmsolver.F90:105-107, 227-229, 355-357)
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
    const size_t smem = sizeof(SweepSmem<AXIS, P, T, RING, Policy>);
    auto kern = ppm_sweep_kernel<AXIS, P, T, RING, Policy, MINB>;
    static bool attr_set = false;  // per instantiation (one process drives one device)
    if (!attr_set) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return -1;
        attr_set = true;
    }
    const long long grid = (a.npencil + P - 1) / P;
    kern<<<(unsigned)grid, P * T, smem, st>>>(a);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

template <class Policy>
static int launch_sweep_policy(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st) {
    if (axis == 0) {
        switch (tile) {
            case 0: return launch_sweep_t<0, 8, 32, 64, Policy>(b, bslot, flags, st);
            case 1: return launch_sweep_t<0, 4, 32, 64, Policy>(b, bslot, flags, st);
            case 2: return launch_sweep_t<0, 8, 16, 32, Policy>(b, bslot, flags, st);
            case 3: return launch_sweep_t<0, 4, 16, 32, Policy>(b, bslot, flags, st);
            case 4: return launch_sweep_t<0, 16, 32, 64, Policy>(b, bslot, flags, st);
            case 5: return launch_sweep_t<0, 12, 32, 64, Policy>(b, bslot, flags, st);
            case 6: return launch_sweep_t<0, 8, 32, 64, Policy, 3>(b, bslot, flags, st);
            case 7: return launch_sweep_t<0, 4, 32, 64, Policy, 5>(b, bslot, flags, st);
        }
    } else if (axis == 1) {
        switch (tile) {
            case 0: return launch_sweep_t<1, 32, 8, 16, Policy>(b, bslot, flags, st);
            case 1: return launch_sweep_t<1, 16, 8, 16, Policy>(b, bslot, flags, st);
            case 2: return launch_sweep_t<1, 32, 4, 16, Policy>(b, bslot, flags, st);
            case 3: return launch_sweep_t<1, 16, 4, 16, Policy>(b, bslot, flags, st);
            case 4: return launch_sweep_t<1, 64, 8, 16, Policy>(b, bslot, flags, st);
            case 5: return launch_sweep_t<1, 32, 12, 32, Policy>(b, bslot, flags, st);
            case 6: return launch_sweep_t<1, 32, 8, 16, Policy, 3>(b, bslot, flags, st);
            case 7: return launch_sweep_t<1, 16, 8, 16, Policy, 5>(b, bslot, flags, st);
        }
    } else if (axis == 2) {
        switch (tile) {
            case 0: return launch_sweep_t<2, 32, 8, 16, Policy>(b, bslot, flags, st);
            case 1: return launch_sweep_t<2, 16, 8, 16, Policy>(b, bslot, flags, st);
            case 2: return launch_sweep_t<2, 32, 4, 16, Policy>(b, bslot, flags, st);
            case 3: return launch_sweep_t<2, 16, 4, 16, Policy>(b, bslot, flags, st);
            case 4: return launch_sweep_t<2, 64, 8, 16, Policy>(b, bslot, flags, st);
            case 5: return launch_sweep_t<2, 32, 12, 32, Policy>(b, bslot, flags, st);
            case 6: return launch_sweep_t<2, 32, 8, 16, Policy, 3>(b, bslot, flags, st);
            case 7: return launch_sweep_t<2, 16, 8, 16, Policy, 5>(b, bslot, flags, st);
        }
    }
    return -1;
}

}  // namespace hp
