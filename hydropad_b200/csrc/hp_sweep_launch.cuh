// hp_sweep_launch.cuh -- tile table and launcher of the fused sweep, shared
// by the FP64 and mixed-precision translation units.
//
// A tile is (P pencils per CTA, T cells per window step, RING slots).  Along
// x a warp covers 32/T pencils x T consecutive cells; along y/z a warp
// covers 32 consecutive pencils (x) x 1 cell.  The best tile depends on the
// grid and the precision; hp_autotune measures them.
#pragma once
#include <cuda_runtime.h>

#include <atomic>

#include "hp_launch.h"
#include "hp_sweep.cuh"

namespace hp {

// Arguments of one sweep of box b along `axis`: the velocities permuted into
// (normal, transverse1, transverse2) of the sweep (ppmsolver.F90:105-107,
// 227-229, 355-357).
static inline SweepArgs make_sweep_args(const Box& b, int axis, int bslot, int flags) {
    SweepArgs a;
    a.f[0] = b.f[0];
    a.f[1] = b.f[1];
    if (axis == 0) { a.f[2] = b.f[2]; a.f[3] = b.f[3]; a.f[4] = b.f[4]; }
    if (axis == 1) { a.f[2] = b.f[3]; a.f[3] = b.f[2]; a.f[4] = b.f[4]; }
    if (axis == 2) { a.f[2] = b.f[4]; a.f[3] = b.f[3]; a.f[4] = b.f[2]; }
    for (int q = 0; q < 4; ++q) a.snap[q] = b.snap[q];
    a.peak = b.peak;
    a.g = b.g[axis];
    // halo planes in the sweep's field order (z sweep: p, rho, vz, vy, vx)
    static const int kPerm[3][5] = {{0, 1, 2, 3, 4}, {0, 1, 3, 2, 4}, {0, 1, 4, 3, 2}};
    const long long plane = (long long)b.nx * b.ny;
    for (int q = 0; q < 5; ++q) {
        a.zlo[q] = b.zlo ? b.zlo + (long long)kPerm[axis][q] * 4 * plane : nullptr;
        a.zhi[q] = b.zhi ? b.zhi + (long long)kPerm[axis][q] * 3 * plane : nullptr;
    }
    a.cho = b.cho;
    a.ctl = b.ctl;
    a.k = b.k;
    a.nx = b.nx; a.ny = b.ny; a.nz = b.nz;
    a.nsweep = axis == 0 ? b.nx : (axis == 1 ? b.ny : b.nz);
    a.npencil = axis == 0 ? (long long)b.ny * b.nz : (axis == 1 ? (long long)b.nx * b.nz : (long long)b.nx * b.ny);
    a.bslot = bslot;
    a.flags = flags;
    return a;
}

// The dynamic shared-memory size of a kernel above 48 KB must be allowed on
// every device that launches it: one bit per device ordinal, per kernel.
// Two host threads that race here both set the attribute (harmless).
static inline int current_device() {
    int dev = 0;
    return cudaGetDevice(&dev) == cudaSuccess ? dev : -1;
}
template <class Kern>
static bool allow_smem(Kern kern, size_t smem, std::atomic<unsigned long long>& done_mask) {
    const int dev = current_device();
    if (dev < 0 || dev >= 64) return false;
    const unsigned long long bit = 1ULL << dev;
    if (done_mask.load(std::memory_order_acquire) & bit) return true;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return false;
    done_mask.fetch_or(bit, std::memory_order_acq_rel);
    return true;
}

template <int AXIS, int P, int T, int RING, class Policy, int MINB = 1, bool GRAV = false, bool PENCIL = false>
static int launch_sweep_t(const Box& b, int bslot, int flags, cudaStream_t st) {
    const SweepArgs a = make_sweep_args(b, AXIS, bslot, flags);
    const size_t smem = sizeof(SweepSmem<AXIS, P, T, RING, Policy, GRAV, PENCIL>);
    auto kern = ppm_sweep_kernel<AXIS, P, T, RING, Policy, MINB, GRAV, PENCIL>;
    static std::atomic<unsigned long long> attr_mask{0};  // per instantiation, one bit per device
    if (!allow_smem(kern, smem, attr_mask)) return -1;
    const long long grid = (a.npencil + P - 1) / P;
    kern<<<(unsigned)grid, P * T, smem, st>>>(a);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

// The tile table: (axis, tile index, P, T, RING, MINB).  MINB > 1 caps the
// registers so that MINB CTAs share an SM: independent barrier domains,
// so one CTA issues while another waits at a barrier.  The pencils per
// CTA of each entry are also in kTilePencils (hp_launch.h); the
// static_asserts below keep the two in step.
#define HP_TILE_TABLE(X)                                                                       \
    X(0, 0, 8, 32, 64, 1) X(0, 1, 4, 32, 64, 1) X(0, 2, 8, 16, 32, 1) X(0, 3, 4, 16, 32, 1)    \
    X(0, 4, 16, 32, 64, 1) X(0, 5, 12, 32, 64, 1) X(0, 6, 8, 32, 64, 3) X(0, 7, 4, 32, 64, 5)  \
    X(0, 8, 8, 32, 64, 2) X(0, 9, 4, 32, 64, 4) X(0, 10, 16, 16, 32, 3)                        \
    X(1, 0, 32, 8, 16, 1) X(1, 1, 16, 8, 16, 1) X(1, 2, 32, 4, 16, 1) X(1, 3, 16, 4, 16, 1)    \
    X(1, 4, 64, 8, 16, 1) X(1, 5, 32, 12, 32, 1) X(1, 6, 32, 8, 16, 3) X(1, 7, 16, 8, 16, 5)   \
    X(1, 8, 32, 8, 16, 2) X(1, 9, 16, 8, 16, 4) X(1, 10, 16, 16, 32, 3)                         \
    X(2, 0, 32, 8, 16, 1) X(2, 1, 16, 8, 16, 1) X(2, 2, 32, 4, 16, 1) X(2, 3, 16, 4, 16, 1)    \
    X(2, 4, 64, 8, 16, 1) X(2, 5, 32, 12, 32, 1) X(2, 6, 32, 8, 16, 3) X(2, 7, 16, 8, 16, 5)   \
    X(2, 8, 32, 8, 16, 2) X(2, 9, 16, 8, 16, 4) X(2, 10, 16, 16, 32, 3)

#define HP_TILE_CHECK(AX, TI, P, T, RING, MINB) \
    static_assert(kTilePencils[AX][TI] == P, "tile table and kTilePencils disagree");
HP_TILE_TABLE(HP_TILE_CHECK)
#undef HP_TILE_CHECK

// GRAV: the instantiation with the gravity source (a box with gforce);
// PENCIL: the non-STENCIL build's full-pencil solver.
template <class Policy, bool GRAV = false, bool PENCIL = false>
static int launch_sweep_policy(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st) {
#define HP_TILE_CASE(AX, TI, P, T, RING, MINB) \
    if (axis == AX && tile == TI)                \
        return launch_sweep_t<AX, P, T, RING, Policy, MINB, GRAV, PENCIL>(b, bslot, flags, st);
    HP_TILE_TABLE(HP_TILE_CASE)
#undef HP_TILE_CASE
    return -1;
}

// Persistent batched sweep: one CTA per resident slot of the GPU (the
// occupancy of the instantiation x the SM count), each draining the queue.
template <int AXIS, int P, int T, int RING, class Policy, int MINB>
static int launch_sweep_batch_t(const BatchLaunch& bl, cudaStream_t st) {
    const size_t smem = sizeof(SweepSmem<AXIS, P, T, RING, Policy>);
    auto kern = ppm_sweep_batch_kernel<AXIS, P, T, RING, Policy, MINB>;
    // per instantiation and device: the attribute, then the resident grid
    static std::atomic<unsigned long long> attr_mask{0};
    static std::atomic<int> grids[64];
    if (!allow_smem(kern, smem, attr_mask)) return -1;
    const int dev = current_device();
    int grid = grids[dev].load(std::memory_order_acquire);
    if (grid == 0) {
        int sms = 0, per_sm = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, P * T, smem) != cudaSuccess) return -1;
        grid = sms * (per_sm > 0 ? per_sm : 1);
        grids[dev].store(grid, std::memory_order_release);
    }
    const int g = bl.nitems < grid ? bl.nitems : grid;
    if (g <= 0) return 0;
    kern<<<g, P * T, smem, st>>>(bl);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

template <class Policy>
static int launch_sweep_batch_policy(const BatchLaunch& bl, int axis, int tile, cudaStream_t st) {
#define HP_TILE_CASE(AX, TI, P, T, RING, MINB) \
    if (axis == AX && tile == TI) return launch_sweep_batch_t<AX, P, T, RING, Policy, MINB>(bl, st);
    HP_TILE_TABLE(HP_TILE_CASE)
#undef HP_TILE_CASE
    return -1;
}

}  // namespace hp
