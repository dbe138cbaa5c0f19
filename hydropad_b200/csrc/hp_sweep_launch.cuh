// hp_sweep_launch.cuh -- tile table and launcher of the fused sweep, shared
// by the FP64 and mixed-precision translation units.
//
// A tile is (P pencils per CTA, T cells per window step, RING slots).  Along
// x a warp covers 32/T pencils x T consecutive cells; along y/z a warp
// covers 32 consecutive pencils (x) x 1 cell.  The best tile depends on the
// grid and the precision; hp_autotune measures them.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>

#include "hp_launch.h"
#include "hp_sweep.cuh"
#include "hp_sweep_ws.cuh"

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
    X(0, 4, 16, 32, 64, 1) X(0, 5, 12, 32, 64, 1) X(0, 6, 8, 32, 64, 3) X(0, 7, 16, 16, 32, 4)  \
    X(0, 8, 16, 32, 64, 2) X(0, 9, 8, 32, 64, 4) X(0, 10, 16, 16, 32, 3)                        \
    X(1, 0, 32, 8, 16, 1) X(1, 1, 16, 8, 16, 1) X(1, 2, 32, 4, 16, 1) X(1, 3, 16, 4, 16, 1)    \
    X(1, 4, 64, 8, 16, 1) X(1, 5, 32, 12, 32, 1) X(1, 6, 32, 8, 16, 3) X(1, 7, 32, 8, 16, 4)   \
    X(1, 8, 64, 8, 16, 2) X(1, 9, 16, 16, 32, 4) X(1, 10, 16, 16, 32, 3)                         \
    X(2, 0, 32, 8, 16, 1) X(2, 1, 16, 8, 16, 1) X(2, 2, 32, 4, 16, 1) X(2, 3, 16, 4, 16, 1)    \
    X(2, 4, 64, 8, 16, 1) X(2, 5, 32, 12, 32, 1) X(2, 6, 32, 8, 16, 3) X(2, 7, 32, 8, 16, 4)   \
    X(2, 8, 64, 8, 16, 2) X(2, 9, 16, 16, 32, 4) X(2, 10, 16, 16, 32, 3)

#define HP_TILE_CHECK(AX, TI, P, T, RING, MINB) \
    static_assert(kTilePencils[AX][TI] == P, "tile table and kTilePencils disagree");
HP_TILE_TABLE(HP_TILE_CHECK)
#undef HP_TILE_CHECK

// ---------------------------------------------------------------------------
// The pipelined sweep (ppm_sweep_ws_kernel): tiles kNumClassicTiles.. of the
// table below, (axis, tile, P, T, NW Newton warps, MINB).
// ---------------------------------------------------------------------------
#define HP_WS_TILE_TABLE(X)                                                                   \
    X(0, 11, 4, 32, 1, 3) X(0, 12, 4, 32, 1, 2) X(0, 13, 8, 32, 1, 1)                         \
    X(1, 11, 16, 8, 1, 3) X(1, 12, 16, 8, 1, 2) X(1, 13, 16, 16, 1, 1)                        \
    X(2, 11, 16, 8, 1, 3) X(2, 12, 16, 8, 1, 2) X(2, 13, 16, 16, 1, 1)

// cuTensorMapEncodeTiled of the driver, through the runtime's entry-point
// query (the library does not link libcuda itself).
static inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// Tensor maps of the five fields of a sweep: x, the rows (nx, ny*nz) in
// boxes of T cells x P rows; y/z, the box (nx, ny, nz) in boxes of 16 x T
// (y) or 16 x 1 x T (z), 128-byte swizzled.  The maps cover this device's
// fields only; no load from them uses cluster multicast.
template <int AXIS, int P, int T>
static bool make_field_maps(const SweepArgs& a, CUtensorMap* tm) {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    for (int q = 0; q < 5; ++q) {
        CUresult r;
        if (AXIS == 0) {
            const cuuint64_t dims[2] = {(cuuint64_t)a.nx, (cuuint64_t)a.ny * (cuuint64_t)a.nz};
            const cuuint64_t strides[1] = {(cuuint64_t)a.nx * 8};
            const cuuint32_t box[2] = {(cuuint32_t)T, (cuuint32_t)P};
            const cuuint32_t es[2] = {1, 1};
            r = enc(&tm[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, a.f[q], dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        } else {
            const cuuint64_t dims[3] = {(cuuint64_t)a.nx, (cuuint64_t)a.ny, (cuuint64_t)a.nz};
            const cuuint64_t strides[2] = {(cuuint64_t)a.nx * 8, (cuuint64_t)a.nx * a.ny * 8};
            const cuuint32_t box[3] = {(cuuint32_t)P, AXIS == 1 ? (cuuint32_t)T : 1u, AXIS == 2 ? (cuuint32_t)T : 1u};
            const cuuint32_t es[3] = {1, 1, 1};
            r = enc(&tm[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, a.f[q], dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        }
        if (r != CUDA_SUCCESS) return false;
    }
    return true;
}

// Whether the pipelined sweep takes this sweep: no gravity source, the
// STENCIL sweep, not a z slab, rows that TMA can address in 16-byte units
// (nx even), and along y/z groups of 16 pencils within one x row.
static inline bool ws_takes(const Box& b, int axis, int flags) {
    if (b.g[0] || b.pencil || (flags & kFlagZHalo)) return false;
    if (b.nx % 2) return false;
    if (axis != 0 && b.nx % 16) return false;
    for (int q = 0; q < 5; ++q)
        if (reinterpret_cast<uintptr_t>(b.f[q]) % 16) return false;
    return true;
}

template <int AXIS, int P, int T, int NW, class Policy, int MINB>
static int launch_sweep_ws_t(const Box& b, int bslot, int flags, cudaStream_t st) {
    using Smem = WsSmem<AXIS, P, T, NW, Policy>;
    using L = WsLayout<AXIS, P, T, NW>;
    WsArgs wa;
    memset(&wa, 0, sizeof wa);
    // the failure-detection test (tests/test_gpu_ws_timeout.py) withholds a
    // completion so that a bounded wait runs out
    const char* withhold = getenv("HP_TEST_WITHHOLD_NEWTON");
    if (withhold && withhold[0] == '1') flags |= kFlagTestWithhold;
    wa.a = make_sweep_args(b, AXIS, bslot, flags);
    if (!make_field_maps<AXIS, P, T>(wa.a, wa.tm)) return -1;
    wa.ngroups = (wa.a.npencil + P - 1) / P;
    wa.wpg = (wa.a.nsweep + 7) / T + 1;  // windows b = -4 + wT up to b <= N + 3
    const size_t smem = sizeof(Smem) + 1024;  // + the 1024-byte alignment of the TMA rows
    auto kern = ppm_sweep_ws_kernel<AXIS, P, T, NW, Policy, MINB>;
    static std::atomic<unsigned long long> attr_mask{0};
    static std::atomic<int> grids[64];
    if (!allow_smem(kern, smem, attr_mask)) return -1;
    const int dev = current_device();
    int grid = grids[dev].load(std::memory_order_acquire);
    if (grid == 0) {
        int sms = 0, per_sm = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, L::kThreads, smem) != cudaSuccess)
            return -1;
        grid = sms * (per_sm > 0 ? per_sm : 1);
        grids[dev].store(grid, std::memory_order_release);
    }
    const long long g = wa.ngroups < grid ? wa.ngroups : grid;
    if (g <= 0) return 0;
    kern<<<(unsigned)g, L::kThreads, smem, st>>>(wa);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

// GRAV: the instantiation with the gravity source (a box with gforce);
// PENCIL: the non-STENCIL build's full-pencil solver.
template <class Policy, bool GRAV = false, bool PENCIL = false>
static int launch_sweep_policy(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st) {
    if (tile >= kNumClassicTiles) {
        if constexpr (!GRAV && !PENCIL) {
            if (ws_takes(b, axis, flags)) {
#define HP_WS_CASE(AX, TI, P, T, NW, MINB) \
    if (axis == AX && tile == TI) return launch_sweep_ws_t<AX, P, T, NW, Policy, MINB>(b, bslot, flags, st);
                HP_WS_TILE_TABLE(HP_WS_CASE)
#undef HP_WS_CASE
                return -1;
            }
        }
        tile = 0;  // a box the pipelined sweep does not take: the same bits from tile 0
    }
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
