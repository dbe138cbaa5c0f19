// hp_launch.h -- host-side launch interface between the C ABI and the
// kernels (internal; not part of the public header).
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "hp_device.cuh"

namespace hp {

// NVTX range over a host-side scope (a sweep, a step, a batch step, a host
// transfer): the timeline of a profiler groups the launches under it.  The
// calls cost nothing measurable when no tool is attached.
struct TraceRange {
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};

// One box resident on the device.
struct Box {
    double* f[5];      // p, rho, vx, vy, vz (natural order), dense (nx,ny,nz), x fastest
    void* snap[4];     // step-start p, vx, vy, vz (cosmo expand): double (FP64 path) or float (mixed), or null
    double* peak;      // density-peak values of the y/z faces (nx*ny*nz + nx*max(ny,nz)), or null
    double* g[3];      // gforce components x, y, z (dense, natural layout), or null: gravity off
    double* zlo;       // slab of a z-split box: 4 halo planes below, [p,rho,vx,vy,vz][4][nx*ny], or null
    double* zhi;       // 3 halo planes above, [5][3][nx*ny], or null
    const double* cho; // cho3d marker of each cell for the full-pencil solver (dense), or null: zeros
    DevCtl* ctl;       // device control block
    Consts k;
    int nx, ny, nz;
    int pencil;        // 1: the non-STENCIL build's full-pencil solver (hydro/ppm.F90); FP64 only
};

// Launches return the number of kernels launched (>= 0) or -1 on a launch error.
int launch_sweep(const Box& b, int axis, int tile, int bslot, int flags, int precision, cudaStream_t st);
int launch_peak_prepass(const Box& b, int axis, int bslot, cudaStream_t st);
int launch_bounds(const Box& b, int slot, cudaStream_t st);
int launch_speed(const Box& b, cudaStream_t st);
int launch_timedet(const Box& b, int advance, cudaStream_t st);

// Number of tile shapes per axis, and the pencils per CTA (P) of each
// (the tile tables in hp_sweep_launch.cuh): tiles 0 .. kNumClassicTiles-1
// run ppm_sweep_kernel (and the batched kernel), the others the pipelined
// ppm_sweep_ws_kernel (single boxes; a box it does not take -- gravity, the
// full-pencil solver, a z slab, a row length it cannot tile -- runs tile 0).
constexpr int kNumClassicTiles = 11;
constexpr int kNumWsTiles = 3;
constexpr int kNumTiles = kNumClassicTiles + kNumWsTiles;
constexpr int kTilePencils[3][kNumClassicTiles] = {{8, 4, 8, 4, 16, 12, 8, 16, 16, 8, 16},
                                            {32, 16, 32, 16, 64, 32, 32, 32, 64, 16, 16},
                                            {32, 16, 32, 16, 64, 32, 32, 32, 64, 16, 16}};

struct BatchLaunch;  // hp_sweep.cuh

// Batched sweep over many boxes (one axis per launch); the counter must be
// zero when the launch starts.
int launch_sweep_batch(const BatchLaunch& bl, int axis, int tile, int precision, cudaStream_t st);
// Peak pre-pass of the boxes of one y/z batch launch.
int launch_peak_prepass_batch(const BatchLaunch& bl, int axis, cudaStream_t st);
// timedet (advance = 1) on n control blocks.
int launch_timedet_batch(DevCtl* const* ctls, int n, cudaStream_t st);
// in = (3, n) interleaved (gforce(3,nx,ny,nz) interior) -> g0, g1, g2.
int launch_deinterleave3(const double* in, double* g0, double* g1, double* g2, long long n, cudaStream_t st);
// Ghosted host-layout planes (contiguous, staged on the device) <-> a dense
// field: the interior of planes zf0.. of the field from `stage`, or the
// ghosted planes zg0.. (periodic ghosts filled) of the field into `stage`.
int launch_planes_to_field(const double* stage, double* f, int nx, int ny, int nb, int zf0, int nplanes,
                           cudaStream_t st);
int launch_field_to_planes(const double* f, double* stage, int nx, int ny, int nz, int nb, int zg0, int nplanes,
                           cudaStream_t st);
// out[i] = (float)in[i], round to nearest even.
int launch_to_f32(const double* in, float* out, long long n, cudaStream_t st);
// out[i] = status word of ctls[i], which is cleared.
int launch_status_gather(DevCtl* const* ctls, int n, unsigned* out, cudaStream_t st);

}  // namespace hp
