// hp_ctx.h -- the single-box context behind the C ABI (internal).
#pragma once
#include <cuda_runtime.h>

#include "../../include/hydropad_b200.h"
#include "hp_device.cuh"
#include "hp_launch.h"

struct hp_ctx {
    hp_params prm;
    int dev;
    cudaStream_t stream;
    hp::Box box;
    hp::DevCtl* ctl_pinned;   // host mirror for reads
    long long sweep_count;    // selects the rho-bound slot
    long long nstep_host;     // host mirror of the step counter (selects nrot)
    const double* host[5];    // attached host arrays (ghosted, Fortran order)
    const double* host_g;     // attached host gforce (3,nx,ny,nz), or null
    int hnx, hny, hnz, hnb;
    bool attached;
    int tile[3];              // sweep tile shape per axis (hp_set_tiles / hp_autotune)
    cudaGraphExec_t graph[6][3];
    int graph_kernels[6][3];
    long long launches;
    double* stage;            // device staging of host-layout planes (host transfers), or null
    size_t stage_bytes;
    int slab;                 // 1: a z slab of a larger periodic box (hp_slab_init)
    int nz_global, z0;
    double* cho_dev;          // attached cho3d (dense) for the full-pencil solver, or null
    const double* host_cho;   // the attached host cho3d array, or null
    long long last_bad_cell;  // first bad cell of the last non-zero status read (hp_bad_cell), or -1
};

namespace hp {
// Sweep order of ppm_lxlylz for nrot = 1..6 (0 = x): xyz, zyx, yzx, xzy, zxy, yxz.
constexpr int kSweepOrder[6][3] = {{0, 1, 2}, {2, 1, 0}, {1, 2, 0}, {0, 2, 1}, {2, 0, 1}, {1, 0, 2}};

// Error code of a device status word.
inline int status_error(unsigned st) {
    if (st & kStatTimeout) return HP_ERR_TIMEOUT;
    if (st & kStatNewton) return HP_ERR_NEWTON;
    if (st & kStatNaN) return HP_ERR_NAN;
    if (st & kStatNegative) return HP_ERR_NEGATIVE_STATE;
    if (st & kStatUnsupported) return HP_ERR_UNSUPPORTED;
    return HP_OK;
}

// nrot of a step (evolve_sys.F90:30-31).
inline int nrot_of_step(long long nstep) { return nstep == 1 ? 1 : (int)(nstep % 6) + 1; }

// Sweep flags of slot s (0..2) of a step: the first sweep zeroes the velmax
// accumulator and snapshots the state for expand, the last applies expand
// and accumulates velmax.
inline int step_flags(const hp_params& p, int s) {
    int flags = 0;
    if (s == 0) {
        flags |= kFlagResetSpeed;
        if (p.cosmo && !p.expand_zero_old) flags |= kFlagSnapshot;
    }
    if (s == 2) {
        flags |= kFlagSpeed;
        if (p.cosmo) flags |= kFlagExpand | (p.expand_zero_old ? kFlagExpandZeroOld : 0);
    }
    return flags;
}
}  // namespace hp
