// hp_device.cuh -- device-resident control block and reduction helpers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "hp_physics.cuh"

namespace hp {

// Status bits accumulated by the kernels (see HP_ERR_* in the C header).
enum : unsigned {
    kStatNewton = 1u,    // Newton for p* exceeded 100 iterations
    kStatNaN = 2u,       // NaN in an updated cell
    kStatNegative = 4u,  // rho <= 0 or p <= 0 in an updated cell
    kStatUnsupported = 8u,  // a case the sweep cannot take (the density-peak fix across z slabs)
    kStatTimeout = 16u,     // a bounded wait of the pipelined sweep gave up (its results are void)
};

// Sweep flags.
enum : int {
    kFlagSnapshot = 1,     // store the step-start p, v (cosmo expand)
    kFlagExpand = 2,       // apply expand.F90 to the updated cells
    kFlagSpeed = 4,        // accumulate velmax of the updated cells
    kFlagResetSpeed = 8,   // zero the velmax accumulator (first sweep of a step)
    kFlagExpandZeroOld = 16,  // expand with vxold = pold3d = 0 (as alloc_arrays.F90:71-74,132-135 leaves them)
    kFlagZHalo = 32,       // z sweep of a slab: the cells beyond its ends come from halo planes
    // failure-detection test of the pipelined sweep: its Newton warps withhold
    // the completion of their first window, so that the main group's bounded
    // wait runs out (set only when HP_TEST_WITHHOLD_NEWTON=1 in the environment)
    kFlagTestWithhold = 64,
};

// Time scalars + bookkeeping, one per box, in device memory so that a whole
// step (sweeps, CFL reduction, timedet) runs without the host.
struct DevCtl {
    StepScalars s;                 // dt, rdtath, at, dat, rat, ath, dath of the current step
    double t, told, thalf, dtold, atnew, datnew, tstop, velmax;
    int nstep;
    int cosmo;
    double cour, ca, dx, dt_cap;
    unsigned long long rho_key[3][2];  // ordered-key min/max of rho, ring of 3 sweep slots
    unsigned long long velmax_key;     // bits of a non-negative double (max accumulator)
    unsigned int status;
    int done;                          // told >= tstop: further steps are no-ops
    // dense index of the first updated cell found with a NaN or a
    // non-positive density or pressure since the status word was last read
    // (-1: none); read together with `status`
    long long bad_cell;
};

// A sweep found cell g of the box non-physical: keep the first such cell.
__device__ __forceinline__ void record_bad_cell(DevCtl* c, long long g) {
    atomicCAS(reinterpret_cast<unsigned long long*>(&c->bad_cell), ~0ULL, (unsigned long long)g);
}

// Order-preserving map double -> uint64 (valid for every non-NaN double).
__device__ __forceinline__ unsigned long long dkey(double x) {
    unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}
__device__ __forceinline__ double dkey_decode(unsigned long long k) {
    unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffULL) : ~k;
    return __longlong_as_double((long long)b);
}
constexpr unsigned long long kKeyPosInf = 0xfff0000000000000ULL;  // dkey(+inf)
constexpr unsigned long long kKeyNegInf = 0x000fffffffffffffULL;  // dkey(-inf)

template <class T>
__device__ __forceinline__ T warp_min(T v) {
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}
template <class T>
__device__ __forceinline__ T warp_max(T v) {
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Block-wide reduction of (min key, max key, velmax key, status) followed by
// one atomic per quantity.  Every thread of the block must call it.
__device__ __forceinline__ void block_flush(unsigned long long kmin, unsigned long long kmax,
                                            unsigned long long kvel, unsigned status,
                                            unsigned long long* gmin, unsigned long long* gmax,
                                            unsigned long long* gvel, unsigned* gstatus,
                                            unsigned long long* red /* smem, >= 4*32 */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    kmin = warp_min(kmin);
    kmax = warp_max(kmax);
    kvel = warp_max(kvel);
    status = __reduce_or_sync(0xffffffffu, status);
    __syncthreads();
    if (lane == 0) {
        red[warp] = kmin;
        red[32 + warp] = kmax;
        red[64 + warp] = kvel;
        red[96 + warp] = status;
    }
    __syncthreads();
    if (warp == 0) {
        kmin = lane < nw ? red[lane] : kKeyPosInf;
        kmax = lane < nw ? red[32 + lane] : 0ULL;
        kvel = lane < nw ? red[64 + lane] : 0ULL;
        status = lane < nw ? (unsigned)red[96 + lane] : 0u;
        kmin = warp_min(kmin);
        kmax = warp_max(kmax);
        kvel = warp_max(kvel);
        status = __reduce_or_sync(0xffffffffu, status);
        if (lane == 0) {
            if (gmin) atomicMin(gmin, kmin);
            if (gmax) atomicMax(gmax, kmax);
            if (gvel) atomicMax(gvel, kvel);
            if (status) atomicOr(gstatus, status);
        }
    }
}

}  // namespace hp
