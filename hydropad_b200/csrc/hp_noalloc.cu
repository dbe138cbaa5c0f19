// hp_noalloc.cu -- one directional sweep without any device allocation.
//
// Some callers cannot call cudaMalloc: a Fortran or C host that owns every
// device array itself (its OpenACC or CUDA data regions hold the state) and
// budgets the device memory on its own, a process whose device memory is
// capped (an MPS client with a memory limit), or a framework whose caching
// allocator owns the device and forbids foreign allocations.
// hp_ppmsolver_noalloc serves them: the caller passes the five state arrays
// (device memory), and every scratch byte the sweep needs -- the control
// block with the time scalars, the rho bounds and the status word, and the
// density-peak values of the y/z faces -- lives in one file-scope
// __device__ array of a fixed size, reserved once per device when the
// library's module is loaded and held until the process exits.
//
// The array is shared by every call: calls that overlap on the GPU (two
// streams, or two host threads) race on it.  Each call re-initialises the
// control block before its kernels run.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <atomic>

#include "../../include/hydropad_b200.h"
#include "hp_device.cuh"
#include "hp_launch.h"

namespace {

// Largest box the entry point accepts, in cells (1,048,576: e.g. 128x128x64
// or 101^3).  The density-peak values need one double per cell plus one per
// pencil of the y/z sweeps (at most cells/8, since every side is >= 8).
constexpr long long kNoAllocMaxCells = 1LL << 20;
constexpr long long kNoAllocPeakSlots = kNoAllocMaxCells + kNoAllocMaxCells / 8;
constexpr size_t kCtlBytes = 4096;  // control block, padded
static_assert(sizeof(hp::DevCtl) <= kCtlBytes, "control block does not fit");

// The scratch array (9 MiB + 4 KiB per device).
static __device__ __align__(256) unsigned char g_hp_noalloc_scratch[kCtlBytes + kNoAllocPeakSlots * sizeof(double)];

// Device address of the array, per device ordinal; filled on the first call
// with that device current.  In host code the symbol itself is only a
// host-side stand-in.  Two host threads making their first call at once
// both look the address up and store the same value.
constexpr int kMaxDevices = 64;
std::atomic<void*> g_scratch_addr[kMaxDevices];

// Initialise the control block of this call from kernel arguments (no
// memcpy from the host): time scalars, the bound slots, status and the
// velmax accumulator all start from a known state.
__global__ void noalloc_ctl_init(hp::DevCtl* c, hp::StepScalars s, double tstop) {
    hp::DevCtl z;
    memset(&z, 0, sizeof z);
    z.s = s;
    z.tstop = tstop;
    z.told = 0.0;  // the sweep only needs `done == 0`
    z.done = 0;
    for (int q = 0; q < 3; ++q) {
        z.rho_key[q][0] = hp::kKeyPosInf;
        z.rho_key[q][1] = hp::kKeyNegInf;
    }
    z.bad_cell = -1;
    *c = z;
}

int noalloc_status(unsigned st) {
    if (st & hp::kStatNewton) return HP_ERR_NEWTON;
    if (st & hp::kStatNaN) return HP_ERR_NAN;
    if (st & hp::kStatNegative) return HP_ERR_NEGATIVE_STATE;
    return HP_OK;
}

}  // namespace

extern "C" int hp_ppmsolver_noalloc(double* p, double* rho, double* vx, double* vy, double* vz, int nx, int ny,
                                    int nz, int ndirection, const hp_params* params, const hp_scalars* scalars,
                                    void* stream) {
    if (!p || !rho || !vx || !vy || !vz || !params || !scalars) return HP_ERR_ARG;
    if (ndirection < 1 || ndirection > 3 || nx < 8 || ny < 8 || nz < 8) return HP_ERR_ARG;
    if ((long long)nx * ny * nz > kNoAllocMaxCells) return HP_ERR_ARG;  // larger than the static scratch
    if (params->precision != HP_PREC_FP64 && params->precision != HP_PREC_MIXED) return HP_ERR_ARG;
    if (params->nbound < 3) return HP_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return HP_ERR_NO_DEVICE;
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess || major != 10)
        return HP_ERR_NO_DEVICE;
    // First call on this device (with it current): look up the array's
    // device address.  Later calls reuse it.
    void* addr = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!addr) {
        if (cudaGetSymbolAddress(&addr, g_hp_noalloc_scratch) != cudaSuccess || !addr) return HP_ERR_CUDA;
        g_scratch_addr[dev].store(addr, std::memory_order_release);
    }
    unsigned char* scratch = static_cast<unsigned char*>(addr);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    hp::Box b;
    memset(&b, 0, sizeof b);
    b.f[0] = p;
    b.f[1] = rho;
    b.f[2] = vx;
    b.f[3] = vy;
    b.f[4] = vz;
    b.ctl = reinterpret_cast<hp::DevCtl*>(scratch);
    b.peak = reinterpret_cast<double*>(scratch + kCtlBytes);
    b.nx = nx;
    b.ny = ny;
    b.nz = nz;
    // constants derived as initialize_parameters.F90:23-24,63-69
    hp::Consts& k = b.k;
    const int nmax = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
    const double g = params->gamma;
    k.dx = 1.0 / (double)nmax;
    k.rdx = 1.0 / k.dx;
    k.gamma = g;
    k.rgamma = 1.0 / g;
    k.gamma1 = (g + 1.0) / (g - 1.0);
    k.rgamma1 = 1.0 / (g - 1.0);
    k.m = (g - 1.0) / (2.0 * g);
    k.rm = 1.0 / k.m;
    k.gf = (g + 1.0) / (2.0 * g);
    k.mingradflat = params->mingradflat;
    k.flatvalue = params->flatvalue;
    k.dmax = params->dmax;
    k.eta1 = params->eta1;
    k.eta2 = params->eta2;
    k.nbound = params->nbound;
    k.nroot = 0;
    k.jrg = 0;
    const double n = k.rm, j = k.rgamma * k.rm;
    if (n == floor(n) && n >= 2.0 && n <= 9.0) {
        k.nroot = (int)n;
        if (fabs(j - rint(j)) < 1e-12 && j >= 1.0 && j <= 9.0) k.jrg = (int)rint(j);
    }
    hp::set_float_consts(k);

    hp::StepScalars sc;
    sc.dt = scalars->dt;
    sc.rdtath = scalars->rdtath;
    sc.at = scalars->at;
    sc.dat = scalars->dat;
    sc.rat = scalars->rat;
    sc.ath = scalars->ath;
    sc.dath = scalars->dath;
    const double tstop = params->tstop > 0.0 ? params->tstop : 1.0e300;

    // control block, rho bounds of the input (slot 0), density-peak
    // pre-pass (only when the bounds admit a peak), the fused sweep
    noalloc_ctl_init<<<1, 1, 0, st>>>(b.ctl, sc, tstop);
    if (cudaPeekAtLastError() != cudaSuccess) return HP_ERR_CUDA;
    if (hp::launch_bounds(b, 0, st) < 0) return HP_ERR_CUDA;
    const int axis = ndirection - 1;
    if (hp::launch_peak_prepass(b, axis, 0, st) < 0) return HP_ERR_CUDA;
    if (hp::launch_sweep(b, axis, 0, 0, 0, params->precision, st) < 0) return HP_ERR_CUDA;
    unsigned status = 0;
    if (cudaMemcpyAsync(&status, &b.ctl->status, sizeof status, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return HP_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return HP_ERR_CUDA;
    return noalloc_status(status);
}
