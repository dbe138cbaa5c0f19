// hp_kernels_fp64.cu -- FP64 sweep instantiations and the small per-step
// kernels (rho bounds, CFL speed, timedet, density-peak pre-pass).
//
// Compiled with --fmad=false: every FP64 operation rounds once, like the
// reference's scalar Fortran, so the FP64 path reproduces the oracle to the
// last bit except where CUDA's pow differs from the host libm by an ulp.
#include <cuda_runtime.h>

#include "hp_device.cuh"
#include "hp_launch.h"
#include "hp_physics.cuh"
#include "hp_sweep.cuh"
#include "hp_sweep_launch.cuh"

namespace hp {

int launch_sweep_grav_fp64(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st);
int launch_sweep_pencil_fp64(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st);

int launch_sweep_fp64(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st) {
    // the full-pencil solver ignores gforce (ppm.F90:93,102)
    if (b.pencil) return launch_sweep_pencil_fp64(b, axis, tile, bslot, flags, st);
    if (b.g[0]) return launch_sweep_grav_fp64(b, axis, tile, bslot, flags, st);
    return launch_sweep_policy<PolicyFP64>(b, axis, tile, bslot, flags, st);
}

// ---------------------------------------------------------------------------
// rho bounds of the resident state into slot `slot`; the other two slots are
// reset.  Feeds the density-peak test of the next sweep.
// ---------------------------------------------------------------------------
__global__ void bounds_reset_kernel(DevCtl* c, int slot) {
    for (int s = 0; s < 3; ++s) {
        c->rho_key[s][0] = kKeyPosInf;
        c->rho_key[s][1] = kKeyNegInf;
    }
    (void)slot;
}

__global__ void bounds_kernel(const double* __restrict__ rho, long long n, DevCtl* c, int slot) {
    __shared__ unsigned long long red[128];
    unsigned long long kmin = kKeyPosInf, kmax = 0ULL;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long kk = dkey(rho[i]);
        kmin = kk < kmin ? kk : kmin;
        kmax = kk > kmax ? kk : kmax;
    }
    block_flush(kmin, kmax, 0ULL, 0u, &c->rho_key[slot][0], &c->rho_key[slot][1], nullptr, &c->status, red);
}

int launch_bounds(const Box& b, int slot, cudaStream_t st) {
    const long long n = (long long)b.nx * b.ny * b.nz;
    bounds_reset_kernel<<<1, 1, 0, st>>>(b.ctl, slot);
    bounds_kernel<<<296, 256, 0, st>>>(b.f[1], n, b.ctl, slot);
    return cudaPeekAtLastError() == cudaSuccess ? 2 : -1;
}

// ---------------------------------------------------------------------------
// speed.F90:17-31: velmax over the resident state (accumulator zeroed first).
// (The sweep's epilogue computes the same maximum for hp_evolve; this kernel
// serves hp_speed.)
// ---------------------------------------------------------------------------
__global__ void speed_kernel(const double* __restrict__ p, const double* __restrict__ rho,
                             const double* __restrict__ vx, const double* __restrict__ vy,
                             const double* __restrict__ vz, long long n, double gamma, DevCtl* c) {
    __shared__ unsigned long long red[128];
    unsigned long long kvel = 0ULL;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double vs = sqrt(gamma * p[i] / rho[i]);
        double vm = fabs(vx[i]) + vs;
        vm = fmax2(vm, fabs(vy[i]) + vs);
        vm = fmax2(vm, fabs(vz[i]) + vs);
        const unsigned long long kb = (unsigned long long)__double_as_longlong(vm);
        kvel = kb > kvel ? kb : kvel;
    }
    block_flush(kKeyPosInf, 0ULL, kvel, 0u, nullptr, nullptr, &c->velmax_key, &c->status, red);
}

int launch_speed(const Box& b, cudaStream_t st) {
    const long long n = (long long)b.nx * b.ny * b.nz;
    if (cudaMemsetAsync(&b.ctl->velmax_key, 0, sizeof(unsigned long long), st) != cudaSuccess) return -1;
    speed_kernel<<<296, 256, 0, st>>>(b.f[0], b.f[1], b.f[2], b.f[3], b.f[4], n, b.k.gamma, b.ctl);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

// ---------------------------------------------------------------------------
// timedet (functions.F90:2-35) / timedet_cosmo (functions.F90:38-151, EdS)
// on the device control block, with velmax from the accumulator.  Advances
// the step counter (when `advance`: the end of an evolve_sys step) and
// raises `done` when told reaches tstop (main.F90:100).
// ---------------------------------------------------------------------------
constexpr double kC0P1 = 0.10000000149011612;   // 0.1 (functions.F90:21,96)
constexpr double kTwo3 = 0.6666666865348816;    // 2.0/3.0 as REAL(4)
constexpr double kMThird = -0.3333333432674408; // -1.0/3.0 as REAL(4)

__device__ void timedet_one(DevCtl* c, int advance) {
    if (c->done) return;
    const double velmax = __longlong_as_double((long long)c->velmax_key);
    c->velmax = velmax;
    if (!c->cosmo) {
        c->s.at = 1.0;
        c->s.ath = 1.0;
        c->s.dat = 0.0;
        c->told = c->t;
        c->dtold = c->s.dt;
        const double rdtc = velmax / (c->cour * c->dx);
        if (velmax == 0.0) c->s.dt = kC0P1;
        else c->s.dt = 1.0 / rdtc;
        c->t = c->t + c->s.dt;
        if (c->t > c->tstop) {
            c->t = c->tstop;
            c->s.dt = c->t - c->told;
        }
        const double dth = 0.5 * c->s.dt;
        c->thalf = c->told + dth;
        c->s.rdtath = c->s.dt / c->s.ath;
    } else {
        c->told = c->t;
        c->dtold = c->s.dt;
        const double rdt = c->nstep > 1 ? 5.0 / (6.0 * c->s.dt) : 0.0;
        c->s.at = pow(c->t, kTwo3);
        c->s.dat = kTwo3 * pow(c->t, kMThird);
        const double dta = pow((1.0 + c->ca) * c->s.at, 1.5) - c->t;
        c->s.rat = 1.0 / c->s.at;
        const double rdtc = velmax / (c->cour * c->dx * c->s.at);
        double dt = 1.0 / fmax2(rdt, rdtc);
        dt = fmin2(dt, dta);
        if (dt >= 10.0) dt = kC0P1;
        if (c->dt_cap > 0.0) dt = fmin2(dt, c->dt_cap);
        c->s.dt = dt;
        c->t = c->t + c->s.dt;
        if (c->t > c->tstop) {
            c->t = c->tstop;
            c->s.dt = c->t - c->told;
        }
        const double dth = 0.5 * c->s.dt;
        c->thalf = c->told + dth;
        c->atnew = pow(c->t, kTwo3);
        c->s.ath = pow(c->thalf, kTwo3);
        c->s.dath = kTwo3 * pow(c->thalf, kMThird);
        c->datnew = kTwo3 * pow(c->t, kMThird);
        c->s.rdtath = c->s.dt / c->s.ath;
    }
    if (advance) c->nstep += 1;
    if (!(c->told < c->tstop)) c->done = 1;
}

__global__ void timedet_kernel(DevCtl* c, int advance) { timedet_one(c, advance); }

// One thread per box of a batch, at the end of a step.
__global__ void timedet_batch_kernel(DevCtl* const* __restrict__ ctls, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) timedet_one(ctls[i], 1);
}

int launch_timedet_batch(DevCtl* const* ctls, int n, cudaStream_t st) {
    if (n <= 0) return 0;
    timedet_batch_kernel<<<(n + 127) / 128, 128, 0, st>>>(ctls, n);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

__global__ void deinterleave3_kernel(const double* __restrict__ in, double* __restrict__ g0,
                                     double* __restrict__ g1, double* __restrict__ g2, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        g0[i] = in[3 * i];
        g1[i] = in[3 * i + 1];
        g2[i] = in[3 * i + 2];
    }
}

int launch_deinterleave3(const double* in, double* g0, double* g1, double* g2, long long n, cudaStream_t st) {
    deinterleave3_kernel<<<592, 256, 0, st>>>(in, g0, g1, g2, n);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

// Host-layout planes <-> dense device field.  A ghosted host array is
// (nxg, nyg, nzg) with nb ghost layers per side, x fastest; `stage` holds
// the ghosted planes zg0 .. zg0+nplanes-1 of it contiguously.
__global__ void planes_to_field_kernel(const double* __restrict__ stage, double* __restrict__ f, int nx, int ny,
                                       int nb, int zf0, int nplanes) {
    const int nxg = nx + 2 * nb, nyg = ny + 2 * nb;
    const long long n = (long long)nx * ny * nplanes;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % nx);
        const int j = (int)((t / nx) % ny);
        const int kz = (int)(t / ((long long)nx * ny));
        f[i + (long long)nx * (j + (long long)ny * (zf0 + kz))] =
            stage[(i + nb) + (long long)nxg * ((j + nb) + (long long)nyg * kz)];
    }
}

// The ghosted planes zg0 .. zg0+nplanes-1 of a field, periodic ghosts
// included (the exchange_mesh fill of a single rank, exchange_mesh.F90:23-41).
__global__ void field_to_planes_kernel(const double* __restrict__ f, double* __restrict__ stage, int nx, int ny,
                                       int nz, int nb, int zg0, int nplanes) {
    const int nxg = nx + 2 * nb, nyg = ny + 2 * nb;
    const long long n = (long long)nxg * nyg * nplanes;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int ig = (int)(t % nxg);
        const int jg = (int)((t / nxg) % nyg);
        const int kz = (int)(t / ((long long)nxg * nyg));
        const int i = ((ig - nb) % nx + nx) % nx;
        const int j = ((jg - nb) % ny + ny) % ny;
        const int k = ((zg0 + kz - nb) % nz + nz) % nz;
        stage[t] = f[i + (long long)nx * (j + (long long)ny * k)];
    }
}

int launch_planes_to_field(const double* stage, double* f, int nx, int ny, int nb, int zf0, int nplanes,
                           cudaStream_t st) {
    planes_to_field_kernel<<<1184, 256, 0, st>>>(stage, f, nx, ny, nb, zf0, nplanes);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}
int launch_field_to_planes(const double* f, double* stage, int nx, int ny, int nz, int nb, int zg0, int nplanes,
                           cudaStream_t st) {
    field_to_planes_kernel<<<1184, 256, 0, st>>>(f, stage, nx, ny, nz, nb, zg0, nplanes);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

// FP64 -> FP32, round to nearest even (Fortran REAL() of a REAL(8), the
// conversion write_var_mpi.F90:55 applies before writing).
__global__ void to_f32_kernel(const double* __restrict__ in, float* __restrict__ out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = __double2float_rn(in[i]);
}

int launch_to_f32(const double* in, float* out, long long n, cudaStream_t st) {
    to_f32_kernel<<<592, 256, 0, st>>>(in, out, n);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

// Status words of a batch's boxes into out[], each cleared.
__global__ void status_gather_kernel(DevCtl* const* __restrict__ ctls, int n, unsigned* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        out[i] = ctls[i]->status;
        ctls[i]->status = 0u;
        ctls[i]->bad_cell = -1;
    }
}

int launch_status_gather(DevCtl* const* ctls, int n, unsigned* out, cudaStream_t st) {
    if (n <= 0) return 0;
    status_gather_kernel<<<(n + 127) / 128, 128, 0, st>>>(ctls, n, out);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

int launch_timedet(const Box& b, int advance, cudaStream_t st) {
    timedet_kernel<<<1, 1, 0, st>>>(b.ctl, advance);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

// ---------------------------------------------------------------------------
// Density-peak pre-pass for y/z sweeps.  The reference gathers the peak test
// with the x-index slot in every direction (ppmsolver.F90:251-252 for y,
// :379-380 for z): for the y face i (between cells i-1 and i of the pencil
// (x, z)) it reads rho3d(iaux, x, z) and vy3d(iaux, x, z), for the z face
// rho3d(iaux, y, x) and vz3d, iaux = i-3 .. i, in its ghosted arrays
// (nx+2nb, ny+2nb, nz+2nb), x fastest, whose ghost layers hold periodic
// copies of the interior (exchange_mesh after every sweep).  Those cells
// belong to other pencils, which the in-place sweep updates concurrently, so
// the values are evaluated here on the pre-sweep state.  The gather is the
// reference's linear index: a column index beyond the ghosted extent runs on
// into the next row or plane (non-cubic boxes), and an index past the end
// of the array reads nothing (NaN: the peak test is false).  Each linear
// index is mapped back to the interior cell whose copy the reference array
// holds there.  Runs only when the rho bounds admit a peak.
//
// Layout of `peak`: the value of face f < N of the pencil at the cell index
// of its right cell f, the last face (f = N) at ncell + pencil.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void peak_prepass_box(const double* __restrict__ rho, const double* __restrict__ vn,
                                                 double* peak, int nx, int ny, int nz, int axis, double dmax,
                                                 int nb, const DevCtl* c, int bslot, long long i0, long long di) {
    const double rmin0 = dkey_decode(c->rho_key[bslot][0]);
    const double rmax0 = dkey_decode(c->rho_key[bslot][1]);
    if (!(rmax0 > dmax * rmin0) || c->done) return;
    const long long n = (long long)nx * ny * nz;
    const long long npencil = axis == 1 ? (long long)nx * nz : (long long)nx * ny;
    const int nsweep = axis == 1 ? ny : nz;
    const long long gx = nx + 2 * nb, gy = ny + 2 * nb, gz = nz + 2 * nb;
    const long long gtot = gx * gy * gz;
    for (long long i = i0; i < n + npencil; i += di) {
        // face f of the pencil whose transverse cell is (x, t): t = z (y sweep) or y (z sweep)
        int x, t, f;
        if (i < n) {
            x = (int)(i % nx);
            const int y = (int)((i / nx) % ny);
            const int z = (int)(i / ((long long)nx * ny));
            if (axis == 1) { f = y; t = z; }
            else { f = z; t = y; }
        } else {
            const long long pid = i - n;
            x = (int)(pid % nx);
            t = (int)(pid / nx);
            f = nsweep;
        }
        // 0-based linear index of rho3d(iaux, x', t') with the ghosted
        // column x' = x + nb (+1 in Fortran) in the row slot (y sweep) or
        // the plane slot (z sweep)
        const long long rowplane = axis == 1 ? ((long long)(x + nb) + gy * (t + nb)) : ((long long)(t + nb) + gy * (x + nb));
        double r[4], u[4];
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            const long long q = (long long)(f + nb - 3 + o) + gx * rowplane;  // iaux - 1 = f + nb + o - 3
            if (q < 0 || q >= gtot) {
                r[o] = u[o] = __longlong_as_double(0x7ff8000000000000ULL);
                continue;
            }
            const long long a = q % gx, bq = (q / gx) % gy, cq = q / (gx * gy);
            const long long ia = ((a - nb) % nx + nx) % nx;
            const long long ib = ((bq - nb) % ny + ny) % ny;
            const long long ic = ((cq - nb) % nz + nz) % nz;
            const long long cell = ia + (long long)nx * (ib + (long long)ny * ic);
            r[o] = rho[cell];
            u[o] = vn[cell];
        }
        peak[i] = peak_value(r[0], r[1], r[2], r[3], u[1], u[2], dmax);
    }
}

__global__ void peak_prepass_kernel(const double* __restrict__ rho, const double* __restrict__ vn, double* peak,
                                    int nx, int ny, int nz, int axis, double dmax, int nb, const DevCtl* c,
                                    int bslot) {
    peak_prepass_box(rho, vn, peak, nx, ny, nz, axis, dmax, nb, c, bslot,
                     blockIdx.x * (long long)blockDim.x + threadIdx.x, (long long)gridDim.x * blockDim.x);
}

// Batch form: blockIdx.y selects the entry (box) of a batched y/z sweep.
__global__ void peak_prepass_batch_kernel(BatchLaunch bl, int axis) {
    const SweepArgs& a = bl.args[bl.ent[blockIdx.y]];
    if (a.peak == nullptr) return;
    peak_prepass_box(a.f[1], a.f[2], const_cast<double*>(a.peak), a.nx, a.ny, a.nz, axis, a.k.dmax, a.k.nbound,
                     a.ctl, a.bslot, blockIdx.x * (long long)blockDim.x + threadIdx.x,
                     (long long)gridDim.x * blockDim.x);
}

int launch_peak_prepass_batch(const BatchLaunch& bl, int axis, cudaStream_t st) {
    if (axis == 0 || bl.nent <= 0) return 0;
    peak_prepass_batch_kernel<<<dim3(64, bl.nent), 256, 0, st>>>(bl, axis);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

int launch_peak_prepass(const Box& b, int axis, int bslot, cudaStream_t st) {
    if (axis == 0 || b.peak == nullptr) return 0;
    const double* vn = axis == 1 ? b.f[3] : b.f[4];
    peak_prepass_kernel<<<592, 256, 0, st>>>(b.f[1], vn, b.peak, b.nx, b.ny, b.nz, axis, b.k.dmax, b.k.nbound,
                                             b.ctl, bslot);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

}  // namespace hp
