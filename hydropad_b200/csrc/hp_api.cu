// hp_api.cu -- C ABI of the B200 PPM hydro step (include/hydropad_b200.h).
//
// Host-side mirror of the reference's call structure: initialize_parameters
// (time init), ppmsolver / ppm_lxlylz (sweeps), speed + timedet (CFL), and
// evolve_sys' hydro loop, over one box whose state stays resident in HBM.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <stddef.h>
#include <string.h>

#include <vector>

#include "../../include/hydropad_b200.h"
#include "hp_ctx.h"
#include "hp_device.cuh"
#include "hp_launch.h"

namespace hp {
int launch_sweep_fp64(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st);
int launch_sweep_mixed(const Box& b, int axis, int tile, int bslot, int flags, cudaStream_t st);

int launch_sweep(const Box& b, int axis, int tile, int bslot, int flags, int precision, cudaStream_t st) {
    return precision == HP_PREC_MIXED ? launch_sweep_mixed(b, axis, tile, bslot, flags, st)
                                      : launch_sweep_fp64(b, axis, tile, bslot, flags, st);
}
}  // namespace hp


namespace {

// REAL(4) literals used by the time initialisation (initialize_parameters.F90)
constexpr double kC0P010 = 0.009999999776482582;  // 0.010
constexpr double kTwo3 = 0.6666666865348816;      // 2.0/3.0
constexpr double kMThird = -0.3333333432674408;   // -1.0/3.0

int cuda_fail(cudaError_t e) {
    if (e == cudaSuccess) return HP_OK;
    if (e == cudaErrorMemoryAllocation) return HP_ERR_OOM;
    return HP_ERR_CUDA;
}
#define HP_CUDA(x)                                       \
    do {                                                 \
        cudaError_t e_ = (x);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_);     \
    } while (0)

// initialize_parameters.F90:133-205 on a host DevCtl.
void init_time(const hp_params& p, hp::DevCtl& c) {
    if (p.cosmo) {
        double at = p.a_start;
        const double tin = pow(at, 1.5);
        c.told = tin;
        c.s.dt = kC0P010 * tin;
        c.dtold = c.s.dt;
        c.t = tin + c.s.dt;
        c.thalf = c.told + c.s.dt / 2.0;
        c.s.at = pow(c.told, kTwo3);
        c.atnew = pow(c.t, kTwo3);
        c.s.dat = kTwo3 * pow(c.told, kMThird);
        c.s.ath = pow(c.told + c.s.dt / 2.0, kTwo3);
        c.s.dath = kTwo3 * pow(c.thalf, kMThird);
        c.datnew = kTwo3 * pow(c.t, kMThird);
        c.s.rat = 1.0 / c.s.at;
        c.s.rdtath = c.s.dt / c.s.ath;
    } else {
        c.told = 0.0;
        c.s.dt = p.dtinit;
        c.dtold = c.s.dt;
        c.t = c.told + c.s.dt;
        c.s.at = 1.0;
        c.atnew = 1.0;
        c.s.dat = 0.0;
        c.s.ath = 1.0;
        c.s.dath = 0.0;
        c.datnew = 0.0;
        c.s.rat = 1.0;
        c.s.rdtath = c.s.dt / c.s.ath;
        c.thalf = c.told + 0.5 * c.s.dt;
    }
}

int copy_ctl_to_device(hp_ctx* x) {
    HP_CUDA(cudaMemcpyAsync(x->box.ctl, x->ctl_pinned, sizeof(hp::DevCtl), cudaMemcpyHostToDevice, x->stream));
    HP_CUDA(cudaStreamSynchronize(x->stream));
    return HP_OK;
}
int copy_ctl_to_host(hp_ctx* x) {
    HP_CUDA(cudaMemcpyAsync(x->ctl_pinned, x->box.ctl, sizeof(hp::DevCtl), cudaMemcpyDeviceToHost, x->stream));
    HP_CUDA(cudaStreamSynchronize(x->stream));
    return HP_OK;
}

// Ghosted Fortran host array <-> dense device field.  The host array is
// moved in contiguous runs of whole (nxg x nyg) planes through a device
// staging buffer (full-speed DMA, unlike a pitched 3-D copy of the
// interior); a kernel extracts the interior on the way in and writes the
// interior plus its periodic ghost layers on the way out, so the host
// array comes back with its ghosts filled (exchange_mesh.F90:23-41 for one
// rank).  All on the context's stream, so each chunk's copy waits for the
// previous chunk's kernel: the stage holds a whole ghosted field up to
// 256 MB (a 256^3 field in one chunk), which keeps those gaps to a few per
// field.
constexpr size_t kStageBytes = size_t(256) << 20;

int ensure_stage(hp_ctx* x, size_t plane_bytes, int nzg) {
    const size_t field = plane_bytes * (size_t)nzg;  // the whole ghosted field
    size_t want = plane_bytes > kStageBytes ? plane_bytes : (kStageBytes / plane_bytes) * plane_bytes;
    if (want > field) want = field;
    if (x->stage && x->stage_bytes >= want) return HP_OK;
    HP_CUDA(cudaStreamSynchronize(x->stream));
    cudaFree(x->stage);
    x->stage = nullptr;
    x->stage_bytes = 0;
    HP_CUDA(cudaMalloc(&x->stage, want));
    x->stage_bytes = want;
    return HP_OK;
}

int upload_field(hp_ctx* x, const double* host, double* f, int nb) {
    const int nx = x->box.nx, ny = x->box.ny, nz = x->box.nz;
    if (nb == 0)
        return cuda_fail(cudaMemcpyAsync(f, host, (size_t)nx * ny * nz * sizeof(double), cudaMemcpyHostToDevice,
                                         x->stream));
    const size_t plane = (size_t)(nx + 2 * nb) * (ny + 2 * nb);
    int rc = ensure_stage(x, plane * sizeof(double), nz + 2 * nb);
    if (rc != HP_OK) return rc;
    const int per = (int)(x->stage_bytes / (plane * sizeof(double)));
    for (int zg = nb; zg < nb + nz; zg += per) {
        const int k = per < nb + nz - zg ? per : nb + nz - zg;
        HP_CUDA(cudaMemcpyAsync(x->stage, host + (size_t)zg * plane, (size_t)k * plane * sizeof(double),
                                cudaMemcpyHostToDevice, x->stream));
        if (hp::launch_planes_to_field(x->stage, f, nx, ny, nb, zg - nb, k, x->stream) < 0) return HP_ERR_CUDA;
        x->launches += 1;
    }
    return HP_OK;
}

int download_field(hp_ctx* x, const double* f, double* host, int nb) {
    const int nx = x->box.nx, ny = x->box.ny, nz = x->box.nz;
    if (nb == 0)
        return cuda_fail(cudaMemcpyAsync(host, f, (size_t)nx * ny * nz * sizeof(double), cudaMemcpyDeviceToHost,
                                         x->stream));
    const int nzg = nz + 2 * nb;
    const size_t plane = (size_t)(nx + 2 * nb) * (ny + 2 * nb);
    int rc = ensure_stage(x, plane * sizeof(double), nzg);
    if (rc != HP_OK) return rc;
    const int per = (int)(x->stage_bytes / (plane * sizeof(double)));
    for (int zg = 0; zg < nzg; zg += per) {
        const int k = per < nzg - zg ? per : nzg - zg;
        if (hp::launch_field_to_planes(f, x->stage, nx, ny, nz, nb, zg, k, x->stream) < 0) return HP_ERR_CUDA;
        x->launches += 1;
        HP_CUDA(cudaMemcpyAsync(host + (size_t)zg * plane, x->stage, (size_t)k * plane * sizeof(double),
                                cudaMemcpyDeviceToHost, x->stream));
    }
    return HP_OK;
}

// One fused sweep on the resident state.
int do_sweep(hp_ctx* x, int axis, int flags) {
    static const char* const kNames[3] = {"hp sweep x", "hp sweep y", "hp sweep z"};
    hp::TraceRange tr(kNames[axis]);
    const int bslot = (int)(x->sweep_count % 3);
    int n = 0;
    if (x->slab && axis == 2) {
        flags |= hp::kFlagZHalo;  // no pre-pass: its transposed gather would cross slabs
    } else if (!x->box.pencil) {  // the full-pencil solver's peak test reads its own window
        n = hp::launch_peak_prepass(x->box, axis, bslot, x->stream);
        if (n < 0) return HP_ERR_CUDA;
    }
    x->launches += n;
    n = hp::launch_sweep(x->box, axis, x->tile[axis], bslot, flags, x->prm.precision, x->stream);
    if (n < 0) return HP_ERR_CUDA;
    x->launches += n;
    x->sweep_count += 1;
    return HP_OK;
}

// One evolve_sys step on the device: three sweeps (the first snapshots the
// state for expand, the last applies expand and accumulates velmax) and
// timedet.  Returns the number of kernels or a negative error.
int enqueue_step(hp_ctx* x, int nrot) {
    int kern = 0;
    for (int s = 0; s < 3; ++s) {
        const long long before = x->launches;
        const int rc = do_sweep(x, hp::kSweepOrder[nrot - 1][s], hp::step_flags(x->prm, s));
        if (rc != HP_OK) return rc;
        kern += (int)(x->launches - before);
    }
    if (hp::launch_timedet(x->box, 1, x->stream) < 0) return HP_ERR_CUDA;
    x->launches += 1;
    return kern + 1;
}

void drop_gravity(hp_ctx* x) {
    for (int q = 0; q < 3; ++q) {
        cudaFree(x->box.g[q]);
        x->box.g[q] = nullptr;
    }
    x->host_g = nullptr;
}

int alloc_gravity(hp_ctx* x) {
    const size_t n = (size_t)x->box.nx * x->box.ny * x->box.nz;
    for (int q = 0; q < 3; ++q)
        if (!x->box.g[q]) {
            const int rc = cuda_fail(cudaMalloc(&x->box.g[q], n * sizeof(double)));
            if (rc != HP_OK) {
                drop_gravity(x);
                return rc;
            }
        }
    return HP_OK;
}

// gforce(3,nx,ny,nz) ghosted Fortran host array -> three dense device
// components: the interior is copied as 24-byte elements, then split.
int upload_gforce(hp_ctx* x, const double* gforce, int nxg, int nyg, int nb) {
    int rc = alloc_gravity(x);
    if (rc != HP_OK) return rc;
    const size_t n = (size_t)x->box.nx * x->box.ny * x->box.nz;
    double* tmp = nullptr;
    if ((rc = cuda_fail(cudaMalloc(&tmp, 3 * n * sizeof(double)))) != HP_OK) return rc;
    cudaMemcpy3DParms prm;
    memset(&prm, 0, sizeof prm);
    const size_t el = 3 * sizeof(double);
    prm.srcPtr = make_cudaPitchedPtr((void*)gforce, (size_t)nxg * el, (size_t)nxg, (size_t)nyg);
    prm.srcPos = make_cudaPos((size_t)nb * el, (size_t)nb, (size_t)nb);
    prm.dstPtr = make_cudaPitchedPtr((void*)tmp, (size_t)x->box.nx * el, (size_t)x->box.nx, (size_t)x->box.ny);
    prm.dstPos = make_cudaPos(0, 0, 0);
    prm.extent = make_cudaExtent((size_t)x->box.nx * el, (size_t)x->box.ny, (size_t)x->box.nz);
    prm.kind = cudaMemcpyHostToDevice;
    rc = cuda_fail(cudaMemcpy3DAsync(&prm, x->stream));
    if (rc == HP_OK && hp::launch_deinterleave3(tmp, x->box.g[0], x->box.g[1], x->box.g[2], (long long)n,
                                                x->stream) < 0)
        rc = HP_ERR_CUDA;
    if (rc == HP_OK) x->launches += 1;
    cudaStreamSynchronize(x->stream);
    cudaFree(tmp);
    return rc;
}

}  // namespace

extern "C" {

const char* hp_strerror(int code) {
    switch (code) {
        case HP_OK: return "ok";
        case HP_ERR_ARG: return "invalid argument";
        case HP_ERR_CUDA: return "CUDA runtime error";
        case HP_ERR_OOM: return "device out of memory";
        case HP_ERR_NEWTON: return "Riemann Newton iteration did not converge in 100 iterations";
        case HP_ERR_NAN: return "NaN in the updated state";
        case HP_ERR_NEGATIVE_STATE: return "non-positive density or pressure in the updated state";
        case HP_ERR_NOT_ATTACHED: return "no state attached";
        case HP_ERR_STATE_MISMATCH: return "host arrays are not the attached state";
        case HP_ERR_NO_DEVICE: return "no usable sm_100 CUDA device";
        case HP_ERR_UNSUPPORTED: return "not supported by this library (the density-peak fix across z slabs)";
        case HP_ERR_TIMEOUT: return "a bounded wait of the pipelined sweep gave up (results void)";
    }
    return "unknown error";
}

int hp_init(const hp_params* p, hp_ctx** out) {
    if (!p || !out) return HP_ERR_ARG;
    *out = nullptr;
    if (p->ngridx < 8 || p->ngridy < 8 || p->ngridz < 8 || p->nbound < 3) return HP_ERR_ARG;
    if (p->precision != HP_PREC_FP64 && p->precision != HP_PREC_MIXED) return HP_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= p->device || p->device < 0) return HP_ERR_NO_DEVICE;
    cudaDeviceProp prop;
    HP_CUDA(cudaGetDeviceProperties(&prop, p->device));
    if (prop.major != 10) return HP_ERR_NO_DEVICE;
    HP_CUDA(cudaSetDevice(p->device));

    hp_ctx* x = new hp_ctx();
    memset(x, 0, sizeof(*x));
    x->prm = *p;
    x->dev = p->device;
    x->box.nx = p->ngridx;
    x->box.ny = p->ngridy;
    x->box.nz = p->ngridz;
    const size_t n = (size_t)p->ngridx * p->ngridy * p->ngridz;
    int rc = HP_OK;
    auto fail = [&](int code) {
        hp_finalize(x);
        return code;
    };
    if (cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(HP_ERR_CUDA);
    for (int q = 0; q < 5; ++q)
        if ((rc = cuda_fail(cudaMalloc(&x->box.f[q], n * sizeof(double)))) != HP_OK) return fail(rc);
    // expand's step-start snapshot: FP64 in the FP64 path, FP32 in the mixed path
    const size_t snap_bytes = p->precision == HP_PREC_MIXED ? sizeof(float) : sizeof(double);
    if (p->cosmo && !p->expand_zero_old)
        for (int q = 0; q < 4; ++q)
            if ((rc = cuda_fail(cudaMalloc(&x->box.snap[q], n * snap_bytes))) != HP_OK) return fail(rc);
    // density-peak values of the y/z faces: one per cell (face f < N of a
    // pencil at its cell f) and one per pencil for the last face
    {
        const size_t ptail = (size_t)p->ngridx * (p->ngridy > p->ngridz ? p->ngridy : p->ngridz);
        if ((rc = cuda_fail(cudaMalloc(&x->box.peak, (n + ptail) * sizeof(double)))) != HP_OK) return fail(rc);
    }
    if ((rc = cuda_fail(cudaMalloc(&x->box.ctl, sizeof(hp::DevCtl)))) != HP_OK) return fail(rc);
    if ((rc = cuda_fail(cudaMallocHost(&x->ctl_pinned, sizeof(hp::DevCtl)))) != HP_OK) return fail(rc);

    // derived constants, initialize_parameters.F90:23-24,63-69
    hp::Consts& k = x->box.k;
    const int nmax = p->ngridx > p->ngridy ? (p->ngridx > p->ngridz ? p->ngridx : p->ngridz)
                                            : (p->ngridy > p->ngridz ? p->ngridy : p->ngridz);
    k.dx = 1.0 / (double)nmax;
    k.rdx = 1.0 / k.dx;
    k.gamma = p->gamma;
    k.rgamma = 1.0 / p->gamma;
    k.gamma1 = (p->gamma + 1.0) / (p->gamma - 1.0);
    k.rgamma1 = 1.0 / (p->gamma - 1.0);
    k.m = (p->gamma - 1.0) / (2.0 * p->gamma);
    k.rm = 1.0 / k.m;
    k.gf = (p->gamma + 1.0) / (2.0 * p->gamma);
    k.mingradflat = p->mingradflat;
    k.flatvalue = p->flatvalue;
    k.dmax = p->dmax;
    k.eta1 = p->eta1;
    k.eta2 = p->eta2;
    k.nbound = p->nbound;
    // exponents of the Riemann solver as multiples of 1/n (see PowRoot)
    k.nroot = 0;
    k.jrg = 0;
    {
        const double n = k.rm, j = k.rgamma * k.rm;
        if (n == floor(n) && n >= 2.0 && n <= 9.0) {
            k.nroot = (int)n;
            if (fabs(j - rint(j)) < 1e-12 && j >= 1.0 && j <= 9.0) k.jrg = (int)rint(j);
        }
    }
    hp::set_float_consts(k);

    hp::DevCtl& c = *x->ctl_pinned;
    memset(&c, 0, sizeof c);
    init_time(*p, c);
    c.tstop = p->tstop;
    c.cosmo = p->cosmo;
    c.cour = p->cour;
    c.ca = p->ca;
    c.dx = k.dx;
    c.dt_cap = p->dt_cap;
    c.nstep = 1;
    c.bad_cell = -1;
    x->last_bad_cell = -1;
    for (int s = 0; s < 3; ++s) {
        c.rho_key[s][0] = hp::kKeyPosInf;
        c.rho_key[s][1] = hp::kKeyNegInf;
    }
    x->nstep_host = 1;
    if ((rc = copy_ctl_to_device(x)) != HP_OK) return fail(rc);
    // zero the state so that a sweep before any attach reads defined memory
    for (int q = 0; q < 5; ++q)
        if ((rc = cuda_fail(cudaMemsetAsync(x->box.f[q], 0, n * sizeof(double), x->stream))) != HP_OK)
            return fail(rc);
    if ((rc = cuda_fail(cudaStreamSynchronize(x->stream))) != HP_OK) return fail(rc);
    *out = x;
    return HP_OK;
}

int hp_finalize(hp_ctx* x) {
    if (!x) return HP_OK;
    cudaSetDevice(x->dev);
    if (x->stream) cudaStreamSynchronize(x->stream);
    for (int r = 0; r < 6; ++r)
        for (int s = 0; s < 3; ++s)
            if (x->graph[r][s]) cudaGraphExecDestroy(x->graph[r][s]);
    for (int q = 0; q < 5; ++q) cudaFree(x->box.f[q]);
    for (int q = 0; q < 4; ++q) cudaFree(x->box.snap[q]);
    cudaFree(x->box.peak);
    cudaFree(x->stage);
    cudaFree(x->box.zlo);
    cudaFree(x->box.zhi);
    for (int q = 0; q < 3; ++q) cudaFree(x->box.g[q]);
    cudaFree(x->cho_dev);
    cudaFree(x->box.ctl);
    if (x->ctl_pinned) cudaFreeHost(x->ctl_pinned);
    if (x->stream) cudaStreamDestroy(x->stream);
    delete x;
    return HP_OK;
}

int hp_set_scalars(hp_ctx* x, const hp_scalars* s) {
    if (!x || !s) return HP_ERR_ARG;
    int rc = copy_ctl_to_host(x);
    if (rc != HP_OK) return rc;
    hp::DevCtl& c = *x->ctl_pinned;
    c.s.dt = s->dt; c.s.rdtath = s->rdtath; c.s.at = s->at; c.s.dat = s->dat; c.s.rat = s->rat;
    c.s.ath = s->ath; c.s.dath = s->dath;
    c.t = s->t; c.told = s->told; c.thalf = s->thalf; c.dtold = s->dtold; c.atnew = s->atnew;
    c.datnew = s->datnew; c.velmax = s->velmax; c.nstep = s->nstep;
    c.done = (c.told < c.tstop) ? 0 : 1;
    x->nstep_host = s->nstep;
    return copy_ctl_to_device(x);
}

int hp_get_scalars(hp_ctx* x, hp_scalars* s) {
    if (!x || !s) return HP_ERR_ARG;
    int rc = copy_ctl_to_host(x);
    if (rc != HP_OK) return rc;
    const hp::DevCtl& c = *x->ctl_pinned;
    s->dt = c.s.dt; s->rdtath = c.s.rdtath; s->at = c.s.at; s->dat = c.s.dat; s->rat = c.s.rat;
    s->ath = c.s.ath; s->dath = c.s.dath;
    s->t = c.t; s->told = c.told; s->thalf = c.thalf; s->dtold = c.dtold; s->atnew = c.atnew;
    s->datnew = c.datnew; s->velmax = c.velmax; s->nstep = c.nstep; s->pad = 0;
    return HP_OK;
}

int hp_attach_state(hp_ctx* x, const double* p3d, const double* rho3d, const double* vx3d, const double* vy3d,
                    const double* vz3d, const double* gforce, int nx, int ny, int nz, int nbound) {
    if (!x || !p3d || !rho3d || !vx3d || !vy3d || !vz3d) return HP_ERR_ARG;
    if (nbound < 0 || nx != x->box.nx + 2 * nbound || ny != x->box.ny + 2 * nbound || nz != x->box.nz + 2 * nbound)
        return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    hp::TraceRange tr("hp attach state (host to device)");
    // gforce is static (initialize_gravity.F90): attaching again with the
    // same array does not upload it again
    if (!gforce) {
        drop_gravity(x);
    } else if (gforce != x->host_g || !x->box.g[0]) {
        const int grc = upload_gforce(x, gforce, nx, ny, nbound);
        if (grc != HP_OK) return grc;
    }
    x->host_g = gforce;
    const double* src[5] = {p3d, rho3d, vx3d, vy3d, vz3d};
    for (int q = 0; q < 5; ++q) {
        const int rc = upload_field(x, src[q], x->box.f[q], nbound);
        if (rc != HP_OK) return rc;
        x->host[q] = src[q];
    }
    x->hnx = nx; x->hny = ny; x->hnz = nz; x->hnb = nbound;
    x->attached = true;
    x->sweep_count = 0;
    const int n = hp::launch_bounds(x->box, 0, x->stream);
    if (n < 0) return HP_ERR_CUDA;
    x->launches += n;
    HP_CUDA(cudaStreamSynchronize(x->stream));
    return HP_OK;
}

int hp_attach_device_state(hp_ctx* x, const double* p, const double* rho, const double* vx, const double* vy,
                           const double* vz) {
    if (!x || !p || !rho || !vx || !vy || !vz) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    const size_t n = (size_t)x->box.nx * x->box.ny * x->box.nz;
    const double* src[5] = {p, rho, vx, vy, vz};
    HP_CUDA(cudaStreamSynchronize(x->stream));
    drop_gravity(x);
    for (int q = 0; q < 5; ++q) {
        HP_CUDA(cudaMemcpyAsync(x->box.f[q], src[q], n * sizeof(double), cudaMemcpyDeviceToDevice, x->stream));
        x->host[q] = nullptr;
    }
    x->hnx = x->box.nx; x->hny = x->box.ny; x->hnz = x->box.nz; x->hnb = 0;
    x->attached = true;
    x->sweep_count = 0;
    const int nk = hp::launch_bounds(x->box, 0, x->stream);
    if (nk < 0) return HP_ERR_CUDA;
    x->launches += nk;
    HP_CUDA(cudaStreamSynchronize(x->stream));
    return HP_OK;
}

int hp_download_state(hp_ctx* x, double* p3d, double* rho3d, double* vx3d, double* vy3d, double* vz3d, int nx,
                      int ny, int nz, int nbound) {
    if (!x || !p3d || !rho3d || !vx3d || !vy3d || !vz3d) return HP_ERR_ARG;
    if (nbound < 0 || nx != x->box.nx + 2 * nbound || ny != x->box.ny + 2 * nbound || nz != x->box.nz + 2 * nbound)
        return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    hp::TraceRange tr("hp download state (device to host)");
    double* dst[5] = {p3d, rho3d, vx3d, vy3d, vz3d};
    for (int q = 0; q < 5; ++q) {
        const int rc = download_field(x, x->box.f[q], dst[q], nbound);
        if (rc != HP_OK) return rc;
    }
    HP_CUDA(cudaStreamSynchronize(x->stream));
    return HP_OK;
}

int hp_attach_device_gforce(hp_ctx* x, const double* gx, const double* gy, const double* gz) {
    if (!x) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    HP_CUDA(cudaStreamSynchronize(x->stream));
    if (!gx && !gy && !gz) {
        drop_gravity(x);
        return HP_OK;
    }
    if (!gx || !gy || !gz) return HP_ERR_ARG;
    int rc = alloc_gravity(x);
    if (rc != HP_OK) return rc;
    const size_t n = (size_t)x->box.nx * x->box.ny * x->box.nz;
    const double* src[3] = {gx, gy, gz};
    for (int q = 0; q < 3; ++q)
        HP_CUDA(cudaMemcpyAsync(x->box.g[q], src[q], n * sizeof(double), cudaMemcpyDeviceToDevice, x->stream));
    HP_CUDA(cudaStreamSynchronize(x->stream));
    x->host_g = nullptr;
    return HP_OK;
}

int hp_write_var(hp_ctx* x, const char* directory, int fp64) {
    if (!x || !directory) return HP_ERR_ARG;
    if (!x->attached) return HP_ERR_NOT_ATTACHED;
    HP_CUDA(cudaSetDevice(x->dev));
    HP_CUDA(cudaStreamSynchronize(x->stream));
    // main.F90:125-135 order and names; field index in box.f (p, rho, vx, vy, vz)
    static const char* kNames[5] = {"rho", "pressure", "vx", "vy", "vz"};
    static const int kField[5] = {1, 0, 2, 3, 4};
    const long long n = (long long)x->box.nx * x->box.ny * x->box.nz;
    const size_t esize = fp64 ? sizeof(double) : sizeof(float);
    // the FP32 copy is staged in the density-peak buffer (n doubles), which
    // holds nothing between steps
    float* f32 = reinterpret_cast<float*>(x->box.peak);
    constexpr size_t kChunk = 64u << 20;  // bytes per pinned staging buffer
    unsigned char* pin[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int rc = HP_OK;
    for (int b = 0; b < 2 && rc == HP_OK; ++b) {
        rc = cuda_fail(cudaMallocHost(&pin[b], kChunk));
        if (rc == HP_OK) rc = cuda_fail(cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming));
    }
    for (int v = 0; v < 5 && rc == HP_OK; ++v) {
        const unsigned char* src;
        if (fp64) {
            src = reinterpret_cast<const unsigned char*>(x->box.f[kField[v]]);
        } else {
            if (hp::launch_to_f32(x->box.f[kField[v]], f32, n, x->stream) < 0) { rc = HP_ERR_CUDA; break; }
            x->launches += 1;
            src = reinterpret_cast<const unsigned char*>(f32);
        }
        char path[4096];
        snprintf(path, sizeof path, "%s/%s%s.bin", directory, kNames[v], fp64 ? ".f64" : "");
        FILE* fp = fopen(path, "wb");
        if (!fp) { rc = HP_ERR_ARG; break; }
        // double-buffered: copy chunk c+1 while chunk c is written
        const size_t total = (size_t)n * esize;
        size_t off = 0, pending = 0;
        int cur = 0;
        while (rc == HP_OK && (off < total || pending)) {
            size_t len = 0;
            if (off < total) {
                len = total - off < kChunk ? total - off : kChunk;
                rc = cuda_fail(cudaMemcpyAsync(pin[cur], src + off, len, cudaMemcpyDeviceToHost, x->stream));
                if (rc == HP_OK) rc = cuda_fail(cudaEventRecord(ev[cur], x->stream));
            }
            if (rc == HP_OK && pending) {
                const int prev = cur ^ 1;
                rc = cuda_fail(cudaEventSynchronize(ev[prev]));
                if (rc == HP_OK && fwrite(pin[prev], 1, pending, fp) != pending) rc = HP_ERR_ARG;
            }
            off += len;
            pending = len;
            cur ^= 1;
            if (len == 0) break;
        }
        if (fclose(fp) != 0 && rc == HP_OK) rc = HP_ERR_ARG;
    }
    cudaStreamSynchronize(x->stream);
    for (int b = 0; b < 2; ++b) {
        if (pin[b]) cudaFreeHost(pin[b]);
        if (ev[b]) cudaEventDestroy(ev[b]);
    }
    return rc;
}

int hp_sync_to_host(hp_ctx* x) {
    if (!x) return HP_ERR_ARG;
    if (!x->attached || !x->host[0]) return HP_ERR_NOT_ATTACHED;  // no host arrays behind a device attach
    return hp_download_state(x, (double*)x->host[0], (double*)x->host[1], (double*)x->host[2], (double*)x->host[3],
                             (double*)x->host[4], x->hnx, x->hny, x->hnz, x->hnb);
}

int hp_ppmsolver(hp_ctx* x, double* p3d, double* rho3d, double* vx3d, double* vy3d, double* vz3d, double* cho3d,
                 double* nes3d, const double* gforce, const int* nx, const int* ny, const int* nz,
                 const int* nbound, const int* ndirection) {
    (void)cho3d;
    (void)nes3d;
    if (!x || !nx || !ny || !nz || !nbound || !ndirection) return HP_ERR_ARG;
    if (!x->attached) return HP_ERR_NOT_ATTACHED;
    if (gforce != x->host_g) return HP_ERR_STATE_MISMATCH;  // the attached gforce (or none)
    if (*ndirection < 1 || *ndirection > 3) return HP_ERR_ARG;
    if (*nx != x->hnx || *ny != x->hny || *nz != x->hnz || *nbound != x->hnb) return HP_ERR_STATE_MISMATCH;
    const double* given[5] = {p3d, rho3d, vx3d, vy3d, vz3d};
    for (int q = 0; q < 5; ++q)
        if (given[q] != x->host[q]) return HP_ERR_STATE_MISMATCH;
    HP_CUDA(cudaSetDevice(x->dev));
    int rc = do_sweep(x, *ndirection - 1, 0);
    if (rc != HP_OK) return rc;
    return hp_synchronize(x);
}

int hp_ppm_lxlylz(hp_ctx* x, int nrot) {
    if (!x || nrot < 1 || nrot > 6 || x->slab) return HP_ERR_ARG;
    if (!x->attached) return HP_ERR_NOT_ATTACHED;
    HP_CUDA(cudaSetDevice(x->dev));
    for (int s = 0; s < 3; ++s) {
        int rc = do_sweep(x, hp::kSweepOrder[nrot - 1][s], 0);
        if (rc != HP_OK) return rc;
    }
    return HP_OK;
}

int hp_speed(hp_ctx* x, double* velmax) {
    if (!x || !velmax) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    if (hp::launch_speed(x->box, x->stream) < 0) return HP_ERR_CUDA;
    x->launches += 1;
    unsigned long long bits = 0;
    HP_CUDA(cudaMemcpyAsync(&bits, &x->box.ctl->velmax_key, sizeof bits, cudaMemcpyDeviceToHost, x->stream));
    HP_CUDA(cudaStreamSynchronize(x->stream));
    memcpy(velmax, &bits, sizeof(double));
    return HP_OK;
}

int hp_timedet(hp_ctx* x, double velmax) {
    if (!x) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    unsigned long long bits;
    memcpy(&bits, &velmax, sizeof bits);
    HP_CUDA(cudaMemcpyAsync(&x->box.ctl->velmax_key, &bits, sizeof bits, cudaMemcpyHostToDevice, x->stream));
    if (hp::launch_timedet(x->box, 0, x->stream) < 0) return HP_ERR_CUDA;
    x->launches += 1;
    HP_CUDA(cudaStreamSynchronize(x->stream));
    return HP_OK;
}

int hp_evolve_async(hp_ctx* x, int nsteps, int use_graph) {
    if (!x || nsteps < 0 || x->slab) return HP_ERR_ARG;  // a slab steps through hp_step_*
    if (!x->attached) return HP_ERR_NOT_ATTACHED;
    HP_CUDA(cudaSetDevice(x->dev));
    for (int it = 0; it < nsteps; ++it) {
        hp::TraceRange tr("hp step");
        const long long nstep = x->nstep_host;
        const int nrot = hp::nrot_of_step(nstep);
        const int slot = (int)(x->sweep_count % 3);
        if (!use_graph) {
            const int n = enqueue_step(x, nrot);
            if (n < 0) return n;
        } else {
            cudaGraphExec_t& g = x->graph[nrot - 1][slot];
            if (!g) {
                cudaGraph_t graph;
                const long long sc0 = x->sweep_count, l0 = x->launches;
                HP_CUDA(cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal));
                const int n = enqueue_step(x, nrot);
                cudaError_t ce = cudaStreamEndCapture(x->stream, &graph);
                if (n < 0) return n;
                HP_CUDA(ce);
                HP_CUDA(cudaGraphInstantiate(&g, graph, 0));
                cudaGraphDestroy(graph);
                x->graph_kernels[nrot - 1][slot] = n;
                x->sweep_count = sc0;  // the capture did not execute anything
                x->launches = l0;
            }
            HP_CUDA(cudaGraphLaunch(g, x->stream));
            x->sweep_count += 3;
            x->launches += x->graph_kernels[nrot - 1][slot];
        }
        x->nstep_host += 1;
    }
    return HP_OK;
}

int hp_evolve(hp_ctx* x, int nsteps, int use_graph) {
    const int rc = hp_evolve_async(x, nsteps, use_graph);
    if (rc != HP_OK) return rc;
    return hp_synchronize(x);
}

int hp_synchronize(hp_ctx* x) {
    if (!x) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    // status, done and the first bad cell are adjacent: one read
    static_assert(offsetof(hp::DevCtl, bad_cell) == offsetof(hp::DevCtl, status) + 8, "DevCtl layout");
    struct {
        unsigned status;
        int done;
        long long bad_cell;
    } rd;
    HP_CUDA(cudaMemcpyAsync(&rd, &x->box.ctl->status, sizeof rd, cudaMemcpyDeviceToHost, x->stream));
    HP_CUDA(cudaMemsetAsync(&x->box.ctl->status, 0, sizeof(unsigned), x->stream));
    HP_CUDA(cudaMemsetAsync(&x->box.ctl->bad_cell, 0xff, sizeof(long long), x->stream));
    HP_CUDA(cudaStreamSynchronize(x->stream));
    if (rd.status) x->last_bad_cell = rd.bad_cell;
    return hp::status_error(rd.status);
}

long long hp_bad_cell(hp_ctx* x) { return x ? x->last_bad_cell : -1; }

void* hp_stream(hp_ctx* x) { return x ? (void*)x->stream : nullptr; }

static void drop_graphs(hp_ctx* x) {
    for (int r = 0; r < 6; ++r)
        for (int s = 0; s < 3; ++s)
            if (x->graph[r][s]) {
                cudaGraphExecDestroy(x->graph[r][s]);
                x->graph[r][s] = nullptr;
            }
}

int hp_set_tiles(hp_ctx* x, int tile_x, int tile_y, int tile_z) {
    if (!x) return HP_ERR_ARG;
    const int t[3] = {tile_x, tile_y, tile_z};
    for (int a = 0; a < 3; ++a)
        if (t[a] < 0 || t[a] >= hp::kNumTiles) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    HP_CUDA(cudaStreamSynchronize(x->stream));
    drop_graphs(x);
    for (int a = 0; a < 3; ++a) x->tile[a] = t[a];
    return HP_OK;
}

int hp_num_tiles(void) { return hp::kNumTiles; }

int hp_get_tiles(hp_ctx* x, int* tiles) {
    if (!x || !tiles) return HP_ERR_ARG;
    for (int a = 0; a < 3; ++a) tiles[a] = x->tile[a];
    return HP_OK;
}

int hp_autotune(hp_ctx* x, int reps) {
    if (!x || reps < 1) return HP_ERR_ARG;
    if (!x->attached) return HP_ERR_NOT_ATTACHED;
    HP_CUDA(cudaSetDevice(x->dev));
    const size_t n = (size_t)x->box.nx * x->box.ny * x->box.nz;
    hp::Box sb = x->box;  // scratch copy of the box: the resident state is not touched
    for (int q = 0; q < 4; ++q) sb.snap[q] = nullptr;
    int rc = HP_OK;
    double* fields[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    hp::DevCtl* sctl = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float best[3] = {1e30f, 1e30f, 1e30f};
    int pick[3] = {x->tile[0], x->tile[1], x->tile[2]};
    const int bslot = (int)(x->sweep_count % 3);
    for (int q = 0; q < 5 && rc == HP_OK; ++q) rc = cuda_fail(cudaMalloc(&fields[q], n * sizeof(double)));
    if (rc == HP_OK) rc = cuda_fail(cudaMalloc(&sctl, sizeof(hp::DevCtl)));
    if (rc == HP_OK) rc = cuda_fail(cudaEventCreate(&e0));
    if (rc == HP_OK) rc = cuda_fail(cudaEventCreate(&e1));
    for (int q = 0; q < 5; ++q) sb.f[q] = fields[q];
    sb.ctl = sctl;
    for (int axis = 0; axis < 3 && rc == HP_OK; ++axis) {
        for (int tile = 0; tile < hp::kNumTiles && rc == HP_OK; ++tile) {
            for (int q = 0; q < 5 && rc == HP_OK; ++q)
                rc = cuda_fail(cudaMemcpyAsync(fields[q], x->box.f[q], n * sizeof(double), cudaMemcpyDeviceToDevice,
                                               x->stream));
            if (rc == HP_OK)
                rc = cuda_fail(cudaMemcpyAsync(sctl, x->box.ctl, sizeof(hp::DevCtl), cudaMemcpyDeviceToDevice,
                                               x->stream));
            if (rc != HP_OK) break;
            // warm-up launch, then reps timed launches (each a full sweep)
            if (hp::launch_sweep(sb, axis, tile, bslot, 0, x->prm.precision, x->stream) < 0) rc = HP_ERR_CUDA;
            if (rc == HP_OK) rc = cuda_fail(cudaEventRecord(e0, x->stream));
            for (int r = 0; r < reps && rc == HP_OK; ++r)
                if (hp::launch_sweep(sb, axis, tile, bslot, 0, x->prm.precision, x->stream) < 0) rc = HP_ERR_CUDA;
            if (rc == HP_OK) rc = cuda_fail(cudaEventRecord(e1, x->stream));
            if (rc == HP_OK) rc = cuda_fail(cudaEventSynchronize(e1));
            float ms = 0.f;
            if (rc == HP_OK) rc = cuda_fail(cudaEventElapsedTime(&ms, e0, e1));
            x->launches += reps + 1;
            if (rc == HP_OK && ms < best[axis]) {
                best[axis] = ms;
                pick[axis] = tile;
            }
        }
    }
    cudaStreamSynchronize(x->stream);
    for (int q = 0; q < 5; ++q) cudaFree(fields[q]);
    cudaFree(sctl);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (rc != HP_OK) return rc;
    return hp_set_tiles(x, pick[0], pick[1], pick[2]);
}

int hp_slab_init(hp_ctx* x, int nz_global, int z0) {
    if (!x || x->slab) return HP_ERR_ARG;
    if (x->box.pencil) return HP_ERR_UNSUPPORTED;
    const int nz = x->box.nz;
    if (nz < 4 || z0 < 0 || nz_global < nz || z0 + nz > nz_global) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    HP_CUDA(cudaStreamSynchronize(x->stream));
    const size_t plane = (size_t)x->box.nx * x->box.ny;
    int rc = cuda_fail(cudaMalloc(&x->box.zlo, 5 * 4 * plane * sizeof(double)));
    if (rc == HP_OK) rc = cuda_fail(cudaMalloc(&x->box.zhi, 5 * 3 * plane * sizeof(double)));
    if (rc != HP_OK) {
        cudaFree(x->box.zlo);
        cudaFree(x->box.zhi);
        x->box.zlo = x->box.zhi = nullptr;
        return rc;
    }
    // dx of the whole box (initialize_parameters.F90:23): 1/max(ngridx, ngridy, nz_global)
    const int nmax = x->box.nx > x->box.ny ? (x->box.nx > nz_global ? x->box.nx : nz_global)
                                           : (x->box.ny > nz_global ? x->box.ny : nz_global);
    x->box.k.dx = 1.0 / (double)nmax;
    hp::set_float_consts(x->box.k);
    x->box.k.rdx = 1.0 / x->box.k.dx;
    if ((rc = copy_ctl_to_host(x)) != HP_OK) return rc;
    x->ctl_pinned->dx = x->box.k.dx;
    if ((rc = copy_ctl_to_device(x)) != HP_OK) return rc;
    drop_graphs(x);
    x->slab = 1;
    x->nz_global = nz_global;
    x->z0 = z0;
    return HP_OK;
}

int hp_slab_get_edges(hp_ctx* x, double* top4, double* bottom3) {
    if (!x || !x->slab || !top4 || !bottom3) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    const size_t plane = (size_t)x->box.nx * x->box.ny;
    const size_t nz = (size_t)x->box.nz;
    for (int q = 0; q < 5; ++q) {
        HP_CUDA(cudaMemcpyAsync(top4 + q * 4 * plane, x->box.f[q] + (nz - 4) * plane, 4 * plane * sizeof(double),
                                cudaMemcpyDeviceToDevice, x->stream));
        HP_CUDA(cudaMemcpyAsync(bottom3 + q * 3 * plane, x->box.f[q], 3 * plane * sizeof(double),
                                cudaMemcpyDeviceToDevice, x->stream));
    }
    HP_CUDA(cudaStreamSynchronize(x->stream));
    return HP_OK;
}

int hp_slab_set_halos(hp_ctx* x, const double* lower4, const double* upper3) {
    if (!x || !x->slab || !lower4 || !upper3) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    const size_t plane = (size_t)x->box.nx * x->box.ny;
    HP_CUDA(cudaMemcpyAsync(x->box.zlo, lower4, 5 * 4 * plane * sizeof(double), cudaMemcpyDeviceToDevice,
                            x->stream));
    HP_CUDA(cudaMemcpyAsync(x->box.zhi, upper3, 5 * 3 * plane * sizeof(double), cudaMemcpyDeviceToDevice,
                            x->stream));
    return HP_OK;
}

int hp_step_axis(hp_ctx* x, int s) {
    if (!x || s < 0 || s > 2) return HP_ERR_ARG;
    return hp::kSweepOrder[hp::nrot_of_step(x->nstep_host) - 1][s];
}

int hp_step_sweep(hp_ctx* x, int s) {
    if (!x || s < 0 || s > 2) return HP_ERR_ARG;
    if (!x->attached) return HP_ERR_NOT_ATTACHED;
    HP_CUDA(cudaSetDevice(x->dev));
    return do_sweep(x, hp::kSweepOrder[hp::nrot_of_step(x->nstep_host) - 1][s], hp::step_flags(x->prm, s));
}

int hp_step_velmax(hp_ctx* x, double* velmax) {
    if (!x || !velmax) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    unsigned long long bits = 0;
    HP_CUDA(cudaMemcpyAsync(&bits, &x->box.ctl->velmax_key, sizeof bits, cudaMemcpyDeviceToHost, x->stream));
    HP_CUDA(cudaStreamSynchronize(x->stream));
    memcpy(velmax, &bits, sizeof(double));
    return HP_OK;
}

int hp_step_finish(hp_ctx* x, double velmax) {
    if (!x) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    unsigned long long bits;
    memcpy(&bits, &velmax, sizeof bits);
    HP_CUDA(cudaMemcpyAsync(&x->box.ctl->velmax_key, &bits, sizeof bits, cudaMemcpyHostToDevice, x->stream));
    if (hp::launch_timedet(x->box, 1, x->stream) < 0) return HP_ERR_CUDA;
    x->launches += 1;
    x->nstep_host += 1;
    return hp_synchronize(x);
}

int hp_device_fields(hp_ctx* x, double** p, double** rho, double** vx, double** vy, double** vz) {
    if (!x) return HP_ERR_ARG;
    if (p) *p = x->box.f[0];
    if (rho) *rho = x->box.f[1];
    if (vx) *vx = x->box.f[2];
    if (vy) *vy = x->box.f[3];
    if (vz) *vz = x->box.f[4];
    return HP_OK;
}

long long hp_launch_count(hp_ctx* x) { return x ? x->launches : 0; }

int hp_set_variant(hp_ctx* x, int variant) {
    if (!x || (variant != HP_VARIANT_STENCIL && variant != HP_VARIANT_PENCIL)) return HP_ERR_ARG;
    if (variant == HP_VARIANT_PENCIL && (x->prm.precision != HP_PREC_FP64 || x->slab)) return HP_ERR_UNSUPPORTED;
    HP_CUDA(cudaSetDevice(x->dev));
    HP_CUDA(cudaStreamSynchronize(x->stream));
    drop_graphs(x);
    x->box.pencil = variant == HP_VARIANT_PENCIL ? 1 : 0;
    return HP_OK;
}

int hp_get_variant(hp_ctx* x) {
    if (!x) return HP_ERR_ARG;
    return x->box.pencil ? HP_VARIANT_PENCIL : HP_VARIANT_STENCIL;
}

int hp_attach_cho(hp_ctx* x, const double* cho3d, int nx, int ny, int nz, int nbound) {
    if (!x) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(x->dev));
    HP_CUDA(cudaStreamSynchronize(x->stream));
    drop_graphs(x);
    if (!cho3d) {
        cudaFree(x->cho_dev);
        x->cho_dev = nullptr;
        x->box.cho = nullptr;
        x->host_cho = nullptr;
        return HP_OK;
    }
    if (nbound < 0 || nx != x->box.nx + 2 * nbound || ny != x->box.ny + 2 * nbound || nz != x->box.nz + 2 * nbound)
        return HP_ERR_ARG;
    if (!x->cho_dev) {
        const size_t n = (size_t)x->box.nx * x->box.ny * x->box.nz;
        int rc = cuda_fail(cudaMalloc(&x->cho_dev, n * sizeof(double)));
        if (rc != HP_OK) return rc;
    }
    int rc = upload_field(x, cho3d, x->cho_dev, nbound);
    if (rc != HP_OK) return rc;
    HP_CUDA(cudaStreamSynchronize(x->stream));
    x->box.cho = x->cho_dev;
    x->host_cho = cho3d;
    return HP_OK;
}

int hp_ppmsolver_pencil(hp_ctx* x, double* p3d, double* rho3d, double* vx3d, double* vy3d, double* vz3d,
                        double* cho3d, double* nes3d, const double* gforce, double* p3dnew, double* rho3dnew,
                        double* vx3dnew, double* vy3dnew, double* vz3dnew, double* cho3dnew, const int* nx,
                        const int* ny, const int* nz, const int* nbound, const int* ndirection) {
    (void)nes3d;
    (void)p3dnew; (void)rho3dnew; (void)vx3dnew; (void)vy3dnew; (void)vz3dnew; (void)cho3dnew;
    if (!x || !nx || !ny || !nz || !nbound || !ndirection) return HP_ERR_ARG;
    if (x->prm.precision != HP_PREC_FP64 || x->slab) return HP_ERR_UNSUPPORTED;
    if (!x->attached) return HP_ERR_NOT_ATTACHED;
    if (gforce != x->host_g || cho3d != x->host_cho) return HP_ERR_STATE_MISMATCH;
    if (*ndirection < 1 || *ndirection > 3) return HP_ERR_ARG;
    if (*nx != x->hnx || *ny != x->hny || *nz != x->hnz || *nbound != x->hnb) return HP_ERR_STATE_MISMATCH;
    const double* given[5] = {p3d, rho3d, vx3d, vy3d, vz3d};
    for (int q = 0; q < 5; ++q)
        if (given[q] != x->host[q]) return HP_ERR_STATE_MISMATCH;
    HP_CUDA(cudaSetDevice(x->dev));
    const int was = x->box.pencil;
    x->box.pencil = 1;
    int rc = do_sweep(x, *ndirection - 1, 0);
    x->box.pencil = was;
    if (rc != HP_OK) return rc;
    return hp_synchronize(x);
}

}  // extern "C"
