/*
 * hydropad_b200.h -- C ABI of the B200 PPM hydro step.
 *
 * Drop-in boundary for Hydropad's STENCIL hydro step.  Each entry point names
 * the reference routine it replaces:
 *
 *   hp_ppmsolver   <- SUBROUTINE ppmsolver(p3d,rho3d,vx3d,vy3d,vz3d,cho3d,nes3d,
 *                                          gforce,nx,ny,nz,nbound,ndirection)
 *                     hydro/ppmsolver.F90:1-5 (STENCIL argument list)
 *   hp_ppm_lxlylz  <- SUBROUTINE ppm_lxlylz          hydro/ppm_lxlylz.F90:1-223
 *                     (+ the exchange_mesh after every sweep,
 *                      hydropad/exchange_mesh.F90:23-41)
 *   hp_speed       <- SUBROUTINE speed               hydropad/speed.F90:2-59
 *   hp_timedet     <- SUBROUTINE timedet / timedet_cosmo
 *                                                    hydropad/functions.F90:2-151
 *   hp_evolve      <- the hydro part of SUBROUTINE evolve_sys, nsteps times
 *                     hydropad/evolve_sys.F90:30-130, main.F90:100-121
 *   hp_attach_state / hp_sync_to_host
 *                  <- the `!$acc update device/host` pairs around every sweep
 *                     (ppmsolver.F90:95, ppm_lxlylz.F90:20), done once per run
 *   hp_set_scalars <- the `!$acc update device(<module scalar list>)`
 *                     hydro/ppmsolver.F90:68-69, hydropad/scalar.F90:98-99
 *
 * Arrays passed by the caller are the reference's module arrays: REAL(8),
 * Fortran column-major (nx,ny,nz) INCLUDING nbound ghost layers per side
 * (hydropad/alloc_arrays.F90:76-78).  The device keeps only the interior,
 * x fastest, and applies the periodic boundary by index wrap, so the ghost
 * layers are an output-only convenience (refreshed by hp_sync_to_host).
 *
 * All functions return HP_OK (0) or a negative HP_ERR_* code; hp_strerror
 * names it.  No function is re-entrant on the same context.
 */
#ifndef HYDROPAD_B200_H
#define HYDROPAD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    HP_OK = 0,
    HP_ERR_ARG = -1,           /* bad argument / shape / unknown direction */
    HP_ERR_CUDA = -2,          /* a CUDA runtime call failed */
    HP_ERR_OOM = -3,           /* device allocation failed */
    HP_ERR_NEWTON = -4,        /* Newton for p* exceeded 100 iterations (riemann.F90:62-65: `stop`) */
    HP_ERR_NAN = -5,           /* NaN in the updated state */
    HP_ERR_NEGATIVE_STATE = -6,/* rho <= 0 or p <= 0 in the updated state */
    HP_ERR_NOT_ATTACHED = -7,  /* sweep requested before hp_attach_state */
    HP_ERR_STATE_MISMATCH = -8,/* host arrays differ from the attached ones */
    HP_ERR_NO_DEVICE = -9,     /* no CUDA device / wrong architecture */
    HP_ERR_UNSUPPORTED = -10,  /* a case this library does not take (the density-peak fix across z slabs) */
    HP_ERR_TIMEOUT = -11       /* a bounded wait inside the pipelined sweep gave up; the sweep's
                                  results are void (no counterpart in the reference) */
};

/* HP_PREC_FP64: every stage in FP64, the reference's arithmetic operation by
 * operation (within 1e-10 relative L1 per field, after 10 steps, of a CPU
 * restatement of the reference's algorithm).
 * HP_PREC_MIXED: reconstruction, tracing, classification, the closed-form
 * Riemann solutions and the Newton iteration of weak faces (pressures
 * within a factor 4, velocity jump at most cL + cR) in FP32; the Newton
 * iteration of strong shocks, the conservative update, the dual-energy
 * switch and the state in FP64 (density within 1e-5 relative L1 of FP64
 * after 100 steps on a 512^3 cosmological box). */
enum { HP_PREC_FP64 = 0, HP_PREC_MIXED = 1 };

/* Namelist values of the run (hydropad/init_sys.F90:12-44) plus the
 * precision choice.  ngrid = interior cells per axis of this box. */
typedef struct {
    int ngridx, ngridy, ngridz;   /* &MESH ngridx/ngridy/ngridz (interior) */
    int nbound;                   /* &MESH nbound (ghosts of the HOST arrays) */
    double gamma;                 /* &PHYSICS gamma */
    double cour, ca, eta1, eta2, dmax;  /* &NUMERICS */
    double flatvalue, mingradflat;      /* &PPM */
    double dtinit, tstop;               /* &TIME */
    int cosmo;                    /* 1: EdS background (-DCOSMO) */
    int expand_zero_old;          /* 1: expand with vxold=pold3d=0 (as allocated) */
    double a_start;               /* initial expansion factor (cosmo) */
    double dt_cap;                /* timedet_cosmo debug cap dt0; <= 0 disables */
    int precision;                /* HP_PREC_FP64 or HP_PREC_MIXED */
    int device;                   /* CUDA device ordinal */
} hp_params;

/* Time scalars of the module `scalar` read by the step (scalar.F90:17-19). */
typedef struct {
    double dt, rdtath, at, dat, rat, ath, dath;
    double t, told, thalf, dtold, atnew, datnew;
    double velmax;
    int nstep;
    int pad;
} hp_scalars;

typedef struct hp_ctx hp_ctx;

/* Allocate the device state for one box and initialise the time scalars as
 * initialize_parameters does (initialize_parameters.F90:133-205). */
int hp_init(const hp_params *params, hp_ctx **ctx);
int hp_finalize(hp_ctx *ctx);

int hp_set_scalars(hp_ctx *ctx, const hp_scalars *s);
int hp_get_scalars(hp_ctx *ctx, hp_scalars *s);

/* Upload the host state (ghosted Fortran arrays) once; it then stays
 * resident in HBM.  gforce: the static gravity force gforce(3,nx,ny,nz)
 * (ghosted, Fortran order, component fastest: hydropad/matrix.F90,
 * initialize_gravity.F90:49-55), or NULL for no gravity source.  It is
 * uploaded as three dense components; attaching again with the same gforce
 * pointer keeps the uploaded copy (the field is static). */
int hp_attach_state(hp_ctx *ctx, const double *p3d, const double *rho3d,
                    const double *vx3d, const double *vy3d, const double *vz3d,
                    const double *gforce, int nx, int ny, int nz, int nbound);

/* Take the state from DEVICE arrays on the context's device (dense
 * (ngridx,ngridy,ngridz) interiors, x fastest; copied, the caller keeps
 * them), e.g. initial conditions generated on the GPU.  The caller's writes
 * must be complete (synchronise the producing stream first).  No host
 * arrays are attached: hp_sync_to_host and hp_ppmsolver then report
 * HP_ERR_NOT_ATTACHED / HP_ERR_STATE_MISMATCH; use hp_download_state.
 * No counterpart in the reference, whose state is born on the host. */
int hp_attach_device_state(hp_ctx *ctx, const double *p, const double *rho,
                           const double *vx, const double *vy, const double *vz);

/* The gravity force from DEVICE arrays (three dense components, x fastest,
 * copied), or all NULL to switch the gravity source off. */
int hp_attach_device_gforce(hp_ctx *ctx, const double *gx, const double *gy,
                            const double *gz);

/* Download the resident state into the attached host arrays (interior) and
 * refill their periodic ghost layers. */
int hp_sync_to_host(hp_ctx *ctx);

/* The end-of-run dump of main.F90:125-135 (write_var_mpi, io/write_var_mpi.F90:
 * 1-65): rho.bin, pressure.bin, vx.bin, vy.bin, vz.bin in `directory`, each
 * the interior (ngridx,ngridy,ngridz) in Fortran order as raw native
 * (little-endian) REAL(4), no header, converted on the device with
 * round-to-nearest.  fp64=1 writes the same layout in REAL(8) to
 * rho.f64.bin, pressure.f64.bin, ... (no counterpart in the reference).
 * Existing files are replaced.  Uses the density-peak buffer as staging. */
int hp_write_var(hp_ctx *ctx, const char *directory, int fp64);

/* Download into arbitrary host arrays of the same shape. */
int hp_download_state(hp_ctx *ctx, double *p3d, double *rho3d, double *vx3d,
                      double *vy3d, double *vz3d, int nx, int ny, int nz,
                      int nbound);

/* Drop-in for ppmsolver: one directional sweep (1=x, 2=y, 3=z) on the
 * resident state.  The host pointers identify the attached state (they must
 * be the attached arrays, gforce included, or NULL when none was attached);
 * cho3d/nes3d are unused under STENCIL and may be NULL.  Scalars and integers are passed by reference, like the Fortran
 * subroutine.  Returns the sweep's error status. */
int hp_ppmsolver(hp_ctx *ctx, double *p3d, double *rho3d, double *vx3d,
                 double *vy3d, double *vz3d, double *cho3d, double *nes3d,
                 const double *gforce, const int *nx, const int *ny,
                 const int *nz, const int *nbound, const int *ndirection);

/* Drop-in for ppm_lxlylz: three sweeps in the order nrot selects
 * (1 xyz, 2 zyx, 3 yzx, 4 xzy, 5 zxy, 6 yxz).  No ghost exchange is needed:
 * the device state is periodic by construction. */
int hp_ppm_lxlylz(hp_ctx *ctx, int nrot);

/* speed: velmax = max over cells of max_d(|v_d| + sqrt(gamma p/rho)). */
int hp_speed(hp_ctx *ctx, double *velmax);

/* timedet (static) or timedet_cosmo (cosmo) on the context's scalars with
 * the given velmax. */
int hp_timedet(hp_ctx *ctx, double velmax);

/* nsteps of evolve_sys' hydro part, entirely on the device: nrot schedule,
 * three fused sweeps, [expand], speed and timedet, no host round trip.
 * use_graph=1 captures one step per nrot value in CUDA graphs and replays
 * them.  Returns the accumulated error status. */
int hp_evolve(hp_ctx *ctx, int nsteps, int use_graph);
/* hp_evolve without the final wait and status read: returns once the steps
 * are enqueued on the context's stream (hp_synchronize reads the status). */
int hp_evolve_async(hp_ctx *ctx, int nsteps, int use_graph);

/* Number of sweep tile shapes per axis (the valid tile indices are
 * 0 .. hp_num_tiles()-1). */
int hp_num_tiles(void);

/* Sweep tile shape per axis (0 .. hp_num_tiles()-1; pencils per CTA x cells per window
 * step).  Results do not depend on the tile, only the speed does.  No
 * reference counterpart (the reference leaves the launch shape to PGI's
 * OpenACC compiler, ppmsolver.F90:96 `!num_gangs ... vector_length`). */
int hp_set_tiles(hp_ctx *ctx, int tile_x, int tile_y, int tile_z);
int hp_get_tiles(hp_ctx *ctx, int *tiles /* [3] */);

/* Time every tile shape of every axis on a scratch copy of the resident
 * state (reps sweeps each) and keep the fastest. */
int hp_autotune(hp_ctx *ctx, int reps);

/* One directional sweep (1=x, 2=y, 3=z) on caller-owned DEVICE arrays,
 * without any device allocation, for callers that cannot allocate: a host
 * that owns every device array and budgets device memory itself (its
 * OpenACC or CUDA data regions hold the state), a process whose device
 * memory is capped, or a framework whose caching allocator owns the device.
 * No counterpart in the reference.
 *   p..vz: device pointers, dense (nx,ny,nz) interior cells, x fastest,
 *          periodic; updated in place.  params: namelist values (nbound >= 3:
 *          the ghost layers of the reference's arrays, which the y/z
 *          density-peak test indexes) and precision; scalars: dt, rdtath,
 *          at, dat, rat, ath, dath.
 *   stream: cudaStream_t (NULL: default stream); the call returns after the
 *          stream has finished the sweep.
 * It takes no gforce: the sweep runs without the gravity source.
 * All scratch (control block + density-peak values) is one static device
 * array of 9 MiB + 4 KiB held by every device that loads the library, so
 * nx*ny*nz may not exceed 1,048,576 cells (HP_ERR_ARG beyond).  The first
 * call on a device looks up the array's address (cudaGetSymbolAddress);
 * make that first call before any stream capture.  Calls share the array:
 * calls that overlap on the GPU race. */
int hp_ppmsolver_noalloc(double *p, double *rho, double *vx, double *vy,
                         double *vz, int nx, int ny, int nz, int ndirection,
                         const hp_params *params, const hp_scalars *scalars,
                         void *stream);

/* ---------------------------------------------------------------------
 * Batches: many independent boxes advanced together.  No counterpart in
 * the reference, which advances one box per run (main.F90:100-121, the
 * time loop over evolve_sys); every member box follows exactly the
 * reference's step (its own nrot, dt, nstep and tstop), so a box advanced
 * in a batch is bitwise identical to the same box advanced alone by
 * hp_evolve with the same tiles.
 *
 * Members are contexts created by hp_init on the batch's device with the
 * batch's precision, with their state attached and no gravity source
 * (hp_batch_add returns HP_ERR_ARG otherwise).  Each sweep of a step is
 * one persistent launch per sweep axis over all members, pulling groups of
 * pencils of any member from one work queue.
 * --------------------------------------------------------------------- */
typedef struct hp_batch hp_batch;

/* capacity: the largest number of members at any time. */
int hp_batch_create(hp_batch **out, int device, int precision, int capacity);
/* Waits for the batch's work; the members stay valid (they are not freed). */
int hp_batch_destroy(hp_batch *b);

/* Add / remove a member between steps.  While it is a member a context is
 * driven only by the batch: call no other hp_* function on it except
 * hp_get_scalars / hp_download_state / hp_sync_to_host after
 * hp_batch_synchronize.  Removing waits for the batch's pending work. */
int hp_batch_add(hp_batch *b, hp_ctx *ctx);
int hp_batch_remove(hp_batch *b, hp_ctx *ctx);
int hp_batch_size(hp_batch *b);

/* Enqueue nsteps evolve_sys steps of every member and return without
 * waiting.  use_graph=1 replays one CUDA graph per nrot while every member
 * is at the same nrot (an ensemble started together); other steps are
 * launched directly.  Errors here are launch errors only; the members'
 * device status is read by hp_batch_synchronize. */
int hp_batch_step(hp_batch *b, int nsteps, int use_graph);

/* Wait for the batch's work.  status[i] (if not NULL; one entry per member
 * in the order of hp_batch_member) receives the error code of member i's
 * device status word since the last call (then cleared); returns the first
 * non-zero one. */
int hp_batch_synchronize(hp_batch *b, int *status);
hp_ctx *hp_batch_member(hp_batch *b, int i);

/* Tile shape per axis of the batched sweeps (as hp_set_tiles), and
 * the autotuner over the current members (on scratch copies of their
 * states; the states are not changed). */
int hp_batch_set_tiles(hp_batch *b, int tile_x, int tile_y, int tile_z);
int hp_batch_get_tiles(hp_batch *b, int *tiles /* [3] */);
int hp_batch_autotune(hp_batch *b, int reps);

/* CUDA stream of the batch (cudaStream_t) and its kernel launch count. */
void *hp_batch_stream(hp_batch *b);
long long hp_batch_launch_count(hp_batch *b);

/* ---------------------------------------------------------------------
 * One box split into z slabs, one per GPU (the reference's Cartesian
 * decomposition along z, init_sys.F90:53-60, with one block per rank).
 * Each slab is a context created by hp_init with ngridz = its own planes;
 * the x and y sweeps are local, the z sweep reads 4 planes below and 3
 * above from halo buffers that the caller refills before every z sweep
 * (the ghost exchange of exchange_mesh.F90 / exchange_var.F90 between
 * ranks), and the CFL velmax of a step is the maximum over the slabs
 * (the MPI_Allreduce of speed.F90).  No counterpart for the step pieces in
 * the reference, whose evolve_sys does all of it in one routine.
 * --------------------------------------------------------------------- */

/* Make ctx the slab of planes [z0, z0 + ngridz) of a periodic box of
 * nz_global planes (ngridz >= 4): dx becomes 1/max(ngridx, ngridy,
 * nz_global), halo buffers are allocated.  Call after hp_init, before the
 * first step.  hp_evolve / hp_ppm_lxlylz then return HP_ERR_ARG (a slab
 * steps through hp_step_*). */
int hp_slab_init(hp_ctx *ctx, int nz_global, int z0);

/* The planes its neighbours need, into caller DEVICE buffers in the halo
 * layout [p, rho, vx, vy, vz][planes][ngridx*ngridy]: top4 = the top 4
 * planes (the lower halo of the slab above), bottom3 = the bottom 3 planes
 * (the upper halo of the slab below).  Returns when the copies are done. */
int hp_slab_get_edges(hp_ctx *ctx, double *top4, double *bottom3);

/* Refill the halos from caller DEVICE buffers of the same layout: lower4 =
 * the 4 planes below the slab (the top4 of the slab below), upper3 = the 3
 * planes above (the bottom3 of the slab above).  The caller's writes to
 * them must be complete; the copies run on the context's stream. */
int hp_slab_set_halos(hp_ctx *ctx, const double *lower4, const double *upper3);

/* A step in pieces (any context, slab or not): hp_step_axis gives the axis
 * (0 x, 1 y, 2 z) of sweep slot s of the current step (the nrot order,
 * evolve_sys.F90:30-31); hp_step_sweep runs that sweep (a slab's z sweep
 * reads its halos; refill them first); hp_step_velmax returns the step's
 * velmax after slot 2; hp_step_finish runs timedet with the given velmax
 * (the maximum over all slabs) and advances the step, returning the status
 * accumulated since the last read.  Sweeps of a slab report
 * HP_ERR_UNSUPPORTED if the density-peak fix could act in the z sweep (its
 * transposed gather reaches across slabs; inert at the namelist dmax). */
int hp_step_axis(hp_ctx *ctx, int s);
int hp_step_sweep(hp_ctx *ctx, int s);
int hp_step_velmax(hp_ctx *ctx, double *velmax);
int hp_step_finish(hp_ctx *ctx, double velmax);

/* Block until the context's stream is idle and return the device status
 * word accumulated since the last call (then cleared). */
int hp_synchronize(hp_ctx *ctx);

/* Dense index (x + nx*(y + ny*z)) of the first updated cell that the last
 * non-zero status word read by hp_synchronize / hp_evolve reported (NaN, or
 * a non-positive density or pressure), or -1.  No counterpart in the
 * reference, which stops with a message only for Newton failures
 * (riemann.F90:62-65). */
long long hp_bad_cell(hp_ctx *ctx);

/* CUDA stream the context launches on (cudaStream_t), for event timing. */
void *hp_stream(hp_ctx *ctx);

/* Device pointers of the resident fields (p, rho, vx, vy, vz), dense
 * (ngridx,ngridy,ngridz) x fastest, for zero-copy access by the caller. */
int hp_device_fields(hp_ctx *ctx, double **p, double **rho, double **vx,
                     double **vy, double **vz);

const char *hp_strerror(int code);

/* Number of kernels launched by this context since creation. */
long long hp_launch_count(hp_ctx *ctx);

/* ---- The non-STENCIL build's full-pencil solver --------------------------
 * A build of the reference without -DSTENCIL sweeps each pencil whole with
 * SUBROUTINE ppm (hydro/ppm.F90:1-662), called by the #else branches of
 * ppmsolver (hydro/ppmsolver.F90:162-190, 290-318, 418-446), writes the
 * *3dnew arrays and copies them back with savetn (hydropad/savetn.F90).
 * Its arithmetic differs from the STENCIL sweep in four places, all kept:
 * the characteristic speeds of cell k use the sound speed of cell k+1
 * (ppm.F90:106-107), the density-peak fix reads cells f-2..f+1 of the
 * sweep's own pencil, pmean takes the cho3d-dependent values at density
 * peaks (ppm.F90:585-594), and the dual-energy switch divides by the largest
 * new total energy of the cell and its neighbours, 0 beyond the pencil's
 * updated cells (ppm.F90:611-621); it has no gravity source (ppm.F90:93,102
 * zero it).  FP64 only; not for z slabs or batches. */
enum { HP_VARIANT_STENCIL = 0, HP_VARIANT_PENCIL = 1 };

/* Select the sweep of hp_ppm_lxlylz, hp_evolve and the step pieces
 * (default HP_VARIANT_STENCIL).  HP_ERR_UNSUPPORTED for a mixed-precision
 * context or a z slab. */
int hp_set_variant(hp_ctx *ctx, int variant);
int hp_get_variant(hp_ctx *ctx);

/* Attach the cho3d array ppm() reads at density peaks (ghosted host array,
 * Fortran order, the shape of the state's arrays; hydropad/matrix.F90), or
 * NULL for zeros (the default).  Uploaded once; the field is static. */
int hp_attach_cho(hp_ctx *ctx, const double *cho3d, int nx, int ny, int nz,
                  int nbound);

/* Drop-in for the non-STENCIL ppmsolver (hydro/ppmsolver.F90:1-5 without
 * STENCIL): one full-pencil sweep of the attached state in place, whatever
 * hp_set_variant selected.  The host pointers identify the attached state
 * as in hp_ppmsolver (cho3d: the attached one, or NULL); the *3dnew arrays
 * are accepted and not written (the resident state is already the new one:
 * a caller's savetn would copy stale host arrays, so drop it, and read the
 * state back with hp_sync_to_host). */
int hp_ppmsolver_pencil(hp_ctx *ctx, double *p3d, double *rho3d, double *vx3d,
                        double *vy3d, double *vz3d, double *cho3d, double *nes3d,
                        const double *gforce, double *p3dnew, double *rho3dnew,
                        double *vx3dnew, double *vy3dnew, double *vz3dnew,
                        double *cho3dnew, const int *nx, const int *ny,
                        const int *nz, const int *nbound, const int *ndirection);

#ifdef __cplusplus
}
#endif
#endif
