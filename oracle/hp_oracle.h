/*
 * hp_oracle.h -- CPU restatement of Hydropad's STENCIL PPM hydro step.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load this library,
 * and only as the checker or the timed CPU baseline -- never as the product.
 *
 * PARITY UNPINNED: the reference is Fortran 90 + OpenACC and no Fortran
 * compiler exists on either machine, and the reference ships no tests, golden
 * vectors or known-answer fixtures.  This restatement follows the reference
 * line by line (file:line cited per function in hp_oracle.c) and is pinned
 * only by physics (exact Sod solution, conservation, axis symmetry) and by an
 * independent second restatement in tests/golden/gen_golden.py.
 *
 * Layout: every field is a Fortran column-major REAL(8) array (nx,ny,nz) with
 * nbound ghost layers per side, exactly as the reference allocates it
 * (hydropad/alloc_arrays.F90:76-78,102-106).  gforce is (3,nx,ny,nz) and may
 * be NULL (gravity off: g == 0).
 */
#ifndef HP_ORACLE_H
#define HP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Module `scalar` values read by the hot path
 * (hydropad/scalar.F90:98-99, hydro/ppmsolver.F90:68-69). */
typedef struct {
    double gamma, rgamma, gamma1, rgamma1, m, rm, gf; /* initialize_parameters.F90:64-69 */
    double mingradflat, flatvalue;                    /* namelist PPM */
    double dmax, eta1, eta2, cour, ca;                /* namelist NUMERICS */
    double dx, rdx;                                   /* initialize_parameters.F90:23-24 */
    double dt, rdtath, at, dat, rat, ath, dath;       /* time scalars of the step */
    double t, told, thalf, dtold, tstop, atnew, datnew;
    double dt_cap;   /* timedet_cosmo debug cap dt0 (functions.F90:49,97); <=0 disables */
    double velmax;
    int    nstep;
    int    cosmo;    /* 1: EdS expanding background (timedet_cosmo + expand) */
    int    expand_zero_old; /* 1: expand with vxold=pold3d=0 (non-STENCIL allocation);
                               0: snapshot of v,p at step start */
    int    pencil;   /* 0: STENCIL sweeps (ppmsolver.F90 #ifdef STENCIL branches);
                        1: the non-STENCIL build's full-pencil ppm() (hydro/ppm.F90) */
} hpo_scalars;

/* Derived constants from gamma, N (initialize_parameters.F90:23-24,63-69). */
void hpo_derive_constants(hpo_scalars *s, double gamma, int ngrid_max);

/* One directional sweep, STENCIL path (hydro/ppmsolver.F90:1-467).
 * ndirection 1=x 2=y 3=z.  Arrays are updated in place; ghosts are read,
 * not written.  Returns the number of Newton failures (reference: `stop`,
 * riemann.F90:62-65) -- the face is then left with the last iterate. */
int hpo_ppmsolver(double *p3d, double *rho3d, double *vx3d, double *vy3d,
                  double *vz3d, const double *gforce, int nx, int ny, int nz,
                  int nbound, int ndirection, const hpo_scalars *s,
                  int nthreads);

/* Periodic ghost fill for one process (exchange_mesh.F90 / exchange_var.F90
 * with npes=1: every Cartesian neighbour is this rank). */
/* One sweep of the non-STENCIL build (ppmsolver.F90:162-190, 290-318,
 * 418-446 -> hydro/ppm.F90 per pencil, then savetn): the same arrays and
 * arguments as hpo_ppmsolver; cho3d (ghosted, or NULL for zeros) is the
 * cho3d array that ppm() reads at density peaks.  The gravity source is
 * ignored, as ppm() zeroes it (ppm.F90:93,102). */
int hpo_ppmsolver_pencil(double *p3d, double *rho3d, double *vx3d, double *vy3d,
                         double *vz3d, const double *cho3d, int nx, int ny, int nz,
                         int nbound, int ndirection, const hpo_scalars *s,
                         int nthreads);

void hpo_exchange_mesh(double *p3d, double *rho3d, double *vx3d, double *vy3d,
                       double *vz3d, int nx, int ny, int nz, int nbound);

/* Three sweeps in the order selected by nrot, ghost refresh after each
 * (hydro/ppm_lxlylz.F90:9-221).  Returns summed Newton failures. */
int hpo_ppm_lxlylz(double *p3d, double *rho3d, double *vx3d, double *vy3d,
                   double *vz3d, const double *gforce, int nx, int ny, int nz,
                   int nbound, int nrot, const hpo_scalars *s, int nthreads);

/* max over interior of max_d(|v_d| + sqrt(gamma p / rho)) (speed.F90:22-31). */
double hpo_speed(const double *p3d, const double *rho3d, const double *vx3d,
                 const double *vy3d, const double *vz3d, int nx, int ny,
                 int nz, int nbound, const hpo_scalars *s);

/* Static timestep (functions.F90:2-35). */
void hpo_timedet(hpo_scalars *s);
/* EdS timestep (functions.F90:38-151, omega_m = 1 branch). */
void hpo_timedet_cosmo(hpo_scalars *s);
/* Time initialisation (initialize_parameters.F90:133-205).  a_start is the
 * initial expansion factor (cosmo only). */
void hpo_init_time(hpo_scalars *s, double dtinit, double a_start);

/* Hubble drag on v and p (hydropad/expand.F90:18-41).  vxold..pold may be
 * NULL when s->expand_zero_old is set. */
void hpo_expand(double *p3d, double *vx3d, double *vy3d, double *vz3d,
                const double *pold, const double *vxold, const double *vyold,
                const double *vzold, int nx, int ny, int nz,
                const hpo_scalars *s);

/* evolve_sys for nsteps steps (hydropad/evolve_sys.F90:30-130 with HYDRO,
 * STENCIL, no NBODY): nrot schedule, ppm_lxlylz, [expand], speed, timedet.
 * Returns summed Newton failures. */
int hpo_evolve(double *p3d, double *rho3d, double *vx3d, double *vy3d,
               double *vz3d, const double *gforce, int nx, int ny, int nz,
               int nbound, hpo_scalars *s, int nsteps, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
