/*
 * hp_oracle.c -- CPU restatement of Hydropad's PPM hydro step: the STENCIL
 * build's sweeps and, for parity with a non-STENCIL build, its full-pencil
 * ppm() (hpo_ppmsolver_pencil).
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline; never the
 * product).  PARITY UNPINNED against the Fortran reference: it cannot be
 * compiled anywhere we run (no gfortran / nvfortran / MPI) and ships no tests
 * or golden vectors.  Every routine below restates one reference routine
 * line by line; the reference file:line is given on each.
 *
 * Fortran-semantics rules followed throughout:
 *  - unsuffixed Fortran literals are REAL(4); their double values are used
 *    (0.16666667 -> 0.1666666716337204 and so on, see the HPO_* constants);
 *  - operators of equal precedence evaluate left to right, `**` with a real
 *    exponent is pow(), `x**2` is x*x;
 *  - build with -ffp-contract=off so no multiply-add is fused.
 *
 * Decisions where the reference is undefined (each also noted in place):
 *  - integrate.F90:75 reads `pmean` uninitialised (HIGHPEAKS undefined).  We
 *    use pmean = (pm1+pm2)*0.5, the non-STENCIL definition (ppm.F90:583).
 *  - order2interp.F90:68-70 keeps a stale `gradleft` when a product is zero;
 *    the stale value is kept here too, starting from 0 at routine entry.
 *  - riemannsolver: a face whose inputs match no wave pattern (NaN inputs)
 *    leaves pm/rhom/vxm undefined in the reference; here they become NaN.
 */
#include "hp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* REAL(4) literals promoted to REAL(8). */
#define HPO_SIXTH   0.1666666716337204      /* 0.16666667 */
#define HPO_THIRD   0.3333333432674408      /* 0.33333333 */
#define HPO_TINY    1.0000000036274937e-15  /* 1e-15      */
#define HPO_TERR    0.0010000000474974513   /* 1e-3       */
#define HPO_C010    0.009999999776482582    /* 0.010      */
#define HPO_C050    0.05000000074505806     /* 0.050      */
#define HPO_C0P1    0.10000000149011612     /* 0.1        */
#define HPO_TWO3    0.6666666865348816      /* 2.0/3.0    */
#define HPO_MTHIRD  (-0.3333333432674408)   /* -1.0/3.0   */
#define HPO_C0P010  0.009999999776482582    /* 0.010      */

/* Fortran MIN / MAX of two or three reals. */
static inline double fmin2(double a, double b) { return b < a ? b : a; }
static inline double fmax2(double a, double b) { return b > a ? b : a; }
static inline double fmin3(double a, double b, double c) { return fmin2(fmin2(a, b), c); }

/* Column-major (nx,ny,nz) index, 1-based like the Fortran source. */
#define IX(i, j, k) ((size_t)((i) - 1) + (size_t)nx * ((size_t)((j) - 1) + (size_t)ny * (size_t)((k) - 1)))

void hpo_derive_constants(hpo_scalars *s, double gamma, int ngrid_max)
{
    /* initialize_parameters.F90:23-24 and :64-69 */
    s->dx = 1.0 / (double)ngrid_max;
    s->rdx = 1.0 / s->dx;
    s->gamma = gamma;
    s->rgamma = 1.0 / gamma;
    s->gamma1 = (gamma + 1.0) / (gamma - 1.0);
    s->rgamma1 = 1.0 / (gamma - 1.0);
    s->m = (gamma - 1.0) / (2.0 * gamma);
    s->rm = 1.0 / s->m;
    s->gf = (gamma + 1.0) / (2.0 * gamma);
}

/* ------------------------------------------------------------------ */
/* hydro/ppm_functs.F90                                                */
/* ------------------------------------------------------------------ */

/* ajside, ppm_functs.F90:167-181 */
static double ajside(double am1, double a, double ap1)
{
    if ((ap1 - a) * (a - am1) > 0.0) {
        double da = 0.5 * (ap1 - am1);
        return fmin3(fabs(da), 2.0 * fabs(a - am1), 2.0 * fabs(ap1 - a)) * da / fabs(da);
    }
    return 0.0;
}

/* fl, ppm_functs.F90:91-105 (uses slot 1 of the two-slot arrays) */
static double fl(const double ajr[3], const double d[3], const double a6[3], double y, const hpo_scalars *s)
{
    double x = y / s->dx;
    return ajr[1] - 0.5 * x * (d[1] - (1.0 - 2.0 * x * HPO_THIRD) * a6[1]);
}

/* fr, ppm_functs.F90:110-124 (uses slot 2) */
static double fr(const double ajl[3], const double d[3], const double a6[3], double y, const hpo_scalars *s)
{
    double x = y / s->dx;
    return ajl[2] + 0.5 * x * (d[2] + (1.0 - 2.0 * x * HPO_THIRD) * a6[2]);
}

/* beta, ppm_functs.F90:129-144 */
static double beta(double ct, double ut, double uc, double pt, double pc, double gc, double sign, const hpo_scalars *s)
{
    double gvc = (-gc + s->dat * uc) * s->rat;
    return -(sign * ((ut - uc) + sign * (pt - pc) / ct + sign * s->dt * (2.0 * s->dat * pc / (ct * s->at)) + s->dt * gvc)) / (2.0 * ct);
}

/* beta0, ppm_functs.F90:149-162 */
static double beta0(double ct, double rhot, double rhoc, double pt, double pc, const hpo_scalars *s)
{
    return (pt - pc) / (ct * ct) + 1.0 / rhot - 1.0 / rhoc + (2.0 * s->dat * pc) / (s->at * ct * ct) * s->dt;
}

/* dda, hydro/dda.F90:1-35.  a[1..5] */
static void dda(const double *a, double *eta, double *ajld, double *ajrd, double dmalf, double dmarg, const hpo_scalars *s)
{
    const double mmmax = 0.0, mmmin = 1.0;
    double deltam2 = HPO_SIXTH * (a[3] - 2.0 * a[2] + a[1]) / (s->dx * s->dx);
    double deltap2 = HPO_SIXTH * (a[5] - 2.0 * a[4] + a[3]) / (s->dx * s->dx);
    double agrad = fabs(a[4] - a[2]) - HPO_C010 * fmin2(fabs(a[4]), fabs(a[2]));
    if (-(deltam2 * deltap2) > 0.0 && agrad > 0.0) {
        double e = -((deltap2 - deltam2) * s->dx * s->dx / (a[4] - a[2]));
        *eta = fmax2(mmmax, fmin2(20.0 * (e - HPO_C050), mmmin));
    } else {
        *eta = 0.0;
    }
    *ajld = a[2] + 0.5 * dmalf;
    *ajrd = a[4] - 0.5 * dmarg;
}

/* correction, ppm_functs.F90:1-86.  a[1..5]; two-slot arrays use [1],[2];
 * acl/acr use [1..3]. */
static void correction(double addp, double addrho, const double *a, double ajl[3], double ajr[3],
                       double deltaa1[3], double a6[3], const double ccc[3], double vi, double vip1,
                       double *atl, double *atr, double acl[4], double acr[4], double flat, int ndda,
                       const hpo_scalars *s)
{
    const double mmmax = 0.0;
    double dmaj = ajside(a[1], a[2], a[3]);
    double dmajp1 = ajside(a[2], a[3], a[4]);
    double dmajp2 = ajside(a[3], a[4], a[5]);
    ajl[2] = a[2] + 0.5 * (a[3] - a[2]) + (dmaj - dmajp1) * HPO_SIXTH;
    ajr[2] = a[3] + 0.5 * (a[4] - a[3]) + (dmajp1 - dmajp2) * HPO_SIXTH;
    if (ndda == 1 && addrho >= addp) {
        double eta, ajld, ajrd;
        dda(a, &eta, &ajld, &ajrd, dmaj, dmajp2, s);
        ajl[2] = (1.0 - eta) * ajl[2] + eta * ajld;
        ajr[2] = (1.0 - eta) * ajr[2] + eta * ajrd;
    }
    deltaa1[2] = ajr[2] - ajl[2];
    a6[2] = 6.0 * (a[3] - 0.5 * (ajl[2] + ajr[2]));
    if ((ajr[2] - a[3]) * (a[3] - ajl[2]) <= 0.0) {
        ajl[2] = a[3];
        ajr[2] = a[3];
    } else if (deltaa1[2] * a6[2] > deltaa1[2] * deltaa1[2]) {
        ajl[2] = 3.0 * a[3] - 2.0 * ajr[2];
    } else if (deltaa1[2] * a6[2] < -(deltaa1[2] * deltaa1[2])) {
        ajr[2] = 3.0 * a[3] - 2.0 * ajl[2];
    }
    ajl[2] = flat * a[3] + (1.0 - flat) * ajl[2];
    ajr[2] = flat * a[3] + (1.0 - flat) * ajr[2];
    deltaa1[2] = ajr[2] - ajl[2];
    a6[2] = 6.0 * (a[3] - 0.5 * (ajl[2] + ajr[2]));

    double cv, y;
    cv = s->dt * (vi + ccc[1]) * s->rat;
    y = fmax2(cv, mmmax);
    *atl = fl(ajr, deltaa1, a6, y, s);
    cv = -(s->dt * (vip1 - ccc[2]) * s->rat);
    y = fmax2(cv, mmmax);
    *atr = fr(ajl, deltaa1, a6, y, s);

    y = s->dt * (vi - ccc[1]) * s->rat;
    acl[1] = fl(ajr, deltaa1, a6, y, s);
    y = s->dt * vi * s->rat;
    acl[2] = fl(ajr, deltaa1, a6, y, s);
    y = s->dt * (vi + ccc[1]) * s->rat;
    acl[3] = fl(ajr, deltaa1, a6, y, s);

    y = -(s->dt * (vip1 - ccc[2]) * s->rat);
    acr[1] = fr(ajl, deltaa1, a6, y, s);
    y = -(s->dt * vip1 * s->rat);
    acr[2] = fr(ajl, deltaa1, a6, y, s);
    y = -(s->dt * (vip1 + ccc[2]) * s->rat);
    acr[3] = fr(ajl, deltaa1, a6, y, s);
}

/* ------------------------------------------------------------------ */
/* hydro/order2interp.F90:1-265, STENCIL call: ngrid=6, nmin=3, nmax=4 */
/* Arrays pres..c are 1-based [1..6] = cells i-3..i+2 of face i.      */
/* ------------------------------------------------------------------ */
typedef struct {
    double jl[3], jr[3], d[3], a6[3];
} slot2;

static void order2interp(const double *pres, const double *rho, const double *vx, const double *vy,
                         const double *vz, const double *g, const double *c, double *pleft,
                         double *pright, double *rholeft, double *rhoright, double *vxleft,
                         double *vxright, double *vyleft, double *vyright, double *vzleft,
                         double *vzright, const hpo_scalars *s)
{
    const int nmin = 3, nmax = 4;
    /* slot (1) starts uninitialised in the reference and is only read in the
     * discarded first iteration; zero it here. */
    slot2 P, R, VX, VY, VZ, G;
    memset(&P, 0, sizeof P); memset(&R, 0, sizeof R); memset(&VX, 0, sizeof VX);
    memset(&VY, 0, sizeof VY); memset(&VZ, 0, sizeof VZ); memset(&G, 0, sizeof G);
    double gradleft = 0.0; /* stale across pairs/variables/iterations (:68-70) */
    double cbar[3];

    for (int i = nmin; i <= nmax; ++i) {
        int mainindex = i - nmin + 1;
        double flat = 0.0;
        cbar[1] = c[i - 1];
        cbar[2] = c[i];

        /* inline flattening, :65-113 */
        const double *vars[5] = {pres, rho, vx, vy, vz};
        for (int v = 0; v < 5; ++v) {
            const double *a = vars[v];
            double gradmax = 0.0;
            for (int ii = 1; ii <= 4; ++ii) {
                int ic = mainindex + ii;
                if (a[ic] * a[ic - 1] != 0.0)
                    gradleft = fabs((a[ic] - a[ic - 1]) / fmin2(a[ic], a[ic - 1]));
                gradmax = fmax2(gradmax, gradleft);
            }
            if (gradmax >= s->mingradflat) flat = s->flatvalue;
        }

        /* shift slot 2 -> slot 1, :120-147 */
        slot2 *all[6] = {&P, &R, &VX, &VY, &VZ, &G};
        for (int v = 0; v < 6; ++v) {
            all[v]->jl[1] = all[v]->jl[2];
            all[v]->jr[1] = all[v]->jr[2];
            all[v]->d[1] = all[v]->d[2];
            all[v]->a6[1] = all[v]->a6[2];
        }

        double addp = fabs(pres[i + 1] - pres[i - 1]) / fmin2(pres[i - 1], pres[i + 1]);
        double addrho = 0.5 * s->gamma * fabs(rho[i + 1] - rho[i - 1]) / fmin2(rho[i - 1], rho[i + 1]);

        double ptl, ptr, pcl[4], pcr[4];
        double rhotl, rhotr, rhocl[4], rhocr[4];
        double vxtl, vxtr, vxcl[4], vxcr[4];
        double vytl, vytr, vycl[4], vycr[4];
        double vztl, vztr, vzcl[4], vzcr[4];
        double gtl, gtr, gcl[4], gcr[4];
        /* a(1..5) = array(mainindex .. mainindex+4): pass base so that a[1]
         * is array[mainindex] */
        correction(addp, addrho, pres + mainindex - 1, P.jl, P.jr, P.d, P.a6, cbar, vx[i - 1], vx[i],
                   &ptl, &ptr, pcl, pcr, flat, 0, s);
        correction(addp, addrho, rho + mainindex - 1, R.jl, R.jr, R.d, R.a6, cbar, vx[i - 1], vx[i],
                   &rhotl, &rhotr, rhocl, rhocr, flat, 1, s);
        correction(addp, addrho, vx + mainindex - 1, VX.jl, VX.jr, VX.d, VX.a6, cbar, vx[i - 1], vx[i],
                   &vxtl, &vxtr, vxcl, vxcr, flat, 0, s);
        correction(addp, addrho, vy + mainindex - 1, VY.jl, VY.jr, VY.d, VY.a6, cbar, vx[i - 1], vx[i],
                   &vytl, &vytr, vycl, vycr, flat, 0, s);
        correction(addp, addrho, vz + mainindex - 1, VZ.jl, VZ.jr, VZ.d, VZ.a6, cbar, vx[i - 1], vx[i],
                   &vztl, &vztr, vzcl, vzcr, flat, 0, s);
        correction(addp, addrho, g + mainindex - 1, G.jl, G.jr, G.d, G.a6, cbar, vx[i - 1], vx[i],
                   &gtl, &gtr, gcl, gcr, flat, 0, s);

        /* negative traced states, :174-190 (the reference also prints) */
        if (ptl < 0.0) ptl = HPO_TINY;
        if (ptr < 0.0) ptr = HPO_TINY;
        if (rhotl < 0.0) rhotl = HPO_TINY;
        if (rhotr < 0.0) rhotr = HPO_TINY;

        double ctl = sqrt(s->gamma * ptl * rhotl);
        double ctr = sqrt(s->gamma * ptr * rhotr);
        double lambdam = (vx[i - 1] - cbar[1]) * s->rat;
        double lambda0 = vx[i - 1] * s->rat;
        double lambdap = (vx[i - 1] + cbar[1]) * s->rat;
        double betaml, betapl, beta0l, betamr, betapr, beta0r;
        double vyl, vzl, vyr, vzr;
        if (lambdam <= 0.0) betaml = 0.0;
        else betaml = beta(ctl, vxtl, vxcl[1], ptl, pcl[1], gcl[1], -1.0, s);
        if (lambdap <= 0.0) { betapl = 0.0; vyl = vytl; vzl = vztl; }
        else { betapl = beta(ctl, vxtl, vxcl[3], ptl, pcl[3], gcl[3], 1.0, s); vyl = vytl; vzl = vztl; }
        if (lambda0 <= 0.0) beta0l = 0.0;
        else { beta0l = beta0(ctl, rhotl, rhocl[2], ptl, pcl[2], s); vyl = vycl[2]; vzl = vzcl[2]; }

        lambdam = (vx[i] - cbar[2]) * s->rat;
        lambda0 = vx[i] * s->rat;
        lambdap = (vx[i] + cbar[2]) * s->rat;
        if (lambdap >= 0.0) betapr = 0.0;
        else betapr = beta(ctr, vxtr, vxcr[3], ptr, pcr[3], gcr[3], 1.0, s);
        if (lambdam >= 0.0) { betamr = 0.0; vyr = vytr; vzr = vztr; }
        else { betamr = beta(ctr, vxtr, vxcr[1], ptr, pcr[1], gcr[1], -1.0, s); vyr = vytr; vzr = vztr; }
        if (lambda0 >= 0.0) beta0r = 0.0;
        else { beta0r = beta0(ctr, rhotr, rhocr[2], ptr, pcr[2], s); vyr = vycr[2]; vzr = vzcr[2]; }

        *pleft = ptl + ctl * ctl * (betapl + betaml);
        if (*pleft <= 0.0) *pleft = ptl;
        *pright = ptr + ctr * ctr * (betapr + betamr);
        if (*pright <= 0.0) *pright = ptr;
        *vxleft = vxtl + ctl * (betapl - betaml);
        *vxright = vxtr + ctr * (betapr - betamr);
        *rholeft = 1.0 / (1.0 / rhotl - betaml - beta0l - betapl);
        if (*rholeft <= 0.0) *rholeft = rhotl;
        *rhoright = 1.0 / (1.0 / rhotr - betamr - beta0r - betapr);
        if (*rhoright <= 0.0) *rhoright = rhotr;
        *vyleft = vyl; *vzleft = vzl; *vyright = vyr; *vzright = vzr;
        /* cleft/cright (:259-260) are computed but unused */
    }
}

/* ------------------------------------------------------------------ */
/* hydro/riemann.F90:1-111                                             */
/* ------------------------------------------------------------------ */
static double rarwave(double f1, double f2, double vt, double vh)   /* :1-9 */
{
    return f2 + vt * (f1 - f2) / (vt - vh);
}

static double rhoshock(double p2, double p1, double rho1, const hpo_scalars *s) /* :14-24 */
{
    return rho1 * (s->gamma1 * p2 / p1 + 1.0) / (s->gamma1 + p2 / p1);
}

/* riemann, :29-111.  Returns 1 on Newton non-convergence (reference: stop). */
static int riemann(double *pstar, double *vstar, double pleft, double pright, double rholeft,
                   double rhoright, double vxleft, double vxright, const hpo_scalars *s)
{
    double err = 1.e10;
    const double terr = HPO_TERR;
    int nnewt = 0;
    const int nnewtmax = 100;
    double kappa = sqrt(s->gamma * (pleft + pright) * (rholeft + rhoright) * 0.25);
    double pcheck = 0.5 * (pleft + pright) + 0.5 * kappa * (vxleft + vxright);
    if (pcheck > 0.0) *pstar = pcheck;
    while (err > terr) {
        nnewt = nnewt + 1;
        if (nnewt > nnewtmax) return 1;
        double pstarold = *pstar;
        double cleft = sqrt(s->gamma * pleft * rholeft);
        double cright = sqrt(s->gamma * pright * rhoright);
        double a, b, vprimel, vprimer;
        double pstup = (1.0 - pow(*pstar / pleft, s->m));
        if (*pstar >= pleft) a = cleft * sqrt(s->gf * *pstar / pleft + s->m);
        else if (pstup == 0.0) a = cleft * sqrt(s->gf * *pstar / pleft + s->m);
        else a = s->m * cleft * (1.0 - *pstar / pleft) / (1.0 - pow(*pstar / pleft, s->m));
        pstup = (1.0 - pow(*pstar / pright, s->m));
        if (*pstar >= pright) b = cright * sqrt(s->gf * *pstar / pright + s->m);
        else if (pstup == 0.0) b = cright * sqrt(s->gf * *pstar / pright + s->m);
        else b = s->m * cright * (1.0 - *pstar / pright) / (1.0 - pow(*pstar / pright, s->m));
        if (*pstar >= pleft) vprimel = -((a * a + cleft * cleft) / (2.0 * a * a * a));
        else vprimel = -((1.0 / cleft) * pow(*pstar / pleft, -s->gf));
        if (*pstar >= pright) vprimer = (b * b + cright * cright) / (2.0 * b * b * b);
        else vprimer = (1.0 / cright) * pow(*pstar / pright, -s->gf);
        double vstarl = vxleft - (*pstar - pleft) / a;
        double vstarr = vxright + (*pstar - pright) / b;
        *pstar = *pstar - (vstarl - vstarr) / (vprimel - vprimer);
        if (*pstar <= 0.0) *pstar = pstarold / 1000.0;
        *vstar = (pleft - pright + a * vxleft + b * vxright) / (a + b);
        err = fabs(pstarold - *pstar) / pstarold;
    }
    return 0;
}

/* riemannsolver, :1-289.  rhobar/vxbar are 1-based [1..6]. */
static int riemannsolver(const double *rhobar, const double *vxbar, double pleft, double pright,
                         double rholeft, double rhoright, double vxleft, double vxright, double vyleft,
                         double vyright, double vzleft, double vzright, double *pm_o, double *rhom_o,
                         double *vxm_o, double *vym_o, double *vzm_o, const hpo_scalars *s)
{
    const double gamma = s->gamma, m = s->m, rm = s->rm, rgamma = s->rgamma, rgamma1 = s->rgamma1;
    int fail = 0;
    double cleft = sqrt(gamma * pleft / rholeft);
    double cright = sqrt(gamma * pright / rhoright);
    double dadt = 1.0 - 0.5 * s->dat * s->dt * s->rat;
    const double mmmax = 0.0;
    double p1, p2, vx1, vx2, rho1, rho2, c1, c2;
    if (pleft <= pright) {
        p1 = pleft; p2 = pright; vx1 = vxleft; vx2 = vxright;
        rho1 = rholeft; rho2 = rhoright; c1 = cleft; c2 = cright;
    } else {
        p1 = pright; p2 = pleft; vx1 = vxleft; vx2 = vxright;
        rho1 = rhoright; rho2 = rholeft; c1 = cright; c2 = cleft;
    }
    (void)vx1; (void)vx2; (void)rho2; (void)c1;
    double dvv = vx1 - vx2;
    double dv2s = (p2 - p1) / sqrt(0.5 * rho1 * ((gamma - 1.0) * p1 + (gamma + 1.0) * p2));
    double dv1s = -((2.0 * c2 / (gamma - 1.0)) * (1.0 - pow(p1 / p2, m)));
    double dv2r = -(2.0 * (c1 + c2) * rgamma1);

    double pm = NAN, vxm = NAN, rhom = NAN;
    double rhoshock1, rhoshock2, vshock1, vshock2, rhocont1, rhocont2;
    double vtail1, vtail2, vhead1, vhead2, zeta, vtleft, vtright;

    if (dvv >= dv2s) {                                                       /* :73-109 */
        pm = fmax2(pleft, pright);
        fail |= riemann(&pm, &vxm, pleft, pright, rholeft, rhoright, vxleft, vxright, s);
        rhoshock1 = rhoshock(pm, pleft, rholeft, s);
        rhoshock2 = rhoshock(pm, pright, rhoright, s);
        if (rhoshock1 == rholeft) vshock1 = 0.0;
        else vshock1 = (rhoshock1 * vxm - rholeft * vxleft) / (rhoshock1 - rholeft);
        if (rhoshock2 == rhoright) vshock2 = 0.0;
        else vshock2 = (rhoshock2 * vxm - rhoright * vxright) / (rhoshock2 - rhoright);
        if (vshock2 < 0.0) { pm = pright; vxm = vxright; rhom = rhoright; }
        else if (vxm <= 0.0 && vshock2 >= 0.0) rhom = rhoshock2;
        else if (vshock1 <= 0.0 && vxm > 0.0) rhom = rhoshock1;
        else { pm = pleft; vxm = vxleft; rhom = rholeft; }
    } else if (dvv < dv2s && dvv >= dv1s) {                                  /* :113-184 */
        pm = pow((cleft + cright + (vxleft - vxright) * (gamma - 1.0) * 0.5) /
                     (cleft / pow(pleft, m) + cright / pow(pright, m)), rm);
        fail |= riemann(&pm, &vxm, pleft, pright, rholeft, rhoright, vxleft, vxright, s);
        if (pleft >= pright) {
            rhoshock2 = rhoshock(pm, pright, rhoright, s);
            rhocont1 = rholeft * pow(pm / pleft, rgamma);
            if (rhoshock2 == rhoright) vshock2 = 0.0;
            else vshock2 = (rhoshock2 * vxm - rhoright * vxright) / (rhoshock2 - rhoright);
            vtail1 = vxm - sqrt(gamma * pm / rhocont1);
            vhead1 = vxleft - cleft;
            if (vshock2 < 0.0) { pm = pright; vxm = vxright; rhom = rhoright; }
            else if (vhead1 >= 0.0) { pm = pleft; vxm = vxleft; rhom = rholeft; }
            else if (vxm <= 0.0 && vshock2 >= 0.0) rhom = rhoshock2;
            else if (vxm > 0.0 && vtail1 <= 0.0) rhom = rhocont1;
            else if (vtail1 > 0.0 && vhead1 <= 0.0) {
                pm = rarwave(pleft, pm, vtail1, vhead1);
                rhom = rarwave(rholeft, rhocont1, vtail1, vhead1);
                vxm = rarwave(vxleft, vxm, vtail1, vhead1);
            }
        } else {
            rhoshock1 = rhoshock(pm, pleft, rholeft, s);
            rhocont2 = rhoright * pow(pm / pright, rgamma);
            if (rhoshock1 == rholeft) vshock1 = 0.0;
            else vshock1 = (rhoshock1 * vxm - rholeft * vxleft) / (rhoshock1 - rholeft);
            vtail2 = vxm + sqrt(gamma * pm / rhocont2);
            vhead2 = vxright + cright;
            if (vshock1 > 0.0) { pm = pleft; vxm = vxleft; rhom = rholeft; }
            else if (vhead2 <= 0.0) { pm = pright; vxm = vxright; rhom = rhoright; }
            else if (vxm >= 0.0 && vshock1 <= 0.0) rhom = rhoshock1;
            else if (vxm < 0.0 && vtail2 >= 0.0) rhom = rhocont2;
            else if (vtail2 < 0.0 && vhead2 >= 0.0) {
                pm = rarwave(pright, pm, vtail2, vhead2);
                rhom = rarwave(rhoright, rhocont2, vtail2, vhead2);
                vxm = rarwave(vxright, vxm, vtail2, vhead2);
            }
        }
    } else if (dvv < dv1s && dvv > dv2r) {                                   /* :188-227 */
        zeta = (cright / cleft) * pow(pleft / pright, m);
        vtleft = vxleft + 2.0 * cleft * rgamma1;
        vtright = vxright - 2.0 * cright * rgamma1;
        vxm = (vtleft * zeta + vtright) / (1.0 + zeta);
        pm = pleft * pow((gamma - 1.0) * (vtleft - vtright) / (2.0 * cleft * (1.0 + zeta)), rm);
        rhocont1 = rholeft * pow(pm / pleft, rgamma);
        rhocont2 = rhoright * pow(pm / pright, rgamma);
        vtail2 = vxm + sqrt(gamma * pm / rhocont2);
        vhead2 = vxright + cright;
        vtail1 = vxm - sqrt(gamma * pm / rhocont1);
        vhead1 = vxleft - cleft;
        if (vhead2 <= 0.0) { pm = pright; vxm = vxright; rhom = rhoright; }
        else if (vhead1 >= 0.0) { pm = pleft; vxm = vxleft; rhom = rholeft; }
        else if (vhead2 > 0.0 && vtail2 <= 0.0) {
            pm = rarwave(pright, pm, vtail2, vhead2);
            rhom = rarwave(rhoright, rhocont2, vtail2, vhead2);
            vxm = rarwave(vxright, vxm, vtail2, vhead2);
        } else if (vxm <= 0.0 && vtail2 > 0.0) rhom = rhocont2;
        else if (vxm > 0.0 && vtail1 <= 0.0) rhom = rhocont1;
        else if (vtail1 > 0.0 && vhead1 <= 0.0) {
            pm = rarwave(pleft, pm, vtail1, vhead1);
            rhom = rarwave(rholeft, rhocont1, vtail1, vhead1);
            vxm = rarwave(vxleft, vxm, vtail1, vhead1);
        }
    } else if (dvv <= dv2r) {                                                /* :231-264 */
        pm = 0.0; vxm = 0.0; rhocont1 = 0.0; rhocont2 = 0.0;
        vtail2 = vxright - 2.0 * cright * rgamma1;
        vhead2 = vxright + cright;
        vtail1 = vxleft - 2.0 * cleft * rgamma1;
        vhead1 = vxleft - cleft;
        if (vhead2 <= 0.0) { pm = pright; vxm = vxright; rhom = rhoright; }
        else if (vhead1 >= 0.0) { pm = pleft; vxm = vxleft; rhom = rholeft; }
        else if (vhead2 > 0.0 && vtail2 <= 0.0) {
            pm = rarwave(pright, pm, vtail2, vhead2);
            rhom = rarwave(rhoright, rhocont2, vtail2, vhead2);
            vxm = rarwave(vxright, vxm, vtail2, vhead2);
        } else if (vtail1 <= 0.0 && vtail2 > 0.0) rhom = 0.0;
        else if (vtail1 > 0.0 && vhead1 <= 0.0) {
            pm = rarwave(pleft, pm, vtail1, vhead1);
            rhom = rarwave(rholeft, rhocont1, vtail1, vhead1);
            vxm = rarwave(vxleft, vxm, vtail1, vhead1);
        }
    }
    double vym, vzm;                                                         /* :269-275 */
    if (vxm >= 0.0) { vym = dadt * vyleft; vzm = dadt * vzleft; }
    else { vym = dadt * vyright; vzm = dadt * vzright; }
    if (rhobar[2] > s->dmax * rhobar[1] && rhobar[3] > s->dmax * rhobar[4]) { /* :279-285 */
        double maxp = (vxbar[2] - vxbar[3]) * fmax2(rhobar[2], rhobar[3]) * fmax2(mmmax, vxbar[2] - vxbar[3]);
        pm = fmax2(pm, maxp);
    }
    *pm_o = pm; *rhom_o = rhom; *vxm_o = vxm; *vym_o = vym; *vzm_o = vzm;
    return fail;
}

/* ------------------------------------------------------------------ */
/* hydro/integrate.F90:1-113, total.F90, internal.F90                  */
/* ------------------------------------------------------------------ */
static double total(double p, double rho, double vx, double vy, double vz, const hpo_scalars *s)
{
    return p * s->rgamma1 + 0.5 * rho * (vx * vx + vy * vy + vz * vz);   /* total.F90:15 */
}
static double internal(double p, const hpo_scalars *s) { return p * s->rgamma1; } /* internal.F90:14 */

static void integrate(double pm1, double pm2, double rhom1, double rhom2, double vxm1, double vxm2,
                      double vym1, double vym2, double vzm1, double vzm2, double *pres, double *rho,
                      double *vx, double *vy, double *vz, double etot, double eint, double ghalf,
                      const hpo_scalars *s)
{
    const double gamma = s->gamma, rgamma1 = s->rgamma1, rdtath = s->rdtath, rdx = s->rdx;
    double flux1, flux2, grav;
    flux1 = rhom1 * vxm1;
    flux2 = rhom2 * vxm2;
    double rhonew = *rho + rdtath * (flux1 - flux2) * rdx;
    flux1 = rhom1 * vxm1 * vxm1 + pm1;
    flux2 = rhom2 * vxm2 * vxm2 + pm2;
    grav = (*rho + rhonew) * ghalf * 0.5;
    double vxnew = (*vx * *rho + rdtath * (flux1 - flux2) * rdx + rdtath * grav) / rhonew;
    flux1 = vym1 * vxm1 * rhom1;
    flux2 = vym2 * vxm2 * rhom2;
    double vynew = (*rho * *vy + rdtath * (flux1 - flux2) * rdx) / rhonew;
    flux1 = vzm1 * vxm1 * rhom1;
    flux2 = vzm2 * vxm2 * rhom2;
    double vznew = (*rho * *vz + rdtath * (flux1 - flux2) * rdx) / rhonew;
    flux1 = (gamma * pm1 * rgamma1 + 0.5 * rhom1 * (vxm1 * vxm1 + vym1 * vym1 + vzm1 * vzm1)) * vxm1;
    flux2 = (gamma * pm2 * rgamma1 + 0.5 * rhom2 * (vxm2 * vxm2 + vym2 * vym2 + vzm2 * vzm2)) * vxm2;
    grav = (*rho * *vx + rhonew * vxnew) * ghalf * 0.5;
    double etotnew = etot + rdtath * (flux1 - flux2) * rdx + rdtath * grav;
    /* pmean: uninitialised in the STENCIL build (HIGHPEAKS undefined,
     * integrate.F90:60-75); defined as in ppm.F90:583. */
    double pmean = (pm1 + pm2) * 0.5;
    double eintnew = eint + rdtath * pmean * (vxm1 - vxm2) * rdx;
    flux1 = (pm1 * vxm1) * rgamma1;
    flux2 = (pm2 * vxm2) * rgamma1;
    eintnew = eintnew + rdtath * (flux1 - flux2) * rdx;
    if (eintnew < 0.0) eintnew = eint;
    double ee2 = etotnew;
    double vvv = vxnew * vxnew + vynew * vynew + vznew * vznew;
    double eeaux = etotnew - 0.5 * rhonew * vvv;
    double ee1 = eeaux / ee2;
    if (ee1 >= s->eta2) eintnew = eeaux;
    double ee0 = eeaux / etotnew;
    double pnew;
    if (ee0 >= s->eta1) pnew = (gamma - 1.0) * eeaux;
    else pnew = (gamma - 1.0) * eintnew;
    if (eintnew <= 0.0) { eintnew = eint; pnew = *pres; }
    if (rhonew <= 0.0) rhonew = *rho;
    *pres = pnew; *rho = rhonew; *vx = vxnew; *vy = vynew; *vz = vznew;
}

/* ------------------------------------------------------------------ */
/* hydro/ppmsolver.F90:1-467 (STENCIL)                                 */
/* ------------------------------------------------------------------ */
int hpo_ppmsolver(double *p3d, double *rho3d, double *vx3d, double *vy3d, double *vz3d,
                  const double *gforce, int nx, int ny, int nz, int nbound, int ndirection,
                  const hpo_scalars *s, int nthreads)
{
    size_t ncell = (size_t)nx * ny * nz;
    /* the 10 face arrays (:54-64) */
    double *pl = calloc(ncell, sizeof(double)), *pr = calloc(ncell, sizeof(double));
    double *rl = calloc(ncell, sizeof(double)), *rr = calloc(ncell, sizeof(double));
    double *ul = calloc(ncell, sizeof(double)), *ur = calloc(ncell, sizeof(double));
    double *vl = calloc(ncell, sizeof(double)), *vr = calloc(ncell, sizeof(double));
    double *wl = calloc(ncell, sizeof(double)), *wr = calloc(ncell, sizeof(double));
    int fails = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    /* Linear Fortran index of rho3d(a,b,c) for the density-peak gather,
     * which the reference performs with the x-index slot for every sweep
     * (:126-127, :251-252, :379-380).  Out of the allocation -> not read. */
#define GIX(a, b, c) ((long)((a) - 1) + (long)nx * ((long)((b) - 1) + (long)ny * (long)((c) - 1)))

    /* ndirection selects the gather: (d1,d2,d3) = loop nest; idx(face,t1,t2) */
    /* R1: reconstruction (:96-117, :215-239, :343-367) */
    int n_sweep = (ndirection == 1) ? nx : (ndirection == 2) ? ny : nz;
    int n_t1 = (ndirection == 1) ? ny : nx;   /* transverse 1 (j in ppmsolver) */
    int n_t2 = (ndirection == 3) ? ny : nz;   /* transverse 2 */
    (void)n_t1; (void)n_t2;
#define CELL(ia, t1, t2) ((ndirection == 1) ? IX((ia), (t1), (t2)) : (ndirection == 2) ? IX((t1), (ia), (t2)) : IX((t1), (t2), (ia)))

    int t1max = (ndirection == 1) ? ny : nx;
    int t2max = (ndirection == 3) ? ny : nz;

#pragma omp parallel for collapse(2) schedule(static)
    for (int t2 = nbound + 1; t2 <= t2max - nbound; ++t2) {
        for (int t1 = nbound + 1; t1 <= t1max - nbound; ++t1) {
            for (int i = nbound + 1; i <= n_sweep - nbound + 1; ++i) {
                double pres[7], rho[7], vx[7], vy[7], vz[7], g[7], c[7];
                for (int ippm = 1; ippm <= 6; ++ippm) {
                    int iaux = i + ippm - 4;
                    size_t q = CELL(iaux, t1, t2);
                    pres[ippm] = p3d[q];
                    rho[ippm] = rho3d[q];
                    if (ndirection == 1) { vx[ippm] = vx3d[q]; vy[ippm] = vy3d[q]; vz[ippm] = vz3d[q]; }
                    else if (ndirection == 2) { vx[ippm] = vy3d[q]; vy[ippm] = vx3d[q]; vz[ippm] = vz3d[q]; }
                    else { vx[ippm] = vz3d[q]; vy[ippm] = vy3d[q]; vz[ippm] = vx3d[q]; }
                    g[ippm] = gforce ? -gforce[3 * q + (size_t)(ndirection - 1)] : -0.0;
                    c[ippm] = sqrt(s->gamma * pres[ippm] / rho[ippm]);
                }
                size_t f = CELL(i, t1, t2);
                order2interp(pres, rho, vx, vy, vz, g, c, &pl[f], &pr[f], &rl[f], &rr[f], &ul[f], &ur[f],
                             &vl[f], &vr[f], &wl[f], &wr[f], s);
            }
        }
    }

    /* R2: Riemann (:119-141, :241-266, :369-394) */
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : fails)
    for (int t2 = nbound + 1; t2 <= t2max - nbound; ++t2) {
        for (int t1 = nbound + 1; t1 <= t1max - nbound; ++t1) {
            for (int i = nbound + 1; i <= n_sweep - nbound + 1; ++i) {
                double rho[7], vx[7];
                for (int ippm = 1; ippm <= 6; ++ippm) {
                    int iaux = i + ippm - 4;
                    long q = (ndirection == 1) ? GIX(iaux, t1, t2) : GIX(iaux, t1, t2);
                    /* x sweep: rho3d(iaux,j,k);  y sweep: rho3d(iaux,j,k) with
                     * j the x index;  z sweep: rho3d(iaux,j,k) with j=y, k=x */
                    if (ndirection == 3) q = GIX(iaux, t2, t1);
                    if (q >= 0 && (size_t)q < ncell) {
                        rho[ippm] = rho3d[q];
                        vx[ippm] = (ndirection == 1) ? vx3d[q] : (ndirection == 2) ? vy3d[q] : vz3d[q];
                    } else {
                        /* outside the allocation (non-cubic boxes only):
                         * NaN makes the peak test false */
                        rho[ippm] = NAN;
                        vx[ippm] = NAN;
                    }
                }
                size_t f = CELL(i, t1, t2);
                double pm, rhom, vxm, vym, vzm;
                fails += riemannsolver(rho, vx, pl[f], pr[f], rl[f], rr[f], ul[f], ur[f], vl[f], vr[f], wl[f],
                                       wr[f], &pm, &rhom, &vxm, &vym, &vzm, s);
                pl[f] = pm; rl[f] = rhom; ul[f] = vxm; vl[f] = vym; wl[f] = vzm;
            }
        }
    }

    /* R3: conservative update (:144-160, :269-288, :397-416) */
#pragma omp parallel for collapse(2) schedule(static)
    for (int t2 = nbound + 1; t2 <= t2max - nbound; ++t2) {
        for (int t1 = nbound + 1; t1 <= t1max - nbound; ++t1) {
            for (int i = nbound + 1; i <= n_sweep - nbound; ++i) {
                size_t q = CELL(i, t1, t2), q1 = CELL(i + 1, t1, t2);
                double etots = total(p3d[q], rho3d[q], vx3d[q], vy3d[q], vz3d[q], s);
                double eints = internal(p3d[q], s);
                double ghalf = gforce ? -gforce[3 * q + (size_t)(ndirection - 1)] : -0.0;
                double *un, *ut1, *ut2;
                if (ndirection == 1) { un = &vx3d[q]; ut1 = &vy3d[q]; ut2 = &vz3d[q]; }
                else if (ndirection == 2) { un = &vy3d[q]; ut1 = &vx3d[q]; ut2 = &vz3d[q]; }
                else { un = &vz3d[q]; ut1 = &vy3d[q]; ut2 = &vx3d[q]; }
                integrate(pl[q], pl[q1], rl[q], rl[q1], ul[q], ul[q1], vl[q], vl[q1], wl[q], wl[q1], &p3d[q],
                          &rho3d[q], un, ut1, ut2, etots, eints, ghalf, s);
            }
        }
    }
#undef CELL
#undef GIX
    free(pl); free(pr); free(rl); free(rr); free(ul); free(ur); free(vl); free(vr); free(wl); free(wr);
    return fails;
}

/* ------------------------------------------------------------------ */
/* hydro/flatten5.F90:1-40: flattening test of one variable over the   */
/* four neighbour pairs of a 5-cell window.  When a pair's product is  */
/* zero, gradleft is not assigned (:17-19): the reference's local is   */
/* then stale or undefined; here it keeps its previous value (0 at the */
/* start of the pencil), which adds nothing new to gradmax or the flag.*/
/* ------------------------------------------------------------------ */
static void flatten5(const double *abar, int *flatyn, double *gradleft, const hpo_scalars *s)
{
    double gradmax = 0.0;
    for (int i = 1; i <= 4; ++i) {
        const int ic = i + 1;
        if (abar[ic] * abar[ic - 1] != 0.0)
            *gradleft = fabs((abar[ic] - abar[ic - 1]) / fmin2(abar[ic], abar[ic - 1]));
        gradmax = fmax2(gradmax, *gradleft);
    }
    if (gradmax >= s->mingradflat) *flatyn = 1;
}

typedef struct {
    double jl[3], jr[3], d[3], a6[3];
} pslot;

static void pslot_shift(pslot *q)
{
    q->jl[1] = q->jl[2]; q->jr[1] = q->jr[2]; q->d[1] = q->d[2]; q->a6[1] = q->a6[2];
}

/* ------------------------------------------------------------------ */
/* hydro/ppm.F90:1-662: one pencil of the non-STENCIL build.  Arrays   */
/* are 1-based [1..ngrid], the whole gathered line with its ghosts;    */
/* nmin = nbound, nmax = ngrid-nbound+1 (ppmsolver.F90:77-79).  pres.. */
/* vz are updated in place over nmin..nmax as the reference does (the  */
/* cells nmin and nmax are ghosts: they keep p and rho and get zero    */
/* velocities, which the ghost fill after the sweep overwrites).       */
/* Differences from the STENCIL path, all as in the reference:         */
/*  - the characteristic speeds of cell k use the sound speed of cell  */
/*    k+1 (cbar = c(i), c(i+1) with vxbar(2), vxbar(3) = cells i-1, i, */
/*    :106-107; order2interp.F90:56-57 has c(i-1), c(i));              */
/*  - the gravity parabola and ghalf are zero (:93,102);               */
/*  - the density-peak fix sees cells i-2..i+1 along the sweep         */
/*    (rhobar(1..4) of the 5-cell window);                             */
/*  - pmean takes the cho-dependent values at density peaks (:585-594);*/
/*  - the dual-energy switch divides by the largest new total energy   */
/*    of the cell and its two neighbours, 0 beyond the line's updated  */
/*    cells (:611-621).                                                */
/* cho may be NULL (zeros).  A face that matches no wave pattern (NaN  */
/* input) gets NaN, as in riemannsolver() here.  Returns the number of */
/* Newton failures.                                                    */
/* ------------------------------------------------------------------ */
static int ppm_pencil(int ngrid, int nmin, int nmax, const double *cho, double *pres, double *rho,
                      double *vx, double *vy, double *vz, const double *c, const double *eint,
                      const double *etot, double *work, const hpo_scalars *s)
{
    const double gamma = s->gamma, rgamma1 = s->rgamma1, rdtath = s->rdtath, rdx = s->rdx, rat = s->rat;
    const double mmmax = 0.0;
    const size_t L = (size_t)ngrid + 2;
    double *pnew = work, *rhonew = work + L, *vxnew = work + 2 * L, *vynew = work + 3 * L;
    double *vznew = work + 4 * L, *etotnew = work + 5 * L, *eintnew = work + 6 * L;
    memset(work, 0, 7 * L * sizeof(double));                               /* :64-71 */
    pslot P, R, VX, VY, VZ;
    memset(&P, 0, sizeof P); memset(&R, 0, sizeof R); memset(&VX, 0, sizeof VX);
    memset(&VY, 0, sizeof VY); memset(&VZ, 0, sizeof VZ);
    double pm[3] = {0, 0, 0}, rhom[3] = {0, 0, 0}, vxm[3] = {0, 0, 0}, vym[3] = {0, 0, 0}, vzm[3] = {0, 0, 0};
    double gradleft = 0.0;
    int fails = 0;
    const int nmid = nmin + 1;
    for (int i = nmin; i <= nmax; ++i) {
        int flatyn = 0;
        double flat = 0.0;
        const int icell = i;
        double pbar[6], rhobar[6], vxbar[6], vybar[6], vzbar[6], cbar[3];
        for (int j = 1; j <= 5; ++j) {                                     /* :95-103 */
            const int ia = icell + j - 3;
            pbar[j] = pres[ia];
            rhobar[j] = rho[ia];
            vxbar[j] = vx[ia];
            vybar[j] = vy[ia];
            vzbar[j] = vz[ia];
        }
        cbar[1] = c[icell];
        cbar[2] = c[icell + 1];
        flatten5(pbar, &flatyn, &gradleft, s);                             /* :119-128 */
        if (flatyn == 1) flat = s->flatvalue;
        flatten5(rhobar, &flatyn, &gradleft, s);
        if (flatyn == 1) flat = s->flatvalue;
        flatten5(vxbar, &flatyn, &gradleft, s);
        if (flatyn == 1) flat = s->flatvalue;
        flatten5(vybar, &flatyn, &gradleft, s);
        if (flatyn == 1) flat = s->flatvalue;
        flatten5(vzbar, &flatyn, &gradleft, s);
        if (flatyn == 1) flat = s->flatvalue;
        pslot_shift(&P); pslot_shift(&R); pslot_shift(&VX); pslot_shift(&VY); pslot_shift(&VZ);  /* :138-165 */
        const double addp = fabs(pbar[4] - pbar[2]) / fmin2(pbar[2], pbar[4]);             /* :169-171 */
        const double addrho = 0.5 * gamma * fabs(rhobar[4] - rhobar[2]) / fmin2(rhobar[2], rhobar[4]);
        double ptl, ptr, rhotl, rhotr, vxtl, vxtr, vytl, vytr, vztl, vztr;
        double pcl[4], pcr[4], rhocl[4], rhocr[4], vxcl[4], vxcr[4], vycl[4], vycr[4], vzcl[4], vzcr[4];
        correction(addp, addrho, pbar, P.jl, P.jr, P.d, P.a6, cbar, vxbar[2], vxbar[3], &ptl, &ptr, pcl, pcr,
                   flat, 0, s);
        correction(addp, addrho, rhobar, R.jl, R.jr, R.d, R.a6, cbar, vxbar[2], vxbar[3], &rhotl, &rhotr, rhocl,
                   rhocr, flat, 1, s);
        correction(addp, addrho, vxbar, VX.jl, VX.jr, VX.d, VX.a6, cbar, vxbar[2], vxbar[3], &vxtl, &vxtr, vxcl,
                   vxcr, flat, 0, s);
        correction(addp, addrho, vybar, VY.jl, VY.jr, VY.d, VY.a6, cbar, vxbar[2], vxbar[3], &vytl, &vytr, vycl,
                   vycr, flat, 0, s);
        correction(addp, addrho, vzbar, VZ.jl, VZ.jr, VZ.d, VZ.a6, cbar, vxbar[2], vxbar[3], &vztl, &vztr, vzcl,
                   vzcr, flat, 0, s);
        /* the g parabola of a zero gbar traces to exactly 0 (gcl = gcr = 0) */
        if (ptl < 0.0) ptl = HPO_TINY;                                     /* :191-207 */
        if (ptr < 0.0) ptr = HPO_TINY;
        if (rhotl < 0.0) rhotl = HPO_TINY;
        if (rhotr < 0.0) rhotr = HPO_TINY;
        const double ctl = sqrt(gamma * ptl * rhotl);                      /* :209-210 */
        const double ctr = sqrt(gamma * ptr * rhotr);
        double lambdam = (vxbar[2] - cbar[1]) * rat, lambda0 = vxbar[2] * rat, lambdap = (vxbar[2] + cbar[1]) * rat;
        double betaml, betapl, beta0l, betamr, betapr, beta0r, vyleft, vzleft, vyright, vzright;
        betaml = (lambdam <= 0.0) ? 0.0 : beta(ctl, vxtl, vxcl[1], ptl, pcl[1], 0.0, -1.0, s);   /* :214-238 */
        betapl = (lambdap <= 0.0) ? 0.0 : beta(ctl, vxtl, vxcl[3], ptl, pcl[3], 0.0, 1.0, s);
        vyleft = vytl;
        vzleft = vztl;
        if (lambda0 <= 0.0) {
            beta0l = 0.0;
        } else {
            beta0l = beta0(ctl, rhotl, rhocl[2], ptl, pcl[2], s);
            vyleft = vycl[2];
            vzleft = vzcl[2];
        }
        lambdam = (vxbar[3] - cbar[2]) * rat;                              /* :240-265 */
        lambda0 = vxbar[3] * rat;
        lambdap = (vxbar[3] + cbar[2]) * rat;
        betapr = (lambdap >= 0.0) ? 0.0 : beta(ctr, vxtr, vxcr[3], ptr, pcr[3], 0.0, 1.0, s);
        betamr = (lambdam >= 0.0) ? 0.0 : beta(ctr, vxtr, vxcr[1], ptr, pcr[1], 0.0, -1.0, s);
        vyright = vytr;
        vzright = vztr;
        if (lambda0 >= 0.0) {
            beta0r = 0.0;
        } else {
            beta0r = beta0(ctr, rhotr, rhocr[2], ptr, pcr[2], s);
            vyright = vycr[2];
            vzright = vzcr[2];
        }
        if (i == nmin) continue;                                           /* :267 */
        double pleft = ptl + ctl * ctl * (betapl + betaml);                /* :269-278 */
        if (pleft <= 0.0) pleft = ptl;
        double pright = ptr + ctr * ctr * (betapr + betamr);
        if (pright <= 0.0) pright = ptr;
        const double vxleft = vxtl + ctl * (betapl - betaml);
        const double vxright = vxtr + ctr * (betapr - betamr);
        double rholeft = 1.0 / (1.0 / rhotl - betaml - beta0l - betapl);
        if (rholeft <= 0.0) rholeft = rhotl;
        double rhoright = 1.0 / (1.0 / rhotr - betamr - beta0r - betapr);
        if (rhoright <= 0.0) rhoright = rhotr;
        pm[1] = pm[2];                                                     /* :310-314 */
        rhom[1] = rhom[2];
        vxm[1] = vxm[2];
        vym[1] = vym[2];
        vzm[1] = vzm[2];
        /* :279-531: the classification and the four wave patterns, the
         * transverse upwinding and the density-peak fix are riemannsolver's
         * (the same statements), with rhobar/vxbar of this 5-cell window */
        fails += riemannsolver(rhobar, vxbar, pleft, pright, rholeft, rhoright, vxleft, vxright, vyleft, vyright,
                               vzleft, vzright, &pm[2], &rhom[2], &vxm[2], &vym[2], &vzm[2], s);
        if (i == nmid) continue;                                           /* :534-535 */
        const int index = icell - 1;                                       /* :544-606 */
        double flux1 = rhom[1] * vxm[1], flux2 = rhom[2] * vxm[2];
        rhonew[index] = rho[index] + rdtath * (flux1 - flux2) * rdx;
        /* grav = (rhoold1d + rhonew) * ghalf * 0.5 with ghalf = 0 (:93): no term */
        flux1 = rhom[1] * vxm[1] * vxm[1] + pm[1];
        flux2 = rhom[2] * vxm[2] * vxm[2] + pm[2];
        vxnew[index] = (vx[index] * rho[index] + rdtath * (flux1 - flux2) * rdx) / rhonew[index];
        flux1 = vym[1] * vxm[1] * rhom[1];
        flux2 = vym[2] * vxm[2] * rhom[2];
        vynew[index] = (rho[index] * vy[index] + rdtath * (flux1 - flux2) * rdx) / rhonew[index];
        flux1 = vzm[1] * vxm[1] * rhom[1];
        flux2 = vzm[2] * vxm[2] * rhom[2];
        vznew[index] = (rho[index] * vz[index] + rdtath * (flux1 - flux2) * rdx) / rhonew[index];
        flux1 = (gamma * pm[1] * rgamma1 + 0.5 * rhom[1] * (vxm[1] * vxm[1] + vym[1] * vym[1] + vzm[1] * vzm[1])) * vxm[1];
        flux2 = (gamma * pm[2] * rgamma1 + 0.5 * rhom[2] * (vxm[2] * vxm[2] + vym[2] * vym[2] + vzm[2] * vzm[2])) * vxm[2];
        etotnew[index] = etot[index] + rdtath * (flux1 - flux2) * rdx;
        double pmean = (pm[1] + pm[2]) * 0.5;
        if (rhobar[2] > s->dmax * rhobar[1] && rhobar[2] > s->dmax * rhobar[3]) {
            const double ch = cho ? cho[index] : 0.0;
            if (ch == 1.0) {
                const double maxp = (vxm[1] - vxm[2]) * rhobar[2] * fmax2(mmmax, vxm[1] - vxm[2]);
                pmean = fmax2(pmean, maxp);
            } else if (ch == 2.0) {
                pmean = (gamma - 1.0) * eint[index];
            }
        }
        eintnew[index] = eint[index] + rdtath * pmean * (vxm[1] - vxm[2]) * rdx;
        flux1 = (pm[1] * vxm[1]) * rgamma1;
        flux2 = (pm[2] * vxm[2]) * rgamma1;
        eintnew[index] = eintnew[index] + rdtath * (flux1 - flux2) * rdx;
        if (eintnew[index] < 0.0) eintnew[index] = eint[index];
    }
    for (int i = nmin; i <= nmax; ++i) {                                   /* :611-638 */
        double eeleft = etotnew[i - 1];
        if (i == nmin) eeleft = 0.0;
        const double ee = etotnew[i];
        double eeright = etotnew[i + 1];
        if (i == nmax) eeright = 0.0;
        const double ee2 = fmax2(fmax2(eeleft, ee), eeright);
        const double vvv = vxnew[i] * vxnew[i] + vynew[i] * vynew[i] + vznew[i] * vznew[i];
        const double eeaux = etotnew[i] - 0.5 * rhonew[i] * vvv;
        const double ee1 = eeaux / ee2;
        if (ee1 >= s->eta2) eintnew[i] = eeaux;
        const double ee0 = eeaux / etotnew[i];
        if (ee0 >= s->eta1) pnew[i] = (gamma - 1.0) * eeaux;
        else pnew[i] = (gamma - 1.0) * eintnew[i];
    }
    for (int i = nmin; i <= nmax; ++i) {                                   /* :646-658 */
        if (eintnew[i] <= 0.0) {
            eintnew[i] = eint[i];
            pnew[i] = pres[i];
        }
        if (rhonew[i] <= 0.0) rhonew[i] = rho[i];
        pres[i] = pnew[i];
        rho[i] = rhonew[i];
        vx[i] = vxnew[i];
        vy[i] = vynew[i];
        vz[i] = vznew[i];
    }
    return fails;
}

/* ppmsolver.F90:162-190, 290-318, 418-446 (#else of STENCIL) and
 * hydropad/savetn.F90: every interior pencil is gathered whole (ghosts
 * included), solved by ppm_pencil, scattered into the new arrays, which
 * then replace the state. */
int hpo_ppmsolver_pencil(double *p3d, double *rho3d, double *vx3d, double *vy3d, double *vz3d,
                         const double *cho3d, int nx, int ny, int nz, int nbound, int ndirection,
                         const hpo_scalars *s, int nthreads)
{
    const size_t ncell = (size_t)nx * ny * nz;
    double *old[5] = {p3d, rho3d, vx3d, vy3d, vz3d};
    double *nw[5];
    for (int q = 0; q < 5; ++q) {
        /* the new arrays keep their contents outside the solved pencils
         * (ghost pencils), which the ghost fill after the sweep replaces */
        nw[q] = malloc(ncell * sizeof(double));
        memcpy(nw[q], old[q], ncell * sizeof(double));
    }
    const int ngrid = (ndirection == 1) ? nx : (ndirection == 2) ? ny : nz;
    const int nmin = nbound, nmax = ngrid - nbound + 1;
    const int t1max = (ndirection == 1) ? ny : nx;
    const int t2max = (ndirection == 3) ? ny : nz;
    int fails = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#define CELL(ia, t1, t2) ((ndirection == 1) ? IX((ia), (t1), (t2)) : (ndirection == 2) ? IX((t1), (ia), (t2)) : IX((t1), (t2), (ia)))
#pragma omp parallel reduction(+ : fails)
    {
        const size_t L = (size_t)ngrid + 2;
        double *buf = malloc(17 * L * sizeof(double));
        double *pres = buf, *rho = buf + L, *vx = buf + 2 * L, *vy = buf + 3 * L, *vz = buf + 4 * L;
        double *c = buf + 5 * L, *eint = buf + 6 * L, *etot = buf + 7 * L, *cho = buf + 8 * L;
        double *work = buf + 9 * L;
        memset(buf, 0, 9 * L * sizeof(double));
#pragma omp for collapse(2) schedule(static)
        for (int t2 = nbound + 1; t2 <= t2max - nbound; ++t2) {
            for (int t1 = nbound + 1; t1 <= t1max - nbound; ++t1) {
                for (int i = 1; i <= ngrid; ++i) {
                    const size_t q = CELL(i, t1, t2);
                    pres[i] = p3d[q];
                    rho[i] = rho3d[q];
                    if (ndirection == 1) { vx[i] = vx3d[q]; vy[i] = vy3d[q]; vz[i] = vz3d[q]; }
                    else if (ndirection == 2) { vx[i] = vy3d[q]; vy[i] = vx3d[q]; vz[i] = vz3d[q]; }
                    else { vx[i] = vz3d[q]; vy[i] = vy3d[q]; vz[i] = vx3d[q]; }
                    eint[i] = internal(pres[i], s);
                    etot[i] = total(pres[i], rho[i], vx[i], vy[i], vz[i], s);
                    cho[i] = cho3d ? cho3d[q] : 0.0;
                    c[i] = sqrt(s->gamma * p3d[q] / rho3d[q]);
                }
                fails += ppm_pencil(ngrid, nmin, nmax, cho, pres, rho, vx, vy, vz, c, eint, etot, work, s);
                for (int i = 1; i <= ngrid; ++i) {
                    const size_t q = CELL(i, t1, t2);
                    nw[0][q] = pres[i];
                    nw[1][q] = rho[i];
                    if (ndirection == 1) { nw[2][q] = vx[i]; nw[3][q] = vy[i]; nw[4][q] = vz[i]; }
                    else if (ndirection == 2) { nw[3][q] = vx[i]; nw[2][q] = vy[i]; nw[4][q] = vz[i]; }
                    else { nw[4][q] = vx[i]; nw[3][q] = vy[i]; nw[2][q] = vz[i]; }
                }
            }
        }
        free(buf);
    }
#undef CELL
    for (int q = 0; q < 5; ++q) {                                          /* savetn.F90:11-21 */
        memcpy(old[q], nw[q], ncell * sizeof(double));
        free(nw[q]);
    }
    return fails;
}

/* ------------------------------------------------------------------ */
/* Ghost fill: exchange_mesh with one rank, periodic in every axis     */
/* (exchange_mesh.F90:23-41 + exchange_var.F90:19-53, neighbours=self) */
/* ------------------------------------------------------------------ */
static void fill_one(double *a, int nx, int ny, int nz, int nb)
{
    /* z faces, then y, then x (each fills full transverse extent, so the
     * corners end up periodic as well) */
    for (int k = 1; k <= nb; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                a[IX(i, j, k)] = a[IX(i, j, nz - 2 * nb + k)];
                a[IX(i, j, nz - nb + k)] = a[IX(i, j, k + nb)];
            }
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= nb; ++j)
            for (int i = 1; i <= nx; ++i) {
                a[IX(i, j, k)] = a[IX(i, ny - 2 * nb + j, k)];
                a[IX(i, ny - nb + j, k)] = a[IX(i, j + nb, k)];
            }
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nb; ++i) {
                a[IX(i, j, k)] = a[IX(nx - 2 * nb + i, j, k)];
                a[IX(nx - nb + i, j, k)] = a[IX(i + nb, j, k)];
            }
}

void hpo_exchange_mesh(double *p3d, double *rho3d, double *vx3d, double *vy3d, double *vz3d, int nx,
                       int ny, int nz, int nbound)
{
    fill_one(rho3d, nx, ny, nz, nbound);
    fill_one(p3d, nx, ny, nz, nbound);
    fill_one(vx3d, nx, ny, nz, nbound);
    fill_one(vy3d, nx, ny, nz, nbound);
    fill_one(vz3d, nx, ny, nz, nbound);
}

/* ppm_lxlylz.F90:9-221: 1 xyz, 2 zyx, 3 yzx, 4 xzy, 5 zxy, 6 yxz */
int hpo_ppm_lxlylz(double *p3d, double *rho3d, double *vx3d, double *vy3d, double *vz3d,
                   const double *gforce, int nx, int ny, int nz, int nbound, int nrot,
                   const hpo_scalars *s, int nthreads)
{
    static const int order[6][3] = {{1, 2, 3}, {3, 2, 1}, {2, 3, 1}, {1, 3, 2}, {3, 1, 2}, {2, 1, 3}};
    int fails = 0;
    for (int k = 0; k < 3; ++k) {
        if (s->pencil)  /* the non-STENCIL build (cho3d of the hydro-only runs: zeros) */
            fails += hpo_ppmsolver_pencil(p3d, rho3d, vx3d, vy3d, vz3d, NULL, nx, ny, nz, nbound,
                                          order[nrot - 1][k], s, nthreads);
        else
            fails += hpo_ppmsolver(p3d, rho3d, vx3d, vy3d, vz3d, gforce, nx, ny, nz, nbound, order[nrot - 1][k],
                                   s, nthreads);
        hpo_exchange_mesh(p3d, rho3d, vx3d, vy3d, vz3d, nx, ny, nz, nbound);
    }
    return fails;
}

/* speed.F90:17-31 */
double hpo_speed(const double *p3d, const double *rho3d, const double *vx3d, const double *vy3d,
                 const double *vz3d, int nx, int ny, int nz, int nbound, const hpo_scalars *s)
{
    double vmax = 0.0;
    for (int k = nbound + 1; k <= nz - nbound; ++k)
        for (int j = nbound + 1; j <= ny - nbound; ++j)
            for (int i = nbound + 1; i <= nx - nbound; ++i) {
                size_t q = IX(i, j, k);
                double vsound = sqrt(s->gamma * p3d[q] / rho3d[q]);
                double a = fabs(vx3d[q]) + vsound, b = fabs(vy3d[q]) + vsound, c = fabs(vz3d[q]) + vsound;
                vmax = fmax2(vmax, a);
                vmax = fmax2(vmax, b);
                vmax = fmax2(vmax, c);
            }
    return vmax;
}

/* timedet, functions.F90:2-35 */
void hpo_timedet(hpo_scalars *s)
{
    s->at = 1.0;
    s->ath = 1.0;
    s->dat = 0.0;
    s->told = s->t;
    s->dtold = s->dt;
    double rdtc = s->velmax / (s->cour * s->dx);
    if (s->velmax == 0.0) s->dt = HPO_C0P1;
    else s->dt = 1.0 / rdtc;
    s->t = s->t + s->dt;
    if (s->t > s->tstop) {
        s->t = s->tstop;
        s->dt = s->t - s->told;
    }
    double dth = 0.5 * s->dt;
    s->thalf = s->told + dth;
    s->rdtath = s->dt / s->ath;
}

/* timedet_cosmo, functions.F90:38-151, omega_m == 1, COSMO defined.  The
 * particle-velocity term (:76-91) is zero without N-body.  The debug cap
 * dt0 = 1e-9 (:49,97) is applied only when s->dt_cap > 0. */
void hpo_timedet_cosmo(hpo_scalars *s)
{
    double rdt, rdtc, dta;
    s->told = s->t;
    s->dtold = s->dt;
    if (s->nstep > 1) rdt = 5.0 / (6.0 * s->dt);
    else rdt = 0.0;
    s->at = pow(s->t, HPO_TWO3);
    s->dat = HPO_TWO3 * pow(s->t, HPO_MTHIRD);
    dta = pow((1.0 + s->ca) * s->at, 1.5) - s->t;
    s->rat = 1.0 / s->at;
    rdtc = s->velmax / (s->cour * s->dx * s->at);
    s->dt = 1.0 / fmax2(rdt, rdtc);
    s->dt = fmin2(s->dt, dta);
    if (s->dt >= 10.0) s->dt = HPO_C0P1;
    if (s->dt_cap > 0.0) s->dt = fmin2(s->dt, s->dt_cap);
    s->t = s->t + s->dt;
    if (s->t > s->tstop) {
        s->t = s->tstop;
        s->dt = s->t - s->told;
    }
    double dth = 0.5 * s->dt;
    s->thalf = s->told + dth;
    s->atnew = pow(s->t, HPO_TWO3);
    s->ath = pow(s->thalf, HPO_TWO3);
    s->dath = HPO_TWO3 * pow(s->thalf, HPO_MTHIRD);
    s->datnew = HPO_TWO3 * pow(s->t, HPO_MTHIRD);
    s->rdtath = s->dt / s->ath;
}

/* initialize_parameters.F90:133-205 */
void hpo_init_time(hpo_scalars *s, double dtinit, double a_start)
{
    if (s->cosmo) {
        s->at = a_start;
        double tin = pow(s->at, 1.5);
        s->told = tin;
        s->dt = HPO_C0P010 * tin;
        s->dtold = s->dt;
        s->t = tin + s->dt;
        s->thalf = s->told + s->dt / 2.0;
        s->at = pow(s->told, HPO_TWO3);
        s->atnew = pow(s->t, HPO_TWO3);
        s->dat = HPO_TWO3 * pow(s->told, HPO_MTHIRD);
        s->ath = pow(s->told + s->dt / 2.0, HPO_TWO3);
        s->dath = HPO_TWO3 * pow(s->thalf, HPO_MTHIRD);
        s->datnew = HPO_TWO3 * pow(s->t, HPO_MTHIRD);
        s->rat = 1.0 / s->at;
        s->rdtath = s->dt / s->ath;
    } else {
        double tin = 0.0;
        s->told = tin;
        s->dt = dtinit;
        s->dtold = s->dt;
        s->t = tin + s->dt;
        s->at = 1.0;
        s->atnew = s->at;
        s->dat = 0.0;
        s->ath = 1.0;
        s->dath = 0.0;
        s->datnew = 0.0;
        s->rat = 1.0 / s->at;
        s->rdtath = s->dt / s->ath;
        s->thalf = s->told + 0.5 * s->dt;
    }
}

/* expand.F90:18-41 over every cell including ghosts */
void hpo_expand(double *p3d, double *vx3d, double *vy3d, double *vz3d, const double *pold,
                const double *vxold, const double *vyold, const double *vzold, int nx, int ny, int nz,
                const hpo_scalars *s)
{
    double afact = s->dt * (s->dath / s->ath);
    double afact1 = 1.0 / (1.0 + afact);
    double afact2 = 1.0 / (2.0 + afact);
    size_t n = (size_t)nx * ny * nz;
    for (size_t q = 0; q < n; ++q) {
        double vxo = s->expand_zero_old ? 0.0 : vxold[q];
        double vyo = s->expand_zero_old ? 0.0 : vyold[q];
        double vzo = s->expand_zero_old ? 0.0 : vzold[q];
        double po = s->expand_zero_old ? 0.0 : pold[q];
        vx3d[q] = (2.0 * vx3d[q] - afact * vxo) * afact2;
        vy3d[q] = (2.0 * vy3d[q] - afact * vyo) * afact2;
        vz3d[q] = (2.0 * vz3d[q] - afact * vzo) * afact2;
        double ppp = p3d[q];
        p3d[q] = (p3d[q] - afact * po) * afact1;
        if (p3d[q] <= 0.0) {
            if (ppp > 0.0) p3d[q] = ppp;
            else p3d[q] = po;
        }
    }
}

/* evolve_sys.F90:30-130 (HYDRO, STENCIL, no NBODY / COOLING / TRACERS),
 * looped like main.F90:100-121. */
int hpo_evolve(double *p3d, double *rho3d, double *vx3d, double *vy3d, double *vz3d,
               const double *gforce, int nx, int ny, int nz, int nbound, hpo_scalars *s, int nsteps,
               int nthreads)
{
    int fails = 0;
    size_t n = (size_t)nx * ny * nz;
    double *snap = NULL;
    if (s->cosmo && !s->expand_zero_old) snap = malloc(4 * n * sizeof(double));
    for (int it = 0; it < nsteps && s->told < s->tstop; ++it) {
        s->nstep += 1;
        int nrot = s->nstep % 6 + 1;
        if (s->nstep == 1) nrot = 1;
        if (snap) {
            memcpy(snap, p3d, n * sizeof(double));
            memcpy(snap + n, vx3d, n * sizeof(double));
            memcpy(snap + 2 * n, vy3d, n * sizeof(double));
            memcpy(snap + 3 * n, vz3d, n * sizeof(double));
        }
        fails += hpo_ppm_lxlylz(p3d, rho3d, vx3d, vy3d, vz3d, gforce, nx, ny, nz, nbound, nrot, s, nthreads);
        if (s->cosmo) {
            hpo_expand(p3d, vx3d, vy3d, vz3d, snap, snap ? snap + n : NULL, snap ? snap + 2 * n : NULL,
                       snap ? snap + 3 * n : NULL, nx, ny, nz, s);
        }
        s->velmax = hpo_speed(p3d, rho3d, vx3d, vy3d, vz3d, nx, ny, nz, nbound, s);
        if (s->cosmo) hpo_timedet_cosmo(s);
        else hpo_timedet(s);
    }
    free(snap);
    return fails;
}
