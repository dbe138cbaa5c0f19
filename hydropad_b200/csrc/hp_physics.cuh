// hp_physics.cuh -- pointwise physics of the PPM step, as device functions.
//
// Each function restates one reference routine (file:line given); operand
// order follows the Fortran left-to-right evaluation so that the FP64 build
// (compiled without FMA contraction) reproduces the reference arithmetic.
// The reconstruction/tracing functions are templated on the real type R so
// the mixed-precision sweep can run them in FP32; the Riemann solver and the
// update are always FP64 (their inputs are widened first).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace hp {

// REAL(4) literals of the reference, promoted to REAL(8).
constexpr double kSixth = 0.1666666716337204;      // 0.16666667  ppm_functs.F90:33-34, dda.F90:198-199
constexpr double kThird = 0.3333333432674408;      // 0.33333333  ppm_functs.F90:103,122
constexpr double kTiny = 1.0000000036274937e-15;   // 1e-15       order2interp.F90:176-189
constexpr double kTerr = 0.0010000000474974513;    // 1e-3        riemann.F90:337
constexpr double kC010 = 0.009999999776482582;     // 0.010       dda.F90:200
constexpr double kC050 = 0.05000000074505806;      // 0.050       dda.F90:203
constexpr int kNewtonMax = 100;                     // riemann.F90:339

// Fortran MIN/MAX of two reals (first operand kept on ties and NaN in b).
template <class R> __device__ __forceinline__ R fmin2(R a, R b) { return b < a ? b : a; }
template <class R> __device__ __forceinline__ R fmax2(R a, R b) { return b > a ? b : a; }

// Scalars of module `scalar` the sweep reads (scalar.F90:98-99).
struct Consts {
    double gamma, rgamma, gamma1, rgamma1, m, rm, gf;
    double mingradflat, flatvalue, dmax, eta1, eta2, dx, rdx;
};
struct StepScalars {
    double dt, rdtath, at, dat, rat, ath, dath;
};

// ajside, ppm_functs.F90:167-181: limited slope of the middle cell.
// Evaluated without a branch (the discarded quotient may be NaN), which keeps
// the warp converged; the selected value is the reference's.
template <class R>
__device__ __forceinline__ R ajside(R am1, R a, R ap1) {
    const R da = R(0.5) * (ap1 - am1);
    const R mn = fmin2(fmin2(fabs(da), R(2) * fabs(a - am1)), R(2) * fabs(ap1 - a));
    const R v = mn * da / fabs(da);
    return ((ap1 - a) * (a - am1) > R(0)) ? v : R(0);
}

// One flattening pair (order2interp.F90:66-71): true when the pair's
// relative jump reaches mingradflat.  A pair whose product is zero does not
// assign gradleft in the reference; it contributes nothing new here.
template <class R>
__device__ __forceinline__ bool flat_pair(R left, R right, R mingradflat) {
    const R g = fabs((right - left) / fmin2(right, left));
    return (right * left != R(0)) && (g >= mingradflat);
}

// Second difference used by dda (dda.F90:198-199), centred on the middle cell.
template <class R>
__device__ __forceinline__ R dda_second(R am1, R a, R ap1, R dx) {
    return R(kSixth) * (ap1 - R(2) * a + am1) / (dx * dx);
}

// Parabola of one cell: edge values, jump and curvature (ppm_functs.F90:29-54).
template <class R>
struct Parabola {
    R jl, jr, d, a6;
};

// correction() without the tracing part: q0..q4 are cells c-2..c+2, dm,d0,dp
// the ajside slopes of c-1,c,c+1.  For rho with addrho >= addp the contact
// steepening of dda() blends in (dda.F90:196-214, ppm_functs.F90:35-40);
// Dm,Dp are the second differences centred on c-1 and c+1.
template <class R>
__device__ __forceinline__ Parabola<R> build_parabola(R q1, R q2, R q3, R dm, R d0, R dp, R flat,
                                                      bool steepen, R Dm, R Dp, R dx) {
    Parabola<R> P;
    R ajl = q1 + R(0.5) * (q2 - q1) + (dm - d0) * R(kSixth);
    R ajr = q2 + R(0.5) * (q3 - q2) + (d0 - dp) * R(kSixth);
    if (steepen) {
        R eta;
        R agrad = fabs(q3 - q1) - R(kC010) * fmin2(fabs(q3), fabs(q1));
        if (-(Dm * Dp) > R(0) && agrad > R(0)) {
            R e = -((Dp - Dm) * dx * dx / (q3 - q1));
            eta = fmax2(R(0), fmin2(R(20) * (e - R(kC050)), R(1)));
        } else {
            eta = R(0);
        }
        R ajld = q1 + R(0.5) * dm;
        R ajrd = q3 - R(0.5) * dp;
        ajl = (R(1) - eta) * ajl + eta * ajld;
        ajr = (R(1) - eta) * ajr + eta * ajrd;
    }
    R d = ajr - ajl;
    R a6 = R(6) * (q2 - R(0.5) * (ajl + ajr));
    if ((ajr - q2) * (q2 - ajl) <= R(0)) {
        ajl = q2;
        ajr = q2;
    } else if (d * a6 > d * d) {
        ajl = R(3) * q2 - R(2) * ajr;
    } else if (d * a6 < -(d * d)) {
        ajr = R(3) * q2 - R(2) * ajl;
    }
    ajl = flat * q2 + (R(1) - flat) * ajl;
    ajr = flat * q2 + (R(1) - flat) * ajr;
    P.jl = ajl;
    P.jr = ajr;
    P.d = ajr - ajl;
    P.a6 = R(6) * (q2 - R(0.5) * (ajl + ajr));
    return P;
}

// fl / fr, ppm_functs.F90:91-124, with x = y/dx precomputed by the caller
// (the same x serves every variable of the cell).
template <class R>
__device__ __forceinline__ R fl(const Parabola<R>& P, R x) {
    return P.jr - R(0.5) * x * (P.d - (R(1) - R(2) * x * R(kThird)) * P.a6);
}
template <class R>
__device__ __forceinline__ R fr(const Parabola<R>& P, R x) {
    return P.jl + R(0.5) * x * (P.d + (R(1) - R(2) * x * R(kThird)) * P.a6);
}

// beta, ppm_functs.F90:129-144 (expanding-coordinate characteristic term).
template <class R>
__device__ __forceinline__ R beta(R ct, R ut, R uc, R pt, R pc, R gc, R sign, R dt, R at, R dat, R rat) {
    R gvc = (-gc + dat * uc) * rat;
    return -(sign * ((ut - uc) + sign * (pt - pc) / ct + sign * dt * (R(2) * dat * pc / (ct * at)) + dt * gvc)) /
           (R(2) * ct);
}

// beta0, ppm_functs.F90:149-162.
template <class R>
__device__ __forceinline__ R beta0(R ct, R rhot, R rhoc, R pt, R pc, R dt, R at, R dat) {
    return (pt - pc) / (ct * ct) + R(1) / rhot - R(1) / rhoc + (R(2) * dat * pc) / (at * ct * ct) * dt;
}

// ------------------------------------------------------------------------
// Riemann solver (FP64 always).  hydro/riemannsolver.F90
// ------------------------------------------------------------------------
__device__ __forceinline__ double rarwave(double f1, double f2, double vt, double vh) {  // :290-298
    return f2 + vt * (f1 - f2) / (vt - vh);
}
__device__ __forceinline__ double rhoshock(double p2, double p1, double rho1, double gamma1) {  // :303-313
    return rho1 * (gamma1 * p2 / p1 + 1.0) / (gamma1 + p2 / p1);
}

// Powers used by the Riemann solver, by exponent: x^m, x^-gf, x^rgamma,
// x^rm (riemannsolver.F90:63,118-119,126,158,192-199; riemann.F90:360-385).
//
// PowExact calls CUDA pow with the run's exponents (the FP64 path).  The
// call is kept out of line so that the solver's many call sites share one
// copy of the power routine's code.
static __device__ __noinline__ double pow_shared(double x, double y) { return pow(x, y); }

struct PowExact {
    __device__ __forceinline__ static double pm(double x, const Consts& k) { return pow_shared(x, k.m); }
    __device__ __forceinline__ static double pgf(double x, const Consts& k) { return pow_shared(x, -k.gf); }
    __device__ __forceinline__ static double prg(double x, const Consts& k) { return pow_shared(x, k.rgamma); }
    __device__ __forceinline__ static double prm(double x, const Consts& k) { return pow_shared(x, k.rm); }
};

// PowRoot: for gamma with integer n = 1/m (= 2 gamma/(gamma-1); 5 for
// gamma = 5/3) every exponent is a multiple of 1/n, since gf = 1 - m and
// rgamma = (2/(gamma-1)) m.  x^(1/n) is seeded in FP32 (hardware log2/exp2)
// and refined by two Newton steps on y^n = x in FP64, which is accurate to
// an ulp or two; the other powers follow by products and one division.
// Falls back to pow() when the exponents are not of that form or x is
// outside the FP32 seed's range.
__device__ __forceinline__ double ipow(double y, int n) {
    double r = y;
    for (int i = 1; i < n; ++i) r *= y;
    return r;
}

static __device__ __noinline__ double root_n(double x, int n) {
    if (!(x > 1e-30 && x < 1e30)) return pow(x, 1.0 / (double)n);
    const float xf = (float)x;
    double y = (double)exp2f(__log2f(xf) * (1.0f / (float)n));
    const double a = (double)(n - 1) / (double)n, b = 1.0 / (double)n;
#pragma unroll 1
    for (int it = 0; it < 2; ++it) y = a * y + b * x / ipow(y, n - 1);
    return y;
}

struct PowRoot {
    // n = 1/m and j = rgamma/m when both are small integers, else 0
    __device__ __forceinline__ static int nroot(const Consts& k) {
        const double n = k.rm;
        return (n == floor(n) && n >= 2.0 && n <= 9.0) ? (int)n : 0;
    }
    __device__ __forceinline__ static int jrg(const Consts& k) {
        const double j = k.rgamma * k.rm;
        return fabs(j - rint(j)) < 1e-12 && j >= 1.0 && j <= 9.0 ? (int)rint(j) : 0;
    }
    __device__ __forceinline__ static double pm(double x, const Consts& k) {
        const int n = nroot(k);
        return n ? root_n(x, n) : pow_shared(x, k.m);
    }
    __device__ __forceinline__ static double pgf(double x, const Consts& k) {
        const int n = nroot(k);
        return n ? root_n(x, n) / x : pow_shared(x, -k.gf);
    }
    __device__ __forceinline__ static double prg(double x, const Consts& k) {
        const int n = nroot(k), j = jrg(k);
        return (n && j) ? ipow(root_n(x, n), j) : pow_shared(x, k.rgamma);
    }
    __device__ __forceinline__ static double prm(double x, const Consts& k) {
        const int n = nroot(k);
        return n ? ipow(x, n) : pow_shared(x, k.rm);
    }
};

// riemann, riemann.F90:318-400 (van Leer Newton for p*).  Returns false when
// more than 100 iterations would be needed (the reference stops the run).
template <class Pow>
__device__ __forceinline__ bool riemann_newton(double& pstar, double& vstar, double pleft, double pright,
                                               double rholeft, double rhoright, double vxleft, double vxright,
                                               const Consts& k) {
    double err = 1.e10;
    int nnewt = 0;
    const double kappa = sqrt(k.gamma * (pleft + pright) * (rholeft + rhoright) * 0.25);
    const double pcheck = 0.5 * (pleft + pright) + 0.5 * kappa * (vxleft + vxright);
    if (pcheck > 0.0) pstar = pcheck;
    const double cleft = sqrt(k.gamma * pleft * rholeft);
    const double cright = sqrt(k.gamma * pright * rhoright);
    while (err > kTerr) {
        nnewt = nnewt + 1;
        if (nnewt > kNewtonMax) return false;
        const double pstarold = pstar;
        double a, b, vprimel, vprimer;
        // pstup (:360,:368) is only consulted on the rarefaction side, so the
        // power is evaluated there alone.
        const double rl = pstar / pleft, rr = pstar / pright;
        if (pstar >= pleft) {
            a = cleft * sqrt(k.gf * pstar / pleft + k.m);
            vprimel = -((a * a + cleft * cleft) / (2.0 * a * a * a));
        } else {
            const double pw = Pow::pm(rl, k);
            if ((1.0 - pw) == 0.0) a = cleft * sqrt(k.gf * pstar / pleft + k.m);
            else a = k.m * cleft * (1.0 - pstar / pleft) / (1.0 - pw);
            vprimel = -((1.0 / cleft) * Pow::pgf(rl, k));
        }
        if (pstar >= pright) {
            b = cright * sqrt(k.gf * pstar / pright + k.m);
            vprimer = (b * b + cright * cright) / (2.0 * b * b * b);
        } else {
            const double pw = Pow::pm(rr, k);
            if ((1.0 - pw) == 0.0) b = cright * sqrt(k.gf * pstar / pright + k.m);
            else b = k.m * cright * (1.0 - pstar / pright) / (1.0 - pw);
            vprimer = (1.0 / cright) * Pow::pgf(rr, k);
        }
        const double vstarl = vxleft - (pstar - pleft) / a;
        const double vstarr = vxright + (pstar - pright) / b;
        pstar = pstar - (vstarl - vstarr) / (vprimel - vprimer);
        if (pstar <= 0.0) pstar = pstarold / 1000.0;
        vstar = (pleft - pright + a * vxleft + b * vxright) / (a + b);
        err = fabs(pstarold - pstar) / pstarold;
    }
    return true;
}

struct FaceState {
    double p, rho, u, v, w;
};

// Wave pattern riemannsolver will take for these states (riemannsolver.F90:
// 32-64, 73, 113, 188, 231): 1 two shocks, 2 shock + rarefaction, 3 two
// rarefactions, 4 vacuum, 5 none (NaN input).  Used only to group problems
// of one pattern into the same warp; the solver decides again itself.
template <class Pow>
__device__ __forceinline__ int riemann_pattern(double pleft, double pright, double rholeft, double rhoright,
                                               double vxleft, double vxright, const Consts& k) {
    const double gamma = k.gamma;
    const double cleft = sqrt(gamma * pleft / rholeft);
    const double cright = sqrt(gamma * pright / rhoright);
    double p1, p2, rho1, c1, c2;
    if (pleft <= pright) {
        p1 = pleft; p2 = pright; rho1 = rholeft; c1 = cleft; c2 = cright;
    } else {
        p1 = pright; p2 = pleft; rho1 = rhoright; c1 = cright; c2 = cleft;
    }
    const double dvv = vxleft - vxright;
    const double dv2s = (p2 - p1) / sqrt(0.5 * rho1 * ((gamma - 1.0) * p1 + (gamma + 1.0) * p2));
    if (dvv >= dv2s) return 1;
    const double dv1s = -((2.0 * c2 / (gamma - 1.0)) * (1.0 - Pow::pm(p1 / p2, k)));
    const double dv2r = -(2.0 * (c1 + c2) * k.rgamma1);
    if (dvv < dv2s && dvv >= dv1s) return 2;
    if (dvv < dv1s && dvv > dv2r) return 3;
    if (dvv <= dv2r) return 4;
    return 5;
}

// riemannsolver, riemannsolver.F90:1-285 without the density-peak fix,
// which the caller applies (it needs neighbouring cells).  Returns false on
// Newton failure.
template <class Pow>
__device__ __forceinline__ bool riemannsolver(const FaceState& L, const FaceState& Rt, FaceState& out,
                                              const Consts& k, const StepScalars& s) {
    const double gamma = k.gamma, rgamma1 = k.rgamma1;
    const double pleft = L.p, pright = Rt.p, rholeft = L.rho, rhoright = Rt.rho;
    const double vxleft = L.u, vxright = Rt.u;
    bool ok = true;
    const double cleft = sqrt(gamma * pleft / rholeft);
    const double cright = sqrt(gamma * pright / rhoright);
    const double dadt = 1.0 - 0.5 * s.dat * s.dt * s.rat;
    double p1, p2, rho1, c1, c2;
    if (pleft <= pright) {
        p1 = pleft; p2 = pright; rho1 = rholeft; c1 = cleft; c2 = cright;
    } else {
        p1 = pright; p2 = pleft; rho1 = rhoright; c1 = cright; c2 = cleft;
    }
    const double dvv = vxleft - vxright;
    const double dv2s = (p2 - p1) / sqrt(0.5 * rho1 * ((gamma - 1.0) * p1 + (gamma + 1.0) * p2));
    double pm = __longlong_as_double(0x7ff8000000000000ULL), vxm = pm, rhom = pm;
    if (dvv >= dv2s) {  // two shocks, :73-109
        pm = fmax2(pleft, pright);
        ok = riemann_newton<Pow>(pm, vxm, pleft, pright, rholeft, rhoright, vxleft, vxright, k);
        const double rhoshock1 = rhoshock(pm, pleft, rholeft, k.gamma1);
        const double rhoshock2 = rhoshock(pm, pright, rhoright, k.gamma1);
        double vshock1, vshock2;
        if (rhoshock1 == rholeft) vshock1 = 0.0;
        else vshock1 = (rhoshock1 * vxm - rholeft * vxleft) / (rhoshock1 - rholeft);
        if (rhoshock2 == rhoright) vshock2 = 0.0;
        else vshock2 = (rhoshock2 * vxm - rhoright * vxright) / (rhoshock2 - rhoright);
        if (vshock2 < 0.0) { pm = pright; vxm = vxright; rhom = rhoright; }
        else if (vxm <= 0.0 && vshock2 >= 0.0) rhom = rhoshock2;
        else if (vshock1 <= 0.0 && vxm > 0.0) rhom = rhoshock1;
        else { pm = pleft; vxm = vxleft; rhom = rholeft; }
    } else {
        const double dv1s = -((2.0 * c2 / (gamma - 1.0)) * (1.0 - Pow::pm(p1 / p2, k)));
        const double dv2r = -(2.0 * (c1 + c2) * rgamma1);
        if (dvv < dv2s && dvv >= dv1s) {  // shock + rarefaction, :113-184
            pm = Pow::prm((cleft + cright + (vxleft - vxright) * (gamma - 1.0) * 0.5) /
                              (cleft / Pow::pm(pleft, k) + cright / Pow::pm(pright, k)),
                          k);
            ok = riemann_newton<Pow>(pm, vxm, pleft, pright, rholeft, rhoright, vxleft, vxright, k);
            if (pleft >= pright) {
                const double rhoshock2 = rhoshock(pm, pright, rhoright, k.gamma1);
                const double rhocont1 = rholeft * Pow::prg(pm / pleft, k);
                double vshock2;
                if (rhoshock2 == rhoright) vshock2 = 0.0;
                else vshock2 = (rhoshock2 * vxm - rhoright * vxright) / (rhoshock2 - rhoright);
                const double vtail1 = vxm - sqrt(gamma * pm / rhocont1);
                const double vhead1 = vxleft - cleft;
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
                const double rhoshock1 = rhoshock(pm, pleft, rholeft, k.gamma1);
                const double rhocont2 = rhoright * Pow::prg(pm / pright, k);
                double vshock1;
                if (rhoshock1 == rholeft) vshock1 = 0.0;
                else vshock1 = (rhoshock1 * vxm - rholeft * vxleft) / (rhoshock1 - rholeft);
                const double vtail2 = vxm + sqrt(gamma * pm / rhocont2);
                const double vhead2 = vxright + cright;
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
        } else if (dvv < dv1s && dvv > dv2r) {  // two rarefactions, :188-227
            const double zeta = (cright / cleft) * Pow::pm(pleft / pright, k);
            const double vtleft = vxleft + 2.0 * cleft * rgamma1;
            const double vtright = vxright - 2.0 * cright * rgamma1;
            vxm = (vtleft * zeta + vtright) / (1.0 + zeta);
            pm = pleft * Pow::prm((gamma - 1.0) * (vtleft - vtright) / (2.0 * cleft * (1.0 + zeta)), k);
            const double rhocont1 = rholeft * Pow::prg(pm / pleft, k);
            const double rhocont2 = rhoright * Pow::prg(pm / pright, k);
            const double vtail2 = vxm + sqrt(gamma * pm / rhocont2);
            const double vhead2 = vxright + cright;
            const double vtail1 = vxm - sqrt(gamma * pm / rhocont1);
            const double vhead1 = vxleft - cleft;
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
        } else if (dvv <= dv2r) {  // vacuum, :231-264
            pm = 0.0; vxm = 0.0;
            const double rhocont1 = 0.0, rhocont2 = 0.0;
            const double vtail2 = vxright - 2.0 * cright * rgamma1;
            const double vhead2 = vxright + cright;
            const double vtail1 = vxleft - 2.0 * cleft * rgamma1;
            const double vhead1 = vxleft - cleft;
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
    }
    // transverse upwinding, :269-275
    double vym, vzm;
    if (vxm >= 0.0) { vym = dadt * L.v; vzm = dadt * L.w; }
    else { vym = dadt * Rt.v; vzm = dadt * Rt.w; }
    out.p = pm; out.rho = rhom; out.u = vxm; out.v = vym; out.w = vzm;
    return ok;
}

// Density-peak pressure fix, riemannsolver.F90:279-285.  r1..r4 / u2,u3 are
// rhobar(1..4) / vxbar(2..3) of the gather (cells f-3..f of the sweep).
__device__ __forceinline__ double peak_value(double r1, double r2, double r3, double r4, double u2, double u3,
                                             double dmax) {
    if (r2 > dmax * r1 && r3 > dmax * r4) {
        return (u2 - u3) * fmax2(r2, r3) * fmax2(0.0, u2 - u3);
    }
    return -__longlong_as_double(0x7ff0000000000000ULL);  // -inf: no fix
}

// total / internal, total.F90:15, internal.F90:14 (natural velocity order).
__device__ __forceinline__ double total_energy(double p, double rho, double vx, double vy, double vz, double rgamma1) {
    return p * rgamma1 + 0.5 * rho * (vx * vx + vy * vy + vz * vz);
}

// integrate, integrate.F90:1-113, without gravity source (g == 0).  f1 is
// the face at i-1/2, f2 at i+1/2; (u,v,w) are the cell's normal and
// transverse velocities of this sweep.  pmean, uninitialised in the
// reference's STENCIL build, is (pm1+pm2)*0.5 as in ppm.F90:583.
__device__ __forceinline__ void integrate(const FaceState& f1, const FaceState& f2, double& pres, double& rho,
                                          double& u, double& v, double& w, double etot, double eint,
                                          const Consts& k, const StepScalars& s) {
    const double gamma = k.gamma, rgamma1 = k.rgamma1, rdtath = s.rdtath, rdx = k.rdx;
    double flux1 = f1.rho * f1.u;
    double flux2 = f2.rho * f2.u;
    double rhonew = rho + rdtath * (flux1 - flux2) * rdx;
    flux1 = f1.rho * f1.u * f1.u + f1.p;
    flux2 = f2.rho * f2.u * f2.u + f2.p;
    const double vxnew = (u * rho + rdtath * (flux1 - flux2) * rdx) / rhonew;
    flux1 = f1.v * f1.u * f1.rho;
    flux2 = f2.v * f2.u * f2.rho;
    const double vynew = (rho * v + rdtath * (flux1 - flux2) * rdx) / rhonew;
    flux1 = f1.w * f1.u * f1.rho;
    flux2 = f2.w * f2.u * f2.rho;
    const double vznew = (rho * w + rdtath * (flux1 - flux2) * rdx) / rhonew;
    flux1 = (gamma * f1.p * rgamma1 + 0.5 * f1.rho * (f1.u * f1.u + f1.v * f1.v + f1.w * f1.w)) * f1.u;
    flux2 = (gamma * f2.p * rgamma1 + 0.5 * f2.rho * (f2.u * f2.u + f2.v * f2.v + f2.w * f2.w)) * f2.u;
    const double etotnew = etot + rdtath * (flux1 - flux2) * rdx;
    const double pmean = (f1.p + f2.p) * 0.5;
    double eintnew = eint + rdtath * pmean * (f1.u - f2.u) * rdx;
    flux1 = (f1.p * f1.u) * rgamma1;
    flux2 = (f2.p * f2.u) * rgamma1;
    eintnew = eintnew + rdtath * (flux1 - flux2) * rdx;
    if (eintnew < 0.0) eintnew = eint;
    // dual energy, :85-98 (STENCIL: ee2 = etotnew)
    const double vvv = vxnew * vxnew + vynew * vynew + vznew * vznew;
    const double eeaux = etotnew - 0.5 * rhonew * vvv;
    const double ee1 = eeaux / etotnew;
    if (ee1 >= k.eta2) eintnew = eeaux;
    const double ee0 = eeaux / etotnew;
    double pnew;
    if (ee0 >= k.eta1) pnew = (gamma - 1.0) * eeaux;
    else pnew = (gamma - 1.0) * eintnew;
    if (eintnew <= 0.0) pnew = pres;
    if (rhonew <= 0.0) rhonew = rho;
    pres = pnew;
    rho = rhonew;
    u = vxnew;
    v = vynew;
    w = vznew;
}

}  // namespace hp
