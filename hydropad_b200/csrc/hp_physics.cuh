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
constexpr double kSixth = 0.1666666716337204;      // 0.16666667  ppm_functs.F90:33-34, dda.F90:17-18
constexpr double kThird = 0.3333333432674408;      // 0.33333333  ppm_functs.F90:103,122
constexpr double kTiny = 1.0000000036274937e-15;   // 1e-15       order2interp.F90:176-189
constexpr double kTerr = 0.0010000000474974513;    // 1e-3        riemann.F90:48
constexpr double kC010 = 0.009999999776482582;     // 0.010       dda.F90:19
constexpr double kC050 = 0.05000000074505806;      // 0.050       dda.F90:22
constexpr int kNewtonMax = 100;                     // riemann.F90:50

// Fortran MIN/MAX of two reals (first operand kept on ties and NaN in b).
template <class R> __device__ __forceinline__ R fmin2(R a, R b) { return b < a ? b : a; }
template <class R> __device__ __forceinline__ R fmax2(R a, R b) { return b > a ? b : a; }

// Scalars of module `scalar` the sweep reads (scalar.F90:98-99).
struct Consts {
    double gamma, rgamma, gamma1, rgamma1, m, rm, gf;
    double mingradflat, flatvalue, dmax, eta1, eta2, dx, rdx;
    int nroot;  // 1/m when it is an integer in [2, 9] (5 for gamma = 5/3), else 0
    int jrg;    // rgamma/m when nroot != 0 and it is an integer in [1, 9], else 0
    int nbound; // ghost layers of the reference's arrays (&MESH nbound): only the
                // y/z density-peak gather, which indexes those arrays, depends on it
    int pad_;
    // FP32 copies for the mixed path's FP32 stages (set_float_consts): the
    // values a conversion in the kernel would give, without the conversion
    // (kernels under register pressure re-convert a constant at each use)
    float fgamma, fgamma1, frgamma1, fm, fgf, frm, frgamma, fdx, fflat, fming;
};
inline void set_float_consts(Consts& k) {
    k.fgamma = float(k.gamma);
    k.fgamma1 = float(k.gamma1);
    k.frgamma1 = float(k.rgamma1);
    k.fm = float(k.m);
    k.fgf = float(k.gf);
    k.frm = float(k.rm);
    k.frgamma = float(k.rgamma);
    k.fdx = float(k.dx);
    k.fflat = float(k.flatvalue);
    k.fming = float(k.mingradflat);
}
// The constants in type T: the FP64 fields, or their FP32 copies.
template <class T> struct KT {
    __device__ __forceinline__ static double gamma(const Consts& k) { return k.gamma; }
    __device__ __forceinline__ static double gamma1(const Consts& k) { return k.gamma1; }
    __device__ __forceinline__ static double rgamma1(const Consts& k) { return k.rgamma1; }
    __device__ __forceinline__ static double dx(const Consts& k) { return k.dx; }
    __device__ __forceinline__ static double flat(const Consts& k) { return k.flatvalue; }
    __device__ __forceinline__ static double ming(const Consts& k) { return k.mingradflat; }
};
template <> struct KT<float> {
    __device__ __forceinline__ static float gamma(const Consts& k) { return k.fgamma; }
    __device__ __forceinline__ static float gamma1(const Consts& k) { return k.fgamma1; }
    __device__ __forceinline__ static float rgamma1(const Consts& k) { return k.frgamma1; }
    __device__ __forceinline__ static float dx(const Consts& k) { return k.fdx; }
    __device__ __forceinline__ static float flat(const Consts& k) { return k.fflat; }
    __device__ __forceinline__ static float ming(const Consts& k) { return k.fming; }
};
struct StepScalars {
    double dt, rdtath, at, dat, rat, ath, dath;
};

// ajside, ppm_functs.F90:167-181: limited slope of the middle cell.
// Evaluated without a branch (the discarded quotient may be NaN), which keeps
// the warp converged; the selected value is the reference's.
//
// The FP32 instantiations (mixed path) below use multiply-adds, reciprocals
// and sign copies where the FP64 ones keep the reference's operations: the
// same values to FP32 rounding.
template <class R>
__device__ __forceinline__ R ajside(R am1, R a, R ap1) {
    const R da = R(0.5) * (ap1 - am1);
    const R mn = fmin2(fmin2(fabs(da), R(2) * fabs(a - am1)), R(2) * fabs(ap1 - a));
    R v;
    if constexpr (sizeof(R) == sizeof(float)) v = copysignf(mn, da);  // da != 0 whenever it is selected
    else v = mn * da / fabs(da);
    return ((ap1 - a) * (a - am1) > R(0)) ? v : R(0);
}

// One flattening pair (order2interp.F90:66-71): true when the pair's
// relative jump reaches mingradflat.  A pair whose product is zero does not
// assign gradleft in the reference; it contributes nothing new here.
template <class R>
__device__ __forceinline__ bool flat_pair(R left, R right, R mingradflat) {
    if constexpr (sizeof(R) == sizeof(float)) {
        return (right * left != 0.0f) && (fabsf(right - left) >= mingradflat * fabsf(fminf(right, left)));
    } else {
        const R g = fabs((right - left) / fmin2(right, left));
        return (right * left != R(0)) && (g >= mingradflat);
    }
}

// Second difference used by dda (dda.F90:17-18), centred on the middle cell.
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
// steepening of dda() blends in (dda.F90:15-33, ppm_functs.F90:35-40);
// Dm,Dp are the second differences centred on c-1 and c+1.
template <class R>
__device__ __forceinline__ Parabola<R> build_parabola(R q1, R q2, R q3, R dm, R d0, R dp, R flat,
                                                      bool steepen, R Dm, R Dp, R dx) {
    Parabola<R> P;
    R ajl, ajr;
    if constexpr (sizeof(R) == sizeof(float)) {
        ajl = fmaf(dm - d0, float(kSixth), fmaf(0.5f, q2 - q1, q1));
        ajr = fmaf(d0 - dp, float(kSixth), fmaf(0.5f, q3 - q2, q2));
    } else {
        ajl = q1 + R(0.5) * (q2 - q1) + (dm - d0) * R(kSixth);
        ajr = q2 + R(0.5) * (q3 - q2) + (d0 - dp) * R(kSixth);
    }
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
    if constexpr (sizeof(R) == sizeof(float)) {
        ajl = fmaf(flat, q2 - ajl, ajl);
        ajr = fmaf(flat, q2 - ajr, ajr);
        P.a6 = fmaf(-3.0f, ajl + ajr, 6.0f * q2);
    } else {
        ajl = flat * q2 + (R(1) - flat) * ajl;
        ajr = flat * q2 + (R(1) - flat) * ajr;
        P.a6 = R(6) * (q2 - R(0.5) * (ajl + ajr));
    }
    P.jl = ajl;
    P.jr = ajr;
    P.d = ajr - ajl;
    return P;
}

// fl / fr, ppm_functs.F90:91-124, with x = y/dx precomputed by the caller
// (the same x serves every variable of the cell).
template <class R>
__device__ __forceinline__ R fl(const Parabola<R>& P, R x) {
    if constexpr (sizeof(R) == sizeof(float)) {
        const float t = fmaf(-2.0f * float(kThird), x, 1.0f);
        return fmaf(-0.5f * x, fmaf(-t, P.a6, P.d), P.jr);
    } else {
        return P.jr - R(0.5) * x * (P.d - (R(1) - R(2) * x * R(kThird)) * P.a6);
    }
}
template <class R>
__device__ __forceinline__ R fr(const Parabola<R>& P, R x) {
    if constexpr (sizeof(R) == sizeof(float)) {
        const float t = fmaf(-2.0f * float(kThird), x, 1.0f);
        return fmaf(0.5f * x, fmaf(t, P.a6, P.d), P.jl);
    } else {
        return P.jl + R(0.5) * x * (P.d + (R(1) - R(2) * x * R(kThird)) * P.a6);
    }
}

// beta, ppm_functs.F90:129-144 (expanding-coordinate characteristic term).
template <class R>
__device__ __forceinline__ R beta(R ct, R ut, R uc, R pt, R pc, R gc, R sign, R dt, R at, R dat, R rat) {
    if constexpr (sizeof(R) == sizeof(float)) {
        // 1/ct is shared by every call of a face side; 1/at = rat
        const float rct = 1.0f / ct;
        const float gvc = (fmaf(dat, uc, -gc)) * rat;
        const float in = fmaf(dt, gvc, fmaf(sign * dt, 2.0f * dat * pc * rct * rat, fmaf(sign * (pt - pc), rct, ut - uc)));
        return -(sign * in) * (0.5f * rct);
    } else {
        R gvc = (-gc + dat * uc) * rat;
        return -(sign * ((ut - uc) + sign * (pt - pc) / ct + sign * dt * (R(2) * dat * pc / (ct * at)) + dt * gvc)) /
               (R(2) * ct);
    }
}

// beta0, ppm_functs.F90:149-162.
template <class R>
__device__ __forceinline__ R beta0(R ct, R rhot, R rhoc, R pt, R pc, R dt, R at, R dat) {
    if constexpr (sizeof(R) == sizeof(float)) {
        const float rct = 1.0f / ct, rct2 = rct * rct;
        return fmaf(pt - pc, rct2, 1.0f / rhot - 1.0f / rhoc) + (2.0f * dat * pc) * (rct2 / at) * dt;
    } else {
        return (pt - pc) / (ct * ct) + R(1) / rhot - R(1) / rhoc + (R(2) * dat * pc) / (at * ct * ct) * dt;
    }
}

struct FaceState {
    double p, rho, u, v, w;
};
// The face state of the mixed path's FP32 solvers.
struct FaceF {
    float p, rho, u, v, w;
};
// A face state in the reconstruction type R (the traced states of stage B).
template <class R> struct FaceOf { using type = FaceState; };
template <> struct FaceOf<float> { using type = FaceF; };

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

// integrate, integrate.F90:1-113.  f1 is the face at i-1/2, f2 at i+1/2;
// (u,v,w) are the cell's normal and transverse velocities of this sweep.
// GRAV adds the source terms of ghalf = -gforce of the cell (:41-44,54-57);
// without it they are exactly zero and left out.  pmean, uninitialised in
// the reference's STENCIL build, is (pm1+pm2)*0.5 as in ppm.F90:583.
// Div::div(a, b) is the division: IEEE for the FP64 path, a refined
// hardware reciprocal for the mixed path.
struct DivIEEE {
    __device__ __forceinline__ static double div(double a, double b) { return a / b; }
};
template <bool GRAV, class Div = DivIEEE>
__device__ __forceinline__ void integrate(const FaceState& f1, const FaceState& f2, double& pres, double& rho,
                                          double& u, double& v, double& w, double etot, double eint,
                                          const Consts& k, const StepScalars& s, double ghalf) {
    const double gamma = k.gamma, rgamma1 = k.rgamma1, rdtath = s.rdtath, rdx = k.rdx;
    double flux1 = f1.rho * f1.u;
    double flux2 = f2.rho * f2.u;
    double rhonew = rho + rdtath * (flux1 - flux2) * rdx;
    flux1 = f1.rho * f1.u * f1.u + f1.p;
    flux2 = f2.rho * f2.u * f2.u + f2.p;
    double vxnew;
    if constexpr (GRAV) {
        const double grav = (rho + rhonew) * ghalf * 0.5;
        vxnew = Div::div(u * rho + rdtath * (flux1 - flux2) * rdx + rdtath * grav, rhonew);
    } else {
        vxnew = Div::div(u * rho + rdtath * (flux1 - flux2) * rdx, rhonew);
    }
    flux1 = f1.v * f1.u * f1.rho;
    flux2 = f2.v * f2.u * f2.rho;
    const double vynew = Div::div(rho * v + rdtath * (flux1 - flux2) * rdx, rhonew);
    flux1 = f1.w * f1.u * f1.rho;
    flux2 = f2.w * f2.u * f2.rho;
    const double vznew = Div::div(rho * w + rdtath * (flux1 - flux2) * rdx, rhonew);
    flux1 = (gamma * f1.p * rgamma1 + 0.5 * f1.rho * (f1.u * f1.u + f1.v * f1.v + f1.w * f1.w)) * f1.u;
    flux2 = (gamma * f2.p * rgamma1 + 0.5 * f2.rho * (f2.u * f2.u + f2.v * f2.v + f2.w * f2.w)) * f2.u;
    double etotnew;
    if constexpr (GRAV) {
        const double grav = (rho * u + rhonew * vxnew) * ghalf * 0.5;
        etotnew = etot + rdtath * (flux1 - flux2) * rdx + rdtath * grav;
    } else {
        etotnew = etot + rdtath * (flux1 - flux2) * rdx;
    }
    const double pmean = (f1.p + f2.p) * 0.5;
    double eintnew = eint + rdtath * pmean * (f1.u - f2.u) * rdx;
    flux1 = (f1.p * f1.u) * rgamma1;
    flux2 = (f2.p * f2.u) * rgamma1;
    eintnew = eintnew + rdtath * (flux1 - flux2) * rdx;
    if (eintnew < 0.0) eintnew = eint;
    // dual energy, :85-98 (STENCIL: ee2 = etotnew)
    const double vvv = vxnew * vxnew + vynew * vynew + vznew * vznew;
    const double eeaux = etotnew - 0.5 * rhonew * vvv;
    const double ee1 = Div::div(eeaux, etotnew);
    if (ee1 >= k.eta2) eintnew = eeaux;
    const double ee0 = Div::div(eeaux, etotnew);
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

// New total energy of a cell from its two faces, ppm.F90:563-567 with the
// gravity term zero (ghalf = 0, :93): the update's and the neighbours' value.
__device__ __forceinline__ double etot_new(const FaceState& f1, const FaceState& f2, double etot, const Consts& k,
                                           const StepScalars& s) {
    const double gamma = k.gamma, rgamma1 = k.rgamma1;
    const double flux1 = (gamma * f1.p * rgamma1 + 0.5 * f1.rho * (f1.u * f1.u + f1.v * f1.v + f1.w * f1.w)) * f1.u;
    const double flux2 = (gamma * f2.p * rgamma1 + 0.5 * f2.rho * (f2.u * f2.u + f2.v * f2.v + f2.w * f2.w)) * f2.u;
    return etot + s.rdtath * (flux1 - flux2) * k.rdx;
}

// The update of the non-STENCIL build's full-pencil solver, ppm.F90:544-606
// (the gravity terms vanish: ghalf = 0, :93) and its dual-energy switch
// and fallbacks, :611-658: the switch divides by the largest new total
// energy of the cell (eeleft, its own, eeright: the neighbours' values, 0
// beyond the pencil's updated cells).  At a density peak (the cell's old
// rho above dmax x each old neighbour's), cho = 1 raises pmean to the
// peak pressure and cho = 2 takes it from the internal energy (:585-594).
template <class Div = DivIEEE>
__device__ __forceinline__ void integrate_pencil(const FaceState& f1, const FaceState& f2, double& pres, double& rho,
                                                 double& u, double& v, double& w, double etot, double eint,
                                                 const Consts& k, const StepScalars& s, double eeleft, double eeright,
                                                 bool peak, double cho) {
    const double gamma = k.gamma, rgamma1 = k.rgamma1, rdtath = s.rdtath, rdx = k.rdx;
    double flux1 = f1.rho * f1.u;
    double flux2 = f2.rho * f2.u;
    double rhonew = rho + rdtath * (flux1 - flux2) * rdx;
    flux1 = f1.rho * f1.u * f1.u + f1.p;
    flux2 = f2.rho * f2.u * f2.u + f2.p;
    const double vxnew = Div::div(u * rho + rdtath * (flux1 - flux2) * rdx, rhonew);
    flux1 = f1.v * f1.u * f1.rho;
    flux2 = f2.v * f2.u * f2.rho;
    const double vynew = Div::div(rho * v + rdtath * (flux1 - flux2) * rdx, rhonew);
    flux1 = f1.w * f1.u * f1.rho;
    flux2 = f2.w * f2.u * f2.rho;
    const double vznew = Div::div(rho * w + rdtath * (flux1 - flux2) * rdx, rhonew);
    const double etotnew = etot_new(f1, f2, etot, k, s);
    double pmean = (f1.p + f2.p) * 0.5;
    if (peak) {
        if (cho == 1.0) {
            const double maxp = (f1.u - f2.u) * rho * fmax2(0.0, f1.u - f2.u);
            pmean = fmax2(pmean, maxp);
        } else if (cho == 2.0) {
            pmean = (gamma - 1.0) * eint;
        }
    }
    double eintnew = eint + rdtath * pmean * (f1.u - f2.u) * rdx;
    flux1 = (f1.p * f1.u) * rgamma1;
    flux2 = (f2.p * f2.u) * rgamma1;
    eintnew = eintnew + rdtath * (flux1 - flux2) * rdx;
    if (eintnew < 0.0) eintnew = eint;
    const double ee2 = fmax2(fmax2(eeleft, etotnew), eeright);
    const double vvv = vxnew * vxnew + vynew * vynew + vznew * vznew;
    const double eeaux = etotnew - 0.5 * rhonew * vvv;
    const double ee1 = Div::div(eeaux, ee2);
    if (ee1 >= k.eta2) eintnew = eeaux;
    const double ee0 = Div::div(eeaux, etotnew);
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
