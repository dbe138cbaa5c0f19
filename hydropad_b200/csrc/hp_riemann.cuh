// hp_riemann.cuh -- exact Riemann solver of the PPM step, split by wave
// pattern (hydro/riemannsolver.F90, hydro/riemann.F90).
//
// riemannsolver.F90 first classifies the face into one of four wave
// patterns (:61-64,73,113,188,231) and then runs very different code for
// each.  The sweep kernel classifies all faces of a window step, groups the
// faces of one pattern into the same warps, and calls the pattern's solver
// below; riemannsolver() chains the same pieces for a single face.  Every
// branch keeps the reference's operand order, so the FP64 instantiation
// follows the Fortran arithmetic.
#pragma once
#include "hp_physics.cuh"

namespace hp {

template <class S = double>
__device__ __forceinline__ S rarwave(S f1, S f2, S vt, S vh) {  // riemann.F90:1-9
    return f2 + vt * (f1 - f2) / (vt - vh);
}
template <class S = double>
__device__ __forceinline__ S rhoshock(S p2, S p1, S rho1, S gamma1) {  // riemann.F90:14-24
    return rho1 * (gamma1 * p2 / p1 + S(1)) / (gamma1 + p2 / p1);
}

// ------------------------------------------------------------------------
// Powers by exponent: x^m, x^-gf, x^rgamma, x^rm
// (riemannsolver.F90:63,118-119,126,158,192-199; riemann.F90:71-96).
// ------------------------------------------------------------------------

// CUDA pow, out of line so that all call sites share one copy of its code.
static __device__ __noinline__ double pow_shared(double x, double y) { return pow(x, y); }

__device__ __forceinline__ double ipow(double y, int n) {
    double r = y;
    for (int i = 1; i < n; ++i) r *= y;
    return r;
}

// z = x^(-1/n) for integer n >= 2, without division: an FP32 estimate
// (hardware log2/exp2, ~2^-22) refined by two Newton steps on z^-n = x,
// z <- z + z (1 - x z^n)/n, each of which squares the relative error.  The
// result is good to a few ulp.  Inputs outside the FP32 range go to pow().
template <int N>
__device__ __forceinline__ double ipow_fixed(double y) {
    double r = y;
#pragma unroll
    for (int i = 1; i < N; ++i) r *= y;
    return r;
}
template <int N, int STEPS = 2>
__device__ __forceinline__ double inv_root_fixed(double x) {
    if (!(x > 1e-30 && x < 1e30)) return pow_shared(x, -1.0 / (double)N);
    double z = (double)exp2f(__log2f((float)x) * (-1.0f / (float)N));
    constexpr double rn = 1.0 / (double)N;
#pragma unroll
    for (int it = 0; it < STEPS; ++it) z = z + z * ((1.0 - x * ipow_fixed<N>(z)) * rn);
    return z;
}
static __device__ __noinline__ double inv_root_any(double x, int n) {
    if (!(x > 1e-30 && x < 1e30)) return pow_shared(x, -1.0 / (double)n);
    double z = (double)exp2f(__log2f((float)x) * (-1.0f / (float)n));
    const double rn = 1.0 / (double)n;
    for (int it = 0; it < 2; ++it) z = z + z * ((1.0 - x * ipow(z, n)) * rn);
    return z;
}
// x^(-(n-1)/n) = x^-gf, the common factor of every power below
template <int STEPS = 2>
__device__ __forceinline__ double pow_mgf(double x, int n) {
    if (n == 5) return ipow_fixed<4>(inv_root_fixed<5, STEPS>(x));
    return ipow(inv_root_any(x, n), n - 1);
}

// gamma enters the Riemann solver only through m = (gamma-1)/(2 gamma),
// gf = 1 - m, rgamma and rm = 1/m.  When n = 1/m is an integer (5 for
// gamma = 5/3; k.nroot) and rgamma = j m with integer j (3 for 5/3; k.jrg),
// every power follows from z = x^(-1/n):  x^-gf = z^(n-1),
// x^m = x z^(n-1), x^rgamma = (x^m)^j, x^rm = x^n.  These agree with pow()
// to a few ulp.  Other gammas use pow().
template <int STEPS>  // Newton steps of the fifth root
struct PowRootBase {
    __device__ __forceinline__ static double pm(double x, const Consts& k) {
        return k.nroot ? x * pow_mgf<STEPS>(x, k.nroot) : pow_shared(x, k.m);
    }
    __device__ __forceinline__ static double pgf(double x, const Consts& k) {
        return k.nroot ? pow_mgf<STEPS>(x, k.nroot) : pow_shared(x, -k.gf);
    }
    // x^m and x^-gf from one root
    __device__ __forceinline__ static void pm_pgf(double x, double& m_, double& gf_, const Consts& k) {
        if (k.nroot) {
            gf_ = pow_mgf<STEPS>(x, k.nroot);
            m_ = x * gf_;
        } else {
            m_ = pow_shared(x, k.m);
            gf_ = pow_shared(x, -k.gf);
        }
    }
    __device__ __forceinline__ static double prg(double x, const Consts& k) {
        if (k.nroot == 5 && k.jrg == 3) return ipow_fixed<3>(pm(x, k));
        return (k.nroot && k.jrg) ? ipow(pm(x, k), k.jrg) : pow_shared(x, k.rgamma);
    }
    __device__ __forceinline__ static double prm(double x, const Consts& k) {
        if (k.nroot == 5) return ipow_fixed<5>(x);
        return k.nroot ? ipow(x, k.nroot) : pow_shared(x, k.rm);
    }
};

// FP64 path: roots to a few ulp, IEEE division, the literal loop body.
// Divisions from the hardware reciprocal estimate refined by two Newton
// steps plus one residual correction (within an ulp or two of the IEEE
// quotient).
__device__ __forceinline__ double rcp_refined(double b) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
    double e = fma(-b, r, 1.0);
    r = fma(r, e, r);
    e = fma(-b, r, 1.0);
    return fma(r, e, r);
}
__device__ __forceinline__ double div_refined(double a, double b) {
    const double r = rcp_refined(b);
    const double q = a * r;
    return fma(r, fma(-b, q, a), q);
}

// FP64 path: the reference's start value; IEEE divisions outside the
// Newton loop, refined reciprocals (an ulp or two) for the two divisions
// inside it -- the iterates then agree with the literal loop to a few ulp.
struct PowRoot : PowRootBase<2> {
    static constexpr bool kShortNewton = false;  // the reference's Newton start value
    __device__ __forceinline__ static double div(double a, double b) { return a / b; }
    __device__ __forceinline__ static double div_loop(double a, double b) { return div_refined(a, b); }
};

// The powers of the mixed path take one Newton step from the FP32 root
// estimate (relative error ~1e-13, far inside the 1e-3 step tolerance of
// the Newton iteration that uses them), and the divisions inside the loop
// one step from the hardware reciprocal (div_loop, ~1e-13).
struct PowRootShort : PowRootBase<1> {
    static constexpr bool kShortNewton = true;
    __device__ __forceinline__ static double div(double a, double b) { return div_refined(a, b); }
    __device__ __forceinline__ static double div_loop(double a, double b) {
        double r;
        asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
        r = fma(r, fma(-b, r, 1.0), r);
        return a * r;
    }
};

// FP32 powers for the mixed path's closed-form two-rarefaction solution.
struct PowF32 {
    __device__ __forceinline__ static float pw(float x, float y) { return exp2f(y * __log2f(x)); }
};

// ------------------------------------------------------------------------
// Classification, riemannsolver.F90:32-64 + the tests at :73,113,188,231.
// Returns 1 two shocks, 2 shock + rarefaction, 3 two rarefactions,
// 4 vacuum, 5 none (NaN input).  cleft/cright are reused by the solvers.
// ------------------------------------------------------------------------
template <class T, class PowT>
__device__ __forceinline__ int riemann_classify(T pleft, T pright, T rholeft, T rhoright, T vxleft, T vxright,
                                                T& cleft, T& cright, const Consts& k) {
    const T gamma = T(KT<T>::gamma(k));
    cleft = sqrt(gamma * pleft / rholeft);
    cright = sqrt(gamma * pright / rhoright);
    T p1, p2, rho1, c1, c2;
    if (pleft <= pright) {
        p1 = pleft; p2 = pright; rho1 = rholeft; c1 = cleft; c2 = cright;
    } else {
        p1 = pright; p2 = pleft; rho1 = rhoright; c1 = cright; c2 = cleft;
    }
    const T dvv = vxleft - vxright;
    const T dv2s = (p2 - p1) / sqrt(T(0.5) * rho1 * ((gamma - T(1)) * p1 + (gamma + T(1)) * p2));
    if (dvv >= dv2s) return 1;
    const T dv1s = -((T(2) * c2 / (gamma - T(1))) * (T(1) - PowT::pm(p1 / p2, k)));
    const T dv2r = -(T(2) * (c1 + c2) * T(KT<T>::rgamma1(k)));
    if (dvv < dv2s && dvv >= dv1s) return 2;
    if (dvv < dv1s && dvv > dv2r) return 3;
    if (dvv <= dv2r) return 4;
    return 5;
}

// FP32 x^m for the mixed classification.
struct PowF32m {
    __device__ __forceinline__ static float pm(float x, const Consts& k) { return PowF32::pw(x, k.fm); }
};

// ------------------------------------------------------------------------
// riemann, riemann.F90:29-111 (van Leer Newton for p*).  Returns false when
// more than 100 iterations would be needed (the reference stops the run).
// ------------------------------------------------------------------------
// Start value of the mixed path's Newton iteration: the two-rarefaction
// estimate p = [(cL + cR + (uL-uR)(gamma-1)/2) / (cL pL^-m + cR pR^-m)]^(1/m)
// (the reference's own start value for the shock-rarefaction pattern,
// riemannsolver.F90:118-119), here in FP32; if it is not a positive finite
// number, the linearised (acoustic) estimate (pL+pR)/2 + kappa (uL-uR)/2;
// 0 if neither is positive.
//
// The reference's guess (riemann.F90:54-56) adds kappa (uL+uR)/2, which in
// the bulk flows of a cosmological box lands far from the root: on a 48^3
// EdS field its Newton faces take 4.9 iterations on average and 7.9 for the
// slowest face of 32 (a warp waits for its slowest lane), the linearised
// estimate 2.2 and 3.0, the two-rarefaction estimate 1.05 and 1.6 (two
// shocks) and 1.01 and 1.1 (shock + rarefaction).  Every start point
// converges to the same root to the 1e-3 step tolerance; p* differs from
// the reference's by a few 1e-7 relative at most.
// FP32 two-rarefaction start value (riemannsolver.F90:118-119), 0 when it
// is not a positive finite number.
__device__ __forceinline__ float newton_start_f32(float pl, float pr, float rl, float rr, float ul, float ur,
                                                  const Consts& k) {
    const float g = k.fgamma, m = k.fm;
    const float cl = sqrtf(g * pl / rl), cr = sqrtf(g * pr / rr);
    const float q = (cl + cr + (ul - ur) * (g - 1.0f) * 0.5f) / (cl / PowF32::pw(pl, m) + cr / PowF32::pw(pr, m));
    float ps;
    if (k.nroot == 5) {
        const float q2 = q * q;
        ps = q2 * q2 * q;
    } else {
        ps = PowF32::pw(q, k.frm);
    }
    return (ps > 0.0f && ps < 3.0e38f) ? ps : 0.0f;
}

__device__ __forceinline__ double mixed_newton_start(double pleft, double pright, double rholeft, double rhoright,
                                                     double vxleft, double vxright, const Consts& k) {
    const float ps = newton_start_f32(float(pleft), float(pright), float(rholeft), float(rhoright), float(vxleft),
                                      float(vxright), k);
    if (ps > 0.0f) return double(ps);
    const double kappa = sqrt(k.gamma * (pleft + pright) * (rholeft + rhoright) * 0.25);
    const double pcheck = 0.5 * (pleft + pright) + 0.5 * kappa * (vxleft - vxright);
    return pcheck > 0.0 ? pcheck : 0.0;
}

// riemann.F90:60-109 with the divisions of the loop body replaced by
// products with reciprocals formed once (or by rsqrt), and u* formed once
// after the loop from the last wave speeds: the same iterates up to a few
// ulp, with a shorter dependency chain per iteration.  Both paths run it in
// FP64 from pstar as given: the FP64 path from the reference's start value
// (riemann_newton below) with IEEE divisions, the mixed path from
// mixed_newton_start (chosen by the caller) with refined reciprocals.
template <class Pow>
__device__ __forceinline__ bool riemann_newton_short(double& pstar, double& vstar, double pleft, double pright,
                                                     double rholeft, double rhoright, double vxleft,
                                                     double vxright, const Consts& k) {
    // Lagrangian sound speeds C = sqrt(gamma p rho) and the reciprocals the
    // loop multiplies by
    double cleft, cright, rpl, rpr, rcl, rcr;
    if constexpr (Pow::kShortNewton) {
        const double c2l = k.gamma * pleft * rholeft, c2r = k.gamma * pright * rhoright;
        rcl = rsqrt(c2l);
        rcr = rsqrt(c2r);
        cleft = c2l * rcl;
        cright = c2r * rcr;
        rpl = Pow::div_loop(1.0, pleft);
        rpr = Pow::div_loop(1.0, pright);
    } else {
        cleft = sqrt(k.gamma * pleft * rholeft);
        cright = sqrt(k.gamma * pright * rhoright);
        rpl = Pow::div(1.0, pleft);
        rpr = Pow::div(1.0, pright);
        rcl = Pow::div(1.0, cleft);
        rcr = Pow::div(1.0, cright);
    }
    // only 1/a and 1/b enter the iteration; u* = (pL-pR + a uL + b uR)/(a+b)
    // is formed once at the end from them
    double ia = 0.0, ib = 0.0;
    bool ok = false;
    for (int nnewt = 1; nnewt <= kNewtonMax; ++nnewt) {
        const double pstarold = pstar;
        const double rl = pstar * rpl, rr = pstar * rpr;
        double vprimel, vprimer;
        if (pstar >= pleft) {
            const double q = k.gf * rl + k.m, rs = rsqrt(q);
            ia = rs * rcl;
            const double ca = cleft * ia;
            vprimel = -0.5 * ia * (1.0 + ca * ca);
        } else {
            double pw, pg;
            Pow::pm_pgf(rl, pw, pg, k);
            if ((1.0 - pw) == 0.0) ia = rsqrt(k.gf * rl + k.m) * rcl;
            else ia = Pow::div_loop(1.0 - pw, k.m * cleft * (1.0 - rl));
            vprimel = -(rcl * pg);  // (1/cl) rl^-gf
        }
        if (pstar >= pright) {
            const double q = k.gf * rr + k.m, rs = rsqrt(q);
            ib = rs * rcr;
            const double cb = cright * ib;
            vprimer = 0.5 * ib * (1.0 + cb * cb);
        } else {
            double pw, pg;
            Pow::pm_pgf(rr, pw, pg, k);
            if ((1.0 - pw) == 0.0) ib = rsqrt(k.gf * rr + k.m) * rcr;
            else ib = Pow::div_loop(1.0 - pw, k.m * cright * (1.0 - rr));
            vprimer = rcr * pg;
        }
        const double vstarl = vxleft - (pstar - pleft) * ia;
        const double vstarr = vxright + (pstar - pright) * ib;
        pstar = pstar - Pow::div_loop(vstarl - vstarr, vprimel - vprimer);
        if (pstar <= 0.0) pstar = pstarold * 0.001;
        if (!(fabs(pstarold - pstar) > kTerr * pstarold)) {
            ok = true;
            break;
        }
    }
    vstar = Pow::div_loop((pleft - pright) * ia * ib + vxleft * ib + vxright * ia, ia + ib);
    return ok;
}

// ------------------------------------------------------------------------
// Weak Newton faces of the mixed path (patterns 6, 7): the iteration of
// riemann.F90:60-109 in FP32.
//
// A two-shock or shock + rarefaction face is weak when its pressures differ
// by at most a factor 4 and its velocity jump uL - uR is at most cL + cR
// (the Eulerian sound speeds of the classification): on the EdS box the
// star pressure of such faces is then at most 10 times the lower side's
// (shock Mach number below about 3).  They are 80-99 % of the Newton faces.
// Strong shocks keep the FP64 iteration, and so does a weak face whose FP32
// iteration fails (a start value or an iterate that is not a positive
// finite number, or no convergence within kNewtonMaxF32 steps).
//
// The rarefaction wave speed a = m c (1 - x)/(1 - x^m) (x = p*/p of the
// side, riemann.F90:74-80) has a 0/0 form at x -> 1 that FP32 cannot
// evaluate as written; with n = 1/m an integer and z = x^(1/n),
// (1 - x)/(1 - z) = 1 + z + ... + z^(n-1) exactly, so a = m c sum_j z^j,
// and x^-gf = z/x.  The face states of the mixed path are FP32 values, so
// the inputs lose nothing in the conversion.
// ------------------------------------------------------------------------
constexpr int kNewtonMaxF32 = 20;

__device__ __forceinline__ bool newton_weak(float pl, float pr, float rl, float rr, float ul, float ur, float cl,
                                            float cr) {
    const float pmin = fminf(pl, pr), pmax = fmaxf(pl, pr);
    const float rmin = fminf(rl, rr), rmax = fmaxf(rl, rr);
    return pmax <= 4.0f * pmin && (ul - ur) <= (cl + cr) && pmin > 1e-18f && pmax < 1e18f && rmin > 1e-18f &&
           rmax < 1e18f;
}

// 1/a and the derivative of u* of one side at p* (x = p*/p of the side);
// sgn = -1 left, +1 right.
__device__ __forceinline__ void wave_f32(float x, float pstar, float p, float c, float rc, float sgn, int nroot,
                                         const Consts& k, float& ia, float& vprime) {
    if (pstar >= p) {  // shock: a = c sqrt(gf x + m)
        ia = rsqrtf(k.fgf * x + k.fm) * rc;
        const float ca = c * ia;
        vprime = sgn * 0.5f * ia * (1.0f + ca * ca);
    } else {  // rarefaction: a = m c (1 + z + ... + z^(n-1)), z = x^(1/n)
        const float z = PowF32::pw(x, k.fm);
        float s = 1.0f;
        for (int j = 1; j < nroot; ++j) s = fmaf(s, z, 1.0f);
        ia = rc / (k.fm * s);
        vprime = sgn * rc * (z / x);
    }
}

__device__ __forceinline__ bool riemann_newton_f32(float& pstar, float& vstar, float pl, float pr, float rl, float rr,
                                                   float ul, float ur, const Consts& k) {
    const int n = k.nroot;
    if (n < 2) return false;
    const float g = k.fgamma;
    const float c2l = g * pl * rl, c2r = g * pr * rr;
    const float rcl = rsqrtf(c2l), rcr = rsqrtf(c2r);
    const float cl = c2l * rcl, cr = c2r * rcr;  // Lagrangian sound speeds
    const float rpl = 1.0f / pl, rpr = 1.0f / pr;
    const float terr = float(kTerr);
    float ia = 0.0f, ib = 0.0f;
    bool ok = false;
    for (int it = 0; it < kNewtonMaxF32; ++it) {
        const float old = pstar;
        float vpl, vpr;
        wave_f32(pstar * rpl, pstar, pl, cl, rcl, -1.0f, n, k, ia, vpl);
        wave_f32(pstar * rpr, pstar, pr, cr, rcr, 1.0f, n, k, ib, vpr);
        const float vsl = ul - (pstar - pl) * ia;
        const float vsr = ur + (pstar - pr) * ib;
        pstar = pstar - (vsl - vsr) / (vpl - vpr);
        if (pstar <= 0.0f) pstar = old * 0.001f;
        if (!(fabsf(old - pstar) > terr * old)) {
            ok = true;
            break;
        }
    }
    vstar = ((pl - pr) * ia * ib + ul * ib + ur * ia) / (ia + ib);
    return ok && pstar > 0.0f && pstar < 3.0e38f && fabsf(vstar) < 3.0e38f;
}

template <class Pow>
__device__ __forceinline__ bool riemann_newton(double& pstar, double& vstar, double pleft, double pright,
                                               double rholeft, double rhoright, double vxleft, double vxright,
                                               const Consts& k) {
    if constexpr (!Pow::kShortNewton) {
        // the reference's start value (riemann.F90:54-56)
        const double kappa = sqrt(k.gamma * (pleft + pright) * (rholeft + rhoright) * 0.25);
        const double pcheck = 0.5 * (pleft + pright) + 0.5 * kappa * (vxleft + vxright);
        if (pcheck > 0.0) pstar = pcheck;
    }
    return riemann_newton_short<Pow>(pstar, vstar, pleft, pright, rholeft, rhoright, vxleft, vxright, k);
}

// Patterns 1 and 2 share the Newton iteration for p*, u* (riemann.F90,
// FP64 in both paths); each has its own start value and its own sampling
// of the solution at the face.  The caller runs one Newton loop for the
// faces of both patterns, so a warp that holds faces of both runs the loop
// once.  S is the type of the sampling (which wave lands on the face, and
// the density behind it): double in the FP64 path, float in the mixed path,
// as its closed two-rarefaction form.

// Start value of pattern 1, two shocks (riemannsolver.F90:77): the larger
// pressure; the mixed path replaces it by the two-rarefaction estimate.
// The FP64 path's riemann_newton then applies the reference's own start
// value when that is positive.
template <class Pow>
__device__ __forceinline__ double start_two_shocks(const FaceState& L, const FaceState& R, const Consts& k) {
    double pm = fmax2(L.p, R.p);
    if constexpr (Pow::kShortNewton) {
        const double st = mixed_newton_start(L.p, R.p, L.rho, R.rho, L.u, R.u, k);
        if (st > 0.0) pm = st;
    }
    return pm;
}

// Sampling of pattern 1 after the Newton solve, riemannsolver.F90:82-109.
// S: the arithmetic type; FS / O: the face-state and result types (FaceState
// and double, or the mixed path's FP32 FaceF and float).
template <class S, class FS = FaceState, class O = double>
__device__ __forceinline__ void sample_two_shocks(const FS& L, const FS& R, O& pm, O& vxm, O& rhom, const Consts& k) {
    const auto pleft = L.p, pright = R.p, rholeft = L.rho, rhoright = R.rho, vxleft = L.u, vxright = R.u;
    const S pmS = S(pm), vxmS = S(vxm), g1 = S(KT<S>::gamma1(k));
    const S rl = S(rholeft), rr = S(rhoright);
    const S rhoshock1 = rhoshock<S>(pmS, S(pleft), rl, g1);
    const S rhoshock2 = rhoshock<S>(pmS, S(pright), rr, g1);
    S vshock1, vshock2;
    if (rhoshock1 == rl) vshock1 = S(0);
    else vshock1 = (rhoshock1 * vxmS - rl * S(vxleft)) / (rhoshock1 - rl);
    if (rhoshock2 == rr) vshock2 = S(0);
    else vshock2 = (rhoshock2 * vxmS - rr * S(vxright)) / (rhoshock2 - rr);
    if (vshock2 < S(0)) { pm = pright; vxm = vxright; rhom = rhoright; }
    else if (vxm <= 0.0 && vshock2 >= S(0)) rhom = O(rhoshock2);
    else if (vshock1 <= S(0) && vxm > 0.0) rhom = O(rhoshock1);
    else { pm = pleft; vxm = vxleft; rhom = rholeft; }
}

// Start value of pattern 2, one shock and one rarefaction
// (riemannsolver.F90:117-119): the reference's two-rarefaction guess, which
// the mixed path forms in FP64 only when its own FP32 estimate fails.
template <class Pow>
__device__ __forceinline__ double start_shock_rarefaction(const FaceState& L, const FaceState& R, double cleft,
                                                          double cright, const Consts& k) {
    if constexpr (Pow::kShortNewton) {
        const double pm = mixed_newton_start(L.p, R.p, L.rho, R.rho, L.u, R.u, k);
        if (pm > 0.0) return pm;
    }
    return Pow::prm((cleft + cright + (L.u - R.u) * (k.gamma - 1.0) * 0.5) /
                        (cleft / Pow::pm(L.p, k) + cright / Pow::pm(R.p, k)),
                    k);
}

// Sampling of pattern 2 after the Newton solve, riemannsolver.F90:124-184,
// with the powers of PowS.
template <class S, class PowS, class FS = FaceState, class O = double>
__device__ __forceinline__ void sample_shock_rarefaction(const FS& L, const FS& R, O cleft, O cright, O& pm, O& vxm,
                                                         O& rhom, const Consts& k) {
    const auto pleft = L.p, pright = R.p, rholeft = L.rho, rhoright = R.rho, vxleft = L.u, vxright = R.u;
    const S gS = S(KT<S>::gamma(k)), pmS = S(pm), vxmS = S(vxm), g1 = S(KT<S>::gamma1(k));
    if (pleft >= pright) {
        const S rr = S(rhoright), rl = S(rholeft);
        const S rhoshock2 = rhoshock<S>(pmS, S(pright), rr, g1);
        const S rhocont1 = rl * PowS::prg(pmS / S(pleft), k);
        S vshock2;
        if (rhoshock2 == rr) vshock2 = S(0);
        else vshock2 = (rhoshock2 * vxmS - rr * S(vxright)) / (rhoshock2 - rr);
        const S vtail1 = vxmS - sqrt(gS * pmS / rhocont1);
        const S vhead1 = S(vxleft) - S(cleft);
        if (vshock2 < S(0)) { pm = pright; vxm = vxright; rhom = rhoright; }
        else if (vhead1 >= S(0)) { pm = pleft; vxm = vxleft; rhom = rholeft; }
        else if (vxm <= 0.0 && vshock2 >= S(0)) rhom = O(rhoshock2);
        else if (vxm > 0.0 && vtail1 <= S(0)) rhom = O(rhocont1);
        else if (vtail1 > S(0) && vhead1 <= S(0)) {
            pm = O(rarwave<S>(S(pleft), pmS, vtail1, vhead1));
            rhom = O(rarwave<S>(rl, rhocont1, vtail1, vhead1));
            vxm = O(rarwave<S>(S(vxleft), vxmS, vtail1, vhead1));
        }
    } else {
        const S rr = S(rhoright), rl = S(rholeft);
        const S rhoshock1 = rhoshock<S>(pmS, S(pleft), rl, g1);
        const S rhocont2 = rr * PowS::prg(pmS / S(pright), k);
        S vshock1;
        if (rhoshock1 == rl) vshock1 = S(0);
        else vshock1 = (rhoshock1 * vxmS - rl * S(vxleft)) / (rhoshock1 - rl);
        const S vtail2 = vxmS + sqrt(gS * pmS / rhocont2);
        const S vhead2 = S(vxright) + S(cright);
        if (vshock1 > S(0)) { pm = pleft; vxm = vxleft; rhom = rholeft; }
        else if (vhead2 <= S(0)) { pm = pright; vxm = vxright; rhom = rhoright; }
        else if (vxm >= 0.0 && vshock1 <= S(0)) rhom = O(rhoshock1);
        else if (vxm < 0.0 && vtail2 >= S(0)) rhom = O(rhocont2);
        else if (vtail2 < S(0) && vhead2 >= S(0)) {
            pm = O(rarwave<S>(S(pright), pmS, vtail2, vhead2));
            rhom = O(rarwave<S>(rr, rhocont2, vtail2, vhead2));
            vxm = O(rarwave<S>(S(vxright), vxmS, vtail2, vhead2));
        }
    }
}

// Pattern 3: two rarefactions, riemannsolver.F90:188-227 (closed form).
// T = double follows the Fortran arithmetic; T = float is the mixed path
// (no Newton iteration is involved).
template <class T, class PowT>
__device__ __forceinline__ void riemann_two_rarefactions(T pleft, T pright, T rholeft, T rhoright, T vxleft,
                                                         T vxright, T cleft, T cright, T& pm, T& vxm, T& rhom,
                                                         const Consts& k) {
    const T gamma = T(KT<T>::gamma(k)), rgamma1 = T(KT<T>::rgamma1(k));
    const T zeta = (cright / cleft) * PowT::pm(pleft / pright, k);
    const T vtleft = vxleft + T(2) * cleft * rgamma1;
    const T vtright = vxright - T(2) * cright * rgamma1;
    vxm = (vtleft * zeta + vtright) / (T(1) + zeta);
    pm = pleft * PowT::prm((gamma - T(1)) * (vtleft - vtright) / (T(2) * cleft * (T(1) + zeta)), k);
    const T rhocont1 = rholeft * PowT::prg(pm / pleft, k);
    const T rhocont2 = rhoright * PowT::prg(pm / pright, k);
    const T vtail2 = vxm + sqrt(gamma * pm / rhocont2);
    const T vhead2 = vxright + cright;
    const T vtail1 = vxm - sqrt(gamma * pm / rhocont1);
    const T vhead1 = vxleft - cleft;
    auto rw = [](T f1, T f2, T vt, T vh) { return f2 + vt * (f1 - f2) / (vt - vh); };
    if (vhead2 <= T(0)) { pm = pright; vxm = vxright; rhom = rhoright; }
    else if (vhead1 >= T(0)) { pm = pleft; vxm = vxleft; rhom = rholeft; }
    else if (vhead2 > T(0) && vtail2 <= T(0)) {
        pm = rw(pright, pm, vtail2, vhead2);
        rhom = rw(rhoright, rhocont2, vtail2, vhead2);
        vxm = rw(vxright, vxm, vtail2, vhead2);
    } else if (vxm <= T(0) && vtail2 > T(0)) rhom = rhocont2;
    else if (vxm > T(0) && vtail1 <= T(0)) rhom = rhocont1;
    else if (vtail1 > T(0) && vhead1 <= T(0)) {
        pm = rw(pleft, pm, vtail1, vhead1);
        rhom = rw(rholeft, rhocont1, vtail1, vhead1);
        vxm = rw(vxleft, vxm, vtail1, vhead1);
    }
}

// FP32 powers of the two-rarefaction form (mixed path).
struct PowRareF32 {
    __device__ __forceinline__ static float pm(float x, const Consts& k) { return PowF32::pw(x, k.fm); }
    __device__ __forceinline__ static float prm(float x, const Consts& k) {
        if (k.nroot == 5) return x * x * x * x * x;
        if (k.nroot) {
            float r = x;
            for (int i = 1; i < k.nroot; ++i) r *= x;
            return r;
        }
        return PowF32::pw(x, k.frm);
    }
    __device__ __forceinline__ static float prg(float x, const Consts& k) { return PowF32::pw(x, k.frgamma); }
};

// Pattern 4: vacuum, riemannsolver.F90:231-264.
__device__ __forceinline__ void riemann_vacuum(const FaceState& L, const FaceState& R, double cleft, double cright,
                                               double& pm, double& vxm, double& rhom, const Consts& k) {
    const double rgamma1 = k.rgamma1;
    const double pleft = L.p, pright = R.p, rholeft = L.rho, rhoright = R.rho, vxleft = L.u, vxright = R.u;
    pm = 0.0;
    vxm = 0.0;
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

// Transverse velocities upwinded by the sign of u* (riemannsolver.F90:269-275).
__device__ __forceinline__ void riemann_finish(const FaceState& L, const FaceState& R, double pm, double vxm,
                                               double rhom, FaceState& out, const StepScalars& s) {
    const double dadt = 1.0 - 0.5 * s.dat * s.dt * s.rat;  // :36
    double vym, vzm;
    if (vxm >= 0.0) { vym = dadt * L.v; vzm = dadt * L.w; }
    else { vym = dadt * R.v; vzm = dadt * R.w; }
    out.p = pm; out.rho = rhom; out.u = vxm; out.v = vym; out.w = vzm;
}

// Pattern of a classified face in the mixed path: the weak two-shock and
// shock + rarefaction faces (newton_weak) become patterns 6 and 7, solved
// with the FP32 iteration.  The FP64 path keeps patterns 1..5.
template <bool kWeakNewton>
__device__ __forceinline__ int solver_pattern(int pattern, float pl, float pr, float rl, float rr, float ul, float ur,
                                              float cl, float cr) {
    if constexpr (kWeakNewton) {
        if ((pattern == 1 || pattern == 2) && newton_weak(pl, pr, rl, rr, ul, ur, cl, cr)) return pattern + 5;
    }
    return pattern;
}

// Solve a face whose pattern is known.  RareT is the arithmetic type of the
// closed two-rarefaction form (double: FP64 path, float: mixed path).  The
// Eulerian sound speeds (riemannsolver.F90:32-33) are recomputed here, in
// the type each pattern works in.  WHICH restricts the code to the Newton
// patterns 1, 2, 6, 7 (kNewtonOnly) or the closed forms 3, 4, 5
// (kClosedOnly), for a caller that only ever sees those (the same
// arithmetic, less code).  Patterns 6 and 7 (mixed path only) are the weak
// faces of patterns 1 and 2: their p*, u* come from the FP32 iteration, or,
// if it fails, from the FP64 one as for patterns 1 and 2.  kFallback (mixed
// path, after riemann_mixed_f32 declined the face) holds the FP64 code
// alone: patterns 1, 2, 4, 5, and pattern 3 straight to its FP64 solution
// (the FP32 closed form is known to have failed); the FP32 branches, which
// the caller has already run, stay out of the kernel's instruction stream.
enum { kAllPatterns = 0, kNewtonOnly = 1, kClosedOnly = 2, kFallback = 3 };
template <class Pow, class RareT, class PowRare, int WHICH = kAllPatterns>
__device__ __forceinline__ bool riemann_by_pattern(int pattern, const FaceState& L, const FaceState& R,
                                                   FaceState& out, const Consts& k, const StepScalars& s) {
    double pm = __longlong_as_double(0x7ff8000000000000ULL), vxm = pm, rhom = pm;
    bool ok = true;
    if constexpr (Pow::kShortNewton && WHICH != kClosedOnly && WHICH != kFallback) {
        if (pattern == 6 || pattern == 7) {
            const float pl = float(L.p), pr = float(R.p), rl = float(L.rho), rr = float(R.rho);
            const float ul = float(L.u), ur = float(R.u);
            float ps = newton_start_f32(pl, pr, rl, rr, ul, ur, k), us = 0.0f;
            if (ps > 0.0f && riemann_newton_f32(ps, us, pl, pr, rl, rr, ul, ur, k)) {
                pm = double(ps);
                vxm = double(us);
                if (pattern == 6) {
                    sample_two_shocks<RareT>(L, R, pm, vxm, rhom, k);
                } else {
                    const float g = k.fgamma;
                    const double cleft = double(sqrtf(g * pl / rl)), cright = double(sqrtf(g * pr / rr));
                    sample_shock_rarefaction<RareT, PowRare>(L, R, cleft, cright, pm, vxm, rhom, k);
                }
                riemann_finish(L, R, pm, vxm, rhom, out, s);
                return true;
            }
            pattern -= 5;  // the FP32 iteration failed: FP64 below
        }
    }
    if (WHICH != kClosedOnly && (pattern == 1 || pattern == 2)) {
        double cleft = 0.0, cright = 0.0;
        if (pattern == 2) {
            if constexpr (Pow::kShortNewton) {
                // mixed path: its start value and its FP32 sampling take the
                // Eulerian sound speeds in FP32 (mixed_newton_start forms the
                // same values); the FP64 ones only when that start fails
                pm = mixed_newton_start(L.p, R.p, L.rho, R.rho, L.u, R.u, k);
                const float g = k.fgamma;
                cleft = double(sqrtf(g * float(L.p) / float(L.rho)));
                cright = double(sqrtf(g * float(R.p) / float(R.rho)));
                if (!(pm > 0.0)) {
                    cleft = sqrt(k.gamma * L.p / L.rho);
                    cright = sqrt(k.gamma * R.p / R.rho);
                    pm = start_shock_rarefaction<Pow>(L, R, cleft, cright, k);
                }
            } else {
                cleft = sqrt(k.gamma * L.p / L.rho);
                cright = sqrt(k.gamma * R.p / R.rho);
                pm = start_shock_rarefaction<Pow>(L, R, cleft, cright, k);
            }
        } else {
            pm = start_two_shocks<Pow>(L, R, k);
        }
        ok = riemann_newton<Pow>(pm, vxm, L.p, R.p, L.rho, R.rho, L.u, R.u, k);
        if (pattern == 1) sample_two_shocks<RareT>(L, R, pm, vxm, rhom, k);
        else sample_shock_rarefaction<RareT, PowRare>(L, R, cleft, cright, pm, vxm, rhom, k);
    } else if (WHICH == kFallback && pattern == 3) {
        // a face at the edge of the vacuum condition: classified and solved
        // again in FP64, as below
        double cl, cr;
        const int p64 = riemann_classify<double, Pow>(L.p, R.p, L.rho, R.rho, L.u, R.u, cl, cr, k);
        if (p64 == 4) riemann_vacuum(L, R, cl, cr, pm, vxm, rhom, k);
        else riemann_two_rarefactions<double, Pow>(L.p, R.p, L.rho, R.rho, L.u, R.u, cl, cr, pm, vxm, rhom, k);
    } else if (WHICH != kNewtonOnly && pattern == 3) {
        const RareT g = RareT(KT<RareT>::gamma(k));
        const RareT pl = RareT(L.p), pr = RareT(R.p), rl = RareT(L.rho), rr = RareT(R.rho);
        const RareT cleft = sqrt(g * pl / rl), cright = sqrt(g * pr / rr);
        // NaN when no branch of the closed form applies (a NaN state), as
        // the undefined values of the reference
        RareT tp = RareT(pm), tv = tp, tr = tp;
        riemann_two_rarefactions<RareT, PowRare>(pl, pr, rl, rr, RareT(L.u), RareT(R.u), cleft, cright, tp, tv, tr,
                                                 k);
        pm = double(tp);
        vxm = double(tv);
        rhom = double(tr);
        if constexpr (sizeof(RareT) < sizeof(double)) {
            // A face at the edge of the vacuum condition (the FP32
            // classification said two rarefactions, the FP32 closed form
            // gives a non-positive star pressure or density, or one below
            // FP32's range): classify and solve it again in FP64.
            if (!(pm > 0.0 && rhom > 0.0 && vxm == vxm)) {
                double cl, cr;
                const int p64 = riemann_classify<double, Pow>(L.p, R.p, L.rho, R.rho, L.u, R.u, cl, cr, k);
                pm = vxm = rhom = __longlong_as_double(0x7ff8000000000000ULL);
                if (p64 == 4) riemann_vacuum(L, R, cl, cr, pm, vxm, rhom, k);
                else riemann_two_rarefactions<double, Pow>(L.p, R.p, L.rho, R.rho, L.u, R.u, cl, cr, pm, vxm, rhom, k);
            }
        }
    } else if (WHICH != kNewtonOnly && pattern == 4) {
        const double cleft = sqrt(k.gamma * L.p / L.rho), cright = sqrt(k.gamma * R.p / R.rho);
        riemann_vacuum(L, R, cleft, cright, pm, vxm, rhom, k);
    }
    riemann_finish(L, R, pm, vxm, rhom, out, s);
    return ok;
}

// The mixed path's FP32 faces on FP32 states: the two-rarefaction closed
// form (pattern 3) and the FP32 Newton of weak faces (patterns 6, 7), the
// same arithmetic as riemann_by_pattern's FP32 branches without widening
// the face states to FP64 and back (the face rings of the mixed path hold
// FP32 values).
// Returns false, with out unset, for every other pattern and for a face
// whose FP32 solution fails (a non-positive or NaN star state, an FP32
// iteration that does not converge); riemann_by_pattern then solves it in
// FP64 (pattern 3, or 1 / 2 for a failed 6 / 7).  The transverse factor
// dadt = 1 - eps (riemannsolver.F90:36, eps = dat dt rat / 2 a few 1e-3)
// enters as v - eps v with eps in FP32: an FP32 dadt would carry its own
// rounding (up to 6e-8 relative) into every transverse flux of every sweep
// with the same sign, while eps v rounds at 1e-10 of v.
__device__ __forceinline__ bool riemann_mixed_f32(int pattern, const FaceF& L, const FaceF& R, FaceF& out,
                                                  const Consts& k, float eps) {
    float pm, vxm, rhom;
    const float g = k.fgamma;
    if (pattern == 3) {
        const float cleft = sqrtf(g * L.p / L.rho), cright = sqrtf(g * R.p / R.rho);
        pm = vxm = rhom = __int_as_float(0x7fc00000);
        riemann_two_rarefactions<float, PowRareF32>(L.p, R.p, L.rho, R.rho, L.u, R.u, cleft, cright, pm, vxm, rhom,
                                                    k);
        if (!(pm > 0.0f && rhom > 0.0f && vxm == vxm)) return false;
    } else if (pattern == 6 || pattern == 7) {
        float ps = newton_start_f32(L.p, R.p, L.rho, R.rho, L.u, R.u, k), us = 0.0f;
        if (!(ps > 0.0f && riemann_newton_f32(ps, us, L.p, R.p, L.rho, R.rho, L.u, R.u, k))) return false;
        pm = ps;
        vxm = us;
        rhom = __int_as_float(0x7fc00000);
        if (pattern == 6) {
            sample_two_shocks<float>(L, R, pm, vxm, rhom, k);
        } else {
            const float cleft = sqrtf(g * L.p / L.rho), cright = sqrtf(g * R.p / R.rho);
            sample_shock_rarefaction<float, PowRareF32>(L, R, cleft, cright, pm, vxm, rhom, k);
        }
    } else {
        return false;
    }
    // transverse velocities upwinded by the sign of u* (riemannsolver.F90:269-275)
    out.p = pm;
    out.rho = rhom;
    out.u = vxm;
    const float vt = vxm >= 0.0f ? L.v : R.v, wt = vxm >= 0.0f ? L.w : R.w;
    out.v = fmaf(-eps, vt, vt);
    out.w = fmaf(-eps, wt, wt);
    return true;
}

// riemannsolver, riemannsolver.F90:1-285, for a single face in FP64 (the
// density-peak fix of :279-285 is applied by the caller).
template <class Pow>
__device__ __forceinline__ bool riemannsolver(const FaceState& L, const FaceState& R, FaceState& out,
                                              const Consts& k, const StepScalars& s) {
    double cleft, cright;
    const int pattern = riemann_classify<double, Pow>(L.p, R.p, L.rho, R.rho, L.u, R.u, cleft, cright, k);
    return riemann_by_pattern<Pow, double, Pow>(pattern, L, R, out, k, s);
}

}  // namespace hp
