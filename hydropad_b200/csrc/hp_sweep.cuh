// hp_sweep.cuh -- the fused directional PPM sweep (one kernel per axis).
//
// Replaces the three OpenACC regions of one ppmsolver call
// (hydro/ppmsolver.F90:96-160 x, :214-288 y, :342-416 z) and the ghost
// exchange that follows it (hydro/ppm_lxlylz.F90:20-21):
//
//   R1 order2interp (flatten + parabolas + characteristic tracing),
//   R2 riemannsolver (exact Riemann problem, Newton for p*),
//   R3 integrate (conservative update + dual energy)
//
// run back to back on the same cells with every intermediate in shared
// memory.  The state is updated in place and read/written exactly once per
// sweep (5 fields x 8 B in + out = 80 B per cell).
//
// Work decomposition.  A CTA owns P whole pencils along the sweep axis and
// walks them with a sliding window of T cells per iteration.  Each cell's
// quantities are computed exactly once (the reference evaluates every
// parabola twice, once per adjacent face) and handed to neighbours through
// ring buffers of RING cells:
//
//   load   cell e                      state ring
//   A      cell e-1: ajside slopes, dda second difference of rho, the
//          flattening flag of the pair (e-1, e)          -> A ring
//   B      cell e-3: flat, parabolas of p, rho, u, v, w, characteristic
//          tracing -> left state of face e-2 (ls ring), right state of
//          face e-3 (registers)
//   C      face e-3: Riemann problem                     -> face ring
//   D      cell e-4: update from faces e-4 and e-3, store (the full-pencil
//          solver of the non-STENCIL build: the new total energy of cell
//          e-4, then the update of cell e-5)
//
// Periodicity is a wrap of the pencil index: the walk starts at cell -4
// (= N-4) and ends at N+3 (N+4); the original values of cells 0..2, which the
// walk re-reads at its end after they have been updated, are kept in a
// small save area.
//
// Thread layout.  Along x (AXIS 0) a warp holds 32 consecutive cells of one
// pencil; along y/z a warp holds 32 neighbouring pencils (consecutive x) at
// the same sweep position for the load and the update (256-byte coalesced
// rows) and 32/T neighbouring pencils x the T cells of the window for the
// stages in between (SweepLayout).
#pragma once
#include "hp_device.cuh"
#include "hp_physics.cuh"
#include "hp_riemann.cuh"

#include <type_traits>

namespace hp {

struct SweepArgs {
    double* f[5];          // p, rho, u (normal), v, w (transverse) of this sweep
    void* snap[4];         // step-start p, vx, vy, vz (natural order) for expand, Policy::SnapT
    const double* peak;    // per-face density-peak values for y/z sweeps (may be null)
    const double* g;       // gforce component along this sweep (natural layout), or null: gravity off
    // z sweep of a slab (kFlagZHalo): the 4 planes below and the 3 planes
    // above the slab, [field][plane][nx*ny] in the sweep's field order
    const double* zlo[5];
    const double* zhi[5];
    // full-pencil sweeps: the cho3d marker of each cell (natural layout), or
    // null for zeros
    const double* cho;
    DevCtl* ctl;
    Consts k;
    int nx, ny, nz;
    int nsweep;            // cells along the sweep axis
    long long npencil;     // pencils in this sweep
    int bslot;             // rho-bound slot this sweep reads (0..2)
    int flags;
};

// Precision policies.  R is the reconstruction/tracing type, Pow the power
// used by the Riemann solver.
struct PolicyFP64 {
    using R = double;          // reconstruction, flattening, tracing
    using Pow = PowRoot;       // powers of the FP64 Riemann solver
    using CT = double;         // wave-pattern classification
    using PowC = PowRoot;
    using RareT = double;      // closed two-rarefaction form
    using PowRare = PowRoot;
    using DivD = DivIEEE;      // divisions of the update
    using SnapT = double;      // step-start snapshot of expand
    static constexpr bool kWeakNewton = false;  // every Newton face in FP64
    static constexpr bool kFaceF32 = false;     // face ring in FP64
};
// Mixed precision: reconstruction, flattening, characteristic tracing and
// the traced face states in FP32; the Riemann solver's Newton for p*, u*,
// the conservative update and the dual-energy switch in FP64; the state in
// HBM stays FP64.
struct PolicyMixed {
    using R = float;             // reconstruction, flattening, tracing
    using Pow = PowRootShort;    // FP64 Newton for p*, u* (patterns 1, 2) and vacuum
    using CT = float;            // wave-pattern classification
    using PowC = PowF32m;
    using RareT = float;         // closed two-rarefaction form: no iteration
    using PowRare = PowRareF32;
    using DivD = PowRootShort;   // update divisions from a refined reciprocal (an ulp or two)
    // expand's step-start snapshot in FP32: it enters the step's end only as
    // afact * v_old / (2 + afact) and afact * p_old / (1 + afact), with afact
    // = dt dath / ath a few 1e-2, so its rounding moves v and p by ~1e-9
    using SnapT = float;
    static constexpr bool kWeakNewton = true;  // weak Newton faces in FP32 (patterns 6, 7)
    static constexpr bool kFaceF32 = true;     // face ring in FP32
};

// Values of the face ring: the traced right state of a face (stage C1),
// replaced by the face's Riemann state (C2), read by the update (D).  In
// the mixed path they are FP32: the traced states are FP32 values, and so
// are the Riemann states except the FP64 Newton's p*, u* of strong shocks
// and the upwinded transverse velocities (dadt v), which are rounded once.
// The update forms the fluxes from them in FP64 as integrate.F90 does
// (products of FP32 values, exact in FP64), so the flux differences of
// neighbouring faces keep their accuracy in bulk flows.  Forming the fluxes
// themselves in FP32 (once per face) made the update 4 % cheaper but
// raised the density L1 against FP64 after 100 steps at 512^3 from 2.8e-6
// to 1.2e-5: a flux rounded to FP32 in a supersonic bulk flow loses the
// small difference between neighbouring faces.
template <class Policy>
using FaceT = typename std::conditional<Policy::kFaceF32, float, double>::type;

template <int AXIS>
__device__ __forceinline__ long long pencil_base(long long pid, int nx, int ny) {
    if (AXIS == 0) return pid * nx;                                     // (y,z) -> x row
    if (AXIS == 1) return (pid % nx) + (long long)nx * ny * (pid / nx);  // (x,z)
    return pid;                                                         // (x,y)
}
template <int AXIS>
__device__ __forceinline__ long long axis_stride(int nx, int ny) {
    return AXIS == 0 ? 1 : (AXIS == 1 ? (long long)nx : (long long)nx * ny);
}

// Ring layout and the thread layout of stages A, B and C1.  Along x a warp
// holds whole pencil windows in both layouts.  Along y/z the load and the
// update keep 32 neighbouring pencils per warp (256-byte rows); when T
// divides 32, stages A, B and C1 re-deal the threads so that a warp holds
// kPw = 32/T neighbouring pencils x the T cells of the window, and those
// stages pass data within the warp.  The y/z ring rows are padded by kPw
// pencils, which keeps both layouts free of shared-memory bank conflicts.
// Along x a warp holds 32/T pencils when T < 32; the slots of its k-th
// pencil are XOR-ed with k*T (RING a multiple of 32), for the same reason.
template <int AXIS, int P, int T, int RING>
struct SweepLayout {
    static constexpr bool kYZWarp = AXIS != 0 && (32 % T) == 0 && (P % (32 / T)) == 0;
    static constexpr int kPw = kYZWarp ? 32 / T : 1;
    static constexpr int kStride = AXIS == 0 ? RING : (kYZWarp ? P + kPw : P);
    static constexpr int kThreads = P * T;
    static constexpr int kCells = kStride * (AXIS == 0 ? P : RING);
    static_assert(AXIS != 0 || T >= 32 || ((32 % T) == 0 && RING % 32 == 0), "x swizzle");
    __device__ __forceinline__ static int idx(int cell, int tp) {
        const int slot = cell & (RING - 1);
        if (AXIS == 0) return tp * RING + (T < 32 ? slot ^ ((tp & (32 / T - 1)) * T) : slot);
        return slot * kStride + tp;
    }
    // cell offset in the window and pencil of thread t in stages A, B, C1
    __device__ __forceinline__ static int wcell(int t) {
        return AXIS == 0 ? t % T : (kYZWarp ? (t & 31) / kPw : t / P);
    }
    __device__ __forceinline__ static int wpencil(int t) {
        return AXIS == 0 ? t / T : (kYZWarp ? (t >> 5) * kPw + (t & 31) % kPw : t % P);
    }
};

// Buckets of the Riemann problems, in the order the solving threads take
// them.  FP64 path: shock + rarefaction with the rarefaction on the left
// (pL >= pR), two shocks, shock + rarefaction with the rarefaction on the
// right (Newton), then the closed forms (patterns 3, 4, 5).  Mixed path
// (W): the weak faces' three (FP32 Newton, patterns 7, 6, 7), the closed
// forms, then the strong faces' three (FP64 Newton, patterns 2, 1, 2): the
// warp that holds the few strong faces of an iteration then shares it with
// closed forms, not with FP32 Newton faces, and the longest warp of the
// stage (run one after the other where a warp holds both) gets shorter.
// The Newton buckets of one precision share the iteration, and neighbouring
// Newton buckets differ in the wave on one side only, so a warp that
// straddles two of them diverges on one side of the loop body.
template <bool W> constexpr int kBucketsOf = W ? 9 : 6;
// 1 + bucket of a face of pattern 1..7 (patterns 2, 7: rare_left = pL >= pR)
template <bool W>
__device__ __forceinline__ int bucket_of(int pattern, bool rare_left) {
    if constexpr (W) {
        if (pattern == 7) return rare_left ? 1 : 3;
        if (pattern == 6) return 2;
        if (pattern == 2) return rare_left ? 7 : 9;
        if (pattern == 1) return 8;
        return pattern + 1;  // 3, 4, 5 -> 4, 5, 6
    } else {
        if (pattern == 2) return rare_left ? 1 : 3;
        if (pattern == 1) return 2;
        return pattern + 1;
    }
}
template <bool W>
__device__ __forceinline__ int pattern_of_bucket(int c) {
    if constexpr (W) {
        if (c == 0 || c == 2) return 7;
        if (c == 1) return 6;
        if (c == 6 || c == 8) return 2;
        if (c == 7) return 1;
        return c;  // 3, 4, 5
    } else {
        if (c == 0 || c == 2) return 2;
        if (c == 1) return 1;
        return c;
    }
}

template <int AXIS, int P, int T, int RING, class Policy, bool GRAV = false, bool PENCIL = false>
struct SweepSmem {
    using R = typename Policy::R;
    static constexpr int kC = SweepLayout<AXIS, P, T, RING>::kCells;
    static constexpr int kG = GRAV ? kC : 1;
    static constexpr int kE = PENCIL ? kC : 1;
    static constexpr int kBuckets = kBucketsOf<Policy::kWeakNewton>;
    double se[kE];              // full-pencil sweeps: new total energy of each cell
    R st[5][kC];                // state ring: p, rho, u, v, w (FP32 copy in the mixed path)
    double sg[kG];              // gravity ring: g = -gforce of this sweep's axis
    R slg[kG];                  // ajside slope of g
    alignas(8) R sl[5][kC];     // ajside slopes (after the walk: the block reduction's buffer)
    R d2[kC];                   // dda second difference of rho
    unsigned char pf[kC];       // flattening flag of pair (c, c+1)
    R ls[5][kC];                // traced left state (face c+1) from cell c
    // traced right state of face f (from cell f), replaced in place by the
    // Riemann state of face f (FaceT): each slot is read and then written by
    // the one thread that solves that face
    FaceT<Policy> rs[5][kC];
    // Riemann problems of the iteration (by the thread index that classified
    // them, a byte when the CTA has at most 256 threads), in buckets
    typename std::conditional<(P * T <= 256), unsigned char, unsigned short>::type work[kBuckets][P * T];
    int bcnt[2][kBuckets];      // bucket fill counts (alternate iterations use alternate rows)
    R sv[5][3 * P];             // original values of cells 0..2 (they only refill the state ring)
};

// The block reduction at the end of a walk (block_flush, 4 x 32 words)
// reuses the slope ring: block_flush starts with a CTA barrier, after which
// no thread reads the ring again in this walk, and the next walk of the
// batched kernel writes it only after its own CTA barriers.
template <class Smem>
__device__ __forceinline__ unsigned long long* red_buffer(Smem& S) {
    static_assert(sizeof(S.sl) >= 128 * sizeof(unsigned long long), "reduction buffer");
    return reinterpret_cast<unsigned long long*>(&S.sl[0][0]);
}

// Barrier between stages that pass data along the pencil only: a warp
// barrier when every warp holds whole pencil windows, else the CTA's.
template <bool kWarp>
__device__ __forceinline__ void pencil_sync() {
    if constexpr (kWarp) __syncwarp();
    else __syncthreads();
}

// ---------------------------------------------------------------------------
// Per-cell stage bodies shared by the sweep kernels (every kernel computes a
// cell's values with these, so they agree bit for bit).
// ---------------------------------------------------------------------------

// Stage A of cell c from cells c-1, c, c+1 (p, rho, u, v, w): the ajside
// slopes, the dda second difference of rho and the flattening flag of the
// pair (c, c+1) (order2interp.F90:65-113, ppm_functs.F90:167-181, dda.F90:17).
template <class R>
__device__ __forceinline__ void slopes_of_cell(const R am[5], const R a0[5], const R ap[5], R ming, R dx, R sl[5],
                                               R& d2, bool& flag) {
    flag = false;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        sl[q] = ajside<R>(am[q], a0[q], ap[q]);
        flag |= flat_pair<R>(a0[q], ap[q], ming);
        if (q == 1) d2 = dda_second<R>(am[q], a0[q], ap[q], dx);
    }
}

// Time scalars of the reconstruction, in its type.
template <class R>
struct TraceScalars {
    R dt, rat, dat, at, dx, gam, flatv;
};

// Stage B of cell c: flattening, the five parabolas (monotonicity, contact
// steepening of rho, flattening) and the characteristic tracing in expanding
// coordinates (order2interp.F90:115-258, ppm_functs.F90:1-162).  q1..q3 are
// cells c-1, c, c+1, dm..dp their slopes, Dm/Dp the second differences of
// rho at c-1 and c+1, fl_any the flattening flags of the pairs c-2 .. c+1.
// Gravity: g1..g3 = -gforce of cells c-1..c+1 and their slopes.  Returns the
// traced left state of face c+1 (`left`) and the right state of face c.
template <class R, bool GRAV, bool PENCIL>
__device__ __forceinline__ void trace_cell(const R q1[5], const R q2[5], const R q3[5], const R dm[5], const R d0[5],
                                           const R dp[5], R Dm, R Dp, bool fl_any, R g1, R g2, R g3, R gdm, R gd0,
                                           R gdp, const TraceScalars<R>& ts, R left[5],
                                           typename FaceOf<R>::type& right) {
    const R dt_ = ts.dt, rat_ = ts.rat, dat_ = ts.dat, at_ = ts.at, dx_ = ts.dx, gam_ = ts.gam;
    const R flat = fl_any ? ts.flatv : R(0);
    const R pm1 = q1[0], p0 = q2[0], pp1 = q3[0];
    const R rm1 = q1[1], r0 = q2[1], rp1 = q3[1];
    const R addp = fabs(pp1 - pm1) / fmin2(pm1, pp1);
    const R addrho = R(0.5) * gam_ * fabs(rp1 - rm1) / fmin2(rm1, rp1);
    const bool steep = addrho >= addp;
    const R u0 = q2[2];
    // sound speed of the characteristic speeds: the cell's own
    // (order2interp.F90:56-57); the full-pencil solver takes the next
    // cell's (ppm.F90:106-107: cbar = c(i), c(i+1) beside vxbar(2),
    // vxbar(3) = cells i-1, i)
    const R cc = PENCIL ? sqrt(gam_ * pp1 / rp1) : sqrt(gam_ * p0 / r0);
    // characteristic speeds of the cell (order2interp.F90:194-196,221-223)
    const R lm = (u0 - cc) * rat_, l0 = u0 * rat_, lp = (u0 + cc) * rat_;
    // x = y/dx of fl/fr (ppm_functs.F90:59-84); the right-side arguments
    // are exact negations of the left-side ones.
    const R yp = dt_ * (u0 + cc) * rat_;
    const R ym = dt_ * (u0 - cc) * rat_;
    const R y0 = dt_ * u0 * rat_;
    const R xp = yp / dx_, xm = ym / dx_, x0 = y0 / dx_;
    const R xtl = (R(0) > yp) ? R(0) / dx_ : xp;    // max(cv,0), atl
    const R xtr = (R(0) > -ym) ? R(0) / dx_ : -xm;  // max(cv,0), atr
    // traced values (t: fl/fr at the face; 1,2,3: the -,0,+
    // characteristics).  All are evaluated, branch-free; the tracing below
    // selects the ones the reference computes.
    R ptl, pc1l, pc2l, pc3l, ptr, pc1r, pc2r, pc3r;
    R rtl, rc2l, rtr, rc2r;
    R utl, uc1l, uc3l, utr, uc1r, uc3r;
    R vtl, vc2l, vtr, vc2r, wtl, wc2l, wtr, wc2r;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        R Dmq = 0, Dpq = 0;
        const bool st = (q == 1) && steep;
        if (q == 1) { Dmq = Dm; Dpq = Dp; }
        const Parabola<R> Pq = build_parabola<R>(q1[q], q2[q], q3[q], dm[q], d0[q], dp[q], flat, st, Dmq, Dpq, dx_);
        const R tl_ = fl(Pq, xtl), tr_ = fr(Pq, xtr);
        if (q == 0) {
            ptl = tl_; ptr = tr_;
            pc1l = fl(Pq, xm); pc2l = fl(Pq, x0); pc3l = fl(Pq, xp);
            pc1r = fr(Pq, -xm); pc2r = fr(Pq, -x0); pc3r = fr(Pq, -xp);
        } else if (q == 1) {
            rtl = tl_; rtr = tr_;
            rc2l = fl(Pq, x0); rc2r = fr(Pq, -x0);
        } else if (q == 2) {
            utl = tl_; utr = tr_;
            uc1l = fl(Pq, xm); uc3l = fl(Pq, xp);
            uc1r = fr(Pq, -xm); uc3r = fr(Pq, -xp);
        } else if (q == 3) {
            vtl = tl_; vtr = tr_;
            vc2l = fl(Pq, x0); vc2r = fr(Pq, -x0);
        } else {
            wtl = tl_; wtr = tr_;
            wc2l = fl(Pq, x0); wc2r = fr(Pq, -x0);
        }
    }
    // negative traced states (order2interp.F90:174-190)
    if (ptl < R(0)) ptl = R(kTiny);
    if (ptr < R(0)) ptr = R(kTiny);
    if (rtl < R(0)) rtl = R(kTiny);
    if (rtr < R(0)) rtr = R(kTiny);
    // g at the -/+ characteristics (order2interp.F90:170-172); gravity
    // off: g == 0
    R gc1l = R(0), gc3l = R(0), gc1r = R(0), gc3r = R(0);
    if constexpr (GRAV) {
        const Parabola<R> Pg = build_parabola<R>(g1, g2, g3, gdm, gd0, gdp, flat, false, R(0), R(0), dx_);
        gc1l = fl(Pg, xm);
        gc3l = fl(Pg, xp);
        gc1r = fr(Pg, -xm);
        gc3r = fr(Pg, -xp);
    }
    // left state of face c+1 (order2interp.F90:192-219,249-258)
    {
        const R ctl = sqrt(gam_ * ptl * rtl);
        const R bm_ = beta<R>(ctl, utl, uc1l, ptl, pc1l, gc1l, R(-1), dt_, at_, dat_, rat_);
        const R bp_ = beta<R>(ctl, utl, uc3l, ptl, pc3l, gc3l, R(1), dt_, at_, dat_, rat_);
        const R b0_ = beta0<R>(ctl, rtl, rc2l, ptl, pc2l, dt_, at_, dat_);
        const R bml = (lm > R(0)) ? bm_ : R(0);
        const R bpl = (lp > R(0)) ? bp_ : R(0);
        const R b0l = (l0 > R(0)) ? b0_ : R(0);
        const R vl = (l0 > R(0)) ? vc2l : vtl;
        const R wl = (l0 > R(0)) ? wc2l : wtl;
        R pl = ptl + ctl * ctl * (bpl + bml);
        if (pl <= R(0)) pl = ptl;
        const R ul = utl + ctl * (bpl - bml);
        R rl = R(1) / (R(1) / rtl - bml - b0l - bpl);
        if (rl <= R(0)) rl = rtl;
        left[0] = pl;
        left[1] = rl;
        left[2] = ul;
        left[3] = vl;
        left[4] = wl;
    }
    // right state of face c (order2interp.F90:221-258)
    {
        const R ctr = sqrt(gam_ * ptr * rtr);
        const R bp_ = beta<R>(ctr, utr, uc3r, ptr, pc3r, gc3r, R(1), dt_, at_, dat_, rat_);
        const R bm_ = beta<R>(ctr, utr, uc1r, ptr, pc1r, gc1r, R(-1), dt_, at_, dat_, rat_);
        const R b0_ = beta0<R>(ctr, rtr, rc2r, ptr, pc2r, dt_, at_, dat_);
        const R bpr = (lp < R(0)) ? bp_ : R(0);
        const R bmr = (lm < R(0)) ? bm_ : R(0);
        const R b0r = (l0 < R(0)) ? b0_ : R(0);
        const R vr = (l0 < R(0)) ? vc2r : vtr;
        const R wr = (l0 < R(0)) ? wc2r : wtr;
        R pr = ptr + ctr * ctr * (bpr + bmr);
        if (pr <= R(0)) pr = ptr;
        const R ur = utr + ctr * (bpr - bmr);
        R rr = R(1) / (R(1) / rtr - bmr - b0r - bpr);
        if (rr <= R(0)) rr = rtr;
        right.p = pr;
        right.rho = rr;
        right.u = ur;
        right.v = vr;
        right.w = wr;
    }
}

// Stage D's epilogue for cell g (updated state p, rho, u, v, w): expand
// with the step-start snapshot (expand.F90:18-41), the store, and the
// step's reductions (rho bounds, speed.F90:25-28 velmax, status).
template <int AXIS, class SnapT>
__device__ __forceinline__ void finish_cell(const SweepArgs& a, long long g, double p, double rho, double u, double v,
                                            double w, double afact, double afact1, double afact2,
                                            unsigned long long& kmin, unsigned long long& kmax,
                                            unsigned long long& kvel, unsigned& status) {
    if (a.flags & kFlagExpand) {
        const bool zero_old = (a.flags & kFlagExpandZeroOld) != 0;
        const double vx_o = zero_old ? 0.0 : double(static_cast<const SnapT*>(a.snap[1])[g]);
        const double vy_o = zero_old ? 0.0 : double(static_cast<const SnapT*>(a.snap[2])[g]);
        const double vz_o = zero_old ? 0.0 : double(static_cast<const SnapT*>(a.snap[3])[g]);
        const double p_o = zero_old ? 0.0 : double(static_cast<const SnapT*>(a.snap[0])[g]);
        const double un_o = AXIS == 0 ? vx_o : (AXIS == 1 ? vy_o : vz_o);
        const double v_o = AXIS == 0 ? vy_o : (AXIS == 1 ? vx_o : vy_o);
        const double w_o = AXIS == 0 ? vz_o : (AXIS == 1 ? vz_o : vx_o);
        u = (2.0 * u - afact * un_o) * afact2;
        v = (2.0 * v - afact * v_o) * afact2;
        w = (2.0 * w - afact * w_o) * afact2;
        const double ppp = p;
        p = (p - afact * p_o) * afact1;
        if (p <= 0.0) p = ppp > 0.0 ? ppp : p_o;
    }
    a.f[0][g] = p;
    a.f[1][g] = rho;
    a.f[2][g] = u;
    a.f[3][g] = v;
    a.f[4][g] = w;
    const unsigned long long kr = dkey(rho);
    kmin = kr < kmin ? kr : kmin;
    kmax = kr > kmax ? kr : kmax;
    if (a.flags & kFlagSpeed) {
        const double vs = sqrt(a.k.gamma * p / rho);
        double vm = fabs(u) + vs;
        vm = fmax2(vm, fabs(v) + vs);
        vm = fmax2(vm, fabs(w) + vs);
        const unsigned long long kb = (unsigned long long)__double_as_longlong(vm);
        kvel = kb > kvel ? kb : kvel;
    }
    if (!(rho == rho) || !(p == p) || !(u == u) || !(v == v) || !(w == w)) {
        status |= kStatNaN;
        record_bad_cell(a.ctl, g);
    } else if (rho <= 0.0 || p <= 0.0) {
        status |= kStatNegative;
        record_bad_cell(a.ctl, g);
    }
}

// One CTA's worth of work: the P pencils pid0 .. pid0+P-1 of the box `a`,
// walked from end to end.  Every thread of the CTA calls it.
// PENCIL: the non-STENCIL build's full-pencil solver (hydro/ppm.F90)
// instead of the STENCIL sweep; see the notes at its four differences.
template <int AXIS, int P, int T, int RING, class Policy, bool GRAV = false, bool PENCIL = false>
__device__ __forceinline__ void sweep_pencils(const SweepArgs& a, long long pid0,
                                              SweepSmem<AXIS, P, T, RING, Policy, GRAV, PENCIL>& S) {
    using R = typename Policy::R;
    using Pow = typename Policy::Pow;
    using CT = typename Policy::CT;
    using L = SweepLayout<AXIS, P, T, RING>;
    static_assert((RING & (RING - 1)) == 0 && RING >= T + 6, "ring too small");
    static_assert(P * T <= 65536, "work items are 16-bit thread indices");
    static_assert(!(GRAV && PENCIL), "the full-pencil solver has no gravity source (ppm.F90:93,102)");
    // the full-pencil solver's update runs one cell later than the STENCIL
    // one (its dual-energy switch reads the new total energy of the next cell)
    constexpr int kLag = PENCIL ? 1 : 0;

    const int tid = threadIdx.x;
    const int tl = AXIS == 0 ? (tid % T) : (tid / P);
    const int tp = AXIS == 0 ? (tid / T) : (tid % P);
    const long long pid = pid0 + tp;
    const bool active = pid < a.npencil;
    // the same in the layout of stages A, B and C1
    const int tlw = L::wcell(tid), tpw = L::wpencil(tid);
    const bool activew = pid0 + tpw < a.npencil;
    const int N = a.nsweep;
    const long long base = pencil_base<AXIS>(active ? pid : 0, a.nx, a.ny);
    const long long stride = axis_stride<AXIS>(a.nx, a.ny);

    const Consts k = a.k;
    const StepScalars sc = a.ctl->s;
    const R dt_ = R(sc.dt), rat_ = R(sc.rat), dat_ = R(sc.dat), at_ = R(sc.at);
    const R dx_ = R(KT<R>::dx(k)), gam_ = R(KT<R>::gamma(k)), flatv_ = R(KT<R>::flat(k)), ming_ = R(KT<R>::ming(k));
    const TraceScalars<R> ts{dt_, rat_, dat_, at_, dx_, gam_, flatv_};
    if (a.ctl->done) return;  // told >= tstop: the time loop has ended (main.F90:100)

    // density-peak fix is possible only if some rho exceeds dmax x another
    // rho (monotone rounding makes this test exact; see the update epilogue)
    const double rmin0 = dkey_decode(a.ctl->rho_key[a.bslot][0]);
    const double rmax0 = dkey_decode(a.ctl->rho_key[a.bslot][1]);
    const bool peak_possible = rmax0 > k.dmax * rmin0;

    if (tid == 0 && pid0 == 0) {  // once per box and sweep
        const int reset = (a.bslot + 2) % 3;
        a.ctl->rho_key[reset][0] = kKeyPosInf;
        a.ctl->rho_key[reset][1] = kKeyNegInf;
        if (a.flags & kFlagResetSpeed) a.ctl->velmax_key = 0ULL;
    }

    // the transverse factor dadt = 1 - dadt_eps of riemann_finish
    // (riemannsolver.F90:36) for the mixed path's FP32 faces
    const float dadt_eps = float(0.5 * sc.dat * sc.dt * sc.rat);
    // expand.F90:18-20
    const double afact = sc.dt * (sc.dath / sc.ath);
    const double afact1 = 1.0 / (1.0 + afact);
    const double afact2 = 1.0 / (2.0 + afact);

    unsigned long long kmin = kKeyPosInf, kmax = 0ULL, kvel = 0ULL;
    unsigned status = 0;

    typename FaceOf<R>::type right;  // right state of face c (cell c), from stage B, in the type R

    // Barriers.  Stages load, A, B and C1 exchange data only along a pencil
    // (ring neighbours e-2 .. e+2).  Along x a warp holds whole pencil
    // windows (T divides 32), so warp barriers order them; along y/z the
    // threads change layout after the load (a CTA barrier) and then hold
    // whole pencil windows for A, B and C1 (warp barriers).  C2 solves any
    // pencil's faces and D reads any thread's C2 result: CTA barriers.
    // The barrier before the load protects the state ring slots that the
    // load overwrites from the previous iteration's stage D, which reads the
    // ring only in the FP64 path and with gravity (the g ring); the mixed
    // path's D reads the cell from global memory instead, so its y/z sweeps
    // need no barrier there (everything else the load writes is read after
    // the next barrier only).
    // Early load (the mixed path's z sweeps): the cells of the next
    // iteration are loaded by each thread as soon as its C2 work is done,
    // before the C2 -> D barrier, which then also publishes them to the
    // layout of stages A-C1.  The threads that finish C2 early load while
    // the Newton faces are still being solved, and the barrier after the
    // load goes.  It needs D to leave the state ring alone (the load then
    // overwrites slots of cells D of this iteration would read) and C2 not
    // to read it (the x sweep's density-peak window does; y/z read the
    // pre-pass's values).  Measured on a late 512^3 state (tile 7): z
    // sweeps 7.76 -> 7.58 ms, whose loads are a plane apart and take the
    // longest; y sweeps 7.58 -> 7.65 ms (the load's registers in the C2
    // region add spills), so y keeps the load at the top.  The load of a wrapped cell e >= N keeps its rule:
    // it reads the save area (written by an earlier load) when D of the
    // iteration before e's could have overwritten cell e-N, which with the
    // early load may not have run yet; either copy holds the original value.
    constexpr bool kWarpPencils = AXIS == 0 && T <= 32 && (32 % T) == 0;
    constexpr bool kWarpStages = kWarpPencils || L::kYZWarp;  // A -> B -> C1 within a warp
    constexpr bool kDReadsRing = sizeof(R) == sizeof(double) || GRAV;
    constexpr bool kEarlyLoad = AXIS == 2 && !kDReadsRing && !PENCIL;
    constexpr bool kW = Policy::kWeakNewton;
    constexpr int kBuckets = kBucketsOf<kW>;
    if (tid < 2 * kBuckets) S.bcnt[tid / kBuckets][tid % kBuckets] = 0;
    int par = 0;  // row of bcnt of this iteration

    using DivD = typename Policy::DivD;
    // D's inputs: the Riemann states of faces d and d+1 of this thread's
    // pencil, and the cell's FP64 state: from the ring in the FP64 path; the
    // mixed path keeps an FP32 ring and reads it again from global memory,
    // which still holds it (only this thread writes cell d)
    auto load_faces = [&](int d, FaceState& f1, FaceState& f2) {
        const int id = L::idx(d, tp), id1 = L::idx(d + 1, tp);
        f1.p = S.rs[0][id];
        f1.rho = S.rs[1][id];
        f1.u = S.rs[2][id];
        f1.v = S.rs[3][id];
        f1.w = S.rs[4][id];
        f2.p = S.rs[0][id1];
        f2.rho = S.rs[1][id1];
        f2.u = S.rs[2][id1];
        f2.v = S.rs[3][id1];
        f2.w = S.rs[4][id1];
    };
    auto cell_state = [&](int d, long long g, double& p, double& rho, double& u, double& v, double& w) {
        if constexpr (sizeof(R) == sizeof(double)) {
            const int id = L::idx(d, tp);
            p = S.st[0][id]; rho = S.st[1][id]; u = S.st[2][id]; v = S.st[3][id]; w = S.st[4][id];
        } else {
            p = a.f[0][g]; rho = a.f[1][g]; u = a.f[2][g]; v = a.f[3][g]; w = a.f[4][g];
        }
    };
    // D's epilogue: expand, store, and the step's reductions
    auto finish = [&](long long g, double p, double rho, double u, double v, double w) {
        finish_cell<AXIS, typename Policy::SnapT>(a, g, p, rho, u, v, w, afact, afact1, afact2, kmin, kmax, kvel,
                                                  status);
    };

    // ---------------- load: cell e of this thread's pencil (load layout) ----------------
    auto load_cell = [&](const int e) {
        if (active && e >= -4 && e <= N + 2) {
            double v[5];
            // Cell e-N (0..2) is overwritten by stage D of the iteration that
            // holds e' = e-N+4+kLag; until then global memory still has the
            // original value (and the save area may not be written yet when
            // the pencil is shorter than one iteration).
            const bool from_save = e >= N && (e + 4) / T > (e - N + 8 + kLag) / T;
            const bool from_halo = AXIS == 2 && (a.flags & kFlagZHalo) && (e < 0 || e >= N);
            if (from_halo) {
                // a z slab's neighbours: planes -4..-1 below, N..N+2 above
                const long long plane = (long long)a.nx * a.ny;
                const long long off = (e < 0 ? (long long)(e + 4) : (long long)(e - N)) * plane + pid;
#pragma unroll
                for (int q = 0; q < 5; ++q) v[q] = (e < 0 ? a.zlo[q] : a.zhi[q])[off];
            } else if (from_save) {
#pragma unroll
                for (int q = 0; q < 5; ++q) v[q] = S.sv[q][(e - N) * P + tp];
            } else {
                const int s = e < 0 ? e + N : (e >= N ? e - N : e);
                const long long g = base + stride * s;
#pragma unroll
                for (int q = 0; q < 5; ++q) v[q] = a.f[q][g];
                if (e >= 0 && e < 3) {
#pragma unroll
                    for (int q = 0; q < 5; ++q) S.sv[q][e * P + tp] = R(v[q]);
                }
                if ((a.flags & kFlagSnapshot) && e >= 0 && e < N) {
                    // natural order p, vx, vy, vz
                    double vx = AXIS == 0 ? v[2] : (AXIS == 1 ? v[3] : v[4]);
                    double vy = AXIS == 0 ? v[3] : (AXIS == 1 ? v[2] : v[3]);
                    double vz = AXIS == 0 ? v[4] : (AXIS == 1 ? v[4] : v[2]);
                    using SnapT = typename Policy::SnapT;
                    static_cast<SnapT*>(a.snap[0])[g] = SnapT(v[0]);
                    static_cast<SnapT*>(a.snap[1])[g] = SnapT(vx);
                    static_cast<SnapT*>(a.snap[2])[g] = SnapT(vy);
                    static_cast<SnapT*>(a.snap[3])[g] = SnapT(vz);
                }
            }
            const int ix = L::idx(e, tp);
#pragma unroll
            for (int q = 0; q < 5; ++q) S.st[q][ix] = R(v[q]);
            if constexpr (GRAV) {
                // g(ippm) = -gforce(d, ...) (ppmsolver.F90:108,230,358); the
                // field never changes, so no save area is needed
                const int s = e < 0 ? e + N : (e >= N ? e - N : e);
                S.sg[ix] = -a.g[base + stride * s];
            }
        }
    };

    if constexpr (kEarlyLoad) load_cell(-4 + tl);
    __syncthreads();
    for (int b = -4; b <= N + 3 + kLag; b += T, par ^= 1) {
        const int e = b + tl;    // load and update layout
        const int ew = b + tlw;  // layout of stages A, B and C1
        if constexpr (!kEarlyLoad) {
            if constexpr (kWarpPencils) __syncwarp();
            else if constexpr (kDReadsRing) __syncthreads();
            load_cell(e);
            pencil_sync<kWarpPencils>();  // y/z: the threads change layout here
        }
        // ---------------- A: cell c = e-1 ----------------
        {
            const int c = ew - 1;
            if (activew && c >= -3 && c <= N + 1) {
                const int im = L::idx(c - 1, tpw), i0 = L::idx(c, tpw), ip = L::idx(c + 1, tpw);
                R am[5], a0[5], ap[5], sl[5], d2;
                bool flag;
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    am[q] = R(S.st[q][im]);
                    a0[q] = R(S.st[q][i0]);
                    ap[q] = R(S.st[q][ip]);
                }
                slopes_of_cell<R>(am, a0, ap, ming_, dx_, sl, d2, flag);
#pragma unroll
                for (int q = 0; q < 5; ++q) S.sl[q][i0] = sl[q];
                S.d2[i0] = d2;
                S.pf[i0] = flag ? 1 : 0;
                if constexpr (GRAV) S.slg[i0] = ajside<R>(R(S.sg[im]), R(S.sg[i0]), R(S.sg[ip]));
            }
        }
        pencil_sync<kWarpStages>();
        // ---------------- B: cell c = e-3 ----------------
        {
            const int c = ew - 3;
            if (activew && c >= -1 && c <= N) {
                int ic[5];
#pragma unroll
                for (int o = 0; o < 5; ++o) ic[o] = L::idx(c - 2 + o, tpw);
                const bool fl_any = S.pf[ic[0]] | S.pf[ic[1]] | S.pf[ic[2]] | S.pf[ic[3]];
                R q1[5], q2[5], q3[5], dm[5], d0[5], dp[5], left[5];
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    q1[q] = R(S.st[q][ic[1]]);
                    q2[q] = R(S.st[q][ic[2]]);
                    q3[q] = R(S.st[q][ic[3]]);
                    dm[q] = S.sl[q][ic[1]];
                    d0[q] = S.sl[q][ic[2]];
                    dp[q] = S.sl[q][ic[3]];
                }
                R g1 = R(0), g2 = R(0), g3 = R(0), gdm = R(0), gd0 = R(0), gdp = R(0);
                if constexpr (GRAV) {
                    g1 = R(S.sg[ic[1]]); g2 = R(S.sg[ic[2]]); g3 = R(S.sg[ic[3]]);
                    gdm = S.slg[ic[1]]; gd0 = S.slg[ic[2]]; gdp = S.slg[ic[3]];
                }
                trace_cell<R, GRAV, PENCIL>(q1, q2, q3, dm, d0, dp, S.d2[ic[1]], S.d2[ic[3]], fl_any, g1, g2, g3, gdm,
                                            gd0, gdp, ts, left, right);
                const int io = ic[2];
#pragma unroll
                for (int q = 0; q < 5; ++q) S.ls[q][io] = left[q];
            }
        }
        pencil_sync<kWarpStages>();
        // ---------------- C: face f = e-3 ----------------
        // The Riemann problems of the iteration are classified by wave
        // pattern and re-dealt to the threads sorted by pattern, so that a
        // warp solves problems of one pattern (the patterns take very
        // different code paths; faces of a smooth flow alternate between
        // them).  C1 classifies and publishes the right states.
        {
            const int f = ew - 3;
            int bucket = 0;  // 1 + bucket of the face, 0: no face
            if (activew && f >= 0 && f <= N) {
                const int io = L::idx(f, tpw);
                S.rs[0][io] = FaceT<Policy>(right.p);
                S.rs[1][io] = FaceT<Policy>(right.rho);
                S.rs[2][io] = FaceT<Policy>(right.u);
                S.rs[3][io] = FaceT<Policy>(right.v);
                S.rs[4][io] = FaceT<Policy>(right.w);
                const int il = L::idx(f - 1, tpw);
                CT cl, cr;
                const CT pl = CT(S.ls[0][il]), pr = CT(right.p);
                const CT rl = CT(S.ls[1][il]), rr = CT(right.rho), ul = CT(S.ls[2][il]), ur = CT(right.u);
                int pattern = riemann_classify<CT, typename Policy::PowC>(pl, pr, rl, rr, ul, ur, cl, cr, k);
                pattern = solver_pattern<kW>(pattern, float(pl), float(pr), float(rl), float(rr), float(ul),
                                             float(ur), float(cl), float(cr));
                bucket = bucket_of<kW>(pattern, pl >= pr);
            }
            // the lanes of one bucket take a run of its slots with one
            // shared-memory atomic (the order of the runs within a bucket
            // varies; every face's result does not)
            const int lane = tid & 31;
            const unsigned peers = __match_any_sync(0xffffffffu, bucket);
            const int leader = __ffs(peers) - 1;
            int off = 0;
            if (bucket && lane == leader) off = atomicAdd(&S.bcnt[par][bucket - 1], __popc(peers));
            off = __shfl_sync(0xffffffffu, off, leader);
            if (bucket) S.work[bucket - 1][off + __popc(peers & ((1u << lane) - 1u))] = tid;
        }
        __syncthreads();
        // C2: solve problem number tid of the buckets laid end to end.
        int pattern = 0, item = 0;
        {
            int idx = tid;
#pragma unroll
            for (int c = 0; c < kBuckets; ++c) {
                const int n = S.bcnt[par][c];
                if (pattern == 0) {
                    if (idx < n) {
                        pattern = pattern_of_bucket<kW>(c);
                        item = S.work[c][idx];
                    } else {
                        idx -= n;
                    }
                }
            }
            // the other row was last read in the previous iteration's C2
            // and is next filled after this iteration's last barrier
            if (tid < kBuckets) S.bcnt[par ^ 1][tid] = 0;
        }
        if (pattern) {
            // the classifying thread's pencil and face
            const int wtp = L::wpencil(item);
            const int f = b - 3 + L::wcell(item);
            const int il = L::idx(f - 1, wtp), io = L::idx(f, wtp);
            // density-peak fix (riemannsolver.F90:279-285): the pressure
            // floor of face f, -inf when the fix does not apply
            auto peak_floor = [&]() -> double {
                if (AXIS == 2 && (a.flags & kFlagZHalo)) {
                    // the transposed gather of the z peak test reaches
                    // across slabs; a slab reports it instead of applying it
                    status |= kStatUnsupported;
                    return -__longlong_as_double(0x7ff0000000000000ULL);
                }
                if constexpr (PENCIL) {
                    // the full-pencil solver's 5-cell window along the sweep:
                    // rhobar(1..4) = cells f-2..f+1, vxbar(2..3) = f-1, f
                    return peak_value(S.st[1][L::idx(f - 2, wtp)], S.st[1][L::idx(f - 1, wtp)],
                                      S.st[1][L::idx(f, wtp)], S.st[1][L::idx(f + 1, wtp)],
                                      S.st[2][L::idx(f - 1, wtp)], S.st[2][L::idx(f, wtp)], k.dmax);
                } else if (AXIS == 0) {
                    return peak_value(S.st[1][L::idx(f - 3, wtp)], S.st[1][L::idx(f - 2, wtp)],
                                      S.st[1][L::idx(f - 1, wtp)], S.st[1][L::idx(f, wtp)],
                                      S.st[2][L::idx(f - 2, wtp)], S.st[2][L::idx(f - 1, wtp)], k.dmax);
                } else {
                    // the reference gathers these with the x index slot
                    // (ppmsolver.F90:251-252, 379-380); a pre-pass has
                    // evaluated them on the pre-sweep state: face f < N at
                    // the index of cell f, face N after the last cell
                    if (f < N) return a.peak[pencil_base<AXIS>(pid0 + wtp, a.nx, a.ny) + stride * f];
                    return a.peak[(long long)a.nx * a.ny * a.nz + pid0 + wtp];
                }
            };
            bool solved = false;
            if constexpr (Policy::kFaceF32) {
                // the mixed path's FP32 faces straight from the FP32 rings
                FaceF lf, rf, of;
                lf.p = S.ls[0][il]; lf.rho = S.ls[1][il]; lf.u = S.ls[2][il]; lf.v = S.ls[3][il];
                lf.w = S.ls[4][il];
                rf.p = S.rs[0][io]; rf.rho = S.rs[1][io]; rf.u = S.rs[2][io]; rf.v = S.rs[3][io];
                rf.w = S.rs[4][io];
                if (riemann_mixed_f32(pattern, lf, rf, of, k, dadt_eps)) {
                    if (peak_possible) of.p = float(fmax2(double(of.p), peak_floor()));
                    S.rs[0][io] = of.p;
                    S.rs[1][io] = of.rho;
                    S.rs[2][io] = of.u;
                    S.rs[3][io] = of.v;
                    S.rs[4][io] = of.w;
                    solved = true;
                } else if (pattern >= 6) {
                    pattern -= 5;  // the FP32 iteration failed: FP64
                }
            }
            if (!solved) {
                FaceState left, rgt, out;
                left.p = double(S.ls[0][il]);
                left.rho = double(S.ls[1][il]);
                left.u = double(S.ls[2][il]);
                left.v = double(S.ls[3][il]);
                left.w = double(S.ls[4][il]);
                rgt.p = S.rs[0][io];
                rgt.rho = S.rs[1][io];
                rgt.u = S.rs[2][io];
                rgt.v = S.rs[3][io];
                rgt.w = S.rs[4][io];
                constexpr int kWhich = Policy::kFaceF32 ? kFallback : kAllPatterns;
                if (!riemann_by_pattern<Pow, typename Policy::RareT, typename Policy::PowRare, kWhich>(
                        pattern, left, rgt, out, k, sc))
                    status |= kStatNewton;
                if (peak_possible) out.p = fmax2(out.p, peak_floor());
                S.rs[0][io] = FaceT<Policy>(out.p);
                S.rs[1][io] = FaceT<Policy>(out.rho);
                S.rs[2][io] = FaceT<Policy>(out.u);
                S.rs[3][io] = FaceT<Policy>(out.v);
                S.rs[4][io] = FaceT<Policy>(out.w);
            }
        }
        if constexpr (kEarlyLoad) {
            if (b + T <= N + 3 + kLag) load_cell(e + T);  // the next iteration's cell
        }
        __syncthreads();
        // ---------------- D: cell d = e-4 ----------------
        if constexpr (PENCIL) {
            // D1: the new total energy of cell e-4, which the dual-energy
            // switch of its neighbours reads (ppm.F90:611-621)
            {
                const int d = e - 4;
                if (active && d >= 0 && d < N) {
                    const long long g = base + stride * d;
                    FaceState f1, f2;
                    load_faces(d, f1, f2);
                    double p, rho, u, v, w;
                    cell_state(d, g, p, rho, u, v, w);
                    // total() of the pencil's order (normal, transverse 1,
                    // transverse 2; ppmsolver.F90:173,301,429)
                    S.se[L::idx(d, tp)] = etot_new(f1, f2, total_energy(p, rho, u, v, w, k.rgamma1), k, sc);
                }
            }
            pencil_sync<kWarpPencils>();
            // D2: the update of cell e-5
            {
                const int d = e - 5;
                if (active && d >= 0 && d < N) {
                    const long long g = base + stride * d;
                    FaceState f1, f2;
                    load_faces(d, f1, f2);
                    double p, rho, u, v, w;
                    cell_state(d, g, p, rho, u, v, w);
                    const double etot = total_energy(p, rho, u, v, w, k.rgamma1);
                    const double eint = p * k.rgamma1;
                    // the neighbours' new total energy, 0 beyond the pencil's
                    // updated cells (ppm.F90:613-617)
                    const double eel = d > 0 ? S.se[L::idx(d - 1, tp)] : 0.0;
                    const double eer = d < N - 1 ? S.se[L::idx(d + 1, tp)] : 0.0;
                    // density peak of the cell against its old neighbours
                    // (ppm.F90:585-586)
                    const bool peak = rho > k.dmax * double(S.st[1][L::idx(d - 1, tp)]) &&
                                      rho > k.dmax * double(S.st[1][L::idx(d + 1, tp)]);
                    const double cho = (peak && a.cho) ? a.cho[g] : 0.0;
                    integrate_pencil<DivD>(f1, f2, p, rho, u, v, w, etot, eint, k, sc, eel, eer, peak, cho);
                    finish(g, p, rho, u, v, w);
                }
            }
        } else {
            const int d = e - 4;
            if (active && d >= 0 && d < N) {
                const long long g = base + stride * d;
                FaceState f1, f2;
                load_faces(d, f1, f2);
                double p, rho, u, v, w;
                cell_state(d, g, p, rho, u, v, w);
                // total() with the natural component order (ppmsolver.F90:149,277,405)
                double etot;
                if (AXIS == 2) etot = total_energy(p, rho, w, v, u, k.rgamma1);
                else etot = total_energy(p, rho, u, v, w, k.rgamma1);
                const double eint = p * k.rgamma1;
                if constexpr (GRAV) {
                    integrate<true, DivD>(f1, f2, p, rho, u, v, w, etot, eint, k, sc, S.sg[L::idx(d, tp)]);
                } else {
                    integrate<false, DivD>(f1, f2, p, rho, u, v, w, etot, eint, k, sc, 0.0);
                }
                finish(g, p, rho, u, v, w);
            }
        }
    }
    block_flush(kmin, kmax, kvel, status, &a.ctl->rho_key[(a.bslot + 1) % 3][0],
                &a.ctl->rho_key[(a.bslot + 1) % 3][1], (a.flags & kFlagSpeed) ? &a.ctl->velmax_key : nullptr,
                &a.ctl->status, red_buffer(S));
}

// One box per launch: CTA b takes pencils b*P .. b*P+P-1.
// MINB > 1 asks the compiler for at most 65536/(P*T*MINB) registers per
// thread so that MINB CTAs fit on one SM (more warps to hide the latency of
// the FP64 Riemann chains, at the price of spills).
template <int AXIS, int P, int T, int RING, class Policy, int MINB = 1, bool GRAV = false, bool PENCIL = false>
__global__ void __launch_bounds__(P* T, MINB) ppm_sweep_kernel(SweepArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto& S = *reinterpret_cast<SweepSmem<AXIS, P, T, RING, Policy, GRAV, PENCIL>*>(smem_raw);
    sweep_pencils<AXIS, P, T, RING, Policy, GRAV, PENCIL>(a, (long long)blockIdx.x * P, S);
}

// Many boxes per launch (the ensemble and the serving batch).  Work item i
// is a group of P pencils of one box: entry e owns the items
// first[e] .. first[e+1]-1 and sweeps box args[arg[e]].  A persistent grid
// pulls items from a queue until it is empty, so boxes of different sizes
// share the SMs without a tail per box.  All boxes of one launch are swept
// along the same axis.
struct BatchLaunch {
    const SweepArgs* args;   // per (box, slot, axis) arguments
    const int* ent;          // arg[0..nent-1], then first[0..nent]
    int nent;
    int nitems;              // first[nent]
    int* counter;            // work queue head, zero before the launch
};

template <int AXIS, int P, int T, int RING, class Policy, int MINB = 1>
__global__ void __launch_bounds__(P* T, MINB) ppm_sweep_batch_kernel(BatchLaunch bl) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto& S = *reinterpret_cast<SweepSmem<AXIS, P, T, RING, Policy>*>(smem_raw);
    __shared__ SweepArgs s_args;
    __shared__ int s_item, s_arg, s_first;
    const int* first = bl.ent + bl.nent;
    for (;;) {
        if (threadIdx.x == 0) {
            const int it = atomicAdd(bl.counter, 1);
            s_item = it;
            if (it < bl.nitems) {
                int lo = 0, hi = bl.nent - 1;  // last entry with first[e] <= it
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (first[mid] <= it) lo = mid;
                    else hi = mid - 1;
                }
                s_arg = bl.ent[lo];
                s_first = first[lo];
            }
        }
        __syncthreads();
        const int it = s_item;
        if (it >= bl.nitems) break;
        {
            static_assert(sizeof(SweepArgs) % 8 == 0, "SweepArgs copy in 8-byte words");
            const unsigned long long* src = reinterpret_cast<const unsigned long long*>(bl.args + s_arg);
            unsigned long long* dst = reinterpret_cast<unsigned long long*>(&s_args);
            for (int w = threadIdx.x; w < (int)(sizeof(SweepArgs) / 8); w += blockDim.x) dst[w] = src[w];
        }
        __syncthreads();
        sweep_pencils<AXIS, P, T, RING, Policy>(s_args, (long long)(it - s_first) * P, S);
        __syncthreads();  // s_item / s_args are rewritten for the next item
    }
}

}  // namespace hp
