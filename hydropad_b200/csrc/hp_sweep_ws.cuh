// hp_sweep_ws.cuh -- the pipelined fused sweep: TMA-staged state, a warp
// group that solves the Newton faces one window behind, persistent CTAs.
//
// The same sweep as ppm_sweep_kernel (hydro/ppmsolver.F90:96-160 x,
// :214-288 y, :342-416 z: order2interp, riemannsolver, integrate on the same
// cells with every intermediate in shared memory) with the per-cell
// arithmetic of the shared stage functions, so it computes the same bits;
// what changes is how the work is ordered on the SM:
//
//   * the state of the CTA's pencils arrives by bulk tensor copies (TMA,
//     cp.async.bulk.tensor) into a ring of 4 windows, one window ahead of
//     the stages that read it, ordered by an mbarrier per ring slot;
//   * the main warp group runs stages A, B, C1 (classification) and the
//     closed-form Riemann problems of window s, and the update of window
//     s-1; the faces that need the Newton iteration for p* (two shocks,
//     shock + rarefaction) go to a queue that a second warp group solves
//     while the main group works on the next window -- the dependent FP64
//     Newton chains no longer stall the CTA at a barrier;
//   * a CTA walks several pencil groups back to back (grid = resident CTAs),
//     and the pipeline runs on across the group boundaries.
//
// Windows.  Window w of a group covers cells b..b+T-1, b = -4 + wT, as the
// windows of ppm_sweep_kernel: load cell e, A at e-1, B at e-3, C at face
// e-3, D at cell e-4.  Windows that lie inside [0, N) come by TMA; the first
// (it wraps around the periodic end) and the last ones (cells N..N+2 are
// the original cells 0..2, kept in a save area) are loaded by the main
// threads.  Ring slot of cell c: (c + 4) mod 4T (state, faces) or mod 2T
// (stage A results).
//
// Synchronisation per window s (main group, barrier 1 = the main threads):
//   main threads wait full[s % 4] (TMA) | main threads load  -> barrier
//   thread 0 issues the TMA of window s+1 (slot of window s-3, dead)
//   A, B, C1 (warp-local) -> barrier -> thread 0 arrives nready[s % 2]
//   closed forms of window s
//   main threads wait ndone[(s-1) % 2] -> barrier -> D of window s-1
// Newton group, window s: wait nready[s % 2], solve, arrive ndone[s % 2].
// Every wait is bounded (hp_tma.cuh); a timeout sets kStatTimeout and ends
// the kernel through a flag that every role polls.
#pragma once
#include <cuda.h>

#include <type_traits>

#include "hp_sweep.cuh"
#include "hp_tma.cuh"

namespace hp {

// Thread and ring layouts.  P pencils x T cells per window; the main group
// has one thread per cell of a window (P*T), the Newton group NW warps.
// Along x (T = 32) a warp holds one pencil's window in every stage.  Along
// y/z (P = 16, one 128-byte row of x per sweep position) the loads and the
// update keep 16 pencils x 2 positions per warp, stages A, B, C1 32/T
// pencils x T positions; the TMA-written state rows use the 128-byte
// swizzle and the other rings rows padded by 32/T pencils, so that both
// layouts access shared memory without bank conflicts.
template <int AXIS, int P, int T, int NW>
struct WsLayout {
    static constexpr int kMain = P * T;
    static constexpr int kMainWarps = kMain / 32;
    static constexpr int kThreads = kMain + 32 * NW;
    static constexpr int kW = P * T;    // cells of one window
    static constexpr int kRing = 4 * T; // state and face slots per pencil
    static constexpr int kRingA = 2 * T;
    static constexpr int kPw = AXIS == 0 ? 1 : 32 / T;
    static constexpr int kPad = AXIS == 0 ? 0 : kPw;
    static constexpr int kStA = AXIS == 0 ? P * kRingA : kRingA * (P + kPad);  // elements per field
    static constexpr int kStF = AXIS == 0 ? P * kRing : kRing * (P + kPad);
    static_assert(kMain % 32 == 0, "whole warps");
    static_assert(T >= 8 && (T & (T - 1)) == 0, "T: a power of two >= 8 (window halos)");
    static_assert(AXIS != 0 || T == 32, "x: one pencil window per warp");
    static_assert(AXIS == 0 || (P == 16 && 32 % T == 0 && P % (32 / T) == 0), "y/z: 16 pencils, 128-byte rows");
    static_assert((kW * 8) % 1024 == 0, "window buffers on 1024-byte boundaries");

    // Ring slot of cell `cell` of a window whose group starts at ring
    // offset `ro` (a multiple of T: the position of the group's first window
    // in the CTA's sequence of windows, modulo 4 windows), so that window s
    // of the sequence fills slot s mod 4 whatever group it belongs to.
    // State ring (TMA destination): x [slot window][pencil][T]; y/z one
    // swizzled 128-byte row of 16 pencils per slot.
    __device__ __forceinline__ static int st(int cell, int tp, int ro) {
        const int s = (cell + 4 + ro) & (kRing - 1);
        if (AXIS == 0) return (s / T) * kW + tp * T + (s % T);
        const int i = s * P + tp;
        return i ^ (((i >> 4) & 7) << 1);
    }
    template <int RING>
    __device__ __forceinline__ static int ring(int cell, int tp, int ro) {
        const int s = (cell + 4 + ro) & (RING - 1);
        if (AXIS == 0) return tp * RING + s;
        return s * (P + kPad) + tp;
    }
    __device__ __forceinline__ static int ai(int cell, int tp, int ro) { return ring<kRingA>(cell, tp, ro); }
    __device__ __forceinline__ static int fi(int cell, int tp, int ro) { return ring<kRing>(cell, tp, ro); }
    // load / update layout: cell offset and pencil of main thread t
    __device__ __forceinline__ static int lcell(int t) { return AXIS == 0 ? t % T : t / P; }
    __device__ __forceinline__ static int lpencil(int t) { return AXIS == 0 ? t / T : t % P; }
    // stages A, B, C1
    __device__ __forceinline__ static int wcell(int t) { return AXIS == 0 ? t % T : (t & 31) / kPw; }
    __device__ __forceinline__ static int wpencil(int t) {
        return AXIS == 0 ? t / T : (t >> 5) * kPw + (t & 31) % kPw;
    }
};

template <int AXIS, int P, int T, int NW, class Policy>
struct WsSmem {
    using R = typename Policy::R;
    using L = WsLayout<AXIS, P, T, NW>;
    double st[5][4 * L::kW];          // state ring (TMA destination), FP64
    FaceT<Policy> rs[5][L::kStF];     // right state of a face, then its Riemann solution
    R ls[5][L::kStF];                 // traced left state of face c+1, at the slot of cell c
    R sl[5][L::kStA];                 // ajside slopes
    R d2[L::kStA];                    // dda second difference of rho
    unsigned char pf[L::kStA];        // flattening flag of the pair (c, c+1)
    double sv[5][3 * P];              // original values of cells 0..2
    unsigned short nq[2][3][L::kW];   // Newton faces of a window (by classifying thread), 3 buckets
    unsigned short cq[3][L::kW];      // closed-form faces of the current window
    int nqcnt[2][3];
    int ntake[2];                     // Newton faces of a window taken so far (chunks of 32)
    int cqcnt[2][3];
    uint64_t full[4];                 // TMA of a ring window complete
    uint64_t nready[2];               // Newton faces of a window queued
    uint64_t ndone[2];                // Newton faces of a window solved
    int abort;                        // a role gave up a wait (every wait polls it)
    unsigned long long red[128];
};

struct WsArgs {
    CUtensorMap tm[5];   // the five fields of the sweep (its order p, rho, u, v, w)
    SweepArgs a;
    long long ngroups;   // pencil groups of P pencils
    int wpg;             // windows per group
};

// Window s of a CTA: its pencil group and its place in the group.
struct WsWin {
    long long pid0;  // first pencil of the group
    int w;           // window of the group
    int b;           // first cell: -4 + w T
    bool tma;        // inside [0, N): loaded by TMA
    int ro;          // ring offset of the group (WsLayout::st)
};
template <int P, int T>
__device__ __forceinline__ WsWin ws_window(long long s, int wpg, int N) {
    WsWin W;
    const long long j = s / wpg;
    W.w = (int)(s - j * wpg);
    W.pid0 = ((long long)blockIdx.x + j * gridDim.x) * P;
    W.b = -4 + W.w * T;
    W.tma = W.w >= 1 && W.b + T <= N;
    W.ro = (int)((s - W.w) & 3) * T;
    return W;
}

template <int AXIS, int P, int T, int NW, class Policy, int MINB>
__global__ void __launch_bounds__(WsLayout<AXIS, P, T, NW>::kThreads, MINB)
    ppm_sweep_ws_kernel(const __grid_constant__ WsArgs wa) {
    using R = typename Policy::R;
    using Pow = typename Policy::Pow;
    using CT = typename Policy::CT;
    using DivD = typename Policy::DivD;
    using L = WsLayout<AXIS, P, T, NW>;
    using Smem = WsSmem<AXIS, P, T, NW, Policy>;
    extern __shared__ __align__(1024) unsigned char ws_smem_raw[];
    // 1024-byte alignment of the swizzled TMA destination
    unsigned char* base = ws_smem_raw + ((1024 - (smem_u32(ws_smem_raw) & 1023)) & 1023);
    Smem& S = *reinterpret_cast<Smem*>(base);

    const SweepArgs& a = wa.a;
    if (a.ctl->done) return;  // told >= tstop: the time loop has ended (main.F90:100)
    const int tid = threadIdx.x;
    const int N = a.nsweep;
    const Consts k = a.k;
    const StepScalars sc = a.ctl->s;
    const R dt_ = R(sc.dt), rat_ = R(sc.rat), dat_ = R(sc.dat), at_ = R(sc.at);
    const R dx_ = R(KT<R>::dx(k)), gam_ = R(KT<R>::gamma(k)), flatv_ = R(KT<R>::flat(k)), ming_ = R(KT<R>::ming(k));
    const TraceScalars<R> ts{dt_, rat_, dat_, at_, dx_, gam_, flatv_};
    const double rmin0 = dkey_decode(a.ctl->rho_key[a.bslot][0]);
    const double rmax0 = dkey_decode(a.ctl->rho_key[a.bslot][1]);
    const bool peak_possible = rmax0 > k.dmax * rmin0;
    const long long stride = axis_stride<AXIS>(a.nx, a.ny);
    const long long ncell = (long long)a.nx * a.ny * a.nz;
    // expand.F90:18-20
    const float dadt_eps = float(0.5 * sc.dat * sc.dt * sc.rat);  // dadt = 1 - dadt_eps (riemannsolver.F90:36)
    const double afact = sc.dt * (sc.dath / sc.ath);
    const double afact1 = 1.0 / (1.0 + afact);
    const double afact2 = 1.0 / (2.0 + afact);

    const long long ngroups = wa.ngroups;
    const long long mygroups =
        (long long)blockIdx.x < ngroups ? (ngroups - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const int wpg = wa.wpg;
    const long long nwin = mygroups * wpg;

    if (tid == 0) {
        for (int i = 0; i < 4; ++i) mbar_init(&S.full[i], 1);
        for (int i = 0; i < 2; ++i) {
            mbar_init(&S.nready[i], 1);
            mbar_init(&S.ndone[i], NW);
        }
        S.abort = 0;
        mbar_init_fence();
        if (blockIdx.x == 0) {  // the CTA of pencil 0: once per box and sweep
            const int reset = (a.bslot + 2) % 3;
            a.ctl->rho_key[reset][0] = kKeyPosInf;
            a.ctl->rho_key[reset][1] = kKeyNegInf;
            if (a.flags & kFlagResetSpeed) a.ctl->velmax_key = 0ULL;
        }
    }
    if (tid < 6) {
        S.nqcnt[tid / 3][tid % 3] = 0;
        S.cqcnt[tid / 3][tid % 3] = 0;
    }
    if (tid < 2) S.ntake[tid] = 0;
    __syncthreads();

    unsigned long long kmin = kKeyPosInf, kmax = 0ULL, kvel = 0ULL;
    unsigned status = 0;

    // the classifying thread's face (window base b) and pencil
    auto item_face = [&](int item, int b) { return b - 3 + L::wcell(item); };
    auto item_pencil = [&](int item) { return L::wpencil(item); };

    // Riemann problem of face f of pencil tp in window W (pattern known),
    // density-peak fix, result in place of the right state.  `which`: the
    // patterns this caller sees (the Newton group: 1, 2; the main group's
    // closed forms: 3, 4, 5), so each role holds only its solver's code.
    auto solve_face = [&](auto which, int pattern, int f, int tp, const WsWin& W) {
        const int il = L::fi(f - 1, tp, W.ro), io = L::fi(f, tp, W.ro);
        // riemannsolver.F90:279-285: the pressure floor of face f
        auto peak_floor = [&]() -> double {
            if (AXIS == 0) {
                // cells f-3 .. f of the pencil, in the reconstruction type
                // as the reference's R1 gather sees them in this path
                return peak_value(double(R(S.st[1][L::st(f - 3, tp, W.ro)])),
                                  double(R(S.st[1][L::st(f - 2, tp, W.ro)])),
                                  double(R(S.st[1][L::st(f - 1, tp, W.ro)])), double(R(S.st[1][L::st(f, tp, W.ro)])),
                                  double(R(S.st[2][L::st(f - 2, tp, W.ro)])),
                                  double(R(S.st[2][L::st(f - 1, tp, W.ro)])), k.dmax);
            } else if (f < N) {  // the transposed gather, evaluated by the pre-pass
                return a.peak[pencil_base<AXIS>(W.pid0 + tp, a.nx, a.ny) + stride * f];
            }
            return a.peak[ncell + W.pid0 + tp];
        };
        if constexpr (Policy::kFaceF32) {
            // the mixed path's FP32 faces straight from the FP32 rings (the
            // same arithmetic as the fused sweep's)
            FaceF lf, rf, of;
            lf.p = S.ls[0][il]; lf.rho = S.ls[1][il]; lf.u = S.ls[2][il]; lf.v = S.ls[3][il]; lf.w = S.ls[4][il];
            rf.p = S.rs[0][io]; rf.rho = S.rs[1][io]; rf.u = S.rs[2][io]; rf.v = S.rs[3][io]; rf.w = S.rs[4][io];
            if (riemann_mixed_f32(pattern, lf, rf, of, k, dadt_eps)) {
                if (peak_possible) of.p = float(fmax2(double(of.p), peak_floor()));
                S.rs[0][io] = of.p;
                S.rs[1][io] = of.rho;
                S.rs[2][io] = of.u;
                S.rs[3][io] = of.v;
                S.rs[4][io] = of.w;
                return;
            }
            if (pattern >= 6) pattern -= 5;  // the FP32 iteration failed: FP64
        }
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
        if (!riemann_by_pattern<Pow, typename Policy::RareT, typename Policy::PowRare, decltype(which)::value>(
                pattern, left, rgt, out, k, sc))
            status |= kStatNewton;
        if (peak_possible) out.p = fmax2(out.p, peak_floor());
        S.rs[0][io] = FaceT<Policy>(out.p);
        S.rs[1][io] = FaceT<Policy>(out.rho);
        S.rs[2][io] = FaceT<Policy>(out.u);
        S.rs[3][io] = FaceT<Policy>(out.v);
        S.rs[4][io] = FaceT<Policy>(out.w);
    };

    // Solve chunks of 32 Newton faces of window W (queue row k) until the
    // queue is drained; called by whole warps of either group (the Newton
    // warps from the window's publication on, the main warps when they reach
    // the window's update and faces remain).
    auto drain_newton = [&](int k, const WsWin& W) {
        const int lane = tid & 31;
        const int n0 = S.nqcnt[k][0], n1 = S.nqcnt[k][1], n2 = S.nqcnt[k][2];
        const int total = n0 + n1 + n2;
        for (;;) {
            int base = 0;
            if (lane == 0) base = atomicAdd(&S.ntake[k], 32);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= total) break;
            const int i = base + lane;
            if (i < total) {
                // the three Newton buckets end to end (shock + rarefaction
                // on the left, two shocks, shock + rarefaction on the right)
                int c = 0, idx = i;
                if (idx >= n0) {
                    idx -= n0;
                    c = 1;
                    if (idx >= n1) {
                        idx -= n1;
                        c = 2;
                    }
                }
                // bit 15 of the item: a weak face (FP32 Newton, patterns 6, 7)
                const int item = S.nq[k][c][idx] & 0x7fff;
                const int pattern = pattern_of_bucket<false>(c) + ((S.nq[k][c][idx] >> 15) ? 5 : 0);
                solve_face(std::integral_constant<int, kNewtonOnly>(), pattern, item_face(item, W.b),
                           item_pencil(item), W);
            }
        }
        __syncwarp();
    };

    if (tid < L::kMain) {
        // ======================= main group =======================
        uint32_t fullph = 0;   // phase parity of full[0..3] (every main thread waits on them)
        uint32_t pending = 0;  // thread 0: ring slots with a TMA in flight
        const int tl = L::lcell(tid), tp = L::lpencil(tid);
        const int tlw = L::wcell(tid), tpw = L::wpencil(tid);
        auto issue_tma = [&](const WsWin& W, int slot) {
            uint64_t* bar = &S.full[slot];
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(bar, 5u * L::kW * 8u);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                double* dst = &S.st[q][slot * L::kW];
                if (AXIS == 0) {
                    tma_load_2d(dst, &wa.tm[q], bar, W.b, (int)W.pid0);
                } else {
                    const int x0 = (int)(W.pid0 % a.nx), t0 = (int)(W.pid0 / a.nx);
                    if (AXIS == 1) tma_load_3d(dst, &wa.tm[q], bar, x0, W.b, t0);
                    else tma_load_3d(dst, &wa.tm[q], bar, x0, t0, W.b);
                }
            }
            pending |= 1u << slot;
        };
        for (long long s = 0; s <= nwin; ++s) {
            if (s < nwin) {
                const WsWin W = ws_window<P, T>(s, wpg, N);
                const bool active = W.pid0 + tp < a.npencil;
                const bool activew = W.pid0 + tpw < a.npencil;
                const long long base = pencil_base<AXIS>(active ? W.pid0 + tp : 0, a.nx, a.ny);
                // ---------------- the state of window s ----------------
                if (!W.tma) {
                    const int e = W.b + tl;
                    if (active && e >= -4 && e <= N + 2) {
                        double v[5];
                        // cell e-N (0..2) is overwritten by the update of window
                        // (e-N+8)/T, run one window later; until then global
                        // memory holds the original value
                        const bool from_save = e >= N && W.w > (e - N + 8) / T + 1;
                        if (from_save) {
#pragma unroll
                            for (int q = 0; q < 5; ++q) v[q] = S.sv[q][(e - N) * P + tp];
                        } else {
                            const int c = e < 0 ? e + N : (e >= N ? e - N : e);
                            const long long g = base + stride * c;
#pragma unroll
                            for (int q = 0; q < 5; ++q) v[q] = a.f[q][g];
                            if (e >= 0 && e < 3) {
#pragma unroll
                                for (int q = 0; q < 5; ++q) S.sv[q][e * P + tp] = v[q];
                            }
                        }
                        const int ix = L::st(e, tp, W.ro);
#pragma unroll
                        for (int q = 0; q < 5; ++q) S.st[q][ix] = v[q];
                    }
                    // a later TMA copy overwrites these slots
                    fence_proxy_async_smem();
                }
                bool bad = false;
                if (W.tma) {
                    // every reader waits for the copy itself (acquire)
                    const int slot = (int)(s & 3);
                    bad = !mbar_wait_bounded(&S.full[slot], (fullph >> slot) & 1u, &S.abort);
                    fullph ^= 1u << slot;
                    if (tid == 0 && !bad) pending &= ~(1u << slot);
                }
                if (named_sync_or(1, L::kMain, bad)) {
                    if (tid == 0) {
                        status |= kStatTimeout;
                        S.abort = 1;
                    }
                    break;
                }
                // prefetch window s+1 into the slot of window s-3 (dead: its last
                // readers, the update of window s-2 and the Newton faces of
                // window s-2, finished before this barrier)
                if (tid == 0 && s + 1 < nwin) {
                    const WsWin W1 = ws_window<P, T>(s + 1, wpg, N);
                    if (W1.tma) issue_tma(W1, (int)((s + 1) & 3));
                }
                const int ew = W.b + tlw;
                // ---------------- A: cell c = ew-1 ----------------
                {
                    const int c = ew - 1;
                    if (activew && c >= -3 && c <= N + 1) {
                        R am[5], a0[5], ap[5], sl[5], d2;
                        bool flag;
                        const int im = L::st(c - 1, tpw, W.ro), i0 = L::st(c, tpw, W.ro), ip = L::st(c + 1, tpw, W.ro);
#pragma unroll
                        for (int q = 0; q < 5; ++q) {
                            am[q] = R(S.st[q][im]);
                            a0[q] = R(S.st[q][i0]);
                            ap[q] = R(S.st[q][ip]);
                        }
                        slopes_of_cell<R>(am, a0, ap, ming_, dx_, sl, d2, flag);
                        const int ia = L::ai(c, tpw, W.ro);
#pragma unroll
                        for (int q = 0; q < 5; ++q) S.sl[q][ia] = sl[q];
                        S.d2[ia] = d2;
                        S.pf[ia] = flag ? 1 : 0;
                    }
                }
                __syncwarp();
                // ---------------- B: cell c = ew-3 ----------------
                typename FaceOf<R>::type right;
                {
                    const int c = ew - 3;
                    if (activew && c >= -1 && c <= N) {
                        const bool fl_any = S.pf[L::ai(c - 2, tpw, W.ro)] | S.pf[L::ai(c - 1, tpw, W.ro)] | S.pf[L::ai(c, tpw, W.ro)] |
                                            S.pf[L::ai(c + 1, tpw, W.ro)];
                        R q1[5], q2[5], q3[5], dm[5], d0[5], dp[5], left[5];
                        const int s1 = L::st(c - 1, tpw, W.ro), s2 = L::st(c, tpw, W.ro), s3 = L::st(c + 1, tpw, W.ro);
                        const int a1 = L::ai(c - 1, tpw, W.ro), a2 = L::ai(c, tpw, W.ro), a3 = L::ai(c + 1, tpw, W.ro);
#pragma unroll
                        for (int q = 0; q < 5; ++q) {
                            q1[q] = R(S.st[q][s1]);
                            q2[q] = R(S.st[q][s2]);
                            q3[q] = R(S.st[q][s3]);
                            dm[q] = S.sl[q][a1];
                            d0[q] = S.sl[q][a2];
                            dp[q] = S.sl[q][a3];
                        }
                        trace_cell<R, false, false>(q1, q2, q3, dm, d0, dp, S.d2[a1], S.d2[a3], fl_any, R(0), R(0),
                                                    R(0), R(0), R(0), R(0), ts, left, right);
                        const int io = L::fi(c, tpw, W.ro);
#pragma unroll
                        for (int q = 0; q < 5; ++q) S.ls[q][io] = left[q];
                    }
                }
                __syncwarp();
                // ---------------- C1: face f = ew-3 ----------------
                {
                    const int f = ew - 3;
                    int bucket = 0;  // 1 + bucket of the face, 0: no face
                    bool weak = false;
                    if (activew && f >= 0 && f <= N) {
                        const int io = L::fi(f, tpw, W.ro);
                        S.rs[0][io] = FaceT<Policy>(right.p);
                        S.rs[1][io] = FaceT<Policy>(right.rho);
                        S.rs[2][io] = FaceT<Policy>(right.u);
                        S.rs[3][io] = FaceT<Policy>(right.v);
                        S.rs[4][io] = FaceT<Policy>(right.w);
                        const int il = L::fi(f - 1, tpw, W.ro);
                        CT cl, cr;
                        const CT pl = CT(S.ls[0][il]), pr = CT(right.p);
                        const CT rl = CT(S.ls[1][il]), rr = CT(right.rho), ul = CT(S.ls[2][il]), ur = CT(right.u);
                        int pattern = riemann_classify<CT, typename Policy::PowC>(pl, pr, rl, rr, ul, ur, cl, cr, k);
                        pattern = solver_pattern<Policy::kWeakNewton>(pattern, float(pl), float(pr), float(rl),
                                                                      float(rr), float(ul), float(ur), float(cl),
                                                                      float(cr));
                        // the weak faces share the Newton queue rows of
                        // patterns 1, 2, marked in bit 15 of their item
                        weak = pattern > 5;
                        bucket = bucket_of<false>(weak ? pattern - 5 : pattern, pl >= pr);
                    }
                    const int lane = tid & 31;
                    const unsigned peers = __match_any_sync(0xffffffffu, bucket);
                    const int leader = __ffs(peers) - 1;
                    int* cnt = bucket == 0 ? nullptr
                                           : (bucket <= 3 ? &S.nqcnt[s & 1][bucket - 1] : &S.cqcnt[s & 1][bucket - 4]);
                    int off = 0;
                    if (bucket && lane == leader) off = atomicAdd(cnt, __popc(peers));
                    off = __shfl_sync(0xffffffffu, off, leader);
                    if (bucket) {
                        const int slotq = off + __popc(peers & ((1u << lane) - 1u));
                        if (bucket <= 3) S.nq[s & 1][bucket - 1][slotq] = (unsigned short)(tid | (weak ? 0x8000 : 0));
                        else S.cq[bucket - 4][slotq] = (unsigned short)tid;
                    }
                }
                named_sync(1, L::kMain);
                if (tid == 0) mbar_arrive(&S.nready[s & 1]);
                // ---------------- C2: the closed forms of window s ----------------
                {
                    int idx = tid, pattern = 0, item = 0;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const int n = S.cqcnt[s & 1][c];
                        if (pattern == 0) {
                            if (idx < n) {
                                pattern = 3 + c;
                                item = S.cq[c][idx];
                            } else {
                                idx -= n;
                            }
                        }
                    }
                    // the other row was read by the previous window's closed
                    // forms and is next filled after the next barrier
                    if (tid < 3) S.cqcnt[(s & 1) ^ 1][tid] = 0;
                    if (pattern)
                        solve_face(std::integral_constant<int, kClosedOnly>(), pattern, item_face(item, W.b),
                                   item_pencil(item), W);
                }
            }
            if (s >= 1) {
                // ---------------- D: the update of window s-1 ----------------
                const long long sp = s - 1;
                // the Newton faces of window s-1 not taken yet, then the
                // chunks still in the Newton warps
                drain_newton((int)(sp & 1), ws_window<P, T>(sp, wpg, N));
                const bool bad = !mbar_wait_bounded(&S.ndone[sp & 1], (uint32_t)((sp >> 1) & 1), &S.abort);
                if (named_sync_or(1, L::kMain, bad)) {
                    if (tid == 0) {
                        status |= kStatTimeout;
                        S.abort = 1;
                    }
                    break;
                }
                // every warp of both groups is done with window s-1's queue
                // (the Newton warps before ndone, the main warps before the
                // barrier); its row is next filled by window s+1, after the
                // next barrier
                if (tid == 0) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) S.nqcnt[sp & 1][c] = 0;
                    S.ntake[sp & 1] = 0;
                }
                const WsWin W = ws_window<P, T>(s - 1, wpg, N);
                const bool active = W.pid0 + tp < a.npencil;
                const int d = W.b - 4 + tl;
                if (active && d >= 0 && d < N) {
                    const long long g = pencil_base<AXIS>(W.pid0 + tp, a.nx, a.ny) + stride * d;
                    const int id = L::fi(d, tp, W.ro), id1 = L::fi(d + 1, tp, W.ro);
                    FaceState f1, f2;
                    f1.p = S.rs[0][id]; f1.rho = S.rs[1][id]; f1.u = S.rs[2][id]; f1.v = S.rs[3][id];
                    f1.w = S.rs[4][id];
                    f2.p = S.rs[0][id1]; f2.rho = S.rs[1][id1]; f2.u = S.rs[2][id1]; f2.v = S.rs[3][id1];
                    f2.w = S.rs[4][id1];
                    const int ic = L::st(d, tp, W.ro);
                    double p = S.st[0][ic], rho = S.st[1][ic], u = S.st[2][ic], v = S.st[3][ic], w = S.st[4][ic];
                    if (a.flags & kFlagSnapshot) {
                        // the step-start state, natural order p, vx, vy, vz
                        using SnapT = typename Policy::SnapT;
                        static_cast<SnapT*>(a.snap[0])[g] = SnapT(p);
                        static_cast<SnapT*>(a.snap[1])[g] = SnapT(AXIS == 0 ? u : (AXIS == 1 ? v : w));
                        static_cast<SnapT*>(a.snap[2])[g] = SnapT(AXIS == 0 ? v : (AXIS == 1 ? u : v));
                        static_cast<SnapT*>(a.snap[3])[g] = SnapT(AXIS == 0 ? w : (AXIS == 1 ? w : u));
                    }
                    // total() with the natural component order (ppmsolver.F90:149,277,405)
                    double etot;
                    if (AXIS == 2) etot = total_energy(p, rho, w, v, u, k.rgamma1);
                    else etot = total_energy(p, rho, u, v, w, k.rgamma1);
                    const double eint = p * k.rgamma1;
                    integrate<false, DivD>(f1, f2, p, rho, u, v, w, etot, eint, k, sc, 0.0);
                    finish_cell<AXIS, typename Policy::SnapT>(a, g, p, rho, u, v, w, afact, afact1, afact2, kmin, kmax, kvel,
                                                              status);
                }
            }
        }
        if (tid == 0) {
            // on an early end: wait (bounded) for the copies still in flight
            // before the CTA's shared memory goes away
            const int never = 0;
            for (int slot = 0; slot < 4; ++slot)
                if (pending & (1u << slot)) {
                    mbar_wait_bounded(&S.full[slot], (fullph >> slot) & 1u, &never);
                    fullph ^= 1u << slot;
                }
        }
    } else {
        // ======================= Newton group =======================
        const int lane = tid & 31;
        for (long long s = 0; s < nwin; ++s) {
            // every lane waits (acquire of the queue); the warp decides together
            const bool ok = mbar_wait_bounded(&S.nready[s & 1], (uint32_t)((s >> 1) & 1), &S.abort);
            if (!__all_sync(0xffffffffu, ok)) {
                status |= kStatTimeout;
                if (lane == 0) S.abort = 1;
                break;
            }
            drain_newton((int)(s & 1), ws_window<P, T>(s, wpg, N));
            const bool withhold = s == 0 && (a.flags & kFlagTestWithhold);
            if (lane == 0 && !withhold) mbar_arrive(&S.ndone[s & 1]);
        }
    }
    block_flush(kmin, kmax, kvel, status, &a.ctl->rho_key[(a.bslot + 1) % 3][0],
                &a.ctl->rho_key[(a.bslot + 1) % 3][1], (a.flags & kFlagSpeed) ? &a.ctl->velmax_key : nullptr,
                &a.ctl->status, S.red);
}

}  // namespace hp
