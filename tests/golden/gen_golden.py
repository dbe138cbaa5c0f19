"""Second, independent restatement of the STENCIL ppmsolver (and of the
non-STENCIL build's full-pencil ppm()) in plain Python, used to generate
golden vectors that pin the C oracle.

The reference (Fortran 90 + OpenACC) cannot be compiled here and ships no
test vectors, so this file transliterates the same routines a second time,
straight from the Fortran, with Python floats (IEEE binary64, one rounding
per operation, ``**`` -> C ``pow``).  Two codings that agree bit for bit
guard against transcription slips in either.  Arrays are 1-based dicts of
Fortran indices to keep the transliteration literal.

    python tests/golden/gen_golden.py      # rewrites tests/golden/*.npz

Sources: hydro/ppmsolver.F90:96-160,214-288,342-416; order2interp.F90;
ppm_functs.F90; dda.F90; riemannsolver.F90; riemann.F90; integrate.F90;
total.F90; internal.F90; for the pencil cases ppm.F90, flatten5.F90 and
ppmsolver.F90:162-190,290-318,418-446.
"""
from __future__ import annotations

import os

import numpy as np

F4 = lambda s: float(np.float32(s))  # REAL(4) literal promoted to REAL(8)
C16, C13, TINY, TERR = F4("0.16666667"), F4("0.33333333"), F4("1e-15"), F4("1e-3")
C010, C050 = F4("0.010"), F4("0.050")


class Sc:
    """Module `scalar` values."""

    def __init__(self, gamma, dx, dt, at, dat, ath, mingradflat=0.25, flatvalue=0.15, dmax=2e10, eta1=1e-3,
                 eta2=0.1):
        self.gamma = gamma
        self.rgamma = 1.0 / gamma
        self.gamma1 = (gamma + 1.0) / (gamma - 1.0)
        self.rgamma1 = 1.0 / (gamma - 1)
        self.m = (gamma - 1.0) / (2.0 * gamma)
        self.rm = 1.0 / self.m
        self.gf = (gamma + 1.0) / (2.0 * gamma)
        self.dx, self.rdx = dx, 1.0 / dx
        self.dt, self.at, self.dat, self.rat = dt, at, dat, 1.0 / at
        self.rdtath = dt / ath
        self.mingradflat, self.flatvalue, self.dmax, self.eta1, self.eta2 = mingradflat, flatvalue, dmax, eta1, eta2


def MIN(*a):
    r = a[0]
    for b in a[1:]:
        if b < r:
            r = b
    return r


def MAX(*a):
    r = a[0]
    for b in a[1:]:
        if b > r:
            r = b
    return r


def ajside(am1, a, ap1):
    if (ap1 - a) * (a - am1) > 0.0:
        da = 0.50 * (ap1 - am1)
        return MIN(abs(da), 2.0 * abs(a - am1), 2.0 * abs(ap1 - a)) * da / abs(da)
    return 0.0


def fl(ajr, d, a6, y, S):
    x = y / S.dx
    return ajr[1] - 0.50 * x * (d[1] - (1.0 - 2.0 * x * C13) * a6[1])


def fr(ajl, d, a6, y, S):
    x = y / S.dx
    return ajl[2] + 0.50 * x * (d[2] + (1.0 - 2.0 * x * C13) * a6[2])


def beta(ct, ut, uc, pt, pc, gc, sign, S):
    gvc = (-gc + S.dat * uc) * S.rat
    return -(sign * ((ut - uc) + sign * (pt - pc) / ct + sign * S.dt * (2.0 * S.dat * pc / (ct * S.at)) + S.dt * gvc)
             / (2 * ct))


def beta0(ct, rhot, rhoc, pt, pc, S):
    return (pt - pc) / (ct * ct) + 1.0 / rhot - 1.0 / rhoc + (2.0 * S.dat * pc) / (S.at * ct * ct) * S.dt


def dda(a, dmalf, dmarg, S):
    deltam2 = C16 * (a[3] - 2.0 * a[2] + a[1]) / (S.dx * S.dx)
    deltap2 = C16 * (a[5] - 2.0 * a[4] + a[3]) / (S.dx * S.dx)
    agrad = abs(a[4] - a[2]) - C010 * MIN(abs(a[4]), abs(a[2]))
    if -(deltam2 * deltap2) > 0.0 and agrad > 0.0:
        eta = -((deltap2 - deltam2) * S.dx * S.dx / (a[4] - a[2]))
        eta = MAX(0.0, MIN(20.0 * (eta - C050), 1.0))
    else:
        eta = 0.0
    return eta, a[2] + 0.50 * dmalf, a[4] - 0.50 * dmarg


def correction(addp, addrho, a, ajl, ajr, d, a6, ccc, vi, vip1, flat, ndda, S):
    dmaj = ajside(a[1], a[2], a[3])
    dmajp1 = ajside(a[2], a[3], a[4])
    dmajp2 = ajside(a[3], a[4], a[5])
    ajl[2] = a[2] + 0.50 * (a[3] - a[2]) + (dmaj - dmajp1) * C16
    ajr[2] = a[3] + 0.50 * (a[4] - a[3]) + (dmajp1 - dmajp2) * C16
    if ndda == 1 and addrho >= addp:
        eta, ajld, ajrd = dda(a, dmaj, dmajp2, S)
        ajl[2] = (1.0 - eta) * ajl[2] + eta * ajld
        ajr[2] = (1.0 - eta) * ajr[2] + eta * ajrd
    d[2] = ajr[2] - ajl[2]
    a6[2] = 6 * (a[3] - 0.50 * (ajl[2] + ajr[2]))
    if (ajr[2] - a[3]) * (a[3] - ajl[2]) <= 0:
        ajl[2] = a[3]
        ajr[2] = a[3]
    elif d[2] * a6[2] > d[2] * d[2]:
        ajl[2] = 3.0 * a[3] - 2.0 * ajr[2]
    elif d[2] * a6[2] < -(d[2] * d[2]):
        ajr[2] = 3.0 * a[3] - 2.0 * ajl[2]
    ajl[2] = flat * a[3] + (1.0 - flat) * ajl[2]
    ajr[2] = flat * a[3] + (1.0 - flat) * ajr[2]
    d[2] = ajr[2] - ajl[2]
    a6[2] = 6 * (a[3] - 0.50 * (ajl[2] + ajr[2]))
    atl = fl(ajr, d, a6, MAX(S.dt * (vi + ccc[1]) * S.rat, 0.0), S)
    atr = fr(ajl, d, a6, MAX(-(S.dt * (vip1 - ccc[2]) * S.rat), 0.0), S)
    acl = {1: fl(ajr, d, a6, S.dt * (vi - ccc[1]) * S.rat, S), 2: fl(ajr, d, a6, S.dt * vi * S.rat, S),
           3: fl(ajr, d, a6, S.dt * (vi + ccc[1]) * S.rat, S)}
    acr = {1: fr(ajl, d, a6, -(S.dt * (vip1 - ccc[2]) * S.rat), S), 2: fr(ajl, d, a6, -(S.dt * vip1 * S.rat), S),
           3: fr(ajl, d, a6, -(S.dt * (vip1 + ccc[2]) * S.rat), S)}
    return atl, atr, acl, acr


def order2interp(pres, rho, vx, vy, vz, g, c, S):
    nmin, nmax = 3, 4
    z0 = np.float64(0.0)
    slots = {k: tuple({1: z0, 2: z0} for _ in range(4)) for k in range(6)}
    gradleft = 0.0
    out = None
    for i in range(nmin, nmax + 1):
        mi = i - nmin + 1
        flat = 0.0
        cbar = {1: c[i - 1], 2: c[i]}
        for arr in (pres, rho, vx, vy, vz):
            gradmax = 0.0
            for ii in range(1, 5):
                ic = mi + ii
                if arr[ic] * arr[ic - 1] != 0.0:
                    gradleft = abs((arr[ic] - arr[ic - 1]) / MIN(arr[ic], arr[ic - 1]))
                gradmax = MAX(gradmax, gradleft)
            if gradmax >= S.mingradflat:
                flat = S.flatvalue
        for k in range(6):
            for sl in slots[k]:
                sl[1] = sl[2]
        addp = abs(pres[i + 1] - pres[i - 1]) / MIN(pres[i - 1], pres[i + 1])
        addrho = 0.50 * S.gamma * abs(rho[i + 1] - rho[i - 1]) / MIN(rho[i - 1], rho[i + 1])
        res = []
        for k, (arr, nd) in enumerate(((pres, 0), (rho, 1), (vx, 0), (vy, 0), (vz, 0), (g, 0))):
            a = {j: arr[mi + j - 1] for j in range(1, 6)}
            ajl, ajr, d, a6 = slots[k]
            res.append(correction(addp, addrho, a, ajl, ajr, d, a6, cbar, vx[i - 1], vx[i], flat, nd, S))
        (ptl, ptr, pcl, pcr), (rhotl, rhotr, rhocl, rhocr), (vxtl, vxtr, vxcl, vxcr) = res[0], res[1], res[2]
        (vytl, vytr, vycl, vycr), (vztl, vztr, vzcl, vzcr), (gtl, gtr, gcl, gcr) = res[3], res[4], res[5]
        if ptl < 0.0:
            ptl = TINY
        if ptr < 0.0:
            ptr = TINY
        if rhotl < 0.0:
            rhotl = TINY
        if rhotr < 0.0:
            rhotr = TINY
        ctl = np.sqrt(S.gamma * ptl * rhotl)
        ctr = np.sqrt(S.gamma * ptr * rhotr)
        lm, l0, lp = (vx[i - 1] - cbar[1]) * S.rat, vx[i - 1] * S.rat, (vx[i - 1] + cbar[1]) * S.rat
        betaml = 0.0 if lm <= 0.0 else beta(ctl, vxtl, vxcl[1], ptl, pcl[1], gcl[1], -1.0, S)
        betapl = 0.0 if lp <= 0.0 else beta(ctl, vxtl, vxcl[3], ptl, pcl[3], gcl[3], 1.0, S)
        vyleft, vzleft = vytl, vztl
        if l0 <= 0.0:
            beta0l = 0.0
        else:
            beta0l = beta0(ctl, rhotl, rhocl[2], ptl, pcl[2], S)
            vyleft, vzleft = vycl[2], vzcl[2]
        lm, l0, lp = (vx[i] - cbar[2]) * S.rat, vx[i] * S.rat, (vx[i] + cbar[2]) * S.rat
        betapr = 0.0 if lp >= 0.0 else beta(ctr, vxtr, vxcr[3], ptr, pcr[3], gcr[3], 1.0, S)
        betamr = 0.0 if lm >= 0.0 else beta(ctr, vxtr, vxcr[1], ptr, pcr[1], gcr[1], -1.0, S)
        vyright, vzright = vytr, vztr
        if l0 >= 0.0:
            beta0r = 0.0
        else:
            beta0r = beta0(ctr, rhotr, rhocr[2], ptr, pcr[2], S)
            vyright, vzright = vycr[2], vzcr[2]
        pleft = ptl + ctl * ctl * (betapl + betaml)
        if pleft <= 0.0:
            pleft = ptl
        pright = ptr + ctr * ctr * (betapr + betamr)
        if pright <= 0.0:
            pright = ptr
        vxleft = vxtl + ctl * (betapl - betaml)
        vxright = vxtr + ctr * (betapr - betamr)
        rholeft = 1.0 / (1.0 / rhotl - betaml - beta0l - betapl)
        if rholeft <= 0.0:
            rholeft = rhotl
        rhoright = 1.0 / (1.0 / rhotr - betamr - beta0r - betapr)
        if rhoright <= 0.0:
            rhoright = rhotr
        out = (pleft, pright, rholeft, rhoright, vxleft, vxright, vyleft, vyright, vzleft, vzright)
    return out


def rarwave(f1, f2, vt, vh):
    return f2 + vt * (f1 - f2) / (vt - vh)


def rhoshock(p2, p1, rho1, S):
    return rho1 * (S.gamma1 * p2 / p1 + 1.0) / (S.gamma1 + p2 / p1)


def riemann(pstar, pl, pr, rl, rr, ul, ur, S):
    err, nnewt = 1.e10, 0
    kappa = np.sqrt(S.gamma * (pl + pr) * (rl + rr) * 0.25)
    pcheck = 0.50 * (pl + pr) + 0.50 * kappa * (ul + ur)
    if pcheck > 0:
        pstar = pcheck
    vstar = float("nan")
    while err > TERR:
        nnewt += 1
        if nnewt > 100:
            raise RuntimeError("convergenza non raggiunta")
        pold = pstar
        cl = np.sqrt(S.gamma * pl * rl)
        cr = np.sqrt(S.gamma * pr * rr)
        pst = 1.0 - (pstar / pl) ** S.m
        if pstar >= pl:
            a = cl * np.sqrt(S.gf * pstar / pl + S.m)
        elif pst == 0.0:
            a = cl * np.sqrt(S.gf * pstar / pl + S.m)
        else:
            a = S.m * cl * (1.0 - pstar / pl) / (1 - (pstar / pl) ** S.m)
        pst = 1.0 - (pstar / pr) ** S.m
        if pstar >= pr:
            b = cr * np.sqrt(S.gf * pstar / pr + S.m)
        elif pst == 0.0:
            b = cr * np.sqrt(S.gf * pstar / pr + S.m)
        else:
            b = S.m * cr * (1.0 - pstar / pr) / (1 - (pstar / pr) ** S.m)
        vpl = -((a * a + cl * cl) / (2 * a * a * a)) if pstar >= pl else -((1.0 / cl) * (pstar / pl) ** (-S.gf))
        vpr = (b * b + cr * cr) / (2 * b * b * b) if pstar >= pr else (1.0 / cr) * (pstar / pr) ** (-S.gf)
        vsl = ul - (pstar - pl) / a
        vsr = ur + (pstar - pr) / b
        pstar = pstar - (vsl - vsr) / (vpl - vpr)
        if pstar <= 0:
            pstar = pold / 1000.0
        vstar = (pl - pr + a * ul + b * ur) / (a + b)
        err = abs(pold - pstar) / pold
    return pstar, vstar


# Faces per wave pattern of the last generated case: two shocks, shock +
# rarefaction, two rarefactions, vacuum (the branch order below), then the
# two-shock and shock + rarefaction faces that are strong (a pressure jump
# above 100 or streams colliding faster than cL + cR).
TALLY = [0] * 6


def _tally(dvv, dv2s, dv1s, dv2r, p1, p2, csum):
    if dvv >= dv2s:
        pat = 0
    elif dvv >= dv1s:
        pat = 1
    elif dvv > dv2r:
        pat = 2
    elif dvv <= dv2r:
        pat = 3
    else:
        return
    TALLY[pat] += 1
    if pat < 2 and (p2 > 100.0 * p1 or dvv > csum):
        TALLY[4 + pat] += 1


def riemannsolver(rhobar, vxbar, pl, pr, rl, rr, ul, ur, vl, vr, wl, wr, S):
    g = S.gamma
    cleft = np.sqrt(g * pl / rl)
    cright = np.sqrt(g * pr / rr)
    dadt = 1.0 - 0.5 * S.dat * S.dt * S.rat
    if pl <= pr:
        p1, p2, rho1, c1, c2 = pl, pr, rl, cleft, cright
    else:
        p1, p2, rho1, c1, c2 = pr, pl, rr, cright, cleft
    dvv = ul - ur
    dv2s = (p2 - p1) / np.sqrt(0.50 * rho1 * ((g - 1) * p1 + (g + 1) * p2))
    dv1s = -((2.0 * c2 / (g - 1.0)) * (1.0 - (p1 / p2) ** S.m))
    dv2r = -(2.0 * (c1 + c2) * S.rgamma1)
    _tally(dvv, dv2s, dv1s, dv2r, p1, p2, cleft + cright)
    pm = vxm = rhom = float("nan")
    if dvv >= dv2s:
        pm, vxm = riemann(MAX(pl, pr), pl, pr, rl, rr, ul, ur, S)
        rs1, rs2 = rhoshock(pm, pl, rl, S), rhoshock(pm, pr, rr, S)
        vs1 = 0.0 if rs1 == rl else (rs1 * vxm - rl * ul) / (rs1 - rl)
        vs2 = 0.0 if rs2 == rr else (rs2 * vxm - rr * ur) / (rs2 - rr)
        if vs2 < 0.0:
            pm, vxm, rhom = pr, ur, rr
        elif vxm <= 0.0 and vs2 >= 0.0:
            rhom = rs2
        elif vs1 <= 0.0 and vxm > 0.0:
            rhom = rs1
        else:
            pm, vxm, rhom = pl, ul, rl
    elif dvv < dv2s and dvv >= dv1s:
        pm = ((cleft + cright + (ul - ur) * (g - 1) * 0.5) / (cleft / pl ** S.m + cright / pr ** S.m)) ** S.rm
        pm, vxm = riemann(pm, pl, pr, rl, rr, ul, ur, S)
        if pl >= pr:
            rs2 = rhoshock(pm, pr, rr, S)
            rc1 = rl * (pm / pl) ** S.rgamma
            vs2 = 0.0 if rs2 == rr else (rs2 * vxm - rr * ur) / (rs2 - rr)
            vt1 = vxm - np.sqrt(g * pm / rc1)
            vh1 = ul - cleft
            if vs2 < 0:
                pm, vxm, rhom = pr, ur, rr
            elif vh1 >= 0.0:
                pm, vxm, rhom = pl, ul, rl
            elif vxm <= 0.0 and vs2 >= 0:
                rhom = rs2
            elif vxm > 0.0 and vt1 <= 0.0:
                rhom = rc1
            elif vt1 > 0.0 and vh1 <= 0.0:
                pm, rhom, vxm = rarwave(pl, pm, vt1, vh1), rarwave(rl, rc1, vt1, vh1), rarwave(ul, vxm, vt1, vh1)
        else:
            rs1 = rhoshock(pm, pl, rl, S)
            rc2 = rr * (pm / pr) ** S.rgamma
            vs1 = 0.0 if rs1 == rl else (rs1 * vxm - rl * ul) / (rs1 - rl)
            vt2 = vxm + np.sqrt(g * pm / rc2)
            vh2 = ur + cright
            if vs1 > 0:
                pm, vxm, rhom = pl, ul, rl
            elif vh2 <= 0.0:
                pm, vxm, rhom = pr, ur, rr
            elif vxm >= 0.0 and vs1 <= 0.0:
                rhom = rs1
            elif vxm < 0.0 and vt2 >= 0.0:
                rhom = rc2
            elif vt2 < 0.0 and vh2 >= 0.0:
                pm, rhom, vxm = rarwave(pr, pm, vt2, vh2), rarwave(rr, rc2, vt2, vh2), rarwave(ur, vxm, vt2, vh2)
    elif dvv < dv1s and dvv > dv2r:
        zeta = (cright / cleft) * (pl / pr) ** S.m
        vtl = ul + 2.0 * cleft * S.rgamma1
        vtr = ur - 2.0 * cright * S.rgamma1
        vxm = (vtl * zeta + vtr) / (1.0 + zeta)
        pm = pl * ((g - 1) * (vtl - vtr) / (2.0 * cleft * (1.0 + zeta))) ** S.rm
        rc1 = rl * (pm / pl) ** S.rgamma
        rc2 = rr * (pm / pr) ** S.rgamma
        vt2, vh2 = vxm + np.sqrt(g * pm / rc2), ur + cright
        vt1, vh1 = vxm - np.sqrt(g * pm / rc1), ul - cleft
        if vh2 <= 0.0:
            pm, vxm, rhom = pr, ur, rr
        elif vh1 >= 0.0:
            pm, vxm, rhom = pl, ul, rl
        elif vh2 > 0.0 and vt2 <= 0.0:
            pm, rhom, vxm = rarwave(pr, pm, vt2, vh2), rarwave(rr, rc2, vt2, vh2), rarwave(ur, vxm, vt2, vh2)
        elif vxm <= 0.0 and vt2 > 0.0:
            rhom = rc2
        elif vxm > 0.0 and vt1 <= 0.0:
            rhom = rc1
        elif vt1 > 0.0 and vh1 <= 0.0:
            pm, rhom, vxm = rarwave(pl, pm, vt1, vh1), rarwave(rl, rc1, vt1, vh1), rarwave(ul, vxm, vt1, vh1)
    elif dvv <= dv2r:
        pm = vxm = rc1 = rc2 = 0.0
        vt2, vh2 = ur - 2.0 * cright * S.rgamma1, ur + cright
        vt1, vh1 = ul - 2.0 * cleft * S.rgamma1, ul - cleft
        if vh2 <= 0.0:
            pm, vxm, rhom = pr, ur, rr
        elif vh1 >= 0.0:
            pm, vxm, rhom = pl, ul, rl
        elif vh2 > 0.0 and vt2 <= 0.0:
            pm, rhom, vxm = rarwave(pr, pm, vt2, vh2), rarwave(rr, rc2, vt2, vh2), rarwave(ur, vxm, vt2, vh2)
        elif vt1 <= 0.0 and vt2 > 0.0:
            rhom = 0.0
        elif vt1 > 0.0 and vh1 <= 0.0:
            pm, rhom, vxm = rarwave(pl, pm, vt1, vh1), rarwave(rl, rc1, vt1, vh1), rarwave(ul, vxm, vt1, vh1)
    if vxm >= 0.0:
        vym, vzm = dadt * vl, dadt * wl
    else:
        vym, vzm = dadt * vr, dadt * wr
    if rhobar[2] > S.dmax * rhobar[1] and rhobar[3] > S.dmax * rhobar[4]:
        maxp = (vxbar[2] - vxbar[3]) * MAX(rhobar[2], rhobar[3]) * MAX(0.0, vxbar[2] - vxbar[3])
        pm = MAX(pm, maxp)
    return pm, rhom, vxm, vym, vzm


# Cells per dual-energy branch of the last generated case: the new internal
# energy from total minus kinetic (eeaux / etot >= eta2), the pressure from
# it (eta1 <= ratio < eta2), the pressure from the separately advected
# internal energy (ratio < eta1).
DUAL = [0] * 3


def integrate(f1, f2, pres, rho, vx, vy, vz, etot, eint, ghalf, S):
    pm1, rhom1, vxm1, vym1, vzm1 = f1
    pm2, rhom2, vxm2, vym2, vzm2 = f2
    g = S.gamma
    fl1, fl2 = rhom1 * vxm1, rhom2 * vxm2
    rhonew = rho + S.rdtath * (fl1 - fl2) * S.rdx
    fl1, fl2 = rhom1 * vxm1 * vxm1 + pm1, rhom2 * vxm2 * vxm2 + pm2
    grav = (rho + rhonew) * ghalf * 0.5
    vxnew = (vx * rho + S.rdtath * (fl1 - fl2) * S.rdx + S.rdtath * grav) / rhonew
    fl1, fl2 = vym1 * vxm1 * rhom1, vym2 * vxm2 * rhom2
    vynew = (rho * vy + S.rdtath * (fl1 - fl2) * S.rdx) / rhonew
    fl1, fl2 = vzm1 * vxm1 * rhom1, vzm2 * vxm2 * rhom2
    vznew = (rho * vz + S.rdtath * (fl1 - fl2) * S.rdx) / rhonew
    fl1 = (g * pm1 * S.rgamma1 + 0.50 * rhom1 * (vxm1 * vxm1 + vym1 * vym1 + vzm1 * vzm1)) * vxm1
    fl2 = (g * pm2 * S.rgamma1 + 0.50 * rhom2 * (vxm2 * vxm2 + vym2 * vym2 + vzm2 * vzm2)) * vxm2
    grav = (rho * vx + rhonew * vxnew) * ghalf * 0.5
    etotnew = etot + S.rdtath * (fl1 - fl2) * S.rdx + S.rdtath * grav
    pmean = (pm1 + pm2) * 0.5  # undefined in the STENCIL build; ppm.F90:583
    eintnew = eint + S.rdtath * pmean * (vxm1 - vxm2) * S.rdx
    fl1, fl2 = (pm1 * vxm1) * S.rgamma1, (pm2 * vxm2) * S.rgamma1
    eintnew = eintnew + S.rdtath * (fl1 - fl2) * S.rdx
    if eintnew < 0:
        eintnew = eint
    vvv = vxnew * vxnew + vynew * vynew + vznew * vznew
    eeaux = etotnew - 0.50 * rhonew * vvv
    if eeaux / etotnew >= S.eta2:
        eintnew = eeaux
    pnew = (g - 1) * eeaux if eeaux / etotnew >= S.eta1 else (g - 1) * eintnew
    DUAL[0 if eeaux / etotnew >= S.eta2 else (1 if eeaux / etotnew >= S.eta1 else 2)] += 1
    if eintnew <= 0.0:
        pnew = pres
    if rhonew <= 0.:
        rhonew = rho
    return pnew, rhonew, vxnew, vynew, vznew


def ppmsolver(F, nb, nd, S, G=None):
    """One STENCIL sweep on ghosted fields F = [p, rho, vx, vy, vz] (numpy,
    Fortran order); returns updated copies.  G: ghosted gforce(3, nx, ny,
    nz) or None (gravity off: g = -0.0)."""
    p3d, r3d, u3d, v3d, w3d = [a.copy(order="F") for a in F]
    nx, ny, nz = p3d.shape
    A = lambda arr, i, j, k: arr[i - 1, j - 1, k - 1]  # Fortran 1-based
    if nd == 1:
        ns, t1r, t2r = nx, range(nb + 1, ny - nb + 1), range(nb + 1, nz - nb + 1)
        cell = lambda s, a, b: (s, a, b)
        roles = (u3d, v3d, w3d)
    elif nd == 2:
        ns, t1r, t2r = ny, range(nb + 1, nx - nb + 1), range(nb + 1, nz - nb + 1)
        cell = lambda s, a, b: (a, s, b)
        roles = (v3d, u3d, w3d)
    else:
        ns, t1r, t2r = nz, range(nb + 1, nx - nb + 1), range(nb + 1, ny - nb + 1)
        cell = lambda s, a, b: (a, b, s)
        roles = (w3d, v3d, u3d)
    faces = {}
    for b in t2r:
        for a in t1r:
            for i in range(nb + 1, ns - nb + 2):
                pr_, rh, vx_, vy_, vz_, g_, c_ = {}, {}, {}, {}, {}, {}, {}
                for ip in range(1, 7):
                    q = cell(i + ip - 4, a, b)
                    pr_[ip], rh[ip] = A(p3d, *q), A(r3d, *q)
                    vx_[ip], vy_[ip], vz_[ip] = A(roles[0], *q), A(roles[1], *q), A(roles[2], *q)
                    g_[ip] = np.float64(-0.0) if G is None else -A(G[nd - 1], *q)
                    c_[ip] = np.sqrt(S.gamma * pr_[ip] / rh[ip])
                faces[(i, a, b)] = order2interp(pr_, rh, vx_, vy_, vz_, g_, c_, S)
    flux = {}
    for b in t2r:
        for a in t1r:
            for i in range(nb + 1, ns - nb + 2):
                # density-peak gather: rho3d(iaux, j, k) with the x-index slot
                # (Fortran storage: a first index beyond its extent runs into
                # the next column; beyond the allocation the test is false)
                rb, vb = {}, {}
                rflat, vflat = r3d.ravel(order="F"), roles[0].ravel(order="F")
                for ip in range(1, 7):
                    ia = i + ip - 4
                    q = (ia, a, b) if nd in (1, 2) else (ia, b, a)
                    lin = (q[0] - 1) + nx * ((q[1] - 1) + ny * (q[2] - 1))
                    if 0 <= lin < rflat.size:
                        rb[ip], vb[ip] = rflat[lin], vflat[lin]
                    else:
                        rb[ip], vb[ip] = float("nan"), float("nan")
                L = faces[(i, a, b)]
                flux[(i, a, b)] = riemannsolver(rb, vb, *L, S)
    out_p, out_r = p3d.copy(order="F"), r3d.copy(order="F")
    out_u, out_v, out_w = u3d.copy(order="F"), v3d.copy(order="F"), w3d.copy(order="F")
    oroles = {1: (out_u, out_v, out_w), 2: (out_v, out_u, out_w), 3: (out_w, out_v, out_u)}[nd]
    for b in t2r:
        for a in t1r:
            for i in range(nb + 1, ns - nb + 1):
                q = cell(i, a, b)
                pz, rz = A(p3d, *q), A(r3d, *q)
                ux, uy, uz = A(u3d, *q), A(v3d, *q), A(w3d, *q)
                etot = pz * S.rgamma1 + 0.5 * rz * (ux * ux + uy * uy + uz * uz)
                eint = pz * S.rgamma1
                ghalf = -0.0 if G is None else -A(G[nd - 1], *q)
                res = integrate(flux[(i, a, b)], flux[(i + 1, a, b)], pz, rz, A(roles[0], *q), A(roles[1], *q),
                                A(roles[2], *q), etot, eint, ghalf, S)
                idx = tuple(x - 1 for x in q)
                out_p[idx], out_r[idx] = res[0], res[1]
                oroles[0][idx], oroles[1][idx], oroles[2][idx] = res[2], res[3], res[4]
    return [out_p, out_r, out_u, out_v, out_w]


# ---------------------------------------------------------------------------
# The non-STENCIL build's full-pencil solver: hydro/ppm.F90 per pencil (with
# flatten5.F90), called by ppmsolver.F90:162-190, 290-318, 418-446 on whole
# gathered lines, then savetn.  Transliterated a second time from the
# Fortran, independently of oracle/hp_oracle.c.
# ---------------------------------------------------------------------------
def flatten5(abar, keep, S):
    """flatten5.F90: 1 when the largest relative jump of the 4 pairs
    reaches mingradflat.  A zero product leaves gradleft as it was (kept in
    keep['g'] across calls; 0 at the start of the pencil)."""
    gradmax = 0.0
    for i in range(1, 5):
        ic = i + 1
        if abar[ic] * abar[ic - 1] != 0.0:
            keep["g"] = abs((abar[ic] - abar[ic - 1]) / MIN(abar[ic], abar[ic - 1]))
        gradmax = MAX(gradmax, keep["g"])
    return 1 if gradmax >= S.mingradflat else 0


def ppm_pencil(pres, rho, vx, vy, vz, c, eint, etot, cho, ngrid, nb, S):
    """ppm.F90:1-662 on one gathered line (1-based dicts over 1..ngrid);
    returns the line's new p, rho, vx, vy, vz (dicts) as the reference
    leaves them (cells nmin..nmax written)."""
    nmin, nmax = nb, ngrid - nb + 1
    nmid = nmin + 1
    z = {i: np.float64(0.0) for i in range(0, ngrid + 2)}  # IEEE division (0/0 -> NaN) at the ghosts
    pnew, rhonew, vxnew, vynew, vznew, etotnew, eintnew = (dict(z) for _ in range(7))
    z0 = np.float64(0.0)
    slots = [tuple({1: z0, 2: z0} for _ in range(4)) for _ in range(5)]
    face = {1: (0.0,) * 5, 2: (0.0,) * 5}
    keep = {"g": 0.0}
    for i in range(nmin, nmax + 1):
        flatyn, flat = 0, 0.0
        bars = [{j: arr[i + j - 3] for j in range(1, 6)} for arr in (pres, rho, vx, vy, vz)]
        pbar, rhobar, vxbar, vybar, vzbar = bars
        cbar = {1: c[i], 2: c[i + 1]}              # ppm.F90:106-107
        for arr in bars:
            if flatten5(arr, keep, S):
                flatyn = 1
            if flatyn == 1:
                flat = S.flatvalue
        for sl4 in slots:
            for sl in sl4:
                sl[1] = sl[2]
        addp = abs(pbar[4] - pbar[2]) / MIN(pbar[2], pbar[4])
        addrho = 0.50 * S.gamma * abs(rhobar[4] - rhobar[2]) / MIN(rhobar[2], rhobar[4])
        res = [correction(addp, addrho, arr, *slots[k], cbar, vxbar[2], vxbar[3], flat, nd, S)
               for k, (arr, nd) in enumerate(((pbar, 0), (rhobar, 1), (vxbar, 0), (vybar, 0), (vzbar, 0)))]
        (ptl, ptr, pcl, pcr), (rhotl, rhotr, rhocl, rhocr), (vxtl, vxtr, vxcl, vxcr) = res[0], res[1], res[2]
        (vytl, vytr, vycl, vycr), (vztl, vztr, vzcl, vzcr) = res[3], res[4]
        if ptl < 0.0:
            ptl = TINY
        if ptr < 0.0:
            ptr = TINY
        if rhotl < 0.0:
            rhotl = TINY
        if rhotr < 0.0:
            rhotr = TINY
        ctl = np.sqrt(S.gamma * ptl * rhotl)
        ctr = np.sqrt(S.gamma * ptr * rhotr)
        lm, l0, lp = (vxbar[2] - cbar[1]) * S.rat, vxbar[2] * S.rat, (vxbar[2] + cbar[1]) * S.rat
        betaml = 0.0 if lm <= 0.0 else beta(ctl, vxtl, vxcl[1], ptl, pcl[1], 0.0, -1.0, S)
        betapl = 0.0 if lp <= 0.0 else beta(ctl, vxtl, vxcl[3], ptl, pcl[3], 0.0, 1.0, S)
        vyleft, vzleft = vytl, vztl
        if l0 <= 0.0:
            beta0l = 0.0
        else:
            beta0l = beta0(ctl, rhotl, rhocl[2], ptl, pcl[2], S)
            vyleft, vzleft = vycl[2], vzcl[2]
        lm, l0, lp = (vxbar[3] - cbar[2]) * S.rat, vxbar[3] * S.rat, (vxbar[3] + cbar[2]) * S.rat
        betapr = 0.0 if lp >= 0.0 else beta(ctr, vxtr, vxcr[3], ptr, pcr[3], 0.0, 1.0, S)
        betamr = 0.0 if lm >= 0.0 else beta(ctr, vxtr, vxcr[1], ptr, pcr[1], 0.0, -1.0, S)
        vyright, vzright = vytr, vztr
        if l0 >= 0.0:
            beta0r = 0.0
        else:
            beta0r = beta0(ctr, rhotr, rhocr[2], ptr, pcr[2], S)
            vyright, vzright = vycr[2], vzcr[2]
        if i == nmin:
            continue
        pleft = ptl + ctl * ctl * (betapl + betaml)
        if pleft <= 0.0:
            pleft = ptl
        pright = ptr + ctr * ctr * (betapr + betamr)
        if pright <= 0.0:
            pright = ptr
        vxleft = vxtl + ctl * (betapl - betaml)
        vxright = vxtr + ctr * (betapr - betamr)
        rholeft = 1.0 / (1.0 / rhotl - betaml - beta0l - betapl)
        if rholeft <= 0.0:
            rholeft = rhotl
        rhoright = 1.0 / (1.0 / rhotr - betamr - beta0r - betapr)
        if rhoright <= 0.0:
            rhoright = rhotr
        face[1] = face[2]
        face[2] = riemannsolver(rhobar, vxbar, pleft, pright, rholeft, rhoright, vxleft, vxright, vyleft, vyright,
                                vzleft, vzright, S)
        if i == nmid:
            continue
        (pm1, rhom1, vxm1, vym1, vzm1), (pm2, rhom2, vxm2, vym2, vzm2) = face[1], face[2]
        ix = i - 1
        rhonew[ix] = rho[ix] + S.rdtath * (rhom1 * vxm1 - rhom2 * vxm2) * S.rdx
        fl1, fl2 = rhom1 * vxm1 * vxm1 + pm1, rhom2 * vxm2 * vxm2 + pm2
        vxnew[ix] = (vx[ix] * rho[ix] + S.rdtath * (fl1 - fl2) * S.rdx) / rhonew[ix]
        fl1, fl2 = vym1 * vxm1 * rhom1, vym2 * vxm2 * rhom2
        vynew[ix] = (rho[ix] * vy[ix] + S.rdtath * (fl1 - fl2) * S.rdx) / rhonew[ix]
        fl1, fl2 = vzm1 * vxm1 * rhom1, vzm2 * vxm2 * rhom2
        vznew[ix] = (rho[ix] * vz[ix] + S.rdtath * (fl1 - fl2) * S.rdx) / rhonew[ix]
        g = S.gamma
        fl1 = (g * pm1 * S.rgamma1 + 0.50 * rhom1 * (vxm1 * vxm1 + vym1 * vym1 + vzm1 * vzm1)) * vxm1
        fl2 = (g * pm2 * S.rgamma1 + 0.50 * rhom2 * (vxm2 * vxm2 + vym2 * vym2 + vzm2 * vzm2)) * vxm2
        etotnew[ix] = etot[ix] + S.rdtath * (fl1 - fl2) * S.rdx
        pmean = (pm1 + pm2) * 0.5
        if rhobar[2] > S.dmax * rhobar[1] and rhobar[2] > S.dmax * rhobar[3]:
            if cho[ix] == 1.0:
                pmean = MAX(pmean, (vxm1 - vxm2) * rhobar[2] * MAX(0.0, vxm1 - vxm2))
            elif cho[ix] == 2.0:
                pmean = (g - 1.0) * eint[ix]
        eintnew[ix] = eint[ix] + S.rdtath * pmean * (vxm1 - vxm2) * S.rdx
        fl1, fl2 = (pm1 * vxm1) * S.rgamma1, (pm2 * vxm2) * S.rgamma1
        eintnew[ix] = eintnew[ix] + S.rdtath * (fl1 - fl2) * S.rdx
        if eintnew[ix] < 0:
            eintnew[ix] = eint[ix]
    for i in range(nmin, nmax + 1):
        eeleft = 0.0 if i == nmin else etotnew[i - 1]
        eeright = 0.0 if i == nmax else etotnew[i + 1]
        ee2 = MAX(eeleft, etotnew[i], eeright)
        vvv = vxnew[i] * vxnew[i] + vynew[i] * vynew[i] + vznew[i] * vznew[i]
        eeaux = etotnew[i] - 0.50 * rhonew[i] * vvv
        if eeaux / ee2 >= S.eta2:
            eintnew[i] = eeaux
        if eeaux / etotnew[i] >= S.eta1:
            pnew[i] = (S.gamma - 1) * eeaux
        else:
            pnew[i] = (S.gamma - 1) * eintnew[i]
    out = [dict(pres), dict(rho), dict(vx), dict(vy), dict(vz)]
    for i in range(nmin, nmax + 1):
        if eintnew[i] <= 0.0:
            pnew[i] = pres[i]
        if rhonew[i] <= 0.0:
            rhonew[i] = rho[i]
        out[0][i], out[1][i], out[2][i], out[3][i], out[4][i] = pnew[i], rhonew[i], vxnew[i], vynew[i], vznew[i]
    return out


def ppmsolver_pencil(F, nb, nd, S, cho3d):
    """One non-STENCIL sweep of the ghosted fields F (savetn included)."""
    p3d, r3d, u3d, v3d, w3d = [a.copy(order="F") for a in F]
    nx, ny, nz = p3d.shape
    A = lambda arr, i, j, k: arr[i - 1, j - 1, k - 1]
    if nd == 1:
        ns, t1r, t2r, cell, roles = nx, range(nb + 1, ny - nb + 1), range(nb + 1, nz - nb + 1), \
            (lambda s, a, b: (s, a, b)), (0, 1, 2)
    elif nd == 2:
        ns, t1r, t2r, cell, roles = ny, range(nb + 1, nx - nb + 1), range(nb + 1, nz - nb + 1), \
            (lambda s, a, b: (a, s, b)), (1, 0, 2)
    else:
        ns, t1r, t2r, cell, roles = nz, range(nb + 1, nx - nb + 1), range(nb + 1, ny - nb + 1), \
            (lambda s, a, b: (a, b, s)), (2, 1, 0)
    vel = (u3d, v3d, w3d)
    new = [a.copy(order="F") for a in (p3d, r3d, u3d, v3d, w3d)]
    for b in t2r:
        for a in t1r:
            pres, rho, vx, vy, vz, c, eint, etot, cho = ({} for _ in range(9))
            for i in range(1, ns + 1):
                q = cell(i, a, b)
                pres[i], rho[i] = A(p3d, *q), A(r3d, *q)
                vx[i], vy[i], vz[i] = (A(vel[r], *q) for r in roles)
                eint[i] = pres[i] * S.rgamma1
                etot[i] = pres[i] * S.rgamma1 + 0.5 * rho[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i])
                cho[i] = A(cho3d, *q)
                c[i] = np.sqrt(S.gamma * pres[i] / rho[i])
            c[ns + 1] = np.float64(0.0)  # never read (cbar(2) of i = nmax <= ns)
            res = ppm_pencil(pres, rho, vx, vy, vz, c, eint, etot, cho, ns, nb, S)
            for i in range(1, ns + 1):
                idx = tuple(x - 1 for x in cell(i, a, b))
                new[0][idx], new[1][idx] = res[0][i], res[1][i]
                for r, f in zip(roles, (res[2], res[3], res[4])):
                    new[2 + r][idx] = f[i]
    return new


def _ghost(a, nb):
    return np.asfortranarray(np.pad(a, nb, mode="wrap"))


def make_case(seed, n=(10, 8, 6), nb=3, peak=False, single=False):
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = tuple(n)
    x = np.linspace(0, 2 * np.pi, shape[0], endpoint=False)[:, None, None]
    rho = 1.0 + 0.4 * np.sin(x) * np.ones(shape) + 0.3 * rng.random(shape)
    p = 0.8 + 0.5 * np.cos(x) * np.ones(shape) + 0.3 * rng.random(shape)
    if peak:
        rho[3::5, :, :] *= 40.0  # two-cell density spikes along x
        rho[4::5, :, :] *= 40.0
    if single:
        rho[6::10, :, :] *= 40.0  # one-cell spikes along x (a peak above both neighbours)
    vel = [0.6 * rng.standard_normal(shape) for _ in range(3)]
    vel[1][:, ::3, :] = 0.0  # exact zeros exercise the stale-gradleft path
    return [_ghost(a, nb) for a in (p, rho, *vel)]


def make_cold(seed, n, nb=3):
    """Cold, fast gas (p ~ 1e-6, sound speed ~ 1.3e-3): velocities of random
    sign whose magnitude spans 1e-3 .. 1 cell by cell, so the ratio of
    internal to total energy spans every branch of the dual-energy switch
    (integrate.F90), down to Mach numbers of several hundred."""
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = tuple(n)
    rho = 1.0 + 0.5 * rng.random(shape)
    p = 1e-6 * (1.0 + rng.random(shape))
    vel = [rng.standard_normal(shape) * 10.0 ** rng.uniform(-3.0, 0.0, shape) for _ in range(3)]
    return [_ghost(a, nb) for a in (p, rho, *vel)]


def make_extreme(seed, n, axis, nb=3):
    """Strong waves along the sweep axis: blocks of 3 cells cycle through
    cold gas (p ~ 1e-2), dense gas (rho ~ 100) and hot gas (p ~ 1e3), and
    the sweep velocity flips between +0.5 and -0.5 (about 4 cold sound
    speeds) every 3 cells, offset from the blocks: streams collide (strong
    two-shock faces), recede (vacuum faces) and meet pressure jumps of 1e5
    (strong shock + rarefaction faces)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = tuple(n)
    i = np.arange(shape[axis])
    sh = [1, 1, 1]
    sh[axis] = shape[axis]
    blk = ((i // 3) % 4).reshape(sh)
    rho = np.where(blk == 1, 100.0, 1.0) * (1.0 + 0.2 * rng.random(shape))
    p = np.where(blk == 2, 1e3, 1e-2) * (1.0 + 0.2 * rng.random(shape))
    vel = [0.05 * rng.standard_normal(shape) for _ in range(3)]
    vel[axis] = vel[axis] + np.where(((i + 1) // 3) % 2 == 0, 0.5, -0.5).reshape(sh)
    return [_ghost(a, nb) for a in (p, rho, *vel)]


CASES = [
    # name, seed, shape, sweep, scalars, peak
    ("static_x", 1, (10, 8, 6), 1, dict(dt=2e-3, at=1.0, dat=0.0, ath=1.0), dict()),
    ("static_y", 2, (8, 10, 6), 2, dict(dt=2e-3, at=1.0, dat=0.0, ath=1.0), dict()),
    ("static_z", 3, (6, 8, 10), 3, dict(dt=2e-3, at=1.0, dat=0.0, ath=1.0), dict()),
    ("cosmo_x", 4, (10, 8, 6), 1, dict(dt=1.5e-3, at=0.05, dat=3.1, ath=0.0502), dict()),
    ("cosmo_z", 5, (8, 8, 8), 3, dict(dt=1.5e-3, at=0.05, dat=3.1, ath=0.0502), dict()),
    ("peak_y", 6, (10, 10, 10), 2, dict(dt=1e-3, at=1.0, dat=0.0, ath=1.0), dict(dmax=2.0)),
    # static gravity source (the Gaussian potential of initialize_gravity.F90,
    # scaled up so the source terms are large)
    ("grav_x", 7, (10, 8, 6), 1, dict(dt=2e-3, at=1.0, dat=0.0, ath=1.0), dict()),
    ("grav_y", 8, (8, 10, 6), 2, dict(dt=1.5e-3, at=0.05, dat=3.1, ath=0.0502), dict()),
    ("grav_z", 9, (6, 8, 10), 3, dict(dt=2e-3, at=1.0, dat=0.0, ath=1.0), dict()),
    # the non-STENCIL build's full-pencil solver; pencil_peak_x: density spikes
    # along the sweep with dmax = 2 and a cho3d of 0, 1, 2
    ("pencil_x", 10, (10, 8, 6), 1, dict(dt=2e-3, at=1.0, dat=0.0, ath=1.0), dict()),
    ("pencil_y", 11, (8, 10, 6), 2, dict(dt=1.5e-3, at=0.05, dat=3.1, ath=0.0502), dict()),
    ("pencil_z", 12, (6, 8, 10), 3, dict(dt=2e-3, at=1.0, dat=0.0, ath=1.0), dict()),
    ("pencil_peak_x", 13, (10, 8, 6), 1, dict(dt=1e-3, at=1.0, dat=0.0, ath=1.0), dict(dmax=2.0)),
    # strong shocks, vacuum and two-rarefaction faces (make_extreme); dt at a
    # Courant number of about 0.32
    ("extreme_x", 7, (12, 8, 8), 1, dict(dt=6e-4, at=1.0, dat=0.0, ath=1.0), dict()),
    ("extreme_z", 8, (8, 8, 12), 3, dict(dt=3e-5, at=0.05, dat=3.1, ath=0.0502), dict()),
    ("extreme_y", 9, (8, 12, 8), 2, dict(dt=6e-4, at=1.0, dat=0.0, ath=1.0), dict()),
    # cold, fast gas over every branch of the dual-energy switch (make_cold);
    # Courant numbers about 0.2
    ("cold_x", 14, (10, 8, 8), 1, dict(dt=1e-2, at=1.0, dat=0.0, ath=1.0), dict()),
    ("cold_z", 15, (8, 8, 10), 3, dict(dt=5e-4, at=0.05, dat=3.1, ath=0.0502), dict()),
]


def gravity_field(shape, nb, alpha=40.0, sigma=0.3):
    """gforce(3, ...) ghosted: phi = alpha exp(-r^2/(2 sigma^2)) at the cell
    centres, central differences phi(i+1) - phi(i-1), periodic."""
    dx = 1.0 / max(shape)
    ax = [(np.arange(n) + 0.5) * dx - 0.5 for n in shape]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    phi = alpha * np.exp(-(X * X + Y * Y + Z * Z) / (2.0 * sigma * sigma))
    g = np.empty((3,) + tuple(n + 2 * nb for n in shape), order="F")
    for d in range(3):
        g[d] = np.pad(np.roll(phi, -1, axis=d) - np.roll(phi, 1, axis=d), nb, mode="wrap")
    return g


def run_case(name, seed, shape, nd, tsc, extra):
    nb = 3
    if name.startswith("extreme"):
        F = make_extreme(seed, shape, nd - 1, nb)
    elif name.startswith("cold"):
        F = make_cold(seed, shape, nb)
    else:
        F = make_case(seed, shape, nb, peak="peak" in name, single=name == "pencil_peak_x")
    S = Sc(5.0 / 3.0, 1.0 / max(shape), **tsc, **extra)
    G = gravity_field(shape, nb) if name.startswith("grav") else None
    if name.startswith("pencil"):
        rng = np.random.Generator(np.random.PCG64(seed + 100))
        cho = _ghost(rng.integers(0, 3, shape).astype(np.float64), nb)
        return F, ppmsolver_pencil(F, nb, nd, S, cho), S, {"cho": cho}
    TALLY[:] = [0] * len(TALLY)
    DUAL[:] = [0] * len(DUAL)
    out = ppmsolver(F, nb, nd, S, G)
    more = {} if G is None else {"gforce": G}
    if name.startswith("extreme"):
        more["patterns"] = np.array(TALLY)
    if name.startswith("cold"):
        more["dual"] = np.array(DUAL)
    return F, out, S, more


def main(names=None):
    """Write the golden files of the named cases (default: all)."""
    np.seterr(all="ignore")  # IEEE results (inf/NaN) instead of warnings, as in Fortran
    here = os.path.dirname(os.path.abspath(__file__))
    for name, seed, shape, nd, tsc, extra in CASES:
        if names and name not in names:
            continue
        F, out, S, more = run_case(name, seed, shape, nd, tsc, extra)
        np.savez_compressed(os.path.join(here, f"{name}.npz"), inp=np.stack(F), out=np.stack(out), nd=nd,
                            shape=np.array(shape), dt=tsc["dt"], at=tsc["at"], dat=tsc["dat"], ath=tsc["ath"],
                            dmax=extra.get("dmax", 2e10), **more)
        print(name, "ok")


if __name__ == "__main__":
    import sys
    main(sys.argv[1:])
