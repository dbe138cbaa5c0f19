"""Exact solution of the 1-D Riemann problem for an ideal gas (textbook
method: Newton iteration on the pressure function, then sampling of the
self-similar wave fan).  Used only as a physics pin of the oracle."""
from __future__ import annotations

import math

import numpy as np


def _f(p, rho, pk, ck, g):
    if p > pk:  # shock
        A = 2.0 / ((g + 1.0) * rho)
        B = (g - 1.0) / (g + 1.0) * pk
        f = (p - pk) * math.sqrt(A / (p + B))
        df = math.sqrt(A / (B + p)) * (1.0 - (p - pk) / (2.0 * (B + p)))
    else:  # rarefaction
        f = 2.0 * ck / (g - 1.0) * ((p / pk) ** ((g - 1.0) / (2.0 * g)) - 1.0)
        df = 1.0 / (rho * ck) * (p / pk) ** (-(g + 1.0) / (2.0 * g))
    return f, df


def star_state(rl, ul, pl, rr, ur, pr, g):
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    p = 0.5 * (pl + pr)
    for _ in range(100):
        fl, dfl = _f(p, rl, pl, cl, g)
        fr, dfr = _f(p, rr, pr, cr, g)
        dp = (fl + fr + ur - ul) / (dfl + dfr)
        p_new = max(p - dp, 1e-12)
        if abs(p_new - p) / (0.5 * (p_new + p)) < 1e-14:
            p = p_new
            break
        p = p_new
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    return p, u


def sample(xi, rl, ul, pl, rr, ur, pr, g):
    """(rho, u, p) at similarity coordinate xi = (x - x0)/t."""
    ps, us = star_state(rl, ul, pl, rr, ur, pr, g)
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    out = np.zeros((len(xi), 3))
    for i, s in enumerate(xi):
        if s <= us:  # left of contact
            if ps > pl:
                sl = ul - cl * math.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if s <= sl:
                    out[i] = (rl, ul, pl)
                else:
                    r = rl * (ps / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pl + 1)
                    out[i] = (r, us, ps)
            else:
                shl = ul - cl
                csl = cl * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - csl
                if s <= shl:
                    out[i] = (rl, ul, pl)
                elif s >= stl:
                    out[i] = (rl * (ps / pl) ** (1 / g), us, ps)
                else:
                    u = 2 / (g + 1) * (cl + (g - 1) / 2 * ul + s)
                    c = 2 / (g + 1) * (cl + (g - 1) / 2 * (ul - s))
                    r = rl * (c / cl) ** (2 / (g - 1))
                    out[i] = (r, u, pl * (c / cl) ** (2 * g / (g - 1)))
        else:
            if ps > pr:
                sr = ur + cr * math.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if s >= sr:
                    out[i] = (rr, ur, pr)
                else:
                    r = rr * (ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1)
                    out[i] = (r, us, ps)
            else:
                shr = ur + cr
                csr = cr * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + csr
                if s >= shr:
                    out[i] = (rr, ur, pr)
                elif s <= str_:
                    out[i] = (rr * (ps / pr) ** (1 / g), us, ps)
                else:
                    u = 2 / (g + 1) * (-cr + (g - 1) / 2 * ur + s)
                    c = 2 / (g + 1) * (cr - (g - 1) / 2 * (ur - s))
                    r = rr * (c / cr) ** (2 / (g - 1))
                    out[i] = (r, u, pr * (c / cr) ** (2 * g / (g - 1)))
    return out
