"""Shared test helpers: run the oracle and the GPU path on the same inputs."""
from __future__ import annotations

import ctypes as C

import numpy as np

from hydropad_b200 import ics
from hydropad_b200.params import HydroParams

NB = 3


def interior(a, nb=NB):
    return a[nb:-nb, nb:-nb, nb:-nb]


def rel_l1(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.abs(b).sum()
    return float(np.abs(a - b).sum() / den) if den > 0 else float(np.abs(a - b).sum())


def sod_state(n, axis=0):
    return ics.sod(n, axis=axis, nb=NB)


def grf_state(n, seed=7):
    return ics.grf_eds(n, seed=seed, nb=NB)


def extreme_state(shape, seed):
    """Strong waves along every axis, periodic ghosts: blocks of 3 cells
    (counted along each axis and summed) cycle through cold gas (p ~ 1e-2),
    dense gas (rho ~ 100) and hot gas (p ~ 1e3), and the velocity along each
    axis flips between +0.5 and -0.5 (about 4 cold sound speeds) every 3
    cells: streams collide (strong two-shock faces), recede (vacuum faces)
    and meet pressure jumps of 1e5 (strong shock + rarefaction faces)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    idx = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    blk = sum(i // 3 for i in idx) % 4
    rho = np.where(blk == 1, 100.0, 1.0) * (1.0 + 0.2 * rng.random(shape))
    p = np.where(blk == 2, 1e3, 1e-2) * (1.0 + 0.2 * rng.random(shape))
    vel = [0.05 * rng.standard_normal(shape) + np.where(((idx[d] + 1) // 3) % 2 == 0, 0.5, -0.5)
           for d in range(3)]
    return tuple(np.asfortranarray(np.pad(a, NB, mode="wrap")) for a in (p, rho, *vel))


def oracle_first_dt(oracle, st, s):
    """dt of the first step from the CFL condition (the harness's choice for
    the configurations; the reference would use dtinit): the clock is put
    back to the initial time and timedet runs on the initial state."""
    s.t = s.told
    s.velmax = st.speed(s)
    lib = oracle.lib()
    if s.cosmo:
        lib.hpo_timedet_cosmo(C.byref(s))
    else:
        lib.hpo_timedet(C.byref(s))


def params_for(shape, cosmo=False, **kw):
    p = HydroParams(shape=tuple(shape), cosmo=cosmo, **kw)
    if cosmo:
        p.tstop = (1.0 + 10.0) ** (-1.5)  # z = 10 (initialize_parameters.F90:85)
    return p
