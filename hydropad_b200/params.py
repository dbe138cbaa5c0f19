"""Run parameters of the hydro step and the derived constants.

Mirrors the namelist groups the hot path reads (hydropad/init_sys.F90:12-44)
and the constants derived from them (hydropad/initialize_parameters.F90:23-24,
63-69).  Namelist values are REAL(8) in the reference, so plain Python floats
are exact mirrors.
"""
from __future__ import annotations

from dataclasses import dataclass, field


@dataclass
class HydroParams:
    """Namelist values used by ppm_lxlylz / ppmsolver / timedet.

    ``shape`` is the interior grid (ngridx, ngridy, ngridz) of one box.
    """

    shape: tuple = (64, 64, 64)
    nbound: int = 3            # &MESH nbound
    gamma: float = 5.0 / 3.0   # &PHYSICS gamma
    cour: float = 0.8          # &NUMERICS cour
    ca: float = 0.02           # &NUMERICS ca
    eta1: float = 1e-3         # &NUMERICS eta1
    eta2: float = 0.1          # &NUMERICS eta2
    dmax: float = 2.0e10       # &NUMERICS dmax
    flatvalue: float = 0.15    # &PPM flatvalue
    mingradflat: float = 0.25  # &PPM mingradflat
    dtinit: float = 0.1        # &TIME dtinit
    tstop: float = 10000.0     # &TIME tstop
    cosmo: bool = False        # -DCOSMO: EdS background (timedet_cosmo + expand)
    a_start: float = 1.0 / 51.0
    dt_cap: float = 0.0        # timedet_cosmo debug cap dt0 (<=0: off)
    expand_zero_old: bool = False  # expand with vxold=pold3d=0 instead of a step-start snapshot
    extra: dict = field(default_factory=dict)

    @property
    def ngrid_max(self) -> int:
        return int(max(self.shape))

    @property
    def dx(self) -> float:
        return 1.0 / float(self.ngrid_max)

    def derived(self) -> dict:
        """initialize_parameters.F90:23-24,64-69."""
        g = self.gamma
        m = (g - 1.0) / (2.0 * g)
        dx = 1.0 / float(self.ngrid_max)
        return dict(dx=dx, rdx=1.0 / dx, rgamma=1.0 / g, gamma1=(g + 1.0) / (g - 1.0),
                    rgamma1=1.0 / (g - 1.0), m=m, rm=1.0 / m, gf=(g + 1.0) / (2.0 * g))
