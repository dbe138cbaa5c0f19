"""Initial conditions for the benchmark configurations.

* :func:`sod` -- the plane-parallel Sod tube (the reference's chooseinit=1/2/3,
  hydropad/initialize_hydro.F90:35-117) with the interface at x=0.5 and its
  periodic mirror at x=0.
* :func:`grf_eds` -- a seeded Gaussian random baryon field on an EdS
  background with linear-theory velocities and uniform temperature (the
  cosmological configurations; reference analogue initvel.F90:31-37).
* :func:`grf_eds_device` -- the same field with the FFT work on the GPU,
  returned as device tensors (serving and large boxes).

The host functions return ``(p, rho, vx, vy, vz)`` as ghosted Fortran-order
float64 arrays ``(N+2nb, ...)`` with periodic ghosts filled.
"""
from __future__ import annotations

import numpy as np

# physical constants of the reference namelists (inputfiles/input.nml)
BOLTZ = 1.380658e-16
MH = 1.6605e-24
MPC_CM = 3.086e24


def _ghost(a: np.ndarray, nb: int) -> np.ndarray:
    out = np.pad(a, nb, mode="wrap")
    return np.asfortranarray(out)


def sod(n, axis: int = 0, nb: int = 3, rho_l=1.0, p_l=1.0, rho_r=0.125, p_r=0.1):
    """Sod tube along ``axis`` on an ``n`` (int or 3-tuple) periodic grid.
    Cell centres x=(i+1/2)/N; left state for x<0.5."""
    shape = (n, n, n) if np.isscalar(n) else tuple(n)
    N = shape[axis]
    x = (np.arange(N) + 0.5) / N
    left = x < 0.5
    sh = [1, 1, 1]
    sh[axis] = N
    rho = np.broadcast_to(np.where(left, rho_l, rho_r).reshape(sh), shape).astype(np.float64)
    p = np.broadcast_to(np.where(left, p_l, p_r).reshape(sh), shape).astype(np.float64)
    z = np.zeros(shape)
    return tuple(_ghost(a, nb) for a in (p, rho, z, z, z))


def eds_time(a_start: float):
    """EdS time variables at a_start as initialize_parameters.F90:133-154
    sets them (t = a^1.5, H = dat/at)."""
    f2 = np.float32(2.0) / np.float32(3.0)
    tin = a_start ** 1.5
    at = tin ** float(f2)
    dat = float(f2) * tin ** float(np.float32(-1.0) / np.float32(3.0))
    return tin, at, dat


def temperature_factor(box_mpc_over_h: float = 1.0, hnow: float = 0.7) -> float:
    """tfact of initialize_parameters.F90:109 (code temperature = T/tfact).

    The code length unit is the box (dx = 1/N, initialize_parameters.F90:23),
    so xnow is taken as the box length; the reference's line 75 divides it by
    ngridx, which would make the code temperature depend on the resolution."""
    box = box_mpc_over_h / hnow
    xnow = MPC_CM * box
    h_sec = hnow / 3.0856e17
    t0h0 = 0.66666666667
    tnow = t0h0 / h_sec
    r = BOLTZ / MH
    return (xnow / tnow) ** 2 / r


def grf_eds(n: int, seed: int = 12345, a_start: float = 1.0 / 51.0, rms: float = 0.5, spectral_index: float = -2.0,
            kc_frac: float = 1.0 / 8.0, temp_k: float = 100.0, rho_floor: float = 1e-2, nb: int = 3,
            gamma: float = 5.0 / 3.0):
    """Gaussian random overdensity with P(k) ~ k^n exp(-(k/kc)^2), k in grid
    units, kc = kc_frac*N, rms delta normalised to ``rms``; rho = max(1+delta,
    rho_floor); v_k = i a H f delta_k k/k^2 (f=1, EdS; k in box units);
    uniform temperature -> p = rho*T/tfact."""
    rng = np.random.Generator(np.random.PCG64(seed))
    white = rng.standard_normal((n, n, n))
    wk = np.fft.rfftn(white)
    kx = np.fft.fftfreq(n) * n
    kz = np.fft.rfftfreq(n) * n
    KX, KY, KZ = np.meshgrid(kx, kx, kz, indexing="ij")
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    k = np.sqrt(k2)
    kc = kc_frac * n
    with np.errstate(divide="ignore", invalid="ignore"):
        pk = np.where(k > 0, k ** spectral_index * np.exp(-(k / kc) ** 2), 0.0)
    dk = wk * np.sqrt(pk)
    delta = np.fft.irfftn(dk, s=(n, n, n), axes=(0, 1, 2))
    norm = rms / delta.std()
    delta *= norm
    dk *= norm
    tin, at, dat = eds_time(a_start)
    hub = dat / at
    fac = at * hub * 1.0  # a H f
    two_pi = 2.0 * np.pi
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = np.where(k2 > 0, 1.0 / (two_pi * k2), 0.0)  # k_phys/k_phys^2 = k_int/(2 pi k_int^2)
    vel = []
    for K in (KX, KY, KZ):
        vk = 1j * fac * dk * K * inv
        vel.append(np.fft.irfftn(vk, s=(n, n, n), axes=(0, 1, 2)))
    rho = np.maximum(1.0 + delta, rho_floor)
    tcode = temp_k / temperature_factor()
    p = rho * tcode
    return tuple(_ghost(np.ascontiguousarray(a), nb) for a in (p, rho, vel[0], vel[1], vel[2]))


def grf_eds_device(n: int, seed: int = 12345, a_start: float = 1.0 / 51.0, rms: float = 0.5,
                   spectral_index: float = -2.0, kc_frac: float = 1.0 / 8.0, temp_k: float = 100.0,
                   rho_floor: float = 1e-2, device="cuda", noise: str = "host"):
    """:func:`grf_eds` with the spectral work on the GPU.

    ``noise="host"``: the white noise is the same PCG64 draw as
    :func:`grf_eds` (generated on the host, so a seed gives the same field on
    every path).  ``noise="device"``: a normal draw of the device's own
    generator (Philox) seeded with ``seed`` -- the same recipe and the same
    field for a given seed and device, a different realisation from the host
    draw, and no host work (the serving engine's choice).  The FFTs, the
    power-spectrum filter and the linear velocities run on ``device`` in
    FP64.  Returns ``(p, rho, vx, vy, vz)`` as contiguous float64 device
    tensors in the device state layout: shape ``(n, n, n)`` indexed
    ``[z, y, x]`` (x fastest), no ghosts -- the input of
    ``Hydro.attach_device``.  With host noise it agrees with :func:`grf_eds`
    to FFT rounding."""
    import torch
    if noise == "device":
        gen = torch.Generator(device=device)
        gen.manual_seed(int(seed))
        white = torch.randn((n, n, n), generator=gen, dtype=torch.float64, device=device)
    else:
        rng = np.random.Generator(np.random.PCG64(seed))
        white = torch.from_numpy(rng.standard_normal((n, n, n))).to(device)  # indexed [x, y, z] like grf_eds
    wk = torch.fft.rfftn(white)
    del white
    f64 = dict(dtype=torch.float64, device=wk.device)
    kx = torch.fft.fftfreq(n, **f64) * n
    kz = torch.fft.rfftfreq(n, **f64) * n
    KX, KY, KZ = kx[:, None, None], kx[None, :, None], kz[None, None, :]
    k2 = KX * KX + KY * KY + KZ * KZ
    k = torch.sqrt(k2)
    kc = kc_frac * n
    pk = torch.where(k > 0, k.pow(spectral_index) * torch.exp(-(k / kc) ** 2), torch.zeros_like(k))
    dk = wk * torch.sqrt(pk)
    del wk, pk, k
    delta = torch.fft.irfftn(dk, s=(n, n, n))
    norm = rms / float(delta.std(correction=0))
    delta *= norm
    dk *= norm
    tin, at, dat = eds_time(a_start)
    fac = at * (dat / at)  # a H f, f = 1
    two_pi = 2.0 * np.pi
    inv = torch.where(k2 > 0, 1.0 / (two_pi * k2), torch.zeros_like(k2))
    del k2
    to_dev = lambda a: a.permute(2, 1, 0).contiguous()  # [x, y, z] -> memory x fastest
    vel = []
    for K in (KX, KY, KZ):
        vk = (1j * fac) * dk * (K * inv)
        vel.append(to_dev(torch.fft.irfftn(vk, s=(n, n, n))))
        del vk
    rho = torch.clamp(1.0 + delta, min=rho_floor)
    tcode = temp_k / temperature_factor()
    p = rho * tcode
    return to_dev(p), to_dev(rho), vel[0], vel[1], vel[2]


def static_gravity(shape, nb: int = 3, alpha: float = 1.0, sigma: float = float(np.float32(0.3)),
                   center=(0.5, 0.5, 0.5)):
    """The reference's static gravity force (initialize_gravity.F90:25-55):
    a Gaussian potential phi = alpha exp(-r^2 / (2 sigma^2)) about
    ``center`` at the cell centres x = (i - 0.5) dx (the integer and 0.5
    in REAL(4), sigma = 0.3 as a REAL(4) literal), and
    gforce(d) = phi(i+1) - phi(i-1) along d, periodic.  Returns the ghosted
    ``gforce(3, nx, ny, nz)`` array (component fastest, Fortran order)."""
    shape = (shape, shape, shape) if np.isscalar(shape) else tuple(int(v) for v in shape)
    dx = 1.0 / float(max(shape))
    ax = []
    for d, n in enumerate(shape):
        i = np.arange(1, n + 1, dtype=np.float32)
        ax.append((i - np.float32(0.5)).astype(np.float64) * dx - center[d])
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    phi = alpha * np.exp(-((X * X + Y * Y) + Z * Z) / (2.0 * (sigma * sigma)))
    g = np.empty((3,) + tuple(n + 2 * nb for n in shape), dtype=np.float64, order="F")
    for d in range(3):
        comp = np.roll(phi, -1, axis=d) - np.roll(phi, 1, axis=d)
        g[d] = np.pad(comp, nb, mode="wrap")
    return g
