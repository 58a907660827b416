"""Seeded synthetic initial conditions for the force-path workloads.

No public dataset is involved: every workload is generated here from a seed
with numpy's PCG64 generator.  Units are G = 1.  Each generator returns a dict
with ``parray`` ([N, 6] float64: x, y, z, m, h, zeta as in the reference's
parray(1:6,p)), ``v`` ([N, 3]), ``sound`` ([N], isothermal c_s), and the
parameters the reference reads from params.dat (``h_fac``, ``thetamaxsqd``,
``alpha``).

The ``h`` column is the smoothing length an IC file would carry.  The
reference stocks the gravity tree with it on the first force evaluation (its
``sph_setup`` calls ``tree_update`` before ``BHhydro_hguess``), so it sets the
MAC's kernel-overlap term of that first evaluation.  It is computed from the
analytic density of each model: h = h_fac * (m / rho)^(1/3).
"""
from __future__ import annotations

import math

import numpy as np

__all__ = [
    "pp_gather_for",
    "h_fac_for",
    "uniform_sphere",
    "plummer",
    "turbulent_core",
    "batched_clouds",
    "protostellar_disc",
]


def pp_gather_for(h_fac: float) -> int:
    """pp_gather = int((4*PI/3)*(KERNRANGE*h_fac)**3), initialize_seren_variables_1.F90:36."""
    pi = 3.1415926536
    x = 2.0 * h_fac
    return int((4.0 * pi / 3.0) * (x * (x * x)))


def h_fac_for(n_neigh: float) -> float:
    """h_fac giving a mean neighbour number n_neigh inside 2h: (3 n / (32 pi))^(1/3)."""
    return (3.0 * n_neigh / (32.0 * math.pi)) ** (1.0 / 3.0)


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _isotropic(rng: np.random.Generator, n: int) -> np.ndarray:
    cos_t = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    sin_t = np.sqrt(np.maximum(0.0, 1.0 - cos_t * cos_t))
    return np.stack([sin_t * np.cos(phi), sin_t * np.sin(phi), cos_t], axis=1)


def _pack(pos, m, h, v, sound, **extra):
    n = pos.shape[0]
    parray = np.zeros((n, 6), dtype=np.float64)
    parray[:, 0:3] = pos
    parray[:, 3] = m
    parray[:, 4] = h
    out = dict(parray=parray, v=np.ascontiguousarray(v, dtype=np.float64),
               sound=np.ascontiguousarray(sound, dtype=np.float64))
    out.update(extra)
    return out


def uniform_sphere(n: int = 32768, seed: int = 1, radius: float = 1.0, mass: float = 1.0,
                   sound: float = 0.1, h_fac: float = 1.2, thetamaxsqd: float = 0.25,
                   alpha: float = 1.0, velocity=None):
    """Cold uniform sphere: r = R u^(1/3) with isotropic directions, equal masses."""
    rng = _rng(seed)
    r = radius * rng.uniform(0.0, 1.0, n) ** (1.0 / 3.0)
    pos = _isotropic(rng, n) * r[:, None]
    m = mass / n
    rho = 3.0 * mass / (4.0 * math.pi * radius ** 3)
    h = h_fac * (m / rho) ** (1.0 / 3.0)
    v = np.zeros((n, 3)) if velocity is None else velocity
    return _pack(pos, m, h, v, np.full(n, sound), h_fac=h_fac, thetamaxsqd=thetamaxsqd,
                 alpha=alpha, name=f"uniform sphere N={n}")


def _ahw_speed_fraction(rng: np.random.Generator, n: int) -> np.ndarray:
    """Aarseth, Henon & Wielen (1974, A&A 37, 183) rejection sampling of
    q = v/v_esc from g(q) = q^2 (1 - q^2)^(7/2), whose maximum is below 0.1."""
    out = np.empty(n)
    filled = 0
    while filled < n:
        k = max(1024, 2 * (n - filled))
        q = rng.uniform(0.0, 1.0, k)
        y = rng.uniform(0.0, 0.1, k)
        acc = q[y < q * q * (1.0 - q * q) ** 3.5]
        take = min(acc.size, n - filled)
        out[filled:filled + take] = acc[:take]
        filled += take
    return out


def plummer(n: int = 1048576, seed: int = 2, a: float = 1.0, mass: float = 1.0,
            rtrunc: float = 20.0, n_neigh: float = 50.0, thetamaxsqd: float = 0.25,
            sound: float = 0.0):
    """Plummer sphere: inverse-CDF radius r = a / sqrt(u^(-2/3) - 1), redrawn
    while r > rtrunc; isotropic angles; AHW velocities.  Gravity-only workload."""
    rng = _rng(seed)
    r = np.empty(n)
    filled = 0
    while filled < n:
        k = 2 * (n - filled) + 16
        u = rng.uniform(0.0, 1.0, k)
        u = u[u > 0.0]
        rr = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        rr = rr[rr <= rtrunc]
        take = min(rr.size, n - filled)
        r[filled:filled + take] = rr[:take]
        filled += take
    pos = _isotropic(rng, n) * r[:, None]
    q = _ahw_speed_fraction(rng, n)
    vesc = math.sqrt(2.0 * mass / a) * (1.0 + (r / a) ** 2) ** (-0.25)
    v = _isotropic(rng, n) * (q * vesc)[:, None]
    m = mass / n
    rho = 3.0 * mass / (4.0 * math.pi * a ** 3) * (1.0 + (r / a) ** 2) ** (-2.5)
    h_fac = h_fac_for(n_neigh)
    h = h_fac * (m / rho) ** (1.0 / 3.0)
    return _pack(pos, m, h, v, np.full(n, sound), h_fac=h_fac, thetamaxsqd=thetamaxsqd,
                 alpha=1.0, name=f"Plummer N={n}")


def turbulent_velocity(pos: np.ndarray, seed: int, ngrid: int = 128, index: float = -4.0,
                       v_rms: float = 0.4, box: float = 2.0) -> np.ndarray:
    """Divergence-free Gaussian random velocity field with power spectrum
    P(k) ~ k^index on an ngrid^3 periodic grid spanning [-box/2, box/2]^3,
    trilinearly interpolated to the particles and scaled to rms speed v_rms."""
    rng = _rng(seed)
    ng = ngrid
    k1 = np.fft.fftfreq(ng) * ng
    kz1 = np.fft.rfftfreq(ng) * ng
    kx, ky, kz = np.meshgrid(k1, k1, kz1, indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = 1.0
    amp = k2 ** (index / 4.0)          # sqrt(P(k)) = k^(index/2)
    amp[0, 0, 0] = 0.0
    comps = []
    for _ in range(3):
        white = rng.standard_normal((ng, ng, ng))
        comps.append(np.fft.rfftn(white) * amp)
    vx, vy, vz = comps
    kdotv = (kx * vx + ky * vy + kz * vz) / k2
    vx = vx - kx * kdotv
    vy = vy - ky * kdotv
    vz = vz - kz * kdotv
    grid = [np.fft.irfftn(c, s=(ng, ng, ng), axes=(0, 1, 2)) for c in (vx, vy, vz)]
    # trilinear interpolation on the periodic grid (cell-centred at (i+0.5)*dx - box/2)
    dx = box / ng
    g = (pos + 0.5 * box) / dx - 0.5
    i0 = np.floor(g).astype(np.int64)
    f = g - i0
    out = np.zeros((pos.shape[0], 3))
    for dxi in (0, 1):
        wx = f[:, 0] if dxi else 1.0 - f[:, 0]
        ix = (i0[:, 0] + dxi) % ng
        for dyi in (0, 1):
            wy = f[:, 1] if dyi else 1.0 - f[:, 1]
            iy = (i0[:, 1] + dyi) % ng
            for dzi in (0, 1):
                wz = f[:, 2] if dzi else 1.0 - f[:, 2]
                iz = (i0[:, 2] + dzi) % ng
                w = wx * wy * wz
                for c in range(3):
                    out[:, c] += w * grid[c][ix, iy, iz]
    out -= out.mean(axis=0)
    rms = math.sqrt(float(np.mean(np.sum(out * out, axis=1))))
    return out * (v_rms / rms)


def turbulent_core(n: int = 4194304, seed: int = 4, sound: float = 0.2, mach: float = 2.0,
                   h_fac: float = 1.2, thetamaxsqd: float = 0.25, alpha: float = 1.0,
                   ngrid: int = 128):
    """Uniform sphere (R = 1, M = 1) with a P(k) ~ k^-4 divergence-free velocity
    field at rms Mach `mach` for isothermal sound speed `sound`."""
    ic = uniform_sphere(n=n, seed=seed, sound=sound, h_fac=h_fac, thetamaxsqd=thetamaxsqd,
                        alpha=alpha)
    ic["v"] = turbulent_velocity(ic["parray"][:, 0:3], seed=seed + 1000003, ngrid=ngrid,
                                 v_rms=mach * sound)
    ic["name"] = f"turbulent core N={n}"
    return ic


def batched_clouds(ncloud: int = 256, nmin: int = 8192, nmax: int = 262144, seed0: int = 1000,
                   h_fac: float = 1.2, thetamaxsqd: float = 0.25):
    """Independent uniform-sphere clouds with log-uniform N and c_s ~ U[0.05, 0.3]."""
    rng = _rng(seed0)
    ns = np.rint(np.exp(rng.uniform(math.log(nmin), math.log(nmax), ncloud))).astype(np.int64)
    cs = rng.uniform(0.05, 0.3, ncloud)
    return [uniform_sphere(n=int(ns[i]), seed=seed0 + i, sound=float(cs[i]), h_fac=h_fac,
                           thetamaxsqd=thetamaxsqd) for i in range(ncloud)]


def protostellar_disc(n: int = 8388608, seed: int = 5, m_sink: float = 1.0, h_sink: float = 0.05,
                      m_disc: float = 0.1, rin: float = 0.1, rout: float = 10.0,
                      h_over_r: float = 0.05, cs1: float = 0.05, h_fac: float = 1.2,
                      thetamaxsqd: float = 0.25):
    """Disc with Sigma ~ 1/R on [rin, rout] (so R is uniform), Gaussian vertical
    profile with H = h_over_r * R, c_s = cs1 * R^-0.25 and Keplerian rotation
    about a central sink plus the isothermal pressure correction
    v_phi^2 = G M(<R) / R + (d ln P / d ln R) c_s^2 with P ~ R^-2.5 at the midplane."""
    rng = _rng(seed)
    R = rng.uniform(rin, rout, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    H = h_over_r * R
    z = rng.standard_normal(n) * H
    pos = np.stack([R * np.cos(phi), R * np.sin(phi), z], axis=1)
    cs = cs1 * R ** (-0.25)
    menc = m_sink + m_disc * (R - rin) / (rout - rin)
    vphi = np.sqrt(np.maximum(menc / R - 2.5 * cs * cs, 0.0))
    v = np.stack([-vphi * np.sin(phi), vphi * np.cos(phi), np.zeros(n)], axis=1)
    m = m_disc / n
    sigma = m_disc / (2.0 * math.pi * R * (rout - rin))
    rho = sigma / (math.sqrt(2.0 * math.pi) * H) * np.exp(-0.5 * (z / H) ** 2)
    h = h_fac * (m / rho) ** (1.0 / 3.0)
    sink = np.array([[0.0, 0.0, 0.0, m_sink, h_sink]])
    return _pack(pos, m, h, v, cs, h_fac=h_fac, thetamaxsqd=thetamaxsqd, alpha=1.0, sink=sink,
                 name=f"disc N={n} + sink")
