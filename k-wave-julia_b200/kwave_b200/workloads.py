"""Seeded synthetic simulation workloads (the benchmark configurations, with reduced-size variants).

No public dataset exists for this path; every medium, source and sensor here is generated from a
seeded ``numpy.random.Generator(PCG64(seed))``.  Random media are Gaussian random fields: white
noise filtered periodically with a Gaussian of standard deviation ``sigma_px`` (an FFT multiply by
exp(-|k|^2 sigma^2 / 2)), then min-max mapped onto the stated range.

Each builder returns a ``Case``: plain parameters and numpy arrays in the reference's Julia index
order, convertible to this package's types (``to_api``) or to any other implementation of the
reference API with the same field names.

  c1  128^2 homogeneous lossless, disc p-source (tone burst), circle sensor recording p
  c2  512^2 heterogeneous c/rho, power law y=1.5 (:stokes), 64-point line p0, full-grid p_max+p_rms
  c3  256^3 heterogeneous c/rho/BonA (ball inclusion), y=1.1 (:no_dispersion), 32x32 ux piston,
      xy plane p + volume p_max
  c4  64 mixed-size 2D heterogeneous absorbing simulations with tone-burst point/disc sources
  c5  Poisson serving stream (70 % 2D 256-1024, 30 % 3D 64^3-192^3)
  elastic3d  256^3 heterogeneous elastic solid (pstd_elastic_3d), p0 ball + sxx point source,
      xy plane p
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any, List, Optional

import numpy as np

from .core import (Additive, KWaveGrid, KWaveMedium, KWaveSensor, KWaveSource, make_ball,
                   make_circle, make_disc, make_time, tone_burst)


@dataclass
class Case:
    name: str
    N: tuple
    d: tuple
    dt: float
    Nt: int
    medium: dict
    source: dict
    sensor: dict
    pml_size: Any = 20
    pml_alpha: Any = 2.0
    smooth_p0: bool = True
    extra_sensors: List[dict] = field(default_factory=list)
    seed: Optional[int] = None

    @property
    def voxels(self) -> int:
        return int(np.prod(self.N))

    def to_api(self):
        """(kgrid, medium, source, sensor, kwargs) in this package's types."""
        args = []
        for n, dd in zip(self.N, self.d):
            args += [n, dd]
        g = KWaveGrid(*args)
        g.dt = self.dt
        g.Nt = self.Nt
        g.t_array = np.arange(self.Nt) * self.dt
        kw = dict(pml_size=self.pml_size, pml_alpha=self.pml_alpha, smooth_p0=self.smooth_p0)
        return g, KWaveMedium(**self.medium), KWaveSource(**self.source), KWaveSensor(**self.sensor), kw


def gaussian_random_field(rng: np.random.Generator, shape, sigma_px: float, lo: float, hi: float):
    """Periodic Gaussian-filtered white noise, min-max mapped onto [lo, hi]."""
    w = rng.standard_normal(shape)
    W = np.fft.fftn(w)
    k2 = np.zeros(shape)
    for ax, n in enumerate(shape):
        kv = 2 * math.pi * np.fft.fftfreq(n)
        s = [1] * len(shape)
        s[ax] = n
        k2 = k2 + kv.reshape(s) ** 2
    f = np.real(np.fft.ifftn(W * np.exp(-k2 * sigma_px ** 2 / 2)))
    f = (f - f.min()) / (f.max() - f.min())
    return lo + (hi - lo) * f


def c1(Nt: Optional[int] = None) -> Case:
    """128^2 homogeneous lossless disc source; Nt from t_end = 1.14 * diag / c (689 steps)."""
    g = KWaveGrid(128, 1e-4, 128, 1e-4)
    make_time(g, 1500.0, t_end=1.14 * math.sqrt(2) * 128e-4 / 1500)
    Nt_ = g.Nt if Nt is None else Nt
    p_mask = make_disc(128, 128, 64, 64, 5)
    tb = tone_burst(1 / g.dt, 1e6, 5)
    sig = np.zeros((int(p_mask.sum()), Nt_))
    sig[:, : min(len(tb), Nt_)] = tb[: min(len(tb), Nt_)]
    return Case("c1_128x128_homogeneous", (128, 128), (1e-4, 1e-4), g.dt, Nt_,
                dict(sound_speed=1500.0, density=1000.0),
                dict(p_mask=p_mask, p=sig, p_mode=Additive),
                dict(mask=make_circle(128, 128, 64, 64, 40), record=["p"]))


def c2(n: int = 512, Nt: int = 2000, seed: int = 2002, record=("p_max", "p_rms")) -> Case:
    """n^2 heterogeneous absorbing (y=1.5, :stokes) line-p0 solve with full-grid aggregates."""
    rng = np.random.Generator(np.random.PCG64(seed))
    c = gaussian_random_field(rng, (n, n), 10.0, 1400.0, 1600.0)
    rho = gaussian_random_field(rng, (n, n), 10.0, 900.0, 1100.0)
    dx = 1e-4
    dt = 0.3 * dx / float(c.max())
    p0 = np.zeros((n, n))
    cx = n // 2  # x index 257 (1-based) at n = 512
    p0[cx, n // 2 - 32: n // 2 + 32] = 1e6  # y 225..288 (1-based) at n = 512
    p0 = np.real(np.fft.ifft2(np.fft.fft2(p0) * np.exp(
        -((2 * math.pi * np.fft.fftfreq(n)[:, None]) ** 2 + (2 * math.pi * np.fft.fftfreq(n)[None, :]) ** 2) / 2)))
    return Case(f"c2_{n}x{n}_heterogeneous_absorbing", (n, n), (dx, dx), dt, Nt,
                dict(sound_speed=c, density=rho, alpha_coeff=0.75, alpha_power=1.5, alpha_mode="stokes"),
                dict(p0=p0),
                dict(mask=np.ones((n, n), dtype=bool), record=list(record)), seed=seed)


def c3(n: int = 256, Nt: int = 1500, seed: int = 3003, piston: int = 32, pml: int = 10,
       plane_record=("p",), volume_record=("p_max",)) -> Case:
    """n^3 heterogeneous nonlinear absorbing (y=1.1) ux piston; plane p + volume p_max."""
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = (n, n, n)
    c = gaussian_random_field(rng, shape, 5.0 * n / 256, 1450.0, 1650.0)
    rho = gaussian_random_field(rng, shape, 5.0 * n / 256, 950.0, 1100.0)
    lo, hi = int(round(60 * n / 256)), int(round(196 * n / 256))
    ctr = rng.integers(lo, hi + 1, size=3)
    bona = np.full(shape, 5.0)
    bona[make_ball(n, n, n, int(ctr[0]), int(ctr[1]), int(ctr[2]), 20 * n / 256)] = 9.0
    dx = 2e-4
    dt = 0.3 * dx / float(c.max())
    u_mask = np.zeros(shape, dtype=bool)
    half = piston // 2
    mid = n // 2
    xs = min(11, n - 1)  # plane x = 12 (1-based)
    u_mask[xs, mid - half: mid + half, mid - half: mid + half] = True
    tb = 0.5 * tone_burst(1 / dt, 1e6, 3)
    sig = np.zeros((int(u_mask.sum()), Nt))
    sig[:, : min(len(tb), Nt)] = tb[: min(len(tb), Nt)]
    plane = np.zeros(shape, dtype=bool)
    plane[:, :, n // 2 - 1] = True  # z = 128 (1-based) at n = 256
    case = Case(f"c3_{n}^3_nonlinear_absorbing", shape, (dx, dx, dx), dt, Nt,
                dict(sound_speed=c, density=rho, alpha_coeff=0.5, alpha_power=1.1,
                     alpha_mode="no_dispersion", BonA=bona),
                dict(u_mask=u_mask, ux=sig, u_mode=Additive),
                dict(mask=plane, record=list(plane_record)), pml_size=pml, seed=seed)
    if volume_record:
        case.extra_sensors = [dict(mask=np.ones(shape, dtype=bool), record=list(volume_record))]
    return case


C4_SIDES = (128, 192, 256, 384, 512, 768, 1024)


def c4_sim(i: int, sides=C4_SIDES, nt_range=(500, 4000)) -> Case:
    """Simulation i of the 64-sim mixed-size batch (seed 4004 + i)."""
    rng = np.random.Generator(np.random.PCG64(4004 + i))
    nx, ny = int(rng.choice(sides)), int(rng.choice(sides))
    c = gaussian_random_field(rng, (nx, ny), 10.0, 1400.0, 1600.0)
    rho = gaussian_random_field(rng, (nx, ny), 10.0, 900.0, 1100.0)
    y = float(rng.uniform(1.0, 2.0))
    Nt = int(rng.integers(nt_range[0], nt_range[1] + 1))
    dx = 1e-4
    dt = 0.3 * dx / float(c.max())
    f0 = float(rng.uniform(0.5e6, 3e6))
    cycles = int(rng.integers(3, 6))
    cx, cy = int(rng.integers(nx // 4, 3 * nx // 4)) + 1, int(rng.integers(ny // 4, 3 * ny // 4)) + 1
    if rng.random() < 0.5:
        p_mask = np.zeros((nx, ny), dtype=bool)
        p_mask[cx - 1, cy - 1] = True
    else:
        p_mask = make_disc(nx, ny, cx, cy, int(rng.integers(2, 7)))
    tb = tone_burst(1 / dt, f0, cycles)
    sig = np.zeros((int(p_mask.sum()), Nt))
    sig[:, : min(len(tb), Nt)] = tb[: min(len(tb), Nt)]
    sensor = np.zeros((nx, ny), dtype=bool)
    sx = min(nx - 1, cx - 1 + nx // 8)
    y0 = max(0, cy - 1 - 8)
    sensor[sx, y0: y0 + 16] = True
    return Case(f"c4_{i}_{nx}x{ny}", (nx, ny), (dx, dx), dt, Nt,
                dict(sound_speed=c, density=rho, alpha_coeff=0.75, alpha_power=y, alpha_mode="no_dispersion"),
                dict(p_mask=p_mask, p=sig, p_mode=Additive),
                dict(mask=sensor, record=["p"]), seed=4004 + i)


def smooth_sides(lo: int, hi: int) -> list:
    """2/3/5-smooth integers in [lo, hi]."""
    out = []
    for n in range(lo, hi + 1):
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            out.append(n)
    return out


def c5_request(i: int, seed: int = 5005, nt_range=(500, 1500)):
    """Request i of the serving stream: (arrival offset s, Case)."""
    rng = np.random.Generator(np.random.PCG64((seed, i)))
    if rng.random() < 0.7:
        sides = smooth_sides(256, 1024)
        nx, ny = int(rng.choice(sides)), int(rng.choice(sides))
        shape = (nx, ny)
    else:
        n3 = int(rng.choice([64, 72, 80, 96, 100, 108, 120, 128, 144, 150, 160, 180, 192]))
        shape = (n3, n3, n3)
    D = len(shape)
    c = gaussian_random_field(rng, shape, 5.0, 1400.0, 1600.0)
    rho = gaussian_random_field(rng, shape, 5.0, 900.0, 1100.0)
    dx = 1e-4
    dt = 0.3 * dx / float(c.max())
    Nt = int(rng.integers(nt_range[0], nt_range[1] + 1))
    ctr = [int(rng.integers(n // 4, 3 * n // 4)) for n in shape]
    p_mask = np.zeros(shape, dtype=bool)
    p_mask[tuple(ctr)] = True
    tb = tone_burst(1 / dt, float(rng.uniform(0.5e6, 3e6)), int(rng.integers(3, 6)))
    sig = np.zeros((1, Nt))
    sig[:, : min(len(tb), Nt)] = tb[: min(len(tb), Nt)]
    sensor = np.zeros(shape, dtype=bool)
    idx = list(ctr)
    idx[0] = min(shape[0] - 1, ctr[0] + shape[0] // 8)
    sl = [idx[0]] + [slice(max(0, ctr[a] - 8), max(0, ctr[a] - 8) + 16) if a == 1 else idx[a] for a in range(1, D)]
    sensor[tuple(sl)] = True
    case = Case(f"c5_{i}_{'x'.join(map(str, shape))}", shape, (dx,) * D, dt, Nt,
                dict(sound_speed=c, density=rho, alpha_coeff=0.75, alpha_power=float(rng.uniform(1.0, 2.0)),
                     alpha_mode="no_dispersion"),
                dict(p_mask=p_mask, p=sig, p_mode=Additive),
                dict(mask=sensor, record=["p"]), pml_size=10 if D == 3 else 20, seed=seed)
    return case


@dataclass
class ElasticCase:
    """An elastic-solver workload (pstd_elastic_2d/3d): medium and source keyword dicts for
    ``ElasticMedium`` / ``ElasticSource``."""
    name: str
    N: tuple
    d: tuple
    dt: float
    Nt: int
    medium: dict
    source: dict
    sensor: dict
    pml_size: Any = 10
    pml_alpha: Any = 2.0
    seed: Optional[int] = None

    @property
    def voxels(self) -> int:
        return int(np.prod(self.N))

    def to_api(self):
        """(kgrid, medium, source, sensor, kwargs) in this package's types."""
        from .core import ElasticMedium, ElasticSource
        args = []
        for n, dd in zip(self.N, self.d):
            args += [n, dd]
        g = KWaveGrid(*args)
        g.dt = self.dt
        g.Nt = self.Nt
        g.t_array = np.arange(self.Nt) * self.dt
        kw = dict(pml_size=self.pml_size, pml_alpha=self.pml_alpha)
        return g, ElasticMedium(**self.medium), ElasticSource(**self.source), KWaveSensor(**self.sensor), kw


def elastic3d(n: int = 256, Nt: int = 1000, seed: int = 6006, pml: int = 10) -> ElasticCase:
    """n^3 heterogeneous elastic solid (cp 2600-3200, cs 1100-1600 m/s, rho 1600-2100 kg/m^3,
    Gaussian random fields of sigma 5 px at 256), a p0 ball of radius 6 px at the centre and a
    3 MHz sxx tone burst at one point; the sensor records p on the xy plane z = n/2."""
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = (n, n, n)
    s = 5.0 * n / 256
    cp = gaussian_random_field(rng, shape, s, 2600.0, 3200.0)
    cs = gaussian_random_field(rng, shape, s, 1100.0, 1600.0)
    rho = gaussian_random_field(rng, shape, s, 1600.0, 2100.0)
    dx = 2e-4
    dt = 0.3 * dx / 3200.0
    mid = n // 2
    p0 = np.zeros(shape)
    p0[make_ball(n, n, n, mid, mid, mid, 6 * n / 256)] = 1e5
    s_mask = np.zeros(shape, dtype=bool)
    s_mask[n // 4, mid - 1, mid - 1] = True
    tb = 1e4 * tone_burst(1 / dt, 3e6, 3)
    sig = np.zeros((1, Nt))
    sig[0, : min(len(tb), Nt)] = tb[: min(len(tb), Nt)]
    plane = np.zeros(shape, dtype=bool)
    plane[:, :, mid - 1] = True
    return ElasticCase(f"elastic3d_{n}^3_heterogeneous", shape, (dx, dx, dx), dt, Nt,
                       dict(sound_speed_compression=cp, sound_speed_shear=cs, density=rho),
                       dict(p0=p0, s_mask=s_mask, sxx=sig),
                       dict(mask=plane, record=["p"]), pml_size=pml, seed=seed)
