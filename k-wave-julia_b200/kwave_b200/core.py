"""Host-side data model and FP64 setup helpers, mirroring KWave.jl's user-facing types.

Arrays use the reference's Julia index order: a 2-D field has shape ``(Nx, Ny)`` and is indexed
``a[x, y]``; a mask's points are taken in column-major (x-fastest) order, as Julia's ``findall``
returns them.  Everything here runs once per simulation on the host in FP64 (the reference runs
it on the host too); the time stepping itself is on the GPU (``solver.py``).

Mirrors:
  KWaveGrid / make_time, grid_size,   KWave.jl/src/grid.jl:120-352
  grid_spacing, k_max, total_grid_points
  KWaveMedium                         KWave.jl/src/medium.jl:248-341
  KWaveSource, SourceMode             KWave.jl/src/source.jl:160-230, types.jl:355
  ElasticMedium, ElasticSource        KWave.jl/src/solver/elastic.jl:22-104
  KWaveSensor, SimulationOutput       KWave.jl/src/sensor.jl:31-87
  get_pml, get_optimal_pml_size       KWave.jl/src/pml.jl:25-121
  smooth                              KWave.jl/src/filter/filters.jl:20-73
  tone_burst                          KWave.jl/src/signal/generation.jl:30-71
  db2neper, neper2db                  KWave.jl/src/material/conversion.jl:9-49
  make_disc/circle/line/ball          KWave.jl/src/geometry/shapes.jl:22-278
"""

from __future__ import annotations

import enum
import math
from dataclasses import dataclass
from typing import Any, Optional, Sequence

import numpy as np


class SourceMode(enum.IntEnum):
    """types.jl:355 -- only Dirichlet is distinguished by the solver; both additive modes add."""
    Dirichlet = 0
    Additive = 1
    AdditiveNoCorrection = 2


Dirichlet = SourceMode.Dirichlet
Additive = SourceMode.Additive
AdditiveNoCorrection = SourceMode.AdditiveNoCorrection


# ---------------------------------------------------------------------------------------------
# grid
# ---------------------------------------------------------------------------------------------

def _wavenumbers(N: int, d: float) -> np.ndarray:
    m = np.arange(N)
    m = np.where(m < (N + 1) // 2, m, m - N)
    return m.astype(np.float64) * (2 * math.pi / (N * d))


class KWaveGrid:
    """``KWaveGrid(Nx, dx[, Ny, dy[, Nz, dz]])`` (grid.jl:196-245)."""

    def __init__(self, *args):
        if len(args) not in (2, 4, 6):
            raise TypeError("KWaveGrid(Nx, dx[, Ny, dy[, Nz, dz]])")
        self.N = tuple(int(n) for n in args[0::2])
        self.d = tuple(float(v) for v in args[1::2])
        for n, dd in zip(self.N, self.d):
            if n < 1 or not dd > 0:
                raise ValueError("grid sizes must be >= 1 and spacings > 0")
        self.dt = 0.0
        self.Nt = 0
        self.t_array = np.zeros(0)

    @property
    def ndim(self) -> int:
        return len(self.N)

    def k_vec(self, dim: int) -> np.ndarray:
        """Wavenumber vector of axis ``dim`` in FFT order (grid.jl:120-130)."""
        return _wavenumbers(self.N[dim], self.d[dim])

    def x_vec(self, dim: int) -> np.ndarray:
        n, dd = self.N[dim], self.d[dim]
        return (np.arange(n) - (n - 1) / 2.0) * dd

    def __getattr__(self, name):
        axes = {"x": 0, "y": 1, "z": 2}
        if len(name) == 2 and name[0] in "Nd" and name[1] in axes and axes[name[1]] < len(self.__dict__.get("N", ())):
            a = axes[name[1]]
            return self.N[a] if name[0] == "N" else self.d[a]
        raise AttributeError(name)

    def total_grid_points(self) -> int:
        return int(np.prod(self.N))


def total_grid_points(grid: KWaveGrid) -> int:
    """grid.jl:260-262."""
    return grid.total_grid_points()


def grid_size(grid: KWaveGrid) -> tuple:
    """grid.jl:269-271: (Nx[, Ny[, Nz]])."""
    return tuple(grid.N)


def grid_spacing(grid: KWaveGrid) -> tuple:
    """grid.jl:278-280: (dx[, dy[, dz]])."""
    return tuple(grid.d)


def k_max(grid: KWaveGrid) -> float:
    """grid.jl:294-296: the Nyquist wavenumber pi / max spacing [rad/m]."""
    return min(math.pi / d for d in grid.d)


def make_time(grid: KWaveGrid, sound_speed, cfl: float = 0.3, t_end: Optional[float] = None):
    """``make_time!`` (grid.jl:320-352): dt = cfl*min(d)/max(c), Nt = ceil(t_end/dt) + 1."""
    c_max = float(np.max(sound_speed))
    c_min = float(np.min(sound_speed))
    dt = cfl * min(grid.d) / c_max
    grid.dt = dt
    if t_end is None:
        diag = math.sqrt(sum((n * dd) ** 2 for n, dd in zip(grid.N, grid.d)))
        t_end = 2.0 * diag / c_min
    Nt = int(math.ceil(t_end / dt)) + 1
    grid.Nt = Nt
    grid.t_array = np.arange(Nt) * dt
    return dt, Nt


# ---------------------------------------------------------------------------------------------
# medium / source / sensor / output
# ---------------------------------------------------------------------------------------------

@dataclass
class KWaveMedium:
    """``KWaveMedium(; sound_speed, density=1.0, alpha_coeff, alpha_power, alpha_mode, BonA)``."""
    sound_speed: Any
    density: Any = 1.0
    alpha_coeff: Any = None
    alpha_power: Optional[float] = None
    alpha_mode: str = "no_absorption"
    BonA: Any = None

    def is_lossless(self) -> bool:  # medium.jl:90
        return self.alpha_coeff is None or self.alpha_mode == "no_absorption"

    def is_homogeneous(self) -> bool:
        return np.ndim(self.sound_speed) == 0 and np.ndim(self.density) == 0

    def is_nonlinear(self) -> bool:
        return self.BonA is not None


@dataclass
class KWaveSource:
    """``KWaveSource(; p0, p_mask, p, p_mode=Additive, u_mask, ux, uy, uz, u_mode=Additive)``."""
    p0: Any = None
    p_mask: Any = None
    p: Any = None
    p_mode: SourceMode = Additive
    u_mask: Any = None
    ux: Any = None
    uy: Any = None
    uz: Any = None
    u_mode: SourceMode = Additive

    def has_p0(self) -> bool:
        return self.p0 is not None

    def has_pressure_source(self) -> bool:
        return self.p_mask is not None and self.p is not None

    def has_velocity_source(self) -> bool:
        return self.u_mask is not None


@dataclass
class ElasticMedium:
    """``ElasticMedium(; sound_speed_compression, sound_speed_shear, density=1000.0,
    alpha_coeff_compression, alpha_coeff_shear, alpha_power)`` (solver/elastic.jl:22-48)."""
    sound_speed_compression: Any
    sound_speed_shear: Any
    density: Any = 1000.0
    alpha_coeff_compression: Any = None
    alpha_coeff_shear: Any = None
    alpha_power: Optional[float] = None


@dataclass
class ElasticSource:
    """``ElasticSource(; s_mask, sxx, syy, szz, sxy, sxz, syz, s_mode=Additive, u_mask, ux, uy,
    uz, u_mode=Additive, p0)`` (solver/elastic.jl:57-104)."""
    s_mask: Any = None
    sxx: Any = None
    syy: Any = None
    szz: Any = None
    sxy: Any = None
    sxz: Any = None
    syz: Any = None
    s_mode: SourceMode = Additive
    u_mask: Any = None
    ux: Any = None
    uy: Any = None
    uz: Any = None
    u_mode: SourceMode = Additive
    p0: Any = None

    def has_stress_source(self) -> bool:  # elastic.jl:106
        return self.s_mask is not None

    def has_velocity_source(self) -> bool:
        return self.u_mask is not None

    def has_p0(self) -> bool:
        return self.p0 is not None


VALID_RECORD_FIELDS = frozenset(["p", "p_max", "p_min", "p_rms", "p_final", "ux", "uy", "uz",
                                 "u_max", "u_rms", "u_final", "I_avg", "I_max"])


@dataclass
class KWaveSensor:
    """``KWaveSensor(; mask, record=[:p], time_reversal_boundary_data, directivity_angle,
    directivity_size, frequency_response)`` (sensor.jl:31-38)."""
    mask: Any = None
    record: Sequence[str] = ("p",)
    time_reversal_boundary_data: Any = None
    directivity_angle: Any = None
    directivity_size: Optional[float] = None
    frequency_response: Any = None

    def is_time_reversal(self) -> bool:
        return self.time_reversal_boundary_data is not None


def validate_record_fields(sensor: KWaveSensor):
    """sensor.jl:52-58."""
    for f in sensor.record:
        if f not in VALID_RECORD_FIELDS:
            raise ValueError(f"Invalid sensor record field: :{f}. Valid fields: "
                             + ", ".join(sorted(VALID_RECORD_FIELDS)))


class SimulationOutput:
    """sensor.jl:76-87 -- ``out["p"]``, ``"p" in out``, ``out.keys()``."""

    def __init__(self, data: dict):
        self.data = data

    def __getitem__(self, key):
        return self.data[key]

    def __contains__(self, key):
        return key in self.data

    def keys(self):
        return self.data.keys()

    def __repr__(self):
        return "SimulationOutput with fields: " + ", ".join(sorted(self.data))


# ---------------------------------------------------------------------------------------------
# setup helpers (FP64, host)
# ---------------------------------------------------------------------------------------------

def get_pml(N: int, d: float, pml_size: int, pml_alpha: float, dt: float, staggered: bool = False):
    """pml.jl:25-56 -- 1-D profile exp(-alpha pos^4 dt) on both ends."""
    pml = np.ones(N)
    for i in range(1, pml_size + 1):
        pos = ((pml_size - i + 0.5) if staggered else (pml_size - i + 1)) / pml_size
        val = math.exp(-(pml_alpha * pos ** 4) * dt)
        pml[i - 1] = val
        pml[N - i] = val
    return pml


def _max_prime_factor(n: int) -> int:
    best, p, m = 1, 2, n
    while p * p <= m:
        while m % p == 0:
            best, m = max(best, p), m // p
        p += 1
    return max(best, m) if m > 1 else best


def get_optimal_pml_size(grid_size, pml_range=range(10, 61)):
    """pml.jl:74-121 -- PML size whose total grid side has the smallest largest prime factor."""
    def one(n):
        scores = [(_max_prime_factor(n + 2 * s), k, s) for k, s in enumerate(pml_range)]
        return min(scores)[2]
    return one(grid_size) if isinstance(grid_size, int) else tuple(one(n) for n in grid_size)


def db2neper(alpha, alpha_power=None):
    """conversion.jl:9, 34 (the two-argument form keeps the reference's 1e-2 factor)."""
    if alpha_power is None:
        return np.asarray(alpha) / (20 * math.log10(math.e))
    return alpha * (1e-2 / (20 * math.log10(math.e))) * (2 * math.pi * 1e6) ** (-alpha_power)


def neper2db(alpha):
    return np.asarray(alpha) * (20 * math.log10(math.e))


def _blackman(N: int) -> np.ndarray:
    if N == 1:
        return np.ones(1)
    n = np.arange(N)
    return 0.42 - 0.5 * np.cos(2 * math.pi * n / (N - 1)) + 0.08 * np.cos(4 * math.pi * n / (N - 1))


def smooth(matrix, restore_max: bool = False) -> np.ndarray:
    """filters.jl:20-60 -- FFT, multiply by the Blackman window circularly shifted by floor(N/2),
    inverse FFT, axis after axis; keep the real part; optionally restore max |.|."""
    m = np.asarray(matrix, dtype=np.float64)
    res = m.astype(np.complex128)
    for d in range(m.ndim):
        shape = [1] * m.ndim
        shape[d] = -1
        win = np.roll(_blackman(m.shape[d]), m.shape[d] // 2).reshape(shape)
        res = np.fft.ifft(np.fft.fft(res, axis=d) * win, axis=d)
    out = np.real(res)
    if restore_max:
        smax = np.max(np.abs(out))
        if smax > 0:
            out = out * (np.max(np.abs(m)) / smax)
    return out


def tone_burst(sample_freq: float, signal_freq: float, num_cycles: int, envelope: str = "gaussian",
               signal_offset: int = 0) -> np.ndarray:
    """generation.jl:30-71."""
    tone_length = num_cycles / signal_freq
    dt = 1.0 / sample_freq
    N = int(round(tone_length / dt))
    t = np.arange(N) * dt
    carrier = np.sin(2 * math.pi * signal_freq * t)
    if envelope == "gaussian":
        sigma = tone_length / (2 * num_cycles)
        env = np.exp(-((t - tone_length / 2) / sigma) ** 2 / 2)
    elif envelope == "rectangular":
        env = np.ones(N)
    elif envelope == "cosine":
        env = 0.5 * (1.0 - np.cos(2 * math.pi * np.arange(N) / (N - 1)))
    else:
        raise ValueError(f"Unknown envelope type: {envelope}. Use :gaussian, :rectangular, or :cosine")
    sig = carrier * env
    return np.concatenate([np.zeros(signal_offset), sig]) if signal_offset > 0 else sig


def make_disc(Nx: int, Ny: int, cx, cy, radius) -> np.ndarray:
    """shapes.jl:22-38 -- filled disc, 1-based centre."""
    i = np.arange(1, Nx + 1)[:, None] - int(round(cx))
    j = np.arange(1, Ny + 1)[None, :] - int(round(cy))
    return i * i + j * j <= radius ** 2


def make_ball(Nx, Ny, Nz, cx, cy, cz, radius) -> np.ndarray:
    """shapes.jl:260-278 -- filled ball, 1-based centre."""
    i = np.arange(1, Nx + 1)[:, None, None] - int(round(cx))
    j = np.arange(1, Ny + 1)[None, :, None] - int(round(cy))
    k = np.arange(1, Nz + 1)[None, None, :] - int(round(cz))
    return i * i + j * j + k * k <= radius ** 2


def make_circle(Nx: int, Ny: int, cx, cy, radius) -> np.ndarray:
    """shapes.jl:56-113 -- midpoint-circle perimeter (full circle)."""
    out = np.zeros((Nx, Ny), dtype=bool)
    cx, cy, r = int(round(cx)), int(round(cy)), int(round(radius))
    x, y, dd = r, 0, 1 - r
    pts = []
    while x >= y:
        pts += [(cx + x, cy + y), (cx - x, cy + y), (cx + x, cy - y), (cx - x, cy - y),
                (cx + y, cy + x), (cx - y, cy + x), (cx + y, cy - x), (cx - y, cy - x)]
        y += 1
        if dd <= 0:
            dd += 2 * y + 1
        else:
            x -= 1
            dd += 2 * (y - x) + 1
    for px, py in pts:
        if 1 <= px <= Nx and 1 <= py <= Ny:
            out[px - 1, py - 1] = True
    return out


def make_line(Nx: int, Ny: int, startpoint, endpoint) -> np.ndarray:
    """shapes.jl:185-218 -- Bresenham line, 1-based end points."""
    out = np.zeros((Nx, Ny), dtype=bool)
    (x1, y1), (x2, y2) = startpoint, endpoint
    dx, dy = abs(x2 - x1), abs(y2 - y1)
    sx, sy = (1 if x1 < x2 else -1), (1 if y1 < y2 else -1)
    err, x, y = dx - dy, x1, y1
    while True:
        if 1 <= x <= Nx and 1 <= y <= Ny:
            out[x - 1, y - 1] = True
        if x == x2 and y == y2:
            return out
        e2 = 2 * err
        if e2 > -dy:
            err -= dy
            x += sx
        if e2 < dx:
            err += dx
            y += sy
