"""CPU restatement of KWave.jl's fluid k-space time-stepping path -- TEST INFRASTRUCTURE ONLY.

This module is the oracle.  It is used as the checker by ``tests/``, by
``__graft_entry__.smoke()`` and as the timed CPU baseline in ``bench.py``.  It is never
imported by the product path (``k-wave-julia_b200/kwave_b200``), which fails loudly when its
CUDA library is missing instead of falling back here.

What it restates (paths relative to the KWave.jl project, ``KWave.jl/src/...``):

* grids, wavenumbers, staggered shift operators, ``make_time!``   -- ``grid.jl:120-153, 196-245, 320-352``
* ``get_pml``                                                    -- ``pml.jl:25-56``
* ``spectral_gradient!``                                          -- ``fft_utils.jl:126-182``
* ``_precompute_absorption``, ``_compute_kappa``                  -- ``solver/first_order.jl:13-42``
* ``kspace_first_order`` 1D/2D/3D drivers                         -- ``solver/first_order.jl:92-728``
* staggered density, p0 initialisation, EOS, time steps,
  source injection, sensor recording/finalisation, post filters   -- ``solver/first_order_steps.jl:40-910``
* sensor data allocation                                          -- ``sensor.jl:94-135``
* setup helpers: ``smooth`` (``filter/filters.jl:20-73``), ``tone_burst``
  (``signal/generation.jl:30-71``), ``db2neper``/``neper2db`` (``material/conversion.jl:34-49``),
  ``make_disc``/``make_circle``/``make_line``/``make_ball`` (``geometry/shapes.jl:22-278``).

Array convention: every grid array has the reference's Julia shape ``(Nx, Ny, Nz)`` and index
order ``a[x, y, z]``; "linear index" means the column-major (x-fastest) index that Julia's
``findall`` returns, i.e. ``a.ravel(order="F")``.  FFTs are scipy's pocketfft over the reversed
axis list, so the halved real-FFT axis is x, exactly like FFTW's ``plan_rfft`` on a Julia array.

Precision: ``dtype=np.float64`` (default) is the FP64 solve every GPU result is compared with.
``dtype=np.float32`` mirrors the reference's ``data_cast=Float32`` mixed-precision semantics
(fields, FFTs and pre-cast operators in FP32; FP64 PML/medium operands promoted per element and
rounded on store) and exists only to size the reference's own FP32 error.

Parity pinning: the reference cannot run in this environment (no Julia), and its test suite pins
no solver output values -- solver-level parity against the Julia binary is therefore unpinned.
This restatement is pinned on (i) every known-answer and property test the reference's own
suite holds for this path (``test/test_fft.jl``, ``test_pml.jl``, ``test_grid.jl``,
``test_filter.jl``, ``test_signal.jl``, ``test_geometry.jl``, ``test_solver_{1,2,3}d.jl``,
``test_absorption.jl``, ``test_time_reversal.jl``), restated in ``tests/test_oracle_kat.py``, and
(ii) a closed-form known answer for the reference's own discrete scheme: with a homogeneous
lossless medium and no PML every Fourier mode evolves by a fixed 2x2 recurrence (kappa applied
once in the EOS, u(-dt/2) = -dt/(2 rho0) dp0/dx as in first_order_steps.jl:86-136), so
the stepped solution must equal that recurrence evaluated mode by mode.  (The reference scheme is
not d'Alembert-exact: it applies kappa once, and its u(-dt/2) has the opposite sign to k-Wave's.)
Solver-level parity therefore rests on this restatement: "parity unpinned" against the Julia
binary, pinned on the reference's own tests and on (ii).
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Any, Optional, Sequence

import numpy as np
import scipy.fft as sfft

# scipy.fft worker threads: all host cores unless KWB_ORACLE_WORKERS says otherwise
_WORKERS = int(os.environ.get("KWB_ORACLE_WORKERS", "0")) or os.cpu_count() or 1

DIRICHLET, ADDITIVE, ADDITIVE_NO_CORRECTION = 0, 1, 2  # types.jl:11 (@enum SourceMode)

VALID_RECORD_FIELDS = frozenset(
    ["p", "p_max", "p_min", "p_rms", "p_final", "ux", "uy", "uz",
     "u_max", "u_rms", "u_final", "I_avg", "I_max"])  # sensor.jl:41-45


# ---------------------------------------------------------------------------------------------
# grid.jl
# ---------------------------------------------------------------------------------------------

def make_wavenumber_vec(N: int, d: float) -> np.ndarray:
    """grid.jl:120-130 -- [0..N/2-1, -N/2..-1]*2pi/(N d) (even N), [0..(N-1)/2, -(N-1)/2..-1] (odd)."""
    dk = 2 * math.pi / (N * d)
    if N % 2 == 0:
        kv = np.concatenate([np.arange(0, N // 2), np.arange(-N // 2, 0)]).astype(np.float64)
    else:
        kv = np.concatenate([np.arange(0, (N - 1) // 2 + 1), np.arange(-((N - 1) // 2), 0)]).astype(np.float64)
    return kv * dk


def make_spatial_vec(N: int, d: float) -> np.ndarray:
    """grid.jl:137-139."""
    return (np.arange(N) - (N - 1) / 2.0) * d


def make_shift_operators(kv: np.ndarray, d: float):
    """grid.jl:149-153 -- exp(+i k d/2), exp(-i k d/2)."""
    return np.exp(1j * kv * d / 2), np.exp(-1j * kv * d / 2)


class KWaveGrid:
    """grid.jl:196-245 -- ``KWaveGrid(Nx, dx[, Ny, dy[, Nz, dz]])``."""

    def __init__(self, *args):
        if len(args) not in (2, 4, 6):
            raise TypeError("KWaveGrid(Nx, dx[, Ny, dy[, Nz, dz]])")
        self.N = tuple(int(n) for n in args[0::2])
        self.d = tuple(float(v) for v in args[1::2])
        self.ndim = len(self.N)
        self.k_vecs = [make_wavenumber_vec(n, dd) for n, dd in zip(self.N, self.d)]
        self.x_vecs = [make_spatial_vec(n, dd) for n, dd in zip(self.N, self.d)]
        self.shift_pos, self.shift_neg = [], []
        for kv, dd in zip(self.k_vecs, self.d):
            sp, sn = make_shift_operators(kv, dd)
            self.shift_pos.append(sp)
            self.shift_neg.append(sn)
        self.dt = 0.0
        self.Nt = 0
        self.t_array = np.zeros(0)

    @property
    def k(self) -> np.ndarray:
        """Full-grid |k| (grid.jl:205, 227-231)."""
        acc = np.zeros(self.N)
        for dim, kv in enumerate(self.k_vecs):
            shape = [1] * self.ndim
            shape[dim] = -1
            acc = acc + kv.reshape(shape) ** 2
        return np.sqrt(acc)

    @property
    def Nx(self):
        return self.N[0]

    @property
    def dx(self):
        return self.d[0]


def make_time(grid: KWaveGrid, sound_speed, cfl: float = 0.3, t_end: Optional[float] = None):
    """grid.jl:320-352 (``make_time!``): dt = cfl*d_min/c_max, Nt = ceil(t_end/dt) + 1."""
    c_max = float(np.max(sound_speed))
    c_min = float(np.min(sound_speed))
    d_min = min(grid.d)
    dt = cfl * d_min / c_max
    grid.dt = dt
    if t_end is None:
        diag = math.sqrt(sum((n * dd) ** 2 for n, dd in zip(grid.N, grid.d)))
        t_end = 2.0 * diag / c_min
    Nt = int(math.ceil(t_end / dt)) + 1
    grid.Nt = Nt
    grid.t_array = np.arange(Nt) * dt
    return dt, Nt


# ---------------------------------------------------------------------------------------------
# pml.jl, material/conversion.jl, filter/filters.jl, signal/generation.jl, geometry/shapes.jl
# ---------------------------------------------------------------------------------------------

def get_pml(N: int, d: float, pml_size: int, pml_alpha: float, dt: float, staggered: bool = False):
    """pml.jl:25-56 -- exp(-alpha*pos^4*dt), pos=(size-i+1)/size or (size-i+0.5)/size, both ends."""
    pml = np.ones(N)
    if pml_size == 0:
        return pml
    for i in range(1, pml_size + 1):
        pos = (pml_size - i + 0.5) / pml_size if staggered else (pml_size - i + 1) / pml_size
        val = math.exp(-(pml_alpha * pos ** 4) * dt)
        pml[i - 1] = val
        pml[N - i] = val
    return pml


def max_prime_factor(n: int) -> int:
    """pml.jl:87-105."""
    if n <= 1:
        return 1
    best, dd, m = 1, 2, n
    while dd * dd <= m:
        while m % dd == 0:
            best = max(best, dd)
            m //= dd
        dd += 1
    if m > 1:
        best = max(best, m)
    return best


def get_optimal_pml_size(grid_size, pml_range=range(10, 61)):
    """pml.jl:74-121."""
    def one(n):
        best_pml, best_score = pml_range[0], 1 << 62
        for s in pml_range:
            score = max_prime_factor(n + 2 * s)
            if score < best_score:
                best_score, best_pml = score, s
        return best_pml
    if isinstance(grid_size, int):
        return one(grid_size)
    return tuple(one(n) for n in grid_size)


def db2neper(alpha_coeff, alpha_power=None):
    """material/conversion.jl:9, 34 -- note the reference's 1e-2 factor."""
    if alpha_power is None:
        return np.asarray(alpha_coeff) / (20 * math.log10(math.e))
    return alpha_coeff * (1e-2 / (20 * math.log10(math.e))) * (2 * math.pi * 1e6) ** (-alpha_power)


def neper2db(alpha_neper):
    """material/conversion.jl:49."""
    return np.asarray(alpha_neper) * (20 * math.log10(math.e))


def blackman_window(N: int) -> np.ndarray:
    """filter/filters.jl:67-73 (symmetric Blackman, denominator N-1)."""
    if N == 1:
        return np.ones(1)
    n = np.arange(N)
    return 0.42 - 0.5 * np.cos(2 * math.pi * n / (N - 1)) + 0.08 * np.cos(4 * math.pi * n / (N - 1))


def smooth(matrix: np.ndarray, restore_max: bool = False, dtype=np.float64) -> np.ndarray:
    """filter/filters.jl:20-60 -- per-axis FFT * fftshift(Blackman) * IFFT, real part, restore max.

    Julia's ``fftshift(x, d)`` is a circular shift by floor(N/2), the same as numpy's; for odd N
    it is not the inverse shift, and the reference keeps that off-by-one, so this does too.
    """
    m = np.asarray(matrix, dtype=dtype)
    cdt = np.complex64 if dtype == np.float32 else np.complex128
    result = m.astype(cdt)
    for d in range(m.ndim):
        N = m.shape[d]
        win = blackman_window(N)
        shape = [1] * m.ndim
        shape[d] = N
        win_fft = np.fft.fftshift(win).reshape(shape).astype(dtype)
        result = sfft.fft(result, axis=d, workers=_WORKERS)
        result = result * win_fft
        result = sfft.ifft(result, axis=d, workers=_WORKERS)
    smoothed = np.real(result).astype(dtype)
    if restore_max:
        orig_max = np.max(np.abs(m))
        smooth_max = np.max(np.abs(smoothed))
        if smooth_max > 0:
            smoothed = smoothed * (orig_max / smooth_max)
    return smoothed.astype(dtype)


def tone_burst(sample_freq: float, signal_freq: float, num_cycles: int, envelope: str = "gaussian",
               signal_offset: int = 0) -> np.ndarray:
    """signal/generation.jl:30-71."""
    tone_length = num_cycles / signal_freq
    dt = 1.0 / sample_freq
    N = int(round(tone_length / dt))  # Julia round: ties to even; numpy/python round match
    t = np.arange(N) * dt
    carrier = np.sin(2 * math.pi * signal_freq * t)
    if envelope == "gaussian":
        t_center = tone_length / 2
        sigma = tone_length / (2 * num_cycles)
        env = np.exp(-((t - t_center) / sigma) ** 2 / 2)
    elif envelope == "rectangular":
        env = np.ones(N)
    elif envelope == "cosine":
        env = np.array([0.5 * (1.0 - math.cos(2 * math.pi * (i - 1) / (N - 1))) for i in range(1, N + 1)])
    else:
        raise ValueError(f"Unknown envelope type: {envelope}")
    sig = carrier * env
    if signal_offset > 0:
        sig = np.concatenate([np.zeros(signal_offset), sig])
    return sig


def make_disc(Nx: int, Ny: int, cx: int, cy: int, radius: float) -> np.ndarray:
    """geometry/shapes.jl:22-38 (1-based centre)."""
    i = np.arange(1, Nx + 1).reshape(-1, 1)
    j = np.arange(1, Ny + 1).reshape(1, -1)
    return (i - int(round(cx))) ** 2 + (j - int(round(cy))) ** 2 <= radius ** 2


def make_ball(Nx, Ny, Nz, cx, cy, cz, radius) -> np.ndarray:
    """geometry/shapes.jl:260-278 (1-based centre)."""
    i = np.arange(1, Nx + 1).reshape(-1, 1, 1)
    j = np.arange(1, Ny + 1).reshape(1, -1, 1)
    k = np.arange(1, Nz + 1).reshape(1, 1, -1)
    return (i - int(round(cx))) ** 2 + (j - int(round(cy))) ** 2 + (k - int(round(cz))) ** 2 <= radius ** 2


def make_circle(Nx: int, Ny: int, cx: int, cy: int, radius: int) -> np.ndarray:
    """geometry/shapes.jl:56-113 -- midpoint circle (full circle only)."""
    mask = np.zeros((Nx, Ny), dtype=bool)
    cx, cy, r = int(round(cx)), int(round(cy)), int(round(radius))

    def setp(px, py):
        if 1 <= px <= Nx and 1 <= py <= Ny:
            mask[px - 1, py - 1] = True

    x, y, dd = r, 0, 1 - r
    while x >= y:
        for px, py in ((cx + x, cy + y), (cx - x, cy + y), (cx + x, cy - y), (cx - x, cy - y),
                       (cx + y, cy + x), (cx - y, cy + x), (cx + y, cy - x), (cx - y, cy - x)):
            setp(px, py)
        y += 1
        if dd <= 0:
            dd += 2 * y + 1
        else:
            x -= 1
            dd += 2 * (y - x) + 1
    return mask


def make_line(Nx: int, Ny: int, startpoint, endpoint) -> np.ndarray:
    """geometry/shapes.jl:185-218 -- Bresenham (1-based points)."""
    mask = np.zeros((Nx, Ny), dtype=bool)
    x1, y1 = startpoint
    x2, y2 = endpoint
    dx, dy = abs(x2 - x1), abs(y2 - y1)
    sx = 1 if x1 < x2 else -1
    sy = 1 if y1 < y2 else -1
    err = dx - dy
    x, y = x1, y1
    while True:
        if 1 <= x <= Nx and 1 <= y <= Ny:
            mask[x - 1, y - 1] = True
        if x == x2 and y == y2:
            break
        e2 = 2 * err
        if e2 > -dy:
            err -= dy
            x += sx
        if e2 < dx:
            err += dx
            y += sy
    return mask


# ---------------------------------------------------------------------------------------------
# medium.jl, source.jl, sensor.jl
# ---------------------------------------------------------------------------------------------

@dataclass
class KWaveMedium:
    """medium.jl:248-306."""
    sound_speed: Any
    density: Any = 1.0
    alpha_coeff: Any = None
    alpha_power: Optional[float] = None
    alpha_mode: str = "no_absorption"
    BonA: Any = None

    def is_lossless(self):  # medium.jl:90
        return self.alpha_coeff is None or self.alpha_mode == "no_absorption"


@dataclass
class KWaveSource:
    """source.jl:160-230."""
    p0: Any = None
    p_mask: Any = None
    p: Any = None
    p_mode: int = ADDITIVE
    u_mask: Any = None
    ux: Any = None
    uy: Any = None
    uz: Any = None
    u_mode: int = ADDITIVE


@dataclass
class KWaveSensor:
    """sensor.jl:31-38."""
    mask: Any = None
    record: Sequence[str] = ("p",)
    time_reversal_boundary_data: Any = None
    directivity_angle: Any = None
    directivity_size: Optional[float] = None
    frequency_response: Any = None


def _is_scalar(x) -> bool:
    return np.ndim(x) == 0


def _flatF(a: np.ndarray) -> np.ndarray:
    """Column-major (Julia linear-index) view of an F-contiguous array."""
    return a.reshape(-1, order="F")


def findall(mask) -> np.ndarray:
    """Julia ``findall`` on a Bool array: sorted column-major linear indices (0-based here)."""
    return np.flatnonzero(np.asarray(mask, dtype=bool).ravel(order="F"))


def _signal_2d(sig) -> np.ndarray:
    """A Vector signal indexes as an n x 1 matrix in the reference (``size(v, 2) == 1``)."""
    s = np.asarray(sig, dtype=np.float64)
    return s.reshape(-1, 1) if s.ndim == 1 else s


def _create_sensor_data(sensor: KWaveSensor, Nt: int) -> dict:
    """sensor.jl:94-135."""
    data: dict = {}
    if sensor.mask is None:
        return data
    m = np.asarray(sensor.mask)
    n_sensor = int(np.count_nonzero(m)) if m.dtype == bool else int(m.shape[1])
    for f in sensor.record:
        if f == "p":
            data["p"] = np.zeros((n_sensor, Nt))
        elif f == "p_max":
            data["p_max"] = np.full(n_sensor, -np.inf)
        elif f == "p_min":
            data["p_min"] = np.full(n_sensor, np.inf)
        elif f in ("p_rms", "p_final", "u_rms", "u_final", "I_avg"):
            data[f] = np.zeros(n_sensor)
        elif f in ("ux", "uy", "uz"):
            data[f] = np.zeros((n_sensor, Nt))
        elif f in ("u_max", "I_max"):
            data[f] = np.full(n_sensor, -np.inf)
    return data


# ---------------------------------------------------------------------------------------------
# fft_utils.jl, solver/first_order.jl helpers
# ---------------------------------------------------------------------------------------------

class _Plans:
    """fft_utils.jl:139-183 -- rfft over all dims with x (axis 0) halved."""

    def __init__(self, shape):
        self.shape = tuple(shape)
        self.nd = len(shape)
        self.axes = tuple(range(self.nd - 1, -1, -1))
        self.s = tuple(self.shape[a] for a in self.axes)
        self.n1 = self.shape[0] // 2 + 1

    def forward(self, f):
        return sfft.rfftn(f, axes=self.axes, workers=_WORKERS)

    def inverse(self, F):
        return sfft.irfftn(F, s=self.s, axes=self.axes, workers=_WORKERS)


def spectral_gradient(f, k_vec, shift_op, plans: _Plans, dim: int, dtype=np.float64):
    """fft_utils.jl:247-303 -- irfft(im * k_d * shift_d * rfft(f)), k/shift truncated to n1 for dim 0."""
    ct = np.complex64 if dtype == np.float32 else np.complex128
    F = plans.forward(f)
    if dim == 0:
        kv = np.asarray(k_vec[: plans.n1], dtype=dtype)
        sv = np.asarray(shift_op[: plans.n1], dtype=ct)
    else:
        kv = np.asarray(k_vec, dtype=dtype)
        sv = np.asarray(shift_op, dtype=ct)
    shape = [1] * plans.nd
    shape[dim] = -1
    kv = kv.reshape(shape)
    sv = sv.reshape(shape)
    F = (1j * kv).astype(ct) * sv * F
    return plans.inverse(F.astype(ct)).astype(dtype)


def compute_kappa(k_grid: np.ndarray, c_ref: float, dt: float) -> np.ndarray:
    """solver/first_order.jl:35-42 -- sinc(c_ref*k*dt/2); 1 only where the argument is exactly 0."""
    arg = c_ref * k_grid * dt / 2
    with np.errstate(invalid="ignore", divide="ignore"):
        kap = np.where(arg == 0, 1.0, np.sin(arg) / np.where(arg == 0, 1.0, arg))
    return kap


@dataclass
class AbsorptionParams:
    """solver/first_order_steps.jl:22-28."""
    tau: float
    eta: float
    nabla1: np.ndarray
    nabla2: np.ndarray
    mode: str


def precompute_absorption(medium: KWaveMedium, k_grid: np.ndarray, c_ref: float):
    """solver/first_order.jl:13-30 (tau = -2 a c^(y-1), eta = 2 a c^(y-1) tan(pi y/2))."""
    if medium.is_lossless():
        return None
    if not _is_scalar(medium.alpha_coeff):
        # T(absorb_tau) on an array raises in the reference (first_order.jl:369)
        raise TypeError("array alpha_coeff is not supported by the reference solver")
    if medium.alpha_power is None:
        raise TypeError("alpha_power must be set when alpha_coeff is set")
    y = float(medium.alpha_power)
    a = db2neper(float(medium.alpha_coeff), y)
    tau = -2 * a * c_ref ** (y - 1)
    eta = 2 * a * c_ref ** (y - 1) * math.tan(math.pi * y / 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        nabla1 = tau * k_grid ** y
        nabla2 = eta * k_grid ** (y - 1)
    return AbsorptionParams(tau, eta, nabla1, nabla2, medium.alpha_mode)


def stagger_density(rho0: np.ndarray, dim: int) -> np.ndarray:
    """solver/first_order_steps.jl:40-52 -- (rho0 + circshift(rho0, -e_dim))/2, periodic."""
    return (rho0 + np.roll(rho0, -1, axis=dim)) / 2


def _compute_pressure(rho_total, rho_total_prev, kappa_r, c0, rho0, BonA, absorb, plans, dt, dtype):
    """solver/first_order_steps.jl:214-290 -- five EOS branches."""
    ct = np.complex64 if dtype == np.float32 else np.complex128
    is_absorbing = absorb is not None and absorb.mode != "no_absorption"
    is_nonlinear = BonA is not None
    if _is_scalar(c0):
        c_sq = dtype(c0) ** 2
        if is_nonlinear:
            tmp = (rho_total * (1 + BonA / 2 * rho_total / rho0)).astype(dtype)
            s1 = plans.forward(tmp)
        else:
            s1 = plans.forward(rho_total)
        if not is_absorbing:
            s1 = (c_sq * kappa_r * s1).astype(ct)
        elif absorb.mode == "no_dispersion" or rho_total_prev is None:
            s1 = (c_sq * kappa_r * (1 + absorb.nabla1) * s1).astype(ct)
        else:
            if is_nonlinear:
                prev_eff = rho_total_prev * (1 + BonA / 2 * rho_total_prev / rho0)
                tmp2 = ((tmp - prev_eff) / dt).astype(dtype)
            else:
                tmp2 = ((rho_total - rho_total_prev) / dt).astype(dtype)
            s2 = plans.forward(tmp2)
            s1 = (c_sq * kappa_r * ((1 + absorb.nabla1) * s1 - absorb.nabla2 * s2)).astype(ct)
        return plans.inverse(s1).astype(dtype)
    if is_nonlinear:
        tmp = (c0 ** 2 * rho_total * (1 + BonA / 2 * rho_total / rho0)).astype(dtype)
    else:
        tmp = (c0 ** 2 * rho_total).astype(dtype)
    s1 = plans.forward(tmp)
    if not is_absorbing:
        s1 = (kappa_r * s1).astype(ct)
    else:
        s1 = (kappa_r * (1 + absorb.nabla1) * s1).astype(ct)
    return plans.inverse(s1).astype(dtype)


def _record(sensor_data, record, p, vel, mask_idx, t_index, Nt):
    """solver/first_order_steps.jl:728-811 (t_index is 1-based, as in the reference)."""
    pf = _flatF(p)[mask_idx].astype(np.float64)
    vf = [_flatF(v)[mask_idx] for v in vel]

    def umag():
        acc = np.zeros(len(mask_idx))
        for v in vf:
            acc = acc + (v * v).astype(np.float64)  # v[idx]^2 in the field type, then promoted
        return np.sqrt(acc)

    def intensity():
        acc = np.zeros(len(mask_idx))
        for v in vf:
            acc = acc + (pf * v.astype(np.float64)) ** 2
        return np.sqrt(acc)

    for f in record:
        if f == "p":
            sensor_data["p"][:, t_index - 1] = pf
        elif f == "p_max":
            sensor_data["p_max"] = np.maximum(sensor_data["p_max"], pf)
        elif f == "p_min":
            sensor_data["p_min"] = np.minimum(sensor_data["p_min"], pf)
        elif f == "p_rms":
            sensor_data["p_rms"] = sensor_data["p_rms"] + (_flatF(p)[mask_idx] ** 2).astype(np.float64)
        elif f == "p_final" and t_index == Nt:
            sensor_data["p_final"] = pf.copy()
        elif f in ("ux", "uy", "uz") and "xyz".index(f[1]) < len(vel):
            sensor_data[f][:, t_index - 1] = vf["xyz".index(f[1])]
        elif f == "u_max":
            sensor_data["u_max"] = np.maximum(sensor_data["u_max"], umag())
        elif f == "u_rms":
            sensor_data["u_rms"] = sensor_data["u_rms"] + umag() ** 2
        elif f == "u_final" and t_index == Nt:
            sensor_data["u_final"] = umag()
        elif f == "I_avg":
            sensor_data["I_avg"] = sensor_data["I_avg"] + intensity() / Nt
        elif f == "I_max":
            sensor_data["I_max"] = np.maximum(sensor_data["I_max"], intensity())


def apply_sensor_directivity(sensor_data, sensor: KWaveSensor, grid: KWaveGrid):
    """solver/first_order_steps.jl:836-873."""
    if sensor.directivity_angle is None or sensor.directivity_size is None or "p" not in sensor_data:
        return
    p_data = sensor_data["p"]
    n_sensor, Nt = p_data.shape
    Fs = 1.0 / grid.dt
    freqs = np.fft.fftfreq(Nt, 1.0 / Fs)
    dmin = grid.dx if grid.ndim == 1 else min(grid.d)
    ang = np.asarray(sensor.directivity_angle, dtype=np.float64)
    for j in range(n_sensor):
        angle = float(ang) if ang.ndim == 0 else float(ang.ravel()[j])
        if math.isclose(angle, 0.0, rel_tol=1.4901161193847656e-08, abs_tol=0.0):
            continue
        fc = np.fft.fft(p_data[j, :])
        kval = 2 * math.pi * np.abs(freqs) / dmin
        arg = kval * sensor.directivity_size * math.sin(angle) / 2
        with np.errstate(invalid="ignore", divide="ignore"):
            dirv = np.where(arg == 0, 1.0, np.sin(arg) / np.where(arg == 0, 1.0, arg))
        p_data[j, :] = np.real(np.fft.ifft(fc * dirv))


def apply_frequency_response(sensor_data, sensor: KWaveSensor, grid: KWaveGrid):
    """solver/first_order_steps.jl:880-910."""
    if sensor.frequency_response is None or "p" not in sensor_data:
        return
    center, bw = sensor.frequency_response
    p_data = sensor_data["p"]
    n_sensor, Nt = p_data.shape
    freqs = np.fft.fftfreq(Nt, grid.dt)
    resp = np.exp(-((np.abs(freqs) - center) ** 2) / (2 * bw ** 2))
    for j in range(n_sensor):
        p_data[j, :] = np.real(np.fft.ifft(np.fft.fft(p_data[j, :]) * resp))


# ---------------------------------------------------------------------------------------------
# kspace_first_order (solver/first_order.jl:92-728)
# ---------------------------------------------------------------------------------------------

def kspace_first_order_as(grid: KWaveGrid, medium: KWaveMedium, source: KWaveSource, sensor: KWaveSensor,
                          pml_size=20, pml_alpha=2.0, smooth_p0: bool = True, dtype=np.float64,
                          max_steps: Optional[int] = None, progress_callback=None) -> dict:
    """Restates ``kspace_first_order_as`` (solver/axisymmetric.jl:26-227): the 2D solver with x
    axial and y radial, whose radial density update carries the cylindrical term u_r / r
    (axisymmetric.jl:183, 186), r = |y_vec| with r = 0 replaced by dy/2 (:100-103).  Time-reversal
    data is not used by that solver (it records the sensor as usual)."""
    if grid.ndim != 2:
        raise TypeError("kspace_first_order_as takes a 2D grid (x axial, y radial)")
    return kspace_first_order(grid, medium, source, sensor, pml_size=pml_size, pml_alpha=pml_alpha,
                              smooth_p0=smooth_p0, dtype=dtype, max_steps=max_steps,
                              progress_callback=progress_callback, _axisymmetric=True)


def radial_distance(grid: KWaveGrid) -> np.ndarray:
    """axisymmetric.jl:100-103 -- r = |y_vec|, with r = 0 replaced by dy / 2."""
    r = np.abs(make_spatial_vec(grid.N[1], grid.d[1]))
    r[r == 0] = grid.d[1] / 2
    return r


def kspace_first_order(grid: KWaveGrid, medium: KWaveMedium, source: KWaveSource, sensor: KWaveSensor,
                       pml_size=20, pml_alpha=2.0, smooth_p0: bool = True, dtype=np.float64,
                       max_steps: Optional[int] = None, progress_callback=None,
                       extra_sensors=(), _axisymmetric: bool = False) -> dict:
    """Restates ``kspace_first_order`` for 1D/2D/3D grids; returns the sensor-data dict.

    Oracle-only conveniences (not in the reference): ``max_steps`` stops the time loop early
    (outputs then describe the prefix); ``extra_sensors`` records further (mask, record) sensors
    in the same loop, returned as a list under the key ``"_extra"``.
    """
    if grid.Nt == 0 or grid.dt == 0:
        raise RuntimeError("Time array not set. Call make_time!(kgrid, sound_speed) before running.")
    for f in sensor.record:
        if f not in VALID_RECORD_FIELDS:
            raise ValueError(f"Invalid sensor record field: :{f}")
    D = grid.ndim
    shape = grid.N
    dt = grid.dt
    Nt = grid.Nt
    ct = np.complex64 if dtype == np.float32 else np.complex128
    psz = tuple(pml_size) if isinstance(pml_size, (tuple, list)) else (pml_size,) * D
    pal = tuple(pml_alpha) if isinstance(pml_alpha, (tuple, list)) else (pml_alpha,) * D

    pml = [get_pml(shape[d], grid.d[d], psz[d], pal[d], dt) for d in range(D)]
    pml_sg = [get_pml(shape[d], grid.d[d], psz[d], pal[d], dt, staggered=True) for d in range(D)]

    def bshape(v, d):
        s = [1] * D
        s[d] = -1
        return v.reshape(s)

    pml = [bshape(v, d) for d, v in enumerate(pml)]
    pml_sg = [bshape(v, d) for d, v in enumerate(pml_sg)]

    plans = _Plans(shape)
    n1 = plans.n1
    c0 = medium.sound_speed if _is_scalar(medium.sound_speed) else np.asarray(medium.sound_speed, np.float64)
    rho0 = medium.density if _is_scalar(medium.density) else np.asarray(medium.density, np.float64)
    BonA = medium.BonA if (medium.BonA is None or _is_scalar(medium.BonA)) else np.asarray(medium.BonA, np.float64)
    if not _is_scalar(c0):
        c0 = float(c0) if np.ndim(c0) == 0 else c0
    c_ref = float(c0) if _is_scalar(c0) else float(np.mean(c0))

    k_full = grid.k
    kappa_r = compute_kappa(k_full, c_ref, dt).astype(dtype)[:n1]
    absorb_f64 = precompute_absorption(medium, k_full, c_ref)
    absorb = None
    if absorb_f64 is not None:
        absorb = AbsorptionParams(dtype(absorb_f64.tau), dtype(absorb_f64.eta),
                                  absorb_f64.nabla1.astype(dtype)[:n1], absorb_f64.nabla2.astype(dtype)[:n1],
                                  absorb_f64.mode)
    k_ops = [grid.k_vecs[d].astype(dtype) for d in range(D)]
    s_pos = [grid.shift_pos[d].astype(ct) for d in range(D)]
    s_neg = [grid.shift_neg[d].astype(ct) for d in range(D)]

    zeros = lambda: np.zeros(shape, dtype=dtype, order="F")
    p = zeros()
    u = [zeros() for _ in range(D)]
    rho = [zeros() for _ in range(D)]
    rho_sg = None if _is_scalar(rho0) else [stagger_density(rho0, d).astype(dtype) for d in range(D)]
    rho_prev = zeros() if (absorb is not None and absorb.mode != "no_dispersion") else None

    sensor_data = _create_sensor_data(sensor, Nt)
    mask_idx = findall(sensor.mask) if (sensor.mask is not None and np.asarray(sensor.mask).dtype == bool) \
        else np.zeros(0, dtype=np.int64)

    extras = []
    for es in extra_sensors:
        es = es if isinstance(es, KWaveSensor) else KWaveSensor(**es)
        extras.append((es, _create_sensor_data(es, Nt), findall(es.mask)))

    tr = sensor.time_reversal_boundary_data is not None and not _axisymmetric
    tr_data = None
    r_row = radial_distance(grid).reshape(1, -1).astype(dtype) if _axisymmetric else None
    if tr:
        tr_data = np.asarray(sensor.time_reversal_boundary_data, dtype=np.float64)
        Nt = tr_data.shape[1]
        grid.Nt = Nt
        tr_idx = mask_idx

    # --- p0 initialisation (solver/first_order_steps.jl:58-191)
    if not tr and source.p0 is not None:
        p0 = np.asarray(source.p0).astype(dtype)
        do_smooth = smooth_p0 and ((D == 1 and shape[0] > 4) or (D > 1 and all(n > 1 for n in shape)))
        if do_smooth:
            p0 = smooth(p0, restore_max=True, dtype=dtype)
        p[...] = p0
        c0_sq = c0 ** 2
        for d in range(D):
            rho[d][...] = p0 / (c0_sq if D == 1 else D * c0_sq)
        for d in range(D):
            g = spectral_gradient(p0, grid.k_vecs[d], grid.shift_pos[d], plans, d, dtype)
            rs = rho0 if _is_scalar(rho0) else stagger_density(rho0, d)
            u[d][...] = -dt / (2 * rs) * g

    has_p_src = source.p_mask is not None and source.p is not None
    has_u_src = source.u_mask is not None
    if has_p_src:
        p_idx = findall(source.p_mask)
        p_sig = _signal_2d(source.p)
    if has_u_src:
        u_idx = findall(source.u_mask)
        u_sigs = [None if s is None else _signal_2d(s) for s in (source.ux, source.uy, source.uz)]

    steps = Nt if max_steps is None else min(Nt, max_steps)
    for t_index in range(1, steps + 1):
        if tr:
            tr_t = Nt - t_index + 1
            c_loc = c0 if _is_scalar(c0) else _flatF(c0)[tr_idx]
            val = tr_data[:, tr_t - 1] / (c_loc ** 2 if D == 1 else D * c_loc ** 2)
            for d in range(D):
                _flatF(rho[d])[tr_idx] = val

        # STEP 1-2: pressure gradient, velocity update with staggered PML
        for d in range(D):
            g = spectral_gradient(p, k_ops[d], s_pos[d], plans, d, dtype)
            rs = rho0 if rho_sg is None else rho_sg[d]
            u[d][...] = pml_sg[d] * (pml_sg[d] * u[d] - dt / rs * g)
        # STEP 3: velocity sources
        if has_u_src:
            for d in range(min(D, 3)):
                sig = u_sigs[d]
                if sig is None:
                    continue
                t_col = min(t_index, sig.shape[1])
                vals = sig[: len(u_idx), t_col - 1]
                uf = _flatF(u[d])
                if source.u_mode == DIRICHLET:
                    uf[u_idx] = vals
                else:
                    uf[u_idx] = uf[u_idx] + vals
        # STEP 4-5: divergence, density update with PML
        for d in range(D):
            g = spectral_gradient(u[d], k_ops[d], s_neg[d], plans, d, dtype)
            if r_row is not None and d == 1:
                g = g + u[1] / r_row  # axisymmetric.jl:183, 186: div u gains u_r / r
            rho[d][...] = pml[d] * (pml[d] * rho[d] - dt * rho0 * g)
        # STEP 6: pressure sources
        if has_p_src:
            t_col = min(t_index, p_sig.shape[1])
            c_loc = c0 if _is_scalar(c0) else _flatF(c0)[p_idx]
            vals = p_sig[: len(p_idx), t_col - 1] / (c_loc ** 2 if D == 1 else D * c_loc ** 2)
            for d in range(D):
                rf = _flatF(rho[d])
                if source.p_mode == DIRICHLET:
                    rf[p_idx] = vals
                else:
                    rf[p_idx] = rf[p_idx] + vals
        # STEP 7: equation of state
        rho_total = rho[0].copy() if D == 1 else np.asarray(sum(rho[1:], rho[0]), dtype=dtype)
        p[...] = _compute_pressure(rho_total, rho_prev, kappa_r, c0, rho0, BonA, absorb, plans, dt, dtype)
        if rho_prev is not None:
            rho_prev[...] = rho_total

        if len(mask_idx) > 0:
            _record(sensor_data, sensor.record, p, u, mask_idx, t_index, Nt)
        for es, esd, eidx in extras:
            if len(eidx) > 0:
                _record(esd, es.record, p, u, eidx, t_index, Nt)
        if progress_callback is not None:
            progress_callback(t_index, Nt, p)

    # finalize (solver/first_order_steps.jl:818-825)
    if "p_rms" in sensor_data:
        sensor_data["p_rms"] = np.sqrt(sensor_data["p_rms"] / Nt)
    if "u_rms" in sensor_data:
        sensor_data["u_rms"] = np.sqrt(sensor_data["u_rms"] / Nt)
    for es, esd, eidx in extras:
        if "p_rms" in esd:
            esd["p_rms"] = np.sqrt(esd["p_rms"] / Nt)
        if "u_rms" in esd:
            esd["u_rms"] = np.sqrt(esd["u_rms"] / Nt)
    if tr:
        sensor_data["p_final"] = _flatF(p).astype(np.float64).copy()
    if extras:
        sensor_data["_extra"] = [esd for _, esd, _ in extras]
    apply_sensor_directivity(sensor_data, sensor, grid)
    apply_frequency_response(sensor_data, sensor, grid)
    return sensor_data


# ---------------------------------------------------------------------------------------------
# pstd_elastic_2d / pstd_elastic_3d (solver/elastic.jl:133-588)
# ---------------------------------------------------------------------------------------------

@dataclass
class ElasticMedium:
    """solver/elastic.jl:22-48."""
    sound_speed_compression: Any
    sound_speed_shear: Any
    density: Any = 1000.0
    alpha_coeff_compression: Any = None
    alpha_coeff_shear: Any = None
    alpha_power: Optional[float] = None


@dataclass
class ElasticSource:
    """solver/elastic.jl:57-104: stress sources on s_mask, velocity sources on u_mask, p0."""
    s_mask: Any = None
    sxx: Any = None
    syy: Any = None
    szz: Any = None
    sxy: Any = None
    sxz: Any = None
    syz: Any = None
    s_mode: int = ADDITIVE
    u_mask: Any = None
    ux: Any = None
    uy: Any = None
    uz: Any = None
    u_mode: int = ADDITIVE
    p0: Any = None


# stress components in the order (xx, yy, zz, xy, xz, yz); sigma_{dj} of axes d, j
STRESS_NAMES = ("sxx", "syy", "szz", "sxy", "sxz", "syz")


def stress_slot(d: int, j: int) -> int:
    """Slot of sigma_{dj} in STRESS_NAMES (symmetric in d, j)."""
    return d if d == j else 2 + d + j


def elastic_lame(medium: ElasticMedium):
    """solver/elastic.jl:168-174, 419-423: lambda = rho (cp^2 - 2 cs^2), mu = rho cs^2.

    With a scalar density the reference writes ``rho0 * (cp^2 - 2 * cs^2)``, which for an array
    ``cp`` or ``cs`` is a matrix power (or a MethodError in 3D), not an element-wise square; that
    combination is rejected here rather than reproduced."""
    cp, cs, rho0 = medium.sound_speed_compression, medium.sound_speed_shear, medium.density
    if _is_scalar(rho0):
        if not (_is_scalar(cp) and _is_scalar(cs)):
            raise TypeError("a scalar density with array wave speeds is evaluated as a matrix power "
                            "(cp^2) by the reference (solver/elastic.jl:169); give the density as an array")
        return float(rho0) * (float(cp) ** 2 - 2 * float(cs) ** 2), float(rho0) * float(cs) ** 2
    rho0 = np.asarray(rho0, np.float64)
    cp = cp if _is_scalar(cp) else np.asarray(cp, np.float64)
    cs = cs if _is_scalar(cs) else np.asarray(cs, np.float64)
    return rho0 * (np.square(cp) - 2 * np.square(cs)), rho0 * np.square(cs)


def elastic_chi(medium: ElasticMedium):
    """solver/elastic.jl:177-195: Kelvin-Voigt factors chi = 2 db2neper(alpha, y) c_ref^(y-1),
    c_ref the (mean) compressional or shear speed; 0 when the coefficient or alpha_power is unset."""
    y = medium.alpha_power
    chi_p = chi_s = 0.0
    if medium.alpha_coeff_compression is not None and y is not None:
        cp = medium.sound_speed_compression
        c_ref = float(cp) if _is_scalar(cp) else float(np.mean(cp))
        chi_p = 2 * db2neper(medium.alpha_coeff_compression, y) * c_ref ** (y - 1)
    if medium.alpha_coeff_shear is not None and y is not None:
        cs = medium.sound_speed_shear
        cs_ref = float(cs) if _is_scalar(cs) else float(np.mean(cs))
        chi_s = 2 * db2neper(medium.alpha_coeff_shear, y) * cs_ref ** (y - 1)
    return chi_p, chi_s


def pstd_elastic(grid: KWaveGrid, medium: ElasticMedium, source: ElasticSource, sensor: KWaveSensor,
                 pml_size=None, pml_alpha=2.0, dtype=np.float64, max_steps: Optional[int] = None,
                 progress_callback=None) -> dict:
    """Restates ``pstd_elastic_2d`` (solver/elastic.jl:133-366) and ``pstd_elastic_3d``
    (:386-588): the stress-velocity PSTD scheme on a staggered grid.

    Per step: the stress divergence (sum over d of d/dx_d sigma_{dj}, staggered +) updates each
    velocity with its own split PML and 1/rho_sg (:236-250, 471-481); velocity sources (:253-276);
    the nine (four in 2D) velocity gradients (staggered -) update the stresses (:279-313, 505-521)
    -- the Kelvin-Voigt factors chi_p, chi_s enter only the 2D homogeneous branch -- then stress
    sources (:316-347), and the sensor records p = -trace(sigma)/D with the velocities (:350-356,
    565-570).  p0 sets every normal stress to -p0 (no smoothing).  Default pml_size is 20 in 2D and
    10 in 3D, as in the reference signatures.  ``max_steps`` (oracle only) stops early.
    """
    if grid.Nt == 0 or grid.dt == 0:
        raise RuntimeError("Time array not set. Call make_time!(kgrid, sound_speed) before running.")
    for f in sensor.record:
        if f not in VALID_RECORD_FIELDS:
            raise ValueError(f"Invalid sensor record field: :{f}")
    D = grid.ndim
    if D not in (2, 3):
        raise TypeError("pstd_elastic_2d / pstd_elastic_3d take a 2D or 3D grid")
    if pml_size is None:
        pml_size = 20 if D == 2 else 10
    shape, dt, Nt = grid.N, grid.dt, grid.Nt
    ct = np.complex64 if dtype == np.float32 else np.complex128
    psz = tuple(pml_size) if isinstance(pml_size, (tuple, list)) else (pml_size,) * D
    pal = tuple(pml_alpha) if isinstance(pml_alpha, (tuple, list)) else (pml_alpha,) * D

    def bshape(v, d):
        s = [1] * D
        s[d] = -1
        return v.reshape(s)

    pml = [bshape(get_pml(shape[d], grid.d[d], psz[d], pal[d], dt), d) for d in range(D)]
    pml_sg = [bshape(get_pml(shape[d], grid.d[d], psz[d], pal[d], dt, staggered=True), d) for d in range(D)]

    lam, mu = elastic_lame(medium)
    homogeneous = _is_scalar(lam)
    chi_p, chi_s = elastic_chi(medium) if D == 2 else (0.0, 0.0)
    rho0 = medium.density if _is_scalar(medium.density) else np.asarray(medium.density, np.float64)
    rho_sg = None if _is_scalar(rho0) else [stagger_density(rho0, d) for d in range(D)]

    plans = _Plans(shape)
    k_ops = [grid.k_vecs[d].astype(dtype) for d in range(D)]
    s_pos = [grid.shift_pos[d].astype(ct) for d in range(D)]
    s_neg = [grid.shift_neg[d].astype(ct) for d in range(D)]

    zeros = lambda: np.zeros(shape, dtype=np.float64, order="F")
    v = [zeros() for _ in range(D)]
    slots = [0, 1, 3] if D == 2 else list(range(6))
    sig = {k: zeros() for k in slots}

    sensor_data = _create_sensor_data(sensor, Nt)
    mask_idx = findall(sensor.mask) if (sensor.mask is not None and np.asarray(sensor.mask).dtype == bool) \
        else np.zeros(0, dtype=np.int64)

    if source.p0 is not None:
        p0 = np.asarray(source.p0, dtype=np.float64)
        for d in range(D):
            sig[d][...] = -p0

    u_idx = findall(source.u_mask) if source.u_mask is not None else None
    s_idx = findall(source.s_mask) if source.s_mask is not None else None
    u_sigs = [None if s is None else _signal_2d(s) for s in (source.ux, source.uy, source.uz)][:D]
    s_sigs = [None if s is None else _signal_2d(s) for s in
              (source.sxx, source.syy, source.szz, source.sxy, source.sxz, source.syz)]

    def inject(fields, sigs, idx, mode, t_index):
        for f, sg in zip(fields, sigs):
            if sg is None:
                continue
            col = sg[:, 0] if sg.shape[1] == 1 else sg[:, min(t_index, sg.shape[1]) - 1]
            vals = col[: len(idx)]
            ff = _flatF(f)
            if mode == DIRICHLET:
                ff[idx] = vals
            else:
                ff[idx] = ff[idx] + vals

    grad = lambda f, d, sp: spectral_gradient(f, k_ops[d], sp[d], plans, d, dtype).astype(np.float64)
    steps = Nt if max_steps is None else min(Nt, max_steps)
    p = zeros()
    for t_index in range(1, steps + 1):
        # stress divergence -> velocities (x, y[, z] terms summed in that order)
        for j in range(D):
            acc = grad(sig[stress_slot(0, j)], 0, s_pos)
            for d in range(1, D):
                acc = acc + grad(sig[stress_slot(d, j)], d, s_pos)
            rs = rho0 if rho_sg is None else rho_sg[j]
            v[j][...] = pml_sg[j] * (pml_sg[j] * v[j] + dt / rs * acc)
        if u_idx is not None:
            inject(v, u_sigs, u_idx, source.u_mode, t_index)
        # velocity gradients dv_j/dx_d
        g = [[grad(v[j], d, s_neg) for d in range(D)] for j in range(D)]  # g[j][d]
        l2m = lam + 2 * mu
        if D == 2:
            dxx, dyy = g[0][0], g[1][1]
            a_xx = l2m * dxx + lam * dyy
            a_yy = lam * dxx + l2m * dyy
            sh = mu * (g[0][1] + g[1][0])
            if homogeneous:
                a_xx = a_xx + chi_p * (l2m * dxx + lam * dyy)
                a_yy = a_yy + chi_p * (lam * dxx + l2m * dyy)
                sh = sh + chi_s * mu * (g[0][1] + g[1][0])
            sig[0][...] = pml[0] * (pml[0] * sig[0] + dt * a_xx)
            sig[1][...] = pml[1] * (pml[1] * sig[1] + dt * a_yy)
            sig[3][...] = pml[0] * pml[1] * (sig[3] + dt * sh)
        else:
            dxx, dyy, dzz = g[0][0], g[1][1], g[2][2]
            sig[0][...] = pml[0] * (pml[0] * sig[0] + dt * (l2m * dxx + lam * (dyy + dzz)))
            sig[1][...] = pml[1] * (pml[1] * sig[1] + dt * (l2m * dyy + lam * (dxx + dzz)))
            sig[2][...] = pml[2] * (pml[2] * sig[2] + dt * (l2m * dzz + lam * (dxx + dyy)))
            sig[3][...] = pml[0] * pml[1] * (sig[3] + dt * mu * (g[0][1] + g[1][0]))
            sig[4][...] = pml[0] * pml[2] * (sig[4] + dt * mu * (g[0][2] + g[2][0]))
            sig[5][...] = pml[1] * pml[2] * (sig[5] + dt * mu * (g[1][2] + g[2][1]))
        if s_idx is not None:
            inject([sig[k] for k in slots], [s_sigs[k] for k in slots], s_idx, source.s_mode, t_index)
        p[...] = -(sum(sig[d] for d in range(D))) / D
        if len(mask_idx) > 0:
            _record(sensor_data, sensor.record, p, v, mask_idx, t_index, Nt)
        if progress_callback is not None:
            progress_callback(t_index, Nt, p)

    if "p_rms" in sensor_data:
        sensor_data["p_rms"] = np.sqrt(sensor_data["p_rms"] / Nt)
    if "u_rms" in sensor_data:
        sensor_data["u_rms"] = np.sqrt(sensor_data["u_rms"] / Nt)
    return sensor_data


def pstd_elastic_2d(grid, medium, source, sensor, pml_size=20, pml_alpha=2.0, **kw) -> dict:
    """solver/elastic.jl:133-366."""
    if grid.ndim != 2:
        raise TypeError("pstd_elastic_2d takes a KWaveGrid2D")
    return pstd_elastic(grid, medium, source, sensor, pml_size=pml_size, pml_alpha=pml_alpha, **kw)


def pstd_elastic_3d(grid, medium, source, sensor, pml_size=10, pml_alpha=2.0, **kw) -> dict:
    """solver/elastic.jl:386-588."""
    if grid.ndim != 3:
        raise TypeError("pstd_elastic_3d takes a KWaveGrid3D")
    return pstd_elastic(grid, medium, source, sensor, pml_size=pml_size, pml_alpha=pml_alpha, **kw)
