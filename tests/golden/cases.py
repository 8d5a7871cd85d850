"""Seeded small cases for the golden fixtures: inputs are rebuilt from these builders, outputs
(FP64 oracle) are stored in tests/golden/<name>.npz by make_golden.py.

Each builder returns (solver, grid_args, dt, Nt, medium, source, sensor, options) with plain
numpy inputs in the reference's index order; ``solver`` names the reference function.
"""
import math

import numpy as np


def _grf(rng, shape, sigma, lo, hi):
    w = rng.standard_normal(shape)
    W = np.fft.fftn(w)
    k2 = np.zeros(shape)
    for ax, n in enumerate(shape):
        kv = 2 * math.pi * np.fft.fftfreq(n)
        s = [1] * len(shape)
        s[ax] = n
        k2 = k2 + kv.reshape(s) ** 2
    f = np.real(np.fft.ifftn(W * np.exp(-k2 * sigma ** 2 / 2)))
    f = (f - f.min()) / (f.max() - f.min())
    return lo + (hi - lo) * f


def fluid_2d():
    """64^2 homogeneous lossless, 3x3 additive pressure source (1 MHz sine), p at 32 points."""
    n, dx, Nt = 64, 1e-4, 120
    dt = 0.3 * dx / 1500.0
    t = np.arange(Nt) * dt
    p_mask = np.zeros((n, n), bool)
    p_mask[30:33, 30:33] = True
    sig = np.vstack([np.sin(2 * math.pi * 1e6 * t)] * 9)
    mask = np.zeros((n, n), bool)
    mask[10, 8:56:3] = True
    mask[50, 8:56:3] = True
    return ("kspace_first_order", (n, dx, n, dx), dt, Nt,
            dict(sound_speed=1500.0, density=1000.0),
            dict(p_mask=p_mask, p=sig), dict(mask=mask, record=["p", "p_max", "p_rms"]), dict(pml_size=10))


def fluid_3d():
    """24^3 heterogeneous nonlinear absorbing medium, smoothed p0 ball, p series and p_max."""
    rng = np.random.default_rng(7001)
    n, dx, Nt = 24, 1e-4, 40
    shape = (n, n, n)
    c = _grf(rng, shape, 2.0, 1450.0, 1600.0)
    rho = _grf(rng, shape, 2.0, 950.0, 1100.0)
    dt = 0.3 * dx / 1600.0
    x = np.arange(n)
    r2 = (x[:, None, None] - 12) ** 2 + (x[None, :, None] - 11) ** 2 + (x[None, None, :] - 12) ** 2
    p0 = np.where(r2 <= 9, 1e5, 0.0)
    mask = np.zeros(shape, bool)
    mask[4, 4:20:2, 12] = True
    mask[18, 12, 4:20:2] = True
    return ("kspace_first_order", (n, dx, n, dx, n, dx), dt, Nt,
            dict(sound_speed=c, density=rho, alpha_coeff=0.75, alpha_power=1.5, alpha_mode="no_dispersion",
                 BonA=6.0),
            dict(p0=p0), dict(mask=mask, record=["p", "p_max", "u_final"]), dict(pml_size=4))


def axisymmetric():
    """64 x 32 axisymmetric grid (x axial, y radial), heterogeneous, p0 on the axis."""
    rng = np.random.default_rng(7002)
    shape = (64, 32)
    dx, Nt = 1e-4, 80
    c = _grf(rng, shape, 3.0, 1450.0, 1600.0)
    dt = 0.3 * dx / 1600.0
    p0 = np.zeros(shape)
    p0[30:34, 14:18] = 1.0
    mask = np.zeros(shape, bool)
    mask[8:56:4, 20] = True
    return ("kspace_first_order_as", (64, dx, 32, dx), dt, Nt,
            dict(sound_speed=c, density=1000.0), dict(p0=p0), dict(mask=mask, record=["p", "uy"]),
            dict(pml_size=6))


def elastic_2d():
    """48^2 heterogeneous elastic solid, additive sxx/sxy sources, p and ux at 24 points."""
    rng = np.random.default_rng(7003)
    shape = (48, 48)
    dx, Nt = 1e-4, 100
    cp = _grf(rng, shape, 3.0, 2600.0, 3100.0)
    cs = _grf(rng, shape, 3.0, 1200.0, 1500.0)
    rho = _grf(rng, shape, 3.0, 1600.0, 2000.0)
    dt = 0.3 * dx / 3100.0
    t = np.arange(Nt) * dt
    s_mask = np.zeros(shape, bool)
    s_mask[24, 24] = s_mask[25, 24] = True
    w = np.sin(2 * math.pi * 2e6 * t)
    mask = np.zeros(shape, bool)
    mask[6:42:3, 10] = True
    mask[6:42:3, 38] = True
    return ("pstd_elastic_2d", (48, dx, 48, dx), dt, Nt,
            dict(sound_speed_compression=cp, sound_speed_shear=cs, density=rho),
            dict(s_mask=s_mask, sxx=1e3 * np.vstack([w, w]), sxy=5e2 * np.vstack([w, w])),
            dict(mask=mask, record=["p", "ux", "u_max"]), dict(pml_size=8))


def elastic_3d():
    """20^3 homogeneous elastic solid, p0 cube, p at 20 points."""
    n, dx, Nt = 20, 1e-4, 40
    dt = 0.3 * dx / 3000.0
    p0 = np.zeros((n, n, n))
    p0[9:12, 9:12, 9:12] = 1e4
    mask = np.zeros((n, n, n), bool)
    mask[3:17:3, 4, 10] = True
    mask[10, 3:17:3, 15] = True
    mask[15, 10, 3:17:3] = True
    mask[4, 15, 3:17:3] = True
    return ("pstd_elastic_3d", (n, dx, n, dx, n, dx), dt, Nt,
            dict(sound_speed_compression=3000.0, sound_speed_shear=1500.0, density=1800.0),
            dict(p0=p0), dict(mask=mask, record=["p", "uz"]), dict(pml_size=4))


CASES = {"fluid_2d": fluid_2d, "fluid_3d": fluid_3d, "axisymmetric": axisymmetric,
         "elastic_2d": elastic_2d, "elastic_3d": elastic_3d}


def run(module, name):
    """Run case `name` through `module` (the oracle kwave_ref or the kwave_b200 package), which
    provides the reference API names."""
    solver, grid_args, dt, Nt, medium, source, sensor, opts = CASES[name]()
    g = module.KWaveGrid(*grid_args)
    g.dt, g.Nt = dt, Nt
    elastic = solver.startswith("pstd_elastic")
    med = (module.ElasticMedium if elastic else module.KWaveMedium)(**medium)
    src = (module.ElasticSource if elastic else module.KWaveSource)(**source)
    out = getattr(module, solver)(g, med, src, module.KWaveSensor(**sensor), **opts)
    return {k: np.asarray(out[k], dtype=np.float64) for k in sensor["record"]}
