"""Axisymmetric solver (kspace_first_order_as, solver/axisymmetric.jl:26-227) on the GPU against
the FP64 oracle: register-FFT sizes, Stockham sizes, an odd radial size (r = dy/2 on the axis),
heterogeneous absorbing media with pressure and velocity sources."""
import math

import numpy as np
import pytest

from _util import assert_parity, oracle_inputs

pytestmark = pytest.mark.gpu
TOL_L2, TOL_MAX = 1e-4, 1e-3


@pytest.fixture(scope="module")
def kb():
    import kwave_b200
    kwave_b200.default_context()
    return kwave_b200


def _case(shape, seed, Nt=120, sources=True):
    from kwave_b200.workloads import Case, gaussian_random_field
    rng = np.random.default_rng(seed)
    Nx, Nr = shape
    c = gaussian_random_field(rng, shape, 3.0, 1450.0, 1600.0)
    rho = gaussian_random_field(rng, shape, 3.0, 950.0, 1100.0)
    dt = 0.3e-4 / 1600
    t = np.arange(Nt) * dt
    p0 = np.zeros(shape)
    p0[Nx // 2 - 2: Nx // 2 + 2, Nr // 2 - 3: Nr // 2 + 3] = 1.0
    src = dict(p0=p0)
    if sources:
        pm = np.zeros(shape, bool)
        pm[Nx // 3, Nr // 2 - 2: Nr // 2 + 2] = True
        um = np.zeros(shape, bool)
        um[2 * Nx // 3, Nr // 2 - 1: Nr // 2 + 1] = True
        src.update(p_mask=pm, p=np.vstack([np.sin(2 * math.pi * 1e6 * t)] * 4),
                   u_mask=um, uy=1e-3 * np.vstack([np.sin(2 * math.pi * 1.5e6 * t)] * 2))
    mask = np.ones(shape, bool)
    return Case(f"as{shape}", shape, (1e-4, 1e-4), dt, Nt,
                dict(sound_speed=c, density=rho, alpha_coeff=0.75, alpha_power=1.5, alpha_mode="no_dispersion",
                     BonA=6.0),
                src, dict(mask=mask, record=["p_final", "p_max", "p_rms", "u_final"]), pml_size=6)


def _gpu(case):
    import kwave_b200 as kb
    g, m, s, sen, opts = case.to_api()
    return kb.kspace_first_order_as(g, m, s, sen, **opts)


def _oracle(case):
    import kwave_ref as K
    g, m, s, sen, opts = oracle_inputs(case)
    return K.kspace_first_order_as(g, m, s, sen, **opts)


@pytest.mark.parametrize("shape", [(128, 64), (64, 128), (96, 48), (72, 45)])
def test_axisymmetric_matches_oracle(kb, shape):
    case = _case(shape, sum(shape))
    assert_parity(_gpu(case), _oracle(case), TOL_L2, TOL_MAX)


def test_axisymmetric_reference_basic_run(kb):
    """test_axisymmetric.jl:2-27 restated on the GPU path (64 x 32, Gaussian p0, p on a line)."""
    Nx, Nr, dx = 64, 32, 1e-4
    g = kb.KWaveGrid(Nx, dx, Nr, dx)
    med = kb.KWaveMedium(sound_speed=1500.0, density=1000.0)
    kb.make_time(g, 1500.0, t_end=2e-6)
    i = np.arange(1, Nx + 1)[:, None]
    j = np.arange(1, Nr + 1)[None, :]
    p0 = np.exp(-(((i - Nx // 2) * dx) ** 2 + ((j - Nr // 2) * dx) ** 2) / (5 * dx) ** 2)
    mask = np.zeros((Nx, Nr), bool)
    mask[Nx // 2 - 1, :] = True
    out = kb.kspace_first_order_as(g, med, kb.KWaveSource(p0=p0), kb.KWaveSensor(mask=mask, record=["p"]))
    assert out["p"].shape == (Nr, g.Nt)
    import kwave_ref as K
    go = K.KWaveGrid(Nx, dx, Nr, dx)
    K.make_time(go, 1500.0, t_end=2e-6)
    ref = K.kspace_first_order_as(go, K.KWaveMedium(sound_speed=1500.0, density=1000.0), K.KWaveSource(p0=p0),
                                  K.KWaveSensor(mask=mask, record=["p"]))
    assert_parity(out, ref, TOL_L2, TOL_MAX)


def test_axisymmetric_rejects_3d_grids(kb):
    g = kb.KWaveGrid(16, 1e-4, 16, 1e-4, 16, 1e-4)
    kb.make_time(g, 1500.0, t_end=1e-7)
    with pytest.raises(TypeError):
        kb.kspace_first_order_as(g, kb.KWaveMedium(sound_speed=1500.0), kb.KWaveSource(p0=np.ones((16, 16, 16))),
                                 kb.KWaveSensor(mask=np.ones((16, 16, 16), bool)))
