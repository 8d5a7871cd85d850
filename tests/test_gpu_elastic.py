"""Elastic solvers (pstd_elastic_2d / pstd_elastic_3d, solver/elastic.jl:133-588) on the GPU
against the FP64 oracle: the reference's own elastic test cases, homogeneous absorbing and
heterogeneous media, stress and velocity sources in both modes, power-of-two and mixed-radix
line lengths, non-square grids, and every sensor field."""
import math

import numpy as np
import pytest

from _util import assert_parity

pytestmark = pytest.mark.gpu
TOL_L2, TOL_MAX = 1e-4, 1e-3


@pytest.fixture(scope="module")
def kb():
    import kwave_b200
    kwave_b200.default_context()
    return kwave_b200


def _run(spec):
    """Run one case through the GPU library and the oracle; spec holds grid, medium, source,
    sensor keyword dicts and the solver options."""
    import kwave_b200 as kb
    import kwave_ref as K
    N, d, dt, Nt = spec["N"], spec["d"], spec["dt"], spec["Nt"]
    args = []
    for n in N:
        args += [n, d]
    g = kb.KWaveGrid(*args)
    g.dt, g.Nt = dt, Nt
    og = K.KWaveGrid(*args)
    og.dt, og.Nt = dt, Nt
    src = dict(spec["source"])
    osrc = {k: (int(v) if k.endswith("_mode") else v) for k, v in src.items()}
    opts = dict(spec.get("opts", {}))
    solve = kb.pstd_elastic_2d if len(N) == 2 else kb.pstd_elastic_3d
    osolve = K.pstd_elastic_2d if len(N) == 2 else K.pstd_elastic_3d
    out = solve(g, kb.ElasticMedium(**spec["medium"]), kb.ElasticSource(**src), kb.KWaveSensor(**spec["sensor"]),
                **opts)
    ref = osolve(og, K.ElasticMedium(**spec["medium"]), K.ElasticSource(**osrc), K.KWaveSensor(**spec["sensor"]),
                 **opts)
    return out, ref


def _homog():
    return dict(sound_speed_compression=3000.0, sound_speed_shear=1500.0, density=1800.0)


def _make_dt(n, dx, c=3000.0):
    return 0.3 * dx / c


# ---- the reference's own elastic tests (test_elastic.jl:44-153), checked against the oracle ----

def test_reference_basic_run_2d(kb):  # test_elastic.jl:44-72
    n, dx = 32, 0.5e-3
    p0 = np.zeros((n, n))
    p0[n // 2 - 1, n // 2 - 1] = 1.0
    mask = np.zeros((n, n), bool)
    mask[4, :] = True
    import kwave_ref as K
    g = K.KWaveGrid(n, dx, n, dx)
    K.make_time(g, 3000.0)
    spec = dict(N=(n, n), d=dx, dt=g.dt, Nt=g.Nt, medium=_homog(), source=dict(p0=p0),
                sensor=dict(mask=mask, record=["p"]))
    out, ref = _run(spec)
    assert out["p"].shape == (mask.sum(), g.Nt)
    assert_parity(out, ref, TOL_L2, TOL_MAX)


def test_reference_stress_source_2d(kb):  # test_elastic.jl:74-101
    import kwave_ref as K
    n, dx = 32, 0.5e-3
    g = K.KWaveGrid(n, dx, n, dx)
    K.make_time(g, 3000.0)
    s_mask = np.zeros((n, n), bool)
    s_mask[4, n // 2 - 1] = True
    sig = np.sin(2 * math.pi * 1e6 * np.arange(g.Nt) * g.dt).reshape(1, -1)
    mask = np.zeros((n, n), bool)
    mask[n // 2 - 1, :] = True
    spec = dict(N=(n, n), d=dx, dt=g.dt, Nt=g.Nt, medium=_homog(),
                source=dict(s_mask=s_mask, sxx=sig, s_mode=kb.Additive), sensor=dict(mask=mask, record=["p"]))
    out, ref = _run(spec)
    assert np.abs(out["p"]).max() > 0
    assert_parity(out, ref, TOL_L2, TOL_MAX)


def test_reference_wave_speeds_2d(kb):  # test_elastic.jl:103-124
    import kwave_ref as K
    n, dx = 64, 0.5e-3
    g = K.KWaveGrid(n, dx, n, dx)
    K.make_time(g, 3000.0)
    p0 = np.zeros((n, n))
    p0[n // 2 - 1, n // 2 - 1] = 1.0
    mask = np.zeros((n, n), bool)
    mask[n // 4 - 1, n // 2 - 1] = True
    spec = dict(N=(n, n), d=dx, dt=g.dt, Nt=g.Nt, medium=_homog(), source=dict(p0=p0),
                sensor=dict(mask=mask, record=["p"]))
    out, ref = _run(spec)
    assert np.abs(out["p"][0]).max() > 0
    assert_parity(out, ref, TOL_L2, TOL_MAX)


def test_reference_basic_run_3d(kb):  # test_elastic.jl:126-153
    import kwave_ref as K
    n, dx = 16, 0.5e-3
    g = K.KWaveGrid(n, dx, n, dx, n, dx)
    K.make_time(g, 3000.0)
    p0 = np.zeros((n, n, n))
    p0[n // 2 - 1, n // 2 - 1, n // 2 - 1] = 1.0
    mask = np.zeros((n, n, n), bool)
    mask[2, :, :] = True
    spec = dict(N=(n, n, n), d=dx, dt=g.dt, Nt=g.Nt, medium=_homog(), source=dict(p0=p0),
                sensor=dict(mask=mask, record=["p"]), opts=dict(pml_size=5))
    out, ref = _run(spec)
    assert out["p"].shape == (mask.sum(), g.Nt)
    assert_parity(out, ref, TOL_L2, TOL_MAX)


# ---- wider cases ---------------------------------------------------------------------------

ALL_FIELDS_2D = ["p", "p_max", "p_min", "p_rms", "p_final", "ux", "uy", "u_max", "u_rms", "u_final",
                 "I_avg", "I_max"]


@pytest.mark.parametrize("shape", [(96, 64), (64, 64), (60, 45), (45, 64)])
def test_homogeneous_absorbing_2d_with_sources(kb, shape):
    """Kelvin-Voigt absorption (2D homogeneous branch), Dirichlet velocity source, additive stress
    source on all three 2D components, every sensor field.  Nx = 45 takes the scalar velocity and
    stress updates (the float4 ones need Nx a multiple of 4)."""
    Nx, Ny = shape
    dx, Nt = 0.2e-3, 150
    dt = _make_dt(Nx, dx)
    t = np.arange(Nt) * dt
    u_mask = np.zeros(shape, bool)
    u_mask[Nx // 3, Ny // 2 - 2: Ny // 2 + 2] = True
    s_mask = np.zeros(shape, bool)
    s_mask[2 * Nx // 3, Ny // 3: Ny // 3 + 3] = True
    burst = np.sin(2 * math.pi * 1.5e6 * t) * np.exp(-((t - 20 * dt) / (8 * dt)) ** 2)
    mask = np.zeros(shape, bool)
    mask[::5, ::7] = True
    medium = dict(_homog(), alpha_coeff_compression=0.5, alpha_coeff_shear=1.0, alpha_power=1.5)
    spec = dict(N=shape, d=dx, dt=dt, Nt=Nt, medium=medium,
                source=dict(u_mask=u_mask, ux=1e-3 * np.vstack([burst] * 4), u_mode=kb.Dirichlet,
                            s_mask=s_mask, sxx=1e3 * burst.reshape(1, -1).repeat(3, 0),
                            syy=-5e2 * burst.reshape(1, -1).repeat(3, 0), sxy=2e2 * burst.reshape(1, -1).repeat(3, 0)),
                sensor=dict(mask=mask, record=ALL_FIELDS_2D), opts=dict(pml_size=8))
    out, ref = _run(spec)
    assert_parity(out, ref, TOL_L2, TOL_MAX)


@pytest.mark.parametrize("shape", [(128, 72), (64, 128), (160, 80), (80, 192)])
def test_heterogeneous_2d(kb, shape):
    """Array speeds and density (no absorption in that branch), Dirichlet stress source, additive
    velocity source, p0."""
    from kwave_b200.workloads import gaussian_random_field
    rng = np.random.default_rng(sum(shape))
    Nx, Ny = shape
    dx, Nt = 0.1e-3, 160
    cp = gaussian_random_field(rng, shape, 4.0, 2500.0, 3200.0)
    cs = gaussian_random_field(rng, shape, 4.0, 1000.0, 1500.0)
    rho = gaussian_random_field(rng, shape, 4.0, 1500.0, 2000.0)
    dt = 0.3 * dx / 3200.0
    t = np.arange(Nt) * dt
    p0 = np.zeros(shape)
    p0[Nx // 2 - 2: Nx // 2 + 2, Ny // 2 - 2: Ny // 2 + 2] = 1e3
    s_mask = np.zeros(shape, bool)
    s_mask[Nx // 4, Ny // 4] = True
    u_mask = np.zeros(shape, bool)
    u_mask[3 * Nx // 4, Ny // 2: Ny // 2 + 5] = True
    mask = np.ones(shape, bool)
    spec = dict(N=shape, d=dx, dt=dt, Nt=Nt,
                medium=dict(sound_speed_compression=cp, sound_speed_shear=cs, density=rho,
                            alpha_coeff_compression=0.5, alpha_power=1.2),
                source=dict(p0=p0, s_mask=s_mask, sxy=1e2 * np.sin(2 * math.pi * 1e6 * t).reshape(1, -1),
                            s_mode=kb.Dirichlet, u_mask=u_mask, uy=1e-4 * np.vstack([np.cos(2 * math.pi * 2e6 * t)] * 5)),
                sensor=dict(mask=mask, record=["p_max", "p_rms", "p_final", "u_final", "u_max"]),
                opts=dict(pml_size=10, pml_alpha=(2.0, 3.0)))
    out, ref = _run(spec)
    assert_parity(out, ref, TOL_L2, TOL_MAX)


def test_homogeneous_3d_cube(kb):
    n, dx, Nt = 64, 0.2e-3, 80
    p0 = np.zeros((n, n, n))
    p0[n // 2 - 3: n // 2 + 3, n // 2 - 3: n // 2 + 3, n // 2 - 3: n // 2 + 3] = 1.0
    mask = np.zeros((n, n, n), bool)
    mask[:, :, n // 2] = True
    spec = dict(N=(n, n, n), d=dx, dt=_make_dt(n, dx), Nt=Nt, medium=_homog(), source=dict(p0=p0),
                sensor=dict(mask=mask, record=["p", "p_max", "uz", "u_rms"]))
    out, ref = _run(spec)
    assert_parity(out, ref, TOL_L2, TOL_MAX)


def test_heterogeneous_3d_all_sources(kb):
    """Non-cubic 3D, array medium, all six stress components (additive) and three velocity
    components (Dirichlet), every sensor field."""
    from kwave_b200.workloads import gaussian_random_field
    rng = np.random.default_rng(33)
    shape = (48, 40, 32)
    dx, Nt = 0.1e-3, 70
    cp = gaussian_random_field(rng, shape, 3.0, 2600.0, 3100.0)
    cs = gaussian_random_field(rng, shape, 3.0, 1100.0, 1500.0)
    rho = gaussian_random_field(rng, shape, 3.0, 1600.0, 2100.0)
    dt = 0.3 * dx / 3100.0
    t = np.arange(Nt) * dt
    s_mask = np.zeros(shape, bool)
    s_mask[10, 20, 16] = s_mask[11, 20, 16] = True
    u_mask = np.zeros(shape, bool)
    u_mask[36, 10:13, 8] = True
    w = np.sin(2 * math.pi * 1.2e6 * t)
    src = dict(s_mask=s_mask, u_mask=u_mask, u_mode=kb.Dirichlet,
               ux=1e-4 * np.vstack([w] * 3), uy=-1e-4 * np.vstack([w] * 3), uz=5e-5 * np.vstack([w] * 3))
    for k, name in enumerate(("sxx", "syy", "szz", "sxy", "sxz", "syz")):
        src[name] = (k + 1) * 1e2 * np.vstack([w] * 2)
    mask = np.zeros(shape, bool)
    mask[::3, ::4, ::5] = True
    rec = ["p", "p_max", "p_min", "p_rms", "p_final", "ux", "uy", "uz", "u_max", "u_rms", "u_final", "I_avg", "I_max"]
    spec = dict(N=shape, d=dx, dt=dt, Nt=Nt,
                medium=dict(sound_speed_compression=cp, sound_speed_shear=cs, density=rho),
                source=src, sensor=dict(mask=mask, record=rec), opts=dict(pml_size=(6, 5, 4)))
    out, ref = _run(spec)
    assert_parity(out, ref, TOL_L2, TOL_MAX)


def test_rejections(kb):
    g = kb.KWaveGrid(32, 1e-4, 32, 1e-4)
    g.dt, g.Nt = 1e-8, 10
    sen = kb.KWaveSensor(mask=np.ones((32, 32), bool), record=["p"])
    # scalar density with array speeds: a matrix power in the reference
    with pytest.raises(TypeError):
        kb.pstd_elastic_2d(g, kb.ElasticMedium(np.full((32, 32), 3000.0), 1500.0, 1800.0), kb.ElasticSource(), sen)
    with pytest.raises(TypeError):
        kb.pstd_elastic_3d(g, kb.ElasticMedium(3000.0, 1500.0, 1800.0), kb.ElasticSource(), sen)


def test_register_and_stockham_paths_agree(kb, monkeypatch):
    """Power-of-two lines run on the register-FFT gradient pass; KWB_FFT_PATH=generic forces the
    shared-memory Stockham pass.  Both match the oracle and each other."""
    from kwave_b200.workloads import elastic3d
    case = elastic3d(64, Nt=60)
    g, m, s, sen, kw = case.to_api()
    outs = {}
    for path in ("default", "generic"):
        if path == "generic":
            monkeypatch.setenv("KWB_FFT_PATH", "generic")
        outs[path] = kb.pstd_elastic_3d(g, m, s, sen, **kw)
    import kwave_ref as K
    args = []
    for n, d in zip(case.N, case.d):
        args += [n, d]
    og = K.KWaveGrid(*args)
    og.dt, og.Nt = case.dt, case.Nt
    ref = K.pstd_elastic_3d(og, K.ElasticMedium(**case.medium), K.ElasticSource(**case.source),
                            K.KWaveSensor(**case.sensor), pml_size=case.pml_size)
    for path in outs:
        assert_parity(outs[path], ref, TOL_L2, TOL_MAX)
    assert_parity(outs["default"], outs["generic"], 1e-5, 1e-4)


def test_served_with_fluid_requests(kb):
    """Elastic and fluid requests served together by the continuous-batching scheduler give the
    same outputs as their blocking solves."""
    from kwave_b200.workloads import elastic3d, c4_sim
    jobs = []
    for n in (32, 48):
        case = elastic3d(n, Nt=40)
        g, m, s, sen, kw = case.to_api()
        jobs.append((g, m, s, sen, kw, kb.pstd_elastic_3d))
    for i in range(2):
        case = c4_sim(i, sides=(128, 192), nt_range=(60, 90))
        g, m, s, sen, kw = case.to_api()
        jobs.append((g, m, s, sen, kw, kb.kspace_first_order))
    reqs = [kb.submit(g, m, s, sen, **kw) for g, m, s, sen, kw, _ in jobs]
    for (g, m, s, sen, kw, solve), r in zip(jobs, reqs):
        served = r.result(timeout=120)
        if solve is kb.pstd_elastic_3d:
            kw = {k: v for k, v in kw.items() if k != "smooth_p0"}
        direct = solve(g, m, s, sen, **kw)
        for k in direct.keys():
            assert np.array_equal(served[k], direct[k]), k
