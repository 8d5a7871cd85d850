"""CPU checks of the host-side mirror: setup helpers agree with the oracle's restatement, and
build_problem turns the reference's arguments into the kwb_problem the C ABI expects."""
import ctypes as C
import math

import numpy as np
import pytest

import kwave_b200 as kb
import kwave_ref as K
from kwave_b200 import workloads as W


def test_setup_helpers_match_oracle():
    rng = np.random.default_rng(5)
    for shape in [(32,), (16, 12), (9, 8, 7)]:
        m = rng.standard_normal(shape)
        assert np.allclose(kb.smooth(m, restore_max=True), K.smooth(m, restore_max=True), atol=1e-12)
    for args in [(40e6, 1e6, 5), (1 / 2e-8, 1e6, 5), (1 / 3.6e-8, 1.3e6, 3)]:
        for env in ("gaussian", "rectangular", "cosine"):
            assert np.array_equal(kb.tone_burst(*args, envelope=env), K.tone_burst(*args, envelope=env)) or \
                np.allclose(kb.tone_burst(*args, envelope=env), K.tone_burst(*args, envelope=env), atol=1e-15)
    assert np.array_equal(kb.make_disc(64, 48, 20, 30, 7), K.make_disc(64, 48, 20, 30, 7))
    assert np.array_equal(kb.make_circle(64, 48, 20, 30, 11), K.make_circle(64, 48, 20, 30, 11))
    assert np.array_equal(kb.make_line(20, 30, (2, 3), (19, 27)), K.make_line(20, 30, (2, 3), (19, 27)))
    assert np.array_equal(kb.make_ball(20, 18, 16, 9, 8, 7, 5), K.make_ball(20, 18, 16, 9, 8, 7, 5))
    for st in (False, True):
        assert np.array_equal(kb.get_pml(50, 1e-4, 12, 2.0, 2e-8, st), K.get_pml(50, 1e-4, 12, 2.0, 2e-8, st))
    assert kb.get_optimal_pml_size((100, 128, 77)) == K.get_optimal_pml_size((100, 128, 77))
    assert kb.db2neper(0.75, 1.5) == K.db2neper(0.75, 1.5)
    g1, g2 = kb.KWaveGrid(128, 1e-4, 96, 2e-4), K.KWaveGrid(128, 1e-4, 96, 2e-4)
    assert kb.make_time(g1, 1500.0) == K.make_time(g2, 1500.0)
    for a in range(2):
        assert np.array_equal(g1.k_vec(a), g2.k_vecs[a])


def test_build_problem_layout():
    n0, n1 = 12, 10
    g = kb.KWaveGrid(n0, 1e-4, n1, 2e-4)
    kb.make_time(g, 1500.0, t_end=1e-6)
    c = np.arange(n0 * n1, dtype=float).reshape(n0, n1) + 1400
    pm = np.zeros((n0, n1), bool)
    pm[3, 2] = pm[1, 5] = pm[7, 2] = True
    sig = np.arange(6.0).reshape(3, 2)
    sm = np.zeros((n0, n1), bool)
    sm[0, 0] = sm[11, 9] = True
    b = kb.build_problem(g, kb.KWaveMedium(sound_speed=c, density=1000.0, alpha_coeff=0.5, alpha_power=1.2,
                                           alpha_mode="stokes", BonA=5.0),
                         kb.KWaveSource(p_mask=pm, p=sig, p_mode=kb.Dirichlet),
                         kb.KWaveSensor(mask=sm, record=["p", "p_rms", "p_rms"]), pml_size=(4, 6), pml_alpha=(2.0, 3.0))
    P = b.problem
    assert P.ndim == 2 and list(P.N) == [n0, n1, 1] and P.Nt == g.Nt
    assert list(P.pml_size)[:2] == [4, 6] and list(P.pml_alpha)[:2] == [2.0, 3.0]
    # column-major (x fastest) linear indices, sorted, as findall returns
    idx = [P.p_index[i] for i in range(P.n_p_index)]
    assert idx == sorted([3 + n0 * 2, 7 + n0 * 2, 1 + n0 * 5])
    # grid arrays go over row-major (NumPy order, reordered on the device): (3, 2) at 3 * n1 + 2
    assert P.row_major == 1
    assert P.c0.count == n0 * n1 and P.c0.data[3 * n1 + 2] == c[3, 2]
    assert P.p_signal.n_rows == 3 and P.p_signal.n_cols == 2 and P.p_signal.data[1] == sig[1, 0]
    assert P.p_mode == 0 and P.alpha_mode == 2 and P.BonA.count == 1
    grp = P.groups[0]
    assert grp.n_index == 2 and grp.dense == 0 and [grp.index[0], grp.index[1]] == [0, n0 * n1 - 1]
    assert grp.record_mask == (1 << 0) | (1 << 3) and grp.record_count[3] == 2


def test_build_problem_dense_cartesian_tr_and_errors():
    g = kb.KWaveGrid(8, 1e-4, 8, 1e-4)
    med = kb.KWaveMedium(sound_speed=1500.0)
    with pytest.raises(RuntimeError, match="make_time"):
        kb.build_problem(g, med, kb.KWaveSource(), kb.KWaveSensor())
    kb.make_time(g, 1500.0, t_end=1e-7)
    b = kb.build_problem(g, med, kb.KWaveSource(), kb.KWaveSensor(mask=np.ones((8, 8), bool), record=["p_max"]))
    assert b.problem.groups[0].dense == 1 and b.problem.groups[0].n_index == 64
    b = kb.build_problem(g, med, kb.KWaveSource(), kb.KWaveSensor(mask=np.zeros((2, 7)), record=["p"]))
    assert b.problem.groups[0].cartesian == 1 and b.problem.groups[0].n_index == 7
    tr = np.ones((4, 9))
    m = np.zeros((8, 8), bool)
    m[0, :4] = True
    b = kb.build_problem(g, med, kb.KWaveSource(p0=np.ones((8, 8))),
                         kb.KWaveSensor(mask=m, time_reversal_boundary_data=tr, record=["p_final"]))
    assert b.problem.tr.n_rows == 4 and b.problem.tr.n_cols == 9 and b.problem.p0.count == 0
    with pytest.raises(ValueError, match="Invalid sensor record field"):
        kb.build_problem(g, med, kb.KWaveSource(), kb.KWaveSensor(mask=m, record=["bogus"]))
    with pytest.raises(TypeError, match="array alpha_coeff"):
        kb.build_problem(g, kb.KWaveMedium(sound_speed=1500.0, alpha_coeff=np.ones((8, 8)), alpha_power=1.5,
                                           alpha_mode="no_dispersion"), kb.KWaveSource(), kb.KWaveSensor())
    with pytest.raises(IndexError, match="BoundsError"):
        kb.build_problem(g, med, kb.KWaveSource(p_mask=m, p=np.ones((2, 3))), kb.KWaveSensor())
    with pytest.raises(TypeError, match="MethodError"):
        kb.build_problem(g, med, kb.KWaveSource(), kb.KWaveSensor(mask=m, record=["I_max"]), data_cast=np.float32)
    with pytest.raises(NotImplementedError):
        kb.kspace_first_order(g, med, kb.KWaveSource(), kb.KWaveSensor(), save_to_disk="/tmp/x.h5")


def test_workloads_are_seeded_and_match_their_configs():
    a, b = W.c2(n=64, Nt=10), W.c2(n=64, Nt=10)
    assert np.array_equal(a.medium["sound_speed"], b.medium["sound_speed"])
    c2 = W.c2(n=512, Nt=2000)
    c = c2.medium["sound_speed"]
    assert c.min() == pytest.approx(1400) and c.max() == pytest.approx(1600)
    assert c2.dt == pytest.approx(0.3e-4 / 1600) and c2.Nt == 2000
    c1 = W.c1()
    assert c1.Nt == 689 and c1.source["p_mask"].sum() == 81 and c1.sensor["mask"].sum() == 228
    assert c1.source["p"].shape == (81, 689)
    c3 = W.c3(n=64, Nt=20, piston=8, pml=4)
    assert c3.source["u_mask"].sum() == 64 and set(np.unique(c3.medium["BonA"])) == {5.0, 9.0}
    sides = {W.c4_sim(i).N for i in range(8)}
    assert all(n in W.C4_SIDES for s in sides for n in s)
    assert W.smooth_sides(256, 300) == [256, 270, 288, 300]


def test_findall_sparse_and_dense_paths_agree():
    """Mask indices: the sparse path (row-major coordinates, sorted) and the column-major ravel
    give the same findall(mask) - 1; an all-true sensor mask becomes a dense group."""
    import kwave_b200 as kb
    from kwave_b200.solver import _findall
    rng = np.random.default_rng(7)
    for shape in ((17, 9), (6, 11, 5)):
        for frac in (0.05, 0.6):
            m = rng.random(shape) < frac
            ref = np.flatnonzero(m.ravel(order="F"))
            assert np.array_equal(_findall(m, shape), ref)
    g = kb.KWaveGrid(8, 1e-4, 6, 1e-4)
    kb.make_time(g, 1500.0, t_end=1e-6)
    b = kb.build_problem(g, kb.KWaveMedium(sound_speed=1500.0), kb.KWaveSource(p0=np.ones((8, 6))),
                         kb.KWaveSensor(mask=np.ones((8, 6), bool), record=["p_max"]))
    assert b.problem.groups[0].dense == 1 and b.problem.groups[0].n_index == 48


def test_post_filter_convolution_form_matches_the_oracle():
    """The device post-filters (kwb_postfilter.cu) apply the reference's
    real(ifft(fft(p) .* H)) as a circular convolution with h = ifft(H), H real and even in |f|
    (first_order_steps.jl:836-910).  Restated here in NumPy on the same steps -- H per distinct
    angle, h by an FP64 cosine sum, p' = h (*) p -- it equals the oracle's FFT filters; rows
    whose angle is 0 get the frequency response only."""
    import kwave_ref as K
    rng = np.random.default_rng(3)
    for n, Nt in ((37, 211), (5, 64), (9, 1)):
        dt = 2e-8
        go = K.KWaveGrid(32, 1e-4, 24, 2e-4)
        go.dt = dt
        ang = rng.uniform(-1.2, 1.2, n)
        ang[[0, n // 2]] = 0.0
        p = rng.standard_normal((n, Nt))
        seno = K.KWaveSensor(mask=np.ones((32, 24), bool), record=["p"])
        seno.directivity_angle, seno.directivity_size, seno.frequency_response = ang, 3e-4, (2e6, 8e5)
        b = {"p": p.copy()}
        K.apply_sensor_directivity(b, seno, go)
        K.apply_frequency_response(b, seno, go)
        k = np.arange(Nt)
        f = np.where(k < (Nt + 1) // 2, k, k - Nt) / (Nt * dt)
        af = np.abs(f)
        out = np.empty_like(p)
        cosT = np.cos(2 * np.pi * np.arange(Nt) / Nt)
        for j in range(n):
            H = np.exp(-((af - 2e6) ** 2) / (2 * (8e5) ** 2))
            if ang[j] != 0.0:
                arg = 2 * np.pi * af / 1e-4 * 3e-4 * np.sin(ang[j]) / 2
                H = H * np.where(arg == 0, 1.0, np.sin(arg) / np.where(arg == 0, 1.0, arg))
            h = np.array([np.dot(H, cosT[(k * m) % Nt]) for m in range(Nt)]) / Nt
            out[j] = [np.dot(h[(m - k) % Nt], p[j]) for m in range(Nt)]
        assert np.allclose(out, b["p"], rtol=0, atol=1e-12 * max(1.0, np.abs(b["p"]).max())), (n, Nt)


def test_build_problem_carries_post_filters():
    """The sensor's directivity and frequency response reach the first sensor group of the ABI
    problem (applied by the library on the device); angle arrays in column-major order, scalar
    angles as one value for every point, short arrays raise as the reference's angle[j] would."""
    g = kb.KWaveGrid(8, 1e-4, 6, 1e-4)
    kb.make_time(g, 1500.0, t_end=1e-6)
    med, src = kb.KWaveMedium(sound_speed=1500.0), kb.KWaveSource(p0=np.ones((8, 6)))
    m = np.zeros((8, 6), bool)
    m[2, 1:4] = True
    ang = np.array([0.1, 0.0, 0.3])
    sen = kb.KWaveSensor(mask=m, record=["p"], directivity_angle=ang, directivity_size=2e-4,
                         frequency_response=(1e6, 3e5))
    b = kb.build_problem(g, med, src, sen)
    grp = b.problem.groups[0]
    assert grp.n_directivity_angle == 3 and grp.directivity_size == 2e-4
    assert [grp.directivity_angle[i] for i in range(3)] == [0.1, 0.0, 0.3]
    assert grp.has_frequency_response == 1 and (grp.frequency_center, grp.frequency_bandwidth) == (1e6, 3e5)
    sen1 = kb.KWaveSensor(mask=m, record=["p"], directivity_angle=0.5, directivity_size=2e-4)
    grp1 = kb.build_problem(g, med, src, sen1).problem.groups[0]
    assert grp1.n_directivity_angle == 1 and grp1.has_frequency_response == 0
    with pytest.raises(IndexError):
        kb.build_problem(g, med, src, kb.KWaveSensor(mask=m, record=["p"], directivity_angle=ang[:2],
                                                     directivity_size=2e-4))
    nofilt = kb.build_problem(g, med, src, kb.KWaveSensor(mask=m, record=["p"])).problem.groups[0]
    assert not nofilt.directivity_angle and nofilt.has_frequency_response == 0


def test_build_problem_elastic():
    """ElasticMedium/ElasticSource -> kwb_problem: speeds, density, Kelvin-Voigt coefficients only
    where the 2D homogeneous branch uses them, stress signals per component, p0 unsmoothed, and
    the reference's error cases."""
    from kwave_b200.solver import build_problem
    n = 16
    g = kb.KWaveGrid(n, 1e-4, n, 1e-4)
    g.dt, g.Nt = 1e-8, 12
    p0 = np.zeros((n, n))
    p0[5, 7] = 3.0
    s_mask = np.zeros((n, n), bool)
    s_mask[2, 3] = s_mask[9, 1] = True
    sig = np.arange(2 * 12, dtype=float).reshape(2, 12)
    src = kb.ElasticSource(s_mask=s_mask, sxx=sig, syy=2 * sig, szz=3 * sig, sxy=4 * sig, s_mode=kb.Dirichlet, p0=p0)
    med = kb.ElasticMedium(3000.0, 1500.0, 1800.0, alpha_coeff_compression=0.5, alpha_coeff_shear=1.0,
                           alpha_power=1.5)
    sen = kb.KWaveSensor(mask=np.ones((n, n), bool), record=["p", "I_avg"])
    P = build_problem(g, med, src, sen, data_cast=np.float32).problem  # I_avg allowed: no MethodError here
    assert P.elastic == 1 and P.c0.count == 1 and P.cs.count == 1 and P.rho0.count == 1
    assert P.cs.data[0] == 1500.0 and P.c0.data[0] == 3000.0 and P.rho0.data[0] == 1800.0
    assert P.alpha_mode != 0 and P.alpha_coeff == 0.5 and P.has_alpha_shear == 1 and P.alpha_coeff_shear == 1.0
    assert P.alpha_power == 1.5
    assert P.n_s_index == 2 and [P.s_index[i] for i in range(2)] == [9 + 1 * n, 2 + 3 * n]  # sorted, column-major
    assert P.s_mode == int(kb.Dirichlet)
    # 2D reads sxx, syy, sxy only (elastic.jl:315-347)
    assert [bool(P.s_signal[k].data) for k in range(6)] == [True, True, False, True, False, False]
    assert P.s_signal[3].n_rows == 2 and P.s_signal[3].n_cols == 12
    # p0 goes over unsmoothed (row-major buffer)
    got = np.ctypeslib.as_array(P.p0.data, shape=(n * n,)).reshape(n, n)
    assert np.array_equal(got, p0)
    # heterogeneous density: chi unused, so no absorption fields
    rho = np.full((n, n), 1800.0)
    P2 = build_problem(g, kb.ElasticMedium(np.full((n, n), 3000.0), 1500.0, rho, alpha_coeff_compression=0.5,
                                           alpha_power=1.5), kb.ElasticSource(p0=p0), sen).problem
    assert P2.alpha_mode == 0 and P2.has_alpha_shear == 0 and P2.c0.count == n * n and P2.rho0.count == n * n
    # 3D: no chi either
    g3 = kb.KWaveGrid(8, 1e-4, 8, 1e-4, 8, 1e-4)
    g3.dt, g3.Nt = 1e-8, 4
    P3 = build_problem(g3, med, kb.ElasticSource(), kb.KWaveSensor(mask=np.ones((8, 8, 8), bool))).problem
    assert P3.elastic == 1 and P3.alpha_mode == 0 and P3.has_alpha_shear == 0
    # errors: scalar density with array speeds (a matrix power in the reference), 1D grids,
    # stress signals with too few rows
    with pytest.raises(TypeError):
        build_problem(g, kb.ElasticMedium(np.full((n, n), 3000.0), 1500.0, 1800.0), kb.ElasticSource(), sen)
    g1 = kb.KWaveGrid(32, 1e-4)
    g1.dt, g1.Nt = 1e-8, 4
    with pytest.raises(TypeError):
        build_problem(g1, med, kb.ElasticSource(), kb.KWaveSensor(mask=np.ones(32, bool)))
    with pytest.raises(IndexError):
        build_problem(g, med, kb.ElasticSource(s_mask=s_mask, sxx=np.ones((1, 12))), sen)


def test_grid_helpers():  # grid.jl:260-296
    g = kb.KWaveGrid(64, 1e-4, 32, 2e-4, 16, 5e-5)
    assert kb.grid_size(g) == (64, 32, 16) and kb.grid_spacing(g) == (1e-4, 2e-4, 5e-5)
    assert kb.total_grid_points(g) == 64 * 32 * 16
    assert kb.k_max(g) == min(math.pi / 1e-4, math.pi / 2e-4, math.pi / 5e-5)
    assert kb.k_max(kb.KWaveGrid(10, 1e-3)) == math.pi / 1e-3
