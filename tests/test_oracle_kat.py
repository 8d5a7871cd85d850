"""Pins the FP64 oracle (oracle/kwave_ref.py) before it is trusted as the checker.

Restates every known-answer and property test the reference's own suite holds for this path
(KWave.jl/test/test_fft.jl, test_pml.jl, test_grid.jl, test_filter.jl, test_signal.jl,
test_geometry.jl, test_solver_{1,2,3}d.jl, test_absorption.jl, test_time_reversal.jl), plus a
closed-form known answer: for a homogeneous lossless medium without PML the reference's discrete
scheme is diagonal in k-space, so each Fourier mode of the stepped solution must equal a 2x2
recurrence evaluated independently here with complex FFTs.
"""
import math

import numpy as np
import pytest

import kwave_ref as K


def grid2(n, d=1e-4):
    return K.KWaveGrid(n, d, n, d)


# ---- test_fft.jl ---------------------------------------------------------------------------

def test_fft_round_trip():  # test_fft.jl:12-22
    plans = K._Plans((32, 32))
    data = np.random.default_rng(0).standard_normal((32, 32))
    assert np.allclose(plans.inverse(plans.forward(data)), data, atol=1e-12, rtol=0)


def test_spectral_gradient_of_sine():  # test_fft.jl:24-56
    n = 64
    g = K.KWaveGrid(n, 1.0, n, 1.0)
    kx = 2 * math.pi / n
    x = g.x_vecs[0]
    f = np.repeat(np.sin(kx * x)[:, None], n, axis=1)
    df = K.spectral_gradient(f, g.k_vecs[0], np.ones(n, complex), K._Plans((n, n)), 0)
    exp = kx * np.cos(kx * x)
    assert np.allclose(df[4:n - 4, n // 2 - 1], exp[4:n - 4], atol=1e-10, rtol=0)


def test_gradient_along_axis_equals_1d_transform():
    """The design fact the line passes rely on: N-D rfft gradient == 1-D FFT along that axis."""
    rng = np.random.default_rng(1)
    for shape in [(16, 12), (15, 10, 8), (8, 9, 10)]:
        g = K.KWaveGrid(*sum(([n, 1e-4] for n in shape), []))
        f = rng.standard_normal(shape)
        for d in range(len(shape)):
            for sh in (g.shift_pos[d], g.shift_neg[d]):
                nd = K.spectral_gradient(f, g.k_vecs[d], sh, K._Plans(shape), d)
                mult = (1j * g.k_vecs[d] * sh).reshape([-1 if a == d else 1 for a in range(len(shape))])
                one = np.real(np.fft.ifft(np.fft.fft(f, axis=d) * mult, axis=d))
                assert np.max(np.abs(nd - one)) < 1e-9 * np.max(np.abs(one))


# ---- test_pml.jl ---------------------------------------------------------------------------

def test_pml_properties():  # test_pml.jl:1-51
    N, s = 64, 10
    pml = K.get_pml(N, 1e-4, s, 2.0, 1e-8)
    assert len(pml) == N
    assert np.allclose(pml[s:N - s], 1.0)
    assert pml[0] < 1.0 and pml[-1] < 1.0
    assert np.all((pml > 0) & (pml <= 1.0))
    for i in range(s):
        assert math.isclose(pml[i], pml[N - 1 - i])
    assert np.all(np.diff(pml[:s]) >= 0)
    stag = K.get_pml(64, 1e-4, 10, 2.0, 1e-8, staggered=True)
    assert len(stag) == 64 and not np.array_equal(stag, pml) and np.allclose(stag[10:54], 1.0)
    assert np.all(K.get_pml(64, 1e-4, 0, 2.0, 1e-8) == 1.0)
    opt = K.get_optimal_pml_size(128)
    assert K.max_prime_factor(128 + 2 * opt) <= 7
    assert len(K.get_optimal_pml_size((64, 128))) == 2


def test_pml_value_formula():
    """pml.jl:40-48 -- exp(-alpha pos^4 dt) with no c/dx scaling (the reference's quirk)."""
    pml = K.get_pml(100, 1e-4, 20, 2.0, 2e-8)
    assert pml[0] == math.exp(-(2.0 * 1.0 ** 4) * 2e-8)
    assert 1 - pml[0] == pytest.approx(4e-8, rel=1e-6)


# ---- test_grid.jl --------------------------------------------------------------------------

def test_grid_construction():  # test_grid.jl:1-63
    g1 = K.KWaveGrid(64, 1e-4)
    assert g1.x_vecs[0][0] == pytest.approx(-(63) / 2 * 1e-4)
    assert g1.k_vecs[0][0] == 0.0 and np.all(g1.k >= 0)
    assert np.allclose(np.abs(g1.shift_pos[0]), 1.0) and np.allclose(np.abs(g1.shift_neg[0]), 1.0)
    g2 = K.KWaveGrid(64, 1e-4, 128, 2e-4)
    assert g2.k.shape == (64, 128) and abs(g2.k[0, 0]) < 1e-15
    for j in range(5):
        for i in range(5):
            assert g2.k[i, j] == pytest.approx(math.sqrt(g2.k_vecs[0][i] ** 2 + g2.k_vecs[1][j] ** 2))
    assert K.KWaveGrid(32, 1e-4, 32, 1e-4, 32, 1e-4).k.shape == (32, 32, 32)
    kv = K.make_wavenumber_vec(8, 1.0)
    assert len(kv) == 8 and kv[0] == 0.0 and kv[4] == -4 * 2 * math.pi / 8
    assert len(K.make_wavenumber_vec(7, 1.0)) == 7


def test_make_time():  # test_grid.jl:65-84
    g = grid2(128)
    dt, Nt = K.make_time(g, 1500.0)
    assert dt == pytest.approx(0.3 * 1e-4 / 1500.0) and Nt > 0 and len(g.t_array) == Nt
    assert g.t_array[1] == pytest.approx(dt)
    dt2, Nt2 = K.make_time(g, 1500.0, t_end=1e-5)
    assert Nt2 == math.ceil(1e-5 / dt2) + 1
    # the 128^2 disc-source workload: dt = 2e-8, Nt = 689
    g = grid2(128)
    assert K.make_time(g, 1500.0, t_end=1.14 * math.sqrt(2) * 128e-4 / 1500) == (2e-8, 689) or \
        (abs(g.dt - 2e-8) < 1e-20 and g.Nt == 689)


# ---- test_filter.jl, test_signal.jl, test_geometry.jl --------------------------------------

def test_smooth_and_conversions():  # test_filter.jl:38-66
    m = np.zeros((32, 32))
    m[9:22, 9:22] = 1.0
    s = K.smooth(m)
    assert s.shape == (32, 32) and s.max() <= m.max() + 0.1
    assert K.smooth(m, restore_max=True).max() == pytest.approx(m.max(), abs=0.1)
    assert float(K.neper2db(K.db2neper(10.0))) == pytest.approx(10.0)
    assert float(K.neper2db(1.0)) == pytest.approx(8.685889638, abs=1e-6)
    assert K.db2neper(0.75, 1.5) > 0 and K.db2neper(1.0, 1.0) > K.db2neper(1.0, 2.0)


def test_smooth_odd_length_shift():
    """Julia's fftshift shifts by floor(N/2) also for odd N; the window is not centred on DC."""
    v = np.zeros(7)
    v[3] = 1.0
    w = K.blackman_window(7)
    exp = np.real(np.fft.ifft(np.fft.fft(v) * np.roll(w, 3)))
    assert np.allclose(K.smooth(v), exp)


def test_tone_burst():  # test_signal.jl:2-23
    sig = K.tone_burst(40e6, 1e6, 5)
    assert len(sig) == 200 and abs(sig[0]) < 0.1 and abs(sig[-1]) < 0.1
    assert 0.5 < np.max(np.abs(sig)) <= 1.0 + 1e-10
    off = K.tone_burst(40e6, 1e6, 5, signal_offset=100)
    assert len(off) == 300 and np.all(off[:100] == 0)
    assert len(K.tone_burst(1 / 2e-8, 1e6, 5)) == 250


def test_geometry():  # test_geometry.jl:2-57
    disc = K.make_disc(64, 64, 32, 32, 10)
    assert disc[31, 31] and not disc[0, 0]
    assert abs(disc.sum() - math.pi * 100) / (math.pi * 100) < 0.1
    assert disc[26, 31] == disc[36, 31]
    circ = K.make_circle(64, 64, 32, 32, 15)
    assert not circ[31, 31] and (circ[46, 31] or circ[16, 31])
    assert abs(circ.sum() - 2 * math.pi * 15) / (2 * math.pi * 15) < 0.3
    ball = K.make_ball(32, 32, 32, 16, 16, 16, 8)
    assert ball[15, 15, 15] and not ball[0, 0, 0]
    assert abs(ball.sum() - 4 / 3 * math.pi * 512) / (4 / 3 * math.pi * 512) < 0.15
    assert K.make_disc(128, 128, 64, 64, 5).sum() == 81
    assert K.make_circle(128, 128, 64, 64, 40).sum() == 228
    line = K.make_line(10, 10, (1, 1), (10, 4))
    assert line[0, 0] and line[9, 3] and line.sum() == 10


# ---- solver property tests (test_solver_{1,2,3}d.jl, test_absorption.jl, test_time_reversal.jl)

def _run2(n, t_end, p0, mask, record, medium=None, **kw):
    g = grid2(n)
    K.make_time(g, 1500.0, t_end=t_end)
    med = medium or K.KWaveMedium(sound_speed=1500.0, density=1000.0)
    out = K.kspace_first_order(g, med, K.KWaveSource(p0=p0), K.KWaveSensor(mask=mask, record=record),
                               smooth_p0=False, **kw)
    return g, out


def test_solver_2d_properties():  # test_solver_2d.jl:1-123
    n = 64
    m = np.zeros((n, n), bool)
    m[n // 2 - 1, n // 2 - 1] = m[n // 2 + 19, n // 2 - 1] = True
    g, out = _run2(n, 5e-6, K.make_disc(n, n, 32, 32, 5).astype(float), m, ["p"])
    assert out["p"].shape == (2, g.Nt) and abs(out["p"][0, 0]) > 0
    g, out = _run2(n, 2e-6, K.make_disc(n, n, 32, 32, 3).astype(float), np.ones((n, n), bool), ["p"])
    assert np.sum(out["p"][:, -1] ** 2) < 10 * np.sum(out["p"][:, 0] ** 2) and np.all(np.isfinite(out["p"]))
    p0 = np.zeros((n, n))
    p0[31, 31] = 1.0
    m = np.zeros((n, n), bool)
    for (i, j) in [(41, 31), (21, 31), (31, 41), (31, 21)]:
        m[i, j] = True
    g, out = _run2(n, 2e-6, p0, m, ["p"])
    mid = out["p"][:, g.Nt // 2 - 1]
    mean = np.mean(np.abs(mid))
    assert np.all(np.abs(mid) / mean < 5.0)
    m = np.zeros((32, 32), bool)
    m[15, 15] = True
    g, out = _run2(32, 1e-6, K.make_disc(32, 32, 16, 16, 3).astype(float), m, ["p", "p_max"])
    assert out["p_max"][0] >= out["p"][0].max() - 1e-10


def test_solver_1d_and_3d_properties():  # test_solver_1d.jl, test_solver_3d.jl
    g = K.KWaveGrid(64, 1e-4)
    K.make_time(g, 1500.0, t_end=1e-6)
    p0 = np.zeros(64)
    p0[29:34] = 1.0
    m = np.zeros(64, bool)
    m[31] = True
    out = K.kspace_first_order(g, K.KWaveMedium(sound_speed=1500.0, density=1000.0), K.KWaveSource(p0=p0),
                               K.KWaveSensor(mask=m, record=["p", "p_max", "p_rms"]), smooth_p0=False)
    assert out["p_max"][0] >= out["p"][0].max() - 1e-10 and out["p_rms"][0] > 0
    n = 24
    g = K.KWaveGrid(n, 1e-4, n, 1e-4, n, 1e-4)
    K.make_time(g, 1500.0, t_end=1e-6)
    m = np.zeros((n, n, n), bool)
    m[11, 11, 11] = True
    out = K.kspace_first_order(g, K.KWaveMedium(sound_speed=1500.0, density=1000.0),
                               K.KWaveSource(p0=K.make_ball(n, n, n, 12, 12, 12, 2).astype(float)),
                               K.KWaveSensor(mask=m, record=["p", "ux", "uy", "uz", "u_max"]),
                               smooth_p0=False, pml_size=8)
    assert all(k in out for k in ("ux", "uy", "uz", "u_max")) and out["u_max"][0] >= 0


def test_absorption_reduces_energy():  # test_absorption.jl:46-82
    n = 64
    p0 = K.make_disc(n, n, 32, 32, 5).astype(float)
    ones = np.ones((n, n), bool)
    _, a = _run2(n, 5e-6, p0, ones, ["p_rms"])
    absorbing = K.KWaveMedium(sound_speed=1500.0, density=1000.0, alpha_coeff=2.0, alpha_power=1.5,
                              alpha_mode="no_dispersion")
    _, b = _run2(n, 5e-6, p0, ones, ["p_rms"], medium=absorbing)
    assert np.sum(b["p_rms"] ** 2) < np.sum(a["p_rms"] ** 2)


def test_time_reversal_peak_at_centre():  # test_time_reversal.jl:2-54
    n = 64
    bm = np.zeros((n, n), bool)
    bm[0, :] = bm[-1, :] = bm[:, 0] = bm[:, -1] = True
    g, fwd = _run2(n, 5e-6, K.make_disc(n, n, 32, 32, 3).astype(float), bm, ["p"])
    g2 = grid2(n)
    K.make_time(g2, 1500.0, t_end=5e-6)
    out = K.kspace_first_order(g2, K.KWaveMedium(sound_speed=1500.0, density=1000.0), K.KWaveSource(),
                               K.KWaveSensor(mask=bm, time_reversal_boundary_data=fwd["p"], record=["p_final"]),
                               smooth_p0=False)
    pk = np.unravel_index(np.argmax(np.abs(out["p_final"].reshape((n, n), order="F"))), (n, n))
    assert abs(pk[0] + 1 - 32) <= 5 and abs(pk[1] + 1 - 32) <= 5


# ---- closed-form known answer --------------------------------------------------------------

@pytest.mark.parametrize("shape", [(96,), (32, 24), (12, 10, 8)])
def test_per_mode_recurrence_matches_stepping(shape):
    D = len(shape)
    c, rho0, d = 1500.0, 1000.0, 1e-4
    g = K.KWaveGrid(*sum(([n, d] for n in shape), []))
    dt = 0.3 * d / c
    g.dt, g.Nt = dt, 40
    rng = np.random.default_rng(3)
    p0 = rng.standard_normal(shape)
    out = K.kspace_first_order(g, K.KWaveMedium(sound_speed=c, density=rho0), K.KWaveSource(p0=p0),
                               K.KWaveSensor(mask=np.ones(shape, bool), record=["p"]),
                               pml_size=0, smooth_p0=False)
    kv = [g.k_vecs[a].reshape([-1 if b == a else 1 for b in range(D)]) for a in range(D)]
    kmag = np.sqrt(sum(k ** 2 for k in kv))
    arg = c * kmag * dt / 2
    kappa = np.where(arg == 0, 1.0, np.sin(arg) / np.where(arg == 0, 1.0, arg))
    Gp = [1j * k * np.exp(1j * k * d / 2) for k in kv]
    Gn = [1j * k * np.exp(-1j * k * d / 2) for k in kv]
    P = np.fft.fftn(p0)
    R = [P / (D * c ** 2) for _ in range(D)]
    U = [-dt / (2 * rho0) * Gp[a] * P for a in range(D)]
    for n in range(1, g.Nt + 1):
        U = [U[a] - dt / rho0 * Gp[a] * P for a in range(D)]
        R = [R[a] - dt * rho0 * Gn[a] * U[a] for a in range(D)]
        P = c ** 2 * kappa * sum(R)
        p = np.real(np.fft.ifftn(P))
        stepped = out["p"][:, n - 1].reshape(shape, order="F")
        assert np.max(np.abs(stepped - p)) <= 1e-10 * np.max(np.abs(p)), n


def test_axisymmetric_basic_run():  # test_axisymmetric.jl:2-27
    Nx, Nr, dx = 64, 32, 1e-4
    g = K.KWaveGrid(Nx, dx, Nr, dx)
    med = K.KWaveMedium(sound_speed=1500.0, density=1000.0)
    K.make_time(g, 1500.0, t_end=2e-6)
    i = np.arange(1, Nx + 1)[:, None]
    j = np.arange(1, Nr + 1)[None, :]
    p0 = np.exp(-(((i - Nx // 2) * dx) ** 2 + ((j - Nr // 2) * dx) ** 2) / (5 * dx) ** 2)
    mask = np.zeros((Nx, Nr), bool)
    mask[Nx // 2 - 1, :] = True
    out = K.kspace_first_order_as(g, med, K.KWaveSource(p0=p0), K.KWaveSensor(mask=mask, record=["p"]))
    assert "p" in out and out["p"].shape == (Nr, g.Nt)
    assert np.all(np.isfinite(out["p"]))


def test_axisymmetric_with_absorption():  # test_axisymmetric.jl:29-50
    Nx = Nr = 64
    dx = 1e-4
    g = K.KWaveGrid(Nx, dx, Nr, dx)
    med = K.KWaveMedium(sound_speed=1500.0, density=1000.0, alpha_coeff=0.5, alpha_power=1.5,
                        alpha_mode="no_dispersion")
    K.make_time(g, 1500.0, t_end=1e-6)
    p0 = np.zeros((Nx, Nr))
    p0[Nx // 2 - 1, Nr // 2 - 1] = 1.0
    mask = np.zeros((Nx, Nr), bool)
    mask[Nx // 2 - 1, 0] = True
    out = K.kspace_first_order_as(g, med, K.KWaveSource(p0=p0), K.KWaveSensor(mask=mask, record=["p_max"]),
                                  pml_size=10)
    assert "p_max" in out and np.isfinite(out["p_max"]).all()


def test_axisymmetric_radial_term():
    """r = |y_vec| never vanishes for an even radial size and is dy/2 at the axis for an odd one
    (axisymmetric.jl:100-103); the u_r / r term changes the solution against the plain 2D solver."""
    g = K.KWaveGrid(32, 1e-4, 16, 1e-4)
    r = K.radial_distance(g)
    assert np.allclose(r, np.abs((np.arange(16) - 7.5) * 1e-4)) and r.min() > 0
    g3 = K.KWaveGrid(32, 1e-4, 15, 1e-4)
    r3 = K.radial_distance(g3)
    assert r3[7] == 0.5e-4 and np.isclose(r3[0], 7e-4)
    K.make_time(g, 1500.0, t_end=1e-6)
    p0 = np.zeros((32, 16))
    p0[15, 6:10] = 1.0
    mask = np.ones((32, 16), bool)
    med = K.KWaveMedium(sound_speed=1500.0, density=1000.0)
    a = K.kspace_first_order_as(g, med, K.KWaveSource(p0=p0), K.KWaveSensor(mask=mask, record=["p_final"]), pml_size=4)
    b = K.kspace_first_order(g, med, K.KWaveSource(p0=p0), K.KWaveSensor(mask=mask, record=["p_final"]), pml_size=4)
    rel = np.linalg.norm(a["p_final"] - b["p_final"]) / np.linalg.norm(b["p_final"])
    assert rel > 1e-3


# ---- test_elastic.jl, and closed-form plane waves of the elastic scheme ----------------------

def _elastic_medium():
    return K.ElasticMedium(sound_speed_compression=3000.0, sound_speed_shear=1500.0, density=1800.0)


def test_elastic_medium_and_source_construction():  # test_elastic.jl:2-42
    em = _elastic_medium()
    assert em.alpha_coeff_compression is None and em.alpha_coeff_shear is None
    em2 = K.ElasticMedium(3000.0, 1500.0, 1800.0, alpha_coeff_compression=0.5, alpha_coeff_shear=1.0,
                          alpha_power=1.5)
    chi_p, chi_s = K.elastic_chi(em2)
    assert chi_p == pytest.approx(2 * K.db2neper(0.5, 1.5) * 3000.0 ** 0.5, rel=1e-15)
    assert chi_s == pytest.approx(2 * K.db2neper(1.0, 1.5) * 1500.0 ** 0.5, rel=1e-15)
    es = K.ElasticSource()
    assert es.s_mask is None and es.p0 is None and es.s_mode == K.ADDITIVE
    lam, mu = K.elastic_lame(em)
    assert lam == 1800.0 * (3000.0 ** 2 - 2 * 1500.0 ** 2) and mu == 1800.0 * 1500.0 ** 2
    with pytest.raises(TypeError):  # the reference evaluates cp^2 as a matrix power here
        K.elastic_lame(K.ElasticMedium(np.full((4, 4), 3000.0), 1500.0, 1800.0))


def test_elastic_2d_basic_runs():  # test_elastic.jl:44-124
    for n, src in ((32, "p0"), (32, "stress"), (64, "p0")):
        g = K.KWaveGrid(n, 0.5e-3, n, 0.5e-3)
        K.make_time(g, 3000.0)
        mask = np.zeros((n, n), bool)
        if src == "p0":
            p0 = np.zeros((n, n))
            p0[n // 2 - 1, n // 2 - 1] = 1.0
            source = K.ElasticSource(p0=p0)
            if n == 64:
                mask[n // 4 - 1, n // 2 - 1] = True
            else:
                mask[4, :] = True
        else:
            s_mask = np.zeros((n, n), bool)
            s_mask[4, n // 2 - 1] = True
            sig = np.sin(2 * math.pi * 1e6 * np.arange(g.Nt) * g.dt).reshape(1, -1)
            source = K.ElasticSource(s_mask=s_mask, sxx=sig, s_mode=K.ADDITIVE)
            mask[n // 2 - 1, :] = True
        r = K.pstd_elastic_2d(g, _elastic_medium(), source, K.KWaveSensor(mask=mask, record=["p"]))
        assert r["p"].shape == (mask.sum(), g.Nt)
        assert np.all(np.isfinite(r["p"])) and np.abs(r["p"]).max() > 0


def test_elastic_3d_basic_run():  # test_elastic.jl:126-153
    n = 16
    g = K.KWaveGrid(n, 0.5e-3, n, 0.5e-3, n, 0.5e-3)
    K.make_time(g, 3000.0)
    p0 = np.zeros((n, n, n))
    p0[n // 2 - 1, n // 2 - 1, n // 2 - 1] = 1.0
    mask = np.zeros((n, n, n), bool)
    mask[2, :, :] = True
    r = K.pstd_elastic_3d(g, _elastic_medium(), K.ElasticSource(p0=p0), K.KWaveSensor(mask=mask, record=["p"]),
                          pml_size=5)
    assert r["p"].shape == (mask.sum(), g.Nt) and np.all(np.isfinite(r["p"]))


def _plane_wave_modes(n, dx, m):
    """Full-FFT wavenumbers of an x line and the staggered gradient multipliers i k e^{+-ik dx/2}."""
    g = K.KWaveGrid(n, dx)
    k = g.k_vecs[0]
    return k, 1j * k * np.exp(1j * k * dx / 2), 1j * k * np.exp(-1j * k * dx / 2)


@pytest.mark.parametrize("D", [2, 3])
def test_elastic_p_wave_matches_leapfrog_recurrence(D):
    """A plane compressional wave along x in a homogeneous medium without PML: per Fourier mode,
    v <- v + dt/rho G+ s_xx; s_xx <- s_xx + dt (lambda + 2 mu) G- v; s_yy (, s_zz) <- ... + dt lambda G- v."""
    n, dx, steps = 32, 0.5e-3, 60
    args = []
    for _ in range(D):
        args += [n, dx]
    g = K.KWaveGrid(*args)
    g.dt, g.Nt = 5e-8, steps
    x = np.arange(n)
    line = np.cos(2 * math.pi * 3 * x / n) + 0.5 * np.sin(2 * math.pi * 5 * x / n)
    p0 = np.broadcast_to(line.reshape((-1,) + (1,) * (D - 1)), g.N).copy()
    mask = np.zeros(g.N, bool)
    mask[(slice(None),) + (1,) * (D - 1)] = True
    rho, cp, cs = 1800.0, 3000.0, 1500.0
    r = K.pstd_elastic(g, K.ElasticMedium(cp, cs, rho), K.ElasticSource(p0=p0),
                       K.KWaveSensor(mask=mask, record=["p", "ux"]), pml_size=0)
    lam, mu = rho * (cp ** 2 - 2 * cs ** 2), rho * cs ** 2
    _, gp, gn = _plane_wave_modes(n, dx, 0)
    S = -np.fft.fft(line)
    T = S.copy()
    V = np.zeros(n, complex)
    p_ref, u_ref = np.zeros((n, steps)), np.zeros((n, steps))
    for t in range(steps):
        V = V + g.dt / rho * gp * S
        S, T = S + g.dt * (lam + 2 * mu) * gn * V, T + g.dt * lam * gn * V
        p_ref[:, t] = np.real(np.fft.ifft(-(S + (D - 1) * T) / D))
        u_ref[:, t] = np.real(np.fft.ifft(V))
    assert np.allclose(r["p"], p_ref, rtol=0, atol=1e-12 * np.abs(p_ref).max())
    assert np.allclose(r["ux"], u_ref, rtol=0, atol=1e-12 * np.abs(u_ref).max())


def test_elastic_s_wave_matches_leapfrog_recurrence():
    """A transverse velocity kick vy = f(x) at step 1 (additive source over the whole grid): a plane
    shear wave, per mode vy <- vy + dt/rho G+ s_xy, s_xy <- s_xy + dt mu G- vy; p stays 0."""
    n, dx, steps = 32, 0.5e-3, 50
    g = K.KWaveGrid(n, dx, n, dx)
    g.dt, g.Nt = 5e-8, steps
    x = np.arange(n)
    line = np.cos(2 * math.pi * 2 * x / n)
    u_mask = np.ones((n, n), bool)
    kick = np.zeros((n * n, steps))
    kick[:, 0] = np.tile(line, n)  # column-major points: x fastest
    mask = np.zeros((n, n), bool)
    mask[:, 3] = True
    rho, cp, cs = 1800.0, 3000.0, 1500.0
    r = K.pstd_elastic_2d(g, K.ElasticMedium(cp, cs, rho), K.ElasticSource(u_mask=u_mask, uy=kick),
                          K.KWaveSensor(mask=mask, record=["p", "uy"]), pml_size=0)
    mu = rho * cs ** 2
    _, gp, gn = _plane_wave_modes(n, dx, 0)
    V = np.zeros(n, complex)
    Sxy = np.zeros(n, complex)
    u_ref = np.zeros((n, steps))
    for t in range(steps):
        V = V + g.dt / rho * gp * Sxy
        if t == 0:
            V = V + np.fft.fft(line)
        Sxy = Sxy + g.dt * mu * gn * V
        u_ref[:, t] = np.real(np.fft.ifft(V))
    assert np.allclose(r["uy"], u_ref, rtol=0, atol=1e-12)
    assert np.abs(r["p"]).max() < 1e-12


def test_elastic_kelvin_voigt_factor_in_2d_homogeneous_branch():
    """With alpha_coeff_compression set, the 2D homogeneous stress update scales the constitutive
    term by (1 + chi_p) (solver/elastic.jl:282-295): the plane P wave follows the leapfrog recurrence
    with (lambda + 2 mu)(1 + chi_p) and lambda (1 + chi_p)."""
    n, dx, steps = 32, 0.5e-3, 40
    g = K.KWaveGrid(n, dx, n, dx)
    g.dt, g.Nt = 5e-8, steps
    x = np.arange(n)
    line = np.cos(2 * math.pi * 4 * x / n)
    p0 = np.repeat(line[:, None], n, axis=1)
    mask = np.zeros((n, n), bool)
    mask[:, 2] = True
    rho, cp, cs = 1800.0, 3000.0, 1500.0
    med = K.ElasticMedium(cp, cs, rho, alpha_coeff_compression=0.8, alpha_coeff_shear=0.3, alpha_power=1.3)
    chi_p, _ = K.elastic_chi(med)
    assert chi_p > 0
    r = K.pstd_elastic_2d(g, med, K.ElasticSource(p0=p0), K.KWaveSensor(mask=mask, record=["p"]), pml_size=0)
    lam, mu = rho * (cp ** 2 - 2 * cs ** 2), rho * cs ** 2
    _, gp, gn = _plane_wave_modes(n, dx, 0)
    S = -np.fft.fft(line)
    T = S.copy()
    V = np.zeros(n, complex)
    p_ref = np.zeros((n, steps))
    for t in range(steps):
        V = V + g.dt / rho * gp * S
        S, T = (S + g.dt * (1 + chi_p) * (lam + 2 * mu) * gn * V, T + g.dt * (1 + chi_p) * lam * gn * V)
        p_ref[:, t] = np.real(np.fft.ifft(-(S + T) / 2))
    assert np.allclose(r["p"], p_ref, rtol=0, atol=1e-12 * np.abs(p_ref).max())
    # a heterogeneous density takes the branch without chi
    r2 = K.pstd_elastic_2d(g, K.ElasticMedium(cp, cs, np.full((n, n), rho), alpha_coeff_compression=0.8,
                                              alpha_power=1.3),
                           K.ElasticSource(p0=p0), K.KWaveSensor(mask=mask, record=["p"]), pml_size=0)
    r0 = K.pstd_elastic_2d(g, K.ElasticMedium(cp, cs, rho), K.ElasticSource(p0=p0),
                           K.KWaveSensor(mask=mask, record=["p"]), pml_size=0)
    assert np.allclose(r2["p"], r0["p"], rtol=0, atol=1e-12 * np.abs(r0["p"]).max())


@pytest.mark.parametrize("j,d", [(0, 1), (0, 2), (1, 0), (1, 2), (2, 0), (2, 1)])
def test_elastic_3d_shear_waves_match_leapfrog_recurrence(j, d):
    """3D: a kick in velocity component j that varies along axis d (j != d) is a plane shear wave
    through the stress slot {j, d}: per mode, v_j <- v_j + dt/rho G+_d s_jd, s_jd <- s_jd + dt mu
    G-_d v_j; p stays 0 and the other velocity components stay 0."""
    n, dx, steps = 16, 0.5e-3, 30
    g = K.KWaveGrid(n, dx, n, dx, n, dx)
    g.dt, g.Nt = 5e-8, steps
    line = np.cos(2 * math.pi * 3 * np.arange(n) / n)
    shape = [1, 1, 1]
    shape[d] = n
    field = np.broadcast_to(line.reshape(shape), (n, n, n))
    kick = np.zeros((n ** 3, steps))
    kick[:, 0] = field.ravel(order="F")  # column-major points of the full mask
    comps = {"ux": None, "uy": None, "uz": None}
    comps["u" + "xyz"[j]] = kick
    mask = np.zeros((n, n, n), bool)
    idx = [4, 5, 6]
    idx[d] = slice(None)
    mask[tuple(idx)] = True
    rec = ["p", "ux", "uy", "uz"]
    rho, cp, cs = 1800.0, 3000.0, 1500.0
    r = K.pstd_elastic_3d(g, K.ElasticMedium(cp, cs, rho),
                          K.ElasticSource(u_mask=np.ones((n, n, n), bool), **comps),
                          K.KWaveSensor(mask=mask, record=rec), pml_size=0)
    mu = rho * cs ** 2
    _, gp, gn = _plane_wave_modes(n, dx, 0)
    V = np.zeros(n, complex)
    Sh = np.zeros(n, complex)
    u_ref = np.zeros((n, steps))
    for t in range(steps):
        V = V + g.dt / rho * gp * Sh
        if t == 0:
            V = V + np.fft.fft(line)
        Sh = Sh + g.dt * mu * gn * V
        u_ref[:, t] = np.real(np.fft.ifft(V))
    assert np.allclose(r["u" + "xyz"[j]], u_ref, rtol=0, atol=1e-12)
    for k in range(3):
        if k != j:
            assert np.abs(r["u" + "xyz"[k]]).max() < 1e-12
    assert np.abs(r["p"]).max() < 1e-9 * mu * dx
