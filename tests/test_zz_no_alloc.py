"""kwb_eos_pressure_noalloc: the equation-of-state step for callers that cannot allocate.

Plugin hosts that own all device memory through their own pools, and real-time loops that must
not allocate after start-up, cannot let a library call cudaMalloc.  These tests call the
no-allocation entry point through the C ABI on caller-owned device buffers and check its
pressure two ways, twice in a row per case (the static scratch keeps the previous call's
contents, which must not leak into the next result):

* against the regular entry point (kwb_solve): one time step with a Dirichlet pressure source on
  every voxel and no other input sets rho_d = s / (D c0^2) everywhere before the equation of
  state, so the recorded p_final is exactly EOS(rho_d);
* against the FP64 oracle's equation of state (``_compute_pressure``, the restatement of
  ``solver/first_order_steps.jl:214-290``) on the same density.

Cases cover 1D, 2D and 3D grids (the 3D case runs the three-spectrum-pass sequence), power-of-two
and 3/5-smooth sides, heterogeneous and scalar sound speed, linear and nonlinear media, and the
lossless and absorbing (no-dispersion) branches.  The file is named to run last in a collected
session.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-4
TOL_MAX = 1e-3

# name: (shape, heterogeneous c0, nonlinear, alpha_mode (0 none, 1 no_dispersion), alpha_power)
CASES = {
    "2d_heterogeneous_nonlinear_absorbing": ((96, 80), True, True, 1, 1.3),
    "3d_heterogeneous_nonlinear_absorbing": ((64, 48, 40), True, True, 1, 1.1),
    "3d_scalar_c_nonlinear_absorbing": ((24, 20, 16), False, True, 1, 1.5),
    "2d_scalar_c_linear_lossless": ((90, 72), False, False, 0, 0.0),
    "1d_heterogeneous_linear_absorbing": ((128,), True, False, 1, 1.8),
}
ALPHA_COEFF = 0.75
DX = 1e-4


def _inputs(shape, het_c, nonlinear, seed):
    from kwave_b200.workloads import gaussian_random_field
    rng = np.random.default_rng(seed)
    sig = 2.0 if min(shape) < 32 else 4.0
    if het_c:
        c = gaussian_random_field(rng, shape, sig, 1400.0, 1600.0)
    else:
        c = 1500.0
    rho0 = gaussian_random_field(rng, shape, sig, 900.0, 1100.0)
    bona = gaussian_random_field(rng, shape, sig, 4.0, 9.0) if nonlinear else None
    s = rng.standard_normal(shape) * 1e6
    return c, rho0, bona, s


def _grid_args(shape):
    args = []
    for n in shape:
        args += [n, DX]
    return args


def _solve_reference(shape, dt, c, rho0, bona, s, alpha_mode, y):
    """p_final of one kwb_solve step whose Dirichlet source fixes rho_d = s/(D c0^2) everywhere."""
    import kwave_b200 as kb
    g = kb.KWaveGrid(*_grid_args(shape))
    g.dt, g.Nt = dt, 1
    kw = dict(sound_speed=c, density=rho0, BonA=bona)
    if alpha_mode:
        kw.update(alpha_coeff=ALPHA_COEFF, alpha_power=y, alpha_mode="no_dispersion")
    src = kb.KWaveSource(p_mask=np.ones(shape, bool), p=s.ravel(order="F")[:, None], p_mode=kb.Dirichlet)
    out = kb.kspace_first_order(g, kb.KWaveMedium(**kw), src,
                                kb.KWaveSensor(mask=np.ones(shape, bool), record=["p_final"]))
    return out["p_final"]


def _oracle_reference(shape, dt, c, rho0, bona, rho_total, alpha_mode, y):
    """The oracle's equation of state on the density the GPU was given (FP64)."""
    import kwave_ref as K
    g = K.KWaveGrid(*_grid_args(shape))
    n1 = shape[0] // 2 + 1
    c_ref = float(c) if np.ndim(c) == 0 else float(np.mean(c))
    kappa = K.compute_kappa(g.k, c_ref, dt)[:n1]
    absorb = None
    if alpha_mode:
        med = K.KWaveMedium(sound_speed=c, density=rho0, alpha_coeff=ALPHA_COEFF, alpha_power=y,
                            alpha_mode="no_dispersion")
        a = K.precompute_absorption(med, g.k, c_ref)
        absorb = K.AbsorptionParams(a.tau, a.eta, a.nabla1[:n1], a.nabla2[:n1], a.mode)
    p = K._compute_pressure(rho_total, None, kappa, c, rho0, bona, absorb, K._Plans(shape), dt, np.float64)
    return np.asarray(p).ravel(order="F")


def _noalloc(lib, shape, dt, c, rho0, bona, s, alpha_mode, y):
    """(p from kwb_eos_pressure_noalloc, the FP32 split density it was given, summed in FP64)."""
    import torch
    D = len(shape)
    dev = torch.device("cuda:0")
    f = lambda a: torch.tensor(np.asarray(a, dtype=np.float32).ravel(order="F"), device=dev)
    c64 = np.asarray(c, dtype=np.float64)
    rho_d32 = np.asarray(s / (D * c64 ** 2), dtype=np.float32)  # the source table's FP64 division, rounded once
    rhos = [f(rho_d32) for _ in range(D)]
    het = np.ndim(c) > 0
    c0sq = f(c64 ** 2) if het else None
    nlq = f((bona / 2.0) / rho0) if bona is not None else None
    p = torch.full((int(np.prod(shape)),), float("nan"), device=dev, dtype=torch.float32)
    rho_ptrs = (C.c_void_p * 3)(*([t.data_ptr() for t in rhos] + [0] * (3 - D)))
    N = (C.c_int64 * 3)(*(list(shape) + [1] * (3 - D)))
    d = (C.c_double * 3)(*([DX] * D + [1.0] * (3 - D)))
    stream = torch.cuda.current_stream(dev).cuda_stream
    c_ref = float(np.mean(c64)) if het else float(c)
    rc = lib.kwb_eos_pressure_noalloc(0, D, N, d, dt, c_ref, alpha_mode, ALPHA_COEFF if alpha_mode else 0.0,
                                      y if alpha_mode else 0.0, rho_ptrs,
                                      C.c_void_p(c0sq.data_ptr() if c0sq is not None else 0),
                                      0.0 if het else float(c) ** 2,
                                      C.c_void_p(nlq.data_ptr() if nlq is not None else 0), 0.0,
                                      1 if bona is not None else 0, C.c_void_p(p.data_ptr()), C.c_void_p(stream))
    assert rc == 0, lib.kwb_noalloc_last_error().decode()
    torch.cuda.synchronize(dev)
    rho_total = D * rho_d32.astype(np.float64)
    return p.cpu().numpy().astype(np.float64), rho_total


def _err(a, b):
    return (float(np.linalg.norm(a - b) / np.linalg.norm(b)), float(np.max(np.abs(a - b)) / np.max(np.abs(b))))


@pytest.fixture(scope="module")
def lib():
    import kwave_b200 as kb
    L = kb.load_library()
    L.kwb_eos_pressure_noalloc.restype = C.c_int
    L.kwb_eos_pressure_noalloc.argtypes = [
        C.c_int, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_double), C.c_double, C.c_double,
        C.c_int32, C.c_double, C.c_double, C.POINTER(C.c_void_p), C.c_void_p, C.c_float,
        C.c_void_p, C.c_float, C.c_int32, C.c_void_p, C.c_void_p]
    L.kwb_noalloc_last_error.restype = C.c_char_p
    L.kwb_noalloc_last_error.argtypes = []
    kb.default_context()
    return L


@pytest.mark.parametrize("name", list(CASES))
def test_noalloc_matches_regular_entry_point_and_oracle_twice(lib, name):
    shape, het_c, nonlinear, alpha_mode, y = CASES[name]
    dt = 0.3 * DX / 1600.0
    for seed in (11, 12):  # two calls in a row, different inputs
        c, rho0, bona, s = _inputs(shape, het_c, nonlinear, seed)
        p, rho_total = _noalloc(lib, shape, dt, c, rho0, bona, s, alpha_mode, y)
        assert np.all(np.isfinite(p))
        p_solve = _solve_reference(shape, dt, c, rho0, bona, s, alpha_mode, y)
        l2, mx = _err(p, p_solve)
        assert l2 <= TOL_L2 and mx <= TOL_MAX, (name, seed, "vs kwb_solve", l2, mx)
        rt = rho_total.reshape(shape, order="F")
        p_oracle = _oracle_reference(shape, dt, c, rho0, bona, rt, alpha_mode, y)
        l2, mx = _err(p, p_oracle)
        assert l2 <= TOL_L2 and mx <= TOL_MAX, (name, seed, "vs oracle", l2, mx)


def test_noalloc_rejects_oversize_grid(lib):
    N = (C.c_int64 * 3)(4096, 4096, 1)
    d = (C.c_double * 3)(1e-4, 1e-4, 1.0)
    rho_ptrs = (C.c_void_p * 3)(1, 1, 0)  # never dereferenced: the size check comes first
    rc = lib.kwb_eos_pressure_noalloc(0, 2, N, d, 1e-8, 1500.0, 0, 0.0, 0.0, rho_ptrs, None, 2.25e6,
                                      None, 0.0, 0, C.c_void_p(1), None)
    assert rc == -2
    assert b"exceeds the no-alloc limit" in lib.kwb_noalloc_last_error()


def test_noalloc_rejects_invalid_absorption(lib):
    N = (C.c_int64 * 3)(64, 64, 1)
    d = (C.c_double * 3)(1e-4, 1e-4, 1.0)
    rho_ptrs = (C.c_void_p * 3)(1, 1, 0)  # never dereferenced: validation comes first
    rc = lib.kwb_eos_pressure_noalloc(0, 2, N, d, 1e-8, 1500.0, 7, 0.5, 1.1, rho_ptrs, None, 2.25e6,
                                      None, 0.0, 0, C.c_void_p(1), None)
    assert rc == -1 and b"alpha_mode" in lib.kwb_noalloc_last_error()
    rc = lib.kwb_eos_pressure_noalloc(0, 2, N, d, 1e-8, 1500.0, 1, float("nan"), 1.1, rho_ptrs, None, 2.25e6,
                                      None, 0.0, 0, C.c_void_p(1), None)
    assert rc == -1 and b"finite" in lib.kwb_noalloc_last_error()
