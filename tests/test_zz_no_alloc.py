"""kwb_eos_pressure_noalloc: the equation-of-state step for callers that cannot allocate.

Plugin hosts that own all device memory through their own pools, and real-time loops that must
not allocate after start-up, cannot let a library call cudaMalloc.  This test calls the
no-allocation entry point through the C ABI on caller-owned device buffers and checks its
pressure against the regular entry point (kwb_solve) on the same density, twice in a row (the
static scratch keeps the previous call's contents, which must not leak into the next result).

Reference pressure: one kwb_solve step with a Dirichlet pressure source on every voxel and no
other input sets rho_d = s / (D c0^2) everywhere before the equation of state, so the recorded
p_final is exactly EOS(rho_d).  The file is named to run last in a collected session.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-4


def _setup(seed):
    import kwave_b200 as kb
    from kwave_b200.workloads import gaussian_random_field
    shape = (96, 80)
    rng = np.random.default_rng(seed)
    c = gaussian_random_field(rng, shape, 4.0, 1400.0, 1600.0)
    rho0 = gaussian_random_field(rng, shape, 4.0, 900.0, 1100.0)
    bona = gaussian_random_field(rng, shape, 4.0, 4.0, 9.0)
    s = rng.standard_normal(shape) * 1e6
    g = kb.KWaveGrid(shape[0], 1e-4, shape[1], 1e-4)
    g.dt, g.Nt = 0.3e-4 / 1600, 1
    med = kb.KWaveMedium(sound_speed=c, density=rho0, alpha_coeff=0.75, alpha_power=1.3,
                         alpha_mode="no_dispersion", BonA=bona)
    src = kb.KWaveSource(p_mask=np.ones(shape, bool), p=s.ravel(order="F")[:, None], p_mode=kb.Dirichlet)
    out = kb.kspace_first_order(g, med, src, kb.KWaveSensor(mask=np.ones(shape, bool), record=["p_final"]))
    return shape, g, c, rho0, bona, s, out["p_final"]


def _noalloc(lib, shape, g, c, rho0, bona, s):
    import torch
    D = len(shape)
    dev = torch.device("cuda:0")
    f = lambda a: torch.tensor(np.asarray(a, dtype=np.float32).ravel(order="F"), device=dev)
    rho_d = f((s / (D * c ** 2)))  # the source table's FP64 division, rounded once
    rhos = [rho_d.clone() for _ in range(D)]
    c0sq = f(c.astype(np.float64) ** 2)
    nlq = f((bona / 2.0) / rho0)
    p = torch.full((int(np.prod(shape)),), float("nan"), device=dev, dtype=torch.float32)
    rho_ptrs = (C.c_void_p * 3)(*([t.data_ptr() for t in rhos] + [0] * (3 - D)))
    N = (C.c_int64 * 3)(*(list(shape) + [1] * (3 - D)))
    d = (C.c_double * 3)(*([1e-4] * D + [1.0] * (3 - D)))
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.kwb_eos_pressure_noalloc(0, D, N, d, g.dt, float(np.mean(c)), 1, 0.75, 1.3,
                                      rho_ptrs, C.c_void_p(c0sq.data_ptr()), 0.0,
                                      C.c_void_p(nlq.data_ptr()), 0.0, 1, C.c_void_p(p.data_ptr()),
                                      C.c_void_p(stream))
    assert rc == 0, lib.kwb_noalloc_last_error().decode()
    torch.cuda.synchronize(dev)
    return p.cpu().numpy().astype(np.float64)


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


def test_noalloc_matches_regular_entry_point_twice(lib):
    for seed in (11, 12):  # two calls in a row, different inputs
        shape, g, c, rho0, bona, s, p_ref = _setup(seed)
        p = _noalloc(lib, shape, g, c, rho0, bona, s)
        assert np.all(np.isfinite(p))
        rel = np.linalg.norm(p - p_ref) / np.linalg.norm(p_ref)
        assert rel <= TOL_L2, rel


def test_noalloc_rejects_oversize_grid(lib):
    N = (C.c_int64 * 3)(4096, 4096, 1)
    d = (C.c_double * 3)(1e-4, 1e-4, 1.0)
    rho_ptrs = (C.c_void_p * 3)(1, 1, 0)  # never dereferenced: the size check comes first
    rc = lib.kwb_eos_pressure_noalloc(0, 2, N, d, 1e-8, 1500.0, 0, 0.0, 0.0, rho_ptrs, None, 2.25e6,
                                      None, 0.0, 0, C.c_void_p(1), None)
    assert rc == -2
    assert b"exceeds the no-alloc limit" in lib.kwb_noalloc_last_error()
