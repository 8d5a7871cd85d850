"""Shared helpers for the parity tests: run a workload Case through the GPU library and the oracle
and compare every output field."""
from __future__ import annotations

import numpy as np


def oracle_inputs(case):
    import kwave_ref as K
    args = []
    for n, d in zip(case.N, case.d):
        args += [n, d]
    g = K.KWaveGrid(*args)
    g.dt = case.dt
    g.Nt = case.Nt
    g.t_array = np.arange(case.Nt) * case.dt
    src = dict(case.source)
    for k in ("p_mode", "u_mode"):
        if k in src:
            src[k] = int(src[k])
    return (g, K.KWaveMedium(**case.medium), K.KWaveSource(**src), K.KWaveSensor(**case.sensor),
            dict(pml_size=case.pml_size, pml_alpha=case.pml_alpha, smooth_p0=case.smooth_p0))


def run_oracle(case, **kw):
    import kwave_ref as K
    g, m, s, sen, opts = oracle_inputs(case)
    opts.update(kw)
    return K.kspace_first_order(g, m, s, sen, extra_sensors=case.extra_sensors, **opts)


def run_gpu(case, **kw):
    import kwave_b200 as kb
    g, m, s, sen, opts = case.to_api()
    opts.update(kw)
    if case.extra_sensors:
        sim = kb.Simulation(g, m, s, sen, extra_sensors=case.extra_sensors, **opts)
        sim.advance(sim.Nt)
        out = sim.outputs()
        sim.close()
        return out
    return kb.kspace_first_order(g, m, s, sen, **opts)


def errors(gpu, ref):
    """(rel-L2, max-abs / max|ref|) of two arrays, ignoring +-inf entries present in both."""
    a = np.asarray(gpu, dtype=np.float64)
    b = np.asarray(ref, dtype=np.float64)
    assert a.shape == b.shape, (a.shape, b.shape)
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin), "non-finite entries differ"
    if not fin.any():
        assert np.array_equal(a, b)
        return 0.0, 0.0
    a, b = a[fin], b[fin]
    nb = np.linalg.norm(b)
    if nb == 0:
        return float(np.linalg.norm(a)), float(np.max(np.abs(a)))
    return float(np.linalg.norm(a - b) / nb), float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def assert_parity(gpu_out, ref_out, tol_l2=1e-4, tol_max=1e-3, fields=None, report=None):
    keys = fields or [k for k in ref_out.keys() if not k.startswith("_")]
    assert set(keys) <= set(gpu_out.keys()), (sorted(gpu_out.keys()), keys)
    res = {}
    for k in keys:
        l2, mx = errors(gpu_out[k], ref_out[k])
        res[k] = (l2, mx)
        assert l2 <= tol_l2 and mx <= tol_max, f"{k}: rel-L2 {l2:.3e}, max {mx:.3e}"
    if report is not None:
        report.update(res)
    return res
