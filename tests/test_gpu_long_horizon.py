"""Full-horizon parity of the two benchmark solves against the FP64 oracle.

The oracle's outputs over every time step are committed as subsampled golden fixtures
(``tests/golden/make_long_golden.py`` wrote them; an FP64 run of the 256^3 x 1500-step solve
takes hours of CPU, far too long to repeat in a test):

* the 512^2 x 2000-step heterogeneous absorbing solve: full-grid p_max and p_rms;
* the 256^3 x 1500-step nonlinear absorbing solve: the pressure series at 1024 points of the
  recorded xy plane and p_max at every 4th voxel along each axis.

The GPU runs the same seeded inputs through the public API.  Gate: relative L2 <= 1e-4 and max
error <= 1e-3 of the field's peak, the hot path's accuracy target, over the whole horizon.
"""
import os

import numpy as np
import pytest

from _util import errors, run_gpu

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-4
TOL_MAX = 1e-3
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _mask(shape, lin):
    m = np.zeros(int(np.prod(shape)), dtype=bool)
    m[lin] = True
    return m.reshape(shape, order="F")


@pytest.fixture(scope="module")
def wl():
    import kwave_b200
    from kwave_b200 import workloads
    kwave_b200.default_context()
    return workloads


def test_c2_full_horizon_against_fp64_golden(wl):
    """512^2, 2000 steps: full-grid p_max and p_rms against the FP64 oracle's."""
    gold = np.load(os.path.join(GOLDEN, "c2_long.npz"))
    case = wl.c2()
    assert int(gold["Nt"]) == case.Nt == 2000
    out = run_gpu(case)
    rep = {}
    for k in ("p_max", "p_rms"):
        l2, mx = errors(out[k], gold[k].astype(np.float64))
        rep[k] = (l2, mx)
        assert l2 <= TOL_L2 and mx <= TOL_MAX, (k, l2, mx)
    print("c2 512^2 x 2000", rep)




def test_c3_full_horizon_against_fp64_golden(wl):
    """256^3, 1500 steps (the nonlinear absorbing workload the throughput is quoted on): the plane
    p series at 1024 sampled points and the volume p_max at every 4th voxel against the FP64
    oracle's run of all 1500 steps."""
    gold = np.load(os.path.join(GOLDEN, "c3_long.npz"))
    case = wl.c3()
    assert int(gold["Nt"]) == case.Nt == 1500
    case.sensor = dict(mask=_mask(case.N, gold["plane_idx"]), record=["p"])
    case.extra_sensors = [dict(mask=_mask(case.N, gold["vol_idx"]), record=["p_max"])]
    out = run_gpu(case)
    rep = {}
    for k, got, ref in (("p", out["p"], gold["p"]), ("p_max", out.extra[0]["p_max"], gold["p_max"])):
        l2, mx = errors(got, ref.astype(np.float64))
        rep[k] = (l2, mx)
        assert l2 <= TOL_L2 and mx <= TOL_MAX, (k, l2, mx)
    print("c3 256^3 x 1500", rep)


def test_sampled_serving_requests_against_fp64_golden(wl):
    """Requests 0, 16 and 22 of the 48-request serving stream (two 2D, one 64^3), served together
    through the continuous-batching scheduler: each p series against the FP64 oracle's
    (tests/golden/serving_sample.npz)."""
    import kwave_b200 as kb
    gold = np.load(os.path.join(GOLDEN, "serving_sample.npz"))
    reqs = {}
    for i in gold["requests"]:
        case = wl.c5_request(int(i), seed=5005, nt_range=(300, 800))
        g, m, s, sen, kw = case.to_api()
        reqs[int(i)] = kb.submit(g, m, s, sen, **kw)
    for i, r in reqs.items():
        l2, mx = errors(r.result()["p"], gold[f"p_{i}"].astype(np.float64))
        assert l2 <= TOL_L2 and mx <= TOL_MAX, (i, l2, mx)
