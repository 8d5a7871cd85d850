"""Golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py from the FP64
oracle on the seeded cases of tests/golden/cases.py): the oracle must still reproduce them, and
the GPU library must match them at the parity gate."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, HERE)

import cases  # noqa: E402
from _util import assert_parity  # noqa: E402


def _fixture(name):
    with np.load(os.path.join(HERE, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_oracle_reproduces_golden(name):
    import kwave_ref
    got = cases.run(kwave_ref, name)
    ref = _fixture(name)
    assert set(got) == set(ref)
    for k in ref:
        scale = max(np.abs(ref[k]).max(), 1e-300)
        assert np.allclose(got[k], ref[k], rtol=0, atol=1e-9 * scale), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_gpu_matches_golden(name):
    import kwave_b200
    got = cases.run(kwave_b200, name)
    assert_parity(got, _fixture(name), 1e-4, 1e-3)


def test_full_horizon_fixtures_are_consistent():
    """The full-horizon FP64 fixtures (make_long_golden.py): shapes, horizons and properties of
    the stored samples; the sampled serving request 16 (324 x 320, 317 steps) is re-run through
    the oracle and reproduced."""
    import make_long_golden as M
    c2 = np.load(os.path.join(HERE, "c2_long.npz"))
    assert int(c2["Nt"]) == 2000 and c2["p_max"].shape == c2["p_rms"].shape == (512 * 512,)
    assert np.all(c2["p_rms"] >= 0) and np.all(np.isfinite(c2["p_max"]))
    assert np.max(c2["p_rms"]) <= np.max(np.abs(c2["p_max"]))
    plane, vol = M.c3_samples(256)
    assert plane.size == 1024 and vol.size == 64 ** 3 and np.all(np.diff(plane) > 0)
    path = os.path.join(HERE, "c3_long.npz")
    if os.path.exists(path):
        c3 = np.load(path)
        assert int(c3["Nt"]) == 1500 and c3["p"].shape == (1024, 1500)
        assert np.array_equal(c3["plane_idx"], plane) and np.array_equal(c3["vol_idx"], vol)
        assert np.all(np.isfinite(c3["p_max"])) and np.all(np.isfinite(c3["p"]))
    sv = np.load(os.path.join(HERE, "serving_sample.npz"))
    assert list(sv["requests"]) == list(M.SERVING_SAMPLE)
    import kwave_ref as K
    from _util import oracle_inputs
    from kwave_b200 import workloads
    case = workloads.c5_request(16, seed=M.SERVING_SEED, nt_range=M.SERVING_NT)
    g, m, s, sen, opts = oracle_inputs(case)
    p = K.kspace_first_order(g, m, s, sen, **opts)["p"]
    ref = sv["p_16"].astype(np.float64)
    assert np.allclose(p, ref, rtol=0, atol=1e-6 * np.abs(ref).max())
