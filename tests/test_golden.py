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
