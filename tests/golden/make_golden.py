"""Writes the golden fixtures tests/golden/<case>.npz: the FP64 oracle's outputs for the seeded
cases in cases.py (the reference itself, Julia, cannot run here; the oracle is pinned on the
reference's own tests and on closed-form answers in tests/test_oracle_kat.py).

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [HERE, os.path.join(HERE, "..", "..", "oracle")]

import cases  # noqa: E402
import kwave_ref  # noqa: E402

if __name__ == "__main__":
    for name in cases.CASES:
        out = cases.run(kwave_ref, name)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(name, {k: v.shape for k, v in out.items()}, os.path.getsize(path), "bytes")
