"""Writes the full-horizon golden fixtures of the two benchmark solves: the FP64 oracle run over
every time step of the 256^3 x 1500-step nonlinear absorbing solve and of the 512^2 x 2000-step
heterogeneous absorbing solve, stored as fixed subsamples (FP32 storage of FP64 values; the
storage rounding, ~6e-8 relative, is far below the 1e-4 parity gate).

    python tests/golden/make_long_golden.py c3     # ~1500 FP64 steps on 256^3: hours of CPU
    python tests/golden/make_long_golden.py c2     # ~2000 FP64 steps on 512^2: minutes
    python tests/golden/make_long_golden.py serving  # the sampled serving requests

Inputs come from the seeded workload builders (``kwave_b200.workloads``), so the GPU tests and
``bench.py`` rebuild bit-identical inputs.  Samples:

* c3_long.npz   ``plane_idx``: 1024 points of the recorded xy plane (every 8th x and y, offset 4),
                ``p``: their pressure series [1024 x 1500]; ``vol_idx``: every 4th voxel along
                each axis (offset 1), ``p_max``: the volume p_max there [262144].
* c2_long.npz   ``p_max``, ``p_rms``: the full-grid aggregates [262144] each.
* serving_sample.npz  for requests 0, 16 and 22 of the 48-request serving stream (Nt 300-800,
                seed 5005): its 16-point sensor line's p series.

Indices are column-major (Julia) linear indices, the order the reference's ``findall`` returns.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "k-wave-julia_b200"),
                os.path.join(ROOT, "tests")]

# serving stream sampled for per-request accuracy: two 2D requests and one 3D request of the 48
SERVING_SEED = 5005
SERVING_NT = (300, 800)
SERVING_SAMPLE = (0, 16, 22)


def c3_samples(n=256):
    """(plane_idx, vol_idx): column-major linear indices of the sampled plane points and voxels."""
    z = n // 2 - 1
    xs = np.arange(4, n, 8)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    plane = np.sort((X + n * Y + n * n * z).ravel(order="F"))
    vs = np.arange(1, n, 4)
    X, Y, Z = np.meshgrid(vs, vs, vs, indexing="ij")
    vol = np.sort((X + n * Y + n * n * Z).ravel(order="F"))
    return plane.astype(np.int64), vol.astype(np.int64)


def _mask(shape, lin):
    m = np.zeros(int(np.prod(shape)), dtype=bool)
    m[lin] = True
    return m.reshape(shape, order="F")


def run_c3(out_path, steps=None):
    import kwave_ref as K
    from _util import oracle_inputs
    from kwave_b200 import workloads
    case = workloads.c3()
    plane_idx, vol_idx = c3_samples(case.N[0])
    case.sensor = dict(mask=_mask(case.N, plane_idx), record=["p"])
    case.extra_sensors = [dict(mask=_mask(case.N, vol_idx), record=["p_max"])]
    g, m, s, sen, opts = oracle_inputs(case)
    t0 = time.time()
    last = [t0]

    def progress(t, nt, p):
        if t % 25 == 0 or t == 1:
            now = time.time()
            print(f"c3 step {t}/{nt}  {now - t0:.0f} s  ({(now - last[0]) / (25 if t > 1 else 1):.2f} s/step)",
                  flush=True)
            last[0] = now

    out = K.kspace_first_order(g, m, s, sen, extra_sensors=case.extra_sensors, max_steps=steps,
                               progress_callback=progress, **opts)
    np.savez_compressed(out_path, plane_idx=plane_idx, p=out["p"].astype(np.float32),
                        vol_idx=vol_idx, p_max=out["_extra"][0]["p_max"].astype(np.float32),
                        Nt=np.int64(case.Nt if steps is None else steps), seconds=np.float64(time.time() - t0))
    print("wrote", out_path, os.path.getsize(out_path), "bytes", f"{time.time() - t0:.0f} s")


def run_c2(out_path, steps=None):
    import kwave_ref as K
    from _util import oracle_inputs
    from kwave_b200 import workloads
    case = workloads.c2()
    g, m, s, sen, opts = oracle_inputs(case)
    t0 = time.time()
    out = K.kspace_first_order(g, m, s, sen, max_steps=steps, **opts)
    np.savez_compressed(out_path, p_max=out["p_max"].astype(np.float32), p_rms=out["p_rms"].astype(np.float32),
                        Nt=np.int64(case.Nt if steps is None else steps), seconds=np.float64(time.time() - t0))
    print("wrote", out_path, os.path.getsize(out_path), "bytes", f"{time.time() - t0:.0f} s")


def run_serving(out_path):
    import kwave_ref as K
    from _util import oracle_inputs
    from kwave_b200 import workloads
    res = {}
    for i in SERVING_SAMPLE:
        case = workloads.c5_request(i, seed=SERVING_SEED, nt_range=SERVING_NT)
        g, m, s, sen, opts = oracle_inputs(case)
        t0 = time.time()
        out = K.kspace_first_order(g, m, s, sen, **opts)
        res[f"p_{i}"] = out["p"].astype(np.float32)
        print(case.name, case.Nt, f"{time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(out_path, requests=np.asarray(SERVING_SAMPLE, np.int64), **res)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


if __name__ == "__main__":
    what = sys.argv[1]
    steps = int(sys.argv[2]) if len(sys.argv) > 2 else None
    dest = sys.argv[3] if len(sys.argv) > 3 else None
    if what == "c3":
        run_c3(dest or os.path.join(HERE, "c3_long.npz"), steps)
    elif what == "c2":
        run_c2(dest or os.path.join(HERE, "c2_long.npz"), steps)
    elif what == "serving":
        run_serving(dest or os.path.join(HERE, "serving_sample.npz"))
    else:
        raise SystemExit(f"unknown fixture {what!r}")
