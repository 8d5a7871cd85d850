"""The FFT schedule autotuner (the role of the reference's FFTW.MEASURE plans,
KWave.jl/src/fft_utils.jl:59-60): every candidate it may pick computes the same fields, and a
measured schedule is cached on disk per device and grid shape and read back by a new process.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from _util import errors

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _cases():
    from kwave_b200.workloads import c2, c3
    return {
        "stockham_2d_270": c2(n=270, Nt=40, record=("p", "p_max", "p_rms")),
        "register_2d_256": c2(n=256, Nt=40, record=("p", "p_max", "p_rms")),
        "stockham_3d_48": c3(n=48, Nt=30, piston=8, pml=6),
        "stockham_3d_96": c3(n=96, Nt=20, piston=8, pml=6),
        "plane_3d_256": c3(n=256, Nt=6),
    }


def _run(kb, case):
    g, m, s, sen, kw = case.to_api()
    sim = kb.Simulation(g, m, s, sen, extra_sensors=case.extra_sensors, **kw)
    sched = sim.schedule()
    sim.advance(sim.Nt)
    out = sim.outputs()
    sim.close()
    return out, sched


@pytest.fixture(scope="module")
def kb():
    import kwave_b200
    kwave_b200.default_context()
    return kwave_b200


def _fields(out):
    f = dict(out.data)
    for i, e in enumerate(out.extra):
        for k, v in e.items():
            f[f"extra{i}_{k}"] = v
    return f


@pytest.mark.parametrize("name", ["stockham_2d_270", "register_2d_256", "stockham_3d_48", "stockham_3d_96",
                                  "plane_3d_256"])
def test_every_candidate_gives_the_same_fields(kb, name, monkeypatch):
    """Candidates 0..5 of every pass (tile variants, TMA or cp.async staging, lines per tile,
    threads per CTA, the plane pass's six variants): fields bit-identical to the size heuristic's;
    the radix orders explored with KWB_TUNE_ORDER=1 agree to FP32 rounding."""
    case = _cases()[name]
    monkeypatch.setenv("KWB_TUNE", "0")
    ref, sched = _run(kb, case)
    assert sched.startswith("heuristic"), sched
    monkeypatch.delenv("KWB_TUNE")
    for pick in range(6 if name == "plane_3d_256" else 4):
        monkeypatch.setenv("KWB_TUNE_PICK", str(pick))
        out, sched = _run(kb, case)
        assert sched.startswith(f"pick {pick}"), sched
        for k, v in _fields(ref).items():
            assert np.array_equal(_fields(out)[k], v), (name, pick, k, sched)
    monkeypatch.setenv("KWB_TUNE_ORDER", "1")
    for pick in range(3):
        monkeypatch.setenv("KWB_TUNE_PICK", str(pick))
        out, sched = _run(kb, case)
        for k, v in _fields(ref).items():
            l2, mx = errors(_fields(out)[k], v)
            assert l2 <= 1e-6 and mx <= 1e-5, (name, pick, k, l2, mx, sched)


_CHILD = r"""
import json, sys
sys.path[:0] = [sys.argv[1]]
import kwave_b200 as kb
from kwave_b200.workloads import c2
case = c2(n=int(sys.argv[2]), Nt=8, record=("p_max",))
g, m, s, sen, kw = case.to_api()
sim = kb.Simulation(g, m, s, sen, **kw)
print(json.dumps(sim.schedule()))
sim.close()
"""


def test_schedule_cache_round_trips(kb, tmp_path):
    """A first process measures the schedule of a grid shape and appends it to the cache file; a
    second process reads it back ("cache") with the same per-pass choices."""
    cache = tmp_path / "fft_schedules.txt"
    env = dict(os.environ, KWB_TUNE_CACHE=str(cache))
    for k in ("KWB_TUNE", "KWB_TUNE_PICK", "KWB_TUNE_ORDER", "KWB_TILE"):
        env.pop(k, None)
    pkg = os.path.join(ROOT, "k-wave-julia_b200")
    run = lambda: json.loads(subprocess.run([sys.executable, "-c", _CHILD, pkg, "384"], env=env, check=True,
                                            capture_output=True, text=True).stdout.strip().splitlines()[-1])
    first = run()
    assert first.startswith("tuned: "), first
    lines = cache.read_text().strip().splitlines()
    assert len(lines) == 1 and "N384x384x1" in lines[0] and "\t" in lines[0]
    second = run()
    assert second.startswith("cache: "), second
    assert second.split(": ", 1)[1] == first.split(": ", 1)[1]
    assert len(cache.read_text().strip().splitlines()) == 1  # nothing re-measured


def test_tuned_schedule_keeps_results(kb, monkeypatch, tmp_path):
    """The measured schedule (whatever it picks) leaves a 2D Stockham solve bit-identical to the
    heuristic's."""
    case = _cases()["stockham_2d_270"]
    monkeypatch.setenv("KWB_TUNE", "0")
    ref, _ = _run(kb, case)
    monkeypatch.delenv("KWB_TUNE")
    monkeypatch.setenv("KWB_TUNE_CACHE", str(tmp_path / "c.txt"))
    out, sched = _run(kb, case)
    assert sched.startswith("tuned") or sched.startswith("cache"), sched
    for k, v in _fields(ref).items():
        assert np.array_equal(_fields(out)[k], v), k
