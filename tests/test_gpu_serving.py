"""Continuous batching on one GPU: results in the mix equal results alone; admission, cancellation
and per-request failures behave; a sampled subset matches the FP64 oracle."""
import math

import numpy as np
import pytest

from _util import assert_parity, run_oracle

pytestmark = pytest.mark.gpu


def _mix():
    from kwave_b200 import workloads as W
    cases = [W.c4_sim(i, sides=(128, 192, 256), nt_range=(60, 160)) for i in range(5)]
    cases += [W.c5_request(i, nt_range=(40, 90)) for i in (3, 7)]
    small3d = W.c3(n=48, Nt=70, piston=8, pml=6)
    cases.append(small3d)
    return cases


def _alone(kb, case):
    g, m, s, sen, kw = case.to_api()
    if case.extra_sensors:
        sim = kb.Simulation(g, m, s, sen, extra_sensors=case.extra_sensors, **kw)
        sim.advance(sim.Nt)
        out = sim.outputs()
        sim.close()
        return out
    return kb.kspace_first_order(g, m, s, sen, **kw)


def test_results_in_the_mix_equal_results_alone():
    import kwave_b200 as kb
    cases = _mix()
    alone = [_alone(kb, c) for c in cases]
    kb.serving_config(max_running=64, chunk_steps=16)
    reqs = []
    for c in cases:
        g, m, s, sen, kw = c.to_api()
        reqs.append(kb.submit(g, m, s, sen, extra_sensors=c.extra_sensors, **kw))
    outs = [r.result(timeout=300) for r in reqs]
    st = kb.serving_stats()
    assert st["peak_running"] >= 2, st  # requests really overlapped
    for c, a, o in zip(cases, alone, outs):
        for k in a.keys():
            assert np.array_equal(a[k], o[k]), (c.name, k)
        for ea, eo in zip(a.extra, o.extra):
            for k in ea:
                assert np.array_equal(ea[k], eo[k]), (c.name, k)
    # a sampled subset against the FP64 oracle (rel-L2 <= 1e-4); cases whose sensors the wave has
    # reached (a sensor the wave has not reached yet sees only the k-space method's pre-arrival
    # tail, where FP32 and FP64 differ by design)
    ref0 = run_oracle(cases[0])
    assert_parity(outs[0], ref0, 1e-4, 1e-3)
    ref7 = run_oracle(cases[7])
    assert_parity(outs[7], ref7, 1e-4, 1e-3)
    assert_parity(outs[7].extra[0], ref7["_extra"][0], 1e-4, 1e-3)


def test_admission_by_memory_cap_serialises():
    import kwave_b200 as kb
    from kwave_b200 import workloads as W
    cases = [W.c4_sim(i, sides=(128,), nt_range=(40, 60)) for i in range(3)]
    g, m, s, sen, kw = cases[0].to_api()
    one = kb.estimate_device_bytes(g, m, s, sen, **kw)
    ctx = kb.Context(0)
    kb.serving_config(max_running=8, chunk_steps=8, mem_cap_bytes=int(one * 1.5), context=ctx)
    reqs = []
    for c in cases:
        g, m, s, sen, kw = c.to_api()
        reqs.append(kb.submit(g, m, s, sen, context=ctx, **kw))
    outs = [r.result(timeout=120) for r in reqs]
    st = kb.serving_stats(context=ctx)
    assert st["peak_running"] == 1 and st["completed"] == 3, st
    for c, o in zip(cases, outs):
        assert np.array_equal(_alone(kb, c)["p"], o["p"])
    ctx.close()


def test_cancel_and_failures_stay_per_request():
    import kwave_b200 as kb
    from kwave_b200 import workloads as W
    ctx = kb.Context(0)
    good = W.c4_sim(1, sides=(128,), nt_range=(50, 50))
    long_ = W.c4_sim(2, sides=(128,), nt_range=(4000, 4000))
    big = W.c4_sim(5, sides=(1024,), nt_range=(50, 50))
    g, m, s, sen, kw = long_.to_api()
    gb, mb, sb, senb, kwb = good.to_api()
    cap = int(1.2 * max(kb.estimate_device_bytes(g, m, s, sen, context=ctx, **kw),
                        kb.estimate_device_bytes(gb, mb, sb, senb, context=ctx, **kwb)))
    kb.serving_config(max_running=4, chunk_steps=4, mem_cap_bytes=cap, context=ctx)
    # an invalid problem is rejected synchronously at submission, like the reference's error()
    nb = 2 * 1031  # a prime factor above 7 and longer than the Bluestein limit: unsupported
    bad_g = kb.KWaveGrid(nb, 1e-4, 16, 1e-4)
    kb.make_time(bad_g, 1500.0, t_end=1e-6)
    with pytest.raises(kb.KWaveB200Error) as e:
        kb.submit(bad_g, kb.KWaveMedium(sound_speed=1500.0), kb.KWaveSource(p0=np.ones((nb, 16))),
                  kb.KWaveSensor(mask=np.ones((nb, 16), bool)), context=ctx)
    assert e.value.code == -2
    r_long = kb.submit(g, m, s, sen, context=ctx, **kw)
    g2, m2, s2, sen2, kw2 = big.to_api()
    r_big = kb.submit(g2, m2, s2, sen2, context=ctx, **kw2)  # larger than the memory cap
    g3, m3, s3, sen3, kw3 = good.to_api()
    r_good = kb.submit(g3, m3, s3, sen3, context=ctx, **kw3)
    r_long.cancel()
    with pytest.raises(kb.KWaveB200Error) as e:
        r_long.result(timeout=120)
    assert e.value.code == -6
    with pytest.raises(kb.KWaveB200Error) as e:
        r_big.result(timeout=120)
    assert e.value.code == -3
    out = r_good.result(timeout=120)
    assert np.array_equal(out["p"], _alone(kb, good)["p"])
    st = kb.serving_stats(context=ctx)
    assert st["cancelled"] == 1 and st["failed"] == 1 and st["completed"] == 1, st
    ctx.close()


def test_wait_timeout_then_completion():
    import kwave_b200 as kb
    from kwave_b200 import workloads as W
    c = W.c4_sim(3, sides=(256,), nt_range=(800, 800))
    g, m, s, sen, kw = c.to_api()
    r = kb.submit(g, m, s, sen, **kw)
    try:
        r.result(timeout=1e-4)
        finished_early = True
    except TimeoutError:
        finished_early = False
    out = r.result(timeout=300)
    assert out["p"].shape[1] == c.Nt and (finished_early or r.latency_s > 0)
