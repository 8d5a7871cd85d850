#!/usr/bin/env python
"""Benchmark of the fluid k-space time-stepping path on B200 (one JSON line on rank 0).

Workload (N = 1): the 256^3 heterogeneous nonlinear absorbing solve (y = 1.1, BonA 5 with a
B/A = 9 ball, 32x32 ux piston, xy-plane p + volume p_max), Nt = 1500, seeded synthetic media.
A "step" is one time step of that simulation.  ``value`` is voxel-steps/s over K device-timed
steps with all fields resident in HBM (CUDA events on the simulation's stream, max over ranks);
``e2e`` is one full solve through the public API from host arrays to FP64 outputs (wall clock,
host<->device copies inside), and ``accuracy`` compares that solve with the FP64 oracle's run of
all 1500 steps (tests/golden/c3_long.npz).  Further keys: ``c2`` (the 512^2 x 2000-step solve,
device-timed, with its accuracy against the oracle's 2000 steps), ``batch`` (64 mixed-size 2D
simulations), ``serving`` (Poisson arrivals, p50/p99, sampled accuracy), ``elastic``,
``comparators`` (the reference's step on cuFFT), ``cpu_baseline``.  Multi-GPU: every rank runs
its own independent simulation (weak scaling; simulations shard with no collective).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config c3|c2]
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "k-wave-julia_b200"))

# DRAM bytes read + written (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the
# dominant kernel, from one capture on a B200 (the x line pass with the EOS operand prefetch and
# the tuned 128-thread tiles; profiles/line_pass_x_eos_256cubed_ncu.md):
#   ncu --set full --clock-control none --kernel-name-base demangled
#       -k 'regex:k_line_fast<.*\(bool\)1, \(int\)[0-9]+, \(int\)2, \(bool\)1>' -s 14 -c 1
#       python bench.py --steps 4 --warmup 3 --no-e2e --no-cpu --no-batch --no-serve --no-elastic
#       --no-cufft --no-c2
# Reads equal the algorithmic bytes; writes land lower because part of each launch's output is
# still in L2 when the launch ends.
NCU_TRAFFIC = {("c3", "line_pass_x_eos_fwd"): 713.9e6}

# Spectral-pass-model words per voxel-step (algorithmic bytes = 4 B x words), per config.
SPM_WORDS = {"c3": 33.0, "c2": 26.0, "c1": 15.01}
UNIT = "Gvoxel-steps/s"
METRIC = "Gvoxel-steps/s (fluid k-space time stepping)"


GOLDEN = os.path.join(ROOT, "tests", "golden")


def rel_errors(gpu, ref):
    """(relative L2, max abs error / max |ref|) of a result against the FP64 oracle's."""
    import numpy as np
    a = np.asarray(gpu, dtype=np.float64).ravel()
    b = np.asarray(ref, dtype=np.float64).ravel()
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b) / nb), float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def c3_accuracy(case, out):
    """Errors of a full 256^3 x 1500-step solve against the FP64 oracle's run of all 1500 steps
    (tests/golden/c3_long.npz): the plane p series at its 1024 sampled points and the volume p_max
    at every 4th voxel along each axis."""
    import numpy as np
    path = os.path.join(GOLDEN, "c3_long.npz")
    if not os.path.exists(path):
        return {"unavailable": "no full-horizon FP64 golden for this workload"}
    gold = np.load(path)
    plane_rows = np.flatnonzero(np.asarray(case.sensor["mask"]).ravel(order="F"))
    rows = np.searchsorted(plane_rows, gold["plane_idx"])
    l2p, mxp = rel_errors(out["p"][rows, :], gold["p"])
    l2v, mxv = rel_errors(out.extra[0]["p_max"][gold["vol_idx"]], gold["p_max"])
    return {"reference": "FP64 oracle, all 1500 steps (tests/golden/c3_long.npz)",
            "p": {"rel_l2": l2p, "max_rel": mxp, "sample": f"{len(rows)} plane points x {gold['p'].shape[1]} steps"},
            "p_max": {"rel_l2": l2v, "max_rel": mxv, "sample": f"{len(gold['vol_idx'])} voxels (every 4th per axis)"}}


def c2_leg(ctx, warmup=40):
    """The 512^2 x 2000-step heterogeneous absorbing solve: every step device-timed in one
    advance (CUDA events), and its full-grid p_max / p_rms against the FP64 oracle's 2000-step
    run (tests/golden/c2_long.npz)."""
    import numpy as np
    import kwave_b200 as kb
    from kwave_b200 import workloads
    warm = workloads.c2(Nt=warmup)
    g, m, s, sen, kw = warm.to_api()
    w = kb.Simulation(g, m, s, sen, context=ctx, **kw)
    w.advance_timed(warmup)
    w.close()
    case = workloads.c2()
    g, m, s, sen, kw = case.to_api()
    sim = kb.Simulation(g, m, s, sen, context=ctx, **kw)
    ms = sim.advance_timed(case.Nt)
    out = sim.outputs()
    sched = sim.schedule()
    sim.close()
    peak, kind = peaks()
    value = case.voxels * case.Nt / (ms / 1e3) / 1e9
    res = {"workload": case.name, "grid": list(case.N), "steps": case.Nt, "ms_per_step": ms / case.Nt,
           "value": value, "unit": UNIT,
           "spm": {"bytes_per_voxel_step": 4.0 * SPM_WORDS["c2"],
                   "frac": 4.0 * SPM_WORDS["c2"] * value / peak, "peak_kind": f"{kind} copy bandwidth"},
           "schedule": sched}
    path = os.path.join(GOLDEN, "c2_long.npz")
    if os.path.exists(path):
        gold = np.load(path)
        acc = {"reference": "FP64 oracle, all 2000 steps (tests/golden/c2_long.npz)"}
        for k in ("p_max", "p_rms"):
            l2, mx = rel_errors(out[k], gold[k])
            acc[k] = {"rel_l2": l2, "max_rel": mx}
        res["accuracy"] = acc
    return res


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_case(name, Nt=None):
    from kwave_b200 import workloads
    if name == "c3":
        return workloads.c3() if Nt is None else workloads.c3(Nt=Nt)
    if name == "c2":
        return workloads.c2() if Nt is None else workloads.c2(Nt=Nt)
    if name == "c1":
        return workloads.c1() if Nt is None else workloads.c1(Nt=Nt)
    raise ValueError(name)


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        try:
            self.file.seek(0)
            rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def barrier_max(pg, local, value):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{local}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, local):
    if pg is not None:
        barrier_max(pg, local, 0.0)


def cufft_comparator(case, steps=20, warmup=3):
    """A comparator timed beside the product, not part of it: the reference's time step written
    with library FFTs -- torch.fft (cuFFT), FP32, on the GPU.  Every spectral derivative is a full
    N-D real FFT pair, as the reference computes it (spectral_gradient!, fft_utils.jl:126-182):
    4D + 2 transforms per step (D gradients of p, D divergences of u, the equation of state), with
    the same PML, staggered densities, nonlinearity, k-space multiplier and velocity source."""
    import numpy as np
    import torch
    from kwave_b200.core import db2neper, get_pml
    from kwave_b200.solver import _findall
    dev = torch.device("cuda", torch.cuda.current_device())
    N = tuple(case.N)
    D = len(N)
    dt = case.dt
    f32 = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float32), device=dev)
    med = case.medium
    c0 = np.asarray(med["sound_speed"], dtype=np.float64)
    r0 = np.asarray(med["density"], dtype=np.float64)
    c0sq, rho0 = f32(c0 ** 2), f32(r0)
    Q = f32(np.asarray(med["BonA"], np.float64) / (2 * r0)) if med.get("BonA") is not None else None
    rho_sg = [0.5 * (rho0 + torch.roll(rho0, -1, dims=a)) for a in range(D)]

    def along(v, a):
        sh = [1] * D
        sh[a] = -1
        return v.reshape(sh)

    pml = [along(f32(get_pml(N[a], case.d[a], case.pml_size, case.pml_alpha, dt)), a) for a in range(D)]
    pml_sg = [along(f32(get_pml(N[a], case.d[a], case.pml_size, case.pml_alpha, dt, staggered=True)), a)
              for a in range(D)]
    # wavenumbers in torch.fft.rfftn's layout (the last axis halved)
    kv = [2 * np.pi * (np.fft.rfftfreq(N[a], case.d[a]) if a == D - 1 else np.fft.fftfreq(N[a], case.d[a]))
          for a in range(D)]
    op = lambda a, sgn: along(torch.as_tensor((1j * kv[a] * np.exp(sgn * 1j * kv[a] * case.d[a] / 2))
                                              .astype(np.complex64), device=dev), a)
    ops_pos = [op(a, 1) for a in range(D)]
    ops_neg = [op(a, -1) for a in range(D)]
    kk = np.sqrt(sum(g ** 2 for g in np.meshgrid(*kv, indexing="ij")))
    c_ref = float(np.mean(c0))
    y = float(med.get("alpha_power") or 1.0)
    tau = -2 * db2neper(float(med.get("alpha_coeff") or 0.0), y) * c_ref ** (y - 1)
    M = torch.as_tensor((np.sinc(c_ref * kk * dt / 2 / np.pi) * (1 + tau * kk ** y)).astype(np.float32), device=dev)
    p = torch.zeros(N, device=dev)
    u = [torch.zeros(N, device=dev) for _ in range(D)]
    rho = [torch.zeros(N, device=dev) for _ in range(D)]
    uidx = usig = None
    if "u_mask" in case.source and case.source.get("ux") is not None:
        lin = _findall(case.source["u_mask"], N)  # column-major order, the signal's row order
        co = np.unravel_index(lin, N, order="F")
        uidx = torch.as_tensor(np.ravel_multi_index(co, N), device=dev)  # the same points, C order
        usig = f32(case.source["ux"])

    def step(t):
        for a in range(D):
            g = torch.fft.irfftn(torch.fft.rfftn(p) * ops_pos[a], s=N)
            u[a] = pml_sg[a] * (pml_sg[a] * u[a] - dt / rho_sg[a] * g)
        if uidx is not None:
            u[0].view(-1)[uidx] += usig[:, min(t, usig.shape[1] - 1)]
        for a in range(D):
            g = torch.fft.irfftn(torch.fft.rfftn(u[a]) * ops_neg[a], s=N)
            rho[a] = pml[a] * (pml[a] * rho[a] - dt * rho0 * g)
        rt = sum(rho[1:], rho[0])
        if Q is not None:
            rt = rt * (1 + Q * rt)
        p.copy_(torch.fft.irfftn(torch.fft.rfftn(c0sq * rt) * M, s=N))

    for t in range(warmup):
        step(t)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for t in range(steps):
        step(warmup + t)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    out = {"what": "the reference's time step with torch.fft (cuFFT) full N-D real FFT pairs, FP32, "
                   f"{4 * D + 2} transforms per step, eager", "ms_per_step": ms,
           "value": float(np.prod(N)) / (ms / 1e3) / 1e9, "unit": UNIT, "steps": steps, "warmup": warmup,
           "finite": bool(torch.isfinite(p).all().item())}
    del p, u, rho, M, rho_sg, pml, pml_sg, ops_pos, ops_neg, c0sq, rho0, Q
    torch.cuda.empty_cache()
    return out


def cpu_baseline(case_name, budget_s=20.0):
    """The FP64 oracle (restatement of the reference algorithm) on the host cores, a bounded
    number of time steps of the same workload; returns voxel-steps/s and the sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _util import oracle_inputs
    import kwave_ref as K
    case = make_case(case_name)
    g, m, s, sen, opts = oracle_inputs(case)
    t0 = time.perf_counter()
    K.kspace_first_order(g, m, s, sen, max_steps=1, **opts)  # warm-up + set-up cost
    one = time.perf_counter() - t0
    steps = max(2, min(case.Nt, int(budget_s / max(one, 1e-3))))
    t0 = time.perf_counter()
    K.kspace_first_order(g, m, s, sen, max_steps=steps, **opts)
    el = time.perf_counter() - t0
    # subtract the per-solve set-up measured by the 1-step run's share (conservative: keep it)
    v = case.voxels * steps / el
    return v, steps, el, os.cpu_count()


def run_reference(args, world, rank):
    if rank != 0:
        return
    v, steps, el, cores = cpu_baseline(args.config, budget_s=min(60.0, 10.0 * max(1, args.steps) ** 0.5))
    val = v / 1e9
    line = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": 1, "ms_per_step": 1e3 * el / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": make_case(args.config, Nt=2).name, "sample": f"first {steps} time steps"},
            "impl": "reference",
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"FP64 NumPy/SciPy restatement of the reference, first {steps} "
                                       f"time steps of the workload, scipy.fft workers={cores}"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def elastic_bench(ctx, n=256, steps=200, warmup=5, cpu=True):
    """The elastic solver (pstd_elastic_3d) on the n^3 heterogeneous elastic workload: device-timed
    steps (CUDA events, CUDA-graph chunks), per-kernel shares and algorithmic bytes, and the FP64
    oracle on the host cores for a 2-step prefix of the same workload."""
    import kwave_b200 as kb
    from kwave_b200 import workloads
    case = workloads.elastic3d(n)
    g, m, s, sen, kw = case.to_api()
    sim = kb.Simulation(g, m, s, sen, context=ctx, **kw)
    sim.advance_timed(warmup)
    ms = sim.advance_timed(steps)
    sim.close()
    prof_sim = kb.Simulation(g, m, s, sen, context=ctx, **kw)
    prof_sim.advance(warmup)
    prof = prof_sim.profile(20)
    prof_sim.close()
    tot = sum(k["total_ms"] for k in prof)
    steps_prof = 20
    bytes_step = sum(k["bytes_per_launch"] * k["launches"] for k in prof) / steps_prof
    peak, peak_kind = peaks()
    ms_step = ms / steps
    out = {"workload": case.name, "grid": list(case.N), "steps": steps, "warmup": warmup,
           "ms_per_step": ms_step, "value": case.voxels / (ms_step / 1e3) / 1e9, "unit": UNIT,
           "bytes_per_voxel_step": bytes_step / case.voxels,
           "achieved_GBps": bytes_step / (ms_step / 1e3) / 1e9, "peak": peak,
           "frac": bytes_step / (ms_step / 1e3) / 1e9 / peak, "peak_kind": f"{peak_kind} copy bandwidth",
           "kernels": {k["name"]: {"avg_us": 1e3 * k["total_ms"] / k["launches"], "share": k["total_ms"] / tot,
                                   "launches_per_step": k["launches"] / steps_prof} for k in prof}}
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import kwave_ref as K
        args = []
        for nn, dd in zip(case.N, case.d):
            args += [nn, dd]
        og = K.KWaveGrid(*args)
        og.dt, og.Nt = case.dt, case.Nt
        t0 = time.perf_counter()
        K.pstd_elastic_3d(og, K.ElasticMedium(**case.medium), K.ElasticSource(**case.source),
                          K.KWaveSensor(**case.sensor), pml_size=case.pml_size, max_steps=2)
        el = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": case.voxels * 2 / el / 1e9, "unit": UNIT, "cores": os.cpu_count(),
                               "kind": "port", "sample": f"FP64 oracle, first 2 time steps incl. set-up ({el:.1f} s)"}
    return out


def batch_bench(ctx, n_sims=64, max_running=64, one_at_a_time=True):
    """Batch workload: n mixed-size 2D simulations, batched (continuous batching, all submitted at once)
    against one-at-a-time blocking solves of the same prepared problems.  Sims/s is measured
    from the first submission to the last completion (host wall clock, device work inside)."""
    import numpy as np
    import kwave_b200 as kb
    from kwave_b200 import workloads as W
    cases = [W.c4_sim(i) for i in range(n_sims)]
    vs = sum(c.voxels * c.Nt for c in cases)

    def prep_all():
        out = []
        for c in cases:
            g, m, s, sen, kw = c.to_api()
            out.append(kb.prepare(g, m, s, sen, context=ctx, **kw))
        return out

    kb.serving_config(max_running=max_running, chunk_steps=32, context=ctx)
    # untimed warm-up: the same 64 grids for 40 steps each through the scheduler and alone (the
    # scheduler's context, first launches and per-kernel attributes are set up outside the timing)
    warm = []
    for i in range(n_sims):
        c = W.c4_sim(i, nt_range=(40, 40))
        g, m, s, sen, kw = c.to_api()
        warm.append(kb.prepare(g, m, s, sen, context=ctx, **kw))
    for r in [kb.submit_prepared(p) for p in warm]:
        r.result()
    for p in warm[:8]:
        kb.solve_prepared(p)
    preps = prep_all()
    t0 = time.perf_counter()
    reqs = [kb.submit_prepared(p) for p in preps]
    outs = [r.result() for r in reqs]
    t_batch = time.perf_counter() - t0
    st = kb.serving_stats(context=ctx)
    res = {"workload": f"{n_sims} mixed-size 2D sims (sides 128-1024, Nt 500-4000, seeds 4004+i)",
           "voxel_steps": vs, "max_running": max_running, "batched_sims_per_s": n_sims / t_batch,
           "batched_Gvoxel_steps_per_s": vs / t_batch / 1e9, "peak_running": st["peak_running"]}
    if not one_at_a_time:
        return res
    preps1 = prep_all()
    t0 = time.perf_counter()
    alone = [kb.solve_prepared(p) for p in preps1]
    t_one = time.perf_counter() - t0
    res.update({"one_at_a_time_sims_per_s": n_sims / t_one, "speedup": t_one / t_batch,
                "results_identical_to_alone": all(np.array_equal(a["p"], b["p"]) for a, b in zip(alone, outs))})
    return res


def serving_bench(ctx, n_req=48, rate=200.0, seed=5005, nt_range=(300, 800), max_running=64, one_at_a_time=True):
    """Serving workload: Poisson arrivals (mean rate 200/s) of mixed 2D/3D requests; latency is arrival to
    completion.  The comparison serves the same arrivals one at a time with blocking solves."""
    import threading
    import numpy as np
    import kwave_b200 as kb
    from kwave_b200 import workloads as W
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
    cases = [W.c5_request(i, seed=seed, nt_range=nt_range) for i in range(n_req)]

    def prep_all():
        out = []
        for c in cases:
            g, m, s, sen, kw = c.to_api()
            out.append(kb.prepare(g, m, s, sen, context=ctx, **kw))
        return out

    preps = prep_all()
    kb.serving_config(max_running=max_running, chunk_steps=32, context=ctx)
    reqs = [None] * n_req
    t0 = time.perf_counter()

    def feeder():
        for i, p in enumerate(preps):
            dt = t0 + arrivals[i] - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            reqs[i] = (time.perf_counter(), kb.submit_prepared(p))

    th = threading.Thread(target=feeder)
    th.start()
    th.join()
    lat = []
    for i in range(n_req):
        ta, r = reqs[i]
        r.result()
        lat.append((r.info["end_ns"] - r.info["submit_ns"]) / 1e9)
    t_end = max(t0 + arrivals[i] + lat[i] for i in range(n_req))
    span = t_end - t0
    q = lambda a, x: float(np.percentile(np.asarray(a), x))
    accuracy = None
    gpath = os.path.join(GOLDEN, "serving_sample.npz")
    if os.path.exists(gpath) and (seed, nt_range, n_req) == (5005, (300, 800), 48):
        gold = np.load(gpath)
        accuracy = {"reference": "FP64 oracle (tests/golden/serving_sample.npz)"}
        for i in gold["requests"]:
            l2, mx = rel_errors(reqs[int(i)][1].result()["p"], gold[f"p_{int(i)}"])
            accuracy[cases[int(i)].name] = {"rel_l2": l2, "max_rel": mx}
    res = {"workload": f"{n_req} Poisson requests at {rate:.0f}/s, 70% 2D 256-1024 / 30% 3D 64^3-192^3, "
                       f"Nt {nt_range[0]}-{nt_range[1]}",
           "max_running": max_running,
           "sims_per_s": n_req / span, "p50_latency_s": q(lat, 50), "p99_latency_s": q(lat, 99),
           "accuracy_sampled": accuracy}
    if not one_at_a_time:
        return res
    preps1 = prep_all()
    t0 = time.perf_counter()
    lat1 = []
    for i, p in enumerate(preps1):
        dt = t0 + arrivals[i] - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        kb.solve_prepared(p)
        lat1.append(time.perf_counter() - (t0 + arrivals[i]))
    span1 = time.perf_counter() - t0
    res["one_at_a_time"] = {"sims_per_s": n_req / span1, "p50_latency_s": q(lat1, 50), "p99_latency_s": q(lat1, 99)}
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=["c3", "c2", "c1"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched mixed-size 2D measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the Poisson serving measurement")
    ap.add_argument("--no-cufft", action="store_true", help="skip the cuFFT-based comparator")
    ap.add_argument("--no-elastic", action="store_true", help="skip the elastic-solver measurement")
    ap.add_argument("--no-c2", action="store_true", help="skip the 512^2 x 2000-step solve")
    args = ap.parse_args()
    world, rank, local, pg = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import numpy as np
    import kwave_b200 as kb

    ctx = kb.Context(local)
    case = make_case(args.config)
    W = max(3, args.warmup)
    K = max(1, min(args.steps, case.Nt - W))
    g, m, s, sen, kw = case.to_api()
    sim = kb.Simulation(g, m, s, sen, extra_sensors=case.extra_sensors, context=ctx, **kw)
    info = sim.info()
    sim.advance_timed(W)
    barrier(pg, local)
    with Clocks(local) as clk:
        ms = sim.advance_timed(K)
    ms = barrier_max(pg, local, ms)
    sim.close()
    vox = case.voxels
    value = world * vox * K / (ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    spm_bytes = 4.0 * SPM_WORDS[args.config]
    spm_frac = spm_bytes * value * 1e9 / world / (peak * 1e9)

    # per-kernel device times (CUDA events around each launch on the simulation's stream)
    prof_sim = kb.Simulation(g, m, s, sen, extra_sensors=case.extra_sensors, context=ctx, **kw)
    prof_sim.advance(W)
    prof = prof_sim.profile(min(20, case.Nt - W))
    prof_sim.close()
    tot = sum(k["total_ms"] for k in prof)
    dom = max(prof, key=lambda k: k["total_ms"])
    dom_avg_s = dom["total_ms"] / dom["launches"] / 1e3
    achieved = dom["bytes_per_launch"] / dom_avg_s / 1e9
    kernels = {k["name"]: {"avg_us": 1e3 * k["total_ms"] / k["launches"], "share": k["total_ms"] / tot,
                           "GBps": (k["bytes_per_launch"] / (k["total_ms"] / k["launches"] / 1e3) / 1e9)
                           if k["bytes_per_launch"] else None} for k in prof}

    e2e = None
    if not args.no_e2e:
        t0 = time.perf_counter()
        sim2 = kb.Simulation(g, m, s, sen, extra_sensors=case.extra_sensors, context=ctx, **kw)
        out = sim2.finish()
        el = time.perf_counter() - t0
        sim2.close()
        h2d = sum(np.asarray(v).nbytes for v in (case.medium["sound_speed"], case.medium["density"],
                                                 case.medium.get("BonA")) if v is not None and np.ndim(v) > 0)
        for v in case.source.values():
            if isinstance(v, np.ndarray) and v.dtype != bool:
                h2d += v.astype(np.float64).nbytes
        d2h = sum(a.nbytes for a in out.data.values()) + sum(a.nbytes for e in out.extra for a in e.values())
        e2e = {"value": world * vox * case.Nt / el / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d / case.Nt), "d2h_bytes_per_step": int(d2h / case.Nt),
               "solve_s": el, "steps": case.Nt}
        accuracy = c3_accuracy(case, out) if args.config == "c3" else None
    else:
        accuracy = None

    c2 = None if (args.no_c2 or args.config == "c2") else c2_leg(ctx)
    batch = None if args.no_batch else batch_bench(ctx)
    serve = None if args.no_serve else serving_bench(ctx)

    elastic = None
    if not args.no_elastic:
        elastic = elastic_bench(ctx, cpu=(rank == 0 and world == 1 and not args.no_cpu))

    comparators = None
    if rank == 0 and world == 1 and not args.no_cufft:
        comparators = {"cufft_reference_step": cufft_comparator(case)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, steps, el, cores = cpu_baseline(args.config)
        cpu = {"value": v / 1e9, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"FP64 NumPy/SciPy restatement of the reference, first {steps} time steps of the "
                         f"same workload ({el:.1f} s), scipy.fft workers={cores}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": case.name, "grid": list(case.N), "Nt": case.Nt,
                       "l2": "inputs larger than L2 (7 FP32 state fields + medium, > 126 MB)",
                       "timing": "CUDA events on the simulation stream, CUDA-graph replay of 32-step chunks"},
            "roofline": {"bound": "hbm", "kernel": dom["name"], "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": NCU_TRAFFIC.get((args.config, dom["name"])),
                         "traffic_unit": "DRAM bytes read + written per launch (ncu)",
                         "algorithmic_bytes": dom["bytes_per_launch"],
                         "peak_kind": f"{peak_kind} copy bandwidth (burst)"},
            "spm": {"bytes_per_voxel_step": spm_bytes, "achieved_GBps": spm_bytes * value * 1e9 / world / 1e9,
                    "frac": spm_frac},
            "kernels": kernels,
            "e2e": e2e,
            "accuracy": accuracy,
            "c2": c2,
            "batch": batch,
            "serving": serve,
            "cpu_baseline": cpu,
            "comparators": comparators,
            "elastic": elastic,
            "clocks": clk.summary(),
            "gpu_launches": info["launches_per_step"] * K + (K // 32),
        }
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
