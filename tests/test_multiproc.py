"""Multi-GPU sharding of independent simulations, exercised on CPU with gloo (world size 2).

Batched simulations are independent units: each rank runs the share ``run_sharded`` /
``shard_jobs`` gives it and ranks exchange nothing while they run; results come together only on
the host at the end.  Without a GPU the library call is replaced by a runner that reads back the
real kwb_problem structs each rank built for its share (grid, time steps, the medium array
through its C pointer), so the sharding of real problems, the no-collective run and the final
gather are tested end to end except for the device work."""
import ctypes as C
import os
import socket

import numpy as np
import torch.multiprocessing as mp

N_JOBS = 5


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _jobs():
    import kwave_b200 as kb
    out = []
    for i, n in enumerate((24, 32, 40, 28, 36)):
        g = kb.KWaveGrid(n, 1e-4, n, 1e-4)
        g.dt, g.Nt = 2e-8, 20 + 5 * i
        c = np.full((n, n), 1500.0 + i)
        p0 = np.zeros((n, n))
        p0[n // 2, n // 2] = 1.0
        mask = np.zeros((n, n), bool)
        mask[n // 3, n // 2] = True
        out.append((g, kb.KWaveMedium(sound_speed=c, density=1000.0), kb.KWaveSource(p0=p0),
                    kb.KWaveSensor(mask=mask, record=["p"]), {"smooth_p0": False}))
    return out


def _readback(device, built):
    """Stand-in for the device: what each built kwb_problem carries."""
    out = []
    for b in built:
        P = b.problem
        n = int(P.N[0] * P.N[1])
        c0 = np.ctypeslib.as_array(C.cast(P.c0.data, C.POINTER(C.c_double)), shape=(n,))
        out.append({"device": device, "N": (int(P.N[0]), int(P.N[1])), "Nt": int(P.Nt), "c0_mean": float(c0.mean()),
                    "groups": int(P.n_groups)})
    return out


def _expected(i, job):
    g = job[0]
    return {"N": tuple(g.N), "Nt": g.Nt, "c0_mean": 1500.0 + i, "groups": 1}


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "k-wave-julia_b200")]
    import torch.distributed as dist
    from kwave_b200 import run_sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    results = run_sharded(_jobs(), runner=_readback)  # world and rank from the process group
    gathered = [None] * world
    dist.all_gather_object(gathered, {"rank": rank, "results": results})
    if rank == 0:
        q.put(gathered)
    dist.destroy_process_group()


def test_two_ranks_shard_a_batch_with_no_overlap():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    owned = [set(g["results"]) for g in gathered]
    assert owned[0].isdisjoint(owned[1]) and owned[0] | owned[1] == set(range(N_JOBS))
    assert owned[0] and owned[1]
    jobs = _jobs()
    for g in gathered:
        for i, r in g["results"].items():
            assert r["device"] == g["rank"]  # each rank on its own LOCAL_RANK device
            assert {k: r[k] for k in ("N", "Nt", "c0_mean", "groups")} == _expected(i, jobs[i])
    # the split balances voxels x steps: longest first onto the least-loaded rank
    from kwave_b200 import shard_jobs
    costs = [j[0].N[0] * j[0].N[1] * j[0].Nt for j in jobs]
    assert [sorted(o) for o in owned] == [shard_jobs(costs, 2, 0), shard_jobs(costs, 2, 1)]


def test_one_process_several_devices():
    """devices=[0, 1, 2]: every share runs in this process, one thread per device."""
    from kwave_b200 import run_sharded
    jobs = _jobs()
    res = run_sharded(jobs, devices=[0, 1, 2], runner=_readback)
    assert sorted(res) == list(range(N_JOBS))
    assert {r["device"] for r in res.values()} == {0, 1, 2}
    for i, r in res.items():
        assert {k: r[k] for k in ("N", "Nt", "c0_mean", "groups")} == _expected(i, jobs[i])
