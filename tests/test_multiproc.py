"""Multi-GPU sharding of independent simulations, exercised on CPU with gloo (world size 2).

Batched simulations are independent units: each rank runs the subset shard_jobs gives it and
ranks exchange nothing while they run; results come together only on the host at the end.
Here each "simulation" is a small oracle solve (CPU), so the sharding, the no-collective run and
the final gather are tested without a GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _jobs():
    import kwave_ref as K
    out = []
    for i, n in enumerate((24, 32, 40, 28, 36)):
        g = K.KWaveGrid(n, 1e-4, n, 1e-4)
        g.dt, g.Nt = 2e-8, 20 + 5 * i
        p0 = np.zeros((n, n))
        p0[n // 2, n // 2] = 1.0
        mask = np.zeros((n, n), bool)
        mask[n // 3, n // 2] = True
        out.append((g, K.KWaveMedium(sound_speed=1500.0, density=1000.0), K.KWaveSource(p0=p0),
                    K.KWaveSensor(mask=mask, record=["p"])))
    return out


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "k-wave-julia_b200"), os.path.join(root, "oracle")]
    import torch.distributed as dist
    import kwave_ref as K
    from kwave_b200.solver import shard_jobs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    jobs = _jobs()
    costs = [g.N[0] * g.N[1] * g.Nt for g, *_ in jobs]
    mine = shard_jobs(costs, world, rank)
    results = {i: K.kspace_first_order(*jobs[i], smooth_p0=False)["p"] for i in mine}
    gathered = [None] * world
    dist.all_gather_object(gathered, {"rank": rank, "mine": mine, "results": results})
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
    owned = [set(g["mine"]) for g in gathered]
    assert owned[0].isdisjoint(owned[1]) and owned[0] | owned[1] == set(range(5))
    assert owned[0] and owned[1]
    import kwave_ref as K
    jobs = _jobs()
    for g in gathered:
        for i, p in g["results"].items():
            assert np.array_equal(p, K.kspace_first_order(*jobs[i], smooth_p0=False)["p"])
