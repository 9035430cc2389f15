"""Host logic of batched ensembles (no GPU): the per-foam law, load balancing
of foams over ranks, and the multi-rank split exercised with gloo ranks on
the CPU (each rank owns whole foams; the only collectives gather per-foam
results, as a multi-GPU ensemble run does with NCCL)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fos import inputs
from fos.ensemble import frame_cost, partition


def test_member_law():
    f = inputs.ensemble_member(5000, 7, 11)
    med = 0.03 * (1000.0 / 5000) ** (1.0 / 3.0)
    assert f.n == 5000 and f.res == 96 and (f.f_low, f.f_high) == (11, 15)
    assert np.all(f.rad >= np.float32(0.4 * med)) and np.all(f.rad <= np.float32(2 * med))
    assert abs(np.median(f.rad) - med) / med < 0.05
    assert (f.pbd_iters, f.pressure_iters, f.jfa_warm, f.jfa_cadence) == (8, 20, 20, 5)
    assert inputs.ensemble_member(100, 7).res == 64 and inputs.ensemble_member(20000, 7).res == 128


def test_partition_covers_and_balances():
    foams = inputs.ensemble()
    for world in (1, 2, 3, 4, 8):
        parts = partition(foams, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(foams)))
        loads = [sum(frame_cost(foams[k]) for k in p) for p in parts]
        opt = max(sum(frame_cost(f) for f in foams) / world,
                  max(frame_cost(f) for f in foams))
        assert max(loads) <= 4.0 / 3.0 * opt + 1e-6
        assert all(p == sorted(p) for p in parts)


def test_partition_is_deterministic_and_validates():
    foams = inputs.ensemble(count=10)
    assert partition(foams, 3) == partition(foams, 3)
    with pytest.raises(ValueError):
        partition(foams, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    foams = inputs.ensemble(count=12, n_range=(200, 2000))
    mine = partition(foams, world)[rank]
    # each rank "runs" its foams: here the per-foam result is the particle count
    # and the mean radius, gathered to every rank as a multi-GPU run gathers stats
    local = {k: (foams[k].n, float(np.mean(foams[k].rad))) for k in mine}
    gathered = [None] * world
    dist.all_gather_object(gathered, local)
    if rank == 0:
        merged = {}
        for d in gathered:
            assert not set(d) & set(merged)
            merged.update(d)
        q.put(sorted(merged.items()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_split_foams_without_overlap():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    foams = inputs.ensemble(count=12, n_range=(200, 2000))
    assert [k for k, _ in got] == list(range(12))
    assert [v[0] for _, v in got] == [f.n for f in foams]
