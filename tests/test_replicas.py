"""Multi-GPU is replicas only: N ranks run N independent instances, with no
collective on the data path. The host side of that (max-over-ranks timing,
whole-job throughput, identical results of identical replicas) runs here as
two gloo ranks on the CPU, with the oracle standing in for each rank's model."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    from fastearth3d_b200 import synth
    from oracle import orc

    # each replica: the same small coupled workload, two steps
    w = synth.Workload("replica", 8, 8, 100.0, 2, 2, "sawtooth", sle=True, visc3d=False, seed=3)
    o = orc.Oracle(w.params(orc.default_params))
    zb, hi = w.reference()
    o.set_reference(zb, hi)
    for s in range(1, 3):
        o.update(w.ice_at(s * 300), w.dt_yr)
    rsl = o.fields()[0]
    local_ms = 10.0 + 5.0 * rank  # stand-in device times of the timed region
    mx = bench.max_over_ranks(local_ms, dist, "cpu")
    gathered = [None] * world
    dist.all_gather_object(gathered, rsl.tolist())
    out[rank] = (mx, bench.replica_throughput(world, 4, mx), gathered)
    dist.destroy_process_group()


def test_replicas_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    for r in range(2):
        mx, thr, gathered = out[r]
        assert mx == 15.0  # the slower rank bounds the job
        assert thr == pytest.approx(2 * 4 / 15e-3)
        # identical inputs give identical replicas (no cross-rank coupling)
        assert np.array_equal(np.array(gathered[0]), np.array(gathered[1]))
