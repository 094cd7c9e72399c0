"""The multi-GPU bookkeeping of bench.py (pofd_affine_b200.ranks) on two
gloo ranks on the CPU: the process group comes up from the torchrun
environment, the timed duration is the maximum over ranks, the proposal
batches of different ranks are disjoint, and the weak-scaled throughput
counts every rank's units over the slowest rank's time."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from pofd_affine_b200.ranks import Ranks
    from pofd_affine_b200 import synth
    rk = Ranks("gloo", timeout_s=60)
    rk.barrier()
    dur = 1.0 + rank  # rank 1 is the slow one
    mx = rk.max_over_ranks(dur)
    tot = rk.sum_over_ranks(rank + 1)
    th = synth.proposals(np.zeros(4, np.float32), 3, 1.0, rng=rk.proposal_seed(0))
    rate = rk.throughput(64, mx)
    out.put((rank, rk.world, mx, tot, th, rate))
    rk.close()


@pytest.mark.timeout(120)
def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, mx0, tot0, th0, rate0), (r1, w1, mx1, tot1, th1, rate1) = res
    assert (r0, r1) == (0, 1) and w0 == w1 == 2
    assert mx0 == mx1 == 2.0
    assert tot0 == tot1 == 3.0
    assert not np.array_equal(th0, th1)
    assert rate0 == rate1 == 2 * 64 / 2.0


def test_single_process_needs_no_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from pofd_affine_b200.ranks import Ranks
    rk = Ranks("gloo")
    assert rk.world == 1 and rk.dist is None
    assert rk.max_over_ranks(3.5) == 3.5
    assert rk.throughput(10, 2.0) == 5.0
    rk.close()
