"""The walker-sharded likelihood's host logic on the CPU, no GPU: the row
partition of a batch over ranks, and, on two gloo ranks, an ensemble whose
likelihood is evaluated in shards (each rank its own rows, then one
all-gather in the layout the device form uses) gives the single-process
chain draw for draw.  The stretch move in this test is the oracle's CPU
restatement (the product ensemble runs on the GPU); what is under test is
the partition and the gather."""
import os
import socket

import numpy as np
import pytest


def test_row_partition_covers_every_batch_once(built_lib):
    from pofd_affine_b200.shard import shard_rows
    for nprop in list(range(0, 40)) + [63, 64, 65, 1000, 4097]:
        for world in range(1, 9):
            spans = [shard_rows(nprop, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nprop
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


K = 4
MEAN = np.array([0.3, -1.0, 2.0, 0.5])
ICOV = np.diag([1.0, 4.0, 0.25, 2.0])


def _gauss(th):
    d = th.astype(np.float64) - MEAN
    return -0.5 * np.einsum("ij,jk,ik->i", d, ICOV, d)


def _start(nw):
    rng = np.random.default_rng(3)
    th = (MEAN + rng.normal(0, 0.5, (nw, K))).astype(np.float32)
    return th, _gauss(th)


def _worker(rank, world, port, nw, nsteps, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import sampler_oracle as so
    from pofd_affine_b200.shard import gather_rows_host, shard_rows
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))

    def sharded(thetas):
        lo, hi = shard_rows(len(thetas), world, rank)
        mine = _gauss(thetas[lo:hi])
        return gather_rows_host(mine, np.zeros(hi - lo, np.int32), len(thetas))

    th, ll = _start(nw)
    ch, cl, nacc = so.stretch_run(th, ll, sharded, nsteps, seed=17)
    out.put((rank, ch, cl, nacc))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("nw", [16, 13])
def test_sharded_chain_equals_single_process_chain(built_lib, nw):
    import sys
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(
        os.path.abspath(__file__))), "oracle"))
    import sampler_oracle as so
    nsteps = 40
    th, ll = _start(nw)
    ref = so.stretch_run(th, ll, lambda t: (_gauss(t), np.zeros(len(t), np.int32)),
                         nsteps, seed=17)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, nw, nsteps, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        r, ch, cl, nacc = q.get(timeout=240)
        res[r] = (ch, cl, nacc)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for r in (0, 1):
        ch, cl, nacc = res[r]
        assert np.array_equal(ch, ref[0])
        assert np.array_equal(cl, ref[1])
        assert np.array_equal(nacc, ref[2])
