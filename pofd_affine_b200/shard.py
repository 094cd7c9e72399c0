"""The batched likelihood split over the GPUs of one node (one process per
GPU, torch.distributed for the process group), the counterpart of the
reference's MPI master/worker farm (affineEnsemble.cc:1233-1521).

Every rank runs the same ensemble (same seed): its likelihood is a
shardedLike, which evaluates this rank's rows of each batch with the rank's
own replica of the likelihood and all-gathers every row's (logL, status)
over NCCL on the ensemble's stream, so the chains are identical on every
rank and to a single-GPU run's.

  * shard_rows(nprop, world, rank)   this rank's rows [lo, hi) of a batch
  * shardedLike(ctx, like, group)     the device form (pofd_shard_*), usable
                                      wherever a batched likelihood is
  * gather_rows_host(...)             the same layout on host arrays with
                                      torch.distributed (any backend), for
                                      host-side batch evaluation across ranks
"""
import ctypes as C

import numpy as np

from ._lib import check, lib


def shard_rows(nprop, world, rank):
    """Rows [lo, hi) of a batch of nprop proposals that rank evaluates:
    lo = nprop rank / world, hi = nprop (rank + 1) / world (integer
    division), so the ranks' row counts differ by at most one."""
    lo, hi = C.c_uint(), C.c_uint()
    check(lib().pofd_shard_rows(int(nprop), int(world), int(rank),
                                C.byref(lo), C.byref(hi)))
    return lo.value, hi.value


def gather_rows_host(logl_rows, status_rows, nprop, group=None):
    """All ranks' rows of a batch from each rank's own rows (this rank's
    shard_rows slice of logL and status), in batch order, on every rank.
    Packs [logL padded to ceil(nprop / world) | status] per rank and does
    one all-gather, the layout the device form uses."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    cap = -(-int(nprop) // world)
    lo, hi = shard_rows(nprop, world, rank)
    if len(logl_rows) != hi - lo or len(status_rows) != hi - lo:
        raise ValueError("rows do not match this rank's share of the batch")
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    send = torch.full((2 * cap,), float("nan"), dtype=torch.float64, device=dev)
    send[:hi - lo] = torch.as_tensor(np.asarray(logl_rows, np.float64))
    send[cap:cap + hi - lo] = torch.as_tensor(np.asarray(status_rows, np.float64))
    recv = torch.empty(world * 2 * cap, dtype=torch.float64, device=dev)
    dist.all_gather_into_tensor(recv, send, group=group)
    recv = recv.cpu().numpy().reshape(world, 2, cap)
    logl = np.empty(nprop)
    status = np.empty(nprop, np.int32)
    for r in range(world):
        a, b = shard_rows(nprop, world, r)
        logl[a:b] = recv[r, 0, :b - a]
        status[a:b] = recv[r, 1, :b - a].astype(np.int32)
    return logl, status


def batch_function(like):
    """(function pointer, handle) of a batched likelihood object of this
    package, with the pofd_batch_loglike_fn signature."""
    from ._lib import support_lib
    from .api1d import calcLike
    from .api2d import calcLikeDouble
    from .mcmc import gaussLike, likeSum
    if isinstance(like, calcLike):
        return C.cast(lib().pofd_like1_eval_batch_device, C.c_void_p), like.h
    if isinstance(like, calcLikeDouble):
        return C.cast(lib().pofd_like2_eval_batch_device, C.c_void_p), like.h
    if isinstance(like, gaussLike):
        return C.cast(support_lib().pofd_gauss_eval_batch_device, C.c_void_p), like.h
    if isinstance(like, likeSum):
        return C.cast(lib().pofd_likesum_eval_batch_device, C.c_void_p), like.h
    if isinstance(like, shardedLike):
        return C.cast(lib().pofd_shard_eval_batch_device, C.c_void_p), like.h
    raise TypeError("unsupported likelihood object")


def unique_id():
    """A new NCCL unique id (128 bytes) for shardedLike."""
    buf = C.create_string_buffer(128)
    check(lib().pofd_nccl_unique_id(buf))
    return buf.raw


class shardedLike:
    """like (this rank's replica) split over the ranks of a torch.distributed
    process group, or, without one, over world ranks given explicitly with a
    shared NCCL unique id (nccl_id from unique_id() on one rank)."""

    def __init__(self, ctx, like, group=None, rank=None, world=None,
                 nccl_id=None):
        if rank is None or world is None or nccl_id is None:
            import torch
            import torch.distributed as dist
            rank, world = dist.get_rank(group), dist.get_world_size(group)
            dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
            t = torch.zeros(128, dtype=torch.uint8, device=dev)
            if rank == 0:
                t[:] = torch.frombuffer(bytearray(unique_id()), dtype=torch.uint8)
            dist.broadcast(t, 0, group=group)
            nccl_id = bytes(t.cpu().numpy().tobytes())
        fn, h = batch_function(like)
        out = C.c_void_p()
        check(lib().pofd_shard_create(ctx.h, nccl_id, int(rank), int(world),
                                      fn, h, C.byref(out)))
        self.h, self.ctx, self.like = out, ctx, like
        self.rank, self.world = int(rank), int(world)

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().pofd_shard_destroy(self.h)
            except Exception:  # interpreter shutdown: the library is gone
                pass
            self.h = None
