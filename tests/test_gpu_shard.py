"""The device form of the walker-sharded likelihood on one GPU (a
one-rank NCCL communicator): evaluating through the shard -- this rank's
rows, the pack, the all-gather and the unpack -- gives the inner
likelihood's values bit for bit, and an ensemble run with the shard as its
likelihood (its steps captured into a CUDA graph with the collective inside)
is the run with the inner likelihood, draw for draw."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_one_rank_shard_is_the_inner_likelihood(gpu_ctx):
    from pofd_affine_b200 import synth
    from pofd_affine_b200.mcmc import affineEnsemble
    from pofd_affine_b200.shard import shardedLike, unique_id
    cfg = synth.config_1d_small(seed=1)
    L = synth.build_like1(cfg, gpu_ctx, ninterp=512)
    S = shardedLike(gpu_ctx, L, rank=0, world=1, nccl_id=unique_id())
    npar = cfg["theta0"].size
    th = synth.proposals(cfg["theta0"], 20, 0.02, rng=4)
    ref, st = L.getLogLikeBatch(th)

    def run(like):
        E = affineEnsemble(gpu_ctx, like, 20, npar, seed=5)
        E.setParamFixed(npar - 1)
        E.initChains(E.generateInitialPosition(cfg["theta0"], 0.03, rng=6))
        E.doSteps(12)
        return E.getChain()

    c1, l1 = run(L)
    c2, l2 = run(S)
    assert np.array_equal(c1, c2)
    assert np.array_equal(l1, l2)
    # a batch through the shard directly
    import ctypes as C
    import torch
    from pofd_affine_b200._lib import lib
    d_th = torch.from_numpy(th).cuda()
    d_ll = torch.empty(20, dtype=torch.float64, device="cuda")
    d_st = torch.empty(20, dtype=torch.int32, device="cuda")
    rc = lib().pofd_shard_eval_batch_device(S.h, 20, C.c_void_p(d_th.data_ptr()), npar,
                                            C.c_void_p(d_ll.data_ptr()),
                                            C.c_void_p(d_st.data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert np.array_equal(d_ll.cpu().numpy(), ref)
    assert np.array_equal(d_st.cpu().numpy(), st)
