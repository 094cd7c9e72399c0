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


def test_delayed_acceptance_through_the_shard(gpu_ctx):
    """Delayed acceptance with the shard as the exact likelihood: the
    survivor batches of stage one go through the shard like any batch, and
    the surrogate (its pairs appended in row order, seeded training) is the
    same network either way, so the chain equals the one through the inner
    likelihood draw for draw -- what keeps the ranks of a sharded ensemble
    in step under delayed acceptance."""
    from pofd_affine_b200 import synth
    from pofd_affine_b200.mcmc import affineEnsemble
    from pofd_affine_b200.shard import shardedLike, unique_id
    from pofd_affine_b200.surrogate import Surrogate
    cfg = synth.config_1d_small(seed=1)
    L = synth.build_like1(cfg, gpu_ctx, ninterp=512)
    S = shardedLike(gpu_ctx, L, rank=0, world=1, nccl_id=unique_id())
    npar = cfg["theta0"].size

    def run(like):
        E = affineEnsemble(gpu_ctx, like, 20, npar, seed=8)
        E.setParamFixed(npar - 1)
        E.initChains(E.generateInitialPosition(cfg["theta0"], 0.03, rng=9))
        E.prepareDA()
        sur = Surrogate(gpu_ctx, npar, list(range(npar - 1)), hidden=256, seed=4)
        E.collectPairs(sur)
        E.doSteps(0, 30)
        sur.train(150, 256, 1e-3)
        E.setSurrogate(sur)
        E.setDAScale(4.0)
        E.doStepsDA(12)
        E.collectPairs(None)
        st = E.daStats()
        ch, cl = E.getChain()
        return ch, cl, st
    c1, l1, s1 = run(L)
    c2, l2, s2 = run(S)
    assert s1 == s2
    assert 0 < s1["stage1_passes"] < s1["proposals"]
    assert np.array_equal(c1, c2)
    assert np.array_equal(l1, l2)
