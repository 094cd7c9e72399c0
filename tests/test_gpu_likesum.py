"""Summed likelihood of fields with different FFT sizes (one launch,
members on forked streams) and the ensemble running on it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_likesum_equals_member_sum(orc, gpu_ctx):
    import torch
    from pofd_affine_b200 import calcLikeDouble, doublebeam, synth
    from pofd_affine_b200._lib import lib
    from pofd_affine_b200.mcmc import affineEnsemble, likeSum
    cfg = synth.config_2d(scale=0.1, n=256, nbins=100)
    rng = np.random.default_rng(4)
    m1, m2 = synth.make_map_pair((60, 50), 6.0, cfg["beam1"], cfg["beam2"],
                                 cfg["knotpos"], cfg["knotvals"],
                                 lambda f: 0.2 + 0 * f, lambda f: -0.35 + 0 * f,
                                 0.0025, 0.0028, rng)
    likes = []
    for n, (a, b) in ((256, cfg["maps"][0]), (128, (m1, m2))):
        L = calcLikeDouble(gpu_ctx, cfg["knotpos"], cfg["sigmapos"],
                           cfg["offsetpos"], n, 64, True, 100)
        L.addBeamSet(doublebeam(cfg["beam1"], cfg["beam2"], 6.0, True, 100, 1e-6))
        L.addDataset(0, a, b, 0.0025, 0.0028)
        L.setRRanges(cfg["theta0"])
        likes.append(L)
    S = likeSum(gpu_ctx, likes)
    th = synth.proposals(cfg["theta0"], 8, 0.02, rng=1, fixed_last=False)
    th[:, -2:] = 1.0
    parts = [L.getLogLikeBatch(th)[0] for L in likes]
    dth = torch.from_numpy(th).cuda()
    dll = torch.empty(8, dtype=torch.float64, device="cuda")
    dst = torch.empty(8, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    for _ in range(2):
        assert lib().pofd_likesum_eval_batch_device(
            S.h, 8, dth.data_ptr(), th.shape[1], dll.data_ptr(), dst.data_ptr(),
            None) == 0
        lib().pofd_ctx_synchronize(gpu_ctx.h)
        assert np.all(dst.cpu().numpy() == 0)
        assert np.array_equal(dll.cpu().numpy(), parts[0] + parts[1])
    # the ensemble on the sum: recorded logL equal the members' sum
    nw, npar = 10, th.shape[1]
    E = affineEnsemble(gpu_ctx, S, nw, npar, seed=3)
    E.setParamFixed(npar - 1)
    E.setParamFixed(npar - 2)
    E.initChains(E.generateInitialPosition(cfg["theta0"], 0.01, rng=2))
    E.doSteps(6)
    ch, cl = E.getChain()
    last = ch[-1]
    ref = sum(L.getLogLikeBatch(last)[0] for L in likes)
    assert np.array_equal(cl[-1], ref)
