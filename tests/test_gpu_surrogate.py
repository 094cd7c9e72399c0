"""The tensor-core surrogate: the tcgen05 GEMM against float64 products of
the same bf16 operands, the network's forward pass and loss gradients
against the CPU oracle, training on a known log-density, and the
delayed-acceptance stretch move (exact posterior, fewer exact evaluations
per accepted move than the plain method)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf16_round(a):
    import mlp_oracle
    return mlp_oracle.bf16(a)


@pytest.mark.parametrize("M,N,K", [(128, 16, 16), (128, 256, 64),
                                   (300, 192, 80), (256, 384, 256),
                                   (77, 512, 32), (1024, 256, 1024)])
def test_bf16_gemm_matches_float64(gpu_ctx, M, N, K):
    import torch
    from pofd_affine_b200.surrogate import bf16_gemm
    rng = np.random.default_rng(M + N + K)
    a = rng.normal(size=(M, K)).astype(np.float32)
    b = rng.normal(size=(N, K)).astype(np.float32)
    A = torch.from_numpy(a).cuda().to(torch.bfloat16).contiguous()
    B = torch.from_numpy(b).cuda().to(torch.bfloat16).contiguous()
    Cg = bf16_gemm(A, B).cpu().numpy().astype(np.float64)
    ref = _bf16_round(a) @ _bf16_round(b).T
    err = np.max(np.abs(Cg - ref)) / np.max(np.abs(ref))
    assert err < 1e-5, err


def test_bounded_wait_times_out_with_a_status(gpu_ctx):
    """The tensor-core kernels' mbarrier wait is bounded: on a barrier that
    nothing arrives on it runs out and the kernel reports that as a status
    the host reads (no trap, no fault); with one arrival it completes.  The
    context stays usable afterwards: a tcgen05 GEMM still matches."""
    import ctypes as C
    import torch
    from pofd_affine_b200._lib import support_lib
    from pofd_affine_b200.surrogate import bf16_gemm
    out = C.c_int(-1)
    for limit in (1, 64, 4096):
        assert support_lib().pofd_wait_check(0, limit, 0, C.byref(out)) == 0
        assert out.value == 1, limit
        assert support_lib().pofd_wait_check(0, limit, 1, C.byref(out)) == 0
        assert out.value == 0, limit
    assert support_lib().pofd_wait_check(0, 0, 0, C.byref(out)) != 0
    assert support_lib().pofd_wait_check(0, (1 << 20) + 1, 0, C.byref(out)) != 0
    torch.cuda.synchronize()
    rng = np.random.default_rng(5)
    a = rng.normal(size=(128, 64)).astype(np.float32)
    b = rng.normal(size=(64, 64)).astype(np.float32)
    A = torch.from_numpy(a).cuda().to(torch.bfloat16).contiguous()
    B = torch.from_numpy(b).cuda().to(torch.bfloat16).contiguous()
    ref = _bf16_round(a) @ _bf16_round(b).T
    err = np.max(np.abs(bf16_gemm(A, B).cpu().numpy() - ref)) / np.max(np.abs(ref))
    assert err < 1e-5, err


def _gauss_pairs(n, k, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(k, k))
    cov = A @ A.T + k * np.eye(k)
    mu = rng.normal(size=k)
    th = (mu + rng.multivariate_normal(np.zeros(k), 2.0 * cov, size=n)).astype(np.float32)
    d = th.astype(np.float64) - mu
    ll = -0.5 * np.einsum("ij,jk,ik->i", d, np.linalg.inv(cov), d)
    return th, ll, mu, cov


def test_forward_and_gradients_match_oracle(gpu_ctx):
    import mlp_oracle
    from pofd_affine_b200.surrogate import Surrogate
    k, H, n = 5, 128, 384
    th, ll, _, _ = _gauss_pairs(n, k, 1)
    npar = k + 1
    thp = np.concatenate([th, np.ones((n, 1), np.float32)], 1)
    S = Surrogate(gpu_ctx, npar, list(range(k)), hidden=H, capacity=4096, seed=3)
    S.addPairs(thp, ll)
    assert S.nPairs() == n
    g, loss = S.gradients(n)  # also fixes the scaling from the pairs
    sc = S.scaling()
    params = [p.astype(np.float64) for p in S.getParams()]
    assert sc["whitened"]
    # the transform whitens the inputs it was fixed on
    x = mlp_oracle.standardise(thp, list(range(k)), sc["mu"], sc["W"])
    cx = np.cov(x[:, :k].astype(np.float64).T)
    assert np.max(np.abs(cx - np.eye(k))) < 0.02
    t = (np.maximum(ll - sc["ymax"], -sc["clip"]) / sc["ys"]).astype(np.float32).astype(np.float64)
    og, oloss = mlp_oracle.gradients(params, H, x, t)
    assert abs(loss - oloss) <= 1e-3 * oloss
    for name, a, b in zip(["W1", "b1", "W2", "b2", "W3", "b3", "w4", "b4"], g, og):
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 2e-2, (name, rel)
    # forward: predictions in logL units
    y, _ = mlp_oracle.forward(params, H, x)
    pred = S.predict(thp)
    assert np.max(np.abs(pred - (sc["ymax"] + sc["ys"] * y))) < 2e-3 * sc["ys"]


def test_training_fits_a_log_density(gpu_ctx):
    from pofd_affine_b200.surrogate import Surrogate
    k = 6
    th, ll, _, _ = _gauss_pairs(12000, k, 2)
    thp = np.concatenate([th, np.ones((len(th), 1), np.float32)], 1)
    S = Surrogate(gpu_ctx, k + 1, list(range(k)), hidden=256, seed=5)
    S.addPairs(thp[:10000], ll[:10000])
    before = S.rms(thp[10000:], ll[10000:])
    S.train(1500, batch=512, lr=1e-3)
    after = S.rms(thp[10000:], ll[10000:])
    assert after < 0.1 * before, (before, after)
    assert after < 0.05 * np.std(ll), (after, np.std(ll))


def test_pair_ring_order_and_training_are_deterministic(gpu_ctx):
    """Pairs enter the ring in row order, invalid rows (bad status,
    non-finite logL) skipped, wrapping at the capacity; two surrogates fed
    the same pairs and trained with the same seed predict bit-identically
    (what lets every rank of a sharded ensemble train the same network)."""
    from pofd_affine_b200.surrogate import Surrogate
    k = 6
    th, ll, _, _ = _gauss_pairs(3000, k, 3)
    thp = np.concatenate([th, np.ones((len(th), 1), np.float32)], 1)
    st = np.zeros(len(th), np.int32)
    st[::7] = -1
    ll = ll.copy()
    ll[5::11] = np.inf
    ok = (st == 0) & np.isfinite(ll)
    nets = []
    for _ in range(2):
        S = Surrogate(gpu_ctx, k + 1, list(range(k)), hidden=256, seed=3,
                      capacity=2048)
        for a in range(0, len(th), 1100):  # batches larger than one block
            S.addPairs(thp[a:a + 1100], ll[a:a + 1100], st[a:a + 1100])
        nets.append(S)
    S = nets[0]
    assert S.nPairs() == 2048
    g_th, g_ll = S.getPairs()
    v_th, v_ll = thp[ok], ll[ok]
    nv = len(v_ll)
    slot = np.arange(nv) % 2048
    exp_th = np.empty((2048, k + 1), np.float32)
    exp_ll = np.empty(2048)
    exp_th[slot], exp_ll[slot] = v_th, v_ll  # later rows overwrite
    assert np.array_equal(g_th, exp_th) and np.array_equal(g_ll, exp_ll)
    for S in nets:
        S.train(200, batch=512, lr=1e-3)
    p0, p1 = nets[0].predict(thp[:256]), nets[1].predict(thp[:256])
    assert np.array_equal(p0, p1)


def test_delayed_acceptance_exact_posterior_and_gain(gpu_ctx):
    """DA keeps the exact posterior (means within 0.1 sigma of the plain
    run and of the truth) and accepts far more of its exact evaluations."""
    from pofd_affine_b200.mcmc import affineEnsemble, gaussLike
    from pofd_affine_b200.surrogate import Surrogate
    k, nw = 6, 64
    _, _, mu, cov = _gauss_pairs(10, k, 7)
    G = gaussLike(gpu_ctx, mu, cov)
    sd = np.sqrt(np.diag(cov))

    def run(da):
        E = affineEnsemble(gpu_ctx, G, nw, k, seed=11 + da)
        E.initChains(E.generateInitialPosition(mu, sd, rng=3))
        S = None
        if da:
            S = Surrogate(gpu_ctx, k, list(range(k)), hidden=256, seed=2)
            E.collectPairs(S)
        E.doSteps(0, initsteps=300)  # burn-in, exact pairs collected
        if da:
            S.train(2000, batch=512, lr=1e-3)
            E.collectPairs(None)
            E.setSurrogate(S)
            base = E.daStats()
            E.doStepsDA(3000)
            st = E.daStats()
            st = {key: st[key] - base[key] for key in st}
        else:
            base = E.daStats()
            E.doSteps(3000)
            st = E.daStats()
            st = {key: st[key] - base[key] for key in st}
        ch, _ = E.getChain()
        tau, ok = E.getAcor()
        return ch.reshape(-1, k).astype(np.float64), st, tau

    sp, stp, taup = run(False)
    sd_, std_, taud = run(True)
    for s in (sp, sd_):
        assert np.all(np.abs(s.mean(0) - mu) < 0.1 * sd)
    assert np.all(np.abs(sd_.mean(0) - sp.mean(0)) < 0.1 * sd)
    assert np.all(np.abs(sd_.std(0) / sp.std(0) - 1) < 0.1)
    acc_plain = stp["accepted"] / stp["exact_evals"]
    acc_da = std_["accepted"] / std_["exact_evals"]
    print("DA stats plain", stp, "da", std_, "tau", taup, taud)
    assert acc_da > 1.5 * acc_plain, (acc_plain, acc_da, std_)
    # effective samples per exact evaluation
    ess_p = nw * 3000 / np.nanmax(taup) / stp["exact_evals"]
    ess_d = nw * 3000 / np.nanmax(taud) / std_["exact_evals"]
    assert ess_d > ess_p, (ess_p, ess_d)


def test_delayed_acceptance_wide_stretch_keeps_posterior(gpu_ctx):
    """A wider stretch for the delayed-acceptance steps (a = 4; plain a = 2)
    keeps the exact posterior (means within 0.1 sigma of the truth, widths
    within 10 %) and gives more effective samples per exact evaluation than
    the plain steps (integrated autocorrelation times, Sokal window)."""
    from pofd_affine_b200.mcmc import affineEnsemble, gaussLike, integrated_time
    from pofd_affine_b200.surrogate import Surrogate
    k, nw, ns = 6, 64, 3000
    _, _, mu, cov = _gauss_pairs(10, k, 7)
    G = gaussLike(gpu_ctx, mu, cov)
    sd = np.sqrt(np.diag(cov))

    def run(da):
        E = affineEnsemble(gpu_ctx, G, nw, k, seed=21 + da)
        E.initChains(E.generateInitialPosition(mu, sd, rng=5))
        S = Surrogate(gpu_ctx, k, list(range(k)), hidden=256, seed=4)
        E.collectPairs(S)
        E.doSteps(0, initsteps=300)
        E.collectPairs(None)
        base = E.daStats()
        if da:
            S.train(2000, batch=512, lr=1e-3)
            E.setSurrogate(S)
            E.setDAScale(4.0)
            E.doStepsDA(ns)
        else:
            E.doSteps(ns)
        st = E.daStats()
        ch, _ = E.getChain()
        tau, _, _ = integrated_time(ch)
        return ch, st["exact_evals"] - base["exact_evals"], np.nanmax(tau)

    cp, ep, tp = run(False)
    cd, ed, td = run(True)
    s = cd.reshape(-1, k).astype(np.float64)
    assert np.all(np.abs(s.mean(0) - mu) < 0.1 * sd)
    assert np.all(np.abs(s.std(0) / sd - 1) < 0.1)
    ess_p = nw * ns / tp / ep
    ess_d = nw * ns / td / ed
    print("wide-stretch DA: ESS per exact evaluation %.4f vs plain %.4f "
          "(tau %.1f vs %.1f, exact evals %d vs %d)" % (ess_d, ess_p, td, tp, ed, ep))
    assert ess_d > 2.0 * ess_p, (ess_p, ess_d)


def test_delayed_acceptance_is_exact_for_any_first_stage(gpu_ctx):
    """Delayed acceptance keeps the exact posterior whatever its first
    stage: with a deliberately wrong first stage (a Gaussian whose mean is
    off by half a standard deviation and whose covariance is 1.5 times too
    wide) in place of the surrogate, a wide stretch (a = 5) and a limit
    through the mean of one parameter (steps outside rejected), the chain's
    means agree with the plain chain's within 4 combined standard errors
    and its widths within 3 %."""
    import ctypes as C
    from pofd_affine_b200._lib import check, lib, support_lib
    from pofd_affine_b200.mcmc import affineEnsemble, gaussLike, integrated_time
    k, nw, ns = 6, 128, 8000
    rng = np.random.default_rng(7)
    A = rng.normal(size=(k, k))
    cov = A @ A.T + k * np.eye(k)
    mu = rng.normal(size=k)
    sd = np.sqrt(np.diag(cov))
    G = gaussLike(gpu_ctx, mu, cov)
    G2 = gaussLike(gpu_ctx, mu + 0.5 * sd, 1.5 * cov)

    def run(da):
        E = affineEnsemble(gpu_ctx, G, nw, k, seed=100 + da)
        E.setParamLimits(0, mu[0], np.inf)
        E.setLimitPolicy(True)
        E.initChains(E.generateInitialPosition(mu, sd, rng=3))
        E.doSteps(0, 500)
        if da:
            fn = C.cast(support_lib().pofd_gauss_eval_batch_device, C.c_void_p)
            check(lib().pofd_ensemble_set_surrogate(E.h, fn, G2.h))
            E.setDAScale(5.0)
            E.doStepsDA(ns)
        else:
            E.doSteps(ns)
        ch, _ = E.getChain()
        tau, _, _ = integrated_time(ch)
        s = ch.reshape(-1, k).astype(np.float64)
        return s.mean(0), s.std(0), np.nanmax(tau)
    mp, sp, tp = run(0)
    md, sdd, td = run(1)
    se = np.sqrt(sp ** 2 * tp / (nw * ns) + sdd ** 2 * td / (nw * ns))
    assert np.all(np.abs(md - mp) < 4 * se), (md - mp) / se
    assert np.all(np.abs(sdd / sp - 1) < 0.03), sdd / sp
