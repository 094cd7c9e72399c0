"""Cross-checks of the oracle's numerical building blocks against numpy and
scipy, and of its 1D P(D) pipeline against an independent numpy
restatement of PDFactory.cc:1031-1243 (given the oracle's R grid)."""
import numpy as np
import pytest
from scipy.interpolate import CubicSpline


def test_natural_spline_matches_scipy(orc):
    rng = np.random.default_rng(3)
    x = np.sort(rng.uniform(0, 10, 40))
    y = np.sin(x) + rng.normal(0, 0.1, 40)
    xq = np.linspace(x[0], x[-1], 1001)
    ref = CubicSpline(x, y, bc_type="natural")(xq)
    got = orc.cspline_eval(x, y, xq)
    assert np.max(np.abs(got - ref)) < 1e-12


@pytest.mark.parametrize("n", [64, 4096, 1000, 3])
def test_rfft_irfft(orc, n):
    rng = np.random.default_rng(n)
    a = rng.normal(size=n)
    assert np.allclose(orc.rfft(a), np.fft.rfft(a), rtol=0, atol=1e-12 * n)
    c = np.fft.rfft(a) + 1j * rng.normal(size=n // 2 + 1)  # non-Hermitian
    ref = np.fft.irfft(c, n) * n  # numpy also drops imag of DC/Nyquist
    assert np.allclose(orc.irfft(c, n), ref, rtol=0, atol=1e-11 * n)


def test_rfft2_irfft2(orc):
    n = 64
    rng = np.random.default_rng(5)
    a = rng.normal(size=(n, n))
    assert np.allclose(orc.rfft2(a), np.fft.rfft2(a), atol=1e-10)
    c = np.fft.rfft2(a)
    assert np.allclose(orc.irfft2(c, n), a * n * n, atol=1e-9)
    # self-conjugate columns are reduced to their Hermitian part
    c2 = c.copy()
    c2[:, 0] += 1j * rng.normal(size=n)
    c2[:, n // 2] += rng.normal(size=n) + 1j * rng.normal(size=n)
    h = c2.copy()
    for j in (0, n // 2):
        col = c2[:, j]
        h[:, j] = 0.5 * (col + np.conj(col[(-np.arange(n)) % n]))
    ref = np.fft.irfft2(h, s=(n, n)) * n * n
    assert np.allclose(orc.irfft2(c2, n), ref, atol=1e-9)


def _split_1d(p, n, dflux, sgpos, sgneg, minflux_R, wrap):
    """PDFactory::findSplitPoint (PDFactory.cc:691-921), pure Python."""
    n1, f1, f2, f3 = 2.5, 5e-14, 1e-5, 5
    peak = max(p)
    n1p, n1n = n1 * sgpos, n1 * sgneg
    bot = int(n1p / dflux)
    top = wrap if n1p > abs(minflux_R) else int(-(n1n + minflux_R) / dflux + wrap + 1)
    mi, mv = bot, p[bot]
    for i in range(bot + 1, top + 1):
        if p[i] < mv:
            mi, mv = i, p[i]
    assert mv <= f2 * peak
    if mi > 17:
        mono = True
        jit = prev = p[mi - 17]
        for i in range(mi - 16, mi):
            if p[i] >= prev:
                mono = False
            jit += p[i]
            prev = p[i]
        if mono:
            return mi
        jit = 1.1 * (jit + mv) / 18
    else:
        jit = f1 * peak
        if mv > jit:
            return mi
    if mv <= 0:
        bi = bot if mi < bot else max(0, mi - 3)
        ti = top - 3 if mi > top - 3 else mi + 3
        for i in range(bi, ti):
            mv = max(mv, p[i])
    if mv > 0:
        jit = min(f3 * mv, jit)
    for i in range(top - 1, bot - 1, -1):
        if p[i] < jit:
            return i + 1
    raise AssertionError("no split")


def _make_like(orc, beams, n=4096, noise=0.002, seed=0):
    from pofd_affine_b200 import synth
    rng = np.random.default_rng(seed)
    kp, kv = synth.knot_model(6, 0.002, 0.4, rng=rng)
    bm = synth.gaussian_beam(3.0)
    img = synth.make_map((128, 128), 6.0, bm, kp, kv, noise, rng)
    L = orc.Like1(kp, n, 512, True, 500)
    L.add_beamset(bm, 6.0, 1e-5, True, 120)
    L.add_dataset(0, img, noise)
    th = np.concatenate([kv, [1.0]]).astype(np.float32)
    L.set_rranges(th)
    return L, th, kp, kv


@pytest.mark.parametrize("noise", [0.002, 0.0005])
def test_pd_pipeline_matches_numpy_restatement(orc, beams, noise):
    L, th, kp, kv = _make_like(orc, beams, 4096, noise)
    pd, info, rv = L.pd(0, 0, th, setlog=False, want_r=True)
    n = rv.size
    dflux, wrap, mfr = info["dflux"], int(info["wrapRidx"]), info["minflux_R"]
    # moments with the reference's lower-edge read (PDFactory.cc:660-666)
    i = np.arange(n)
    cf = np.where(i <= wrap, i * dflux, (i - wrap - 1) * dflux + mfr)
    w = np.ones(n)
    w[0] = 0
    w[wrap] = 0.5
    mn = np.sum(w * cf * rv)
    var = np.sum(w * cf * cf * rv)
    if wrap < n - 1:
        mn -= 0.5 * mfr * rv[wrap - 1]
        var -= mfr * 0.5 * mfr * rv[wrap - 1]
    assert abs(mn - info["mn"]) <= 1e-12 * abs(mn)
    assert abs(var - info["var_noi"]) <= 1e-12 * abs(var)
    sg = np.sqrt(var)
    doshift = sg > dflux and abs(mn) > dflux
    assert doshift == bool(info["doshift"])
    shift = -mn if doshift else 0.0
    rt = np.fft.rfft(rv)
    k = np.arange(rt.size)
    iflux = 2 * np.pi / (n * dflux)
    p = np.exp(rt.real - rt[0].real) * np.exp(1j * (rt.imag - shift * iflux * k))
    p[0] = 1.0
    p = p * np.exp(-0.5 * noise ** 2 * (iflux * k) ** 2)
    p[0] = 1.0
    pofd = np.fft.irfft(p, n) * n
    pofd[pofd < 0] = 0
    sgpos = np.sqrt(var + noise ** 2)
    sgneg = noise if 9 * noise ** 2 > var else sgpos
    split = _split_1d(list(pofd), n, dflux, sgpos, sgneg, mfr, wrap)
    assert split == int(info["splitidx"])
    q = np.concatenate([pofd[split:], pofd[:split]])
    tot = (0.5 * q[0] + q[1:-1].sum() + 0.5 * q[-1]) * dflux
    q = q / tot
    assert np.max(np.abs(q - pd)) <= 1e-10 * q.max()
    mean = (np.sum(np.arange(1, n - 1) * q[1:-1]) + 0.5 * (n - 1) * q[-1]) * dflux ** 2
    assert abs(-mean - info["pd_minflux"]) <= 1e-10 * abs(mean)


def test_loglike_matches_numpy_gather(orc, beams):
    L, th, kp, kv = _make_like(orc, beams)
    lp, info = L.pd(0, 0, th, setlog=True)
    di = L.dataset_info(0, 0)
    bins = L.dataset_bins(0, 0)
    n = lp.size
    mf, df = info["pd_minflux"], info["dflux"]
    ll = 0.0
    for i, c in enumerate(bins):
        if c == 0:
            continue
        x = di["bincent0"] + i * di["bindelta"]
        if x < mf:
            ll += c * lp[0]
        elif x > mf + (n - 2) * df:
            ll += c * lp[-1]
        else:
            d = (x - mf) / df
            j = int(d)
            t = d - j
            ll += ((1 - t) * lp[j] + t * lp[j + 1]) * c
    ll = np.log(2.0) * ll
    expect = (ll - di["like_offset"]) / di["like_norm"]
    assert abs(L.loglike(th) - expect) < 1e-6


def test_like_batch_threads_match_serial(orc, beams):
    L, th, kp, kv = _make_like(orc, beams)
    rng = np.random.default_rng(9)
    thetas = np.tile(th, (6, 1))
    thetas[:, :-1] += rng.normal(0, 0.02, (6, th.size - 1)).astype(np.float32)
    thetas[3, 2] = np.nan
    ll1, st1 = L.loglike_batch(thetas, 1)
    ll4, st4 = L.loglike_batch(thetas, 4)
    assert list(st1) == list(st4)
    assert st1[3] == -1 and np.isnan(ll1[3])
    ok = st1 == 0
    assert np.array_equal(ll1[ok], ll4[ok])


@pytest.mark.parametrize("n", [8, 32, 256, 4096, 65536])
def test_fast_real_fft_against_numpy(orc, n):
    """The timed CPU baseline's radix-4 real transforms (oracle/fastfft.cc)
    against numpy's, forward and unnormalised inverse, 1D and 2D."""
    rng = np.random.default_rng(n)
    x = rng.normal(size=n)
    X = np.fft.rfft(x)
    Y = X * np.exp(0.1j * rng.normal(size=X.size))
    orc.set_fast_fft(True)
    try:
        f = orc.rfft(x)
        y = orc.irfft(Y, n)
        if n <= 256:
            x2 = rng.normal(size=(n, n))
            X2 = np.fft.rfft2(x2)
            Y2 = X2 * np.exp(0.1j * rng.normal(size=X2.shape))
            f2 = orc.rfft2(x2)
            y2 = orc.irfft2(Y2, n)
    finally:
        orc.set_fast_fft(False)
    assert np.max(np.abs(f - X)) < 1e-14 * np.abs(X).max()
    yr = np.fft.irfft(Y, n) * n
    assert np.max(np.abs(y - yr)) < 1e-14 * np.abs(yr).max()
    if n <= 256:
        assert np.max(np.abs(f2 - X2)) < 1e-14 * np.abs(X2).max()
        y2r = np.fft.irfft2(Y2, (n, n)) * n * n
        assert np.max(np.abs(y2 - y2r)) < 1e-14 * np.abs(y2r).max()


def test_fast_fft_likelihood_agrees(orc):
    """The oracle's log-likelihood with the fast transforms (the timed CPU
    baseline) against the radix-2 parity form."""
    from pofd_affine_b200 import synth
    cfg = synth.config_1d_small(seed=3)
    O = orc.Like1(cfg["knotpos"], 8192, 512, True, 500)
    O.add_beamset(cfg["beams"][0], 6.0, 1e-5, True, 120)
    O.add_dataset(0, cfg["maps"][0], cfg["sigmas"][0])
    O.set_rranges(cfg["theta0"])
    th = synth.proposals(cfg["theta0"], 4, 0.02, rng=5)
    l0, s0 = O.loglike_batch(th, 2)
    orc.set_fast_fft(True)
    try:
        l1, s1 = O.loglike_batch(th, 2)
    finally:
        orc.set_fast_fft(False)
    assert list(s0) == list(s1)
    assert np.max(np.abs(l1 - l0)) < 1e-6
