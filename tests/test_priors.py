"""Priors, bonus parameters and regularisation of the 1D likelihood.

Reference: calcLike::getLogLike adds, once for all beam sets, a Gaussian
prior on the sigma multiplier about 1, Gaussian priors on <S> (CFIRB) and
<S^2> (Poisson), then alpha times the log-slope penalty
(calcLike.cc:918-952, numberCountsKnotsSpline.cc:540-559); the bonus
parameters <S>, <S^2> are the integrals of numberCountsKnotsSpline.cc:
300-343, filled after the sigma multiplier (calcLike.cc:958-980).

CPU tests pin the oracle: its integrals against an independent adaptive
quadrature and the reference's golden values, and its prior terms against a
restatement in numpy.  GPU tests compare the CUDA path with the oracle:
log-likelihoods within 1e-6 absolute, bonus integrals within 1e-12
relative.
"""
import numpy as np
import pytest

LL_TOL = 1e-6
HALF_LOG_2PI = 0.918938517570495605469
LOGFAC = np.log2(10.0)


def _small(seed=3, n=4096, ni=512, nbins=400):
    from pofd_affine_b200 import synth
    rng = np.random.default_rng(seed)
    kp, kv = synth.knot_model(6, 0.002, 0.4, rng=rng)
    bm = synth.gaussian_beam(3.0)
    img = synth.make_map((128, 128), 6.0, bm, kp, kv, 0.002, rng)
    th = np.concatenate([kv, [1.0]]).astype(np.float32)
    return dict(kp=kp, kv=kv, bm=bm, img=img, th=th, n=n, ni=ni,
                nbins=nbins)


def _oracle(orc, s):
    O = orc.Like1(s["kp"], s["n"], s["ni"], True, s["nbins"])
    O.add_beamset(s["bm"], 6.0, 1e-5, True, 120)
    O.add_dataset(0, s["img"], 0.002)
    O.set_rranges(s["th"])
    return O


def _penalty(kp, theta):
    """numberCountsKnotsSpline::differenceRegularize without alpha."""
    lk = np.log2(np.asarray(kp, np.float64))
    lv = LOGFAC * np.asarray(theta[:len(kp)], np.float64)
    sl = np.diff(lv) / np.diff(lk)
    return -np.sum((sl - sl.mean()) ** 2)


def _independent_bonus(kp, theta):
    from scipy.integrate import quad
    from scipy.interpolate import CubicSpline
    kp = np.asarray(kp, np.float64)
    lk = np.log2(kp)
    lv = LOGFAC * np.asarray(theta[:len(kp)], np.float64)
    cs = CubicSpline(lk, lv, bc_type="natural")
    out = []
    for a in (1, 2):
        tot = 0.0
        for i in range(len(kp) - 1):
            v, _ = quad(lambda s: s ** a * 2.0 ** cs(np.log2(s)), kp[i],
                        kp[i + 1], epsrel=1e-13, limit=200)
            tot += v
        out.append(tot)
    return np.array(out)


def test_oracle_bonus_matches_independent_quadrature(orc):
    s = _small()
    O = _oracle(orc, s)
    rng = np.random.default_rng(0)
    for k in range(3):
        th = s["th"].copy()
        th[:6] += rng.normal(0, 0.1, 6).astype(np.float32)
        b = O.bonus(th)
        ref = _independent_bonus(s["kp"], th)
        assert np.allclose(b, ref, rtol=1e-12, atol=0)


def test_oracle_prior_terms(orc):
    s = _small()
    O = _oracle(orc, s)
    th = s["th"].copy()
    th[6] = 1.07
    base = O.loglike(th)
    b = O.bonus(th)
    cases = [
        (dict(sigma=0.05), -(HALF_LOG_2PI + np.log(0.05)
                             + 0.5 * ((float(th[6]) - 1.0) / 0.05) ** 2)),
        (dict(cfirb=(b[0] * 1.1, b[0] * 0.05)),
         -(HALF_LOG_2PI + np.log(b[0] * 0.05) + 0.5 * (0.1 / 0.05) ** 2)),
        (dict(poisson=(b[1] * 0.9, b[1] * 0.2)),
         -(HALF_LOG_2PI + np.log(b[1] * 0.2) + 0.5 * (0.1 / 0.2) ** 2)),
        (dict(alpha=3.5), 3.5 * _penalty(s["kp"], th)),
    ]
    for kw, term in cases:
        O.set_priors(**kw)
        assert abs((O.loglike(th) - base) - term) < 1e-8 * max(1, abs(term))
    O.set_priors()
    assert O.loglike(th) == base


# ------------------------------------------------------------------ GPU
def _both(orc, ctx, s):
    from pofd_affine_b200 import beam, calcLike
    O = _oracle(orc, s)
    G = calcLike(ctx, s["kp"], s["n"], s["ni"], True, s["nbins"])
    G.addBeamSet(beam(s["bm"], 6.0, True, 120, 1e-5))
    G.addDataset(0, s["img"], 0.002)
    G.setRRanges(s["th"])
    return O, G


def _batch(s, nprop=12, seed=5):
    rng = np.random.default_rng(seed)
    th = np.repeat(s["th"][None, :], nprop, 0)
    th[:, :6] += rng.normal(0, 0.05, (nprop, 6)).astype(np.float32)
    th[:, 6] = rng.uniform(0.9, 1.1, nprop).astype(np.float32)
    return th


@pytest.mark.gpu
def test_gpu_bonus_matches_oracle_and_golden(orc, gpu_ctx, golden):
    s = _small()
    O, G = _both(orc, gpu_ctx, s)
    th = _batch(s)
    bg = G.getBonus(th)
    bo = np.array([O.bonus(t) for t in th])
    assert np.max(np.abs(bg / bo - 1)) < 1e-12
    # the reference's own integration test (model_test.cc:196-212)
    g, c = golden["integrals1"], golden["counts1"]
    s5 = dict(s, kp=np.array(c["knotpos_f32"], np.float64),
              th=np.array(c["knotval"] + [1.0], np.float32))
    O5, G5 = _both(orc, gpu_ctx, s5)
    b5 = G5.getBonus(s5["th"])[0]
    assert np.max(np.abs(b5 / O5.bonus(s5["th"]) - 1)) < 1e-12
    assert abs(b5[0] - g["flux_per_area"][0]) < g["flux_per_area"][1]
    assert abs(b5[1] - g["fluxsq_per_area"][0]) < g["fluxsq_per_area"][1]


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["sigma", "cfirb", "poisson", "alpha",
                                  "all", "off"])
def test_gpu_priors_match_oracle(orc, gpu_ctx, case):
    s = _small()
    O, G = _both(orc, gpu_ctx, s)
    th = _batch(s)
    b0 = O.bonus(s["th"])
    kw = {}
    if case in ("sigma", "all"):
        kw["sigma"] = 0.04
    if case in ("cfirb", "all"):
        kw["cfirb"] = (b0[0] * 1.05, b0[0] * 0.03)
    if case in ("poisson", "all"):
        kw["poisson"] = (b0[1] * 0.95, b0[1] * 0.1)
    if case in ("alpha", "all"):
        kw["alpha"] = 2.0
    G.getLogLikeBatch(th)  # graphs captured before the priors change
    O.set_priors(**kw)
    if "sigma" in kw:
        G.setSigmaPrior(kw["sigma"])
    if "cfirb" in kw:
        G.setCFIRBPrior(*kw["cfirb"])
    if "poisson" in kw:
        G.setPoissonPrior(*kw["poisson"])
    if "alpha" in kw:
        G.setRegularizationAlpha(kw["alpha"])
    lg, st = G.getLogLikeBatch(th)
    assert np.all(st == 0)
    lo, _ = O.loglike_batch(th)
    assert np.max(np.abs(lg - lo)) < LL_TOL
    if case == "all":
        # unsetting restores the plain likelihood
        G.unsetSigmaPrior()
        G.unsetCFIRBPrior()
        G.unsetPoissonPrior()
        G.setRegularizationAlpha(0.0)
        O.set_priors()
        lg2, _ = G.getLogLikeBatch(th)
        assert np.max(np.abs(lg2 - O.loglike_batch(th)[0])) < LL_TOL


@pytest.mark.gpu
def test_gpu_prior_setter_errors(gpu_ctx):
    from pofd_affine_b200 import PofdError
    s = _small()
    from pofd_affine_b200 import calcLike
    G = calcLike(gpu_ctx, s["kp"], s["n"], s["ni"], True, s["nbins"])
    for bad in (lambda: G.setCFIRBPrior(-1.0, 1.0),
                lambda: G.setCFIRBPrior(1.0, -1.0),
                lambda: G.setPoissonPrior(-1.0, 1.0),
                lambda: G.setRegularizationAlpha(-0.5),
                lambda: G.setSigmaPrior(0.0)):
        with pytest.raises(PofdError):
            bad()


@pytest.mark.gpu
def test_gpu_fill_bonus_params(orc, gpu_ctx):
    s = _small()
    O, G = _both(orc, gpu_ctx, s)
    th = _batch(s)
    th9 = np.concatenate([th, np.full((th.shape[0], 2), np.nan, np.float32)],
                         1)
    f = G.fillBonusParams(th9)
    bo = np.array([O.bonus(t) for t in th])
    assert np.array_equal(f[:, :7], th)
    assert np.array_equal(f[:, 7:], bo.astype(np.float32))


@pytest.mark.gpu
def test_gpu_ensemble_records_bonus_params(orc, gpu_ctx):
    """Walkers over knots + sigma + two bonus slots: every recorded row
    carries the <S>, <S^2> of its own knot values (pofdMCMC.cc:354-360)."""
    from pofd_affine_b200.mcmc import affineEnsemble
    s = _small()
    O, G = _both(orc, gpu_ctx, s)
    np_ = 9
    E = affineEnsemble(gpu_ctx, G, 16, np_, seed=11)
    E.setParamFixed(6)
    E.setParamBonus(7)
    E.setParamBonus(8)
    theta0 = np.concatenate([s["th"], [0.0, 0.0]]).astype(np.float32)
    sig = np.concatenate([np.full(6, 0.02), [0.0, 0.0, 0.0]])
    E.initChains(E.generateInitialPosition(theta0, sig, rng=1))
    E.doSteps(6)
    ch, ll = E.getChain()
    rows = ch.reshape(-1, np_)
    assert np.all(np.isfinite(ll))
    assert np.all(np.isfinite(rows[:, 7:]))
    idx = np.random.default_rng(0).choice(len(rows), 20, replace=False)
    for r in rows[idx]:
        assert np.array_equal(r[7:], O.bonus(r[:7]).astype(np.float32))
