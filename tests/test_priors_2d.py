"""Priors, bonus parameters and regularisation of the 2D likelihood.

Reference: calcLikeDouble::getLogLike adds per band a Gaussian prior on the
sigma multiplier, on <S_b> (CFIRB) and on <S_b^2> (Poisson), then alpha
times the band-1 log-slope penalty (calcLikeDouble.cc:1236-1276); the bonus
parameters <S1>, <S2>, <S1^2>, <S2^2> are numberCountsDoubleLogNormal::
splineInt (numberCountsDoubleLogNormal.cc:1549-1631), filled after the two
sigma multipliers (calcLikeDouble.cc:1283-1310).

CPU tests pin the oracle's integrals against the reference's golden values
(model_test.cc:681-702) and an independent adaptive quadrature, and its
prior terms against numpy.  GPU tests compare the CUDA path with the oracle:
log-likelihoods within 1e-6 absolute, integrals within 1e-12 relative.
"""
import numpy as np
import pytest

from test_gpu_2d import build2, spec2

LL_TOL = 1e-6
HALF_LOG_2PI = 0.918938517570495605469
LOGFAC = np.log2(10.0)


def _independent(kp, sk, sv, ok, ov, kv, a, b, min_sigma=0.0):
    """S1^(a+b) n1 exp(b mu + b^2/2 sigma^2) integrated with scipy, broken
    at every knot; colour curves constant (1 knot), linear (2) or natural
    cubic (3+), clamped outside their knots."""
    from scipy.integrate import quad
    from scipy.interpolate import CubicSpline
    kp = np.asarray(kp, np.float64)
    cs = CubicSpline(np.log2(kp), LOGFAC * np.asarray(kv, np.float64),
                     bc_type="natural")

    def curve(x, v):
        x, v = np.asarray(x, np.float64), np.asarray(v, np.float64)
        if len(x) == 1:
            return lambda s: v[0]
        if len(x) == 2:
            return lambda s: np.interp(s, x, v)
        c = CubicSpline(x, v, bc_type="natural")
        return lambda s: v[0] if s <= x[0] else (v[-1] if s >= x[-1]
                                                 else float(c(s)))
    sg, mu = curve(sk, sv), curve(ok, ov)

    def f(s):
        sig = max(sg(s), min_sigma)
        return (s ** (a + b) * np.exp(b * mu(s) + 0.5 * b * b * sig * sig)
                * 2.0 ** cs(np.log2(s)))
    pts = sorted(set(list(kp) + [x for x in list(sk) + list(ok)
                                 if kp[0] < x < kp[-1]]))
    return sum(quad(f, pts[i], pts[i + 1], epsrel=1e-13, limit=400)[0]
               for i in range(len(pts) - 1))


def test_oracle_integrals_golden_and_independent(orc, golden):
    m, g = golden["model2"], golden["integrals2"]
    c = orc.Counts2(m["knotpos_f32"], m["sigmapos_f32"], m["offsetpos_f32"])
    c.set(m["pvals"])
    assert abs(c.spline_int(0, 0) - g["ns"][0]) < g["ns"][1]
    assert abs(c.spline_int(1, 0) - g["flux_per_area1"][0]) < g["flux_per_area1"][1]
    assert abs(c.spline_int(0, 1) - g["flux_per_area2"][0]) < g["flux_per_area2"][1]
    for nsig, noff in ((2, 1), (3, 3), (1, 2)):
        s = spec2(nsig=nsig, noff=noff, shape=(32, 32))
        K = len(s["kp"])
        th = s["th"].astype(np.float64)
        c = orc.Counts2(s["kp"], s["sk"], s["ok"])
        c.set(s["th"])
        sv, ov = th[K:K + nsig], th[K + nsig:K + nsig + noff]
        for a, b in ((1, 0), (0, 1), (2, 0), (0, 2)):
            ref = _independent(s["kp"], s["sk"], sv, s["ok"], ov, th[:K], a, b)
            assert abs(c.spline_int(a, b) / ref - 1) < 1e-11, (nsig, noff, a, b)


def test_oracle_prior_terms_2d(orc):
    s = spec2(shape=(48, 48), n=128, nedge=32)
    O = orc.Like2(s["kp"], s["sk"], s["ok"], s["n"], s["nedge"], s["edge"],
                  s["nbins"], s["bin_data"])
    O.add_beamset(s["b1"], s["b2"], s["ps"], s["minval"], True, s["nh"])
    m1, m2 = s["maps"][0]
    O.add_dataset(0, m1, m2, *s["noise"])
    O.set_rranges(s["th"])
    th = s["th"].copy()
    th[-2], th[-1] = 1.05, 0.97
    base = O.loglike(th)
    b = O.bonus(th)
    K = len(s["kp"])
    lk = np.log2(s["kp"])
    sl = np.diff(LOGFAC * th[:K].astype(np.float64)) / np.diff(lk)
    pen = -np.sum((sl - sl.mean()) ** 2)
    sm = [float(th[-2]), float(th[-1])]
    cases = [
        (dict(sigma=(0.05, None)), -(HALF_LOG_2PI + np.log(0.05)
                                     + 0.5 * ((sm[0] - 1) / 0.05) ** 2)),
        (dict(sigma=(None, 0.1)), -(HALF_LOG_2PI + np.log(0.1)
                                    + 0.5 * ((sm[1] - 1) / 0.1) ** 2)),
        (dict(cfirb=(None, (b[1] * 1.2, b[1] * 0.1))),
         -(HALF_LOG_2PI + np.log(b[1] * 0.1) + 0.5 * 2.0 ** 2)),
        (dict(poisson=((b[2] * 0.8, b[2] * 0.4), None)),
         -(HALF_LOG_2PI + np.log(b[2] * 0.4) + 0.5 * 0.5 ** 2)),
        (dict(alpha=1.5), 1.5 * pen),
    ]
    for kw, term in cases:
        O.set_priors(**kw)
        assert abs((O.loglike(th) - base) - term) < 1e-8 * max(1, abs(term))
    O.set_priors()
    assert O.loglike(th) == base


# ------------------------------------------------------------------ GPU
def _batch(s, nprop=6, seed=4):
    rng = np.random.default_rng(seed)
    th = np.repeat(s["th"][None, :], nprop, 0)
    K = len(s["kp"])
    th[:, :K] += rng.normal(0, 0.04, (nprop, K)).astype(np.float32)
    th[:, -2:] = rng.uniform(0.92, 1.08, (nprop, 2)).astype(np.float32)
    return th


@pytest.mark.gpu
@pytest.mark.parametrize("curves", [(3, 3), (2, 1), (1, 2)])
def test_gpu_bonus_2d_matches_oracle(orc, gpu_ctx, curves):
    s = spec2(nsig=curves[0], noff=curves[1], shape=(48, 48))
    O, G = build2(orc, gpu_ctx, s)
    th = _batch(s)
    bg = G.getBonus(th)
    bo = np.array([O.bonus(t) for t in th])
    assert np.max(np.abs(bg / bo - 1)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["sigma", "cfirb", "poisson", "alpha",
                                  "all"])
def test_gpu_priors_2d_match_oracle(orc, gpu_ctx, case):
    s = spec2(shape=(48, 48))
    O, G = build2(orc, gpu_ctx, s)
    th = _batch(s)
    b0 = O.bonus(s["th"])
    kw = dict(sigma=[None, None], cfirb=[None, None], poisson=[None, None],
              alpha=0.0)
    if case in ("sigma", "all"):
        kw["sigma"] = [0.05, 0.08]
    if case in ("cfirb", "all"):
        kw["cfirb"] = [(b0[0] * 1.04, b0[0] * 0.03), (b0[1] * 0.97, b0[1] * 0.05)]
    if case in ("poisson", "all"):
        kw["poisson"] = [(b0[2] * 1.1, b0[2] * 0.2), (b0[3] * 0.9, b0[3] * 0.3)]
    if case in ("alpha", "all"):
        kw["alpha"] = 0.7
    G.getLogLikeBatch(th)  # graphs captured before the priors change
    O.set_priors(**kw)
    for b in range(2):
        if kw["sigma"][b] is not None:
            G.setSigmaPrior(b, kw["sigma"][b])
        if kw["cfirb"][b] is not None:
            G.setCFIRBPrior(b, *kw["cfirb"][b])
        if kw["poisson"][b] is not None:
            G.setPoissonPrior(b, *kw["poisson"][b])
    if kw["alpha"]:
        G.setRegularizationAlpha(kw["alpha"])
    lg, st = G.getLogLikeBatch(th)
    assert np.all(st == 0)
    lo, _ = O.loglike_batch(th)
    assert np.max(np.abs(lg - lo)) < LL_TOL
    if case == "all":
        for b in range(2):
            G.unsetSigmaPrior(b)
            G.unsetCFIRBPrior(b)
            G.unsetPoissonPrior(b)
        G.setRegularizationAlpha(0.0)
        O.set_priors()
        lg2, _ = G.getLogLikeBatch(th)
        assert np.max(np.abs(lg2 - O.loglike_batch(th)[0])) < LL_TOL


@pytest.mark.gpu
def test_gpu_fill_bonus_2d_and_ensemble(orc, gpu_ctx):
    from pofd_affine_b200.mcmc import affineEnsemble
    s = spec2(shape=(48, 48))
    O, G = build2(orc, gpu_ctx, s)
    th = _batch(s)
    nm = G.nmodel
    thb = np.concatenate([th, np.full((th.shape[0], 4), np.nan, np.float32)], 1)
    f = G.fillBonusParams(thb)
    assert np.array_equal(f[:, :th.shape[1]], th)
    bo = np.array([O.bonus(t) for t in th])
    assert np.array_equal(f[:, nm + 2:], bo.astype(np.float32))
    np_ = th.shape[1] + 4
    E = affineEnsemble(gpu_ctx, G, 12, np_, seed=3)
    for p in range(len(s["kp"]), np_):
        if p >= nm + 2:
            E.setParamBonus(p)
        else:
            E.setParamFixed(p)
    theta0 = np.concatenate([s["th"], np.zeros(4)]).astype(np.float32)
    sig = np.zeros(np_)
    sig[:len(s["kp"])] = 0.02
    E.initChains(E.generateInitialPosition(theta0, sig, rng=2))
    E.doSteps(3)
    ch, ll = E.getChain()
    rows = ch.reshape(-1, np_)
    assert np.all(np.isfinite(ll))
    for r in rows[::5]:
        assert np.array_equal(r[nm + 2:], O.bonus(r[:nm + 2]).astype(np.float32))
