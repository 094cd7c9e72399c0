"""Chain output and the pofd_affine_getStats restatement (CPU).

The number counts are pinned to the reference's model test
(model_test.cc:182-192: log10 dN/dS at 0.003, 0.007, 0.015 Jy and at the
interior knots); the two-band colour curves to the reference's
two-band counts (model_test.cc:646-677) and to the oracle's sigma / offset
restatement; the accumulator to a direct restatement of
statsAccumulator::accumulateStats; the chain writer by a round trip."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def test_number_counts_against_reference_goldens():
    from pofd_affine_b200 import stats
    g = json.load(open(os.path.join(HERE, "golden", "reference_goldens.json")))["counts1"]
    kp = np.array(g["knotpos_f32"])
    th = np.array(g["knotval"], np.float32)
    got = np.log10(stats.numberCounts(kp, th, g["testpos"]))
    assert np.max(np.abs(got - np.array(g["testval_log10"]))) < g["tol"]
    inner = np.log10(stats.numberCounts(kp, th, kp[1:-1]))
    assert np.max(np.abs(inner - th[1:-1])) < g["interior_tol"]
    assert stats.numberCounts(kp, th, [kp[0] * 0.99, kp[-1]]).tolist() == [0.0, 0.0]


def _reference_accumulate(working, plevels=(0.683, 0.954, 0.997)):
    w = np.sort(np.asarray(working, np.float32), axis=1)
    n1, n2 = w.shape
    mean = np.empty(n1, np.float32)
    med = np.empty(n1, np.float32)
    snake = np.empty((3, n1, 2), np.float32)
    for j in range(n1):
        acc = float(w[j, 0])
        for k in range(1, n2):
            acc += float(w[j, k])
        mean[j] = np.float32(acc / n2)
        med[j] = w[j, n2 // 2]
        for k, p in enumerate(plevels):
            lo = np.float32(0.5) * (np.float32(1.0) - np.float32(p)) * np.float32(n2)
            hi = np.float32(0.5) * (np.float32(1.0) + np.float32(p)) * np.float32(n2)
            il, iu = int(lo), int(hi)
            snake[k, j, 0] = w[j, il] + (w[j, il + 1] - w[j, il]) * (lo - np.float32(il))
            snake[k, j, 1] = w[j, iu] + (w[j, iu + 1] - w[j, iu]) * (hi - np.float32(iu))
    return mean, med, snake


def test_accumulate_stats_restates_the_reference():
    from pofd_affine_b200 import stats
    rng = np.random.default_rng(2)
    work = rng.normal(size=(7, 1500)).astype(np.float32)
    m, md, sn = stats.accumulateStats(work)
    rm, rmd, rsn = _reference_accumulate(work)
    assert np.array_equal(m, rm) and np.array_equal(md, rmd)
    assert np.array_equal(sn, rsn)
    # a Gaussian's intervals
    big = rng.normal(size=(1, 200000)).astype(np.float32)
    _, _, s2 = stats.accumulateStats(big)
    assert abs(s2[0, 0, 0] + 1.0) < 0.02 and abs(s2[0, 0, 1] - 1.0) < 0.02
    assert abs(s2[1, 0, 1] - 2.0) < 0.03


def test_number_counts_stats_and_chain_round_trip(tmp_path):
    from pofd_affine_b200 import stats
    g = json.load(open(os.path.join(HERE, "golden", "reference_goldens.json")))["counts1"]
    kp = np.array(g["knotpos_f32"])
    th0 = np.array(g["knotval"], np.float32)
    rng = np.random.default_rng(5)
    nsteps, nw = 60, 10
    chain = (th0 + rng.normal(0, 0.05, (nsteps, nw, 5))).astype(np.float32)
    chain = np.concatenate([chain, np.ones((nsteps, nw, 1), np.float32)], 2)
    logl = -np.sum((chain[..., :5] - th0) ** 2, axis=2)
    r = stats.numberCountsStats(chain, logl, kp, nflux=64, thin=3)
    assert r["nsamples"] == (nsteps * nw + 2) // 3
    i = np.unravel_index(np.argmax(logl), logl.shape)
    assert np.array_equal(r["best_params"], chain[i])
    assert np.all(r["snake"][0, :, 0] <= r["median"]) and np.all(r["median"] <= r["snake"][0, :, 1])
    mid = np.log10(stats.numberCounts(kp, th0, r["flux"]))
    assert np.max(np.abs(r["median"] - mid)) < 0.1
    assert abs(r["flux"][0] - kp[0]) < 1e-9 and r["flux"][-1] < kp[-1]
    path = str(tmp_path / "chain.npz")
    stats.writeChain(path, chain, logl, param_names=["k%d" % k for k in range(5)] + ["sigmult"],
                     param_states=[0, 0, 0, 0, 0, 1], acceptance=np.full(nw, 0.3),
                     acor=np.full(6, 4.0), knotpos=kp, model="numberCountsKnotsSpline")
    back = stats.readChain(path)
    assert np.array_equal(back["chain"], chain) and np.array_equal(back["likelihood"], logl)
    assert list(back["param_states"]) == [0, 0, 0, 0, 0, 1]
    assert str(back["model"]) == "numberCountsKnotsSpline"
    raw = np.load(path)
    assert raw["chain"].shape == (nw, nsteps, 6)  # the reference's [walker][step][param]


def _counts2_from_curves(stats, m, f1, f2):
    """dN/dS1 dS2 = n1(S1) lognormal(S2/S1; offset(S1), sigma(S1)) / S2
    (numberCountsDoubleLogNormal::getNumberCountsInner) from the stats
    module's band-1 counts and colour curves."""
    K, NS = len(m["knotpos_f32"]), len(m["sigmapos_f32"])
    p = np.array(m["pvals"], np.float32)
    f1, f2 = np.asarray(f1, float), np.asarray(f2, float)
    n1 = stats.numberCounts(m["knotpos_f32"], p[:K], f1)
    sg = stats.colourCurve(m["sigmapos_f32"], p[K:K + NS], f1, 0.0)
    mu = stats.colourCurve(m["offsetpos_f32"], p[K + NS:], f1)
    t = (np.log(f2 / f1) - mu) / sg
    return n1 * np.exp(-0.5 * t * t) / (np.sqrt(2 * np.pi) * sg * f2)


def test_colour_curves_against_reference_goldens_and_oracle(orc, golden):
    from pofd_affine_b200 import stats
    g, m = golden["counts2"], golden["model2"]
    got = _counts2_from_curves(stats, m, g["f1"], g["f2"])
    assert np.all(np.abs(got / np.array(g["counts"]) - 1) < g["reltol"])
    # one, two and five sigma / offset knots against the oracle's restatement
    f1 = np.concatenate([np.geomspace(0.001, 0.06, 200), [0.002, 0.02, 0.04]])
    for sp, op in (([0.01], [0.03]), ([0.002, 0.02], [0.003, 0.03]),
                   ([0.002, 0.005, 0.01, 0.02, 0.04], [0.002, 0.004, 0.01, 0.02, 0.04])):
        kp = m["knotpos_f32"]
        th = np.concatenate([np.array(m["pvals"][:5]),
                             0.1 + 0.05 * np.arange(len(sp)),
                             -0.03 + 0.02 * np.sin(np.arange(len(op)))]).astype(np.float32)
        c = orc.Counts2(kp, sp, op)
        c.set(th)
        sig, off = np.empty(len(f1)), np.empty(len(f1))
        rc = orc.lib().orc_counts2_sigma_offset(c.h, len(f1), f1, sig, off)
        assert rc == 0
        ms = stats.colourCurve(sp, th[5:5 + len(sp)], f1, 0.0)
        mo = stats.colourCurve(op, th[5 + len(sp):], f1)
        assert np.max(np.abs(ms - sig)) < 1e-12 and np.max(np.abs(mo - off)) < 1e-12


def test_setup_fluxes_and_best_fit_rules():
    from pofd_affine_b200 import stats
    s = stats.setupFluxes(0.002, 0.05, 11)
    assert s.dtype == np.float32 and s[0] == np.float32(0.002)
    assert abs(s[-1] / np.float32(0.05) - 1) < 1e-6
    assert np.allclose(np.diff(np.log(s.astype(float))), np.log(25) / 10, rtol=1e-5)
    lin = stats.setupFluxes(1.0, 2.0, 5, logspace=False)
    assert lin.tolist() == [1.0, 1.25, 1.5, 1.75, 2.0]
    # the first maximum wins, NaN never does unless it is the first entry
    ch = np.arange(12, dtype=np.float32).reshape(3, 2, 2)  # [step][walker][param]
    ll = np.array([[1.0, np.nan], [5.0, 2.0], [5.0, np.nan]])
    r = stats.numberCountsStats(np.concatenate([ch, ch], 2), ll, [0.01, 0.1], nflux=4, thin=1)
    assert r["best_loglike"] == 5.0 and r["best_params"][0] == 4.0
    ll2 = ll.copy()
    ll2[0, 0] = np.nan
    r2 = stats.numberCountsStats(np.concatenate([ch, ch], 2), ll2, [0.01, 0.1], nflux=4, thin=1)
    assert np.isnan(r2["best_loglike"]) and r2["best_params"][0] == 0.0


def test_double_lognormal_stats_on_a_synthetic_chain(golden):
    from pofd_affine_b200 import stats
    m = golden["model2"]
    kp, sp, op = m["knotpos_f32"], m["sigmapos_f32"], m["offsetpos_f32"]
    th0 = np.array(m["pvals"], np.float32)
    rng = np.random.default_rng(9)
    nsteps, nw = 40, 12
    chain = (th0 + rng.normal(0, 0.01, (nsteps, nw, len(th0)))).astype(np.float32)
    logl = -np.sum((chain - th0) ** 2, axis=2)
    r = stats.doubleLogNormalStats(chain, logl, kp, sp, op, nflux=50, thin=2)
    assert r["nsamples"] == nsteps * nw // 2
    b1 = r["band1"]
    truth = np.log10(stats.numberCounts(kp, th0[:5], b1["flux"]))
    assert np.max(np.abs(b1["median"] - truth)) < 0.05
    sg = r["sigma"]
    assert abs(sg["flux"][0] - sp[0]) < 1e-9 and abs(sg["flux"][-1] / sp[-1] - 1) < 1e-6
    assert np.max(np.abs(sg["median"] - stats.colourCurve(sp, th0[5:7], sg["flux"]))) < 0.01
    # one offset knot: the offset curve spans the sigma knots (the range before it)
    assert np.array_equal(r["offset"]["flux"], sg["flux"])
    assert np.allclose(r["offset"]["median"], th0[7], atol=0.01)
    rr = stats.doubleLogNormalStats(chain, logl, kp, sp, op, nflux=50, thin=2, ratios=True)
    s = stats.colourCurve(sp, th0[5:7], sg["flux"])
    want = np.sqrt(np.exp(2 * th0[7] + s * s) * np.expm1(s * s))
    assert np.max(np.abs(rr["sigma"]["median"] / want - 1)) < 0.1
    assert np.allclose(rr["offset"]["median"], np.exp(th0[7] + 0.5 * s * s), rtol=0.02)
    for c in (r["band1"], r["sigma"], r["offset"], rr["sigma"]):
        lo, hi = c["snake"][2, :, 0], c["snake"][2, :, 1]
        assert np.all(lo <= c["median"]) and np.all(c["median"] <= hi)


def test_band_range_rounding_rules():
    """The top of the flux grid: pulled in by 1e-4 of the range in double
    for the 1D model's double knots, then converted to float
    (numberCountsKnotsSplineStats.cc:156-159); in float arithmetic for the
    two-band model's float knots (numberCountsDoubleLogNormalStats.cc:212-214).
    The two rules differ by a float ulp on a good share of knot pairs."""
    from pofd_affine_b200 import stats
    rng = np.random.default_rng(5)
    differ = 0
    for _ in range(2000):
        k = np.sort(rng.uniform(1e-4, 1.0, 2))
        lo1, hi1 = stats._band_range(k, double_knots=True)
        assert lo1 == np.float32(k[0])
        assert hi1 == np.float32(k[1] - 1e-4 * (k[1] - k[0]))
        lo2, hi2 = stats._band_range(k)
        f0, f1 = np.float32(k[0]), np.float32(k[1])
        assert hi2 == np.float32(float(f1) - 1e-4 * float(np.float32(f1 - f0)))
        differ += hi1 != hi2
    assert differ > 0
