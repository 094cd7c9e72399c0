"""Chain output and the pofd_affine_getStats restatement (CPU).

The number counts are pinned to the reference's model test
(model_test.cc:182-192: log10 dN/dS at 0.003, 0.007, 0.015 Jy and at the
interior knots); the accumulator to a direct restatement of
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
