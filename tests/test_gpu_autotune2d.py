"""The 2D launch-shape autotuner: every value of every knob keeps the
oracle's log-likelihood (within 1e-6), and the autotuner picks among the
candidates, reports times, and leaves its choice in place."""
import numpy as np
import pytest

from test_gpu_2d import build2, spec2

pytestmark = pytest.mark.gpu

LL_TOL = 1e-6


def _setup(orc, gpu_ctx):
    s = spec2(n=512, nedge=128, shape=(64, 64))
    O, G = build2(orc, gpu_ctx, s)
    rng = np.random.default_rng(11)
    th = np.repeat(s["th"][None, :], 6, 0)
    th[:, :6] += rng.normal(0, 0.03, (6, 6)).astype(np.float32)
    lo, so = O.loglike_batch(th, 6)
    assert np.all(so == 0)
    return G, th, lo


@pytest.mark.parametrize("knob,values", [("rgrid_rows", [2, 8, 4]),
                                         ("edge_rows", [4, 16, 8]),
                                         ("fft_mode", [0, 1])])
def test_every_2d_knob_value_keeps_parity(orc, gpu_ctx, knob, values):
    G, th, lo = _setup(orc, gpu_ctx)
    for v in values:
        G.setTuning(**{knob: v})
        assert G.getTuning()[knob] == v
        lg, st = G.getLogLikeBatch(th)
        assert np.all(st == 0)
        assert np.max(np.abs(lg - lo)) < LL_TOL, (knob, v)


def test_2d_autotune_picks_from_the_candidates(orc, gpu_ctx):
    G, th, lo = _setup(orc, gpu_ctx)
    r = G.autotune(th, reps=3)
    assert r["fft_mode"] in (0, 1)
    assert r["rgrid_rows"] in (2, 4, 8)
    assert r["edge_rows"] in (4, 8, 16)
    assert 0 < r["ms"] <= r["untuned_ms"]
    assert G.getTuning() == {k: r[k] for k in G.TUNING_KEYS}
    lg, st = G.getLogLikeBatch(th)
    assert np.all(st == 0)
    assert np.max(np.abs(lg - lo)) < LL_TOL
