"""The launch-shape autotuner of the 1D engine: every knob value it may
pick gives the oracle's log-likelihood (within the 1e-6 parity tolerance),
and autotune() returns a choice from the candidate sets with a measured
time."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LL_TOL = 1e-6


def _setup(orc, ctx, n=8192):
    from pofd_affine_b200 import beam, calcLike, synth
    cfg = synth.config_1d_batched(seed=2, scale=0.1)
    L = calcLike(ctx, cfg["knotpos"], n, 1024, True, 500)
    O = orc.Like1(cfg["knotpos"], n, 1024, True, 500)
    for b in cfg["beams"]:
        L.addBeamSet(beam(b, 6.0, True, 150))
        O.add_beamset(b, 6.0, 1e-5, True, 150)
    for m, bi, s in zip(cfg["maps"], cfg["map_beam"], cfg["sigmas"]):
        L.addDataset(bi, m, s)
        O.add_dataset(bi, m, s)
    L.setRRanges(cfg["theta0"])
    O.set_rranges(cfg["theta0"])
    th = synth.proposals(cfg["theta0"], 12, 0.03, rng=7)
    return L, O, th


@pytest.mark.parametrize("knob,values", [("rfill_per", [4, 8, 16]),
                                         ("rnodes_threads", [64, 128, 256]),
                                         ("spec_blocks", [1, 2, 32]),
                                         ("own_fft", [0, 1]),
                                         ("rfill_mode", [0, 1, 2, 3])])
def test_every_knob_value_keeps_parity(orc, gpu_ctx, knob, values):
    L, O, th = _setup(orc, gpu_ctx)
    lo, _ = O.loglike_batch(th, 4)
    for v in values:
        L.setTuning(**{knob: v})
        assert L.getTuning()[knob] == v
        lg, st = L.getLogLikeBatch(th)
        assert np.all(st == 0)
        assert np.max(np.abs(lg - lo)) < LL_TOL, (knob, v)


def test_autotune_picks_from_the_candidates(orc, gpu_ctx):
    L, O, th = _setup(orc, gpu_ctx)
    before, _ = L.getLogLikeBatch(th)
    r = L.autotune(th, reps=5)
    assert r["rfill_per"] in (4, 8, 16)
    assert r["rnodes_threads"] in (64, 128, 256)
    assert r["spec_blocks"] in (1, 2, 4, 8, 16, 32)
    assert r["own_fft"] in (0, 1)
    assert r["rfill_mode"] in (0, 1, 2, 3)
    assert 0 < r["ms"] <= r["untuned_ms"]
    assert L.getTuning() == {k: r[k] for k in L.TUNING_KEYS}
    after, st = L.getLogLikeBatch(th)
    assert np.all(st == 0)
    assert np.max(np.abs(after - before)) < 1e-7
    lo, _ = O.loglike_batch(th, 4)
    assert np.max(np.abs(after - lo)) < LL_TOL
