"""The library's own FP64 four-step FFT path of the 1D likelihood against
the cuFFT path on the same engine: R spectrum, P(D) and log-likelihood
agree to rounding at every supported size, and the own path is the one in
use by default."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [4096, 8192, 16384, 32768, 65536, 131072])
def test_own_fft_matches_cufft(orc, gpu_ctx, n):
    from pofd_affine_b200 import beam, calcLike, synth
    cfg = synth.config_1d_batched(seed=2, scale=0.1)
    L = calcLike(gpu_ctx, cfg["knotpos"], n, 1024, True, 500)
    for b in cfg["beams"]:
        L.addBeamSet(beam(b, 6.0, True, 150))
    for m, bi, s in zip(cfg["maps"], cfg["map_beam"], cfg["sigmas"]):
        L.addDataset(bi, m, s)
    L.setRRanges(cfg["theta0"])
    th = synth.proposals(cfg["theta0"], 9, 0.03, rng=n)
    th[4, -1] = 1.1
    L.setFFT(0)  # the own FFT (by default only from n = 8192)
    assert L.ownFFT()
    lo, so = L.getLogLikeBatch(th)
    po, io = L.getPD(1, 0, th[0], setLog=False)
    L.setFFT(1)
    assert not L.ownFFT()
    lc, sc = L.getLogLikeBatch(th)
    pc, ic = L.getPD(1, 0, th[0], setLog=False)
    L.setFFT(0)
    assert list(so) == list(sc)
    ok = so == 0
    assert np.max(np.abs(lo[ok] - lc[ok])) < 1e-7
    # the default R grid fill (running products over runs of one node
    # interval, inside the forward pass A) against the others -- one exp2
    # per point materialised or inside the forward pass A, the runs
    # materialised: values within ~1e-13 relative, moments grouped
    # differently
    d0 = L.getTuning()["rfill_mode"]
    assert d0 == 3
    for rf in (0, 1, 2):
        L.setTuning(rfill_mode=rf)
        lu, su = L.getLogLikeBatch(th)
        pu, iu = L.getPD(1, 0, th[0], setLog=False)
        assert list(su) == list(so)
        assert np.max(np.abs(lu[ok] - lo[ok])) < 1e-7
        du = int(io["splitidx"] - iu["splitidx"])
        assert np.max(np.abs(np.roll(po, du) - pu)) <= 1e-10 * pu.max()
    L.setTuning(rfill_mode=d0)
    # where the P(D) tail lies at the transform's rounding floor (large n),
    # the first bin below the reference's split threshold is set by rounding
    # and can differ between any two FFTs; the unwrapped arrays are then the
    # same wrapped P(D) rotated differently, with equal log-likelihoods
    ds = int(io["splitidx"] - ic["splitidx"])
    assert np.max(np.abs(np.roll(po, ds) - pc)) <= 1e-12 * pc.max()
    if ds:
        tail = np.roll(po, ds)[:abs(ds)] if ds > 0 else np.roll(po, ds)[ds:]
        assert np.max(tail) < 1e-9 * pc.max()
    # and the oracle, on one proposal
    O = orc.Like1(cfg["knotpos"], n, 1024, True, 500)
    for b in cfg["beams"]:
        O.add_beamset(b, 6.0, 1e-5, True, 150)
    for m, bi, s in zip(cfg["maps"], cfg["map_beam"], cfg["sigmas"]):
        O.add_dataset(bi, m, s)
    O.set_rranges(cfg["theta0"])
    ol, ost = O.loglike_batch(th[:3], 3)
    assert np.max(np.abs(ol - lo[:3])) < 1e-6


def test_own_fft_not_used_for_other_sizes(gpu_ctx):
    from pofd_affine_b200 import beam, calcLike, synth
    cfg = synth.config_1d_small(seed=1)
    for n in (2048, 3000, 262144):
        L = calcLike(gpu_ctx, cfg["knotpos"], n, 512, True, 300)
        L.addBeamSet(beam(cfg["beams"][0], 6.0, True, 120))
        L.addDataset(0, cfg["maps"][0], 0.0025)
        L.setRRanges(cfg["theta0"])
        assert not L.ownFFT()
    # n = 4096: cuFFT by default (the faster one there), the own FFT on request
    L = calcLike(gpu_ctx, cfg["knotpos"], 4096, 512, True, 300)
    L.addBeamSet(beam(cfg["beams"][0], 6.0, True, 120))
    L.addDataset(0, cfg["maps"][0], 0.0025)
    L.setRRanges(cfg["theta0"])
    assert not L.ownFFT() and L.getTuning()["own_fft"] == 0
    L.setFFT(0)
    assert L.ownFFT() and L.getTuning()["own_fft"] == 1
