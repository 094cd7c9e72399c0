"""The 1D likelihood at the exact shapes that are benchmarked, against the
oracle, through the C ABI.

* the batched workload the throughput line is measured on: 10 knots over
  1-800 mJy, three beam sets (FWHM 3.0 / 4.2 / 6.0 px, 150-bin beam
  histograms), full-size maps 2000x2000 @ 2.0 mJy, 1200x900 @ 3.1 mJy and
  600x600 @ 5.0 mJy, n = 65536, 2048 interpolation nodes, 1000 data bins,
  built exactly as the benchmark builds it, 16 proposals of which four carry
  a sigma multiplier other than 1;
* the plain fit the MCMC comparison runs: 6 knots, one 256x256 map,
  n = 4096, 2048 nodes, 1000 bins;
* the same fit with the counts raised a hundredfold, so that confusion
  dominates the noise and the split search takes its jitter branch.

Tolerances (the parity bar): log-likelihood within 1e-6 absolute, P(D)
within 1e-10 of its peak, statuses identical.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LL_TOL = 1e-6
P_TOL = 1e-10


def _oracle(orc, cfg):
    O = orc.Like1(cfg["knotpos"], cfg["fftsize"], cfg["ninterp"], True,
                  cfg["nbins"])
    for b in cfg["beams"]:
        O.add_beamset(b, cfg["pixsize"], 1e-5, True, cfg["nbeamhist"])
    for m, bi, s in zip(cfg["maps"], cfg["map_beam"], cfg["sigmas"]):
        O.add_dataset(bi, m, s)
    O.set_rranges(cfg["theta0"])
    return O


def _compare(orc, gpu_ctx, cfg, nprop, seed, sigmult_rows=()):
    from pofd_affine_b200 import synth
    G = synth.build_like1(cfg, gpu_ctx)
    O = _oracle(orc, cfg)
    th = synth.proposals(cfg["theta0"], nprop, 0.02, rng=seed)
    for k, v in sigmult_rows:
        th[k, -1] = v
    lg, sg = G.getLogLikeBatch(th)
    lo, so = O.loglike_batch(th, min(nprop, os.cpu_count() or 1))
    assert list(sg) == list(so)
    ok = sg == 0
    assert ok.sum() >= nprop - 1
    err = float(np.max(np.abs(lg[ok] - lo[ok])))
    assert err < LL_TOL, err
    # P(D) of every beam set for one proposal with a sigma multiplier.  Where
    # the split search takes its jitter branch (the P(D) tail reaches the
    # transform's rounding floor, as at n = 65536), the first bin below the
    # jitter estimate is set by rounding noise and can differ between any
    # two FFTs; the unwrapped arrays are then the same wrapped P(D) rotated
    # differently, and the bins between the two splits are at the noise
    # floor (the log-likelihood above is unaffected).
    k = sigmult_rows[0][0] if sigmult_rows else 0
    for b in range(len(cfg["beams"])):
        pg, ig = G.getPD(b, 0, th[k], setLog=False)
        po, io = O.pd(b, 0, th[k], setlog=False)
        ds = int(ig["splitidx"]) - int(io["splitidx"])
        if ds:
            assert abs(ds) < 0.01 * pg.size
            tail = pg[-ds:] if ds > 0 else pg[:-ds]
            assert np.max(tail) < 1e-9 * pg.max()
        assert np.max(np.abs(np.roll(po, -ds) - pg)) <= P_TOL * po.max()
    return err


def test_batched_workload_full_size(orc, gpu_ctx):
    from pofd_affine_b200 import synth
    cfg = synth.config_1d_batched(seed=2)
    err = _compare(orc, gpu_ctx, cfg, 16, 4242,
                   sigmult_rows=((3, 0.9), (7, 1.1), (11, 0.95), (15, 1.2)))
    print("1D batched workload, full size: max |dlogL| = %.3g" % err)


def test_plain_fit_exact_shape(orc, gpu_ctx):
    from pofd_affine_b200 import synth
    cfg = synth.config_1d_small(seed=1)
    assert (cfg["fftsize"], cfg["ninterp"], cfg["nbins"]) == (4096, 2048, 1000)
    assert cfg["maps"][0].shape == (256, 256)
    err = _compare(orc, gpu_ctx, cfg, 16, 77, sigmult_rows=((5, 1.1),))
    print("1D plain fit: max |dlogL| = %.3g" % err)


def test_plain_fit_confusion_dominated(orc, gpu_ctx):
    from pofd_affine_b200 import synth
    cfg = synth.config_1d_small(seed=1, norm_scale=100.0)
    err = _compare(orc, gpu_ctx, cfg, 16, 78, sigmult_rows=((2, 0.9),))
    print("1D confusion-dominated fit: max |dlogL| = %.3g" % err)
