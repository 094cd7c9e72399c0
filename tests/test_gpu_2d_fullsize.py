"""The 2D likelihood at the full sizes that are benchmarked, against the
oracle, through the C ABI.

* the 2D plain workload: a 1500 x 1500 map pair, 500 x 500 data bins, an
  n = 2048 grid with 256 edge points;
* the second field of the two-field fit: an 800 x 600 pair on an n = 1024
  grid with 128 edge points.

The reference normalises the P(D) and takes its means with one sequential
sum each over the n^2 cells (PDDouble.cc:142-208, 355-447).  That chain's
rounding (a few 1e-12 relative at n = 2048) moves a log-likelihood summed
over 2.25 M pixels by ~1e-5.  The library's default tree sums are exact to
~1e-16, so by default it differs from the reference (and the oracle, which
follows the reference's order) by that rounding.  With the reference-order
mode on (setReferenceSums) the library sums in the reference's own order
and the log-likelihood must agree within the parity bar of 1e-6.  The
default mode is checked against the oracle's P(D) renormalised with exact
sums, to the same 1e-6.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LL_TOL = 1e-6
P_TOL = 1e-10


def _exact_trap(p):
    w1 = np.ones(p.shape[0])
    w1[0] = w1[-1] = 0.5
    w2 = np.ones(p.shape[1])
    w2[0] = w2[-1] = 0.5
    W = np.outer(w1, w2) * p
    a = np.arange(p.shape[0], dtype=np.float64)
    b = np.arange(p.shape[1], dtype=np.float64)
    return (math.fsum(W.ravel()), math.fsum((W * a[:, None]).ravel()),
            math.fsum((W * b[None, :]).ravel()))


def _oracle(orc, cfg):
    O = orc.Like2(cfg["knotpos"], cfg["sigmapos"], cfg["offsetpos"],
                  cfg["fftsize"], cfg["nedge"], True, cfg["nbins"])
    O.add_beamset(cfg["beam1"], cfg["beam2"], cfg["pixsize"], cfg["minval"],
                  True, cfg["nbeamhist"])
    for (m1, m2), (s1, s2) in zip(cfg["maps"], cfg["sigmas"]):
        O.add_dataset(0, m1, m2, s1, s2)
    O.set_rranges(cfg["theta0"])
    return O


def _proposals(cfg, nprop, seed):
    from pofd_affine_b200 import synth
    th = synth.proposals(cfg["theta0"], nprop, 0.01, rng=seed,
                         fixed_last=False)
    th[:, -2:] = 1.0
    th[0] = cfg["theta0"]
    if nprop > 2:
        th[2, -2:] = (1.05, 0.95)  # sigma multipliers other than 1
    return th


def _check(orc, gpu_ctx, cfg, nprop, seed):
    from pofd_affine_b200 import synth
    G = synth.build_like2(cfg, gpu_ctx)
    O = _oracle(orc, cfg)
    th = _proposals(cfg, nprop, seed)
    lo, so = O.loglike_batch(th, nprop)
    assert np.all(so == 0), so
    # default (tree sums)
    lg, sg = G.getLogLikeBatch(th)
    assert np.all(sg == 0), sg
    # the reference's summation order
    G.setReferenceSums(True)
    lr, sr = G.getLogLikeBatch(th)
    assert np.all(sr == 0), sr
    err_ref = float(np.max(np.abs(lr - lo)))
    assert err_ref < LL_TOL, (lr, lo)
    # P(D) and split indices of the central proposal, both modes
    po, io = O.pd(0, 0, th[0], setlog=False)
    pr, ir = G.getPD(0, 0, th[0], setLog=False)
    assert ir["split1"] == io["split1"] and ir["split2"] == io["split2"]
    assert np.max(np.abs(pr - po)) <= P_TOL * po.max()
    G.setReferenceSums(False)
    pg, ig = G.getPD(0, 0, th[0], setLog=False)
    assert ig["split1"] == io["split1"] and ig["split2"] == io["split2"]
    assert np.max(np.abs(pg - po)) <= P_TOL * po.max()

    # the default mode against the oracle's P(D) normalised with exact sums
    info = O.dataset_info(0, 0)
    bins = O.dataset_bins(0, 0)
    d1, d2 = io["dflux1"], io["dflux2"]

    def ll(p, mf1, mf2):
        raw = orc.loglike_binned2(p, mf1, mf2, d1, d2, bins, info["bincent01"],
                                  info["bincent02"], info["bindelta1"],
                                  info["bindelta2"])
        return (raw - info["like_offset"]) / info["like_norm"]

    # the vectorised gather restates the oracle's own
    assert abs(ll(po, io["pd_minflux1"], io["pd_minflux2"]) - lo[0]) < LL_TOL
    tot, s1, s2 = _exact_trap(po)
    norm_err = tot * d1 * d2 - 1.0
    pn = po / (tot * d1 * d2)
    assert abs(ll(pn, -s1 / tot * d1, -s2 / tot * d2) - lg[0]) < LL_TOL
    assert abs(norm_err) < 1e-10
    return err_ref, float(np.max(np.abs(lg - lo)))


def test_full_size_2d_parity(orc, gpu_ctx):
    from pofd_affine_b200 import synth
    cfg = synth.config_2d()
    e_ref, e_tree = _check(orc, gpu_ctx, cfg, 3, 31)
    print("2D n=2048, 1500^2 maps: |dlogL| reference-order sums %.3g, "
          "tree sums %.3g" % (e_ref, e_tree))


def test_two_field_second_field_full_size(orc, gpu_ctx):
    from pofd_affine_b200 import synth
    _, cfg = synth.config_2d_two_fields()
    assert cfg["fftsize"] == 1024 and cfg["maps"][0][0].shape == (800, 600)
    e_ref, e_tree = _check(orc, gpu_ctx, cfg, 3, 32)
    print("2D n=1024, 800x600 maps: |dlogL| reference-order sums %.3g, "
          "tree sums %.3g" % (e_ref, e_tree))
