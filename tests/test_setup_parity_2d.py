"""Host-side set-up of the 2D product path (doublebeam sign split and
histograms, 2D data binning, likelihood offsets, frozen R ranges including
the Brent maximum-flux solve) against the oracle, bit for bit.  Runs on a
host-only context (no GPU)."""
import numpy as np
import pytest

KNOTS = np.array([0.002, 0.006, 0.02, 0.07, 0.25])
SIGK = np.array([0.004, 0.05])
OFFK = np.array([0.003, 0.03, 0.2])
THETA = np.array([6.4, 5.1, 3.5, 2.0, 0.3, 0.12, 0.25, -0.3, -0.35, -0.2,
                  1.0, 1.0], np.float32)


@pytest.mark.parametrize("n1,n2,minval,nh", [
    ("band1", "band2", 1e-6, 0), ("band1", "band2", 1e-6, 40),
    ("band12_0", "band12_1", 1e-7, 0), ("band12_0", "band12_1", 1e-7, 30),
    ("band12_0", "band12_1", 0.01, 100)])
def test_beam2_info_and_terms_bit_exact(orc, beams, host_ctx, n1, n2, minval,
                                        nh):
    from pofd_affine_b200 import doublebeam
    ps = float(beams[n1 + "_pixsize"])
    ob = orc.Beam2(beams[n1], beams[n2], ps, minval, nh)
    pb = doublebeam(beams[n1], beams[n2], ps, nh > 0, nh, minval)
    oi, pi = ob.info(), pb.info()
    for k in oi:
        assert np.array_equal(oi[k], pi[k]), k


def _pair(orc, host_ctx, beam_pairs, maps, sigmas, nbins=120, n=256,
          nedge=64, exp_conf=(0.0, 0.0), nh=40):
    from pofd_affine_b200 import calcLikeDouble, doublebeam
    O = orc.Like2(KNOTS, SIGK, OFFK, n, nedge, True, nbins)
    P = calcLikeDouble(host_ctx, KNOTS, SIGK, OFFK, n, nedge, True, nbins)
    for (b1, b2, ps, mv) in beam_pairs:
        O.add_beamset(b1, b2, ps, mv, True, nh, exp_conf[0], exp_conf[1])
        P.addBeamSet(doublebeam(b1, b2, ps, True, nh, mv), exp_conf[0],
                     exp_conf[1])
    for (m1, m2, b), (s1, s2) in zip(maps, sigmas):
        O.add_dataset(b, m1, m2, s1, s2, 0.8)
        P.addDataset(b, m1, m2, s1, s2, 0.8)
    O.set_rranges(THETA)
    P.setRRanges(THETA)
    return O, P


def test_binning_offsets_rranges_bit_exact(orc, beams, host_ctx):
    from pofd_affine_b200 import synth
    rng = np.random.default_rng(5)
    g1, g2 = synth.gaussian_beam(3.0), synth.gaussian_beam(3.0, 9.0 * 1.0)
    bp = [(g1, g2 * 0.9, 6.0, 1e-6),
          (beams["band12_0"], beams["band12_1"], 8.0, 1e-7)]
    maps = [(rng.normal(0, 0.003, (40, 50)), rng.normal(0, 0.004, (40, 50)), 0),
            (rng.normal(0, 0.002, 1999), rng.normal(0, 0.0025, 1999), 0),
            (rng.normal(0, 0.004, (30, 30)) + 0.02 * rng.random((30, 30)) ** 6,
             rng.normal(0, 0.003, (30, 30)), 1)]
    O, P = _pair(orc, host_ctx, bp, maps, [(0.003, 0.004), (0.002, 0.0025),
                                          (0.004, 0.003)],
                 exp_conf=(0.001, 0.0015))
    for bs, nds in ((0, 2), (1, 1)):
        assert np.array_equal(O.rrange(bs), P.getRRange(bs)), bs
        for ds in range(nds):
            oi = O.dataset_info(bs, ds)
            pi = P.datasetInfo(bs, ds)
            for k in oi:
                assert oi[k] == pi[k], (bs, ds, k)
            assert np.array_equal(O.dataset_bins(bs, ds), pi["bins"])
    # the beam pair with negative parts gives a range below zero in both bands
    r = P.getRRange(1)
    assert r[0] < 0 and r[2] < 0


def test_rrange_uses_brent_maxflux(orc, host_ctx):
    """The band-2 upper range comes from the maximum of exp(offset + 3
    sigma)-style colour extent found by Brent's method on the knot range; a
    change of the offset curve must move it identically in both."""
    from pofd_affine_b200 import synth
    g = synth.gaussian_beam(3.0)
    rng = np.random.default_rng(8)
    m = (rng.normal(0, 0.003, 900), rng.normal(0, 0.003, 900), 0)
    O, P = _pair(orc, host_ctx, [(g, g, 6.0, 1e-6)], [m], [(0.003, 0.003)])
    th2 = THETA.copy()
    th2[7:10] = [0.2, -0.1, 0.4]
    O.set_rranges(th2)
    P.setRRanges(th2)
    assert np.array_equal(O.rrange(0), P.getRRange(0))


def test_unbinned_ranges_and_info(orc, host_ctx):
    """Unbinned data: no bins, R ranges from the raw data extremes."""
    from pofd_affine_b200 import calcLikeDouble, doublebeam, synth
    g = synth.gaussian_beam(3.0)
    rng = np.random.default_rng(9)
    m1 = rng.normal(0, 0.003, 700) + 0.05 * rng.random(700) ** 9
    m2 = rng.normal(0, 0.004, 700)
    O = orc.Like2(KNOTS, SIGK, OFFK, 256, 64, True, 50, False)
    P = calcLikeDouble(host_ctx, KNOTS, SIGK, OFFK, 256, 64, True, 50, False)
    O.add_beamset(g, g, 6.0, 1e-6, True, 40)
    P.addBeamSet(doublebeam(g, g, 6.0, True, 40, 1e-6))
    O.add_dataset(0, m1, m2, 0.003, 0.004)
    P.addDataset(0, m1, m2, 0.003, 0.004)
    O.set_rranges(THETA)
    P.setRRanges(THETA)
    assert np.array_equal(O.rrange(0), P.getRRange(0))
    oi, pi = O.dataset_info(0, 0), P.datasetInfo(0, 0)
    for k in oi:
        assert oi[k] == pi[k], k
    assert pi["nbins"] == 0 and pi["bins"].size == 0


def test_invalid_configurations_rejected(host_ctx):
    from pofd_affine_b200 import PofdError, calcLikeDouble
    with pytest.raises(PofdError):
        calcLikeDouble(host_ctx, KNOTS, SIGK, OFFK, 8, 4)  # below 16
    with pytest.raises(PofdError):
        calcLikeDouble(host_ctx, KNOTS[:1], SIGK, OFFK, 256, 16)
    L = calcLikeDouble(host_ctx, KNOTS, SIGK, OFFK, 256, 16, True, 50)
    with pytest.raises(PofdError):
        L.addDataset(0, np.zeros(10), np.zeros(10), 0.1, 0.1)  # no beam set
