"""Host-side set-up of the product library (beam selection and histogram,
data binning, likelihood offsets, frozen R ranges) against the oracle,
bit for bit.  Runs on a host-only context (no GPU)."""
import numpy as np
import pytest


@pytest.mark.parametrize("name,minval,nh", [
    ("band1", 1e-5, 0), ("band1", 1e-5, 120), ("band12_0", 1e-5, 0),
    ("band12_0", 1e-5, 200), ("band12_0", 0.02, 200), ("band2", 0.0, 50)])
def test_beam_terms_bit_exact(orc, beams, host_ctx, name, minval, nh):
    from pofd_affine_b200 import beam
    pix = beams[name]
    ps = float(beams[name + "_pixsize"])
    ob = orc.Beam1(pix, ps, minval, nh)
    pb = beam(pix, ps, nh > 0, nh, minval)
    oi, pi = ob.info(), pb.info()
    for k in oi:
        if np.isnan(oi[k]):
            assert np.isnan(pi[k]), k
        else:
            assert oi[k] == pi[k], k
    for neg in (False, True):
        w, ie = pb.terms(neg)
        if oi["poshist"]:
            ow = ob.array(2 if neg else 0)
            oie = ob.array(3 if neg else 1)
        else:
            oie = ob.array(5 if neg else 4)
            ow = np.ones_like(oie)
        assert np.array_equal(w, ow) and np.array_equal(ie, oie)


def _pair(orc, host_ctx, maps, beam_pix, sigmas, nbins=300, exp_conf=0.0,
          ps=6.0, nh=120, bin_data=True):
    from pofd_affine_b200 import beam, calcLike
    knots = np.array([0.002, 0.005, 0.02, 0.08, 0.3])
    th = np.array([6.5, 5.2, 3.4, 1.9, 0.1, 1.0], np.float32)
    O = orc.Like1(knots, 2048, 256, bin_data, nbins)
    P = calcLike(host_ctx, knots, 2048, 256, bin_data, nbins)
    for bp in beam_pix:
        O.add_beamset(bp, ps, 1e-5, True, nh, exp_conf)
        P.addBeamSet(beam(bp, ps, True, nh, 1e-5), exp_conf)
    for (m, b), s in zip(maps, sigmas):
        O.add_dataset(b, m, s, 1.3)
        P.addDataset(b, m, s, 1.3)
    O.set_rranges(th)
    P.setRRanges(th)
    return O, P


def test_binning_offsets_rranges_bit_exact(orc, beams, host_ctx):
    from pofd_affine_b200 import synth
    rng = np.random.default_rng(11)
    b0 = synth.gaussian_beam(3.0)
    b1 = beams["band12_0"]  # has a negative part
    maps = [(rng.normal(0, 0.003, (64, 80)) + 0.01 * rng.random((64, 80)) ** 8, 0),
            (rng.normal(0, 0.002, 3001), 0),
            (rng.normal(0, 0.004, (50, 50)), 1)]
    O, P = _pair(orc, host_ctx, maps, [b0, b1], [0.003, 0.002, 0.004],
                 exp_conf=0.0011)
    for bs, nds in ((0, 2), (1, 1)):
        assert np.array_equal(O.rrange(bs), P.getRRange(bs))
        for ds in range(nds):
            oi = O.dataset_info(bs, ds)
            pi = P.datasetInfo(bs, ds)
            for k in oi:
                assert oi[k] == pi[k], (bs, ds, k)
            assert np.array_equal(O.dataset_bins(bs, ds), pi["bins"])
    # the negative beam's range covers the data minimum
    assert P.getRRange(1)[0] < 0


def test_unbinned_and_single_bin(orc, host_ctx):
    from pofd_affine_b200 import synth
    b0 = synth.gaussian_beam(4.2)
    rng = np.random.default_rng(2)
    maps = [(rng.normal(0, 0.003, 500), 0)]
    O, P = _pair(orc, host_ctx, maps, [b0], [0.003], nbins=1)
    assert np.array_equal(O.dataset_bins(0, 0), P.datasetInfo(0, 0)["bins"])
    O, P = _pair(orc, host_ctx, maps, [b0], [0.003], bin_data=False)
    assert np.array_equal(O.rrange(0), P.getRRange(0))
