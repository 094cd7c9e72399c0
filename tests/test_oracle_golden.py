"""Pins the CPU oracle to the reference's own golden values
(test/model_test.cc of aconley/pofd_affine 0.5.1, transcribed with their
tolerances in tests/golden/reference_goldens.json)."""
import numpy as np


def _k1(g):
    c = g["counts1"]
    return np.array(c["knotpos_f32"]), np.array(c["knotval"], np.float32)


def test_counts1_at_knots_and_test_points(orc, golden):
    kp, kv = _k1(golden)
    c = golden["counts1"]
    got = np.log10(orc.counts1(kp, kv, kp[1:-1]))
    assert np.allclose(got, kv[1:-1], atol=c["interior_tol"])
    got = np.log10(orc.counts1(kp, kv, c["testpos"]))
    assert np.allclose(got, c["testval_log10"], atol=c["tol"])


def test_counts1_integrals(orc, golden):
    kp, kv = _k1(golden)
    g = golden["integrals1"]
    ns, s1, s2 = orc.integrals1(kp, kv)
    assert abs(ns - g["ns"][0]) < g["ns"][1]
    assert abs(s1 - g["flux_per_area"][0]) < g["flux_per_area"][1]
    assert abs(s2 - g["fluxsq_per_area"][0]) < g["fluxsq_per_area"][1]


def test_rrange1(orc, golden, beams):
    kp, kv = _k1(golden)
    b = orc.Beam1(beams["band1"], float(beams["band1_pixsize"]), 1e-5)
    lo, hi = orc.rrange1(kp, kv, b)
    assert lo == 0.0
    assert abs(hi - golden["rrange1"]["upper"][0]) < golden["rrange1"]["upper"][1]


def test_R1_raw_and_histogrammed(orc, golden, beams):
    kp, kv = _k1(golden)
    r = golden["R1"]
    for nh in (0, 120):
        b = orc.Beam1(beams["band1"], float(beams["band1_pixsize"]), 1e-5, nh)
        if nh:
            assert b.info()["poshist"] == 1
        for scalar in (True, False):
            got = orc.getR1(kp, kv, b, r["flux"], scalar)
            assert np.all(np.abs(got / np.array(r["R"]) - 1) < r["reltol"])
        assert np.all(orc.getR1(kp, kv, b, r["zero_at"], True) == 0.0)


def test_R1_negative_beam(orc, golden, beams):
    kp, kv = _k1(golden)
    r = golden["R1neg"]
    exp = np.array(r["R"])
    for nh in (0, 200):
        b = orc.Beam1(beams["band12_0"], float(beams["band12_0_pixsize"]),
                      1e-5, nh)
        assert b.info()["pixsize"] == 8.0
        assert bool(b.info()["poshist"]) == (nh > 0)
        assert bool(b.info()["neghist"]) == (nh > 0)
        for scalar in (True, False):
            got = orc.getR1(kp, kv, b, r["flux"], scalar)
            rel = np.where(exp > 0, np.abs(got / np.where(exp > 0, exp, 1) - 1),
                           np.abs(got))
            assert np.all(rel < r["tol"]), (nh, scalar, got)


def _model2(orc, g, sigmapos=None, pvals=None):
    m = g["model2"]
    c = orc.Counts2(m["knotpos_f32"], sigmapos or m["sigmapos_f32"],
                    m["offsetpos_f32"])
    c.set(pvals or m["pvals"])
    return c


def test_model2_range_and_maxflux(orc, golden, beams):
    m = golden["model2"]
    c = _model2(orc, golden)
    mf = c.maxflux()
    assert abs(mf[0] - m["maxflux"][0]) < m["maxflux"][1]
    assert abs(mf[1] - m["maxflux"][2]) < m["maxflux"][3]
    b = orc.Beam2(beams["band1"], beams["band2"], 4.0, 1e-6)
    mm = b.minmax(0)
    assert abs(mm[1] - m["beam_max1"][0]) < m["beam_max1"][1]
    assert abs(mm[3] - m["beam_max2"][0]) < m["beam_max2"][1]
    rr = c.rrange(b)
    assert rr[0] == 0.0 and rr[2] == 0.0
    assert abs(rr[1] - m["rrange_upper1"][0]) < m["rrange_upper1"][1]
    assert abs(rr[3] - m["rrange_upper2"][0]) < m["rrange_upper2"][1]


def test_counts2(orc, golden):
    g = golden["counts2"]
    c = _model2(orc, golden)
    got = c.counts(g["f1"], g["f2"])
    assert np.all(np.abs(got / np.array(g["counts"]) - 1) < g["reltol"])


def test_R2_raw_and_histogrammed(orc, golden, beams):
    r = golden["R2"]
    for sp, nh in ((r["sigmapos_f32"], 0),
                   (golden["R2hist"]["sigmapos_f32"], golden["R2hist"]["nhist"])):
        c = _model2(orc, golden, sp, r["pvals"])
        b = orc.Beam2(beams["band1"], beams["band2"], 4.0, 1e-6, nh)
        if nh:
            assert b.info()["ishist"][0]
        got = c.getR_scalar(b, r["f1"], r["f2"])
        assert np.all(np.abs(got / np.array(r["R"]) - 1) < r["reltol"])
        grid = c.getR(b, r["grid_f1"], r["grid_f2"]).ravel()
        assert np.all(np.abs(grid / np.array(r["grid_R"]) - 1) < r["reltol"])


def test_R2_negative_beam(orc, golden, beams):
    r = golden["R2neg"]
    c = _model2(orc, golden, r["sigmapos_f32"], r["pvals"])
    exp = np.array(r["grid_R"])
    for nh in (0, 200):
        b = orc.Beam2(beams["band12_0"], beams["band12_1"], 8.0, 1e-7, nh)
        if nh:
            assert list(b.info()["ishist"]) == r["hist_flags"]
        got = c.getR_scalar(b, r["f1"], r["f2"])
        assert np.all(np.abs(got / np.array(r["R"]) - 1) < r["reltol"])
        for f1, f2 in r["zero_at"]:
            assert c.getR_scalar(b, [f1], [f2])[0] == 0.0
        grid = c.getR(b, r["grid_f1"], r["grid_f2"]).ravel()
        rel = np.where(exp > 0, np.abs(grid / np.where(exp > 0, exp, 1) - 1),
                       np.abs(grid))
        assert np.all(rel < r["reltol"])
