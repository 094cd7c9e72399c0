"""2D (two-band) CUDA path against the oracle, through the C ABI.

Tolerances: R grid and P(D) within 1e-10 relative to their maxima,
log-likelihood within 1e-6 absolute; split indices and status codes exact.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P_TOL = 1e-10
LL_TOL = 1e-6


def _beam2d(beams, name):
    return beams[name].reshape(tuple(beams[name + "_dims"])[::-1])


def spec2(seed=0, n=256, nedge=64, edge=True, shape=(96, 96), noise=(0.0025,
          0.003), nbins=120, nh=40, beams_pair=None, ps=6.0, minval=1e-6,
          ndata=1, nsig=3, noff=3, bin_data=True):
    """A small two-band fit of the log-normal colour model."""
    from pofd_affine_b200 import synth
    rng = np.random.default_rng(seed)
    kp, kv = synth.knot_model(6, 0.002, 0.4, rng=rng)
    sk = np.logspace(np.log10(0.003), np.log10(0.3), nsig)
    sv = np.linspace(0.15, 0.3, nsig).astype(np.float32)
    ok = np.logspace(np.log10(0.003), np.log10(0.3), noff)
    ov = (np.log(0.7) + rng.normal(0, 0.05, noff)).astype(np.float32)
    if beams_pair is None:
        b1, b2 = synth.gaussian_beam(3.0), synth.gaussian_beam(3.0) ** 0.6
    else:
        b1, b2 = beams_pair
    sfn = lambda f: np.interp(f, sk, sv)  # noqa: E731
    ofn = lambda f: np.interp(f, ok, ov)  # noqa: E731
    maps = [synth.make_map_pair(shape, ps, b1, b2, kp, kv, sfn, ofn,
                                noise[0], noise[1], rng)
            for _ in range(ndata)]
    th = np.concatenate([kv, sv, ov, [1.0, 1.0]]).astype(np.float32)
    return dict(kp=kp, sk=sk, ok=ok, b1=b1, b2=b2, maps=maps, noise=noise,
                th=th, n=n, nedge=nedge, edge=edge, nbins=nbins, nh=nh, ps=ps,
                minval=minval, bin_data=bin_data)


def build2(orc, ctx, s):
    from pofd_affine_b200 import calcLikeDouble, doublebeam
    O = orc.Like2(s["kp"], s["sk"], s["ok"], s["n"], s["nedge"], s["edge"],
                  s["nbins"], s["bin_data"])
    G = calcLikeDouble(ctx, s["kp"], s["sk"], s["ok"], s["n"], s["nedge"],
                       s["edge"], s["nbins"], s["bin_data"])
    O.add_beamset(s["b1"], s["b2"], s["ps"], s["minval"], s["nh"] > 0,
                  s["nh"])
    G.addBeamSet(doublebeam(s["b1"], s["b2"], s["ps"], s["nh"] > 0, s["nh"],
                            s["minval"]))
    for m1, m2 in s["maps"]:
        O.add_dataset(0, m1, m2, *s["noise"])
        G.addDataset(0, m1, m2, *s["noise"])
    O.set_rranges(s["th"])
    G.setRRanges(s["th"])
    return O, G


CASES = {
    "hist": {},
    "raw": dict(nh=0, shape=(48, 48)),
    "neg": "neg",
    "noedge": dict(edge=False),
    "n384": dict(n=384, nedge=96),
    "onesig": dict(nsig=1, noff=1),
    "twosig": dict(nsig=2, noff=2),
}


def _case(beams, name):
    kw = CASES[name]
    if kw == "neg":
        kw = dict(beams_pair=(_beam2d(beams, "band12_0"),
                              _beam2d(beams, "band12_1")), ps=8.0,
                  minval=1e-7, nh=30)
    return spec2(**kw)


@pytest.mark.parametrize("case", list(CASES))
def test_r_grid_and_pd_match_oracle(orc, gpu_ctx, beams, case):
    s = _case(beams, case)
    O, G = build2(orc, gpu_ctx, s)
    po, io, ro = O.pd(0, 0, s["th"], setlog=False, want_r=True)
    rg = G.getR(0, s["th"])
    scale = np.max(np.abs(ro))
    assert np.max(np.abs(rg - ro)) <= 1e-12 * scale
    pg, ig = G.getPD(0, 0, s["th"], setLog=False)
    for k in ("split1", "split2"):
        assert ig[k] == io[k], k
    # moments are sums in another order: last-bit differences only
    for k in ("mn1", "mn2", "var1", "var2", "shift1", "shift2", "sg1pos",
              "sg1neg", "sg2pos", "sg2neg", "pd_minflux1", "pd_minflux2"):
        assert abs(ig[k] - io[k]) <= 1e-10 * max(abs(io[k]), 1e-300), k
    assert np.max(np.abs(pg - po)) <= P_TOL * po.max()
    lg, _ = G.getPD(0, 0, s["th"], setLog=True)
    lo, _ = O.pd(0, 0, s["th"], setlog=True)
    big = po > 1e-6 * po.max()
    assert np.max(np.abs(lg[big] - lo[big])) < 1e-9


@pytest.mark.parametrize("case", ["hist", "neg", "noedge", "multi",
                                  "unbinned", "unbinned_neg"])
def test_loglike_batch_matches_oracle(orc, gpu_ctx, beams, case):
    from pofd_affine_b200 import synth
    if case == "multi":
        s = spec2(ndata=3, shape=(64, 64))
    elif case == "unbinned":
        s = spec2(bin_data=False, shape=(40, 50))
    elif case == "unbinned_neg":
        s = spec2(bin_data=False, shape=(40, 40),
                  beams_pair=(_beam2d(beams, "band12_0"),
                              _beam2d(beams, "band12_1")), ps=8.0,
                  minval=1e-7, nh=30)
    else:
        s = _case(beams, case)
    O, G = build2(orc, gpu_ctx, s)
    th = synth.proposals(s["th"], 10, 0.02, rng=6, fixed_last=False)
    th[:, -2:] = 1.0
    th[3, -2] = 1.05   # band-1 sigma multiplier
    th[4, -1] = 0.97   # band-2 sigma multiplier
    th[6, -1] = -0.5   # negative multiplier -> bad_like
    th[8, 2] = np.nan  # invalid model
    lo, so = O.loglike_batch(th, 4)
    lg, sg = G.getLogLikeBatch(th)
    assert list(sg) == list(so)
    ok = so == 0
    assert np.max(np.abs(lg[ok] - lo[ok])) < LL_TOL
    assert lg[6] == 1e25
    assert np.isnan(lg[8]) and sg[8] == -1
    ll, inv = G.getLogLike(th[0])
    assert not inv and abs(ll - lo[0]) < LL_TOL


def test_two_beam_sets_and_repeat_stability(orc, gpu_ctx, beams):
    from pofd_affine_b200 import calcLikeDouble, doublebeam, synth
    a = spec2(seed=4)
    b = spec2(seed=5, beams_pair=(_beam2d(beams, "band1"),
                                  _beam2d(beams, "band2")), ps=4.0,
              shape=(64, 48))
    O = orc.Like2(a["kp"], a["sk"], a["ok"], 256, 64, True, 100)
    G = calcLikeDouble(gpu_ctx, a["kp"], a["sk"], a["ok"], 256, 64, True, 100)
    for i, s in enumerate((a, b)):
        O.add_beamset(s["b1"], s["b2"], s["ps"], 1e-6, True, 40)
        G.addBeamSet(doublebeam(s["b1"], s["b2"], s["ps"], True, 40, 1e-6))
        for m1, m2 in s["maps"]:
            O.add_dataset(i, m1, m2, *s["noise"])
            G.addDataset(i, m1, m2, *s["noise"])
    O.set_rranges(a["th"])
    G.setRRanges(a["th"])
    th = synth.proposals(a["th"], 9, 0.02, rng=3, fixed_last=False)
    th[:, -2:] = 1.0
    lo, so = O.loglike_batch(th, 4)
    first, sg = G.getLogLikeBatch(th)
    assert list(sg) == list(so)
    assert np.max(np.abs(first - lo)) < LL_TOL
    for _ in range(3):  # eager, capture, replay
        assert np.array_equal(first, G.getLogLikeBatch(th)[0])
    G.getLogLikeBatch(th[:4])
    assert np.array_equal(first, G.getLogLikeBatch(th)[0])


def test_device_pointer_entry_point_2d(orc, gpu_ctx):
    import torch
    from pofd_affine_b200 import synth
    s = spec2(seed=7)
    O, G = build2(orc, gpu_ctx, s)
    th = synth.proposals(s["th"], 6, 0.02, rng=2, fixed_last=False)
    th[:, -2:] = 1.0
    ref, _ = G.getLogLikeBatch(th)
    dth = torch.from_numpy(th).cuda()
    dll = torch.empty(6, dtype=torch.float64, device="cuda")
    dst = torch.empty(6, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    G.getLogLikeDevice(6, dth.data_ptr(), th.shape[1], dll.data_ptr(),
                       dst.data_ptr(), stream)
    torch.cuda.synchronize()
    assert np.array_equal(dll.cpu().numpy(), ref)
    assert np.all(dst.cpu().numpy() == 0)


@pytest.mark.parametrize("edge", [True, False])
def test_pdfactory2_matches_likelihood(orc, gpu_ctx, edge):
    """PDFactoryDouble on the likelihood's own ranges gives the likelihood's
    R grid and P(D), which the oracle's PDFactoryDouble reproduces."""
    from pofd_affine_b200 import PDFactoryDouble, doublebeam
    s = spec2(seed=11, edge=edge)
    O, G = build2(orc, gpu_ctx, s)
    rr = G.getRRange(0)
    F = PDFactoryDouble(gpu_ctx, s["nedge"])
    F.initPD(s["n"], rr[0], rr[1], rr[2], rr[3], s["kp"], s["sk"], s["ok"],
             s["th"][:-2], doublebeam(s["b1"], s["b2"], s["ps"], True, s["nh"],
                                      s["minval"]), edge)
    assert np.array_equal(F.getR(), G.getR(0, s["th"]))
    pf, inf = F.getPD(s["noise"][0], s["noise"][1], setLog=False)
    pg, ig = G.getPD(0, 0, s["th"], setLog=False)
    assert np.max(np.abs(pf - pg)) <= 1e-13 * pg.max()
    assert inf["minflux1"] == ig["pd_minflux1"] and inf["dflux2"] == ig["dflux2"]
    po, io = O.pd(0, 0, s["th"], setlog=False)
    assert np.max(np.abs(pf - po)) <= 1e-10 * po.max()
