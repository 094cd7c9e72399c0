"""Data-map ingestion on the GPU (mean subtraction and binning of maps in
device memory) against the host set-up, at the benchmarked map sizes: the
bin counts, bin centres and widths, pixel counts and likelihood offsets are
identical, and so are the log-likelihoods of the two likelihoods, bit for
bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same_info(a, b):
    for k in a:
        if k == "bins":
            assert np.array_equal(a[k], b[k])
        else:
            assert a[k] == b[k], (k, a[k], b[k])


def test_1d_ingestion_matches_host(gpu_ctx):
    import torch
    from pofd_affine_b200 import beam, calcLike, synth
    cfg = synth.config_1d_batched(seed=2)
    hostL = synth.build_like1(cfg, gpu_ctx)
    devL = calcLike(gpu_ctx, cfg["knotpos"], cfg["fftsize"], cfg["ninterp"], True,
                    cfg["nbins"])
    for b in cfg["beams"]:
        devL.addBeamSet(beam(b, cfg["pixsize"], True, cfg["nbeamhist"], 1e-5))
    keep = []
    for m, bi, s in zip(cfg["maps"], cfg["map_beam"], cfg["sigmas"]):
        d = torch.from_numpy(np.ascontiguousarray(m, np.float64).ravel()).cuda()
        devL.addDatasetDevice(bi, d.data_ptr(), d.numel(), s)
        keep.append(d)
    devL.setRRanges(cfg["theta0"])
    for b in range(3):
        _same_info(hostL.datasetInfo(b, 0), devL.datasetInfo(b, 0))
    th = synth.proposals(cfg["theta0"], 8, 0.02, rng=5)
    lh, sh = hostL.getLogLikeBatch(th)
    ld, sd = devL.getLogLikeBatch(th)
    assert list(sh) == list(sd)
    assert np.array_equal(lh, ld)


def test_2d_ingestion_matches_host(gpu_ctx):
    import torch
    from pofd_affine_b200 import synth
    from pofd_affine_b200.api2d import calcLikeDouble, doublebeam
    cfg = synth.config_2d()
    hostL = synth.build_like2(cfg, gpu_ctx)
    devL = calcLikeDouble(gpu_ctx, cfg["knotpos"], cfg["sigmapos"], cfg["offsetpos"],
                          cfg["fftsize"], cfg["nedge"], True, cfg["nbins"])
    devL.addBeamSet(doublebeam(cfg["beam1"], cfg["beam2"], cfg["pixsize"], True,
                               cfg["nbeamhist"], cfg["minval"]))
    (m1, m2), (s1, s2) = cfg["maps"][0], cfg["sigmas"][0]
    d1 = torch.from_numpy(np.ascontiguousarray(m1, np.float64).ravel()).cuda()
    d2 = torch.from_numpy(np.ascontiguousarray(m2, np.float64).ravel()).cuda()
    devL.addDatasetDevice(0, d1.data_ptr(), d2.data_ptr(), d1.numel(), s1, s2)
    devL.setRRanges(cfg["theta0"])
    _same_info(hostL.datasetInfo(0, 0), devL.datasetInfo(0, 0))
    th = np.repeat(cfg["theta0"][None, :], 2, 0)
    lh, sh = hostL.getLogLikeBatch(th)
    ld, sd = devL.getLogLikeBatch(th)
    assert list(sh) == list(sd)
    assert np.array_equal(lh, ld)


def test_standalone_binning_and_its_errors(gpu_ctx):
    import ctypes as C
    import torch
    from pofd_affine_b200._lib import lib
    rng = np.random.default_rng(9)
    x = rng.normal(0.0, 0.003, 100000)
    d = torch.from_numpy(x.copy()).cuda()
    bins = torch.zeros(50, dtype=torch.int32, device="cuda")
    info = np.zeros(3)
    assert lib().pofd_data_bin_device(C.c_void_p(d.data_ptr()), x.size, 1, 50,
                                      C.c_void_p(bins.data_ptr()), info, None) == 0
    # the host rules restated: sequential mean, then the bin index rule
    m = x[0]
    for v in x[1:]:
        m += v
    m /= x.size
    y = x - m
    assert info[0] == m
    assert np.array_equal(d.cpu().numpy(), y)
    lo, hi = y.min(), y.max()
    bd = (hi - lo) / 49
    idx = ((y - lo) * (1.0 / bd) + 0.5).astype(np.uint32)
    assert info[1] == lo and info[2] == bd
    assert np.array_equal(bins.cpu().numpy(), np.bincount(idx, minlength=50))
    assert lib().pofd_data_bin_device(C.c_void_p(d.data_ptr()), x.size, 0, 0,
                                      C.c_void_p(bins.data_ptr()), info, None) < 0
