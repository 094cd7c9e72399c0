"""The allocation-free entry point pofd_pd1_loglike_noalloc, through the C
ABI, against the regular entry point pofd_like1_eval_batch.

The no-alloc entry point serves callers that cannot allocate GPU memory when
they evaluate (device memory owned by another allocator, or no tolerance for
the synchronisation cudaMalloc/cudaFree imply).  It takes a wrapped P(D)
(the inverse-FFT output) in caller-owned device memory and returns the
dataset's log-likelihood term; here that P(D) is formed from the oracle's R
grid with numpy's FFT, and the result must equal the regular entry point's
log-likelihood for the same proposal within the parity tolerance, on two
calls in a row (the shared static scratch keeps the previous call's
contents).  This file is collected last so that a stop-at-first-failure run
has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LL_TOL = 1e-6


def _wrapped_pd(rv, info, sigma):
    """PDFactory::initPD/getPD up to the inverse FFT (PDFactory.cc:1094-1199)
    from an R grid, with numpy's FFT."""
    n = rv.size
    dflux = info["dflux"]
    shift = info["shift"] if info["doshift"] else 0.0
    rt = np.fft.rfft(rv)
    k = np.arange(rt.size)
    iflux = 2 * np.pi / (n * dflux)
    p = np.exp(rt.real - rt[0].real) * np.exp(1j * (rt.imag - shift * iflux * k))
    p[0] = 1.0
    p = p * np.exp(-0.5 * sigma * sigma * (iflux * k) ** 2)
    p[0] = 1.0
    return np.fft.irfft(p, n) * n


def _jitter_branch(raw, info, sigma):
    """True when the reference's split search (PDFactory.cc:756-921) finds
    no monotonic descent before the minimum and takes its jitter-estimate
    branch on this wrapped P(D)."""
    dflux = info["dflux"]
    sgpos = np.sqrt(info["var_noi"] + sigma * sigma)
    sgneg = sigma if 9 * sigma * sigma > info["var_noi"] else sgpos
    bot = int(2.5 * sgpos / dflux)
    mfr, wr = info["minflux_R"], int(info["wrapRidx"])
    top = wr if 2.5 * sgpos > abs(mfr) else int(-(2.5 * sgneg + mfr) / dflux
                                                 + wr + 1)
    p = np.where(raw > 0, raw, 0.0)
    mi = bot + int(np.argmin(p[bot:top + 1]))
    return mi > 17 and not np.all(np.diff(p[mi - 17:mi + 1]) < 0)


# (knots, knot range, FWHM px, beam histogram bins, noise, map, n, nodes,
# data bins): a noise-dominated P(D) whose split is the first minimum, and
# the 65536-point P(D) of the batched workload's first beam set, which
# reaches the rounding floor and takes the jitter branch
CASES = {
    "monotone": (6, 0.002, 0.4, 3.0, 120, 0.002, (128, 128), 8192, 512, 500),
    "jitter": (10, 0.001, 0.8, 3.0, 150, 0.002, (400, 400), 65536, 2048, 1000),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_matches_regular_entry_point(orc, gpu_ctx, case):
    import torch
    from pofd_affine_b200 import beam, calcLike, synth
    from pofd_affine_b200._lib import lib

    nk, smin, smax, fwhm, nh, sigma, shape, n, ni, nb = CASES[case]
    rng = np.random.default_rng(21)
    kp, kv = synth.knot_model(nk, smin, smax, rng=rng)
    bm = synth.gaussian_beam(fwhm)
    img = synth.make_map(shape, 6.0, bm, kp, kv, sigma, rng)
    th = np.concatenate([kv, [1.0]]).astype(np.float32)

    G = calcLike(gpu_ctx, kp, n, ni, True, nb)
    G.addBeamSet(beam(bm, 6.0, True, nh))
    G.addDataset(0, img, sigma)
    G.setRRanges(th)
    ref, st = G.getLogLikeBatch(th[None, :])
    assert st[0] == 0

    O = orc.Like1(kp, n, ni, True, nb)
    O.add_beamset(bm, 6.0, 1e-5, True, nh)
    O.add_dataset(0, img, sigma)
    O.set_rranges(th)
    _, info, rv = O.pd(0, 0, th, setlog=False, want_r=True)
    raw = _wrapped_pd(rv, info, sigma)
    assert _jitter_branch(raw, info, sigma) == (case == "jitter")

    di = G.datasetInfo(0, 0)
    nz = np.nonzero(di["bins"])[0]
    d_pd = torch.from_numpy(raw).cuda()
    d_idx = torch.from_numpy(nz.astype(np.int32)).cuda()
    d_cnt = torch.from_numpy(di["bins"][nz].astype(np.float64)).cuda()
    d_out = torch.zeros(3, dtype=torch.float64, device="cuda")
    d_st = torch.full((1,), 99, dtype=torch.int32, device="cuda")

    outs = []
    for _ in range(2):
        rc = lib().pofd_pd1_loglike_noalloc(
            C.c_void_p(d_pd.data_ptr()), n, info["dflux"], info["minflux_R"],
            int(info["wrapRidx"]), info["var_noi"], sigma,
            C.c_void_p(d_idx.data_ptr()), C.c_void_p(d_cnt.data_ptr()),
            int(nz.size), di["bincent0"], di["bindelta"], di["like_offset"],
            di["like_norm"], C.c_void_p(d_out.data_ptr()),
            C.c_void_p(d_st.data_ptr()), None)
        assert rc == 0
        torch.cuda.synchronize()
        assert int(d_st.item()) == 0
        out = d_out.cpu().numpy().copy()
        assert abs(out[0] - ref[0]) < LL_TOL, (out[0], ref[0])
        assert int(out[1]) == int(info["splitidx"])
        outs.append(out)
    assert np.array_equal(outs[0], outs[1])


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu_ctx):
    from pofd_affine_b200._lib import lib
    dummy = C.c_void_p(1)
    rc = lib().pofd_pd1_loglike_noalloc(dummy, 262144 + 1, 1e-5, 0.0, 1000,
                                        1e-6, 1e-3, dummy, dummy, 1, 0.0, 1.0,
                                        0.0, 1.0, dummy, dummy, None)
    assert rc == -10
    assert b"262144" in lib().pofd_last_error()
