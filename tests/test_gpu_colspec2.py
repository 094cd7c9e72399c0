"""The 2D likelihood's fused column path (FFT mode 1: batched 1D row
transforms around the library's column-transform + spectrum kernel) against
the 2D-transform path (mode 0) on the same engine and against the oracle.

Tolerances: P(D) within 1e-10 of its maximum, log-likelihood within 1e-6
absolute against the oracle and 1e-7 between the two GPU paths; split
indices and status codes exact.
"""
import numpy as np
import pytest

from test_gpu_2d import build2, spec2

pytestmark = pytest.mark.gpu

P_TOL = 1e-10
LL_TOL = 1e-6


def _batch(s, nprop=5, seed=3):
    rng = np.random.default_rng(seed)
    th = np.repeat(s["th"][None, :], nprop, 0)
    th[:, :6] += rng.normal(0, 0.03, (nprop, 6)).astype(np.float32)
    th[:, -2:] = rng.uniform(0.95, 1.05, (nprop, 2)).astype(np.float32)
    return th


@pytest.mark.parametrize("n,nedge", [(512, 128), (1024, 128), (2048, 256)])
def test_fused_columns_match_2d_path_and_oracle(orc, gpu_ctx, n, nedge):
    s = spec2(n=n, nedge=nedge, shape=(64, 64))
    O, G = build2(orc, gpu_ctx, s)
    th = _batch(s)
    assert G.fusedColumns()
    lf, sf = G.getLogLikeBatch(th)
    pf, inf = G.getPD(0, 0, th[0], setLog=False)
    G.setFFT(0)
    assert not G.fusedColumns()
    l0, s0 = G.getLogLikeBatch(th)
    p0, in0 = G.getPD(0, 0, th[0], setLog=False)
    G.setFFT(1)
    assert G.fusedColumns()
    assert list(sf) == list(s0)
    ok = sf == 0
    assert ok.any()
    assert np.max(np.abs(lf[ok] - l0[ok])) < 1e-7
    assert (inf["split1"], inf["split2"]) == (in0["split1"], in0["split2"])
    assert np.max(np.abs(pf - p0)) <= P_TOL * p0.max()
    # and the oracle on two proposals
    lo, so = O.loglike_batch(th[:2], 2)
    assert list(so) == list(sf[:2])
    assert np.max(np.abs(lo - lf[:2])) < LL_TOL


def test_fused_columns_several_datasets_and_no_noise(orc, gpu_ctx):
    """A beam set with two datasets (the column kernel runs once per
    dataset), and the noiseless P(D) of the factory path."""
    s = spec2(n=512, nedge=128, shape=(48, 48), ndata=2)
    O, G = build2(orc, gpu_ctx, s)
    th = _batch(s, nprop=4, seed=8)
    lf, sf = G.getLogLikeBatch(th)
    G.setFFT(0)
    l0, s0 = G.getLogLikeBatch(th)
    G.setFFT(1)
    assert list(sf) == list(s0)
    assert np.max(np.abs(lf - l0)) < 1e-7
    lo, _ = O.loglike_batch(th[:2], 2)
    assert np.max(np.abs(lo - lf[:2])) < LL_TOL


def test_fused_columns_not_used_for_other_sizes(orc, gpu_ctx):
    s = spec2(n=384, nedge=96, shape=(40, 40))
    O, G = build2(orc, gpu_ctx, s)
    assert not G.fusedColumns()
    ll, st = G.getLogLikeBatch(s["th"][None, :])
    lo, _ = O.loglike_batch(s["th"][None, :])
    assert np.abs(ll[0] - lo[0]) < LL_TOL


def test_fused_columns_largest_size(orc, gpu_ctx):
    """n = 4096 (one column per block) against the 2D-transform path."""
    s = spec2(n=4096, nedge=256, shape=(48, 48))
    O, G = build2(orc, gpu_ctx, s)
    th = _batch(s, nprop=2, seed=5)
    assert G.fusedColumns()
    lf, sf = G.getLogLikeBatch(th)
    pf, inf = G.getPD(0, 0, th[0], setLog=False)
    G.setFFT(0)
    l0, s0 = G.getLogLikeBatch(th)
    p0, in0 = G.getPD(0, 0, th[0], setLog=False)
    assert list(sf) == list(s0)
    ok = sf == 0
    assert ok.any()
    assert np.max(np.abs(lf[ok] - l0[ok])) < 1e-7
    assert (inf["split1"], inf["split2"]) == (in0["split1"], in0["split2"])
    assert np.max(np.abs(pf - p0)) <= P_TOL * p0.max()
