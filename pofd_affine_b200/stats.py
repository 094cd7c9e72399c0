"""Chain output and posterior summaries of 1D number-counts fits.

writeChain stores a recorded chain in the layout of the reference's HDF5
output (affineEnsemble::writeToHDF5: Chains/Chain [nwalkers][nsteps][nparams],
Chains/Likelihood [nwalkers][nsteps], per-parameter names and states,
acceptance fractions, autocorrelation lengths) as an .npz file; there is no
HDF5 library here, so the container is numpy's.

numberCountsStats restates pofd_affine_getStats for the knot-spline model
(numberCountsKnotsSplineStats::build, numberCountsKnotsSplineStats.cc:62-180,
with statsAccumulator::accumulateStats, statsAccumulator.cc:43-75): the chain
read walker-major, every thin-th sample kept, the best-fit parameters at the
highest likelihood, and per parameter and per flux point of log10 dN/dS the
mean, the median and the 68.3 / 95.4 / 99.7 % intervals ("snake") from the
sorted samples by fractional-index interpolation.
"""
import numpy as np

PLEVELS = (0.683, 0.954, 0.997)


def accumulateStats(working):
    """working [n1][n2] (float32, n2 samples per row) -> mean, median [n1]
    and snake [nprob][n1][2], as statsAccumulator::accumulateStats: the
    mean summed in double in sorted order, the median the n2/2-th sorted
    value, the interval ends interpolated at fractional indices
    (1 -/+ p) n2 / 2 of the sorted samples."""
    w = np.sort(np.asarray(working, np.float32), axis=1)
    n1, n2 = w.shape
    # a running (sequential) double sum in sorted order, as the reference's
    mean = (np.cumsum(w.astype(np.float64), axis=1)[:, -1] / n2).astype(np.float32)
    median = w[:, n2 // 2].copy()
    snake = np.empty((len(PLEVELS), n1, 2), np.float32)
    for k, p in enumerate(PLEVELS):
        for side, frac in ((0, np.float32(0.5) * (np.float32(1.0) - np.float32(p)) * np.float32(n2)),
                           (1, np.float32(0.5) * (np.float32(1.0) + np.float32(p)) * np.float32(n2))):
            i = int(frac)
            i1 = min(i + 1, n2 - 1)
            snake[k, :, side] = w[:, i] + (w[:, i1] - w[:, i]) * (frac - np.float32(i))
    return mean, median, snake


def _natural_spline(x, y):
    """Second derivatives of the natural cubic spline through (x, y)."""
    n = len(x)
    m = np.zeros(n)
    if n < 3:
        return m
    h = np.diff(x)
    A = np.zeros((n - 2, n - 2))
    r = np.empty(n - 2)
    for i in range(1, n - 1):
        if i > 1:
            A[i - 1, i - 2] = h[i - 1]
        A[i - 1, i - 1] = 2.0 * (h[i - 1] + h[i])
        if i < n - 2:
            A[i - 1, i] = h[i]
        r[i - 1] = 6.0 * ((y[i + 1] - y[i]) / h[i] - (y[i] - y[i - 1]) / h[i - 1])
    m[1:-1] = np.linalg.solve(A, r)
    return m


def numberCounts(knotpos, log10vals, flux):
    """dN/dS of the knot-spline model (numberCountsKnotsSpline::
    getNumberCounts): 2^spline(log2 S) of the natural cubic spline through
    (log2 S_k, log2(10) * theta_k), 0 outside [S_0, S_{K-1})."""
    lk = np.log2(np.asarray(knotpos, np.float64))
    lv = np.log2(10.0) * np.asarray(log10vals, np.float64)
    m = _natural_spline(lk, lv)
    s = np.atleast_1d(np.asarray(flux, np.float64))
    out = np.zeros(s.shape)
    inside = (s >= knotpos[0]) & (s < knotpos[-1])
    u = np.log2(s[inside])
    j = np.clip(np.searchsorted(lk, u, side="right") - 1, 0, len(lk) - 2)
    h = lk[j + 1] - lk[j]
    a = (lk[j + 1] - u) / h
    b = (u - lk[j]) / h
    v = (a * lv[j] + b * lv[j + 1] +
         ((a ** 3 - a) * m[j] + (b ** 3 - b) * m[j + 1]) * h * h / 6.0)
    out[inside] = np.exp2(v)
    return out


def numberCountsStats(chain, logl, knotpos, nflux=1024, thin=5, logspace=True):
    """pofd_affine_getStats for a knot-spline chain.  chain
    [nsteps][nwalkers][nparams] and logl [nsteps][nwalkers] as the ensemble
    records them (reordered here walker-major, as the reference's file
    holds them).  Returns a dict: best_loglike, best_params, param_mean,
    param_median, param_snake [3][nparams][2], flux [nflux], mean, median,
    snake [3][nflux][2] of log10 dN/dS."""
    ch = np.transpose(np.asarray(chain, np.float32), (1, 0, 2))  # walker-major
    ll = np.transpose(np.asarray(logl, np.float64), (1, 0))
    nw, ns, npar = ch.shape
    flat = ch.reshape(nw * ns, npar)
    lflat = ll.reshape(nw * ns)
    best = int(np.argmax(lflat)) if np.isfinite(lflat).any() else 0
    nsamp = (nw * ns + thin - 1) // thin
    samples = flat[::thin][:nsamp]
    pmean, pmed, psnake = accumulateStats(samples.T)
    K = len(knotpos)
    lo, hi = float(knotpos[0]), float(knotpos[-1])
    hi -= 1e-4 * (hi - lo)  # counts are 0 at the last knot
    if logspace:
        flux = np.exp(np.log(lo) + (np.log(hi) - np.log(lo)) * np.arange(nflux) / (nflux - 1))
    else:
        flux = lo + (hi - lo) * np.arange(nflux) / (nflux - 1)
    flux = flux.astype(np.float32).astype(np.float64)
    working = np.empty((nflux, nsamp), np.float32)
    for i, p in enumerate(samples):
        with np.errstate(divide="ignore"):
            working[:, i] = np.log10(numberCounts(knotpos, p[:K], flux))
    mean, median, snake = accumulateStats(working)
    return {"best_loglike": float(lflat[best]), "best_params": flat[best].copy(),
            "param_mean": pmean, "param_median": pmed, "param_snake": psnake,
            "flux": flux, "mean": mean, "median": median, "snake": snake,
            "plevels": PLEVELS, "nsamples": nsamp}


def writeChain(path, chain, logl, param_names=None, param_states=None,
               acceptance=None, acor=None, **metadata):
    """Write a recorded chain ([nsteps][nwalkers][nparams] as recorded) in
    the reference's output layout: chain [nwalkers][nsteps][nparams],
    likelihood [nwalkers][nsteps], plus parameter names and states
    (FIXED 1, ACIGNORE 2, BONUS 4), acceptance fractions, acor lengths and
    any further metadata."""
    ch = np.transpose(np.asarray(chain, np.float32), (1, 0, 2))
    ll = np.transpose(np.asarray(logl, np.float64), (1, 0))
    npar = ch.shape[2]
    names = np.array(param_names if param_names is not None
                     else ["p%d" % i for i in range(npar)])
    states = np.asarray(param_states if param_states is not None
                        else np.zeros(npar, np.int32), np.int32)
    extra = {k: np.asarray(v) for k, v in metadata.items()}
    np.savez(path, chain=ch, likelihood=ll, param_names=names,
             param_states=states,
             acceptance=np.asarray(acceptance if acceptance is not None else [],
                                   np.float64),
             acor=np.asarray(acor if acor is not None else [], np.float64),
             **extra)


def readChain(path):
    """The arrays writeChain stored, with chain / likelihood back in the
    recorded order ([nsteps][nwalkers]...)."""
    z = np.load(path, allow_pickle=False)
    out = {k: z[k] for k in z.files}
    out["chain"] = np.transpose(out["chain"], (1, 0, 2))
    out["likelihood"] = np.transpose(out["likelihood"], (1, 0))
    return out
