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
sorted samples by fractional-index interpolation.  doubleLogNormalStats
does the same for the two-band log-normal colour model
(numberCountsDoubleLogNormalStats::build,
numberCountsDoubleLogNormalStats.cc:96-282): band-1 log10 dN/dS and the
colour model's sigma and offset curves (or, as ratios, sigma and mean of
f2/f1) against band-1 flux.
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
            with np.errstate(invalid="ignore"):  # -inf log counts give NaN, as in C
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


def _spline_eval(x, y, m, u):
    """The cubic with second derivatives m through (x, y) at u (inside
    [x_0, x_{n-1}]); linear where m is zero."""
    j = np.clip(np.searchsorted(x, u, side="right") - 1, 0, len(x) - 2)
    h = x[j + 1] - x[j]
    a = (x[j + 1] - u) / h
    b = (u - x[j]) / h
    return (a * y[j] + b * y[j + 1] +
            ((a ** 3 - a) * m[j] + (b ** 3 - b) * m[j + 1]) * h * h / 6.0)


def numberCounts(knotpos, log10vals, flux):
    """dN/dS of the knot-spline model (numberCountsKnotsSpline::
    getNumberCounts, and numberCountsDoubleLogNormal::getBand1NumberCounts,
    numberCountsDoubleLogNormal.cc:1272-1283): 2^spline(log2 S) of the
    natural cubic spline through (log2 S_k, log2(10) * theta_k), 0 outside
    [S_0, S_{K-1})."""
    lk = np.log2(np.asarray(knotpos, np.float64))
    lv = np.log2(10.0) * np.asarray(log10vals, np.float64)
    m = _natural_spline(lk, lv)
    s = np.atleast_1d(np.asarray(flux, np.float64))
    out = np.zeros(s.shape)
    inside = (s >= knotpos[0]) & (s < knotpos[-1])
    out[inside] = np.exp2(_spline_eval(lk, lv, m, np.log2(s[inside])))
    return out


def colourCurve(knotpos, vals, flux, floor=None):
    """The colour model's sigma or offset at band-1 flux
    (numberCountsDoubleLogNormal::getSigmaInner / getOffsetInner,
    numberCountsDoubleLogNormal.cc:1172-1195): constant for one knot, held
    at the end values outside the knots, linear between two knots, the
    natural cubic spline in flux for more; sigma is floored at the model's
    minimum (0 unless set)."""
    k = np.asarray(knotpos, np.float64)
    v = np.asarray(vals, np.float64)
    s = np.atleast_1d(np.asarray(flux, np.float64))
    if len(k) == 1:
        out = np.full(s.shape, v[0])
    else:
        out = np.empty(s.shape)
        lo, hi = s <= k[0], s >= k[-1]
        mid = ~(lo | hi)
        out[lo], out[hi] = v[0], v[-1]
        out[mid] = _spline_eval(k, v, _natural_spline(k, v), s[mid])
        if floor is not None:
            out[mid] = np.maximum(out[mid], floor)
    return out


def setupFluxes(minval, maxval, n, logspace=True):
    """n flux points from minval to maxval (float limits), log or linearly
    spaced, accumulated in double and stored as float
    (statsAccumulator::setupFluxes, statsAccumulator.cc:13-33)."""
    lo, hi = float(np.float32(minval)), float(np.float32(maxval))
    i = np.arange(n, dtype=np.float64)
    if logspace:
        llo = np.log(lo)
        return np.exp(llo + (np.log(hi) - llo) / (n - 1) * i).astype(np.float32)
    return (lo + (hi - lo) / (n - 1) * i).astype(np.float32)


def _band_range(knotpos, double_knots=False):
    """The reference's flux range of a counts curve: the first knot to just
    below the last (the counts are 0 at the last knot), passed on as float.
    The two-band model holds its knots as float and pulls the top in float
    arithmetic (numberCountsDoubleLogNormalStats.cc:212-214); the 1D model
    holds double knots and pulls the top in double before the conversion
    (numberCountsKnotsSplineStats.cc:156-159): double_knots=True."""
    if double_knots:
        lo, hi = float(knotpos[0]), float(knotpos[-1])
        return np.float32(lo), np.float32(hi - 1e-4 * (hi - lo))
    lo, hi = np.float32(knotpos[0]), np.float32(knotpos[-1])
    d = np.float32(hi - lo)
    return lo, np.float32(float(hi) - 1e-4 * float(d))


def _read_walker_major(chain, logl, thin):
    """Flatten a recorded chain walker-major (the order of the reference's
    file), pick the best-fit sample (the first maximum; NaN likelihoods
    never win, and a NaN first entry wins outright, as the reference's
    scan from like[0] does) and every thin-th sample."""
    ch = np.transpose(np.asarray(chain, np.float32), (1, 0, 2))
    ll = np.transpose(np.asarray(logl, np.float64), (1, 0))
    nw, ns, npar = ch.shape
    flat = ch.reshape(nw * ns, npar)
    lflat = ll.reshape(nw * ns)
    if np.isnan(lflat[0]):
        best = 0
    else:
        best = int(np.argmax(np.where(np.isnan(lflat), -np.inf, lflat)))
    nsamp = (nw * ns + thin - 1) // thin
    return flat, lflat, best, flat[::thin][:nsamp], nsamp


def numberCountsStats(chain, logl, knotpos, nflux=1024, thin=5, logspace=True):
    """pofd_affine_getStats for a knot-spline chain.  chain
    [nsteps][nwalkers][nparams] and logl [nsteps][nwalkers] as the ensemble
    records them (reordered here walker-major, as the reference's file
    holds them).  Returns a dict: best_loglike, best_params, param_mean,
    param_median, param_snake [3][nparams][2], flux [nflux], mean, median,
    snake [3][nflux][2] of log10 dN/dS."""
    flat, lflat, best, samples, nsamp = _read_walker_major(chain, logl, thin)
    pmean, pmed, psnake = accumulateStats(samples.T)
    K = len(knotpos)
    flux = setupFluxes(*_band_range(knotpos, double_knots=True), nflux,
                       logspace).astype(np.float64)
    working = np.empty((nflux, nsamp), np.float32)
    for i, p in enumerate(samples):
        with np.errstate(divide="ignore"):
            working[:, i] = np.log10(numberCounts(knotpos, p[:K], flux))
    mean, median, snake = accumulateStats(working)
    return {"best_loglike": float(lflat[best]), "best_params": flat[best].copy(),
            "param_mean": pmean, "param_median": pmed, "param_snake": psnake,
            "flux": flux, "mean": mean, "median": median, "snake": snake,
            "plevels": PLEVELS, "nsamples": nsamp}


def doubleLogNormalStats(chain, logl, knotpos, sigmapos, offsetpos,
                         nflux=1024, thin=5, logspace=True, ratios=False,
                         min_sigma=0.0):
    """pofd_affine_getStats for a two-band log-normal colour chain (the
    parameter vector: log10 band-1 counts at knotpos, then the sigma values
    at sigmapos, then the offsets at offsetpos, then any sigma multipliers
    and bonus parameters).  Returns the parameter summaries as
    numberCountsStats does plus three curves of nflux points, each with
    mean, median and snake [3][nflux][2]: "band1" (log10 dN/dS1 against
    S1), "sigma" and "offset" (the colour model's sigma and offset against
    S1, or with ratios=True the sigma and the mean of f2/f1,
    sqrt(exp(2 mu + s^2) expm1(s^2)) and exp(mu + s^2 / 2)).  The sigma
    curve spans the sigma knots when there are two or more, else the
    band-1 range; the offset curve the offset knots when there are two or
    more, else the range of the curve before it."""
    flat, lflat, best, samples, nsamp = _read_walker_major(chain, logl, thin)
    pmean, pmed, psnake = accumulateStats(samples.T)
    K, NS, NO = len(knotpos), len(sigmapos), len(offsetpos)
    lo, hi = _band_range(knotpos)
    s1 = setupFluxes(lo, hi, nflux, logspace).astype(np.float64)
    if NS > 1:
        lo, hi = np.float32(sigmapos[0]), np.float32(sigmapos[-1])
    ssig = setupFluxes(lo, hi, nflux, logspace).astype(np.float64)
    if NO > 1:
        lo, hi = np.float32(offsetpos[0]), np.float32(offsetpos[-1])
    soff = setupFluxes(lo, hi, nflux, logspace).astype(np.float64)
    w1 = np.empty((nflux, nsamp), np.float32)
    ws = np.empty((nflux, nsamp), np.float32)
    wo = np.empty((nflux, nsamp), np.float32)
    for i, p in enumerate(samples):
        cnt, sv, ov = p[:K], p[K:K + NS], p[K + NS:K + NS + NO]
        with np.errstate(divide="ignore"):
            w1[:, i] = np.log10(numberCounts(knotpos, cnt, s1))
        if ratios:
            sg = colourCurve(sigmapos, sv, ssig, min_sigma).astype(np.float32)
            mu = colourCurve(offsetpos, ov, ssig).astype(np.float32)
            s2 = sg.astype(np.float64) ** 2
            ws[:, i] = np.sqrt(np.exp(2 * mu.astype(np.float64) + s2) * np.expm1(s2))
            sg = colourCurve(sigmapos, sv, soff, min_sigma).astype(np.float32)
            mu = colourCurve(offsetpos, ov, soff).astype(np.float32)
            wo[:, i] = np.exp(mu.astype(np.float64) + 0.5 * sg.astype(np.float64) ** 2)
        else:
            ws[:, i] = colourCurve(sigmapos, sv, ssig, min_sigma)
            wo[:, i] = colourCurve(offsetpos, ov, soff)
    out = {"best_loglike": float(lflat[best]), "best_params": flat[best].copy(),
           "param_mean": pmean, "param_median": pmed, "param_snake": psnake,
           "plevels": PLEVELS, "nsamples": nsamp, "ratios": bool(ratios)}
    for name, flux, work in (("band1", s1, w1), ("sigma", ssig, ws), ("offset", soff, wo)):
        m, md, sn = accumulateStats(work)
        out[name] = {"flux": flux, "mean": m, "median": md, "snake": sn}
    return out


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
