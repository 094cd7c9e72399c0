"""Python mirror of the reference's affine-invariant ensemble sampler.

  * affineEnsemble  affineEnsemble (affineEnsemble.h:60-200) over a batched
                    likelihood of this library (calcLike, calcLikeDouble,
                    gaussLike): setParamFixed / setParamBonus /
                    setParamIgnoreAcor, doSteps(nsteps, initsteps),
                    doBurnIn (fixed burn), getAcor, getAcceptanceFrac, and the
                    recorded chain.
  * acor            Goodman's acor (affineChainSet.cc:884-951).
  * integrated_time the integrated autocorrelation time with Sokal's
                    automatic window (no counterpart in the reference).
  * gaussLike       a multivariate Gaussian test likelihood on the device.
"""
import ctypes as C

import numpy as np

from ._lib import PofdError, check, lib, support_lib  # noqa: F401

FIXED, ACIGNORE, BONUS = 1, 2, 4  # mcmc_affine (global_settings.h:57)


def acor(x):
    """(mean, sigma, tau, ok) of a series by Goodman's acor; ok is False
    when the series is shorter than 50 (then only the mean is set)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    m, s, t = C.c_double(), C.c_double(), C.c_double()
    rc = check(lib().pofd_acor(x, x.size, C.byref(m), C.byref(s),
                               C.byref(t)))
    return m.value, s.value, t.value, rc == 0


def _autocorr_1d(x):
    """Normalised autocorrelation function of a series (FFT, zero-padded to
    at least twice its length so that the circular correlation is the
    linear one)."""
    x = np.asarray(x, dtype=np.float64)
    n = x.size
    m = 1
    while m < 2 * n:
        m *= 2
    f = np.fft.rfft(x - x.mean(), n=m)
    acf = np.fft.irfft(f * np.conjugate(f), n=m)[:n]
    return acf / acf[0] if acf[0] > 0 else np.zeros(n)


def integrated_time(chain, c=5.0):
    """Integrated autocorrelation time per parameter of an ensemble chain
    [nsteps][nwalkers][nparams] with Sokal's automatic window: the
    autocorrelation function is averaged over the walkers (Goodman & Weare
    2010), tau(M) = 1 + 2 sum_{t=1..M} rho(t), and M is the first window
    with M >= c tau(M) (Sokal 1997, sec. 3; c = 5 as in emcee).  Unlike
    acor's fixed 10-lag window this estimate does not saturate for long
    correlation times.  Returns (tau [nparams], window [nparams],
    converged [nparams]): converged is False when no window up to the chain
    length satisfies the rule (tau is then a lower bound)."""
    ch = np.asarray(chain, dtype=np.float64)
    nsteps, nwalkers, npar = ch.shape
    tau = np.full(npar, np.nan)
    win = np.zeros(npar, dtype=int)
    conv = np.zeros(npar, dtype=bool)
    for p in range(npar):
        if np.all(ch[:, :, p] == ch[0, 0, p]):
            continue  # a fixed parameter
        rho = np.mean([_autocorr_1d(ch[:, k, p]) for k in range(nwalkers)],
                      axis=0)
        taus = 2.0 * np.cumsum(rho) - 1.0
        ok = np.arange(taus.size) >= c * taus
        if np.any(ok):
            m = int(np.argmax(ok))
            conv[p] = True
        else:
            m = taus.size - 1
        tau[p], win[p] = taus[m], m
    return tau, win, conv


class gaussLike:
    """log N(theta[:k]; mean, cov) up to a constant, batched on the GPU."""

    def __init__(self, ctx, mean, cov):
        from ._lib import support_lib
        mean = np.ascontiguousarray(mean, dtype=np.float64)
        icov = np.ascontiguousarray(np.linalg.inv(np.asarray(cov, np.float64)))
        h = C.c_void_p()
        check(support_lib().pofd_gauss_create(ctx.device, mean.size, mean,
                                              icov, C.byref(h)))
        self.h, self.ctx, self.k = h, ctx, mean.size

    def __del__(self):
        if getattr(self, "h", None):
            try:
                from ._lib import support_lib
                support_lib().pofd_gauss_destroy(self.h)
            except Exception:  # interpreter shutdown: the library is gone
                pass
            self.h = None


class likeSum:
    """Sum of likelihoods (calcLike / calcLikeDouble / gaussLike) over the
    same parameters, members evaluated concurrently."""

    def __init__(self, ctx, likes=()):
        h = C.c_void_p()
        check(lib().pofd_likesum_create(ctx.h, C.byref(h)))
        self.h, self.ctx, self.members = h, ctx, []
        for L in likes:
            self.add(L)

    def add(self, like):
        from .api1d import calcLike
        from .api2d import calcLikeDouble
        if isinstance(like, calcLike):
            check(lib().pofd_likesum_add_like1(self.h, like.h))
        elif isinstance(like, calcLikeDouble):
            check(lib().pofd_likesum_add_like2(self.h, like.h))
        elif isinstance(like, gaussLike):
            fn = C.cast(support_lib().pofd_gauss_eval_batch_device, C.c_void_p)
            check(lib().pofd_likesum_add(self.h, fn, like.h))
        else:
            raise PofdError(-10, "unsupported likelihood object")
        self.members.append(like)

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().pofd_likesum_destroy(self.h)
            except Exception:  # interpreter shutdown: the library is gone
                pass
            self.h = None


class affineEnsemble:
    """Batched stretch-move ensemble (one process, one GPU)."""

    def __init__(self, ctx, like, nwalkers, nparams, scalefac=2.0, seed=0):
        h = C.c_void_p()
        check(lib().pofd_ensemble_create(ctx.h, int(nwalkers), int(nparams),
                                         float(scalefac), int(seed),
                                         C.byref(h)))
        self.h, self.ctx, self.like = h, ctx, like
        self.nwalkers, self.nparams = int(nwalkers), int(nparams)
        self.state = np.zeros(self.nparams, dtype=np.int32)
        self.lo = np.full(self.nparams, -np.inf, np.float32)
        self.hi = np.full(self.nparams, np.inf, np.float32)
        self.nsteps_done = 0
        from .api1d import calcLike
        from .api2d import calcLikeDouble
        if isinstance(like, calcLike):
            check(lib().pofd_ensemble_use_like1(h, like.h))
        elif isinstance(like, calcLikeDouble):
            check(lib().pofd_ensemble_use_like2(h, like.h))
        elif isinstance(like, gaussLike):
            fn = C.cast(support_lib().pofd_gauss_eval_batch_device, C.c_void_p)
            check(lib().pofd_ensemble_set_likelihood(h, fn, like.h))
        elif isinstance(like, likeSum):
            fn = C.cast(lib().pofd_likesum_eval_batch_device, C.c_void_p)
            check(lib().pofd_ensemble_set_likelihood(h, fn, like.h))
        else:
            from .shard import shardedLike
            if not isinstance(like, shardedLike):
                raise PofdError(-10, "unsupported likelihood object")
            fn = C.cast(lib().pofd_shard_eval_batch_device, C.c_void_p)
            check(lib().pofd_ensemble_set_likelihood(h, fn, like.h))

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().pofd_ensemble_destroy(self.h)
            except Exception:  # interpreter shutdown: the library is gone
                pass
            self.h = None

    # ---------------------------------------------------------- set-up
    def _state(self, i, bits):
        self.state[i] |= bits
        check(lib().pofd_ensemble_set_param_state(self.h, int(i),
                                                  int(self.state[i])))

    def setParamFixed(self, i):
        self._state(i, FIXED | ACIGNORE)

    def setParamIgnoreAcor(self, i):
        self._state(i, ACIGNORE)

    def setParamBonus(self, i):
        self._state(i, ACIGNORE | BONUS)

    def setParamLimits(self, i, lo=-np.inf, hi=np.inf):
        self.lo[i], self.hi[i] = lo, hi
        check(lib().pofd_ensemble_set_param_limits(self.h, int(i), float(lo),
                                                   float(hi)))

    def setErrorPolicy(self, reject_failures):
        """False (default): a failed likelihood evaluation stops the run as
        in the reference; True: the step is rejected and counted."""
        check(lib().pofd_ensemble_set_error_policy(self.h,
                                                   1 if reject_failures else 0))

    def setLimitPolicy(self, reject_outside):
        """False (default): a step outside the parameter limits redraws z
        (up to 40 times) as in the reference; True: it is rejected, which
        keeps the move exact where the posterior reaches a limit."""
        self.reject_outside = bool(reject_outside)
        check(lib().pofd_ensemble_set_limit_policy(self.h,
                                                   1 if reject_outside else 0))

    def getFailures(self):
        n = C.c_ulonglong()
        check(lib().pofd_ensemble_failures(self.h, C.byref(n)))
        return n.value

    def setTemperature(self, t):
        check(lib().pofd_ensemble_set_temperature(self.h, float(t)))

    def generateInitialPosition(self, theta0, sigma, rng=None,
                                maxtrials=1000):
        """Walkers theta0 + sigma * N(0, 1) per free parameter, redrawn
        until inside the limits (initFileKnots::generateRandomKnotValues);
        fixed parameters keep theta0, bonus ones are NaN."""
        rng = np.random.default_rng(rng)
        theta0 = np.asarray(theta0, np.float32)
        sigma = np.broadcast_to(np.asarray(sigma, np.float64), theta0.shape)
        w = np.empty((self.nwalkers, self.nparams), np.float32)
        for k in range(self.nwalkers):
            for p in range(self.nparams):
                if self.state[p] & BONUS:
                    w[k, p] = np.nan
                    continue
                if self.state[p] & FIXED or sigma[p] == 0:
                    w[k, p] = theta0[p]
                    continue
                for _ in range(maxtrials):
                    v = np.float32(theta0[p] + sigma[p] * rng.standard_normal())
                    if self.lo[p] <= v <= self.hi[p]:
                        break
                else:
                    raise PofdError(-10, "Couldn't generate initial value")
                w[k, p] = v
        return w

    def initChains(self, walkers, logl=None):
        w = np.ascontiguousarray(walkers, dtype=np.float32)
        if w.shape != (self.nwalkers, self.nparams):
            raise PofdError(-10, "walkers must be [nwalkers, nparams]")
        lp = None
        if logl is not None:
            self._l0 = np.ascontiguousarray(logl, dtype=np.float64)
            lp = self._l0.ctypes.data_as(C.c_void_p)
        check(lib().pofd_ensemble_init(self.h, w, lp))
        self.nsteps_done = 0

    # ------------------------------------------------------------ steps
    def sync(self):
        """Wait for the ensemble's queued work (reads the record counter)."""
        self.nRecorded()

    def doSteps(self, nsteps, initsteps=0):
        """initsteps unrecorded steps, then nsteps recorded ones."""
        if initsteps:
            check(lib().pofd_ensemble_do_steps(self.h, int(initsteps), 0))
            self.nsteps_done += int(initsteps)
        if nsteps:
            check(lib().pofd_ensemble_do_steps(self.h, int(nsteps), 1))
            self.nsteps_done += int(nsteps)

    def doBurnIn(self, nburn):
        """Fixed burn-in (the -f mode): nburn unrecorded steps."""
        self.doSteps(0, nburn)

    def clearChain(self):
        check(lib().pofd_ensemble_clear_chain(self.h))

    # ------------------------------------------------ delayed acceptance
    def setSurrogate(self, sur):
        """First stage of delayed acceptance: a Surrogate."""
        fn = C.cast(lib().pofd_surrogate_predict_device, C.c_void_p)
        check(lib().pofd_ensemble_set_surrogate(self.h, fn, sur.h))
        self.sur = sur

    def setDAScale(self, a):
        """Stretch parameter of the delayed-acceptance steps (0: the plain
        steps' scalefac)."""
        check(lib().pofd_ensemble_set_da_scale(self.h, float(a)))

    def collectPairs(self, sur):
        """Append every exact evaluation to sur's training pairs (None
        stops)."""
        check(lib().pofd_ensemble_collect_pairs(self.h,
                                                sur.h if sur else None))
        self.collector = sur

    def prepareDA(self):
        """One exact evaluation of every survivor batch size (plans and
        graphs made before sampling)."""
        check(lib().pofd_ensemble_prepare_da(self.h))

    def doStepsDA(self, nsteps, record=True):
        check(lib().pofd_ensemble_do_steps_da(self.h, int(nsteps),
                                              1 if record else 0))
        self.nsteps_done += int(nsteps)

    def daStats(self):
        """{proposals, stage1_passes, exact_evals, accepted} since init."""
        o = (C.c_ulonglong * 4)()
        check(lib().pofd_ensemble_da_stats(self.h, o))
        return dict(zip(["proposals", "stage1_passes", "exact_evals",
                         "accepted"], [int(v) for v in o]))

    # ---------------------------------------------------------- results
    def nRecorded(self):
        n = C.c_uint()
        check(lib().pofd_ensemble_nrecorded(self.h, C.byref(n)))
        return n.value

    def getChain(self):
        n = self.nRecorded()
        th = np.empty((n, self.nwalkers, self.nparams), np.float32)
        ll = np.empty((n, self.nwalkers), np.float64)
        if n:
            check(lib().pofd_ensemble_chain(self.h,
                                            th.ctypes.data_as(C.c_void_p),
                                            ll.ctypes.data_as(C.c_void_p)))
        return th, ll

    def getLast(self):
        th = np.empty((self.nwalkers, self.nparams), np.float32)
        ll = np.empty(self.nwalkers, np.float64)
        check(lib().pofd_ensemble_last(self.h, th.ctypes.data_as(C.c_void_p),
                                       ll.ctypes.data_as(C.c_void_p)))
        return th, ll

    def getNAccept(self):
        out = np.empty(self.nwalkers, np.uint32)
        check(lib().pofd_ensemble_naccept(self.h, out))
        return out

    def checkpoint(self, path):
        """Write the sampler's resumable state to path (.npz): the current
        walkers and log-likelihoods, the generator's step counter and seed,
        the accepted-step counts and the steps taken.  The recorded chain is
        not part of it (read it with getChain before)."""
        th, ll = self.getLast()
        step, seed = C.c_ulonglong(), C.c_ulonglong()
        check(lib().pofd_ensemble_get_counter(self.h, C.byref(step),
                                              C.byref(seed)))
        np.savez(path, walkers=th, logl=ll, step=np.uint64(step.value),
                 seed=np.uint64(seed.value), naccept=self.getNAccept(),
                 nsteps_done=np.int64(self.nsteps_done),
                 shape=np.array([self.nwalkers, self.nparams]))

    def resume(self, path):
        """Continue from a checkpoint written by checkpoint(): same walker
        count, parameter count and seed required.  Parameter states, limits,
        the likelihood and the temperature are the caller's to set as
        before.  The plain stretch-move chain then continues exactly as the
        uninterrupted run would."""
        z = np.load(path)
        if list(z["shape"]) != [self.nwalkers, self.nparams]:
            raise PofdError(-10, "checkpoint is for another ensemble shape")
        step, seed = C.c_ulonglong(), C.c_ulonglong()
        check(lib().pofd_ensemble_get_counter(self.h, C.byref(step),
                                              C.byref(seed)))
        if int(z["seed"]) != seed.value:
            raise PofdError(-10, "checkpoint was written with another seed")
        self.initChains(z["walkers"], z["logl"])
        check(lib().pofd_ensemble_set_counter(self.h, int(z["step"])))
        check(lib().pofd_ensemble_set_naccept(
            self.h, np.ascontiguousarray(z["naccept"], np.uint32)))
        self.nsteps_done = int(z["nsteps_done"])

    def writeChain(self, path, param_names=None, **metadata):
        """The recorded chain with its likelihoods, the parameter states,
        the acceptance fractions and acor lengths, in the reference's output
        layout (affineEnsemble::writeToHDF5), as .npz (stats.writeChain)."""
        from .stats import writeChain
        th, ll = self.getChain()
        tau = self.getAcor()[0] if self.nRecorded() > 1 else np.full(self.nparams, np.nan)
        writeChain(path, th, ll, param_names=param_names, param_states=self.state,
                   acceptance=self.getAcceptanceFrac(), acor=tau,
                   nsteps_done=self.nsteps_done, **metadata)

    def getAcceptanceFrac(self):
        return self.getNAccept() / max(self.nsteps_done, 1)

    def getAcor(self):
        """(tau[nparams], ok): NaN for ignored parameters."""
        tau = np.empty(self.nparams)
        rc = check(lib().pofd_ensemble_acor(self.h, tau))
        return tau, rc == 0

    def getESS(self):
        """nwalkers * nrecorded / max tau (acor over the recorded chain)."""
        tau, ok = self.getAcor()
        t = np.nanmax(tau) if np.any(np.isfinite(tau)) else np.nan
        return self.nwalkers * self.nRecorded() / t, tau, ok

    def getIntegratedTime(self, c=5.0):
        """integrated_time of the recorded chain over the parameters that
        are neither fixed nor ignored for acor: (tau [nparams] with NaN for
        the others, converged)."""
        ch, _ = self.getChain()
        tau, _, conv = integrated_time(ch, c)
        for p in range(self.nparams):
            if self.state[p] & (FIXED | ACIGNORE):
                tau[p] = np.nan
                conv[p] = True
        return tau, bool(np.all(conv))
