"""Fixed-burn MCMC runs of the plain and the delayed-acceptance stretch move
(the single-process counterpart of pofd_affine_mcmc's fixed-burn mode,
pofdMCMC / affineEnsemble::doBurnIn with a fixed burn, then doSteps), with
effective samples per second from the integrated autocorrelation time
(Sokal's automatic window; the reference's acor reported beside it).

  * run_plain(E, nburn, nsteps)
  * run_da(E, S, nburn, nsteps, ...)   burn-in pairs train the surrogate,
                                       which is refreshed every `refresh`
                                       new exact evaluations
"""
import time

import numpy as np


def _summary(E, wall, nsteps):
    """Effective samples of the recorded chain: the integrated
    autocorrelation time with Sokal's automatic window (mcmc.integrated_time)
    sets ESS = nwalkers nsteps / max tau; the reference's acor (fixed 10-lag
    window, which saturates on long correlation times) is reported beside
    it."""
    from .mcmc import integrated_time
    ch, cl = E.getChain()
    tau, ok = E.getAcor()
    finite = np.isfinite(tau)
    tmax = float(np.max(tau[finite])) if np.any(finite) else float("nan")
    ti, win, conv = integrated_time(ch)
    for p in range(E.nparams):
        if E.state[p] & 3:  # fixed or ignored
            ti[p] = np.nan
            conv[p] = True
    fi = np.isfinite(ti)
    timax = float(np.max(ti[fi])) if np.any(fi) else float("nan")
    ess = E.nwalkers * nsteps / timax if np.isfinite(timax) else float("nan")
    ess_acor = E.nwalkers * nsteps / tmax if np.isfinite(tmax) else float("nan")
    return {"wall_s": wall, "tau_acor": [float(t) for t in tau],
            "tau_acor_max": tmax, "acor_ok": bool(ok),
            "tau": [float(t) for t in ti], "tau_max": timax,
            "tau_converged": bool(np.all(conv)),
            "steps_per_tau": nsteps / timax if np.isfinite(timax) else float("nan"),
            "failures": E.getFailures(),
            "ess": ess, "ess_per_s": ess / wall, "ess_acor": ess_acor,
            "chain": ch, "logl": cl}


def run_plain(E, nburn, nsteps):
    """Burn-in (unrecorded) then nsteps recorded plain steps; the timed
    region is the whole run."""
    t0 = time.perf_counter()
    E.doSteps(0, nburn)
    E.sync()
    t1 = time.perf_counter()
    base = E.daStats()
    E.doSteps(nsteps)
    wall = time.perf_counter() - t0
    st = E.daStats()
    out = _summary(E, wall, nsteps)
    out["stats"] = {k: st[k] - base[k] for k in st}
    out["burn_s"] = t1 - t0
    out["ess_per_s_after_burn"] = out["ess"] / (wall - out["burn_s"])
    return out


def run_da(E, S, nburn, nsteps, train_iters=2000, batch=512, lr=1e-3,
           refresh=5000, refresh_iters=400, chunk=25, holdout=None,
           da_scale=0.0, refresh_decay=False):
    """Burn-in with exact evaluations collected as training pairs, train,
    then delayed-acceptance steps in chunks, retraining on all pairs held
    after every `refresh` new exact evaluations.  The timed region includes
    the training.  da_scale: stretch parameter of the delayed-acceptance
    steps (0: the plain one).  The surrogate RMS error is reported on
    holdout (theta, logl) pairs when given, and on the exact pairs the run
    evaluated after its last training (never trained on).  The likelihood's
    plans and graphs for every survivor batch size are made before the timed
    region (prepareDA), as the plain run's are by its first step."""
    E.prepareDA()
    E.setDAScale(da_scale)
    t0 = time.perf_counter()
    E.collectPairs(S)
    E.doSteps(0, nburn)
    E.sync()
    t1 = time.perf_counter()
    t_burn = t1 - t0
    npairs_burn = S.nPairs()
    S.train(train_iters, batch, lr)
    t_train = time.perf_counter() - t1
    trained_on = npairs_burn
    E.setSurrogate(S)
    base = E.daStats()
    last = base["exact_evals"]
    done = 0
    nrefresh = 0
    while done < nsteps:
        k = min(chunk, nsteps - done)
        E.doStepsDA(k)
        done += k
        st = E.daStats()
        if st["exact_evals"] - last >= refresh and done < nsteps:
            t1 = time.perf_counter()
            trained_on = S.nPairs()
            # with refresh_decay the k-th retraining uses lr / (k + 1): the
            # surrogate -- hence the first-stage kernel -- changes less and
            # less (diminishing adaptation)
            S.train(refresh_iters, batch,
                    lr / (nrefresh + 1) if refresh_decay else lr)
            t_train += time.perf_counter() - t1
            last = st["exact_evals"]
            nrefresh += 1
    wall = time.perf_counter() - t0
    E.collectPairs(None)
    st = E.daStats()
    out = _summary(E, wall, nsteps)
    out["stats"] = {k: st[k] - base[k] for k in st}
    out["train_s"] = t_train
    out["burn_s"] = t_burn
    out["training_pairs_burn"] = npairs_burn
    out["refreshes"] = nrefresh
    out["da_scale"] = da_scale
    # after the common burn-in; the training stays in
    out["ess_per_s_after_burn"] = out["ess"] / (wall - t_burn)
    s = out["stats"]
    out["stage1_rate"] = s["stage1_passes"] / max(s["proposals"], 1)
    out["stage2_rate"] = s["accepted"] / max(s["stage1_passes"], 1)
    if holdout is not None:
        out["surrogate_rms"] = S.rms(*holdout)
    th, ll = S.getPairs()
    if th.shape[0] - trained_on >= 100:
        th, ll = th[trained_on:], ll[trained_on:]
        ok = np.isfinite(ll)
        out["surrogate_rms_untrained_pairs"] = S.rms(th[ok], ll[ok])
        out["untrained_pairs"] = int(ok.sum())
    return out


def find_start(loglike, x0, rounds=4, maxfev=2000, bounds=None):
    """A starting point near the likelihood maximum for the walkers: Powell's
    method (scipy) on -loglike from x0, restarted `rounds` times (each
    restart renews the search directions).  loglike(x) returns the summed
    log-likelihood of the free parameters x, or None for a rejected point.
    This replaces the hand-made init files of the reference's drivers
    (initFileKnots) for synthetic fits whose generating parameters are not
    the likelihood maximum.  bounds: (lo, hi) per parameter, as the
    sampler's limits (the result stays strictly inside)."""
    from scipy.optimize import minimize
    lo = hi = None
    if bounds is not None:
        # a margin keeps float32 rounding of the result inside the limits
        lo = np.array([b[0] + 1e-4 * max(1.0, abs(b[0])) for b in bounds])
        hi = np.array([b[1] - 1e-4 * max(1.0, abs(b[1])) for b in bounds])

    def f(x):
        if lo is not None and (np.any(x < lo) or np.any(x > hi)):
            return 1e300  # outside the sampler's limits
        v = loglike(x)
        return 1e300 if v is None or not np.isfinite(v) else -v
    x = np.asarray(x0, dtype=np.float64).copy()
    if lo is not None:
        x = np.clip(x, lo, hi)
    best = f(x)
    for _ in range(rounds):
        r = minimize(f, x, method="Powell",
                     options=dict(maxfev=maxfev, xtol=1e-6, ftol=1e-9))
        if r.fun < best:
            best, x = r.fun, r.x
    return x, -best


def laplace_covariance(loglike_batch, x0, h, bounds=None):
    """Covariance of the Laplace approximation at a likelihood maximum x0:
    the inverse of minus the Hessian of the log-likelihood by central
    differences with steps h (per parameter), all 1 + 2k + 2k(k-1)
    evaluations in one batch (loglike_batch(X [m][k]) -> logL [m], None
    entries for rejected points).  A Hessian that is not negative definite
    is made so by flipping its negative eigenvalues' signs."""
    x0 = np.asarray(x0, np.float64)
    h = np.broadcast_to(np.asarray(h, np.float64), x0.shape)
    k = x0.size
    pts = [x0]
    for i in range(k):
        for si in (1, -1):
            e = x0.copy()
            e[i] += si * h[i]
            pts.append(e)
    pairs = [(i, j) for i in range(k) for j in range(i + 1, k)]
    for i, j in pairs:
        for si, sj in ((1, 1), (1, -1), (-1, 1), (-1, -1)):
            e = x0.copy()
            e[i] += si * h[i]
            e[j] += sj * h[j]
            pts.append(e)
    X = np.array(pts)
    if bounds is not None:
        lo = np.array([b[0] for b in bounds])
        hi = np.array([b[1] for b in bounds])
        X = np.clip(X, lo, hi)
    L = np.asarray(loglike_batch(X), np.float64)
    f0 = L[0]
    H = np.empty((k, k))
    for i in range(k):
        H[i, i] = (L[1 + 2 * i] - 2 * f0 + L[2 + 2 * i]) / (h[i] * h[i])
    off = 1 + 2 * k
    for q, (i, j) in enumerate(pairs):
        a, b, c, d = L[off + 4 * q:off + 4 * q + 4]
        H[i, j] = H[j, i] = (a - b - c + d) / (4 * h[i] * h[j])
    w, V = np.linalg.eigh(-0.5 * (H + H.T))
    w = np.abs(w)
    w[w < 1e-12 * w.max()] = 1e-12 * w.max()
    return (V / w) @ V.T


def posterior_agreement(a, b, free):
    """(max over free parameters of |mean_a - mean_b| / sd_b, the same in
    units of the standard error of the difference sqrt(var_a / ESS_a,p +
    var_b / ESS_b,p), ESS_p = nwalkers nsteps / tau_p with each parameter's
    own integrated autocorrelation time)."""
    ca = a["chain"].reshape(-1, a["chain"].shape[-1])[:, free].astype(np.float64)
    cb = b["chain"].reshape(-1, b["chain"].shape[-1])[:, free].astype(np.float64)
    d = np.abs(ca.mean(0) - cb.mean(0))
    ta = np.asarray(a["tau"], np.float64)[free]
    tb = np.asarray(b["tau"], np.float64)[free]
    ea, eb = ca.shape[0] / ta, cb.shape[0] / tb
    se = np.sqrt(ca.var(0) / ea + cb.var(0) / eb)
    return float(np.max(d / cb.std(0))), float(np.max(d / se))


DA_PAIRS = 20000       # exact burn-in pairs the surrogate first trains on
DA_REFRESH = 5000      # retrain after this many new exact evaluations
DA_SCALE_2D = 5.0      # stretch parameter of the delayed-acceptance steps


def compare_two_fields_2d(ctx, nsteps, npre, nburn=None, plain_control=False,
                          train_iters=2000, da_scale=DA_SCALE_2D,
                          refresh=DA_REFRESH):
    """Plain vs delayed acceptance on the two-field 2D fit (a 1500x1500 pair
    on a 2048^2 grid and an 800x600 pair on a 1024^2 grid in one summed
    likelihood, 14 free parameters, 128 walkers).

    Both methods start from the same walkers, made untimed: a bounded Powell
    maximum of the likelihood (the synthetic maps' generating parameters lie
    several hundred log-likelihood units below it), walkers drawn from the
    Laplace approximation there (finite-difference Hessian) and npre plain
    steps.  Each run then burns nburn steps (default: enough
    for 20k exact pairs, on which the surrogate first trains) and records
    nsteps; the surrogate is retrained every `refresh` (5k) new exact
    evaluations, and
    the delayed-acceptance steps use the stretch parameter da_scale (the
    plain steps the reference's 2).  With plain_control a second plain run
    (another seed) gives the plain-vs-plain agreement the DA-vs-plain
    agreement is compared with.  Every run rejects steps outside the
    parameter limits (affineEnsemble.setLimitPolicy): the third sigma knot's
    posterior reaches its lower limit, where the reference's redrawing of z
    biases a chain, and more so the wider the stretch."""
    from . import synth
    from .mcmc import affineEnsemble, likeSum
    from .surrogate import Surrogate
    a, b = synth.config_2d_two_fields()
    if nburn is None:
        nburn = -(-DA_PAIRS // 128)
    La, Lb = synth.build_like2(a, ctx), synth.build_like2(b, ctx)
    S2 = likeSum(ctx, [La, Lb])
    npar = a["theta0"].size
    nfree = npar - 2
    lims = ([(float(a["theta0"][p]) - 2.0, float(a["theta0"][p]) + 2.0)
             for p in range(8)] + [(0.02, 1.0)] * 3 + [(-2.0, 1.0)] * 3)

    def loglike(x):
        t = a["theta0"].astype(np.float64).copy()
        t[:nfree] = x
        t = t.astype(np.float32)[None, :]
        (la, sa), (lb, sb) = La.getLogLikeBatch(t), Lb.getLogLikeBatch(t)
        return None if sa[0] != 0 or sb[0] != 0 else la[0] + lb[0]
    xopt, lopt = find_start(loglike, a["theta0"][:nfree], bounds=lims)
    x0 = a["theta0"].copy()
    x0[:nfree] = xopt

    def loglike_batch(X):
        t = np.repeat(a["theta0"][None, :].astype(np.float64), X.shape[0], 0)
        t[:, :nfree] = X
        t = t.astype(np.float32)
        (la, sa), (lb, sb) = La.getLogLikeBatch(t), Lb.getLogLikeBatch(t)
        return np.where((sa == 0) & (sb == 0), la + lb, -np.inf)
    cov = laplace_covariance(loglike_batch, xopt, 1e-3, bounds=lims)

    def ens(seed, start=None):
        E = affineEnsemble(ctx, S2, 128, npar, seed=seed)
        E.setParamFixed(npar - 2)
        E.setParamFixed(npar - 1)
        for p, (lo, hi) in enumerate(lims):
            E.setParamLimits(p, lo, hi)
        E.setErrorPolicy(True)  # unphysical corners reject instead of stop
        # the posterior of the third sigma knot reaches its lower limit:
        # steps outside the limits are rejected (exact for the truncated
        # posterior) rather than redrawn, for every run alike
        E.setLimitPolicy(True)
        if start is None:
            # walkers drawn from the Laplace approximation at the maximum,
            # inside the limits
            rng = np.random.default_rng(seed)
            lo = np.array([l for l, _ in lims])
            hi = np.array([h for _, h in lims])
            w = np.repeat(x0[None, :].astype(np.float64), 128, 0)
            k = 0
            while k < 128:
                d = rng.multivariate_normal(xopt, cov)
                if np.all(d > lo) and np.all(d < hi):
                    w[k, :nfree] = d
                    k += 1
            E.initChains(w.astype(np.float32))
        else:
            E.initChains(*start)
        return E
    E0 = ens(30)
    E0.doSteps(0, npre)
    start = E0.getLast()
    plain = run_plain(ens(31, start), nburn, nsteps)
    ch = plain["chain"].reshape(-1, npar)
    rng = np.random.default_rng(1)
    pick = rng.choice(ch.shape[0], 2000, replace=False)
    hold = (ch[pick], plain["logl"].reshape(-1)[pick])
    S = Surrogate(ctx, npar, list(range(nfree)), hidden=384, seed=9)
    da = run_da(ens(32, start), S, nburn, nsteps, train_iters=train_iters,
                refresh=refresh, holdout=hold, da_scale=da_scale)
    free = list(range(nfree))
    out = {"plain": plain, "da": da, "start_loglike": lopt,
           "agreement": posterior_agreement(da, plain, free)}
    if plain_control:
        plain2 = run_plain(ens(41, start), nburn, nsteps)
        out["plain_control"] = plain2
        out["agreement_plain_control"] = posterior_agreement(plain2, plain, free)
        # the two plain chains side by side (twice the walkers, the mean of
        # their autocorrelation times): the better estimate of the plain
        # posterior to hold DA against
        pooled = {"chain": np.concatenate([plain["chain"], plain2["chain"]], 1),
                  "tau": 0.5 * (np.asarray(plain["tau"]) + np.asarray(plain2["tau"]))}
        out["agreement_pooled"] = posterior_agreement(da, pooled, free)
    return out


SUMMARY_KEYS = ("wall_s", "burn_s", "tau_max", "tau_acor_max", "tau_converged",
                "steps_per_tau", "ess", "ess_per_s", "ess_per_s_after_burn",
                "failures")
DA_KEYS = ("train_s", "training_pairs_burn", "refreshes", "da_scale",
           "surrogate_rms", "surrogate_rms_untrained_pairs", "untrained_pairs",
           "stage1_rate", "stage2_rate", "stats")


def summarise(r):
    """The comparison of compare_two_fields_2d as plain numbers: both runs'
    wall times, autocorrelation times and effective samples per second, the
    ratios over the whole run and after the common burn-in, and the
    posterior-mean agreements (in sigma and in standard errors) of DA vs
    plain and, when run, of plain vs plain."""
    def pick(run, keys):
        return {k: run[k] for k in keys if k in run}
    out = {"plain": pick(r["plain"], SUMMARY_KEYS + ("stats",)),
           "da": pick(r["da"], SUMMARY_KEYS + DA_KEYS),
           "ess_per_s_ratio": r["da"]["ess_per_s"] / r["plain"]["ess_per_s"],
           "ess_per_s_ratio_after_burn": (r["da"]["ess_per_s_after_burn"] /
                                          r["plain"]["ess_per_s_after_burn"]),
           "posterior_mean_shift_sigma": r["agreement"][0],
           "posterior_mean_shift_se": r["agreement"][1],
           "start_loglike": r["start_loglike"]}
    if "plain_control" in r:
        out["plain_control"] = pick(r["plain_control"], SUMMARY_KEYS)
        out["plain_vs_plain_shift_sigma"] = r["agreement_plain_control"][0]
        out["plain_vs_plain_shift_se"] = r["agreement_plain_control"][1]
        out["posterior_mean_shift_sigma_vs_pooled_plain"] = r["agreement_pooled"][0]
        out["posterior_mean_shift_se_vs_pooled_plain"] = r["agreement_pooled"][1]
    return out


def _main(argv=None):
    """python -m pofd_affine_b200.runner two-fields-2d --steps 3000 --pre 300"""
    import argparse
    import json
    from . import Context
    p = argparse.ArgumentParser()
    p.add_argument("case", choices=["two-fields-2d"])
    p.add_argument("--steps", type=int, default=3000)
    p.add_argument("--pre", type=int, default=300)
    p.add_argument("--burn", type=int, default=None)
    p.add_argument("--da-scale", type=float, default=DA_SCALE_2D)
    p.add_argument("--save", default=None,
                   help="write the three chains (every --thin-th step) to this .npz")
    p.add_argument("--thin", type=int, default=10)
    p.add_argument("--refresh", type=int, default=DA_REFRESH,
                   help="retrain after this many new exact evaluations")
    p.add_argument("--no-control", action="store_true",
                   help="skip the second plain run")
    a = p.parse_args(argv)
    r = compare_two_fields_2d(Context(0), a.steps, a.pre, a.burn,
                              plain_control=not a.no_control,
                              da_scale=a.da_scale, refresh=a.refresh)
    summ = summarise(r)
    summ.update(steps=a.steps, pre=a.pre, burn=a.burn)
    if a.save:
        np.savez_compressed(a.save, **{
            "%s_%s" % (k, f): r[k][f][::a.thin]
            for k in ("plain", "da", "plain_control") if k in r
            for f in ("chain", "logl")})
    print(json.dumps(summ))


if __name__ == "__main__":
    _main()
