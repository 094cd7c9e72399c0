"""Fixed-burn MCMC runs of the plain and the delayed-acceptance stretch move
(the single-process counterpart of pofd_affine_mcmc's fixed-burn mode,
pofdMCMC / affineEnsemble::doBurnIn with a fixed burn, then doSteps), with
effective samples per second measured by acor.

  * run_plain(E, nburn, nsteps)
  * run_da(E, S, nburn, nsteps, ...)   burn-in pairs train the surrogate,
                                       which is refreshed every `refresh`
                                       new exact evaluations
"""
import time

import numpy as np


def _summary(E, wall, nsteps):
    ch, cl = E.getChain()
    tau, ok = E.getAcor()
    finite = np.isfinite(tau)
    tmax = float(np.max(tau[finite])) if np.any(finite) else float("nan")
    ess = E.nwalkers * nsteps / tmax if np.isfinite(tmax) else float("nan")
    return {"wall_s": wall, "tau": [float(t) for t in tau], "tau_max": tmax,
            "failures": E.getFailures(),
            "acor_ok": bool(ok), "ess": ess, "ess_per_s": ess / wall,
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
           refresh=5000, refresh_iters=300, chunk=25, holdout=None):
    """Burn-in with exact evaluations collected as training pairs, train,
    then delayed-acceptance steps in chunks, retraining after every
    `refresh` new exact evaluations.  The timed region includes the
    training.  holdout (theta, logl) gives the surrogate RMS error.  The
    likelihood's plans and graphs for every survivor batch size are made
    before the timed region (prepareDA), as the plain run's are by its
    first step."""
    E.prepareDA()
    t0 = time.perf_counter()
    E.collectPairs(S)
    E.doSteps(0, nburn)
    E.sync()
    t1 = time.perf_counter()
    t_burn = t1 - t0
    S.train(train_iters, batch, lr)
    t_train = time.perf_counter() - t1
    E.setSurrogate(S)
    base = E.daStats()
    last = base["exact_evals"]
    done = 0
    while done < nsteps:
        k = min(chunk, nsteps - done)
        E.doStepsDA(k)
        done += k
        st = E.daStats()
        if st["exact_evals"] - last >= refresh and done < nsteps:
            t1 = time.perf_counter()
            S.train(refresh_iters, batch, lr)
            t_train += time.perf_counter() - t1
            last = st["exact_evals"]
    wall = time.perf_counter() - t0
    E.collectPairs(None)
    st = E.daStats()
    out = _summary(E, wall, nsteps)
    out["stats"] = {k: st[k] - base[k] for k in st}
    out["train_s"] = t_train
    out["burn_s"] = t_burn
    # after the common burn-in; the training stays in
    out["ess_per_s_after_burn"] = out["ess"] / (wall - t_burn)
    s = out["stats"]
    out["stage1_rate"] = s["stage1_passes"] / max(s["proposals"], 1)
    out["stage2_rate"] = s["accepted"] / max(s["stage1_passes"], 1)
    if holdout is not None:
        out["surrogate_rms"] = S.rms(*holdout)
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


def posterior_agreement(a, b, free):
    """(max over free parameters of |mean_a - mean_b| / sd_b, the same in
    units of the standard error of the difference sqrt(var_a / ESS_a +
    var_b / ESS_b))."""
    ca = a["chain"].reshape(-1, a["chain"].shape[-1])[:, free].astype(np.float64)
    cb = b["chain"].reshape(-1, b["chain"].shape[-1])[:, free].astype(np.float64)
    d = np.abs(ca.mean(0) - cb.mean(0))
    se = np.sqrt(ca.var(0) / a["ess"] + cb.var(0) / b["ess"])
    return float(np.max(d / cb.std(0))), float(np.max(d / se))


def compare_two_fields_2d(ctx, nsteps, npre, nburn=150, plain_control=False,
                          train_iters=1000):
    """Plain vs delayed acceptance on the two-field 2D fit (a 1500x1500 pair
    on a 2048^2 grid and an 800x600 pair on a 1024^2 grid in one summed
    likelihood, 14 free parameters, 128 walkers).

    Both methods start from the same walkers, made untimed: a bounded Powell
    maximum of the likelihood (the synthetic maps' generating parameters lie
    several hundred log-likelihood units below it), a 1e-3 ball around it
    and npre plain steps.  Each run then burns nburn steps and records
    nsteps.  With plain_control a second plain run (another seed) gives the
    plain-vs-plain agreement the DA-vs-plain agreement is compared with."""
    from . import synth
    from .mcmc import affineEnsemble, likeSum
    from .surrogate import Surrogate
    a, b = synth.config_2d_two_fields()
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

    def ens(seed, start=None):
        E = affineEnsemble(ctx, S2, 128, npar, seed=seed)
        E.setParamFixed(npar - 2)
        E.setParamFixed(npar - 1)
        for p, (lo, hi) in enumerate(lims):
            E.setParamLimits(p, lo, hi)
        E.setErrorPolicy(True)  # unphysical corners reject instead of stop
        if start is None:
            sig = np.r_[np.full(nfree, 1e-3), 0, 0]
            E.initChains(E.generateInitialPosition(x0, sig, rng=seed))
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
                holdout=hold)
    free = list(range(nfree))
    out = {"plain": plain, "da": da, "start_loglike": lopt,
           "agreement": posterior_agreement(da, plain, free)}
    if plain_control:
        plain2 = run_plain(ens(41, start), nburn, nsteps)
        out["plain_control"] = plain2
        out["agreement_plain_control"] = posterior_agreement(plain2, plain, free)
    return out


def _main(argv=None):
    """python -m pofd_affine_b200.runner two-fields-2d --steps 1500 --pre 1000"""
    import argparse
    import json
    from . import Context
    p = argparse.ArgumentParser()
    p.add_argument("case", choices=["two-fields-2d"])
    p.add_argument("--steps", type=int, default=1500)
    p.add_argument("--pre", type=int, default=1000)
    p.add_argument("--burn", type=int, default=150)
    a = p.parse_args(argv)
    r = compare_two_fields_2d(Context(0), a.steps, a.pre, a.burn, plain_control=True)
    keep = ("wall_s", "burn_s", "tau_max", "ess", "ess_per_s", "ess_per_s_after_burn")
    summ = {"steps": a.steps, "pre": a.pre, "burn": a.burn,
            "start_loglike": r["start_loglike"],
            "plain": {k: r["plain"][k] for k in keep},
            "plain_control": {k: r["plain_control"][k] for k in keep},
            "da": {k: r["da"][k] for k in keep + ("train_s", "surrogate_rms",
                                                  "stage1_rate", "stage2_rate")},
            "da_vs_plain_shift_sigma_se": r["agreement"],
            "plain_vs_plain_shift_sigma_se": r["agreement_plain_control"],
            "ess_per_s_ratio": r["da"]["ess_per_s"] / r["plain"]["ess_per_s"],
            "ess_per_s_ratio_after_burn": (r["da"]["ess_per_s_after_burn"] /
                                           r["plain"]["ess_per_s_after_burn"])}
    print(json.dumps(summ))


if __name__ == "__main__":
    _main()
