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
    base = E.daStats()
    E.doSteps(nsteps)
    wall = time.perf_counter() - t0
    st = E.daStats()
    out = _summary(E, wall, nsteps)
    out["stats"] = {k: st[k] - base[k] for k in st}
    return out


def run_da(E, S, nburn, nsteps, train_iters=2000, batch=512, lr=1e-3,
           refresh=5000, refresh_iters=300, chunk=25, holdout=None):
    """Burn-in with exact evaluations collected as training pairs, train,
    then delayed-acceptance steps in chunks, retraining after every
    `refresh` new exact evaluations.  The timed region includes the
    training.  holdout (theta, logl) gives the surrogate RMS error."""
    t0 = time.perf_counter()
    E.collectPairs(S)
    E.doSteps(0, nburn)
    t1 = time.perf_counter()
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
    s = out["stats"]
    out["stage1_rate"] = s["stage1_passes"] / max(s["proposals"], 1)
    out["stage2_rate"] = s["accepted"] / max(s["stage1_passes"], 1)
    if holdout is not None:
        out["surrogate_rms"] = S.rms(*holdout)
    return out


def posterior_agreement(a, b, free):
    """(max over free parameters of |mean_a - mean_b| / sd_b, the same in
    units of the standard error of the difference sqrt(var_a / ESS_a +
    var_b / ESS_b))."""
    ca = a["chain"].reshape(-1, a["chain"].shape[-1])[:, free].astype(np.float64)
    cb = b["chain"].reshape(-1, b["chain"].shape[-1])[:, free].astype(np.float64)
    d = np.abs(ca.mean(0) - cb.mean(0))
    se = np.sqrt(ca.var(0) / a["ess"] + cb.var(0) / b["ess"])
    return float(np.max(d / cb.std(0))), float(np.max(d / se))
