"""CPU restatement of the stretch-move ensemble and of acor -- test
infrastructure only (the product sampler is pofd_affine_b200/csrc/ensemble.cu).

  * philox4x32_10     Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11), the
                      counter-based generator the product keys by (step,
                      walker, draw), so that a CPU run reproduces a GPU run
                      draw for draw.
  * stretch_run       affineEnsemble::doMasterStep (affineEnsemble.cc:
                      1233-1284), generateNewStep (1144-1228), generateZ
                      (116-126) and the acceptance rule (1360-1433), with a
                      Python batched log-likelihood.
  * acor              affineChainSet::acor (affineChainSet.cc:884-951).
  * average_series    affineChainSet::getAverageParamVector (824-867).
"""
import math

import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF
FIXED, ACIGNORE, BONUS = 1, 2, 4
MAXITERS = 40


def philox4x32_10(ctr, key):
    c0, c1, c2, c3 = ctr
    k0, k1 = key
    for _ in range(10):
        p0 = M0 * c0
        p1 = M1 * c2
        hi0, lo0 = (p0 >> 32) & MASK, p0 & MASK
        hi1, lo1 = (p1 >> 32) & MASK, p1 & MASK
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & MASK, lo1, (hi0 ^ c3 ^ k1) & MASK, lo0
        k0 = (k0 + W0) & MASK
        k1 = (k1 + W1) & MASK
    return c0, c1, c2, c3


def draw(seed, step, walker, tag):
    return philox4x32_10((step & MASK, (step >> 32) & MASK, walker & MASK,
                          tag & MASK), (seed & MASK, (seed >> 32) & MASK))


def u01f(x):
    return np.float32(x >> 8) * np.float32(1.0 / 16777216.0)


def u01d(a, b):
    v = ((a >> 5) << 26) | (b >> 6)
    return float(v) * (1.0 / 9007199254740992.0)


def gen_z(a, x):
    val = (a - 1.0) * float(u01f(x)) + 1.0
    return np.float32(val * val / a)


def stretch_run(theta, logl, loglike_batch, nsteps, seed, scalefac=2.0,
                state=None, lo=None, hi=None, temp=1.0, step0=0,
                reject_outside=False):
    """Runs nsteps full steps from walkers theta [nw, np] (float32) with
    log-likelihoods logl; loglike_batch(thetas) -> (logl, status).  Returns
    the chain [nsteps, nw, np], its logl [nsteps, nw] and accept counts.
    reject_outside: a step outside the limits is rejected instead of
    redrawing z (the product's opt-in limit policy)."""
    theta = np.array(theta, dtype=np.float32)
    logl = np.array(logl, dtype=np.float64)
    nw, npar = theta.shape
    state = np.zeros(npar, int) if state is None else np.asarray(state)
    lo = np.full(npar, -np.inf, np.float32) if lo is None else np.asarray(lo, np.float32)
    hi = np.full(npar, np.inf, np.float32) if hi is None else np.asarray(hi, np.float32)
    nfixed = int(np.sum((state & FIXED) != 0))
    zexp = float(npar - nfixed - 1)
    nh0 = nw // 2
    chain = np.empty((nsteps, nw, npar), np.float32)
    chl = np.empty((nsteps, nw))
    nacc = np.zeros(nw, int)
    for k in range(nsteps):
        step = step0 + k
        for half in (0, 1):
            idx = range(nh0) if half == 0 else range(nh0, nw)
            pmin, prange = (nh0, nw - nh0) if half == 0 else (0, nh0)
            props, zs = [], []
            for i in idx:
                r = draw(seed, step, i, half << 16)
                j = pmin + ((r[0] * prange) >> 32)
                z = gen_z(scalefac, r[1])
                it = 0
                while True:
                    omz = np.float32(1.0) - z
                    y = np.empty(npar, np.float32)
                    ok = True
                    for p in range(npar):
                        if state[p] & FIXED:
                            y[p] = theta[i, p]
                        elif state[p] & BONUS:
                            y[p] = np.nan
                        else:
                            y[p] = np.float32(z * theta[i, p]) + np.float32(omz * theta[j, p])
                            if not (lo[p] <= y[p] <= hi[p]):
                                ok = False
                    if ok or reject_outside or it > MAXITERS:
                        break
                    z = gen_z(scalefac, draw(seed, step, i, (half << 16) | (it + 1))[0])
                    it += 1
                if not ok:
                    if not reject_outside:
                        raise RuntimeError("Unable to generate new step")
                    y = theta[i].copy()  # evaluated, then rejected
                    z = np.float32(np.nan)
                props.append(y)
                zs.append(z)
            ln, st = loglike_batch(np.array(props))
            for t, i in enumerate(idx):
                if st[t] == 1 or np.isnan(zs[t]):
                    continue
                if st[t] != 0 or not math.isfinite(ln[t]):
                    raise RuntimeError("Invalid likelihood")
                prob = math.exp(zexp * math.log(float(zs[t])) +
                                (ln[t] - logl[i]) / temp)
                if prob >= 1.0:
                    take = True
                else:
                    r = draw(seed, step, i, (half << 16) | 0x8000)
                    take = u01d(r[0], r[1]) < prob
                if take:
                    theta[i] = props[t]
                    logl[i] = ln[t]
                    nacc[i] += 1
        chain[k] = theta
        chl[k] = logl
    return chain, chl, nacc


def average_series(chain, p):
    """Walker-averaged series of parameter p (float32), summed in double
    from walker 0 upward."""
    n, nw, _ = chain.shape
    out = np.empty(n, np.float32)
    for s in range(n):
        cum = float(chain[s, 0, p])
        for k in range(1, nw):
            cum += float(chain[s, k, p])
        out[s] = np.float32((1.0 / nw) * cum)
    return out


def acor(x, L=None, maxlag=10, minfac=5, winmult=5, sigma=float("nan"),
         tau=float("nan")):
    """(mean, sigma, tau, status); x (float32) is overwritten like the
    reference's in-place recursion.  sigma and tau are the reference's
    in/out arguments: a series too short to estimate leaves them as given."""
    if L is None:
        L = len(x)
    invL = 1.0 / L
    mean = float(x[0])
    for i in range(1, L):
        mean += float(x[i])
    mean *= invL
    for i in range(L):
        x[i] = np.float32(float(x[i]) - mean)
    if L < minfac * maxlag:
        return mean, sigma, tau, 1
    C = [0.0] * (maxlag + 1)
    imax = L - maxlag
    for i in range(imax):
        for s in range(maxlag + 1):
            C[s] += float(np.float32(x[i]) * np.float32(x[i + s]))  # float product
    inv = 1.0 / imax
    C = [c * inv for c in C]
    D = C[0]
    for s in range(1, maxlag + 1):
        D += 2 * C[s]
    sigma = math.sqrt(D * invL)
    tau = D / C[0]
    if tau * winmult < maxlag:
        return mean, sigma, tau, 0
    Lh = L // 2
    for i in range(Lh):
        x[i] = np.float32(x[2 * i]) + np.float32(x[2 * i + 1])  # float sum
    _, sigma, tau, _ = acor(x, Lh, maxlag, minfac, winmult, sigma, tau)
    D = 0.25 * sigma * sigma * L
    tau = D / C[0]
    sigma = math.sqrt(D * invL)
    return mean, sigma, tau, 0
