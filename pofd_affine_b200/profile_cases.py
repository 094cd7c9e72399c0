"""Small fixed workloads to run under a profiler (one GPU, a few hundred MB
on the device, a handful of launches per kernel).

    python -m pofd_affine_b200.profile_cases 1d [--batch P] [--reps R]
    python -m pofd_affine_b200.profile_cases 2d [--batch P] [--reps R]
    python -m pofd_affine_b200.profile_cases surrogate [--batch M] [--reps R]

1d: the 1D batched configuration (n = 65536, three beam sets and maps);
2d: the 2D plain configuration (n = 2048, 1500 x 1500 map pair); both run
R likelihood batches of P proposals.  surrogate: R Adam steps of the
H = 256 network on minibatches of M pairs.
"""
import argparse
import sys


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("case", choices=["1d", "2d", "surrogate"])
    p.add_argument("--batch", type=int, default=8)
    p.add_argument("--reps", type=int, default=2)
    a = p.parse_args(argv)
    import numpy as np
    from . import Context, synth
    ctx = Context(0)
    if a.case == "1d":
        cfg = synth.config_1d_batched(seed=2)
        L = synth.build_like1(cfg, ctx)
        th = synth.proposals(cfg["theta0"], a.batch, 0.02, rng=1)
    elif a.case == "2d":
        cfg = synth.config_2d()
        L = synth.build_like2(cfg, ctx)
        th = synth.proposals(cfg["theta0"], a.batch, 0.02, rng=1,
                             fixed_last=False)
        th[:, -2:] = 1.0
    else:
        from .surrogate import Surrogate
        rng = np.random.default_rng(0)
        th = rng.normal(size=(8192, 7)).astype(np.float32)
        ll = -0.5 * (th[:, :6] ** 2).sum(1)
        S = Surrogate(ctx, 7, list(range(6)), hidden=256, seed=1)
        S.addPairs(th, ll)
        for _ in range(a.reps):
            S.train(1, a.batch)
        print("surrogate: %d Adam steps of batch %d" % (a.reps, a.batch))
        return 0
    L.reserve(a.batch)
    for _ in range(a.reps):
        ll, st = L.getLogLikeBatch(th)
    print("%s: %d batches of %d, status %s" % (a.case, a.reps, a.batch,
                                               sorted(set(st.tolist()))))
    return 0


if __name__ == "__main__":
    sys.exit(main())
