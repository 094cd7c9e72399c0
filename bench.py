#!/usr/bin/env python
"""P(D)+logL evaluations per second on one B200 (or N, weak scaling).

Workload: the 1D batched configuration -- a 10-knot spline model over
1-800 mJy, three beam sets (Gaussian FWHM 3.0 / 4.2 / 6.0 px at 6", 150-bin
beam histograms) with one map each (2000x2000 at 2.0 mJy, 1200x900 at
3.1 mJy, 600x600 at 5.0 mJy noise; seeded synthetic, mean-subtracted, 1000
data bins), FFT size n = 65536, 2048 R interpolation nodes.  A step is one
launch sequence evaluating the full likelihood (all beam sets and datasets)
for a batch of 128 proposals (128 walkers); each rank evaluates its own
batch (weak scaling, no data-path collective).

    python bench.py [--gpus N] [--steps K] [--warmup W]
    python bench.py --impl reference ...   # the CPU path on host cores

Prints one JSON line (rank 0).  At N = 1 the line also carries, under
"workloads" and "mcmc", the 2D plain workload (n = 2048, 64 proposals per
launch) and the plain vs delayed-acceptance MCMC comparisons (effective
samples per second) on the 1D and the two-field 2D fits.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BATCH = 128
METRIC = "P(D)+logL evals/s"
WORKLOAD = ("1D batched plain method: 10-knot spline 1-800 mJy, 3 beam sets "
            "(FWHM 3.0/4.2/6.0 px, 150-bin beam histograms), maps 2000x2000 "
            "@2.0 mJy, 1200x900 @3.1 mJy, 600x600 @5.0 mJy, n=65536, "
            "ninterp=2048, 1000 data bins, 128 proposals per launch")


def args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cpu-seconds", type=float, default=12.0,
                   help="CPU-baseline sample length")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-2d", action="store_true")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the default launch shapes (skip the autotuner)")
    p.add_argument("--no-mcmc", action="store_true")
    p.add_argument("--no-sharded", action="store_true",
                   help="skip the walker-sharded ensemble run (N > 1)")
    p.add_argument("--mcmc-2d", type=int, default=1,
                   help="include the two-field 2D MCMC comparison")
    p.add_argument("--mcmc-steps", type=int, default=3000,
                   help="recorded steps of each 2D MCMC run")
    p.add_argument("--profile-case", choices=["1d", "2d", "surrogate"],
                   help="run a small fixed workload for a profiler and exit "
                        "(--batch proposals or pairs, --reps repetitions)")
    p.add_argument("--batch", type=int, default=8)
    p.add_argument("--reps", type=int, default=2)
    return p.parse_args()


# ------------------------------------------------------- profiler workloads
def profile_case(a):
    """Small fixed workloads to run under a profiler (one GPU, a few hundred
    MB on the device, a handful of launches per kernel).  1d: the 1D batched
    configuration (n = 65536, three beam sets and maps); 2d: the 2D plain
    configuration (n = 2048, 1500 x 1500 map pair); both run `reps`
    likelihood batches of `batch` proposals.  surrogate: `reps` Adam steps of
    the H = 256 network on minibatches of `batch` pairs."""
    from pofd_affine_b200 import Context, synth
    ctx = Context(0)
    if a.profile_case == "surrogate":
        from pofd_affine_b200.surrogate import Surrogate
        rng = np.random.default_rng(0)
        th = rng.normal(size=(8192, 7)).astype(np.float32)
        ll = -0.5 * (th[:, :6] ** 2).sum(1)
        S = Surrogate(ctx, 7, list(range(6)), hidden=256, seed=1)
        S.addPairs(th, ll)
        for _ in range(a.reps):
            S.train(1, a.batch)
        print("surrogate: %d Adam steps of batch %d" % (a.reps, a.batch))
        return
    if a.profile_case == "1d":
        cfg = synth.config_1d_batched(seed=2)
        L = synth.build_like1(cfg, ctx)
        th = synth.proposals(cfg["theta0"], a.batch, 0.02, rng=1)
    else:
        cfg = synth.config_2d()
        L = synth.build_like2(cfg, ctx)
        th = synth.proposals(cfg["theta0"], a.batch, 0.02, rng=1,
                             fixed_last=False)
        th[:, -2:] = 1.0
    L.reserve(a.batch)
    for _ in range(a.reps):
        ll, st = L.getLogLikeBatch(th)
    print("%s: %d batches of %d, status %s" % (a.profile_case, a.reps,
                                               a.batch, sorted(set(st.tolist()))))


# --------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx = [], []
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------- CPU baseline
CPU_FFT = ("radix-4 Stockham real FFT (oracle/fastfft.cc, AVX2/FMA clone "
           "when the CPU has it), the counterpart of the reference's "
           "FFTW_MEASURE plans")


def _oracle1(cfg):
    """The oracle's calcLike for the 1D workload, with the fast transforms
    of the timed CPU baseline switched on."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    pyoracle.set_fast_fft(True)
    O = pyoracle.Like1(cfg["knotpos"], cfg["fftsize"], cfg["ninterp"], True,
                       cfg["nbins"])
    for b in cfg["beams"]:
        O.add_beamset(b, cfg["pixsize"], 1e-5, True, cfg["nbeamhist"])
    for m, bi, s in zip(cfg["maps"], cfg["map_beam"], cfg["sigmas"]):
        O.add_dataset(bi, m, s)
    O.set_rranges(cfg["theta0"])
    return O


def cpu_fft_share(O, cfg, th, reps=4):
    """Share of one single-threaded CPU evaluation spent in the real
    transforms: one forward per beam set and one inverse per dataset, timed
    alone, against the evaluation."""
    import pyoracle
    n = cfg["fftsize"]
    x = np.random.default_rng(0).normal(size=n)
    X = np.fft.rfft(x)
    nb, nd = len(cfg["beams"]), len(cfg["maps"])
    O.loglike_batch(th[:1], 1)
    t0 = time.perf_counter()
    for _ in range(reps):
        O.loglike_batch(th[:1], 1)
    t_eval = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        for _ in range(nb):
            pyoracle.rfft(x)
        for _ in range(nd):
            pyoracle.irfft(X, n)
    t_fft = (time.perf_counter() - t0) / reps
    return {"eval_ms_1thread": 1e3 * t_eval, "fft_ms": 1e3 * t_fft,
            "fft_share": t_fft / t_eval}


def cpu_baseline(cfg, seconds, nthreads=None):
    """The oracle port of the reference path (calcLike::getLogLike per
    proposal) on the host cores, thread farm over proposals."""
    from pofd_affine_b200 import synth
    nthreads = nthreads or os.cpu_count() or 1
    O = _oracle1(cfg)
    th = synth.proposals(cfg["theta0"], 4 * nthreads, 0.02, rng=99)
    share = cpu_fft_share(O, cfg, th)
    O.loglike_batch(th[:nthreads], nthreads)  # builds the thread copies
    done, t0 = 0, time.perf_counter()
    while True:
        O.loglike_batch(th, nthreads)
        done += th.shape[0]
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return {"value": done / el, "unit": "evals/s", "cores": nthreads,
            "kind": "port", "fft": CPU_FFT, "fft_share_1thread": share,
            "sample": "%d proposals of the workload in %.1f s on %d threads "
                      "(oracle restatement of the reference CPU path with a "
                      "%s; the reference needs GSL/FFTW/cfitsio/HDF5/MPI, "
                      "absent here)" % (done, el, nthreads, CPU_FFT)}


def reference_arm(a, cfg):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cpu = os.cpu_count() or 1
    from pofd_affine_b200 import synth
    O = _oracle1(cfg)
    per_step = BATCH  # the GPU arm's launch: ~0.1 s of host work per step
    th = synth.proposals(cfg["theta0"], per_step, 0.02, rng=99)
    for _ in range(a.warmup):
        O.loglike_batch(th, cpu)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        O.loglike_batch(th, cpu)
    el = time.perf_counter() - t0
    v = per_step * a.steps / el
    line = {"metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": 0,
            "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * el / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD,
                       "proposals_per_step": per_step,
                       "fftsize": cfg["fftsize"],
                       "beam_sets": len(cfg["beams"]),
                       "datasets": len(cfg["maps"])},
            "cpu_baseline": {"value": v, "unit": "evals/s", "cores": cpu,
                             "kind": "port",
                             "fft": CPU_FFT,
                             "sample": "%d proposals per step, %d steps, %d "
                                       "threads (oracle restatement of the "
                                       "reference CPU path, %s)"
                                       % (per_step, a.steps, cpu, CPU_FFT)},
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- roofline
def noise_cuts(L, cfg, theta):
    """Per beam set and dataset, the own-FFT path's noise cut-off (bins k
    with min(k, m - k) > kc carry exp(-sigma^2 w_k^2 / 2) < e^-760, i.e.
    exactly 0; the same formula as the library's noise_cut), with the grid
    step of each beam set from the library and sigma = the dataset's noise
    (the proposals keep the sigma multiplier at 1)."""
    n = cfg["fftsize"]
    m = n // 2
    sets = []
    for b in range(len(cfg["beams"])):
        dflux = L.getPD(b, 0, theta, setLog=False)[1]["dflux"]
        iflux = 2 * np.pi / (n * dflux)
        kcs = []
        for d, bi in enumerate(cfg["map_beam"]):
            if bi != b:
                continue
            x = np.sqrt(1520.0) / (cfg["sigmas"][d] * iflux)
            kcs.append(m if x >= m else int(np.ceil(x)) + 1)
        sets.append(kcs)
    return sets


def stage_bytes(stage, P, B, D, n, cuts=None):
    """Algorithmic HBM bytes per launch of an HBM-bound stage (one
    compulsory FP64 read/write of each array it streams).  With the noise
    cut-offs of the own-FFT path (noise_cuts), the bins that path skips:
    forward pass B writes only bins with min(k, m - k) <= kc of the beam
    set (the widest of its datasets), the spectrum reads only those pairs
    and writes, per dataset, only the 256-bin rows the inverse pass A reads,
    and pass A reads only those rows."""
    nc = n // 2 + 1
    m = n // 2
    row = 16.0 * m  # one complex row of m points
    fwd = 4.0 * row * P * B
    spec = 8.0 * n * P * B + 8.0 * n * P * D
    inv = 4.0 * row * P * D
    if cuts is not None:
        k = np.arange(m)
        kmin = np.minimum(k, m - k)
        a = np.arange(m // 256)
        rmin = np.minimum(256 * a, m - 256 * a - 255)
        fwd = inv = spec = 0.0
        for kcs in cuts:
            kset = max(kcs) if kcs else m
            f = float(np.mean(kmin <= kset))
            fwd += P * row * (3.0 + f)
            spec += P * 32.0 * (min(kset, m // 2) + 1)
            for kc in kcs:
                g = float(np.mean(rmin <= kc))
                spec += P * row * g
                inv += P * row * (3.0 + g)
    # forward pass B alone (pass A fused with the R fill): reads the rows,
    # writes the bins inside the cut-off
    fwdB = 2.0 * row * P * B
    if cuts is not None:
        fwdB = 0.0
        for kcs in cuts:
            kset = max(kcs) if kcs else m
            fwdB += P * row * (1.0 + float(np.mean(kmin <= kset)))
    return {
        # own FFT path (n = 2m, m complex per row): passes A and B each read
        # and write the rows; the spectrum reads Z and writes one row per
        # dataset
        "k_fftA1+k_fftB1": fwd,
        "k_fftAR1": row * P * B,                              # write pass A rows
        "k_fftB1": fwdB,
        "k_spectrum1f": spec,
        "k_fftA1+k_fftB1_inv": inv,
        "k_rfill1": 8.0 * n * P * B,                         # write R
        "k_spectrum1": 16.0 * nc * P * B + 16.0 * nc * P * D,  # read R~, write per-dataset spectra
        "k_pscan1": 8.0 * n * P * D,                          # read P(D)
        "cufft_d2z": 8.0 * n * P * B + 16.0 * nc * P * B,
        "cufft_z2d": 16.0 * nc * P * D + 8.0 * n * P * D,
    }.get(stage)


def stage_flops(stage, P, B, n, rfill_mode=3):
    """Algorithmic FP64 flops per launch of the FP64-bound R-grid stages.
    One exp2 per point (fill modes 0 and 1): 35 per grid point (grid flux
    and interval offset 3, the cubic 6, the table exp2 21, the dflux scale
    1, the two moment terms 4).  Running products over runs of <= 16 points
    (modes 2 and 3): 8 per point (three products, the grid flux and the
    moment terms) plus, per run, the cubic's value and three differences at
    its first point (≈ 29) and four table exp2 (84), counted for full
    16-point runs -- 15 per point, a lower bound (runs cut at node
    intervals are shorter).  Every grid point is counted (the R range, hence
    the grid, is set to the span the spline covers).  A complex element of
    the fused forward pass A adds 5 log2(m1) (its m1-point DFT) + 12 (the
    inter-stage and outgoing twiddle products)."""
    m = n // 2
    per_pt = 35.0 if rfill_mode in (0, 1) else 8.0 + 113.0 / 16.0
    rpts = per_pt * n * P * B
    if stage == "k_rfill1":
        return rpts
    if stage == "k_fftAR1":
        return rpts + (5.0 * np.log2(m // 256) + 12.0) * m * P * B
    return None


def read_traffic(stage, per_proposal=False):
    """DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of a stage
    from the committed ncu summaries: the line
    'traffic_bytes_per_launch[<stage>]: N' -- or, for a stage captured on a
    smaller batch than the bench's and scaled by the caller,
    'traffic_bytes_per_proposal[<stage>]: N' -- in any profiles/*.md, else
    'traffic_bytes_per_launch: N' in profiles/<stage>_1d_batched.md."""
    import glob
    key = "traffic_bytes_per_%s[%s]:" % (
        "proposal" if per_proposal else "launch", stage)
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        try:
            for line in open(path):
                if line.strip().startswith(key):
                    return float(line.split("]:")[1].split()[0])
        except (OSError, ValueError):
            pass
    if per_proposal:
        return None
    path = os.path.join(ROOT, "profiles", "%s_1d_batched.md" % stage)
    try:
        for line in open(path):
            if line.strip().startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1].split()[0])
    except (OSError, ValueError):
        pass
    return None


# ------------------------------------------------------------ 2D workload
BATCH_2D = 64


def cpu_baseline_2d(cfg, seconds, nthreads=None):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from pofd_affine_b200 import synth
    pyoracle.set_fast_fft(True)
    nthreads = nthreads or os.cpu_count() or 1
    O = pyoracle.Like2(cfg["knotpos"], cfg["sigmapos"], cfg["offsetpos"],
                       cfg["fftsize"], cfg["nedge"], True, cfg["nbins"])
    O.add_beamset(cfg["beam1"], cfg["beam2"], cfg["pixsize"], cfg["minval"],
                  True, cfg["nbeamhist"])
    for (m1, m2), (s1, s2) in zip(cfg["maps"], cfg["sigmas"]):
        O.add_dataset(0, m1, m2, s1, s2)
    O.set_rranges(cfg["theta0"])
    th = synth.proposals(cfg["theta0"], nthreads, 0.02, rng=98,
                         fixed_last=False)
    th[:, -2:] = 1.0
    done, t0 = 0, time.perf_counter()
    while True:
        O.loglike_batch(th, nthreads)
        done += th.shape[0]
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return {"value": done / el, "unit": "evals/s", "cores": nthreads,
            "kind": "port",
            "fft": CPU_FFT,
            "sample": "%d proposals of the 2D workload in %.1f s on %d "
                      "threads (oracle restatement of the reference CPU path, "
                      "%s)" % (done, el, nthreads, CPU_FFT)}


def roofline_2d(L, cfg, thetas, stages, P):
    """Rooflines of the two dominant 2D kernels from the stage times.
    k_rgrid2 (FP64): every active colour term of every main-grid row is
    evaluated once per column, 25 flops each (the table exp2 21, the
    squared offset 3, the weighted add 1); the active terms per proposal
    are counted by the library for the first proposal and taken for all.
    k_colspec2 (HBM): per proposal it reads the row-transformed R spectrum
    and writes one column-transformed spectrum per dataset, 16 n (n/2+1)
    bytes each."""
    import ctypes as C
    from pofd_affine_b200._lib import support_lib
    n = cfg["fftsize"]
    nc = n // 2 + 1
    main, edge = L.activeTerms(thetas[0])
    pk = C.c_double()
    support_lib().pofd_fp64_peak(0, C.byref(pk))
    hb = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm_peak = hb.get("hbm_gbs", 6650.0)
    out = {"active_terms_per_proposal": {"main_rows": main, "edge_rows": edge}}
    ms = stages.get("k_rgrid2")
    if ms:
        flops = 25.0 * main * (n - 1) * P
        ach = flops / (ms * 1e-3) / 1e12
        tp = read_traffic("k_rgrid2", per_proposal=True)
        out["roofline_rgrid2"] = {
            "bound": "fp64", "kernel": "k_rgrid2", "ms_per_launch": ms,
            "algorithmic_flops": flops, "achieved": ach, "peak": pk.value,
            "unit": "TFLOP/s", "frac": ach / pk.value,
            "traffic": tp * P if tp else None,
            "peak_source": "measured (pofd_fp64_peak DFMA loop)"}
    ms = stages.get("k_r0sum2+k_colspec2")
    if ms:
        nds = len(cfg["maps"])
        nbytes = 16.0 * n * nc * (1 + nds) * P
        ach = nbytes / (ms * 1e-3) / 1e9
        tp = read_traffic("k_colspec2", per_proposal=True)
        out["roofline_colspec2"] = {
            "bound": "hbm", "kernel": "k_r0sum2+k_colspec2", "ms_per_launch": ms,
            "algorithmic_bytes": nbytes, "achieved": ach, "peak": hbm_peak,
            "unit": "GB/s", "frac": ach / hbm_peak,
            "traffic": tp * P if tp else None,
            "peak_source": "measured" if "hbm_gbs" in hb else "fallback"}
    return out


def measure_2d(a, ctx, stream):
    import torch
    from pofd_affine_b200 import synth
    cfg = synth.config_2d()
    L = synth.build_like2(cfg, ctx)
    L.reserve(BATCH_2D)
    npar = cfg["theta0"].size
    host = []
    for k in range(2):
        t = synth.proposals(cfg["theta0"], BATCH_2D, 0.02, rng=300 + k,
                            fixed_last=False)
        t[:, -2:] = 1.0
        host.append(t)
    dth = [torch.from_numpy(h).cuda() for h in host]
    dll = torch.empty(BATCH_2D, dtype=torch.float64, device="cuda")
    dst = torch.empty(BATCH_2D, dtype=torch.int32, device="cuda")
    sptr = stream.cuda_stream
    ref, st = L.getLogLikeBatch(host[0])
    assert np.all(st == 0), st
    tuning = L.autotune(host[0], reps=3) if not a.no_autotune else L.getTuning()
    steps = max(3, a.steps // 50)
    for k in range(max(a.warmup, 3)):
        L.getLogLikeDevice(BATCH_2D, dth[k % 2].data_ptr(), npar,
                           dll.data_ptr(), dst.data_ptr(), sptr)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(steps):
        L.getLogLikeDevice(BATCH_2D, dth[k % 2].data_ptr(), npar,
                           dll.data_ptr(), dst.data_ptr(), sptr)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    t0 = time.perf_counter()
    for k in range(steps):
        L.getLogLikeBatch(host[k % 2])
    e2e_s = time.perf_counter() - t0
    stages = L.profileStages(host[0], reps=3)
    roof = roofline_2d(L, cfg, host[0], stages, BATCH_2D)
    out = {"workload": "2D plain method: 8-knot counts 2-500 mJy, log-normal "
                       "colour (3 sigma + 3 offset knots), FWHM 3.0/4.2 px "
                       "beams in 100-bin 2D histograms, 1500x1500 map pair, "
                       "500x500 data bins, n=2048, nedge=256, 64 proposals "
                       "per launch",
           "value": BATCH_2D * steps / (ms * 1e-3), "unit": "evals/s",
           "steps": steps, "ms_per_step": ms / steps,
           "e2e": {"value": BATCH_2D * steps / e2e_s, "unit": "evals/s",
                   "h2d_bytes_per_step": BATCH_2D * npar * 4,
                   "d2h_bytes_per_step": BATCH_2D * 12},
           "stage_ms": stages, "gpu_launches": L.kernelsPerEval() * steps,
           "autotune": tuning}
    out.update(roof)
    if not a.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_2d(cfg, a.cpu_seconds)
    return out


# ---------------------------------------------------------------- MCMC
def _device_ms(fn, reps=50):
    """Mean device time of fn() (which enqueues on torch's current stream)
    by CUDA events, after one warm call."""
    import torch
    fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def setup_times(ctx, cfg, cfg2=None):
    """Set-up cost of the data maps: mean subtraction and binning on the
    host (addDataset from host arrays) against the GPU path (one H2D copy of
    the pixels, then addDatasetDevice), for the 2000x2000 map of the 1D
    workload and the 1500x1500 pair of the 2D one; both give identical bins
    (the GPU tests check that).  Wall-clock seconds, best of three."""
    import torch
    from pofd_affine_b200 import beam, calcLike
    m = np.ascontiguousarray(cfg["maps"][0], np.float64).ravel()
    pinned = torch.from_numpy(m).pin_memory()
    b = beam(cfg["beams"][0], cfg["pixsize"], True, cfg["nbeamhist"], 1e-5)

    def fresh():
        L = calcLike(ctx, cfg["knotpos"], cfg["fftsize"], cfg["ninterp"], True,
                     cfg["nbins"])
        L.addBeamSet(b)
        return L
    t_host, t_dev = [], []
    for _ in range(3):
        L = fresh()
        t0 = time.perf_counter()
        L.addDataset(0, m, cfg["sigmas"][0])
        t_host.append(time.perf_counter() - t0)
        L = fresh()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d = pinned.to("cuda", non_blocking=True)
        torch.cuda.synchronize()
        L.addDatasetDevice(0, d.data_ptr(), d.numel(), cfg["sigmas"][0])
        t_dev.append(time.perf_counter() - t0)
    out = {"map_2000x2000": {"host_s": min(t_host), "gpu_s": min(t_dev),
                             "pixels": int(m.size), "nbins": cfg["nbins"]}}
    if cfg2 is not None:
        from pofd_affine_b200.api2d import calcLikeDouble, doublebeam
        (m1, m2), (s1, s2) = cfg2["maps"][0], cfg2["sigmas"][0]
        a1 = np.ascontiguousarray(m1, np.float64).ravel()
        a2 = np.ascontiguousarray(m2, np.float64).ravel()
        p1, p2 = torch.from_numpy(a1).pin_memory(), torch.from_numpy(a2).pin_memory()
        bm = doublebeam(cfg2["beam1"], cfg2["beam2"], cfg2["pixsize"], True,
                        cfg2["nbeamhist"], cfg2["minval"])

        def fresh2():
            L2 = calcLikeDouble(ctx, cfg2["knotpos"], cfg2["sigmapos"],
                                cfg2["offsetpos"], cfg2["fftsize"], cfg2["nedge"],
                                True, cfg2["nbins"])
            L2.addBeamSet(bm)
            return L2
        t_host, t_dev = [], []
        for _ in range(3):
            L2 = fresh2()
            t0 = time.perf_counter()
            L2.addDataset(0, a1, a2, s1, s2)
            t_host.append(time.perf_counter() - t0)
            L2 = fresh2()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            d1 = p1.to("cuda", non_blocking=True)
            d2 = p2.to("cuda", non_blocking=True)
            torch.cuda.synchronize()
            L2.addDatasetDevice(0, d1.data_ptr(), d2.data_ptr(), d1.numel(), s1, s2)
            t_dev.append(time.perf_counter() - t0)
        out["pair_1500x1500"] = {"host_s": min(t_host), "gpu_s": min(t_dev),
                                 "pixels": int(a1.size),
                                 "nbins": "%dx%d" % (cfg2["nbins"], cfg2["nbins"])}
    return out


def sharded_ensemble(a, ctx, L, cfg, rk):
    """One 128-walker stretch-move ensemble over the 1D workload's
    likelihood with each half-step's 64 proposals split over the ranks
    (shardedLike: each rank its rows, one NCCL all-gather of logL and
    status), every rank running the same ensemble.  Reports steps/s (the
    slowest rank's time) and whether the recorded chains are identical on
    every rank (a checksum reduced with min and max over ranks)."""
    import torch
    from pofd_affine_b200.mcmc import affineEnsemble
    from pofd_affine_b200.shard import shardedLike
    S = shardedLike(ctx, L)
    npar = cfg["theta0"].size
    E = affineEnsemble(ctx, S, 128, npar, seed=123)
    E.setParamFixed(npar - 1)
    E.initChains(E.generateInitialPosition(cfg["theta0"], 0.02, rng=7))
    E.doSteps(0, max(a.warmup, 3))
    E.sync()
    rk.barrier()
    nsteps = 20
    t0 = time.perf_counter()
    E.doSteps(nsteps)
    E.sync()
    dt = rk.max_over_ranks(time.perf_counter() - t0)
    ch, cl = E.getChain()
    h = float(np.sum(ch.astype(np.float64) * np.arange(1, ch.size + 1).reshape(ch.shape))
              + np.sum(cl))
    lo = -rk.max_over_ranks(-h)
    hi = rk.max_over_ranks(h)
    del E, S
    torch.cuda.synchronize()
    return {"workload": "128 walkers on the 1D batched workload, 64 proposals "
                        "per half-step split over %d ranks" % rk.world,
            "steps": nsteps, "steps_per_s": nsteps / dt,
            "evals_per_s": 128 * nsteps / dt,
            "chains_identical_on_all_ranks": bool(lo == hi),
            "scaling": "strong (one ensemble)"}


def mcmc_1d(ctx, cpu=True):
    """Plain vs delayed-acceptance stretch move on the 1D plain fit (6
    knots, n = 4096, 40 walkers, fixed burn 200, 500 recorded steps), with
    the cost of one half-ensemble's exact likelihood and of its surrogate
    screening (the 1D exact step is latency-bound, so the screening cannot
    save much)."""
    import ctypes as C
    import torch
    from pofd_affine_b200 import runner, synth
    from pofd_affine_b200._lib import lib
    from pofd_affine_b200.mcmc import affineEnsemble
    from pofd_affine_b200.surrogate import Surrogate
    cfg = synth.config_1d_small(seed=1)
    L = synth.build_like1(cfg, ctx)
    npar = cfg["theta0"].size
    nk = npar - 1
    # launch shapes for the half-ensemble batches the runs evaluate (at this
    # size cuFFT can beat the own FFT)
    tuning = L.autotune(synth.proposals(cfg["theta0"], 20, 0.02, rng=3), reps=20)

    def ens(seed):
        E = affineEnsemble(ctx, L, 40, npar, seed=seed)
        E.setParamFixed(nk)
        for p in range(nk):  # knot limits of an initialisation file
            E.setParamLimits(p, cfg["theta0"][p] - 2.0, cfg["theta0"][p] + 2.0)
        E.initChains(E.generateInitialPosition(cfg["theta0"], 0.05, rng=seed))
        return E
    plain = runner.run_plain(ens(21), 200, 500)
    ch = plain["chain"].reshape(-1, npar)
    rng = np.random.default_rng(0)
    pick = rng.choice(ch.shape[0], 2000, replace=False)
    hold = (ch[pick], plain["logl"].reshape(-1)[pick])
    S = Surrogate(ctx, npar, list(range(nk)), hidden=256, seed=7)
    da = runner.run_da(ens(22), S, 200, 500, train_iters=1000, holdout=hold)
    out = _mcmc_summary("1D plain fit: 6 knots 2-400 mJy, n=4096, one "
                        "256x256 map, 40 walkers, burn 200, 500 steps; MLP "
                        "6 -> 3x256 SiLU -> 1", plain, da, list(range(nk)))
    # one half-ensemble (20 proposals): exact likelihood vs surrogate
    th = torch.from_numpy(np.ascontiguousarray(ch[:20])).cuda()
    ll = torch.empty(20, dtype=torch.float64, device="cuda")
    st = torch.empty(20, dtype=torch.int32, device="cuda")
    sp = torch.cuda.current_stream().cuda_stream
    exact_ms = _device_ms(lambda: L.getLogLikeDevice(
        20, th.data_ptr(), npar, ll.data_ptr(), st.data_ptr(), sp))
    sur_ms = _device_ms(lambda: lib().pofd_surrogate_predict_device(
        S.h, 20, C.c_void_p(th.data_ptr()), npar, C.c_void_p(ll.data_ptr()),
        C.c_void_p(st.data_ptr()), C.c_void_p(sp)))
    out["half_step_ms"] = {"exact_20": exact_ms, "surrogate_20": sur_ms}
    out["autotune"] = tuning
    if cpu:
        c = cpu_mcmc_1d()
        c["gpu_plain_ess_per_s_ratio"] = out["plain"]["ess_per_s"] / c["ess_per_s"]
        out["cpu_plain"] = c
    return out


def cpu_mcmc_1d(nthreads=None, nburn=200, nsteps=500, nwalkers=40):
    """The plain stretch move of mcmc_1d on the host: the oracle's sampler
    (the same Philox draws and acceptance rule as the GPU ensemble) over the
    oracle port's likelihood, each half-ensemble's proposals farmed over
    nthreads host threads (the reference's master/worker farm), the same
    walkers, limits, burn-in and recorded steps as the GPU plain run, ESS
    from the same estimator.  Reported twice: over the whole wall time, and
    over the time spent inside the likelihood calls only (the share a
    compiled sampler could not avoid)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sampler_oracle as so
    from pofd_affine_b200 import synth
    from pofd_affine_b200.mcmc import integrated_time
    nthreads = nthreads or os.cpu_count() or 1
    cfg = synth.config_1d_small(seed=1)
    O = _oracle1(cfg)
    th0 = np.asarray(cfg["theta0"], np.float32)
    npar = th0.size
    nk = npar - 1
    state = np.zeros(npar, int)
    state[nk] = so.FIXED
    lo = np.full(npar, -np.inf, np.float32)
    hi = np.full(npar, np.inf, np.float32)
    lo[:nk], hi[:nk] = th0[:nk] - 2.0, th0[:nk] + 2.0
    # the walkers of affineEnsemble.generateInitialPosition(theta0, 0.05,
    # rng=21): the same draws in the same order
    rng = np.random.default_rng(21)
    w = np.empty((nwalkers, npar), np.float32)
    for k in range(nwalkers):
        for p in range(npar):
            if state[p] & so.FIXED:
                w[k, p] = th0[p]
                continue
            while True:
                v = np.float32(th0[p] + 0.05 * rng.standard_normal())
                if lo[p] <= v <= hi[p]:
                    break
            w[k, p] = v
    t_like = [0.0]

    def like(th):
        t = time.perf_counter()
        r = O.loglike_batch(np.ascontiguousarray(th, np.float32), nthreads)
        t_like[0] += time.perf_counter() - t
        return r

    like(w[:nthreads])  # builds the thread copies (untimed)
    t_like[0] = 0.0
    t0 = time.perf_counter()
    ll, st = like(w)
    ch, cl, _ = so.stretch_run(w, ll, like, nburn, 21, state=state, lo=lo,
                               hi=hi)
    ch, cl, nacc = so.stretch_run(ch[-1], cl[-1], like, nsteps, 21,
                                  state=state, lo=lo, hi=hi, step0=nburn)
    wall = time.perf_counter() - t0
    tau, _, conv = integrated_time(ch)
    tau[nk] = np.nan
    tmax = float(np.nanmax(tau))
    ess = nwalkers * nsteps / tmax
    return {"workload": "the 1D plain fit of mcmc_1d on the host: %d walkers, "
                        "burn %d, %d recorded steps" % (nwalkers, nburn, nsteps),
            "kind": "port", "cores": nthreads,
            "sample": "oracle sampler (Python) over the oracle port's "
                      "likelihood with a %s, each half-ensemble farmed over "
                      "%d threads" % (CPU_FFT, nthreads),
            "wall_s": wall, "likelihood_s": t_like[0],
            "evals": nwalkers * (nburn + nsteps + 1),
            "tau_max": tmax, "tau_converged": bool(np.all(conv[:nk])),
            "acceptance": float(np.mean(nacc)) / nsteps,
            "ess": ess, "ess_per_s": ess / wall,
            "ess_per_s_likelihood_only": ess / t_like[0]}


def mcmc_2d(ctx, nsteps=3000):
    """Plain vs delayed acceptance on the two-field 2D fit (2048^2 and
    1024^2 grids in one launch, 14 free parameters, 128 walkers), from a
    shared equilibrated start, with a plain-vs-plain control
    (runner.compare_two_fields_2d, runner.summarise)."""
    from pofd_affine_b200 import runner
    npre = 2000  # ~10 autocorrelation times: a shared start at equilibrium
    r = runner.compare_two_fields_2d(ctx, nsteps, npre, plain_control=True)
    out = runner.summarise(r)
    out["workload"] = ("2D two-field fit: 1500x1500 pair on 2048^2 + 800x600 "
                       "pair on 1024^2 in one launch, 14 free parameters, "
                       "128 walkers, shared start (Powell maximum, walkers "
                       "from its Laplace approximation, %d plain steps, "
                       "untimed), burn %d steps (20k exact pairs), %d "
                       "recorded steps; DA: MLP 14 -> 3x384 SiLU -> 1 trained "
                       "on the burn-in pairs, retrained every 5k exact "
                       "evaluations, stretch a = %g (plain a = 2); every "
                       "run rejects steps outside the parameter limits"
                       % (npre, -(-runner.DA_PAIRS // 128), nsteps,
                          runner.DA_SCALE_2D))
    return out


def _mcmc_summary(name, plain, da, free):
    from pofd_affine_b200 import runner
    shift = runner.posterior_agreement(da, plain, free)
    keep = runner.SUMMARY_KEYS + ("stats",)
    return {"workload": name,
            "plain": {k: plain[k] for k in keep},
            "da": dict({k: da[k] for k in keep},
                       **{k: da[k] for k in runner.DA_KEYS if k in da}),
            "ess_per_s_ratio": da["ess_per_s"] / plain["ess_per_s"],
            # both methods share the burn-in; after it, DA's time includes
            # its training
            "ess_per_s_ratio_after_burn": (da["ess_per_s_after_burn"] /
                                           plain["ess_per_s_after_burn"]),
            "posterior_mean_shift_sigma": shift[0],
            "posterior_mean_shift_se": shift[1]}


def main():
    a = args()
    if a.profile_case:
        profile_case(a)
        return
    from pofd_affine_b200 import synth
    cfg = synth.config_1d_batched(seed=2)
    if a.impl == "reference":
        reference_arm(a, cfg)
        return

    import torch
    from pofd_affine_b200.ranks import Ranks
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rk = Ranks("nccl")
    rank, world, local = rk.rank, rk.world, rk.local
    from pofd_affine_b200 import Context, build
    build.build()
    from pofd_affine_b200._lib import support_lib
    import ctypes as C

    ctx = Context(local)
    L = synth.build_like1(cfg, ctx)
    L.reserve(BATCH)
    npar = cfg["theta0"].size
    nbatches = 4  # distinct resident proposal batches, cycled
    host = [synth.proposals(cfg["theta0"], BATCH, 0.02, rng=rk.proposal_seed(k))
            for k in range(nbatches)]
    # launch shapes chosen by the library's autotuner on this workload
    tuning = L.autotune(host[0], reps=10) if not a.no_autotune else L.getTuning()
    dth = [torch.from_numpy(h).cuda() for h in host]
    dll = [torch.empty(BATCH, dtype=torch.float64, device="cuda")
           for _ in range(nbatches)]
    dst = [torch.empty(BATCH, dtype=torch.int32, device="cuda")
           for _ in range(nbatches)]
    # a dedicated stream: the library reads a NULL stream as "the context's
    # own stream", so the events must sit on the stream we pass
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream

    def step(k):
        j = k % nbatches
        L.getLogLikeDevice(BATCH, dth[j].data_ptr(), npar, dll[j].data_ptr(),
                           dst[j].data_ptr(), sptr)

    # correctness gate: device path equals the host path, all statuses ok
    ref_ll, ref_st = L.getLogLikeBatch(host[0])
    step(0)
    torch.cuda.synchronize()
    assert np.all(ref_st == 0), ref_st
    assert np.array_equal(dll[0].cpu().numpy(), ref_ll)

    for k in range(max(a.warmup, 3)):
        step(k)
    torch.cuda.synchronize()
    rk.barrier()
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(a.steps):
        step(k)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = rk.max_over_ranks(e0.elapsed_time(e1))
    value = rk.throughput(BATCH * a.steps, ms * 1e-3)

    # end to end through the public API with host buffers
    L.getLogLikeBatch(host[1])
    rk.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(a.steps):
        L.getLogLikeBatch(host[k % nbatches])
    torch.cuda.synchronize()
    e2e_s = rk.max_over_ranks(time.perf_counter() - t0)
    e2e = rk.throughput(BATCH * a.steps, e2e_s)

    # per-stage device times of the same launch sequence (CUDA events)
    stages = L.profileStages(host[0], reps=5)
    own = {k: v for k, v in stages.items() if k.startswith("k_")}
    dom = max(own, key=own.get)
    B, D, n = 3, 3, cfg["fftsize"]
    hb = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm_peak = hb.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in hb else "fallback"
    cuts = noise_cuts(L, cfg, cfg["theta0"]) if L.ownFFT() else None
    nbytes = stage_bytes(dom, BATCH, B, D, n, cuts)
    rmode = L.getTuning()["rfill_mode"]
    nflops = stage_flops(dom, BATCH, B, n, rmode)

    def fp64_roof(k):
        # FP64-bound R grid fill (fused with the forward pass A): algorithmic
        # FP64 flops against the measured FP64 FMA peak
        fl = stage_flops(k, BATCH, B, n, rmode)
        pk = C.c_double()
        support_lib().pofd_fp64_peak(local, C.byref(pk))
        ach = fl / (own[k] * 1e-3) / 1e12
        return {"bound": "fp64", "kernel": k, "ms_per_launch": own[k],
                "achieved": ach, "peak": pk.value, "unit": "TFLOP/s",
                "frac": ach / pk.value,
                "peak_source": "measured (pofd_fp64_peak DFMA loop)",
                "algorithmic_flops": fl,
                "flops_basis": ("R fill by running products: 15 FP64 flops per "
                                "grid point (three products, grid flux and moment "
                                "terms, per-run set-up amortised)"
                                if rmode >= 2 else
                                "R fill with one table exp2 per grid point: 35 "
                                "FP64 flops per point")
                               + ("; plus the pass-A DFT, 5 log2(m1) + 12 per "
                                  "complex element" if k == "k_fftAR1" else ""),
                # the run-based fills have their own captures
                "traffic": read_traffic(k + ("@runs" if rmode >= 2 else ""))}

    if nflops is not None:
        roof = fp64_roof(dom)
    elif nbytes is not None:
        ach = nbytes / (own[dom] * 1e-3) / 1e9
        traffic = read_traffic(dom)
        roof = {"bound": "hbm", "kernel": dom, "achieved": ach,
                "peak": hbm_peak, "unit": "GB/s", "frac": ach / hbm_peak,
                "traffic": traffic, "algorithmic_bytes": nbytes,
                "ms_per_launch": own[dom], "peak_source": peak_src}
    else:
        # FP64-bound R builder: FP64 flops of the R terms against the
        # measured FP64 FMA peak
        pk = C.c_double()
        support_lib().pofd_fp64_peak(local, C.byref(pk))
        roof = {"bound": "fp64", "kernel": dom, "ms_per_launch": own[dom],
                "peak": pk.value, "unit": "TFLOP/s",
                "peak_source": "measured (pofd_fp64_peak DFMA loop)",
                "achieved": None, "frac": None,
                "traffic": read_traffic(dom)}
    # the longest HBM-bound stage beside it (the dominant one is FP64 bound)
    hbm_stages = {k: v for k, v in own.items()
                  if stage_flops(k, BATCH, B, n, rmode) is None
                  and stage_bytes(k, BATCH, B, D, n, cuts) is not None}
    roof_hbm = None
    if hbm_stages:
        hs = max(hbm_stages, key=hbm_stages.get)
        hb_bytes = stage_bytes(hs, BATCH, B, D, n, cuts)
        ach_h = hb_bytes / (own[hs] * 1e-3) / 1e9
        roof_hbm = {"bound": "hbm", "kernel": hs, "achieved": ach_h,
                    "peak": hbm_peak, "unit": "GB/s", "frac": ach_h / hbm_peak,
                    "algorithmic_bytes": hb_bytes, "ms_per_launch": own[hs],
                    "peak_source": peak_src}
    # the longest FP64-bound stage beside it (the dominant one is HBM bound)
    fp_stages = {k: v for k, v in own.items()
                 if stage_flops(k, BATCH, B, n, rmode) is not None}
    roof_fp64 = None
    if fp_stages:
        fs = max(fp_stages, key=fp_stages.get)
        if fs != dom:
            roof_fp64 = fp64_roof(fs)
    hbm_pipe = sum(stage_bytes(s, BATCH, B, D, n, cuts) or 0 for s in stages)
    nk = L.kernelsPerEval()

    extra = {}
    if world > 1 and not a.no_sharded:
        # every rank takes part (collectives); rank 0 reports
        sh = sharded_ensemble(a, ctx, L, cfg, rk)
        if rank == 0:
            extra["sharded_ensemble"] = sh
    if rank == 0 and world == 1:
        if not a.no_2d:
            extra["workloads"] = {"2d": measure_2d(a, ctx, stream)}
        from pofd_affine_b200 import synth as _s
        extra["setup"] = setup_times(ctx, cfg, None if a.no_2d else _s.config_2d())
        if not a.no_mcmc:
            extra["mcmc"] = {"1d": mcmc_1d(ctx, cpu=not a.no_cpu_baseline)}
            if a.mcmc_2d:
                extra["mcmc"]["2d_two_fields"] = mcmc_2d(ctx, a.mcmc_steps)

    if rank == 0:
        cpu = None
        if not a.no_cpu_baseline and world == 1:
            cpu = cpu_baseline(cfg, a.cpu_seconds)
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded maps of the workload's shapes)",
            "config": {"workload": WORKLOAD, "proposals_per_step": BATCH,
                       "fftsize": n, "beam_sets": B, "datasets": D,
                       "autotune": tuning,
                       "l2": "working set per step ~400 MB > 126 MB L2 "
                             "(no flush needed)"},
            "e2e": {"value": e2e, "unit": "evals/s",
                    "h2d_bytes_per_step": BATCH * npar * 4,
                    "d2h_bytes_per_step": BATCH * (8 + 4)},
            "roofline": roof,
            "roofline_hbm_stage": roof_hbm,
            "roofline_fp64_stage": roof_fp64,
            "stage_ms": stages,
            "pipeline_hbm_bytes_per_step": hbm_pipe,
            "gpu_launches": nk * a.steps,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    rk.close()


if __name__ == "__main__":
    main()
