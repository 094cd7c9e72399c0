"""Python mirror of the reference's 1D interfaces, backed by libpofd_b200.

Names and argument meanings follow aconley/pofd_affine 0.5.1:
  * beam        beam::beam(file, histogram, NBINS, MINVAL)  (beam.h:69), from
                an in-memory pixel array instead of a FITS file
  * PDFactory   initPD(n, minflux, maxflux, model, beam) / getPD(sigma, setLog)
                (PDFactory.h:136-140); the model is (knot positions, log10
                knot values)
  * calcLike    readDataFromFiles grouping by beam (calcLike.cc:688-758) from
                arrays, setRRanges(p) (calcLike.cc:827), getLogLike(p) ->
                (logL, pars_invalid) (calcLike.h:275), plus getLogLikeBatch
                for many proposals in one launch sequence.
Errors the reference raises as affineExcept surface as PofdError with the
matching POFD_E_* code.
"""
import ctypes as C
from collections import namedtuple

import numpy as np

from . import _lib
from ._lib import check, lib, PofdError  # noqa: F401

PD = namedtuple("PD", ["pd", "minflux", "dflux", "logflat"])


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Context:
    """One GPU (device >= 0) or a host-only context (device = -1)."""

    def __init__(self, device=0):
        h = C.c_void_p()
        check(lib().pofd_ctx_create(int(device), C.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            lib().pofd_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(lib().pofd_ctx_synchronize(self.h))

    def stream(self):
        s = C.c_void_p()
        check(lib().pofd_ctx_stream(self.h, C.byref(s)))
        return s.value


class beam:
    """1D beam: pixels with |value| > minval, optionally log-histogrammed."""

    def __init__(self, pix, pixsize, histogram=False, nbins=120, minval=1e-5):
        pix = _f64(pix).ravel()
        h = C.c_void_p()
        check(lib().pofd_beam1_create(pix, pix.size, float(pixsize),
                                      float(minval),
                                      int(nbins) if histogram else 0,
                                      C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().pofd_beam1_destroy(self.h)
            except Exception:  # interpreter shutdown: the library is gone
                pass
            self.h = None

    def info(self):
        o = np.empty(15)
        check(lib().pofd_beam1_info(self.h, o))
        keys = ["haspos", "hasneg", "npos", "nneg", "poshist", "neghist",
                "nposhist", "nneghist", "minpos", "maxpos", "minneg",
                "maxneg", "pixsize", "totpos", "totneg"]
        return dict(zip(keys, o))

    def hasPos(self):
        return bool(self.info()["haspos"])

    def hasNeg(self):
        return bool(self.info()["hasneg"])

    def getMinMaxPos(self):
        i = self.info()
        return i["minpos"], i["maxpos"]

    def getMinMaxNeg(self):
        i = self.info()
        return i["minneg"], i["maxneg"]

    def terms(self, negative_side=False):
        """(weights, inverse beam) the R sum runs over for one side."""
        n = C.c_size_t()
        check(lib().pofd_beam1_terms(self.h, int(negative_side), C.byref(n),
                                     None, None))
        w = np.empty(n.value)
        ie = np.empty(n.value)
        check(lib().pofd_beam1_terms(self.h, int(negative_side), C.byref(n),
                                     _lib.ptr(w), _lib.ptr(ie)))
        return w, ie


class PDFactory:
    """1D P(D) factory on the GPU (PDFactory.h)."""

    def __init__(self, ctx, ninterp=2048):
        self.ctx = ctx
        h = C.c_void_p()
        check(lib().pofd_pdfactory1_create(ctx.h, int(ninterp), C.byref(h)))
        self.h = h
        self.n = 0

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().pofd_pdfactory1_destroy(self.h)
            except Exception:  # interpreter shutdown: the library is gone
                pass
            self.h = None

    def initPD(self, n, minflux, maxflux, knotpos, knotvals, bm):
        kp, kv = _f64(knotpos), _f32(knotvals)
        check(lib().pofd_pdfactory1_initpd(self.h, int(n), float(minflux),
                                           float(maxflux), kp.size, kp, kv,
                                           bm.h))
        self.n = int(n)
        return True

    def getPD(self, sigma, setLog=True):
        out = np.empty(self.n)
        mf, df = C.c_double(), C.c_double()
        check(lib().pofd_pdfactory1_getpd(self.h, float(sigma), int(setLog),
                                          out, C.byref(mf), C.byref(df)))
        return PD(out, mf.value, df.value, bool(setLog))

    def getR(self):
        """R times dflux on the wrapped n-point grid."""
        out = np.empty(self.n)
        check(lib().pofd_pdfactory1_get_r(self.h, out))
        return out


class calcLike:
    """1D likelihood over beam sets and datasets (calcLike.h)."""

    def __init__(self, ctx, knotpos, fftsize=131072, ninterp=2048,
                 bin_data=True, nbins=1000):
        self.ctx = ctx
        self.knotpos = _f64(knotpos)
        self.nknots = self.knotpos.size
        self.fftsize = int(fftsize)
        h = C.c_void_p()
        check(lib().pofd_like1_create(ctx.h, self.nknots, self.knotpos,
                                      self.fftsize, int(ninterp),
                                      int(bin_data), int(nbins), C.byref(h)))
        self.h = h
        self.nbeamsets = 0
        self.ndatasets = []
        self._beams = []

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().pofd_like1_destroy(self.h)
            except Exception:  # interpreter shutdown: the library is gone
                pass
            self.h = None

    # ---- set-up
    def addBeamSet(self, bm, exp_conf=0.0):
        idx = check(lib().pofd_like1_add_beamset(self.h, bm.h,
                                                 float(exp_conf)))
        self._beams.append(bm)
        self.nbeamsets += 1
        self.ndatasets.append(0)
        return idx

    def addDataset(self, beamset, data, sigma_base, like_norm=1.0,
                   meansub=True):
        d = _f64(data).ravel()
        check(lib().pofd_like1_add_dataset(self.h, int(beamset), d, d.size,
                                           int(meansub), float(sigma_base),
                                           float(like_norm)))
        self.ndatasets[beamset] += 1

    def addDatasetDevice(self, beamset, data_ptr, ndata, sigma_base,
                         like_norm=1.0, meansub=True):
        """A dataset whose ndata pixels are in device memory at data_ptr
        (double; mean-subtracted in place when meansub): mean subtraction
        and binning on the GPU, bit-identical to addDataset's."""
        check(lib().pofd_like1_add_dataset_device(
            self.h, int(beamset), C.c_void_p(int(data_ptr)), int(ndata),
            int(bool(meansub)), float(sigma_base), float(like_norm)))

    def readDataFromArrays(self, datasets, beams, sigmas, like_norms=None,
                           meansub=True, exp_conf=0.0):
        """Group datasets by beam object, as readDataFromFiles groups by
        beam file (calcLike.cc:688-758).  Beam sets keep first-use order."""
        if like_norms is None:
            like_norms = [1.0] * len(datasets)
        if not (len(datasets) == len(beams) == len(sigmas) == len(like_norms)):
            raise PofdError(-10, "datasets, beams, sigmas, like_norms differ "
                                 "in length")
        index = {}
        for d, b, s, ln in zip(datasets, beams, sigmas, like_norms):
            if id(b) not in index:
                index[id(b)] = self.addBeamSet(b, exp_conf)
            self.addDataset(index[id(b)], d, s, ln, meansub)

    def readDataFromFiles(self, datafiles, beamfiles, sigmas, like_norms,
                          ignore_mask=False, meansub=False, minbeamval=1e-5,
                          histogram=False, nbeamhist=120, exp_conf=0.0):
        """calcLike::readDataFromFiles (calcLike.cc:688-758): the datasets
        grouped into beam sets by beam file, the groups in the order of their
        file names (the reference keys a std::map by them), each group's
        datasets in input order; FITS files read as fitsData::readData and
        beam::readFile.  Returns the beam set index of each dataset."""
        from . import fitsio
        n = len(datafiles)
        if n == 0:
            raise PofdError(-10, "No datafiles")
        if not (n == len(beamfiles) == len(sigmas) == len(like_norms)):
            raise PofdError(-10, "datafiles, beamfiles, sigmas, like_norms "
                                 "not same length")
        sets = {}
        for bf in sorted(set(beamfiles)):
            pix, ps = fitsio.readBeam(bf)
            sets[bf] = self.addBeamSet(beam(pix, ps, histogram, nbeamhist,
                                            minbeamval), exp_conf)
        for df, bf, s_, ln in sorted(zip(datafiles, beamfiles, sigmas,
                                         like_norms),
                                     key=lambda r: sets[r[1]]):
            self.addDataset(sets[bf], fitsio.readData(df, ignore_mask),
                            s_, ln, meansub)
        return [sets[bf] for bf in beamfiles]

    def setRRanges(self, p):
        th = _f32(p)
        check(lib().pofd_like1_set_rranges(self.h, th, th.size))

    def getR(self, beamset, p):
        """The R grid (times dflux) of a beam set for parameters p."""
        th = _f32(p)
        out = np.empty(self.fftsize)
        check(lib().pofd_like1_get_r(self.h, int(beamset), th, th.size, out))
        return out

    def getRRange(self, beamset):
        out = np.empty(2)
        check(lib().pofd_like1_get_rrange(self.h, int(beamset), out))
        return out

    def datasetInfo(self, beamset, ds):
        o = np.empty(9)
        check(lib().pofd_like1_dataset_info(self.h, int(beamset), int(ds), o,
                                            None))
        keys = ["ndata", "nbins", "bincent0", "bindelta", "like_offset",
                "sigma_base", "like_norm", "minflux", "maxflux"]
        info = dict(zip(keys, o))
        nb = int(info["nbins"])
        bins = np.zeros(nb, dtype=np.uint32)
        if nb:
            check(lib().pofd_like1_dataset_info(self.h, int(beamset), int(ds),
                                                o, _lib.ptr(bins)))
        info["bins"] = bins
        return info

    def reserve(self, max_batch):
        check(lib().pofd_like1_reserve(self.h, int(max_batch)))

    # ---- evaluation
    def getLogLike(self, p):
        th = _f32(p)
        ll = C.c_double()
        inv = C.c_int()
        check(lib().pofd_like1_loglike(self.h, th, th.size, C.byref(ll),
                                       C.byref(inv)))
        return ll.value, bool(inv.value)

    def getLogLikeBatch(self, thetas):
        th = _f32(thetas)
        if th.ndim != 2:
            raise PofdError(-10, "thetas must be [nprop, npar]")
        nprop, npar = th.shape
        ll = np.empty(nprop)
        st = np.empty(nprop, dtype=np.int32)
        check(lib().pofd_like1_eval_batch(self.h, nprop, th.ctypes.data, npar,
                                          ll.ctypes.data, st.ctypes.data))
        return ll, st

    def getLogLikeDevice(self, nprop, theta_ptr, npar, logl_ptr, status_ptr,
                         stream=None):
        """Enqueue on device pointers (ints) without synchronising."""
        check(lib().pofd_like1_eval_batch_device(
            self.h, int(nprop), C.c_void_p(theta_ptr), int(npar),
            C.c_void_p(logl_ptr), C.c_void_p(status_ptr),
            C.c_void_p(stream) if stream else None))

    def getPD(self, beamset, ds, p, setLog=True):
        th = _f32(p)
        out = np.empty(self.fftsize)
        info = np.empty(12)
        check(lib().pofd_like1_pd(self.h, int(beamset), int(ds), th, th.size,
                                  int(setLog), out, _lib.ptr(info)))
        keys = ["dflux", "minflux_R", "wrapRidx", "mn", "var_noi", "doshift",
                "shift", "splitidx", "sgpos", "sgneg", "pd_minflux", "unused"]
        return out, dict(zip(keys, info))

    def getRNodes(self, beamset, p, ninterp, negative_side=False):
        th = _f32(p)
        x = np.empty(ninterp)
        r = np.empty(ninterp)
        check(lib().pofd_like1_rnodes(self.h, int(beamset),
                                      int(negative_side), th, th.size, x, r))
        return x, r

    def profileStages(self, thetas, reps=5):
        """{stage name: mean device ms} for one launch sequence."""
        th = _f32(thetas)
        nprop, npar = th.shape
        ms = np.zeros(16)
        ns = C.c_int()
        check(lib().pofd_like1_profile(self.h, nprop, th.ravel(), npar,
                                       int(reps), ms, C.byref(ns)))
        return {lib().pofd_like1_stage_name(self.h, i).decode(): ms[i]
                for i in range(ns.value)}

    # priors (calcLike.h:251-269): added once to the summed log-likelihood
    def setSigmaPrior(self, width):
        check(lib().pofd_like1_set_sigma_prior(self.h, 1, float(width)))

    def unsetSigmaPrior(self):
        check(lib().pofd_like1_set_sigma_prior(self.h, 0, 0.0))

    def setCFIRBPrior(self, mean, sigma):
        check(lib().pofd_like1_set_cfirb_prior(self.h, 1, float(mean),
                                               float(sigma)))

    def unsetCFIRBPrior(self):
        check(lib().pofd_like1_set_cfirb_prior(self.h, 0, 0.0, 0.0))

    def setPoissonPrior(self, mean, sigma):
        check(lib().pofd_like1_set_poisson_prior(self.h, 1, float(mean),
                                                 float(sigma)))

    def unsetPoissonPrior(self):
        check(lib().pofd_like1_set_poisson_prior(self.h, 0, 0.0, 0.0))

    def setRegularizationAlpha(self, alpha):
        check(lib().pofd_like1_set_regularization(self.h, float(alpha)))

    def getBonus(self, thetas):
        """<S>, <S^2> (numberCountsKnotsSpline::getFluxPerArea /
        getFluxSqPerArea) of each row: [nprop, 2]."""
        th = _f32(thetas)
        if th.ndim == 1:
            th = th[None, :]
        th = np.ascontiguousarray(th)
        out = np.empty((th.shape[0], 2))
        check(lib().pofd_like1_bonus(self.h, th.shape[0], th.ravel(),
                                     th.shape[1], out.ravel()))
        return out

    def fillBonusParams(self, thetas):
        """calcLike::fillBonusParams on rows with nknots + 3 or more
        entries: a copy with <S>, <S^2> after the sigma multiplier (float,
        as the reference's paramSet holds them)."""
        th = np.array(_f32(thetas), copy=True)
        one = th.ndim == 1
        if one:
            th = th[None, :]
        k = len(self.knotpos)
        if th.shape[1] < k + 3:
            raise PofdError(-10, "Not enough room to fill")
        b = self.getBonus(th)
        th[:, k + 1:k + 3] = b.astype(np.float32)
        return th[0] if one else th

    TUNING_KEYS = ("own_fft", "rfill_per", "rnodes_threads", "spec_blocks",
                   "rfill_mode")

    def autotune(self, thetas, reps=20):
        """Choose the launch shapes by timing the graph-captured launch
        sequence on these rows; returns the chosen knobs with the best and
        the untuned time per launch (ms)."""
        th = np.ascontiguousarray(_f32(thetas))
        if th.ndim != 2:
            raise PofdError(-10, "thetas must be [nprop, npar]")
        out = np.zeros(7)
        check(lib().pofd_like1_autotune(self.h, th.shape[0], th.ravel(),
                                        th.shape[1], int(reps),
                                        out.ctypes.data_as(C.c_void_p)))
        d = {k: int(v) for k, v in zip(self.TUNING_KEYS, out[:5])}
        d["ms"], d["untuned_ms"] = float(out[5]), float(out[6])
        return d

    def getTuning(self):
        k = np.zeros(len(self.TUNING_KEYS), dtype=np.int32)
        check(lib().pofd_like1_get_tuning(self.h, k))
        return {n: int(v) for n, v in zip(self.TUNING_KEYS, k)}

    def setTuning(self, **knobs):
        cur = self.getTuning()
        cur.update(knobs)
        k = np.array([cur[n] for n in self.TUNING_KEYS], dtype=np.int32)
        check(lib().pofd_like1_set_tuning(self.h, k))

    def setFFT(self, mode):
        """0: own FP64 FFT where the size allows (default), 1: cuFFT."""
        check(lib().pofd_like1_set_fft(self.h, int(mode)))

    def ownFFT(self):
        v = C.c_int()
        check(lib().pofd_like1_fft_info(self.h, C.byref(v)))
        return bool(v.value)

    def kernelsPerEval(self):
        k = C.c_int()
        check(lib().pofd_like1_kernels_per_eval(self.h, C.byref(k)))
        return k.value
