"""Python mirror of the reference's 2D (two-band) interfaces.

  * PDFactoryDouble PDFactoryDouble::initPD / getPD (PDFactoryDouble.h:142-148)
  * doublebeam      doublebeam::doublebeam(file1, file2, histogram, NBINS,
                    MINVAL) (doublebeam.h:81) from two in-memory pixel arrays
  * calcLikeDouble  calcLikeDouble (calcLikeDouble.h:192-347) with the
                    log-normal colour model: setRRanges(p), getLogLike(p) ->
                    (logL, pars_invalid), getLogLikeBatch, getPD, getR.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib, PofdError  # noqa: F401


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class doublebeam:
    """Two-band beam split into pp/pn/np/nn sign components."""

    def __init__(self, pix1, pix2, pixsize, histogram=False, nbins=150,
                 minval=1e-6):
        p1, p2 = _f64(pix1).ravel(), _f64(pix2).ravel()
        if p1.size != p2.size:
            raise PofdError(-10, "beams must have the same size")
        h = C.c_void_p()
        check(lib().pofd_beam2_create(p1, p2, p1.size, float(pixsize),
                                      float(minval),
                                      int(nbins) if histogram else 0,
                                      C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().pofd_beam2_destroy(self.h)
            except Exception:  # interpreter shutdown: the library is gone
                pass
            self.h = None

    def info(self):
        o = np.empty(17)
        check(lib().pofd_beam2_info(self.h, o))
        return {"hassign": o[0:4].astype(bool), "npix": o[4:8].astype(int),
                "ishist": o[8:12].astype(bool), "nhist": o[12:16].astype(int),
                "pixsize": o[16]}


class PDFactoryDouble:
    """2D P(D) factory on the GPU (PDFactoryDouble.h)."""

    def __init__(self, ctx, nedge=256):
        h = C.c_void_p()
        check(lib().pofd_pdfactory2_create(ctx.h, int(nedge), C.byref(h)))
        self.h, self.ctx, self.n = h, ctx, 0

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().pofd_pdfactory2_destroy(self.h)
            except Exception:  # interpreter shutdown: the library is gone
                pass
            self.h = None

    def initPD(self, n, minflux1, maxflux1, minflux2, maxflux2, knotpos,
               sigmapos, offsetpos, params, bm, setEdge=True):
        k, sg, o = _f64(knotpos), _f64(sigmapos), _f64(offsetpos)
        check(lib().pofd_pdfactory2_initpd(
            self.h, int(n), float(minflux1), float(maxflux1), float(minflux2),
            float(maxflux2), k.size, k, sg.size, sg, o.size, o, _f32(params),
            bm.h, int(bool(setEdge))))
        self.n = int(n)
        self._beam = bm
        return True

    def getPD(self, sigma1, sigma2, setLog=True):
        out = np.empty(self.n * self.n)
        info = np.empty(4)
        check(lib().pofd_pdfactory2_getpd(self.h, float(sigma1), float(sigma2),
                                          int(setLog), out, info))
        return out.reshape(self.n, self.n), dict(zip(
            ["minflux1", "dflux1", "minflux2", "dflux2"], info))

    def getR(self):
        out = np.empty(self.n * self.n)
        check(lib().pofd_pdfactory2_get_r(self.h, out))
        return out.reshape(self.n, self.n)


class calcLikeDouble:
    """2D likelihood over beam sets and datasets."""

    def __init__(self, ctx, knotpos, sigmapos, offsetpos, fftsize=4096,
                 nedge=256, edge_integ=True, nbins=1000, bin_data=True):
        self.ctx = ctx
        k, s, o = _f64(knotpos), _f64(sigmapos), _f64(offsetpos)
        self.nmodel = k.size + s.size + o.size
        self.fftsize = int(fftsize)
        h = C.c_void_p()
        check(lib().pofd_like2_create(ctx.h, k.size, k, s.size, s, o.size, o,
                                      self.fftsize, int(nedge),
                                      int(edge_integ), int(bool(bin_data)),
                                      int(nbins), C.byref(h)))
        self.h = h
        self._beams = []

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().pofd_like2_destroy(self.h)
            except Exception:  # interpreter shutdown: the library is gone
                pass
            self.h = None

    def addBeamSet(self, bm, exp_conf1=0.0, exp_conf2=0.0):
        idx = check(lib().pofd_like2_add_beamset(self.h, bm.h,
                                                 float(exp_conf1),
                                                 float(exp_conf2)))
        self._beams.append(bm)
        return idx

    def addDataset(self, beamset, data1, data2, sigma1, sigma2,
                   like_norm=1.0, meansub=True):
        a, b = _f64(data1).ravel(), _f64(data2).ravel()
        if a.size != b.size:
            raise PofdError(-10, "band maps differ in size")
        check(lib().pofd_like2_add_dataset(self.h, int(beamset), a, b, a.size,
                                           int(meansub), float(sigma1),
                                           float(sigma2), float(like_norm)))

    def addDatasetDevice(self, beamset, d1_ptr, d2_ptr, ndata, sigma1, sigma2,
                         like_norm=1.0, meansub=True):
        """A two-band dataset whose ndata pixels per band are in device
        memory (double; mean-subtracted in place when meansub): mean
        subtraction and 2D binning on the GPU, bit-identical to
        addDataset's."""
        check(lib().pofd_like2_add_dataset_device(
            self.h, int(beamset), C.c_void_p(int(d1_ptr)), C.c_void_p(int(d2_ptr)),
            int(ndata), int(bool(meansub)), float(sigma1), float(sigma2),
            float(like_norm)))

    def readDataFromFiles(self, datafiles1, datafiles2, beamfiles1, beamfiles2,
                          sigmas1, sigmas2, like_norms, ignore_mask=False,
                          meansub=False, minbeamval=1e-6, histogram=False,
                          nbeamhist=150, exp_conf1=0.0, exp_conf2=0.0):
        """calcLikeDouble::readDataFromFiles (calcLikeDouble.cc:932-1030):
        datasets grouped into beam sets by the pair of beam files (key
        "file1:file2", groups in key order as the reference's std::map),
        each group's datasets in input order; the two bands' maps read as
        fitsDataDouble::readData, the beams as doublebeam's.  Returns the
        beam set index of each dataset."""
        from . import fitsio
        n = len(datafiles1)
        if n != len(datafiles2):
            raise PofdError(-10, "Datafiles1 and datafile2 not same length")
        if n == 0:
            raise PofdError(-10, "No datafiles")
        if not (n == len(beamfiles1) == len(beamfiles2) == len(sigmas1)
                == len(sigmas2) == len(like_norms)):
            raise PofdError(-10, "datafiles, beamfiles, sigmas, like_norms "
                                 "not same length")
        keys = [b1 + ":" + b2 for b1, b2 in zip(beamfiles1, beamfiles2)]
        sets = {}
        for k in sorted(set(keys)):
            i = keys.index(k)
            p1, ps1 = fitsio.readBeam(beamfiles1[i])
            p2, ps2 = fitsio.readBeam(beamfiles2[i])
            if abs((ps1 - ps2) / ps1) > 1e-5:  # doublebeam.cc:263-270
                raise PofdError(-10, "Pixel scale in %s doesn't match that of %s"
                                % (beamfiles2[i], beamfiles1[i]))
            sets[k] = self.addBeamSet(doublebeam(p1, p2, ps1, histogram,
                                                 nbeamhist, minbeamval),
                                      exp_conf1, exp_conf2)
        order = sorted(range(n), key=lambda i: sets[keys[i]])
        for i in order:
            d1, d2 = fitsio.readData2(datafiles1[i], datafiles2[i], ignore_mask)
            self.addDataset(sets[keys[i]], d1, d2, sigmas1[i], sigmas2[i],
                            like_norms[i], meansub)
        return [sets[k] for k in keys]

    def setRRanges(self, p):
        th = _f32(p)
        check(lib().pofd_like2_set_rranges(self.h, th, th.size))

    def getRRange(self, beamset):
        out = np.empty(4)
        check(lib().pofd_like2_get_rrange(self.h, int(beamset), out))
        return out

    def datasetInfo(self, beamset, ds):
        o = np.empty(10)
        check(lib().pofd_like2_dataset_info(self.h, int(beamset), int(ds), o,
                                            None))
        keys = ["ndata", "nbins", "bincent01", "bincent02", "bindelta1",
                "bindelta2", "like_offset", "sigma_base1", "sigma_base2",
                "like_norm"]
        info = dict(zip(keys, o))
        nb = int(info["nbins"])
        bins = np.zeros(max(nb * nb, 1), dtype=np.uint32)
        check(lib().pofd_like2_dataset_info(self.h, int(beamset), int(ds), o,
                                            _lib.ptr(bins)))
        info["bins"] = bins[:nb * nb].reshape(nb, nb)
        return info

    def reserve(self, max_batch):
        check(lib().pofd_like2_reserve(self.h, int(max_batch)))

    def getLogLike(self, p):
        th = _f32(p)
        ll = C.c_double()
        inv = C.c_int()
        check(lib().pofd_like2_loglike(self.h, th, th.size, C.byref(ll),
                                       C.byref(inv)))
        return ll.value, bool(inv.value)

    def getLogLikeBatch(self, thetas):
        th = _f32(thetas)
        if th.ndim != 2:
            raise PofdError(-10, "thetas must be [nprop, npar]")
        nprop, npar = th.shape
        ll = np.empty(nprop)
        st = np.empty(nprop, dtype=np.int32)
        check(lib().pofd_like2_eval_batch(self.h, nprop, th.ctypes.data, npar,
                                          ll.ctypes.data, st.ctypes.data))
        return ll, st

    # priors per band (calcLikeDouble.h:310-341); band 0 or 1
    def setSigmaPrior(self, band, width):
        check(lib().pofd_like2_set_sigma_prior(self.h, int(band), 1,
                                               float(width)))

    def unsetSigmaPrior(self, band):
        check(lib().pofd_like2_set_sigma_prior(self.h, int(band), 0, 0.0))

    def setCFIRBPrior(self, band, mean, sigma):
        check(lib().pofd_like2_set_cfirb_prior(self.h, int(band), 1,
                                               float(mean), float(sigma)))

    def unsetCFIRBPrior(self, band):
        check(lib().pofd_like2_set_cfirb_prior(self.h, int(band), 0, 0.0,
                                               0.0))

    def setPoissonPrior(self, band, mean, sigma):
        check(lib().pofd_like2_set_poisson_prior(self.h, int(band), 1,
                                                 float(mean), float(sigma)))

    def unsetPoissonPrior(self, band):
        check(lib().pofd_like2_set_poisson_prior(self.h, int(band), 0, 0.0,
                                                 0.0))

    def setRegularizationAlpha(self, alpha):
        check(lib().pofd_like2_set_regularization(self.h, float(alpha)))

    def getBonus(self, thetas):
        """<S1>, <S2>, <S1^2>, <S2^2> of each row: [nprop, 4]."""
        th = _f32(thetas)
        if th.ndim == 1:
            th = th[None, :]
        th = np.ascontiguousarray(th)
        out = np.empty((th.shape[0], 4))
        check(lib().pofd_like2_bonus(self.h, th.shape[0], th.ravel(),
                                     th.shape[1], out.ravel()))
        return out

    def fillBonusParams(self, thetas):
        """calcLikeDouble::fillBonusParams on rows with nmodel + 6 or more
        entries: a copy with <S1>, <S2>, <S1^2>, <S2^2> after the two sigma
        multipliers (as floats)."""
        th = np.array(_f32(thetas), copy=True)
        one = th.ndim == 1
        if one:
            th = th[None, :]
        k = self.nmodel
        if th.shape[1] < k + 6:
            raise PofdError(-10, "Not enough room to fill")
        th[:, k + 2:k + 6] = self.getBonus(th).astype(np.float32)
        return th[0] if one else th

    def getLogLikeDevice(self, nprop, theta_ptr, npar, logl_ptr, status_ptr,
                         stream=None):
        check(lib().pofd_like2_eval_batch_device(
            self.h, int(nprop), C.c_void_p(theta_ptr), int(npar),
            C.c_void_p(logl_ptr), C.c_void_p(status_ptr),
            C.c_void_p(stream) if stream else None))

    def getPD(self, beamset, ds, p, setLog=True):
        th = _f32(p)
        n = self.fftsize
        out = np.empty(n * n)
        info = np.empty(16)
        check(lib().pofd_like2_pd(self.h, int(beamset), int(ds), th, th.size,
                                  int(setLog), out, _lib.ptr(info)))
        keys = ["dflux1", "dflux2", "mn1", "mn2", "var1", "var2", "shift1",
                "shift2", "split1", "split2", "pd_minflux1", "pd_minflux2",
                "sg1pos", "sg1neg", "sg2pos", "sg2neg"]
        return out.reshape(n, n), dict(zip(keys, info))

    def getR(self, beamset, p):
        th = _f32(p)
        n = self.fftsize
        out = np.empty(n * n)
        check(lib().pofd_like2_get_r(self.h, int(beamset), th, th.size, out))
        return out.reshape(n, n)

    def profileStages(self, thetas, reps=3):
        th = _f32(thetas)
        nprop, npar = th.shape
        ms = np.zeros(16)
        ns = C.c_int()
        check(lib().pofd_like2_profile(self.h, nprop, th.ravel(), npar,
                                       int(reps), ms, C.byref(ns)))
        return {lib().pofd_like2_stage_name_now(self.h, i).decode(): ms[i]
                for i in range(ns.value)}

    def setFFT(self, mode):
        """1: 1D cuFFT row transforms around the library's fused column
        transform + spectrum kernel (default, n a power of two in
        [512, 4096]); 0: 2D cuFFT transforms with the spectrum kernel between
        them."""
        check(lib().pofd_like2_set_fft(self.h, int(mode)))

    def setReferenceSums(self, on):
        """Sum the P(D) integral and means in the reference's sequential
        row-major order (PDDouble.cc:142-208, 355-447) instead of the
        default tree sums; slow, for parity checks."""
        check(lib().pofd_like2_set_reference_sums(self.h, 1 if on else 0))

    TUNING_KEYS = ("fft_mode", "rgrid_rows", "edge_rows")

    def autotune(self, thetas, reps=5):
        """Choose the launch shapes by timing the graph-captured launch
        sequence on these rows; returns the chosen knobs with the best and
        the untuned time per launch (ms)."""
        th = np.ascontiguousarray(_f32(thetas))
        if th.ndim != 2:
            raise PofdError(-10, "thetas must be [nprop, npar]")
        out = np.zeros(5)
        check(lib().pofd_like2_autotune(self.h, th.shape[0], th.ravel(),
                                        th.shape[1], int(reps),
                                        out.ctypes.data_as(C.c_void_p)))
        d = {k: int(v) for k, v in zip(self.TUNING_KEYS, out[:3])}
        d["ms"], d["untuned_ms"] = float(out[3]), float(out[4])
        return d

    def getTuning(self):
        k = np.zeros(len(self.TUNING_KEYS), dtype=np.int32)
        check(lib().pofd_like2_get_tuning(self.h, k))
        return {n: int(v) for n, v in zip(self.TUNING_KEYS, k)}

    def setTuning(self, **knobs):
        cur = self.getTuning()
        cur.update(knobs)
        k = np.array([cur[n] for n in self.TUNING_KEYS], dtype=np.int32)
        check(lib().pofd_like2_set_tuning(self.h, k))

    def activeTerms(self, p):
        """(main-row, edge-row) active colour terms of one proposal's R
        grid, summed over rows and beam sets (the R builders' work per
        column)."""
        th = _f32(p)
        out = (C.c_longlong * 2)()
        check(lib().pofd_like2_active_terms(self.h, th, th.size, out))
        return int(out[0]), int(out[1])

    def fusedColumns(self):
        """True when the fused column path is the one in use."""
        k = C.c_int()
        check(lib().pofd_like2_fft_info(self.h, C.byref(k)))
        return bool(k.value)

    def kernelsPerEval(self):
        k = C.c_int()
        check(lib().pofd_like2_kernels_per_eval(self.h, C.byref(k)))
        return k.value
