"""ctypes wrapper of the CPU oracle (oracle/_build/libpofd_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker or the timed CPU baseline.  The
product package never imports this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "_build", "libpofd_oracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")

_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        build()
    L = C.CDLL(LIBPATH)
    V, I, D, U, P, I64 = (C.c_void_p, C.c_int, C.c_double, C.c_uint,
                          C.c_void_p, C.c_int64)
    sigs = {
        "orc_last_error": (C.c_char_p, []),
        "orc_cspline_eval": (I, [I, _dp, _dp, I, _dp, _dp]),
        "orc_set_fast_fft": (I, [I]),
        "orc_rfft": (I, [I, _dp, _dp]),
        "orc_irfft": (I, [I, _dp, _dp]),
        "orc_rfft2": (I, [I, _dp, _dp]),
        "orc_irfft2": (I, [I, _dp, _dp]),
        "orc_beam1_new": (V, [_dp, I64, D, D, U]),
        "orc_beam1_free": (None, [V]),
        "orc_beam1_info": (I, [V, _dp]),
        "orc_beam1_array": (I, [V, I, _dp]),
        "orc_counts1_eval": (I, [I, _dp, _fp, I, _dp, _dp]),
        "orc_counts1_getR": (I, [I, _dp, _fp, V, I, _dp, _dp, I]),
        "orc_counts1_rrange": (I, [I, _dp, _fp, V, _dp]),
        "orc_counts1_integrals": (I, [I, _dp, _fp, _dp]),
        "orc_like1_new": (V, [I, _dp, U, U, I, U]),
        "orc_like1_free": (None, [V]),
        "orc_like1_add_beamset": (I, [V, _dp, I64, D, D, I, U, D]),
        "orc_like1_add_dataset": (I, [V, I, _dp, I64, I, D, D]),
        "orc_like1_set_rranges": (I, [V, _fp, I]),
        "orc_like1_get_rrange": (I, [V, I, _dp]),
        "orc_like1_dataset_info": (I, [V, I, I, _dp]),
        "orc_like1_dataset_bins": (I, [V, I, I, _up]),
        "orc_like1_eval": (I, [V, _fp, I, _dp]),
        "orc_like1_set_priors": (I, [V, _dp]),
        "orc_like2_set_priors": (I, [V, _dp]),
        "orc_like2_bonus": (I, [V, _fp, I, _dp]),
        "orc_like1_bonus": (I, [V, _fp, I, _dp]),
        "orc_like1_eval_batch": (I, [V, I, _fp, I, _dp, _ip, I]),
        "orc_like1_pd": (I, [V, I, I, _fp, I, I, _dp, P, P]),
        "orc_like1_rinterp": (I, [V, I, _fp, I, I, _dp, _dp]),
        "orc_beam2_new": (V, [_dp, _dp, I64, D, D, U]),
        "orc_beam2_free": (None, [V]),
        "orc_beam2_info": (I, [V, _dp]),
        "orc_beam2_array": (I, [V, I, I, _dp]),
        "orc_beam2_minmax": (I, [V, I, _dp]),
        "orc_counts2_new": (V, [I, _dp, I, _dp, I, _dp]),
        "orc_counts2_free": (None, [V]),
        "orc_counts2_set": (I, [V, _fp, I]),
        "orc_counts2_spline_int": (I, [V, D, D, _dp]),
        "orc_counts2_eval": (I, [V, I, _dp, _dp, _dp]),
        "orc_counts2_getR": (I, [V, V, I, _dp, I, _dp, _dp]),
        "orc_counts2_getR_scalar": (I, [V, V, I, _dp, _dp, _dp]),
        "orc_counts2_maxflux": (I, [V, _dp]),
        "orc_counts2_rrange": (I, [V, V, _dp]),
        "orc_counts2_sigma_offset": (I, [V, I, _dp, _dp, _dp]),
        "orc_like2_new": (V, [I, _dp, I, _dp, I, _dp, U, U, I, I, U]),
        "orc_like2_free": (None, [V]),
        "orc_like2_add_beamset": (I, [V, _dp, _dp, I64, D, D, I, U, D, D]),
        "orc_like2_add_dataset": (I, [V, I, _dp, _dp, I64, I, D, D, D]),
        "orc_like2_set_rranges": (I, [V, _fp, I]),
        "orc_like2_get_rrange": (I, [V, I, _dp]),
        "orc_like2_dataset_info": (I, [V, I, I, _dp]),
        "orc_like2_dataset_bins": (I, [V, I, I, _up]),
        "orc_like2_eval": (I, [V, _fp, I, _dp]),
        "orc_like2_eval_batch": (I, [V, I, _fp, I, _dp, _ip, I]),
        "orc_like2_pd": (I, [V, I, I, _fp, I, I, _dp, P, P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("oracle error %d: %s" % (code, msg))
        self.code = code


def _chk(st):
    if st < 0:
        raise OracleError(st, lib().orc_last_error().decode())
    return st


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ----------------------------------------------------------------- numerics
def cspline_eval(x, y, xq):
    x, y, xq = f64(x), f64(y), f64(xq)
    out = np.empty_like(xq)
    _chk(lib().orc_cspline_eval(len(x), x, y, len(xq), xq, out))
    return out


def set_fast_fft(on):
    """Route the oracle's real transforms (powers of two >= 8) to the fast
    radix-4 transforms (oracle/fastfft.hh) -- for the timed CPU baseline --
    or back to the radix-2 parity form.  Process-wide."""
    _chk(lib().orc_set_fast_fft(1 if on else 0))


def rfft(a):
    a = f64(a)
    n = len(a)
    out = np.empty(2 * (n // 2 + 1))
    _chk(lib().orc_rfft(n, a, out))
    return out.view(np.complex128)


def irfft(c, n):
    c = np.ascontiguousarray(c, dtype=np.complex128).view(np.float64)
    out = np.empty(n)
    _chk(lib().orc_irfft(n, c, out))
    return out


def rfft2(a):
    a = f64(a)
    n = a.shape[0]
    out = np.empty(2 * n * (n // 2 + 1))
    _chk(lib().orc_rfft2(n, a.ravel(), out))
    return out.view(np.complex128).reshape(n, n // 2 + 1)


def irfft2(c, n):
    c = np.ascontiguousarray(c, dtype=np.complex128).ravel().view(np.float64)
    out = np.empty(n * n)
    _chk(lib().orc_irfft2(n, c, out))
    return out.reshape(n, n)


# ----------------------------------------------------------------- 1D beam
class Beam1:
    def __init__(self, pix, pixsize, minval=1e-5, nhist=0):
        pix = f64(pix).ravel()
        self.h = lib().orc_beam1_new(pix, len(pix), pixsize, minval, nhist)
        if not self.h:
            raise OracleError(-10, lib().orc_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_beam1_free(self.h)

    def info(self):
        o = np.empty(15)
        lib().orc_beam1_info(self.h, o)
        keys = ["haspos", "hasneg", "npos", "nneg", "poshist", "neghist",
                "nposhist", "nneghist", "minpos", "maxpos", "minneg",
                "maxneg", "pixsize", "totpos", "totneg"]
        return dict(zip(keys, o))

    def array(self, which):
        inf = self.info()
        n = {0: inf["nposhist"], 1: inf["nposhist"], 2: inf["nneghist"],
             3: inf["nneghist"], 4: inf["npos"], 5: inf["nneg"]}[which]
        out = np.empty(int(n))
        lib().orc_beam1_array(self.h, which, out)
        return out


def counts1(knots, theta, s):
    knots, theta, s = f64(knots), f32(theta), f64(s)
    out = np.empty_like(s)
    _chk(lib().orc_counts1_eval(len(knots), knots, theta, len(s), s, out))
    return out


def getR1(knots, theta, beam, flux, scalar=False):
    knots, theta, flux = f64(knots), f32(theta), f64(flux)
    out = np.empty_like(flux)
    _chk(lib().orc_counts1_getR(len(knots), knots, theta, beam.h, len(flux),
                                flux, out, int(scalar)))
    return out


def rrange1(knots, theta, beam):
    knots, theta = f64(knots), f32(theta)
    out = np.empty(2)
    _chk(lib().orc_counts1_rrange(len(knots), knots, theta, beam.h, out))
    return out


def integrals1(knots, theta):
    knots, theta = f64(knots), f32(theta)
    out = np.empty(3)
    _chk(lib().orc_counts1_integrals(len(knots), knots, theta, out))
    return out


# ---------------------------------------------------------- 1D likelihood
class Like1:
    def __init__(self, knots, fftsize, ninterp=2048, bin_data=True,
                 nbins=1000):
        self.knots = f64(knots)
        self.fftsize = fftsize
        self.h = lib().orc_like1_new(len(self.knots), self.knots, fftsize,
                                     ninterp, int(bin_data), nbins)
        self.nsets = 0
        self.nds = []

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_like1_free(self.h)

    def add_beamset(self, beampix, pixsize, minval=1e-5, histogram=True,
                    nbeamhist=120, exp_conf=0.0):
        b = f64(beampix).ravel()
        idx = _chk(lib().orc_like1_add_beamset(self.h, b, len(b), pixsize,
                                               minval, int(histogram),
                                               nbeamhist, exp_conf))
        self.nsets += 1
        self.nds.append(0)
        return idx

    def add_dataset(self, beamset, data, sigma_base, like_norm=1.0,
                    meansub=True):
        d = f64(data).ravel()
        _chk(lib().orc_like1_add_dataset(self.h, beamset, d, len(d),
                                         int(meansub), sigma_base, like_norm))
        self.nds[beamset] += 1

    def set_rranges(self, theta):
        th = f32(theta)
        _chk(lib().orc_like1_set_rranges(self.h, th, len(th)))

    def rrange(self, bs):
        out = np.empty(2)
        _chk(lib().orc_like1_get_rrange(self.h, bs, out))
        return out

    def dataset_info(self, bs, ds):
        o = np.empty(9)
        _chk(lib().orc_like1_dataset_info(self.h, bs, ds, o))
        keys = ["ndata", "nbins", "bincent0", "bindelta", "like_offset",
                "sigma_base", "like_norm", "minflux", "maxflux"]
        return dict(zip(keys, o))

    def dataset_bins(self, bs, ds):
        nb = int(self.dataset_info(bs, ds)["nbins"])
        out = np.empty(nb, dtype=np.uint32)
        _chk(lib().orc_like1_dataset_bins(self.h, bs, ds, out))
        return out

    def loglike(self, theta):
        th = f32(theta)
        out = np.empty(1)
        _chk(lib().orc_like1_eval(self.h, th, len(th), out))
        return out[0]

    def set_priors(self, sigma=None, cfirb=None, poisson=None, alpha=0.0):
        """sigma: prior width on the sigma multiplier; cfirb, poisson:
        (mean, sigma) on <S> and <S^2>; alpha: regularisation multiplier
        (calcLike.h:184-195).  None turns a prior off."""
        v = np.zeros(9)
        if sigma is not None:
            v[0], v[1] = 1.0, sigma
        if cfirb is not None:
            v[2], v[3], v[4] = 1.0, cfirb[0], cfirb[1]
        if poisson is not None:
            v[5], v[6], v[7] = 1.0, poisson[0], poisson[1]
        v[8] = alpha
        _chk(lib().orc_like1_set_priors(self.h, v))

    def bonus(self, theta):
        """<S> and <S^2> of the model at theta (calcLike.cc:958-980)."""
        th = f32(theta)
        out = np.empty(2)
        _chk(lib().orc_like1_bonus(self.h, th, len(th), out))
        return out

    def loglike_batch(self, thetas, nthreads=1):
        th = f32(thetas)
        nprop, npar = th.shape
        out = np.empty(nprop)
        st = np.empty(nprop, dtype=np.int32)
        _chk(lib().orc_like1_eval_batch(self.h, nprop, th.ravel(), npar, out,
                                        st, nthreads))
        return out, st

    def pd(self, bs, ds, theta, setlog=True, want_r=False):
        th = f32(theta)
        out = np.empty(self.fftsize)
        dbg = np.empty(12)
        rv = np.empty(self.fftsize) if want_r else None
        _chk(lib().orc_like1_pd(self.h, bs, ds, th, len(th), int(setlog), out,
                                _ptr(dbg), _ptr(rv)))
        keys = ["dflux", "minflux_R", "wrapRidx", "mn", "var_noi", "doshift",
                "shift", "splitidx", "sgpos", "sgneg", "pd_minflux", "r0"]
        info = dict(zip(keys, dbg))
        return (out, info, rv) if want_r else (out, info)

    def rinterp(self, bs, theta, ninterp, neg=False):
        th = f32(theta)
        x = np.empty(ninterp)
        r = np.empty(ninterp)
        _chk(lib().orc_like1_rinterp(self.h, bs, th, len(th), int(neg), x, r))
        return x, r


# ----------------------------------------------------------------- 2D beam
class Beam2:
    def __init__(self, pix1, pix2, pixsize, minval=1e-6, nhist=0):
        p1, p2 = f64(pix1).ravel(), f64(pix2).ravel()
        self.h = lib().orc_beam2_new(p1, p2, len(p1), pixsize, minval, nhist)
        if not self.h:
            raise OracleError(-10, lib().orc_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_beam2_free(self.h)

    def info(self):
        o = np.empty(17)
        lib().orc_beam2_info(self.h, o)
        return {"hassign": o[0:4].astype(bool), "npix": o[4:8].astype(int),
                "ishist": o[8:12].astype(bool), "nhist": o[12:16].astype(int),
                "pixsize": o[16]}

    def nterms(self, sgn):
        inf = self.info()
        if not inf["hassign"][sgn]:
            return 0
        return int(inf["nhist"][sgn] if inf["ishist"][sgn]
                   else inf["npix"][sgn])

    def array(self, sgn, which):
        out = np.empty(self.nterms(sgn))
        _chk(lib().orc_beam2_array(self.h, sgn, which, out))
        return out

    def minmax(self, sgn):
        out = np.empty(4)
        lib().orc_beam2_minmax(self.h, sgn, out)
        return out


class Counts2:
    def __init__(self, knots, sigmapos, offsetpos):
        k, s, o = f64(knots), f64(sigmapos), f64(offsetpos)
        self.npar = len(k) + len(s) + len(o)
        self.h = lib().orc_counts2_new(len(k), k, len(s), s, len(o), o)
        if not self.h:
            raise OracleError(-10, lib().orc_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_counts2_free(self.h)

    def set(self, theta):
        th = f32(theta)
        _chk(lib().orc_counts2_set(self.h, th, len(th)))

    def counts(self, f1, f2):
        f1, f2 = f64(f1), f64(f2)
        out = np.empty_like(f1)
        _chk(lib().orc_counts2_eval(self.h, len(f1), f1, f2, out))
        return out

    def getR(self, beam, f1, f2):
        f1, f2 = f64(f1), f64(f2)
        out = np.empty(len(f1) * len(f2))
        _chk(lib().orc_counts2_getR(self.h, beam.h, len(f1), f1, len(f2), f2,
                                    out))
        return out.reshape(len(f1), len(f2))

    def getR_scalar(self, beam, f1, f2):
        f1, f2 = f64(f1), f64(f2)
        out = np.empty_like(f1)
        _chk(lib().orc_counts2_getR_scalar(self.h, beam.h, len(f1), f1, f2,
                                           out))
        return out

    def maxflux(self):
        out = np.empty(2)
        _chk(lib().orc_counts2_maxflux(self.h, out))
        return out

    def spline_int(self, alpha, beta):
        out = np.empty(1)
        _chk(lib().orc_counts2_spline_int(self.h, float(alpha), float(beta),
                                          out))
        return out[0]

    def rrange(self, beam):
        out = np.empty(4)
        _chk(lib().orc_counts2_rrange(self.h, beam.h, out))
        return out

    def sigma_offset(self, f1):
        f1 = f64(f1)
        s = np.empty_like(f1)
        o = np.empty_like(f1)
        _chk(lib().orc_counts2_sigma_offset(self.h, len(f1), f1, s, o))
        return s, o


class Like2:
    def __init__(self, knots, sigmapos, offsetpos, fftsize, nedge=256,
                 edge_integ=True, nbins=1000, bin_data=True):
        k, s, o = f64(knots), f64(sigmapos), f64(offsetpos)
        self.fftsize = fftsize
        self.h = lib().orc_like2_new(len(k), k, len(s), s, len(o), o, fftsize,
                                     nedge, int(edge_integ), int(bool(bin_data)),
                                     nbins)
        if not self.h:
            raise OracleError(-10, lib().orc_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_like2_free(self.h)

    def add_beamset(self, pix1, pix2, pixsize, minval=1e-6, histogram=True,
                    nbeamhist=150, exp_conf1=0.0, exp_conf2=0.0):
        p1, p2 = f64(pix1).ravel(), f64(pix2).ravel()
        return _chk(lib().orc_like2_add_beamset(self.h, p1, p2, len(p1),
                                                pixsize, minval,
                                                int(histogram), nbeamhist,
                                                exp_conf1, exp_conf2))

    def add_dataset(self, bs, d1, d2, sigma1, sigma2, like_norm=1.0,
                    meansub=True):
        a, b = f64(d1).ravel(), f64(d2).ravel()
        _chk(lib().orc_like2_add_dataset(self.h, bs, a, b, len(a),
                                         int(meansub), sigma1, sigma2,
                                         like_norm))

    def set_rranges(self, theta):
        th = f32(theta)
        _chk(lib().orc_like2_set_rranges(self.h, th, len(th)))

    def rrange(self, bs):
        out = np.empty(4)
        _chk(lib().orc_like2_get_rrange(self.h, bs, out))
        return out

    def dataset_info(self, bs, ds):
        o = np.empty(10)
        _chk(lib().orc_like2_dataset_info(self.h, bs, ds, o))
        keys = ["ndata", "nbins", "bincent01", "bincent02", "bindelta1",
                "bindelta2", "like_offset", "sigma_base1", "sigma_base2",
                "like_norm"]
        return dict(zip(keys, o))

    def dataset_bins(self, bs, ds):
        nb = int(self.dataset_info(bs, ds)["nbins"])
        out = np.empty(nb * nb, dtype=np.uint32)
        _chk(lib().orc_like2_dataset_bins(self.h, bs, ds, out))
        return out.reshape(nb, nb)

    def loglike(self, theta):
        th = f32(theta)
        out = np.empty(1)
        _chk(lib().orc_like2_eval(self.h, th, len(th), out))
        return out[0]

    def set_priors(self, sigma=(None, None), cfirb=(None, None),
                   poisson=(None, None), alpha=0.0):
        """Per band: sigma width, (mean, sigma) on <S_b>, (mean, sigma) on
        <S_b^2>; None turns a prior off (calcLikeDouble.h:213-232)."""
        v = np.zeros(17)
        for b in range(2):
            q = v[8 * b:8 * b + 8]
            if sigma[b] is not None:
                q[0], q[1] = 1.0, sigma[b]
            if cfirb[b] is not None:
                q[2], q[3], q[4] = 1.0, cfirb[b][0], cfirb[b][1]
            if poisson[b] is not None:
                q[5], q[6], q[7] = 1.0, poisson[b][0], poisson[b][1]
        v[16] = alpha
        _chk(lib().orc_like2_set_priors(self.h, v))

    def bonus(self, theta):
        """<S1>, <S2>, <S1^2>, <S2^2> (calcLikeDouble.cc:1283-1310)."""
        th = f32(theta)
        out = np.empty(4)
        _chk(lib().orc_like2_bonus(self.h, th, len(th), out))
        return out

    def loglike_batch(self, thetas, nthreads=1):
        th = f32(thetas)
        nprop, npar = th.shape
        out = np.empty(nprop)
        st = np.empty(nprop, dtype=np.int32)
        _chk(lib().orc_like2_eval_batch(self.h, nprop, th.ravel(), npar, out,
                                        st, nthreads))
        return out, st

    def pd(self, bs, ds, theta, setlog=True, want_r=False):
        th = f32(theta)
        n = self.fftsize
        out = np.empty(n * n)
        dbg = np.empty(16)
        rv = np.empty(n * n) if want_r else None
        _chk(lib().orc_like2_pd(self.h, bs, ds, th, len(th), int(setlog), out,
                                _ptr(dbg), _ptr(rv)))
        keys = ["dflux1", "dflux2", "mn1", "mn2", "var1", "var2", "shift1",
                "shift2", "split1", "split2", "pd_minflux1", "pd_minflux2",
                "sg1pos", "sg1neg", "sg2pos", "sg2neg"]
        info = dict(zip(keys, dbg))
        pdv = out.reshape(n, n)
        return (pdv, info, rv.reshape(n, n)) if want_r else (pdv, info)


# ------------------------------------------------ vectorised 2D gather
def loglike_binned2(pd, minflux1, minflux2, dflux1, dflux2, bins, bc1, bc2,
                    bd1, bd2):
    """PDDouble::getLogLikeBinned (PDDouble.cc:1103-1222) vectorised over the
    non-zero bins of a linear (not log) normalised P(D): log2 of the P(D)
    is bilinearly interpolated at the bin centres (clamped at the edges,
    last cell clamped as in the restatement above), summed with the bin
    counts and returned in natural-log units."""
    pd = np.asarray(pd, dtype=np.float64)
    n1, n2 = pd.shape
    lp = np.where(pd > 0, np.log2(np.where(pd > 0, pd, 1.0)), -30.0)
    i, j = np.nonzero(bins)
    cnt = bins[i, j].astype(np.float64)
    c1 = bc1 + i * bd1
    c2 = bc2 + j * bd2
    max1 = minflux1 + (n1 - 1) * dflux1
    max2 = minflux2 + (n2 - 1) * dflux2
    x = (c1 - minflux1) / dflux1
    y = (c2 - minflux2) / dflux2
    i1 = np.clip(x.astype(np.int64), 0, n1 - 1)
    i2 = np.clip(y.astype(np.int64), 0, n2 - 1)
    t = x - i1
    u = y - i2
    in1 = (c1 >= minflux1) & (c1 <= max1)
    in2 = (c2 >= minflux2) & (c2 <= max2)
    e1 = np.where(c1 < minflux1, 0, n1 - 1)
    e2 = np.where(c2 < minflux2, 0, n2 - 1)
    a1 = np.where(i1 > n1 - 2, n1 - 2, i1)
    t = np.where(i1 > n1 - 2, 1.0, t)
    a2 = np.where(i2 > n2 - 2, n2 - 2, i2)
    u = np.where(i2 > n2 - 2, 1.0, u)
    bil = ((1 - t) * ((1 - u) * lp[a1, a2] + u * lp[a1, a2 + 1]) +
           t * ((1 - u) * lp[a1 + 1, a2] + u * lp[a1 + 1, a2 + 1]))
    iv = np.where(in1 & in2, bil,
                  np.where(in1, lp[i1, e2], np.where(in2, lp[e1, i2], lp[e1, e2])))
    return float(np.sum(cnt * iv)) * np.log(2.0)
