"""Seeded synthetic inputs of the benchmark configurations.

The reference ships no simulator; these generators make maps with the
shapes, sizes and value distributions of the benchmark configurations:
a knot power-law number-count model with jittered knots, circular Gaussian
beams, Poisson source draws convolved with the beam, white noise and mean
subtraction; for two bands a log-normal colour S2/S1.

Units: fluxes in Jy, pixel sizes in arcsec, counts in sources / deg^2 / Jy.
"""
import numpy as np

ARCSEC2_PER_DEG2 = 3600.0 ** 2


def gaussian_beam(fwhm_px, nfwhm=9.0):
    """Peak-normalised circular Gaussian on an odd square map about
    nfwhm * FWHM pixels wide."""
    npix = int(np.ceil(nfwhm * fwhm_px))
    if npix % 2 == 0:
        npix += 1
    c = npix // 2
    y, x = np.mgrid[0:npix, 0:npix]
    sig = fwhm_px / np.sqrt(8.0 * np.log(2.0))
    return np.exp(-0.5 * ((x - c) ** 2 + (y - c) ** 2) / sig ** 2)


def knot_model(nknots, smin, smax, slope=-2.7, norm=1e4, s0=0.010,
               jitter=0.1, rng=None):
    """Knots log-spaced over [smin, smax] with log10 dN/dS from a power law
    norm * (S/s0)^slope, each jittered by N(0, jitter) dex.  Returns
    (positions float64, log10 values float32)."""
    rng = np.random.default_rng(rng)
    pos = np.logspace(np.log10(smin), np.log10(smax), nknots)
    val = np.log10(norm) + slope * np.log10(pos / s0)
    if jitter:
        val = val + rng.normal(0.0, jitter, nknots)
    return pos, val.astype(np.float32)


def _natural_spline(x, y):
    from scipy.interpolate import CubicSpline
    return CubicSpline(x, y, bc_type="natural")


def counts_on_grid(knotpos, log10vals, s):
    """dN/dS of the knot model (natural cubic spline in log2-log2 space)."""
    spl = _natural_spline(np.log2(knotpos), np.log2(10.0) * np.asarray(
        log10vals, dtype=np.float64))
    out = np.exp2(spl(np.log2(s)))
    out[(s < knotpos[0]) | (s >= knotpos[-1])] = 0.0
    return out


def draw_fluxes(knotpos, log10vals, area_deg2, rng):
    """Poisson number of sources over the area, fluxes by inverse CDF."""
    lo, hi = np.log(knotpos[0]), np.log(knotpos[-1])
    u = np.linspace(lo, hi, 20001)
    s = np.exp(u)
    dn = counts_on_grid(knotpos, log10vals, s) * s  # per d ln S
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (dn[1:] + dn[:-1]) *
                                           np.diff(u))])
    ntot = cdf[-1] * area_deg2
    nsrc = rng.poisson(ntot)
    r = rng.uniform(0.0, cdf[-1], nsrc)
    return np.exp(np.interp(r, cdf, u))


def _convolve(img, beam):
    ny, nx = img.shape
    by, bx = beam.shape
    k = np.zeros_like(img)
    k[:by, :bx] = beam
    k = np.roll(k, (-(by // 2), -(bx // 2)), axis=(0, 1))
    return np.fft.irfft2(np.fft.rfft2(img) * np.fft.rfft2(k), s=img.shape)


def make_map(shape, pixsize, beam, knotpos, log10vals, sigma_noise, rng):
    """Mean-subtracted map: Poisson sources placed on pixels, convolved with
    the beam (periodic), plus white noise sigma_noise."""
    rng = np.random.default_rng(rng)
    ny, nx = shape
    area = ny * nx * pixsize ** 2 / ARCSEC2_PER_DEG2
    f = draw_fluxes(knotpos, log10vals, area, rng)
    img = np.zeros(shape)
    iy = rng.integers(0, ny, f.size)
    ix = rng.integers(0, nx, f.size)
    np.add.at(img, (iy, ix), f)
    img = _convolve(img, beam)
    img += rng.normal(0.0, sigma_noise, shape)
    return img - img.mean()


def make_map_pair(shape, pixsize, beam1, beam2, knotpos, log10vals,
                  sigma_fn, offset_fn, sigma1, sigma2, rng):
    """Two-band maps: band 1 as make_map, band 2 fluxes S2 = S1 * exp(g),
    g ~ N(offset(S1), sigma(S1)^2) (the log-normal colour model)."""
    rng = np.random.default_rng(rng)
    ny, nx = shape
    area = ny * nx * pixsize ** 2 / ARCSEC2_PER_DEG2
    f1 = draw_fluxes(knotpos, log10vals, area, rng)
    g = rng.normal(offset_fn(f1), sigma_fn(f1))
    f2 = f1 * np.exp(g)
    iy = rng.integers(0, ny, f1.size)
    ix = rng.integers(0, nx, f1.size)
    m1 = np.zeros(shape)
    m2 = np.zeros(shape)
    np.add.at(m1, (iy, ix), f1)
    np.add.at(m2, (iy, ix), f2)
    m1 = _convolve(m1, beam1) + rng.normal(0.0, sigma1, shape)
    m2 = _convolve(m2, beam2) + rng.normal(0.0, sigma2, shape)
    return m1 - m1.mean(), m2 - m2.mean()


# ------------------------------------------------------------ configurations
def config_1d_small(seed=1, norm_scale=1.0):
    """1D plain fit: 6 knots over 2-400 mJy, FWHM 3 px beam at 6", 120-bin
    beam histogram, n = 4096, one 256x256 map at 2.5 mJy noise, 1000 data
    bins.  norm_scale multiplies the counts (100 makes the map confusion
    dominated: the split search then takes its jitter branch)."""
    rng = np.random.default_rng(seed)
    kp, kv = knot_model(6, 0.002, 0.400, norm=1e4 * norm_scale, rng=rng)
    bm = gaussian_beam(3.0)
    img = make_map((256, 256), 6.0, bm, kp, kv, 0.0025, rng)
    return dict(knotpos=kp, knotvals=kv, fftsize=4096, ninterp=2048,
                nbins=1000, beams=[bm], pixsize=6.0, nbeamhist=120,
                maps=[img], map_beam=[0], sigmas=[0.0025],
                theta0=np.concatenate([kv, [1.0]]).astype(np.float32))


def config_1d_batched(seed=2, scale=1.0):
    """1D batched fit: 10 knots over 1-800 mJy, three beam sets (FWHM 3.0,
    4.2, 6.0 px, 150-bin histograms) with one map each (2000x2000 at
    2.0 mJy, 1200x900 at 3.1 mJy, 600x600 at 5.0 mJy), n = 65536, 1000 data
    bins.  scale < 1 shrinks the maps (for fast tests)."""
    rng = np.random.default_rng(seed)
    kp, kv = knot_model(10, 0.001, 0.800, rng=rng)
    fw = [3.0, 4.2, 6.0]
    shapes = [(2000, 2000), (1200, 900), (600, 600)]
    sig = [0.0020, 0.0031, 0.0050]
    beams = [gaussian_beam(f) for f in fw]
    maps = []
    for sh, b, s in zip(shapes, beams, sig):
        sh = (max(32, int(sh[0] * scale)), max(32, int(sh[1] * scale)))
        maps.append(make_map(sh, 6.0, b, kp, kv, s, rng))
    return dict(knotpos=kp, knotvals=kv, fftsize=65536, ninterp=2048,
                nbins=1000, beams=beams, pixsize=6.0, nbeamhist=150,
                maps=maps, map_beam=[0, 1, 2], sigmas=sig,
                theta0=np.concatenate([kv, [1.0]]).astype(np.float32))


def build_like1(cfg, ctx, fftsize=None, ninterp=None, nbins=None):
    """calcLike for a 1D configuration (beam sets in config order)."""
    from .api1d import beam, calcLike
    L = calcLike(ctx, cfg["knotpos"], fftsize or cfg["fftsize"],
                 ninterp or cfg["ninterp"], True, nbins or cfg["nbins"])
    bms = [beam(b, cfg["pixsize"], True, cfg["nbeamhist"], 1e-5)
           for b in cfg["beams"]]
    for b in bms:
        L.addBeamSet(b, 0.0)
    for m, bi, s in zip(cfg["maps"], cfg["map_beam"], cfg["sigmas"]):
        L.addDataset(bi, m, s, 1.0, True)
    L.setRRanges(cfg["theta0"])
    return L


def proposals(theta0, nprop, scale=0.02, rng=None, fixed_last=True):
    """Walker-like proposals: theta0 plus N(0, scale) on the knot values."""
    rng = np.random.default_rng(rng)
    th = np.tile(np.asarray(theta0, dtype=np.float32), (nprop, 1))
    nfree = th.shape[1] - (1 if fixed_last else 0)
    th[:, :nfree] += rng.normal(0.0, scale, (nprop, nfree)).astype(np.float32)
    return th


def config_2d(seed=3, scale=1.0, n=2048, nbins=500):
    """2D plain fit: 8 band-1 knots over 2-500 mJy (power law, jittered),
    log-normal colour with 3 sigma knots (0.15-0.3) and 3 offset knots
    (about ln 0.7), both log-spaced over 2-500 mJy; Gaussian beams FWHM 3.0
    and 4.2 px at 6" on 39x39 maps, minval 1e-6, 100-bin 2D histogram; a
    1500x1500 map pair at 2.5 / 2.8 mJy noise; n = 2048, nedge = 256,
    500x500 data bins.  scale < 1 shrinks the maps (for fast tests)."""
    rng = np.random.default_rng(seed)
    kp, kv = knot_model(8, 0.002, 0.500, rng=rng)
    sk = np.logspace(np.log10(0.002), np.log10(0.5), 3)
    sv = np.array([0.15, 0.22, 0.3], np.float32)
    ok = sk.copy()
    ov = (np.log(0.7) + rng.normal(0, 0.02, 3)).astype(np.float32)
    b1 = gaussian_beam(3.0, nfwhm=39 / 3.0)
    b2 = gaussian_beam(4.2)
    sig_fn = lambda f: np.interp(f, sk, sv)  # noqa: E731
    off_fn = lambda f: np.interp(f, ok, ov)  # noqa: E731
    sh = (max(32, int(1500 * scale)), max(32, int(1500 * scale)))
    m1, m2 = make_map_pair(sh, 6.0, b1, b2, kp, kv, sig_fn, off_fn, 0.0025,
                           0.0028, rng)
    theta0 = np.concatenate([kv, sv, ov, [1.0, 1.0]]).astype(np.float32)
    return dict(knotpos=kp, knotvals=kv, sigmapos=sk, sigmavals=sv,
                offsetpos=ok, offsetvals=ov, beam1=b1, beam2=b2, pixsize=6.0,
                nbeamhist=100, minval=1e-6, maps=[(m1, m2)], sigmas=[(0.0025,
                                                                     0.0028)],
                fftsize=n, nedge=256, nbins=nbins, theta0=theta0)


def build_like2(cfg, ctx):
    from .api2d import calcLikeDouble, doublebeam
    L = calcLikeDouble(ctx, cfg["knotpos"], cfg["sigmapos"], cfg["offsetpos"],
                       cfg["fftsize"], cfg["nedge"], True, cfg["nbins"])
    bm = doublebeam(cfg["beam1"], cfg["beam2"], cfg["pixsize"], True,
                    cfg["nbeamhist"], cfg["minval"])
    L.addBeamSet(bm)
    for (m1, m2), (s1, s2) in zip(cfg["maps"], cfg["sigmas"]):
        L.addDataset(0, m1, m2, s1, s2)
    L.setRRanges(cfg["theta0"])
    return L


def config_2d_two_fields(seed=5, scale=1.0):
    """2D joint fit of two fields with different FFT sizes: the 2D plain
    configuration's 1500x1500 pair on a 2048^2 grid plus an 800x600 pair
    (same sources model, noise 2.5 / 2.8 mJy) on a 1024^2 grid; 14 model
    parameters (8 knots, 3 sigma, 3 offset) plus two fixed sigma
    multipliers."""
    a = config_2d(seed=seed, scale=scale)
    rng = np.random.default_rng(seed + 100)
    sk, sv, ok, ov = a["sigmapos"], a["sigmavals"], a["offsetpos"], a["offsetvals"]
    sig_fn = lambda f: np.interp(f, sk, sv)  # noqa: E731
    off_fn = lambda f: np.interp(f, ok, ov)  # noqa: E731
    sh = (max(32, int(800 * scale)), max(32, int(600 * scale)))
    m1, m2 = make_map_pair(sh, 6.0, a["beam1"], a["beam2"], a["knotpos"],
                           a["knotvals"], sig_fn, off_fn, 0.0025, 0.0028, rng)
    b = dict(a)
    b.update(maps=[(m1, m2)], fftsize=1024, nedge=128)
    return a, b
