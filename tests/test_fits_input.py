"""FITS input (pofd_fits_read_data / pofd_fits_read_beam) on the CPU.

Files written here by a minimal FITS writer cover the reference's reading
rules (fitsData.cc:56-316, beam.cc:295-395): the "image"/"IMAGE" extension
or the primary HDU, the "mask"/"MASK" extension (non-zero pixels dropped,
file order kept), mean subtraction, PIXSIZE then PIXSCALE, the "[k]" HDU
selector, BITPIX -64/-32/16/8 with BSCALE/BZERO, and the reference's
errors.  Where the reference's test data are present, the reader is checked
against the committed beam fixtures made by an independent reader
(tests/golden/make_fixtures.py).
"""
import os

import numpy as np
import pytest

# the reference's own test FITS files (test/testdata in its tree), when a
# checkout is named by POFD_REFERENCE_DIR; skipped otherwise
REFDATA = os.path.join(os.environ.get("POFD_REFERENCE_DIR", ""), "test", "testdata") \
    if os.environ.get("POFD_REFERENCE_DIR") else ""


def _card(key, value=None, comment=""):
    if value is None:
        s = key.ljust(8)
    else:
        if isinstance(value, bool):
            v = ("T" if value else "F").rjust(20)
        elif isinstance(value, str):
            v = ("'" + value.ljust(8) + "'").ljust(20)
        elif isinstance(value, int):
            v = str(value).rjust(20)
        else:
            v = ("%.17G" % value).rjust(20)
        s = key.ljust(8) + "= " + v + (" / " + comment if comment else "")
    return s.ljust(80)[:80]


def _hdu(arr, bitpix, primary, extname=None, keys=()):
    arr = np.asarray(arr)
    cards = [_card("SIMPLE", True) if primary else _card("XTENSION", "IMAGE"),
             _card("BITPIX", bitpix), _card("NAXIS", arr.ndim)]
    for i, d in enumerate(arr.shape[::-1]):
        cards.append(_card("NAXIS%d" % (i + 1), int(d)))
    if not primary:
        cards += [_card("PCOUNT", 0), _card("GCOUNT", 1)]
    if extname:
        cards.append(_card("EXTNAME", extname))
    for k, v in keys:
        cards.append(_card(k, v))
    cards.append(_card("END"))
    head = "".join(cards).encode("ascii")
    head += b" " * (-len(head) % 2880)
    dt = {-64: ">f8", -32: ">f4", 16: ">i2", 32: ">i4", 8: "u1"}[bitpix]
    data = np.ascontiguousarray(arr).astype(dt).tobytes()
    data += b"\0" * (-len(data) % 2880)
    return head + data


def _write(path, *hdus):
    with open(path, "wb") as f:
        for h in hdus:
            f.write(h)
    return str(path)


def test_primary_image_and_beam_keywords(tmp_path):
    from pofd_affine_b200 import fitsio
    rng = np.random.default_rng(1)
    img = rng.normal(size=(7, 5))
    f = _write(tmp_path / "a.fits", _hdu(img, -64, True, keys=[("PIXSIZE", 6.0)]))
    d = fitsio.readData(f)
    assert np.array_equal(d, img.ravel())  # file order: first axis fastest
    b, ps = fitsio.readBeam(f)
    assert ps == 6.0 and np.array_equal(b, img)
    g = _write(tmp_path / "b.fits", _hdu(img, -64, True, keys=[("PIXSCALE", 4.5)]))
    assert fitsio.readBeam(g)[1] == 4.5


def test_image_and_mask_extensions(tmp_path):
    from pofd_affine_b200 import fitsio
    rng = np.random.default_rng(2)
    img = rng.normal(size=(6, 9))
    mask = (rng.uniform(size=img.shape) < 0.3).astype(np.int32)
    f = _write(tmp_path / "m.fits", _hdu(np.zeros((1, 1)), -64, True),
               _hdu(img, -64, False, "IMAGE"), _hdu(mask, 32, False, "MASK"))
    d = fitsio.readData(f)
    assert np.array_equal(d, img.ravel()[mask.ravel() == 0])
    assert np.array_equal(fitsio.readData(f, ignore_mask=True), img.ravel())
    # mean subtraction as fitsData::meanSubtract: sum in order, / n
    keep = img.ravel()[mask.ravel() == 0]
    m = keep[0]
    for v in keep[1:]:
        m += v
    m /= keep.size
    assert np.array_equal(fitsio.readData(f, meansub=True), keep - m)
    # lower-case extension names, HDU selector
    g = _write(tmp_path / "l.fits", _hdu(np.ones((2, 2)), -64, True),
               _hdu(img, -64, False, "image"), _hdu(mask, 16, False, "mask"))
    assert np.array_equal(fitsio.readData(g), img.ravel()[mask.ravel() == 0])
    assert np.array_equal(fitsio.readData(g + "[0]", ignore_mask=True), np.ones(4))


def test_scaled_integer_and_float32_images(tmp_path):
    from pofd_affine_b200 import fitsio
    raw = np.arange(-6, 6, dtype=np.int16).reshape(3, 4)
    f = _write(tmp_path / "s.fits", _hdu(raw, 16, True,
                                         keys=[("BSCALE", 0.5), ("BZERO", 10.0),
                                               ("PIXSIZE", 1.0)]))
    assert np.array_equal(fitsio.readData(f), 10.0 + 0.5 * raw.ravel())
    img = np.linspace(-1, 1, 12, dtype=np.float32).reshape(3, 4)
    g = _write(tmp_path / "f.fits", _hdu(img, -32, True, keys=[("PIXSIZE", 2.0)]))
    assert np.array_equal(fitsio.readBeam(g)[0], img.astype(np.float64))
    u8 = np.arange(12, dtype=np.uint8).reshape(3, 4)
    h = _write(tmp_path / "u.fits", _hdu(u8, 8, True))
    assert np.array_equal(fitsio.readData(h), u8.ravel().astype(np.float64))


def test_reference_errors(tmp_path):
    from pofd_affine_b200 import PofdError, fitsio
    img = np.ones((4, 4))
    nopix = _write(tmp_path / "n.fits", _hdu(img, -64, True))
    with pytest.raises(PofdError, match="pixel scale"):
        fitsio.readBeam(nopix)
    cube = _write(tmp_path / "c.fits", _hdu(np.ones((2, 3, 4)), -64, True,
                                            keys=[("PIXSIZE", 1.0)]))
    with pytest.raises(PofdError, match="not 2D"):
        fitsio.readBeam(cube)
    with pytest.raises(PofdError, match="not 2D"):
        fitsio.readData(cube)
    allm = _write(tmp_path / "x.fits", _hdu(img, -64, True),
                  _hdu(np.ones((4, 4), np.int32), 32, False, "MASK"))
    with pytest.raises(PofdError, match="All data masked"):
        fitsio.readData(allm)
    bad = _write(tmp_path / "y.fits", _hdu(img, -64, True),
                 _hdu(np.zeros((4, 3), np.int32), 32, False, "MASK"))
    with pytest.raises(PofdError, match="first dimension"):
        fitsio.readData(bad)
    with pytest.raises(PofdError, match="opening"):
        fitsio.readData(str(tmp_path / "missing.fits"))
    junk = tmp_path / "j.fits"
    junk.write_bytes(b"not a fits file" * 300)
    with pytest.raises(PofdError):
        fitsio.readData(str(junk))


@pytest.mark.skipif(not REFDATA or not os.path.isdir(REFDATA),
                    reason="POFD_REFERENCE_DIR not set or its test data absent")
def test_reference_beam_files_match_fixtures():
    from pofd_affine_b200 import fitsio
    here = os.path.dirname(os.path.abspath(__file__))
    g = np.load(os.path.join(here, "golden", "beams.npz"))
    for name, fn in [("band1", "band1_beam.fits"), ("band2", "band2_beam.fits"),
                     ("band12_0", "band12_beam_f100.fits[0]"),
                     ("band12_1", "band12_beam_f100.fits[1]")]:
        b, ps = fitsio.readBeam(os.path.join(REFDATA, fn))
        assert np.array_equal(b.ravel(), g[name])
        assert list(b.shape[::-1]) == list(g[name + "_dims"])
        assert ps == float(g[name + "_pixsize"])


def test_two_band_masks_as_the_reference(tmp_path):
    """fitsDataDouble.cc:338-395: both masked -> dropped where mask1 & mask2
    share a bit; one mask -> dropped where it is non-zero."""
    from pofd_affine_b200 import PofdError, fitsio
    rng = np.random.default_rng(4)
    a, b = rng.normal(size=(5, 6)), rng.normal(size=(5, 6))
    m1 = rng.integers(0, 4, size=a.shape).astype(np.int32)
    m2 = rng.integers(0, 4, size=a.shape).astype(np.int32)
    f1 = _write(tmp_path / "1.fits", _hdu(a, -64, True), _hdu(m1, 32, False, "MASK"))
    f2 = _write(tmp_path / "2.fits", _hdu(b, -64, True), _hdu(m2, 32, False, "MASK"))
    f2n = _write(tmp_path / "2n.fits", _hdu(b, -64, True))
    d1, d2 = fitsio.readData2(f1, f2)
    keep = (m1 & m2).ravel() == 0
    assert np.array_equal(d1, a.ravel()[keep]) and np.array_equal(d2, b.ravel()[keep])
    d1, d2 = fitsio.readData2(f1, f2n)
    keep = m1.ravel() == 0
    assert np.array_equal(d1, a.ravel()[keep]) and np.array_equal(d2, b.ravel()[keep])
    d1, d2 = fitsio.readData2(f1, f2, meansub=True)
    k = (m1 & m2).ravel() == 0
    for d, x in ((d1, a.ravel()[k]), (d2, b.ravel()[k])):
        m = x[0]
        for v in x[1:]:
            m += v
        assert np.array_equal(d, x - m / x.size)
    small = _write(tmp_path / "s.fits", _hdu(np.ones((2, 2)), -64, True))
    with pytest.raises(PofdError, match="not the same size"):
        fitsio.readData2(f1, small)


def test_read_data_from_files_groups_like_the_reference(tmp_path):
    """calcLike::readDataFromFiles: beam sets keyed by beam file in name
    order, datasets in input order inside a set (host-only context)."""
    from pofd_affine_b200 import Context, calcLike, synth
    ctx = Context(-1)
    bm = synth.gaussian_beam(3.0)
    bz = _write(tmp_path / "z_beam.fits", _hdu(bm, -64, True, keys=[("PIXSIZE", 6.0)]))
    ba = _write(tmp_path / "a_beam.fits", _hdu(bm ** 1.2, -64, True,
                                               keys=[("PIXSIZE", 6.0)]))
    rng = np.random.default_rng(0)
    maps = [rng.normal(0, 0.002, (40, 40)) for _ in range(3)]
    files = [_write(tmp_path / ("m%d.fits" % i), _hdu(m, -64, True))
             for i, m in enumerate(maps)]
    kp, kv = synth.knot_model(6, 0.002, 0.4, rng=rng)
    L = calcLike(ctx, kp, 4096, 256, True, 100)
    idx = L.readDataFromFiles(files, [bz, ba, bz], [0.002, 0.003, 0.004],
                              [1.0, 1.0, 1.0], meansub=True)
    assert idx == [1, 0, 1]  # a_beam sorts first
    info = L.datasetInfo(1, 1)
    assert info["sigma_base"] == 0.004  # second dataset of the z_beam set


@pytest.mark.gpu
def test_likelihood_from_files_equals_from_arrays(gpu_ctx, tmp_path):
    from pofd_affine_b200 import beam, calcLike, calcLikeDouble, doublebeam, synth
    rng = np.random.default_rng(6)
    kp, kv = synth.knot_model(6, 0.002, 0.4, rng=rng)
    bm = synth.gaussian_beam(3.0)
    img = synth.make_map((96, 96), 6.0, bm, kp, kv, 0.002, rng)
    bf = _write(tmp_path / "b.fits", _hdu(bm, -64, True, keys=[("PIXSIZE", 6.0)]))
    df = _write(tmp_path / "d.fits", _hdu(img, -64, True))
    th = np.concatenate([kv, [1.0]]).astype(np.float32)
    A = calcLike(gpu_ctx, kp, 4096, 512, True, 300)
    A.readDataFromFiles([df], [bf], [0.002], [1.0], meansub=True, histogram=True)
    A.setRRanges(th)
    B = calcLike(gpu_ctx, kp, 4096, 512, True, 300)
    B.addBeamSet(beam(bm, 6.0, True, 120, 1e-5))
    B.addDataset(0, img, 0.002, 1.0, True)
    B.setRRanges(th)
    la, sa = A.getLogLikeBatch(th[None, :])
    lb, sb = B.getLogLikeBatch(th[None, :])
    assert sa[0] == 0 and la[0] == lb[0]
    # 2D
    b1, b2 = synth.gaussian_beam(3.0), synth.gaussian_beam(3.0) ** 0.6
    sk = np.logspace(np.log10(0.003), np.log10(0.3), 2)
    ok = np.array([0.01])
    sv = np.array([0.2, 0.25], np.float32)
    ov = np.array([np.log(0.7)], np.float32)
    m1, m2 = synth.make_map_pair((64, 64), 6.0, b1, b2, kp, kv,
                                 lambda f: np.interp(f, sk, sv),
                                 lambda f: 0 * f + ov[0], 0.0025, 0.003, rng)
    f1 = _write(tmp_path / "m1.fits", _hdu(m1, -64, True))
    f2 = _write(tmp_path / "m2.fits", _hdu(m2, -64, True))
    g1 = _write(tmp_path / "b1.fits", _hdu(b1, -64, True, keys=[("PIXSIZE", 6.0)]))
    g2 = _write(tmp_path / "b2.fits", _hdu(b2, -64, True, keys=[("PIXSIZE", 6.0)]))
    th2 = np.concatenate([kv, sv, ov, [1.0, 1.0]]).astype(np.float32)
    C2 = calcLikeDouble(gpu_ctx, kp, sk, ok, 256, 64, True, 100, True)
    C2.readDataFromFiles([f1], [f2], [g1], [g2], [0.0025], [0.003], [1.0],
                         meansub=True, histogram=True, nbeamhist=40)
    C2.setRRanges(th2)
    D2 = calcLikeDouble(gpu_ctx, kp, sk, ok, 256, 64, True, 100, True)
    D2.addBeamSet(doublebeam(b1, b2, 6.0, True, 40, 1e-6))
    D2.addDataset(0, m1, m2, 0.0025, 0.003, 1.0, True)
    D2.setRRanges(th2)
    lc, sc = C2.getLogLikeBatch(th2[None, :])
    ld, sd = D2.getLogLikeBatch(th2[None, :])
    assert sc[0] == 0 and lc[0] == ld[0]
