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

REFDATA = "/root/reference/test/testdata"


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


@pytest.mark.skipif(not os.path.isdir(REFDATA), reason="reference test data absent")
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
