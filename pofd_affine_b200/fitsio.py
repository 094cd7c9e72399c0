"""FITS input of data and beam maps through the library's reader (no GPU).

readData mirrors fitsData::readData(file, ignore_mask, meansub)
(fitsData.cc:56-316): the image of an "image"/"IMAGE" extension, else of the
primary HDU ("file.fits[k]" selects HDU k), minus the pixels a "mask"/"MASK"
extension marks non-zero, in file order.  readBeam mirrors beam::readFile
(beam.cc:295-395): the primary HDU (or HDU k) as an [ny][nx] array and its
PIXSIZE (else PIXSCALE) keyword.
"""
import ctypes as C

import numpy as np

from ._lib import check, lib


def readData(path, ignore_mask=False, meansub=False):
    n = C.c_size_t()
    p = str(path).encode()
    check(lib().pofd_fits_read_data(p, int(ignore_mask), int(meansub), None, 0,
                                    C.byref(n)))
    out = np.empty(n.value)
    check(lib().pofd_fits_read_data(p, int(ignore_mask), int(meansub),
                                    out.ctypes.data_as(C.c_void_p), out.size,
                                    C.byref(n)))
    return out


def readData2(path1, path2, ignore_mask=False, meansub=False):
    """The two bands' maps as fitsDataDouble::readData reads them
    (fitsDataDouble.cc:304-430): with masks in both files a pixel is dropped
    where the two mask values share a set bit, with one mask where it is
    non-zero."""
    n = C.c_size_t()
    a, b = str(path1).encode(), str(path2).encode()
    check(lib().pofd_fits_read_data2(a, b, int(ignore_mask), int(meansub), None,
                                     None, 0, C.byref(n)))
    o1, o2 = np.empty(n.value), np.empty(n.value)
    check(lib().pofd_fits_read_data2(a, b, int(ignore_mask), int(meansub),
                                     o1.ctypes.data_as(C.c_void_p),
                                     o2.ctypes.data_as(C.c_void_p), o1.size,
                                     C.byref(n)))
    return o1, o2


def readBeam(path):
    """(pixels [ny][nx], pixsize in arcsec)."""
    nx, ny, ps = C.c_size_t(), C.c_size_t(), C.c_double()
    p = str(path).encode()
    check(lib().pofd_fits_read_beam(p, None, 0, C.byref(nx), C.byref(ny),
                                    C.byref(ps)))
    out = np.empty(nx.value * ny.value)
    check(lib().pofd_fits_read_beam(p, out.ctypes.data_as(C.c_void_p), out.size,
                                    C.byref(nx), C.byref(ny), C.byref(ps)))
    return out.reshape(ny.value, nx.value), ps.value
