"""Regenerate the committed golden fixtures from the reference's test data.

Run in a container where the reference tree is mounted (it is not needed at
test time):

    python tests/golden/make_fixtures.py <reference checkout>   (or POFD_REFERENCE_DIR)

Writes, next to this script:
  * beams.npz -- the reference's test beams (test/testdata/band1_beam.fits,
    band2_beam.fits and both HDUs of band12_beam_f100.fits) as float64 pixel
    arrays in file order plus their PIXSIZE keyword.  A minimal FITS reader
    (2880-byte header blocks, BITPIX -64/-32 big-endian images) replaces
    cfitsio.
  * reference_goldens.json -- the golden values the reference's own unit
    tests assert (test/model_test.cc), transcribed with their file:line,
    inputs and tolerances.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _parse_header(buf, off):
    cards = {}
    pos = off
    while True:
        block = buf[pos:pos + 2880].decode("ascii")
        pos += 2880
        done = False
        for i in range(0, 2880, 80):
            card = block[i:i + 80]
            key = card[:8].strip()
            if key == "END":
                done = True
                break
            if card[8:10] == "= ":
                val = card[10:].split("/")[0].strip()
                cards[key] = val
        if done:
            return cards, pos


def read_fits_image(path, hdu=0):
    buf = open(path, "rb").read()
    off = 0
    for k in range(hdu + 1):
        cards, data_off = _parse_header(buf, off)
        naxis = int(cards["NAXIS"])
        dims = [int(cards["NAXIS%d" % (i + 1)]) for i in range(naxis)]
        bitpix = int(cards["BITPIX"])
        nbytes = abs(bitpix) // 8 * int(np.prod(dims)) if naxis else 0
        if k == hdu:
            dt = {-64: ">f8", -32: ">f4"}[bitpix]
            arr = np.frombuffer(buf, dtype=dt, count=int(np.prod(dims)),
                                offset=data_off).astype(np.float64)
            pix = cards.get("PIXSIZE", cards.get("PIXSCALE"))
            return arr.copy(), dims, float(pix)
        off = data_off + ((nbytes + 2879) // 2880) * 2880
    raise ValueError("HDU not found")


def main(refroot):
    td = os.path.join(refroot, "test", "testdata")
    out = {}
    for name, fn, hdu in [("band1", "band1_beam.fits", 0),
                          ("band2", "band2_beam.fits", 0),
                          ("band12_0", "band12_beam_f100.fits", 0),
                          ("band12_1", "band12_beam_f100.fits", 1)]:
        arr, dims, pix = read_fits_image(os.path.join(td, fn), hdu)
        out[name] = arr
        out[name + "_dims"] = np.array(dims, dtype=np.int64)
        out[name + "_pixsize"] = np.array(pix)
    np.savez_compressed(os.path.join(HERE, "beams.npz"), **out)

    f32 = lambda xs: [float(np.float32(x)) for x in xs]  # noqa: E731
    goldens = {
        "source": "aconley/pofd_affine 0.5.1 test/model_test.cc",
        "counts1": {
            "cite": "model_test.cc:171-192",
            "knotpos_f32": f32([0.002, 0.005, 0.010, 0.020, 0.050]),
            "knotval": [10.0, 7.0, 5.0, 4.0, -1.0],
            "interior_tol": 1e-4,
            "testpos": [0.003, 0.007, 0.015],
            "testval_log10": [8.69422, 5.88217, 4.53303],
            "tol": 1e-3,
        },
        "integrals1": {
            "cite": "model_test.cc:196-212",
            "ns": [3.12022e6, 1e4],
            "flux_per_area": [7386.67, 1.0],
            "fluxsq_per_area": [18.132, 0.01],
        },
        "rrange1": {
            "cite": "model_test.cc:216-236 (band1_beam.fits, minval 1e-5)",
            "lower": 0.0, "upper": [0.0488993, 1e-4],
        },
        "R1": {
            "cite": "model_test.cc:241-316 (band1_beam.fits raw and 120-bin"
                    " histogram, minval 1e-5)",
            "flux": [0.003, 0.011, 0.03],
            "R": [1891.52, 0.817009, 0.000313631],
            "reltol": 1e-3,
            "zero_at": [-0.001, 0.1],
        },
        "R1neg": {
            "cite": "model_test.cc:320-394 (band12_beam_f100.fits[0], minval"
                    " 1e-5, raw and makeHistogram(200))",
            "flux": [-0.03, -0.003, -1e-4, 0.003, 0.03],
            "R": [0.0, 0.019075718, 11916638.0, 969.44687, 7.2612855e-5],
            "tol": 1e-3,
        },
        "model2": {
            "cite": "model_test.cc:574-640",
            "knotpos_f32": f32([0.002, 0.005, 0.010, 0.020, 0.040]),
            "sigmapos_f32": f32([0.002, 0.020]),
            "offsetpos_f32": f32([0.03]),
            "pvals": [8.0, 6.0, 4.0, 3.3, 2.0, 0.1, 0.2, -0.03],
            "maxflux": [0.040, 1e-5, 0.067957, 1e-3],
            "beam_max1": [0.97798554, 1e-5],
            "beam_max2": [0.98850347, 1e-5],
            "rrange_upper1": [0.039119421, 1e-4],
            "rrange_upper2": [0.0671758809, 1e-4],
        },
        "integrals2": {
            "cite": "model_test.cc:681-702 (the model2 model)",
            "ns": [57266.8, 10.0],
            "flux_per_area1": [152.262, 0.1],
            "flux_per_area2": [148.585, 0.1],
        },
        "counts2": {
            "cite": "model_test.cc:646-677",
            "f1": [0.003, 0.011, 0.011, 0.03],
            "f2": [0.003, 0.010, 0.015, 0.028],
            "counts": [2.09837e+10, 1.67999e+06, 94125.8, 29739.2],
            "reltol": 1e-3,
        },
        "R2": {
            "cite": "model_test.cc:761-820 (sigma knot 0.015, values"
                    " 0.15/-0.03, band1/band2 beams raw, minval 1e-6)",
            "sigmapos_f32": f32([0.015]),
            "pvals": [8.0, 6.0, 4.0, 3.3, 2.0, 0.15, -0.03],
            "f1": [0.003, 0.011, 0.011, 0.03],
            "f2": [0.003, 0.010, 0.015, 0.028],
            "R": [76926.027, 9.6701326, 11.520839, 0.12455423],
            "grid_f1": [0.003, 0.011, 0.02],
            "grid_f2": [0.003, 0.015],
            "grid_R": [76926.027, 0.024892799, 1.2063052e-15, 11.520839,
                       1.9838477e-34, 0.21958590],
            "reltol": 1e-3,
        },
        "R2hist": {
            "cite": "model_test.cc:824-885 (sigma knot 0.020, 150-bin"
                    " histogram)",
            "sigmapos_f32": f32([0.020]),
            "nhist": 150,
        },
        "R2neg": {
            "cite": "model_test.cc:889-991 (band12_beam_f100.fits[0/1],"
                    " minval 1e-7, mu -0.3, raw then makeHistogram(200))",
            "sigmapos_f32": f32([0.015]),
            "pvals": [8.0, 6.0, 4.0, 3.3, 2.0, 0.15, -0.3],
            "f1": [-2e-4, -2e-4, 0.003, 0.011],
            "f2": [-3e-4, 1e-4, 0.002, 0.010],
            "R": [1.596908e8, 12727124, 75840.624, 20.409118],
            "zero_at": [[0.050, 0.030], [0.050, -0.030], [-0.050, 0.030],
                        [-0.050, -0.030]],
            "grid_f1": [-3e-4, -1e-4, 1e-3],
            "grid_f2": [-2e-4, 0.5e-3],
            "grid_R": [37281355, 771.54407, 45388812, 49.613048, 0.0,
                       7762.3524],
            "hist_flags": [True, False, False, True],
            "reltol": 1e-3,
        },
    }
    with open(os.path.join(HERE, "reference_goldens.json"), "w") as f:
        json.dump(goldens, f, indent=1)
    print("wrote", os.path.join(HERE, "beams.npz"), "and reference_goldens.json")


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("POFD_REFERENCE_DIR")
    if not src:
        sys.exit("usage: make_fixtures.py <reference checkout> (or set POFD_REFERENCE_DIR)")
    main(src)
