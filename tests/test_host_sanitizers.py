"""The host-side set-up code (csrc/setup.cc: beam selection and histograms,
data binning, spline systems, quadrature, flux grids; csrc/fits.cc: FITS
input) built with AddressSanitizer and UndefinedBehaviorSanitizer and run on
small cases, malformed FITS input included.  Any report aborts the program
(-fno-sanitize-recover), so the test passes only on a clean run.  No GPU."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "pofd_affine_b200", "csrc")

DRIVER = r"""
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>
#include "setup.hh"
#include "fits.hh"
using namespace pofd;
int main(int argc, char** argv) {
  const std::string dir = argv[1];
  // 1D beam: selection, histogram, terms; a beam with negative lobes
  std::vector<double> pix(27 * 27), pixn(27 * 27);
  for (int i = 0; i < 27; ++i)
    for (int j = 0; j < 27; ++j) {
      const double r2 = (i - 13.0) * (i - 13.0) + (j - 13.0) * (j - 13.0);
      pix[i * 27 + j] = std::exp(-0.5 * r2 / 1.62);
      pixn[i * 27 + j] = pix[i * 27 + j] - 0.05 * std::exp(-0.5 * r2 / 20.0);
    }
  for (const auto* p : {&pix, &pixn}) {
    Beam1 b;
    b.build(p->data(), p->size(), 6.0, 1e-5);
    b.histogram(120);
    std::vector<double> w, ie;
    b.terms(false, w, ie);
    if (b.hasneg) b.terms(true, w, ie);
    const auto rr = rrange_knots(0.5, b);
    std::printf("beam %zu %zu %g %g\n", b.pos.size(), b.neg.size(), rr.first, rr.second);
  }
  // 2D beam with all four sign components
  std::vector<double> p2(pixn.size());
  for (size_t i = 0; i < p2.size(); ++i) p2[i] = -pixn[(i * 7) % pixn.size()];
  Beam2 b2;
  b2.build(pixn.data(), p2.data(), pixn.size(), 6.0, 1e-6);
  b2.histogram(50);
  std::printf("beam2 %zu %zu %zu %zu\n", b2.nterms(0), b2.nterms(1), b2.nterms(2), b2.nterms(3));
  // data: mean subtraction and binning, 1D and 2D, a one-pixel map
  Data1 d;
  for (int i = 0; i < 5000; ++i) d.data.push_back(0.003 * std::sin(0.1 * i) + 1e-4 * i);
  d.meanSubtract();
  d.applyBinning(300);
  Data1 one;
  one.data = {0.5};
  one.applyBinning(10);
  Data2 dd;
  for (int i = 0; i < 4000; ++i) {
    dd.d1.push_back(std::cos(0.01 * i));
    dd.d2.push_back(std::sin(0.013 * i));
  }
  dd.meanSubtract();
  dd.applyBinning(64, 48);
  // spline systems, grids, quadrature
  std::vector<double> xn(2048);
  for (int i = 0; i < 2048; ++i) xn[i] = 1e-7 * std::pow(2.0, i * 0.01);
  SplineSystem ss;
  ss.factor(xn);
  RGrid1 g;
  g.init(4096, -0.01, 0.8);
  RGrid2Axis a;
  a.init(512, -0.02, 0.4);
  std::vector<double> lk = {std::log2(0.002), std::log2(0.01), std::log2(0.05), std::log2(0.4)};
  KnotQuadrature kq;
  kq.build(lk.data(), 4, 8, 20);
  kq.build_breaks(lk.data(), 4, {std::log2(0.004), std::log2(0.02)}, 8, 20);
  NatSpline ns;
  double xs[3] = {0.0, 1.0, 2.0}, ys[3] = {1.0, 3.0, 2.0};
  ns.init(xs, ys, 3);
  // FITS files written by the test, then malformed ones: every error is an
  // exception, never a read out of bounds
  const std::vector<double> dm = fits_read_data(dir + "/m.fits", false, true);
  const FitsBeam fb = fits_read_beam(dir + "/b.fits");
  std::vector<double> x1, x2;
  fits_read_data2(dir + "/m.fits", dir + "/m.fits", false, false, &x1, &x2);
  int errors = 0;
  for (const char* f : {"/trunc_head.fits", "/trunc_data.fits", "/junk.fits", "/nofile.fits",
                        "/cube.fits", "/negaxis.fits", "/bigaxis.fits", "/negpcount.fits",
                        "/gcount0.fits"}) {
    try {
      fits_read_data(dir + f, false, false);
    } catch (const Error&) {
      ++errors;
    }
  }
  // beams with corrupt axis sizes are rejected as well
  for (const char* f : {"/negaxis.fits", "/bigaxis.fits"}) {
    try {
      fits_read_beam(dir + f);
    } catch (const Error&) {
      ++errors;
    }
  }
  std::printf("fits %zu %ld %ld %zu errors %d\n", dm.size(), fb.nx, fb.ny, x1.size(), errors);
  return 0;
}
"""


def _raw_header(cards, nbytes_data=2880):
    """A primary HDU written card by card (no validation): 80-character
    cards, END, padded to 2880-byte blocks, then nbytes_data of zeros."""
    txt = "".join(c.ljust(80)[:80] for c in cards + ["END"])
    txt = txt.ljust((len(txt) + 2879) // 2880 * 2880)
    return txt.encode("ascii") + b"\0" * nbytes_data


def _card(key, val):
    return "%-8s= %20s" % (key, val)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_setup_and_fits_under_asan_ubsan(tmp_path):
    from test_fits_input import _hdu, _write
    img = np.random.default_rng(1).normal(size=(20, 30))
    mask = np.zeros((20, 30), np.int32)
    mask[3:6] = 1
    m = _write(tmp_path / "m.fits", _hdu(img, -64, True), _hdu(mask, 32, False, "MASK"))
    _write(tmp_path / "b.fits", _hdu(img[:9, :9], -32, True, keys=[("PIXSIZE", 4.0)]))
    raw = open(m, "rb").read()
    (tmp_path / "trunc_head.fits").write_bytes(raw[:1000])
    (tmp_path / "trunc_data.fits").write_bytes(raw[:2880 + 1000])
    (tmp_path / "junk.fits").write_bytes(b"\x00\xff" * 3000)
    _write(tmp_path / "cube.fits", _hdu(np.ones((2, 3, 4)), -64, True))
    base = [_card("SIMPLE", "T"), _card("BITPIX", -64), _card("NAXIS", 2)]
    (tmp_path / "negaxis.fits").write_bytes(_raw_header(
        base + [_card("NAXIS1", -1), _card("NAXIS2", -1)]))
    (tmp_path / "bigaxis.fits").write_bytes(_raw_header(
        base + [_card("NAXIS1", 2 ** 32), _card("NAXIS2", 2 ** 32)]))
    (tmp_path / "negpcount.fits").write_bytes(_raw_header(
        base + [_card("NAXIS1", 4), _card("NAXIS2", 4), _card("PCOUNT", -100)]))
    (tmp_path / "gcount0.fits").write_bytes(_raw_header(
        base + [_card("NAXIS1", 4), _card("NAXIS2", 4), _card("GCOUNT", 0)]))
    src = tmp_path / "drv.cc"
    src.write_text(DRIVER)
    exe = tmp_path / "drv"
    flags = ["-std=c++17", "-O1", "-g", "-fsanitize=address,undefined",
             "-fno-sanitize-recover=all", "-fno-omit-frame-pointer"]
    subprocess.check_call(["g++"] + flags + [str(src), os.path.join(CSRC, "setup.cc"),
                                             os.path.join(CSRC, "fits.cc"), "-I", CSRC,
                                             "-o", str(exe)])
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True,
                       env=env, timeout=300)
    assert r.returncode == 0, r.stderr[-4000:]
    assert "errors 11" in r.stdout
    assert "fits 510 9 9 510" in r.stdout  # 600 pixels, 3 rows of 30 masked


ORACLE_DRIVER = r"""
#include <cmath>
#include <cstdio>
#include <vector>
#include "pofd_oracle.h"
int main() {
  // a small 1D likelihood through the CPU oracle (test infrastructure),
  // two beam sets, binned and unbinned data, a batch on two threads
  std::vector<double> pix(27 * 27);
  for (int i = 0; i < 27; ++i)
    for (int j = 0; j < 27; ++j) {
      const double r2 = (i - 13.0) * (i - 13.0) + (j - 13.0) * (j - 13.0);
      pix[i * 27 + j] = std::exp(-0.5 * r2 / 1.62);
    }
  double knots[5] = {0.002, 0.005, 0.02, 0.08, 0.3};
  std::vector<double> data(3000);
  for (int i = 0; i < 3000; ++i) data[i] = 0.004 * std::sin(0.37 * i) + 0.001 * std::cos(1.3 * i);
  float th[6] = {6.5f, 5.2f, 3.4f, 1.9f, 0.1f, 1.0f};
  for (int binned = 0; binned < 2; ++binned) {
    void* L = orc_like1_new(5, knots, 2048, 256, binned, 200);
    const int b0 = orc_like1_add_beamset(L, pix.data(), pix.size(), 6.0, 1e-5, 1, 120, 0.0);
    const int b1 = orc_like1_add_beamset(L, pix.data(), pix.size(), 6.0, 1e-5, 0, 0, 0.0);
    orc_like1_add_dataset(L, b0, data.data(), data.size(), 1, 0.003, 1.0);
    orc_like1_add_dataset(L, b1, data.data(), data.size() / 2, 1, 0.004, 1.0);
    orc_like1_set_rranges(L, th, 6);
    double ll = 0.0;
    const int st = orc_like1_eval(L, th, 6, &ll);
    std::vector<float> ths(4 * 6);
    for (int k = 0; k < 4; ++k)
      for (int p = 0; p < 6; ++p) ths[k * 6 + p] = th[p] + 0.01f * k * (p < 5);
    std::vector<double> lls(4);
    std::vector<int> sts(4);
    orc_like1_eval_batch(L, 4, ths.data(), 6, lls.data(), sts.data(), 2);
    orc_set_fast_fft(1);
    double llf = 0.0;
    const int stf = orc_like1_eval(L, th, 6, &llf);
    orc_set_fast_fft(0);
    std::printf("oracle binned %d status %d finite %d fast %d %d\n", binned, st,
                std::isfinite(ll) ? 1 : 0, stf, std::fabs(llf - ll) < 1e-6 ? 1 : 0);
    orc_like1_free(L);
  }
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_oracle_under_asan_ubsan(tmp_path):
    odir = os.path.join(ROOT, "oracle")
    src = tmp_path / "odrv.cc"
    src.write_text(ORACLE_DRIVER)
    exe = tmp_path / "odrv"
    flags = ["-std=c++17", "-O1", "-g", "-pthread", "-ffp-contract=off",
             "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
             "-fno-omit-frame-pointer"]
    subprocess.check_call(["g++"] + flags + [str(src), os.path.join(odir, "pofd_oracle.cc"),
                                             os.path.join(odir, "numerics.cc"),
                                             os.path.join(odir, "fastfft.cc"), "-I", odir,
                                             "-o", str(exe)])
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-4000:]
    assert "oracle binned 0 status 0 finite 1 fast 0 1" in r.stdout
    assert "oracle binned 1 status 0 finite 1 fast 0 1" in r.stdout
