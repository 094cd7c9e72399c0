"""The header-only C++ shim (include/pofd_b200.hpp) compiles against the C
ABI, links libpofd_b200.so and raises the reference-style exceptions; the
set-up half runs on a host-only context (no GPU)."""
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROG = r"""
#include <cstdio>
#include <vector>
#include <cmath>
#include "pofd_b200.hpp"
int main() {
  pofd_b200::Context ctx(-1);
  std::vector<double> beam(27 * 27);
  for (int i = 0; i < 27; ++i)
    for (int j = 0; j < 27; ++j) {
      double r2 = (i - 13) * (i - 13) + (j - 13) * (j - 13);
      beam[i * 27 + j] = std::exp(-0.5 * r2 / (1.274 * 1.274));
    }
  pofd_b200::Beam1 bm(beam.data(), beam.size(), 6.0, true, 120, 1e-5);
  double knots[5] = {0.002, 0.005, 0.02, 0.08, 0.3};
  pofd_b200::Like1 like(ctx, 5, knots, 2048, 256, true, 200);
  int bs = like.addBeamSet(bm);
  std::vector<double> data(1000);
  for (int i = 0; i < 1000; ++i) data[i] = 0.002 * std::sin(0.37 * i);
  like.addDataset(bs, data.data(), data.size(), 0.002);
  float th[6] = {6.5f, 5.2f, 3.4f, 1.9f, 0.1f, 1.0f};
  like.setRRanges(th, 6);
  int code = 0;
  try {
    bool inv = false;
    like.getLogLike(th, 6, inv);   // needs a GPU: host-only context throws
  } catch (const pofd_b200::Exception& e) {
    code = e.code();
  }
  try {
    std::vector<double> zero(25, 0.0);
    pofd_b200::Beam1 bad(zero.data(), zero.size(), 6.0);
  } catch (const pofd_b200::Exception& e) {
    std::printf("beam %d\n", e.code());
  }
  std::printf("loglike %d\n", code);
  // the 2D classes: set-up on the host, evaluation needs a GPU
  std::vector<double> beam2(27 * 27);
  for (size_t i = 0; i < beam2.size(); ++i) beam2[i] = std::pow(beam[i], 0.6);
  pofd_b200::Beam2 bm2(beam.data(), beam2.data(), beam.size(), 6.0, true, 40, 1e-6);
  double sk[2] = {0.003, 0.3}, ok[1] = {0.01};
  pofd_b200::Like2 like2(ctx, 5, knots, 2, sk, 1, ok, 256, 64, true, true, 100);
  int bs2 = like2.addBeamSet(bm2);
  std::vector<double> d2(1000);
  for (int i = 0; i < 1000; ++i) d2[i] = 0.0025 * std::cos(0.41 * i);
  like2.addDataset(bs2, data.data(), d2.data(), data.size(), 0.002, 0.0025);
  float th2[10] = {6.5f, 5.2f, 3.4f, 1.9f, 0.1f, 0.2f, 0.25f, -0.3f, 1.0f, 1.0f};
  int code2 = 0;
  try {
    like2.setRRanges(th2, 10);
    bool inv = false;
    like2.getLogLike(th2, 10, inv);
  } catch (const pofd_b200::Exception& e) {
    code2 = e.code();
  }
  std::printf("loglike2 %d\n", code2);
  return 0;
}
"""


def test_cpp_shim_compiles_links_and_throws(built_lib, tmp_path):
    src = tmp_path / "shim.cc"
    src.write_text(PROG)
    exe = tmp_path / "shim"
    libdir = os.path.dirname(built_lib)
    subprocess.check_call(["g++", "-std=c++17", "-O1", str(src), "-I",
                           os.path.join(ROOT, "include"), "-L", libdir,
                           "-lpofd_b200", "-Wl,-rpath," + libdir, "-o",
                           str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True,
                         check=True).stdout
    assert "beam -10" in out
    assert "loglike -11" in out
    assert "loglike2 -11" in out


PROG_FILES = r"""
#include <cstdio>
#include <string>
#include <vector>
#include "pofd_b200.hpp"
int main(int argc, char** argv) {
  const std::string dir = argv[1];
  pofd_b200::Context ctx(-1);
  double knots[5] = {0.002, 0.005, 0.02, 0.08, 0.3};
  pofd_b200::Like1 like(ctx, 5, knots, 2048, 256, true, 100);
  like.readDataFromFiles({dir + "/d0.fits", dir + "/d1.fits", dir + "/d2.fits"},
                         {dir + "/z_beam.fits", dir + "/a_beam.fits", dir + "/z_beam.fits"},
                         {0.002, 0.003, 0.004}, {1.0, 1.0, 1.0}, false, true, 1e-5, true, 120);
  double info[9];
  pofd_like1_dataset_info(like.get(), 1, 1, info, nullptr);
  std::printf("set1ds1 ndata %g sigma %g\n", info[0], info[5]);
  pofd_like1_dataset_info(like.get(), 0, 0, info, nullptr);
  std::printf("set0ds0 ndata %g sigma %g\n", info[0], info[5]);
  double sk[2] = {0.003, 0.3}, ok[1] = {0.01};
  pofd_b200::Like2 like2(ctx, 5, knots, 2, sk, 1, ok, 256, 64, true, true, 50);
  like2.readDataFromFiles({dir + "/d0.fits"}, {dir + "/d1.fits"}, {dir + "/z_beam.fits"},
                          {dir + "/a_beam.fits"}, {0.002}, {0.003}, {1.0}, false, true, 1e-6,
                          true, 40);
  double info10[10];
  pofd_like2_dataset_info(like2.get(), 0, 0, info10, nullptr);
  std::printf("like2 ndata %g sigma2 %g\n", info10[0], info10[8]);
  return 0;
}
"""


def test_cpp_shim_reads_data_from_files(built_lib, tmp_path):
    """readDataFromFiles with the reference's signature and grouping: the
    a_beam group comes first (file-name order), the z_beam group holds the
    first and third datasets in input order; the masked map loses its
    masked pixels."""
    from test_fits_input import _hdu, _write
    from pofd_affine_b200 import synth
    bm = synth.gaussian_beam(3.0)
    _write(tmp_path / "z_beam.fits", _hdu(bm, -64, True, keys=[("PIXSIZE", 6.0)]))
    _write(tmp_path / "a_beam.fits", _hdu(bm ** 1.2, -64, True, keys=[("PIXSIZE", 6.0)]))
    rng = np.random.default_rng(3)
    for i in range(3):
        m = rng.normal(0, 0.002, (30, 30))
        if i == 2:
            mask = np.zeros((30, 30), np.int32)
            mask[:5] = 1
            _write(tmp_path / ("d%d.fits" % i), _hdu(m, -64, True),
                   _hdu(mask, 32, False, "MASK"))
        else:
            _write(tmp_path / ("d%d.fits" % i), _hdu(m, -64, True))
    src = tmp_path / "files.cc"
    src.write_text(PROG_FILES)
    exe = tmp_path / "files"
    libdir = os.path.dirname(built_lib)
    subprocess.check_call(["g++", "-std=c++17", "-O1", str(src), "-I",
                           os.path.join(ROOT, "include"), "-L", libdir,
                           "-lpofd_b200", "-Wl,-rpath," + libdir, "-o", str(exe)])
    out = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True,
                         check=True).stdout
    assert "set1ds1 ndata 750 sigma 0.004" in out
    assert "set0ds0 ndata 900 sigma 0.003" in out
    assert "like2 ndata 900 sigma2 0.003" in out
