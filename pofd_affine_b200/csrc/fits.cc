// fits.cc -- reading the FITS images the reference's drivers take: the data
// maps with their optional mask (fitsData::readData, fitsData.cc:56-316;
// fitsDataDouble::readData reads one map per band and masks them jointly,
// fitsDataDouble.cc:304-430) and the beam maps with their pixel size
// (beam::readFile, beam.cc:295-395; doublebeam reads two).
//
// A FITS file is a sequence of header-data units (HDUs): a header of
// 80-character "KEYWORD = value" cards in 2880-byte blocks ending at END,
// then the data, big-endian, padded to a 2880-byte multiple.  This reader
// handles images (BITPIX 8, 16, 32, 64, -32, -64, with BSCALE/BZERO), walks
// the HDUs by their sizes (NAXISn, PCOUNT, GCOUNT) and selects one by number
// (the cfitsio "file.fits[k]" suffix) or by EXTNAME.  Checksums are not
// verified.
#include "fits.hh"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

namespace pofd {

namespace {

constexpr size_t kBlock = 2880;

struct Hdu {
  std::map<std::string, std::string> keys;  // values as written (quotes stripped)
  size_t data_off = 0;                      // byte offset of the data
  size_t data_bytes = 0;                    // unpadded data size
  int bitpix = 0;
  std::vector<long> naxes;
};

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
  while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
  return s.substr(a, b - a);
}

// Value field of a card: a quoted string (quotes removed, '' unescaped) or
// the text before a '/' comment.
std::string card_value(const std::string& card) {
  std::string v = card.size() > 10 ? card.substr(10) : std::string();
  size_t i = 0;
  while (i < v.size() && v[i] == ' ') ++i;
  if (i < v.size() && v[i] == '\'') {
    std::string out;
    for (size_t j = i + 1; j < v.size(); ++j) {
      if (v[j] == '\'') {
        if (j + 1 < v.size() && v[j + 1] == '\'') {
          out += '\'';
          ++j;
        } else {
          break;
        }
      } else {
        out += v[j];
      }
    }
    return trim(out);
  }
  const size_t slash = v.find('/');
  return trim(slash == std::string::npos ? v : v.substr(0, slash));
}

long key_long(const Hdu& h, const std::string& k, long dflt, bool required,
              const std::string& path) {
  auto it = h.keys.find(k);
  if (it == h.keys.end()) {
    if (required) throw Error(POFD_E_ARG, "FITS header of " + path + " lacks " + k);
    return dflt;
  }
  return std::stol(it->second);
}

double key_double(const Hdu& h, const std::string& k, double dflt) {
  auto it = h.keys.find(k);
  if (it == h.keys.end()) return dflt;
  std::string v = it->second;
  for (auto& c : v)
    if (c == 'D' || c == 'd') c = 'E';  // Fortran exponent
  return std::stod(v);
}

std::vector<Hdu> scan(const std::string& path, const std::string& buf) {
  std::vector<Hdu> hdus;
  size_t pos = 0;
  while (pos + kBlock <= buf.size()) {
    Hdu h;
    bool end = false;
    size_t p = pos;
    while (!end) {
      if (p + kBlock > buf.size()) throw Error(POFD_E_ARG, "FITS header of " + path + " is truncated");
      for (size_t c = 0; c < kBlock; c += 80) {
        const std::string card = buf.substr(p + c, 80);
        const std::string key = trim(card.substr(0, 8));
        if (key == "END") {
          end = true;
          break;
        }
        if (card.size() >= 10 && card[8] == '=' && card[9] == ' ')
          h.keys[key] = card_value(card);
      }
      p += kBlock;
    }
    if (hdus.empty() && h.keys.find("SIMPLE") == h.keys.end())
      throw Error(POFD_E_ARG, path + " is not a FITS file");
    h.bitpix = static_cast<int>(key_long(h, "BITPIX", 0, true, path));
    const long naxis = key_long(h, "NAXIS", 0, true, path);
    // FITS standard 4.4.1: 0 <= NAXIS <= 999, NAXISn >= 0, PCOUNT >= 0,
    // GCOUNT >= 1; the data size is |BITPIX|/8 * GCOUNT * (PCOUNT + prod
    // NAXISn), computed with overflow checks so that a corrupt header ends
    // in an error instead of a wrapped size
    if (naxis < 0 || naxis > 999) throw Error(POFD_E_ARG, "Invalid NAXIS in " + path);
    auto bad_size = [&]() { return Error(POFD_E_ARG, "Invalid data size in FITS header of " + path); };
    size_t prod = naxis > 0 ? 1 : 0;
    for (long a = 1; a <= naxis; ++a) {
      const long na = key_long(h, "NAXIS" + std::to_string(a), 0, true, path);
      if (na < 0) throw Error(POFD_E_ARG, "Negative NAXIS" + std::to_string(a) + " in " + path);
      h.naxes.push_back(na);
      if (__builtin_mul_overflow(prod, static_cast<size_t>(na), &prod)) throw bad_size();
    }
    const long pcount = key_long(h, "PCOUNT", 0, false, path);
    const long gcount = key_long(h, "GCOUNT", 1, false, path);
    if (pcount < 0) throw Error(POFD_E_ARG, "Negative PCOUNT in " + path);
    if (gcount < 1) throw Error(POFD_E_ARG, "GCOUNT below 1 in " + path);
    size_t elems = 0, bytes = 0, padded = 0, next = 0;
    if (__builtin_add_overflow(prod, static_cast<size_t>(pcount), &elems) ||
        __builtin_mul_overflow(elems, static_cast<size_t>(gcount), &elems) ||
        __builtin_mul_overflow(elems, static_cast<size_t>(std::abs(h.bitpix) / 8), &bytes) ||
        __builtin_add_overflow(bytes, kBlock - 1, &padded) ||
        __builtin_add_overflow(p, padded / kBlock * kBlock, &next))
      throw bad_size();
    h.data_off = p;
    h.data_bytes = bytes;
    hdus.push_back(h);
    // the next header starts after this one's data, inside the file; a data
    // block that runs past the end is caught where the data is read
    if (next <= pos) throw bad_size();
    pos = next;
  }
  if (hdus.empty()) throw Error(POFD_E_ARG, path + " is not a FITS file");
  return hdus;
}

// "file.fits[k]" -> ("file.fits", k); no suffix -> (path, -1)
std::pair<std::string, int> split_selector(const std::string& spec) {
  if (!spec.empty() && spec.back() == ']') {
    const size_t lb = spec.rfind('[');
    if (lb != std::string::npos) {
      const std::string inner = spec.substr(lb + 1, spec.size() - lb - 2);
      if (!inner.empty() && inner.find_first_not_of("0123456789") == std::string::npos)
        return {spec.substr(0, lb), std::stoi(inner)};
    }
  }
  return {spec, -1};
}

std::string read_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw Error(POFD_E_ARG, "Error opening input file: " + path);
  std::ostringstream s;
  s << f.rdbuf();
  return s.str();
}

int find_ext(const std::vector<Hdu>& hdus, const char* name) {
  for (size_t i = 1; i < hdus.size(); ++i) {
    auto it = hdus[i].keys.find("EXTNAME");
    if (it != hdus[i].keys.end() && it->second == name) return static_cast<int>(i);
  }
  return -1;
}

// Pixel values of a 2D image HDU, file order (first axis fastest), as
// doubles with BSCALE/BZERO applied.
std::vector<double> pixels(const std::string& path, const std::string& buf, const Hdu& h,
                           long* nx, long* ny, const char* what) {
  if (h.naxes.size() != 2) throw Error(POFD_E_ARG, std::string(what) + " in " + path + " is not 2D");
  *nx = h.naxes[0];
  *ny = h.naxes[1];
  const size_t n = static_cast<size_t>(*nx) * static_cast<size_t>(*ny);
  const int bp = h.bitpix;
  const size_t nb = static_cast<size_t>(std::abs(bp) / 8);
  if (h.data_off + n * nb > buf.size()) throw Error(POFD_E_ARG, "FITS data of " + path + " is truncated");
  const double bscale = key_double(h, "BSCALE", 1.0), bzero = key_double(h, "BZERO", 0.0);
  std::vector<double> out(n);
  const unsigned char* d = reinterpret_cast<const unsigned char*>(buf.data()) + h.data_off;
  for (size_t i = 0; i < n; ++i) {
    uint64_t u = 0;
    for (size_t b = 0; b < nb; ++b) u = (u << 8) | d[i * nb + b];
    double v;
    switch (bp) {
      case 8: v = static_cast<double>(static_cast<uint8_t>(u)); break;
      case 16: v = static_cast<double>(static_cast<int16_t>(static_cast<uint16_t>(u))); break;
      case 32: v = static_cast<double>(static_cast<int32_t>(static_cast<uint32_t>(u))); break;
      case 64: v = static_cast<double>(static_cast<int64_t>(u)); break;
      case -32: {
        const uint32_t w = static_cast<uint32_t>(u);
        float f;
        std::memcpy(&f, &w, 4);
        v = static_cast<double>(f);
        break;
      }
      case -64: std::memcpy(&v, &u, 8); break;
      default: throw Error(POFD_E_ARG, "Unsupported BITPIX in " + path);
    }
    out[i] = (bscale == 1.0 && bzero == 0.0) ? v : bzero + bscale * v;
  }
  return out;
}

}  // namespace

namespace {

struct ImageMask {
  std::vector<double> data;
  std::vector<unsigned int> mask;  // empty: no mask (or ignored)
};

// The image of a data file and, unless ignored, its mask extension
// (fitsData.cc:94-275, fitsDataDouble.cc:94-295): the selected HDU, else an
// "image"/"IMAGE" extension, else the primary; the mask from a
// "mask"/"MASK" extension, read as unsigned integers.
ImageMask read_image_mask(const std::string& spec, bool ignore_mask) {
  const auto sel = split_selector(spec);
  const std::string& path = sel.first;
  const std::string buf = read_file(path);
  const std::vector<Hdu> hdus = scan(path, buf);
  int ih = sel.second;
  if (ih < 0) {
    ih = find_ext(hdus, "image");
    if (ih < 0) ih = find_ext(hdus, "IMAGE");
    if (ih < 0) ih = 0;
  }
  if (ih >= static_cast<int>(hdus.size())) throw Error(POFD_E_ARG, "No HDU " + std::to_string(ih) + " in " + path);
  long nx = 0, ny = 0;
  ImageMask im;
  im.data = pixels(path, buf, hdus[ih], &nx, &ny, "Image");
  if (im.data.empty()) throw Error(POFD_E_ARG, "Image in " + path + " is empty");
  if (!ignore_mask) {
    int mh = find_ext(hdus, "mask");
    if (mh < 0) mh = find_ext(hdus, "MASK");
    if (mh >= 0) {
      long mx = 0, my = 0;
      const std::vector<double> m = pixels(path, buf, hdus[mh], &mx, &my, "Mask");
      if (m.empty()) throw Error(POFD_E_ARG, "Mask present zero extent");
      if (mx != nx) throw Error(POFD_E_ARG, "Mask does not match image extent along first dimension");
      if (my != ny) throw Error(POFD_E_ARG, "Mask does not match image extent along second dimension");
      im.mask.resize(m.size());
      for (size_t i = 0; i < m.size(); ++i) im.mask[i] = static_cast<unsigned int>(m[i]);
    }
  }
  return im;
}

}  // namespace

std::vector<double> fits_read_data(const std::string& spec, bool ignore_mask, bool meansub) {
  ImageMask im = read_image_mask(spec, ignore_mask);
  std::vector<double> data;
  if (im.mask.empty()) {
    data.swap(im.data);
  } else {
    // keep the pixels whose mask is 0, in file order (fitsData.cc:286-312)
    data.reserve(im.data.size());
    for (size_t i = 0; i < im.data.size(); ++i)
      if (im.mask[i] == 0u) data.push_back(im.data[i]);
    if (data.empty()) throw Error(POFD_E_ARG, "All data masked");
  }
  if (meansub) {
    Data1 d;
    d.data = data;
    d.meanSubtract();
    data.swap(d.data);
  }
  return data;
}

void fits_read_data2(const std::string& spec1, const std::string& spec2, bool ignore_mask,
                     bool meansub, std::vector<double>* out1, std::vector<double>* out2) {
  ImageMask a = read_image_mask(spec1, ignore_mask);
  ImageMask b = read_image_mask(spec2, ignore_mask);
  if (a.data.size() != b.data.size())
    throw Error(POFD_E_ARG, "Data from file1 and file2 not the same size");
  const size_t n = a.data.size();
  Data2 d;
  if (a.mask.empty() && b.mask.empty()) {
    d.d1.swap(a.data);
    d.d2.swap(b.data);
  } else {
    // fitsDataDouble.cc:338-395: with both masks a pixel is dropped only
    // where the two mask values share a set bit (mask1 & mask2); with one,
    // where that mask is non-zero
    const bool both = !a.mask.empty() && !b.mask.empty();
    for (size_t i = 0; i < n; ++i) {
      const unsigned int m = both ? (a.mask[i] & b.mask[i]) : (a.mask.empty() ? b.mask[i] : a.mask[i]);
      if (m == 0u) {
        d.d1.push_back(a.data[i]);
        d.d2.push_back(b.data[i]);
      }
    }
    if (d.d1.empty()) throw Error(POFD_E_ARG, "All data masked");
  }
  if (meansub) d.meanSubtract();
  out1->swap(d.d1);
  out2->swap(d.d2);
}

FitsBeam fits_read_beam(const std::string& spec) {
  const auto sel = split_selector(spec);
  const std::string& path = sel.first;
  const std::string buf = read_file(path);
  const std::vector<Hdu> hdus = scan(path, buf);
  const int ih = sel.second < 0 ? 0 : sel.second;
  if (ih >= static_cast<int>(hdus.size())) throw Error(POFD_E_ARG, "No HDU " + std::to_string(ih) + " in " + path);
  const Hdu& h = hdus[ih];
  FitsBeam b;
  if (h.keys.count("PIXSIZE")) b.pixsize = key_double(h, "PIXSIZE", 0.0);
  else if (h.keys.count("PIXSCALE")) b.pixsize = key_double(h, "PIXSCALE", 0.0);
  else throw Error(POFD_E_ARG, "Unable to find pixel scale information in " + path);
  if (h.naxes.size() != 2) throw Error(POFD_E_ARG, "Input BEAM is not 2D");
  long nx = 0, ny = 0;
  b.pix = pixels(path, buf, h, &nx, &ny, "Beam");
  b.nx = nx;
  b.ny = ny;
  return b;
}

}  // namespace pofd
