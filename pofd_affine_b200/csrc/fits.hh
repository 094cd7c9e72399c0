// fits.hh -- FITS image reading for the data and beam maps (fits.cc).
#ifndef POFD_FITS_HH
#define POFD_FITS_HH

#include <string>
#include <vector>

#include "setup.hh"

namespace pofd {

// fitsData::readData (fitsData.cc:56-316): the image of an "image"/"IMAGE"
// extension, else of the primary HDU (or of HDU k with a "[k]" suffix),
// without the pixels a "mask"/"MASK" extension marks non-zero (unless
// ignore_mask), in file order, mean-subtracted on request.
std::vector<double> fits_read_data(const std::string& spec, bool ignore_mask, bool meansub);

// fitsDataDouble::readData (fitsDataDouble.cc:304-430): the two bands'
// images read as above, the same number of pixels in each, masked jointly.
void fits_read_data2(const std::string& spec1, const std::string& spec2, bool ignore_mask,
                     bool meansub, std::vector<double>* out1, std::vector<double>* out2);

struct FitsBeam {
  std::vector<double> pix;  // file order, first axis fastest
  long nx = 0, ny = 0;
  double pixsize = 0.0;     // PIXSIZE, else PIXSCALE
};
// beam::readFile (beam.cc:295-395): the primary HDU (or HDU k of "[k]").
FitsBeam fits_read_beam(const std::string& spec);

}  // namespace pofd
#endif
