// Minimal FITS primary-image I/O for the command-line tools (FITS standard 4.0; no cfitsio).
#pragma once
#include <string>
#include <vector>

namespace svdi_io {
// Reads a 1-D or 2-D primary image converted to float (any BITPIX, BSCALE/BZERO applied).
// naxes[1] is 1 for a 1-D image (archive/pipe_interface.cpp:34-46). Throws std::runtime_error.
std::vector<float> read_fits_image(const std::string& path, long naxes[2]);
// Writes a 2-D FLOAT_IMG (BITPIX -32), NAXIS1 = axis0 (fast axis); overwrites.
void write_fits_2d(const std::string& path, const float* values, long axis0, long axis1);
}
