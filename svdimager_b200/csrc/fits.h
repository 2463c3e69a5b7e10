// Minimal FITS primary-image I/O for the command-line tools (FITS standard 4.0; no cfitsio).
#pragma once
#include <string>
#include <vector>

namespace svdi_io {
// Reads a 1-D or 2-D primary image converted to float (any BITPIX, BSCALE/BZERO applied).
// naxes[1] is 1 for a 1-D image (archive/pipe_interface.cpp:34-46). Throws std::runtime_error.
std::vector<float> read_fits_image(const std::string& path, long naxes[2]);
// Writes a 2-D FLOAT_IMG (BITPIX -32), NAXIS1 = axis0 (fast axis); overwrites. extra_cards are
// complete 80-character header cards placed before END.
void write_fits_2d(const std::string& path, const float* values, long axis0, long axis1,
                   const std::vector<std::string>& extra_cards = {});
// World coordinates of an N x N SIN-projected dirty image (FITS WCS paper II): reference pixel at the
// image centre (0-based N / 2, the imager's phase centre), cell_rad per pixel, RA decreasing along
// axis 1 as the imager's reprojection lays the image out, phase centre (ra_deg, dec_deg).
std::vector<std::string> sin_wcs_cards(long image_size, double cell_rad, double ra_deg, double dec_deg);
// sin_wcs_cards for the phase centre in the environment variable SVDI_FITS_WCS ("ra_deg,dec_deg"),
// none when it is unset (the reference writes bare images). Throws on a malformed value.
std::vector<std::string> wcs_cards_from_env(long image_size, double cell_rad);
}
