// sharedlibrary_gpu Visreal.fits Visimag.fits B.fits V.fits Image_Size Number_of_Rows Cell_Size Out.fits
// Same argument order and behaviour as the archive CLI (archive/pipe_interface.cpp:139-186): reads
// the four FITS inputs as float, calls FIpipe, writes the image (overwriting). Unlike the
// reference it checks argc (usage, exit 2) and the array sizes, and reports FIpipe errors.
#include <chrono>
#include <cstdio>
#include <exception>
#include <iostream>
#include <string>
#include <vector>

#include "fits.h"
#include "svdimager_b200.h"

int main(int argc, char** argv) {
    if (argc != 9) {
        std::cerr << "Usage: " << argv[0]
                  << " Visreal.fits Visimag.fits B.fits V.fits Image_Size Number_of_Rows Cell_Size Output_Name.fits\n";
        return 2;
    }
    try {
        long nv[2], ni[2], nb[2], nV[2];
        std::vector<float> visreal = svdi_io::read_fits_image(argv[1], nv);
        std::vector<float> visimag = svdi_io::read_fits_image(argv[2], ni);
        std::vector<float> bin = svdi_io::read_fits_image(argv[3], nb);
        std::vector<float> vin = svdi_io::read_fits_image(argv[4], nV);
        const size_t image_size = std::stoul(argv[5]);
        const size_t num_baselines = std::stoul(argv[6]);
        const float cell_size = std::stof(argv[7]);
        const std::string out = argv[8];
        if (visreal.size() < num_baselines || visimag.size() < num_baselines || bin.size() < 3 * num_baselines ||
            vin.size() < 9) {
            std::cerr << "input FITS arrays are shorter than Number_of_Rows\n";
            return 1;
        }
        std::vector<float> dirty(image_size * image_size, 0.0f);
        const auto t0 = std::chrono::high_resolution_clock::now();
        const int st = FIpipe(visreal.data(), visimag.data(), bin.data(), vin.data(), dirty.data(), num_baselines,
                              image_size, cell_size);
        const auto t1 = std::chrono::high_resolution_clock::now();
        if (st != 0) {
            std::cerr << "FIpipe failed: " << svdi_last_error() << "\n";
            return 1;
        }
        std::cout << "Time elapsed: " << std::chrono::duration<double, std::milli>(t1 - t0).count() << " ms"
                  << std::endl;
        svdi_io::write_fits_2d(out, dirty.data(), (long)image_size, (long)image_size,
                               svdi_io::wcs_cards_from_env((long)image_size, cell_size));
        return 0;
    } catch (const std::exception& ex) {
        std::cerr << "sharedlibrary_gpu failed: " << ex.what() << "\n";
        return 1;
    }
}
