// svd_integrated_imager_gpu Snapshots Image_Size Cell_Size Snapshot_Index Output_Name.fits
// Argument order and exit codes of SVDIntegratedImager.cu:1763-1854 (argc != 6: usage, exit 2;
// errors: message, exit 1). The first argument is a snapshot bundle (svdimager_b200/bundle.py),
// which stands in for a Measurement Set: this library reads no casacore tables.
#include <chrono>
#include <exception>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "bundle.h"
#include "fits.h"
#include "svdimager_b200.h"

int main(int argc, char** argv) {
    if (argc != 6) {
        std::cerr << "Usage: " << argv[0] << " MeasurementSet Image_Size Cell_Size Snapshot_Index Output_Name.fits\n";
        return 2;
    }
    try {
        const std::string ms_path(argv[1]);
        const size_t image_size = std::stoul(argv[2]);
        const float cell_size = std::stof(argv[3]);
        const size_t snapshot_index = std::stoul(argv[4]);
        const std::string output_name(argv[5]);
        if (image_size == 0) throw std::runtime_error("Image_Size must be greater than zero");
        if (cell_size <= 0.0f) throw std::runtime_error("Cell_Size must be greater than zero");
        const auto total_start = std::chrono::high_resolution_clock::now();
        std::cerr << "Reading snapshots by TIME: " << ms_path << '\n';
        size_t total = 0;
        svdi_io::HostSnapshot s = svdi_io::read_bundle_snapshot(ms_path, snapshot_index, total);
        std::cerr << "Found " << total << " TIME snapshot(s)\n";
        std::cerr << "Selected snapshot " << s.index << " time " << s.time << " rows " << s.num_rows << " samples "
                  << s.num_samples << '\n';
        svdi_host_ms h{};
        h.num_rows = s.num_rows;
        h.num_channels = s.num_channels;
        h.num_samples = s.num_samples;
        h.uvw = s.uvw.data();
        h.frequencies_hz = s.frequencies_hz.data();
        h.vis0_real = s.vis0_real.data();
        h.vis0_imag = s.vis0_imag.data();
        h.vis3_real = s.vis3_real.data();
        h.vis3_imag = s.vis3_imag.data();
        h.flag0 = s.flag0.data();
        h.flag3 = s.flag3.data();
        h.weight0 = s.weight0.data();
        h.weight3 = s.weight3.data();
        h.array_center_x = s.array_center_x;
        svdi_device_buffers dev{};
        if (svdi_preprocess_measurement_set(&h, &dev, 0) != 0) throw std::runtime_error(svdi_last_error());
        std::vector<float> dirty(image_size * image_size, 0.0f);
        const int st = svdi_fipipe_device(&dev, dirty.data(), image_size, cell_size);
        svdi_free_device_buffers(&dev);
        if (st != 0) throw std::runtime_error(std::string("FIpipeDevice failed: ") + svdi_last_error());
        svdi_io::write_fits_2d(output_name, dirty.data(), (long)image_size, (long)image_size,
                               svdi_io::wcs_cards_from_env((long)image_size, cell_size));
        const auto total_stop = std::chrono::high_resolution_clock::now();
        std::cerr << "Wrote image FITS: " << output_name << '\n';
        std::cout << "Total pipeline time: "
                  << std::chrono::duration<double>(total_stop - total_start).count() * 1000.0 << " ms" << std::endl;
        return 0;
    } catch (const std::exception& ex) {
        std::cerr << "Integrated SVD imager failed: " << ex.what() << '\n';
        return 1;
    }
}
