// C++ main-path entry points with the reference's types and linkage (include/svdimager_b200_sii.hpp),
// over the C ABI. Replaces preprocess_measurement_set_gpu (SVDIntegratedImager.cu:635-853),
// FIpipeDevice (:1498-1761) and free_device_preprocess_buffers (:855-865) for callers compiled
// against the reference's declarations (:39-86).
#include "svdimager_b200_sii.hpp"

#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

#include "svdimager_b200.h"

namespace {

// The C descriptor (FP64 rotation, engine) of every live DevicePreprocessBuffers, by d_vis_real.
std::mutex g_mu;
std::map<const float*, svdi_device_buffers> g_live;

[[noreturn]] void fail(const char* what) {
    throw std::runtime_error(std::string(what) + ": " + svdi_last_error());
}

void check_size(std::size_t got, std::size_t want, const char* name) {
    if (got != want)
        throw std::runtime_error(std::string("HostMeasurementSetData.") + name + " has " + std::to_string(got) +
                                 " elements, expected " + std::to_string(want));
}

}  // namespace

void preprocess_measurement_set_gpu(const HostMeasurementSetData& h, DevicePreprocessBuffers& out) {
    if (h.num_samples == 0) throw std::runtime_error("No visibility samples available for preprocessing.");
    if (h.num_rows * h.num_channels != h.num_samples)
        throw std::runtime_error("num_samples must equal num_rows * num_channels");
    check_size(h.uvw.size(), 3 * h.num_rows, "uvw");
    check_size(h.frequencies_hz.size(), h.num_channels, "frequencies_hz");
    check_size(h.vis0_real.size(), h.num_samples, "vis0_real");
    check_size(h.vis0_imag.size(), h.num_samples, "vis0_imag");
    check_size(h.vis3_real.size(), h.num_samples, "vis3_real");
    check_size(h.vis3_imag.size(), h.num_samples, "vis3_imag");
    check_size(h.flag0.size(), h.num_samples, "flag0");
    check_size(h.flag3.size(), h.num_samples, "flag3");
    check_size(h.weight0.size(), h.num_samples, "weight0");
    check_size(h.weight3.size(), h.num_samples, "weight3");
    svdi_host_ms c{};
    c.num_rows = h.num_rows;
    c.num_channels = h.num_channels;
    c.num_samples = h.num_samples;
    c.uvw = h.uvw.data();
    c.frequencies_hz = h.frequencies_hz.data();
    c.vis0_real = h.vis0_real.data();
    c.vis0_imag = h.vis0_imag.data();
    c.vis3_real = h.vis3_real.data();
    c.vis3_imag = h.vis3_imag.data();
    c.flag0 = h.flag0.data();
    c.flag3 = h.flag3.data();
    c.weight0 = h.weight0.data();
    c.weight3 = h.weight3.data();
    c.array_center_x = h.array_center_x;
    svdi_device_buffers d{};
    // the reference fills d_bin, so this does too (want_bin = 1)
    if (svdi_preprocess_measurement_set(&c, &d, 1) != SVDI_OK) fail("preprocess_measurement_set_gpu");
    out.d_bin = d.d_bin;
    out.d_vin = d.d_vin;
    out.d_vis_real = d.d_vis_real;
    out.d_vis_imag = d.d_vis_imag;
    out.num_samples = d.num_samples;
    std::lock_guard<std::mutex> lk(g_mu);
    g_live[d.d_vis_real] = d;
}

int FIpipeDevice(const DevicePreprocessBuffers& b, float* dirty_image, std::size_t image_size, float cell_size) {
    svdi_device_buffers d{};
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_live.find(b.d_vis_real);
        if (it == g_live.end() || it->second.num_samples != b.num_samples)
            throw std::runtime_error("FIpipeDevice: buffers were not filled by preprocess_measurement_set_gpu");
        d = it->second;
    }
    if (image_size == 0) throw std::runtime_error("Image_Size must be greater than zero");
    if (!(cell_size > 0.0f)) throw std::runtime_error("Cell_Size must be greater than zero");
    if (svdi_fipipe_device(&d, dirty_image, image_size, cell_size) != SVDI_OK) fail("FIpipeDevice");
    return 0;
}

void free_device_preprocess_buffers(DevicePreprocessBuffers& b) {
    svdi_device_buffers d{};
    bool found = false;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_live.find(b.d_vis_real);
        if (it != g_live.end()) {
            d = it->second;
            g_live.erase(it);
            found = true;
        }
    }
    if (found) svdi_free_device_buffers(&d);
    b.d_bin = nullptr;
    b.d_vin = nullptr;
    b.d_vis_real = nullptr;
    b.d_vis_imag = nullptr;
    b.num_samples = 0;
}
