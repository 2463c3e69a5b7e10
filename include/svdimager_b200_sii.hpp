// svdimager_b200 — C++ main-path entry points with the reference's own types and linkage.
//
// A caller written against SVDIntegratedImager.cu (its `main`, or any code that includes the same
// declarations) links against libsvdimager_b200.so unchanged: the types below are layout- and
// name-identical to SVDIntegratedImager.cu:39-69 and the functions have the C++ linkage and
// signatures of SVDIntegratedImager.cu:76-86 (mangled names included). They wrap the C ABI of
// svdimager_b200.h: svdi_preprocess_measurement_set, svdi_fipipe_device, svdi_free_device_buffers.
//
// Behaviour kept from the reference:
//   - errors throw std::runtime_error (SVDIntegratedImager.cu:384-407); FIpipeDevice returns 0;
//   - DevicePreprocessBuffers holds device arrays the library allocated: d_bin [num_samples][3]
//     float rotated baselines in wavelengths, d_vin [9] float row-major basis, d_vis_real /
//     d_vis_imag [num_samples] collapsed visibilities; free_device_preprocess_buffers releases them
//     and zeroes the fields;
//   - slab + bucket-K Chebyshev semantics and the simplified SIN reprojection of the main path.
// Added: the FP64 rotation the B200 path images from (separable r = s[chan] q[row]) lives beside
// the four reference arrays, keyed by d_vis_real; a DevicePreprocessBuffers not filled by
// preprocess_measurement_set_gpu makes FIpipeDevice throw instead of reading stray memory.
#ifndef SVDIMAGER_B200_SII_HPP
#define SVDIMAGER_B200_SII_HPP

#include <cstddef>
#include <cstdint>
#include <vector>

// SVDIntegratedImager.cu:39-54
struct HostMeasurementSetData {
    std::size_t num_rows = 0;
    std::size_t num_channels = 0;
    std::size_t num_samples = 0;
    std::vector<float> uvw;
    std::vector<float> frequencies_hz;
    std::vector<float> vis0_real;
    std::vector<float> vis0_imag;
    std::vector<float> vis3_real;
    std::vector<float> vis3_imag;
    std::vector<std::uint8_t> flag0;
    std::vector<std::uint8_t> flag3;
    std::vector<float> weight0;
    std::vector<float> weight3;
    float array_center_x = 0.0f;
};

// SVDIntegratedImager.cu:63-69
struct DevicePreprocessBuffers {
    float* d_bin = nullptr;
    float* d_vin = nullptr;
    float* d_vis_real = nullptr;
    float* d_vis_imag = nullptr;
    std::size_t num_samples = 0;
};

// SVDIntegratedImager.cu:76-79 (defined there at :635-853)
void preprocess_measurement_set_gpu(const HostMeasurementSetData& host_data,
                                    DevicePreprocessBuffers& device_buffers);

// SVDIntegratedImager.cu:80 (defined there at :855-865)
void free_device_preprocess_buffers(DevicePreprocessBuffers& device_buffers);

// SVDIntegratedImager.cu:81-86 (defined there at :1498-1761). dirty_image is a HOST array of
// image_size * image_size floats.
int FIpipeDevice(const DevicePreprocessBuffers& preprocess_buffers, float* dirty_image,
                 std::size_t image_size, float cell_size);

#endif  // SVDIMAGER_B200_SII_HPP
