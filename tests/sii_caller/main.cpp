// A main-path caller written against the reference's declarations (SVDIntegratedImager.cu:39-86),
// as its own `main` (:1773-1854) uses them: fill HostMeasurementSetData, preprocess, image, free.
// Linked against libsvdimager_b200.so by tests/test_sii_cpp.py.
//
//   sii_caller snapshot.bin image.bin
// snapshot.bin: uint64 num_rows, num_channels, image_size; float cell_size, array_center_x; then
// uvw, frequencies_hz, vis0_real, vis0_imag, vis3_real, vis3_imag (float), flag0, flag3 (uint8),
// weight0, weight3 (float). image.bin: image_size^2 floats.
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "svdimager_b200_sii.hpp"

template <typename T>
static void read_into(std::FILE* f, std::vector<T>& v, std::size_t n) {
    v.resize(n);
    if (std::fread(v.data(), sizeof(T), n, f) != n) throw std::runtime_error("short read");
}

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s snapshot.bin image.bin\n", argv[0]);
        return 2;
    }
    try {
        std::FILE* f = std::fopen(argv[1], "rb");
        if (!f) throw std::runtime_error("cannot open input");
        std::uint64_t hdr[3];
        float fc[2];
        if (std::fread(hdr, 8, 3, f) != 3 || std::fread(fc, 4, 2, f) != 2) throw std::runtime_error("short header");
        HostMeasurementSetData h;
        h.num_rows = hdr[0];
        h.num_channels = hdr[1];
        h.num_samples = h.num_rows * h.num_channels;
        h.array_center_x = fc[1];
        const std::size_t n = h.num_samples;
        read_into(f, h.uvw, 3 * h.num_rows);
        read_into(f, h.frequencies_hz, h.num_channels);
        read_into(f, h.vis0_real, n);
        read_into(f, h.vis0_imag, n);
        read_into(f, h.vis3_real, n);
        read_into(f, h.vis3_imag, n);
        read_into(f, h.flag0, n);
        read_into(f, h.flag3, n);
        read_into(f, h.weight0, n);
        read_into(f, h.weight3, n);
        std::fclose(f);
        const std::size_t N = hdr[2];
        std::vector<float> image(N * N, 0.0f);

        // buffers never filled by preprocess_measurement_set_gpu: the call must throw
        bool threw = false;
        try {
            DevicePreprocessBuffers empty;
            FIpipeDevice(empty, image.data(), N, fc[0]);
        } catch (const std::runtime_error&) {
            threw = true;
        }
        if (!threw) throw std::runtime_error("FIpipeDevice accepted unfilled buffers");

        DevicePreprocessBuffers buffers;
        preprocess_measurement_set_gpu(h, buffers);
        if (!buffers.d_bin || !buffers.d_vin || !buffers.d_vis_real || !buffers.d_vis_imag || buffers.num_samples != n)
            throw std::runtime_error("DevicePreprocessBuffers not filled");
        const int rc = FIpipeDevice(buffers, image.data(), N, fc[0]);
        free_device_preprocess_buffers(buffers);
        if (rc != 0) throw std::runtime_error("FIpipeDevice returned non-zero");
        if (buffers.d_bin || buffers.d_vin || buffers.d_vis_real || buffers.d_vis_imag || buffers.num_samples)
            throw std::runtime_error("free_device_preprocess_buffers left fields set");

        std::FILE* o = std::fopen(argv[2], "wb");
        if (!o || std::fwrite(image.data(), 4, image.size(), o) != image.size()) throw std::runtime_error("write failed");
        std::fclose(o);
        std::printf("sii_caller: ok\n");
        return 0;
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "sii_caller failed: %s\n", ex.what());
        return 1;
    }
}
