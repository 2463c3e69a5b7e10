// Snapshot bundle reader (stand-in for the casacore Measurement Set reader of
// SVDIntegratedImager.cu:180-378). Layout documented in svdimager_b200/bundle.py.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace svdi_io {
struct HostSnapshot {  // HostMeasurementSetData (SVDIntegratedImager.cu:39-54)
    size_t num_rows = 0, num_channels = 0, num_samples = 0;
    std::vector<float> uvw, frequencies_hz, vis0_real, vis0_imag, vis3_real, vis3_imag, weight0, weight3;
    std::vector<uint8_t> flag0, flag3;
    float array_center_x = 0.0f;
    double time = 0.0;
    size_t index = 0;
};
// Groups rows by TIME in ascending order (std::map, SVDIntegratedImager.cu:333-355) and reads the
// snapshot_index-th group. total_snapshots receives the number of groups. Throws on error.
HostSnapshot read_bundle_snapshot(const std::string& path, size_t snapshot_index, size_t& total_snapshots);
}
