#include "bundle.h"

#include <cstring>
#include <fstream>
#include <map>
#include <stdexcept>

namespace svdi_io {

HostSnapshot read_bundle_snapshot(const std::string& path, size_t snapshot_index, size_t& total_snapshots) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open snapshot bundle: " + path);
    char magic[8];
    f.read(magic, 8);
    if (!f || std::memcmp(magic, "SVDIMS01", 8) != 0) throw std::runtime_error("not a snapshot bundle: " + path);
    uint64_t hdr[4];
    double ac[3];
    f.read(reinterpret_cast<char*>(hdr), sizeof(hdr));
    f.read(reinterpret_cast<char*>(ac), sizeof(ac));
    const size_t R = hdr[0], C = hdr[1], P = hdr[2];
    const bool has_w = hdr[3] != 0;
    if (!f || R == 0 || C == 0) throw std::runtime_error("empty snapshot bundle: " + path);
    if (P < 4) throw std::runtime_error("DATA has fewer than 4 polarisations in " + path);
    std::vector<double> time(R), uvw(R * 3), freq(C);
    f.read(reinterpret_cast<char*>(time.data()), R * 8);
    f.read(reinterpret_cast<char*>(uvw.data()), R * 24);
    f.read(reinterpret_cast<char*>(freq.data()), C * 8);
    if (!f) throw std::runtime_error("truncated snapshot bundle: " + path);
    std::map<double, std::vector<size_t>> groups;
    for (size_t r = 0; r < R; ++r) groups[time[r]].push_back(r);
    total_snapshots = groups.size();
    if (snapshot_index >= groups.size())
        throw std::runtime_error("Snapshot_Index is outside available TIME snapshots");
    auto it = groups.begin();
    std::advance(it, (long)snapshot_index);
    const std::vector<size_t>& rows = it->second;

    HostSnapshot s;
    s.index = snapshot_index;
    s.time = it->first;
    s.num_rows = rows.size();
    s.num_channels = C;
    s.num_samples = s.num_rows * C;
    s.array_center_x = (float)ac[0];
    for (size_t c = 0; c < C; ++c) s.frequencies_hz.push_back((float)freq[c]);
    s.uvw.resize(s.num_rows * 3);
    const size_t n = s.num_samples;
    s.vis0_real.resize(n); s.vis0_imag.resize(n); s.vis3_real.resize(n); s.vis3_imag.resize(n);
    s.flag0.resize(n); s.flag3.resize(n);
    s.weight0.assign(n, 1.0f); s.weight3.assign(n, 1.0f);
    const std::streamoff data_off = 8 + 32 + 24 + (std::streamoff)R * 8 + (std::streamoff)R * 24 + (std::streamoff)C * 8;
    const std::streamoff flag_off = data_off + (std::streamoff)(R * C * P * 8);
    const std::streamoff wt_off = flag_off + (std::streamoff)(R * C * P);
    std::vector<float> drow(C * P * 2), wrow(C * P);
    std::vector<uint8_t> frow(C * P);
    for (size_t lr = 0; lr < rows.size(); ++lr) {
        const size_t r = rows[lr];
        for (int a = 0; a < 3; ++a) s.uvw[lr * 3 + a] = (float)uvw[r * 3 + a];
        f.seekg(data_off + (std::streamoff)(r * C * P * 8));
        f.read(reinterpret_cast<char*>(drow.data()), (std::streamsize)(C * P * 8));
        f.seekg(flag_off + (std::streamoff)(r * C * P));
        f.read(reinterpret_cast<char*>(frow.data()), (std::streamsize)(C * P));
        if (has_w) {
            f.seekg(wt_off + (std::streamoff)(r * C * P * 4));
            f.read(reinterpret_cast<char*>(wrow.data()), (std::streamsize)(C * P * 4));
        }
        if (!f) throw std::runtime_error("truncated snapshot bundle: " + path);
        for (size_t c = 0; c < C; ++c) {
            const size_t k = lr + c * s.num_rows;  // channel-major (SVDIntegratedImager.cu:90-92)
            s.vis0_real[k] = drow[(c * P + 0) * 2 + 0];
            s.vis0_imag[k] = drow[(c * P + 0) * 2 + 1];
            s.vis3_real[k] = drow[(c * P + 3) * 2 + 0];
            s.vis3_imag[k] = drow[(c * P + 3) * 2 + 1];
            s.flag0[k] = frow[c * P + 0] ? 1 : 0;
            s.flag3[k] = frow[c * P + 3] ? 1 : 0;
            if (has_w) {
                s.weight0[k] = wrow[c * P + 0];
                s.weight3[k] = wrow[c * P + 3];
            }
        }
    }
    return s;
}
}  // namespace svdi_io
