// Minimal FITS primary-image I/O, written from the FITS standard: 2880-byte blocks, 80-column
// header cards, big-endian data.
#include "fits.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <stdexcept>

namespace svdi_io {
namespace {
constexpr size_t kBlock = 2880;

std::string card(const std::string& key, const std::string& value) {
    std::string s = key;
    s.resize(8, ' ');
    s += "= ";
    std::string v = value;
    if (v.size() < 20) v = std::string(20 - v.size(), ' ') + v;
    s += v;
    s.resize(80, ' ');
    return s;
}

template <typename T>
T be(const unsigned char* p) {
    unsigned char b[sizeof(T)];
    for (size_t i = 0; i < sizeof(T); ++i) b[i] = p[sizeof(T) - 1 - i];
    T v;
    std::memcpy(&v, b, sizeof(T));
    return v;
}
}  // namespace

std::vector<float> read_fits_image(const std::string& path, long naxes[2]) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open FITS file: " + path);
    std::vector<unsigned char> raw((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    std::map<std::string, std::string> hdr;
    size_t pos = 0;
    bool end = false;
    while (!end) {
        if (pos + kBlock > raw.size()) throw std::runtime_error("truncated FITS header: " + path);
        for (size_t c = 0; c < kBlock; c += 80) {
            std::string line(reinterpret_cast<const char*>(&raw[pos + c]), 80);
            std::string key = line.substr(0, 8);
            key.erase(key.find_last_not_of(' ') + 1);
            if (key == "END") {
                end = true;
                break;
            }
            if (line.compare(8, 2, "= ") == 0) {
                std::string v = line.substr(10);
                const size_t slash = v.find('/');
                if (slash != std::string::npos && v.find('\'') == std::string::npos) v = v.substr(0, slash);
                v.erase(0, v.find_first_not_of(' '));
                v.erase(v.find_last_not_of(' ') + 1);
                hdr[key] = v;
            }
        }
        pos += kBlock;
    }
    auto geti = [&](const std::string& k) -> long {
        auto it = hdr.find(k);
        if (it == hdr.end()) throw std::runtime_error("FITS keyword missing: " + k);
        return std::stol(it->second);
    };
    auto getd = [&](const std::string& k, double d) -> double {
        auto it = hdr.find(k);
        return it == hdr.end() ? d : std::stod(it->second);
    };
    const long naxis = geti("NAXIS");
    if (naxis == 1) {
        naxes[0] = geti("NAXIS1");
        naxes[1] = 1;
    } else if (naxis == 2) {
        naxes[0] = geti("NAXIS1");
        naxes[1] = geti("NAXIS2");
    } else {
        throw std::runtime_error("unsupported NAXIS in " + path);
    }
    const long bitpix = geti("BITPIX");
    const double bscale = getd("BSCALE", 1.0), bzero = getd("BZERO", 0.0);
    const size_t n = (size_t)naxes[0] * (size_t)naxes[1];
    const size_t bytes = (size_t)std::labs(bitpix) / 8;
    if (pos + n * bytes > raw.size()) throw std::runtime_error("truncated FITS data: " + path);
    std::vector<float> out(n);
    const unsigned char* p = &raw[pos];
    for (size_t i = 0; i < n; ++i, p += bytes) {
        double v;
        switch (bitpix) {
            case 8: v = *p; break;
            case 16: v = be<int16_t>(p); break;
            case 32: v = be<int32_t>(p); break;
            case 64: v = (double)be<int64_t>(p); break;
            case -32: v = be<float>(p); break;
            case -64: v = be<double>(p); break;
            default: throw std::runtime_error("unsupported BITPIX in " + path);
        }
        out[i] = (float)(v * bscale + bzero);
    }
    return out;
}

std::string num_card(const std::string& key, double v) {
    char buf[32];
    std::snprintf(buf, sizeof(buf), "%.15E", v);
    return card(key, buf);
}

std::string str_card(const std::string& key, const std::string& v) {
    std::string q = "'" + v;
    if (q.size() < 9) q.resize(9, ' ');
    q += "'";
    std::string s = key;
    s.resize(8, ' ');
    s += "= " + q;
    s.resize(80, ' ');
    return s;
}

std::vector<std::string> sin_wcs_cards(long image_size, double cell_rad, double ra_deg, double dec_deg) {
    const double cell_deg = cell_rad * 180.0 / 3.14159265358979323846;
    const double crpix = (double)(image_size / 2) + 1.0;  // FITS pixels count from 1
    return {str_card("CTYPE1", "RA---SIN"), num_card("CRVAL1", ra_deg), num_card("CRPIX1", crpix),
            num_card("CDELT1", -cell_deg),   str_card("CUNIT1", "deg"),
            str_card("CTYPE2", "DEC--SIN"), num_card("CRVAL2", dec_deg), num_card("CRPIX2", crpix),
            num_card("CDELT2", cell_deg),    str_card("CUNIT2", "deg"),
            str_card("RADESYS", "ICRS"),     num_card("EQUINOX", 2000.0), str_card("BUNIT", "JY/BEAM")};
}

std::vector<std::string> wcs_cards_from_env(long image_size, double cell_rad) {
    const char* env = std::getenv("SVDI_FITS_WCS");
    if (!env || !*env) return {};
    double ra = 0.0, dec = 0.0;
    char tail = 0;
    if (std::sscanf(env, "%lf,%lf%c", &ra, &dec, &tail) != 2 || !(dec >= -90.0 && dec <= 90.0))
        throw std::runtime_error("SVDI_FITS_WCS must be \"ra_deg,dec_deg\"");
    return sin_wcs_cards(image_size, cell_rad, ra, dec);
}

void write_fits_2d(const std::string& path, const float* values, long axis0, long axis1,
                   const std::vector<std::string>& extra_cards) {
    std::string h = card("SIMPLE", "T") + card("BITPIX", "-32") + card("NAXIS", "2") +
                    card("NAXIS1", std::to_string(axis0)) + card("NAXIS2", std::to_string(axis1));
    for (const auto& c : extra_cards) {
        std::string cc = c;
        cc.resize(80, ' ');
        h += cc;
    }
    std::string endc = "END";
    endc.resize(80, ' ');
    h += endc;
    h.resize((h.size() + kBlock - 1) / kBlock * kBlock, ' ');
    const size_t n = (size_t)axis0 * (size_t)axis1;
    std::vector<unsigned char> body((n * 4 + kBlock - 1) / kBlock * kBlock, 0);
    for (size_t i = 0; i < n; ++i) {
        unsigned char b[4];
        std::memcpy(b, &values[i], 4);
        body[i * 4 + 0] = b[3];
        body[i * 4 + 1] = b[2];
        body[i * 4 + 2] = b[1];
        body[i * 4 + 3] = b[0];
    }
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) throw std::runtime_error("Failed to create FITS file: " + path);
    f.write(h.data(), (std::streamsize)h.size());
    f.write(reinterpret_cast<const char*>(body.data()), (std::streamsize)body.size());
    if (!f) throw std::runtime_error("Failed to write FITS image: " + path);
}
}  // namespace svdi_io
